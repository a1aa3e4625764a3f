// cryo_physics.cu -- neighbour passes of the rate evaluation
// (Solver::evaluate_rates, sph_solver.cu:449-480).  One thread per particle
// over the cell-sorted arrays; every neighbour loop visits the reference's
// 27-cell order (for_each_neighbor in cryo_common.cuh).
#include "cryo_kernels.cuh"

// exact (default) or fast: see CRYO_FIELD_KERNELS in cryo_kernels.cuh
#ifndef CRYO_FIELD_NS
#define CRYO_FIELD_NS exact
#endif

namespace cryo {
namespace CRYO_FIELD_NS {

#define PARTICLE_LOOP(i, n) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// compute_density_summation (SPH_kernels.cu:6-34); with fuse_eos the
// equation of state (navier_stokes.cu:5-14) is applied in the same pass.
__global__ void __launch_bounds__(kBlock) k_density(Params P, View V, int fuse_eos) {
  // with lists: the walls' constants from the wall list, then the fluid
  // particles from the fluid list (a warp runs one kind of work)
  if (P.use_lists) {
    const Range wr = wall_range(P, V);
    PARTICLE_LOOP(t, wr.count) {
      const int i = particle_at(wr, t);
      reinterpret_cast<float*>(V.mrps + i)[3] = 1.0f / P.vol0;
      V.rmin[i] = P.support;
    }
  }
  const Range fr = fluid_range(P, V);
  PARTICLE_LOOP(t, fr.count) {
    const int i = particle_at(fr, t);
    const float4 xpi = V.xp[i];
    const int ph = ph_of(xpi);
    float* mr = reinterpret_cast<float*>(V.mrps + i);
    if (!is_fluid(ph)) {
      mr[3] = 1.0f / P.vol0;
      V.rmin[i] = P.support;
      continue;
    }
    const V3 xi = xyz(xpi);
    float sum = 0.0f, r2min = P.support2;
    for_each_nbr_quads(P, V, i, xi, [&](int j, float4, V3, float r2) {
      sum += kernel_W(P, sqrtf(r2));
      if (j != i && r2 < r2min) r2min = r2;
    });
    mr[3] = sum;
    V.rmin[i] = sqrtf(r2min);
    float rho = mr[1];
    if (P.density_mode == CRYO_DENSITY_SUMMATION) {
      rho = (ph == kLiquid ? V.vt[i].w : mr[0]) * sum;
      mr[1] = rho;
    }
    const float Ti = V.vT[i].w;
    if (fuse_eos) mr[2] = eos_pressure(P, ph, rho, Ti);
    V.aux[i] = make_float4(mr[0] / rho, 1.0f / sum, sound_speed(P, ph, Ti), 0.0f);
  }
}

// The per-particle factors of View::aux from the current fields (for
// operator-level passes run on fields set from outside).
__global__ void __launch_bounds__(kBlock) k_aux(Params P, View V) {
  const int n = V.dyn->n;
  PARTICLE_LOOP(i, n) {
    const int ph = ph_of(V.xp[i]);
    if (!is_fluid(ph)) continue;
    const float4 mr = V.mrps[i];
    V.aux[i] = make_float4(mr.x / mr.y, 1.0f / mr.w, sound_speed(P, ph, V.vT[i].w), 0.0f);
  }
}

// normalize_initial_masses (SPH_kernels.cu:36-54)
__global__ void __launch_bounds__(kBlock) k_normalize_masses(Params P, View V) {
  const int n = V.dyn->n;
  PARTICLE_LOOP(i, n) {
    const float4 xpi = V.xp[i];
    if (!is_fluid(ph_of(xpi))) continue;
    float sum = 0.0f;
    for_each_nbr(P, V, i, xyz(xpi), [&](int, float4, V3, float r2) {
      sum += kernel_W(P, sqrtf(r2));
    });
    if (sum > 0.0f) {
      float* mr = reinterpret_cast<float*>(V.mrps + i);
      const float m = mr[1] / sum;
      mr[0] = m;
      V.vt[i].w = m;
    }
  }
}

// compute_equation_of_state (navier_stokes.cu:5-14)
__global__ void __launch_bounds__(kBlock) k_eos(Params P, View V) {
  const int n = V.dyn->n;
  PARTICLE_LOOP(i, n) {
    const int ph = ph_of(V.xp[i]);
    if (is_fluid(ph)) {
      float* mr = reinterpret_cast<float*>(V.mrps + i);
      mr[2] = eos_pressure(P, ph, mr[1], V.vT[i].w);
    }
  }
}

// compute_wall_boundary (navier_stokes.cu:16-69)
__global__ void __launch_bounds__(kBlock) k_wall(Params P, View V) {
  const DynState* dyn = V.dyn;
  const Range rg = wall_range(P, V);
  const V3 g = v3(dyn->fr.gravity[0], dyn->fr.gravity[1], dyn->fr.gravity[2]);
  PARTICLE_LOOP(t, rg.count) {
    const int i = particle_at(rg, t);
    const float4 xpi = V.xp[i];
    if (ph_of(xpi) != kWall) continue;
    const V3 xi = xyz(xpi);
    float sw[2] = {0, 0}, sp[2] = {0, 0}, sgr[2] = {0, 0};
    float srho = 0.0f;
    V3 sv{0, 0, 0};
    for_each_nbr(P, V, i, xi, [&](int j, float4 xj, V3 rwf, float r2) {
      const int phj = ph_of(xj);
      if (!is_fluid(phj)) return;
      const float w = kernel_W(P, sqrtf(r2));
      const float4 mr = __ldg(V.mrps + j);
      const float rhoj = mr.y;
      const int k = phase_index(phj);
      sw[k] += w;
      sp[k] += mr.z * w;
      sgr[k] += dot(g, rwf) * rhoj * w;
      srho += rhoj * w;
      sv += xyz(__ldg(V.vT + j)) * w;
    });
    float pw[2];
    for (int k = 0; k < 2; ++k) {
      pw[k] = sw[k] > 0.0f ? (sp[k] + sgr[k]) / sw[k] : P.p_bg;
      if (P.clamp_neg && pw[k] < 0.0f) pw[k] = 0.0f;
    }
    if (!(sw[0] > 0.0f) && sw[1] > 0.0f) pw[0] = pw[1];
    if (!(sw[1] > 0.0f) && sw[0] > 0.0f) pw[1] = pw[0];
    float* mr = reinterpret_cast<float*>(V.mrps + i);
    mr[2] = pw[0];
    V.nrm[i].w = (sw[0] + sw[1]) > 0.0f ? sw[0] / (sw[0] + sw[1]) : 0.0f;
    const float swt = sw[0] + sw[1];
    V3 vw;
    if (swt > 0.0f) {
      mr[1] = srho / swt;
      vw = sv * (-1.0f / swt);
    } else {
      mr[1] = P.rho0[0];
      vw = V3{0, 0, 0};
    }
    V.vwp[i] = f4(vw, pw[1]);
    V.a4[i] = make_float4(0.0f, 0.0f, 0.0f, V.a4[i].w);
  }
}

// compute_interface_fields (surface_tension.cu:5-85).  With heat_sum the FP64
// sum of heat_w over fluid particles (sph_solver.cu:101-104) is reduced in the
// same pass and heat_inv_norm is set (sph_solver.cu:466-472); the CSF unit
// normal (smooth_interface_normals without smoothing, surface_tension.cu:91-101)
// is written when the CSF model is active.
template <int TAPE>
__global__ void __launch_bounds__(kBlock) k_interface(Params P, View V, Reduce R, int heat_sum) {
  __shared__ double sh[kBlock / 32];
  const Range rg = fluid_range(P, V);
  const int nch = num_chunks(rg.count);
  const bool write_ns = P.csf_active && !P.csf_smooth;
  const int own_lo = V.dyn->own_lo, own_hi = V.dyn->own_hi, n_sorted = V.dyn->n_sorted;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int t = c * kChunk + threadIdx.x;
    double hsum[1] = {0.0};
    if (t < rg.count) {
      const int i = particle_at(rg, t);
      const float4 xpi = V.xp[i];
      const int ph = ph_of(xpi);
      if (is_fluid(ph)) {
        const V3 xi = xyz(xpi);
        const float ci = ph == kLiquid ? 1.0f : 0.0f;
        V3 gradc{0, 0, 0}, wall_n{0, 0, 0}, akn{0, 0, 0}, gradphi{0, 0, 0};
        float s_all = 0, s_other = 0, ww = 0, hw = 0;
        auto wall_term = [&](int j, float4 xj, V3 rij, float r) {
          const float vw = P.vol0 * kernel_W(P, r);
          ww += vw;
          if (fl_of(xj) & kHeated) hw += vw;
          const float4 nj = __ldg(V.nrm + j);
          wall_n += xyz(nj) * vw;
          gradphi += kernel_gradW(P, rij, r) * P.vol0;
          if (P.wall_colour) gradc += kernel_gradW(P, rij, r) * (P.vol0 * (nj.w - ci));
        };
        if (!TAPE && !P.has_vapor && P.st_model != CRYO_ST_AKINCI) {
          // A tank without vapour: every fluid neighbour is liquid, so its
          // colour term is gw * (V_j * 0) (a zero, which leaves the sum as
          // it is) and s_other stays 0, making alpha 0 whatever s_all is;
          // only the wall neighbours change the outputs.
          for_each_nbr(P, V, i, xi, [&](int j, float4 xj, V3 rij, float r2) {
            if (ph_of(xj) == kWall) wall_term(j, xj, rij, sqrtf(r2));
          });
        } else {
          for_each_nbr_pf(P, V, i, xi, V.aux, [&](int j, float4 xj, V3 rij, float r2, const float4& auxj) {
            const float r = sqrtf(r2);
            const int phj = ph_of(xj);
            if (phj == kWall) {
              wall_term(j, xj, rij, r);
              return;
            }
            const float w = kernel_W(P, r);
            const float Vj = auxj.x;  // m_j / rho_j
            s_all += Vj * w;
            if (phj != ph) s_other += Vj * w;
            if (j == i) return;
            // a neighbour of the same phase adds gw * (V_j * 0) to the colour
            // gradient, a zero that leaves the sum as it is; only Akinci's
            // normal needs its gradient
            if (phj == ph && P.st_model != CRYO_ST_AKINCI) return;
            const V3 gw = kernel_gradW(P, rij, r);
            const float cj = phj == kLiquid ? 1.0f : 0.0f;
            gradc += gw * (Vj * (cj - ci));
            if (phj == kLiquid) akn += gw * Vj;
          });
        }
        if (TAPE) {
          const int tn = V.tape_n;
          V.tape[3 * tn + i] = f4(gradc, s_all);
          V.tape[4 * tn + i] = f4(wall_n, s_other);
          V.tape[5 * tn + i] = make_float4(ww, 0.0f, 0.0f, 0.0f);
        }
        const float alpha = s_all > 0.0f ? s_other / s_all : 0.0f;
        V.wall_w[i] = ww;
        V.heat_w[i] = hw;
        if (owned(own_lo, own_hi, n_sorted, i)) hsum[0] = (double)hw;
        if (P.st_model == CRYO_ST_AKINCI) {
          V.nrm[i] = f4(ph == kLiquid ? akn * (-P.h) : V3{0, 0, 0}, alpha);
        } else {
          const float gmag = norm(gradc);
          V3 vwi{0, 0, 0};
          if (P.wetting_model != 0 && ww > 0.0f && gmag > P.normal_eps && norm2(wall_n) > 0.0f) {
            const V3 nw = normalized(wall_n);
            const V3 nh = gradc / gmag;
            const V3 tan_in = nh - nw * dot(nh, nw);
            const float tm = norm(tan_in);
            if (tm > 1e-6f) {
              const float cos_d = -dot(nh, nw);
              const float delta_w = 2.0f * norm(gradphi);
              const float coeff = 2.0f * P.sigma / (P.rho0[0] + P.rho0[1]);
              vwi = tan_in * (-(P.cos_theta - cos_d) * coeff * gmag * delta_w / tm);
            }
          }
          V.vwp[i] = f4(vwi, V.vwp[i].w);
          if (P.wetting_model != 1 && ww > 0.0f && gmag > P.normal_eps) {
            const V3 nw = normalized(wall_n);
            const V3 nh = gradc / gmag;
            V3 t = nh - nw * dot(nh, nw);
            const float tmag = norm(t);
            if (norm2(nw) > 0.0f && tmag > 1e-6f) {
              t = t / tmag;
              const V3 target = nw * (-P.cos_theta) + t * P.sin_theta;
              const float beta = clampf(ww / P.wall_adhesion_weight, 0.0f, 1.0f);
              const V3 blended = normalized(nh * (1.0f - beta) + target * beta);
              gradc = blended * gmag;
            }
          }
          V.nrm[i] = f4(gradc, alpha);
          if (write_ns) {
            const float gm = norm(gradc);
            const V3 ns = gm > P.normal_eps ? gradc / gm : V3{0, 0, 0};
            V.ns4[i] = f4(ns, V.ns4[i].w);
          }
        }
      }
    }
    if (heat_sum) publish_chunk<1>(R, c, hsum, sh);
  }
  if (heat_sum && last_block(R.ticket)) {
    DynState* dyn = V.dyn;
    const double S = block_sum_partials(R, 0, nch);
    if (threadIdx.x != 0) return;
    dyn->heat_sum = S;
    if (P.slab) return;  // the slabs set heat_inv_norm from their combined sums
    if (heat_sum == 2 || dyn->thermal_on) {
      if (P.heat_power != 0.0f) {
        dyn->heat_inv_norm = S > 0 ? (float)(1.0 / S) : 0.0f;
      } else {
        dyn->heat_inv_norm = 0.0f;
      }
    }
  }
}

template __global__ void k_interface<0>(Params, View, Reduce, int);
template __global__ void k_interface<1>(Params, View, Reduce, int);

// compute_sps_viscosity (navier_stokes.cu:71-119)
__global__ void __launch_bounds__(kBlock) k_sps(Params P, View V) {
  const int n = V.dyn->n;
  const int own_lo = V.dyn->own_lo, own_hi = V.dyn->own_hi, n_sorted = V.dyn->n_sorted;  // a slab skips its ghosts
  PARTICLE_LOOP(i, n) {
    if (!owned(own_lo, own_hi, n_sorted, i)) continue;
    const float4 xpi = V.xp[i];
    if (!is_fluid(ph_of(xpi))) {
      V.nu_t[i] = 0.0f;
      continue;
    }
    const V3 vi = xyz(V.vT[i]);
    float L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for_each_nbr(P, V, i, xyz(xpi), [&](int j, float4 xj, V3 rij, float r2) {
      if (j == i) return;
      const V3 gw = kernel_gradW(P, rij, sqrtf(r2));
      V3 vj;
      float Vj;
      if (ph_of(xj) == kWall) {
        if (!P.no_slip) return;
        vj = xyz(__ldg(V.vwp + j));
        Vj = P.vol0;
      } else {
        vj = xyz(__ldg(V.vT + j));
        Vj = __ldg(V.aux + j).x;  // m_j / rho_j
      }
      const V3 dv = (vj - vi) * Vj;
      const float dvc[3] = {dv.x, dv.y, dv.z};
      const float gwc[3] = {gw.x, gw.y, gw.z};
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) L[a][b] += dvc[a] * gwc[b];
    });
    float ss = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const float sab = 0.5f * (L[a][b] + L[b][a]);
        ss += sab * sab;
      }
    const float smag = sqrtf(2.0f * ss);
    const float l = P.smagorinsky_cs * P.dx;
    V.nu_t[i] = l * l * smag;
  }
}

// smooth_interface_normals (surface_tension.cu:87-118)
__global__ void __launch_bounds__(kBlock) k_smooth_normals(Params P, View V) {
  const int n = V.dyn->n;
  const int own_lo = V.dyn->own_lo, own_hi = V.dyn->own_hi, n_sorted = V.dyn->n_sorted;  // a slab skips its ghosts
  PARTICLE_LOOP(i, n) {
    if (!owned(own_lo, own_hi, n_sorted, i)) continue;
    const float4 xpi = V.xp[i];
    if (!is_fluid(ph_of(xpi))) continue;
    const V3 gi = xyz(V.nrm[i]);
    const float gmag = norm(gi);
    const float kap = V.ns4[i].w;
    if (!(gmag > P.normal_eps)) {
      V.ns4[i] = make_float4(0.0f, 0.0f, 0.0f, kap);
      continue;
    }
    if (!P.csf_smooth) {
      V.ns4[i] = f4(gi / gmag, kap);
      continue;
    }
    V3 acc{0, 0, 0};
    for_each_nbr(P, V, i, xyz(xpi), [&](int j, float4 xj, V3, float r2) {
      if (!is_fluid(ph_of(xj))) return;
      const V3 gj = xyz(__ldg(V.nrm + j));
      const float gjm = norm(gj);
      if (!(gjm > P.normal_eps)) return;
      const float4 mr = __ldg(V.mrps + j);
      acc += gj * ((mr.x / mr.y) * kernel_W(P, sqrtf(r2)) / gjm);
    });
    V.ns4[i] = f4(normalized(acc), kap);
  }
}

// Fused force pass: compute_transport_acceleration (SPH_kernels.cu:56-104),
// compute_momentum (navier_stokes.cu:121-245), apply_csf_surface_tension
// (surface_tension.cu:120-177) or apply_akinci_surface_tension (:179-213),
// compute_density_rate (SPH_kernels.cu:162-203), compute_thermal_rates
// (phase_change.cu:31-75) and the dt maxima (sph_solver.cu:59-99, 475-479),
// in one neighbour loop.  Each sub-pass reads only what the previous passes
// wrote, never what this pass writes, so fusing keeps the reference's values.
template <int WHAT>
__global__ void __launch_bounds__(FORCES_BLOCK, forces_min_blocks(WHAT)) k_forces_t(Params P, View V, int what_rt) {
  // WHAT >= 0: the sub-pass set is a compile-time constant (the step path);
  // -1: read at run time (operator-level calls)
  const int what = WHAT >= 0 ? WHAT : what_rt;
  DynState* dyn = V.dyn;
  const int n = dyn->n;
  const bool thermal = ((what & FORCE_THERMAL) && dyn->thermal_on) || (what & FORCE_THERMAL_ALWAYS);
  const float dt = dyn->dt;
  const V3 origin = v3(dyn->fr.frame_origin[0], dyn->fr.frame_origin[1], dyn->fr.frame_origin[2]);
  const float h = P.h;
  const float eta2 = 0.01f * h * h;
  const float r_guard = 0.6f * P.dx;
  const bool tvf_stress = P.tvf && P.tvf_stress;
  const float inv_gamma = 1.0f / P.tait_gamma;
  const float csf_coeff = 2.0f * P.sigma / (P.rho0[0] + P.rho0[1]);
  const bool iso_walls = P.wall_bc == CRYO_WALL_ISOTHERMAL;
  const int own_lo = dyn->own_lo, own_hi = dyn->own_hi, n_sorted = dyn->n_sorted;
  float vmax_l = 0.0f, amax_l = 0.0f, tv_l = 0.0f, sr_l = 0.0f, nut_l = 0.0f;

  // walls (and, without lists, every particle that is not fluid): zero outputs
  {
    const Range wr = P.use_lists ? wall_range(P, V) : Range{nullptr, n};
    PARTICLE_LOOP(t, wr.count) {
      const int i = particle_at(wr, t);
      if (is_fluid(ph_of(V.xp[i]))) continue;
      if (what & FORCE_TRANSPORT) V.ab4[i] = make_float4(0.0f, 0.0f, 0.0f, V.ab4[i].w);
      if (what & FORCE_MOMENTUM) {
        V.a4[i] = make_float4(0.0f, 0.0f, 0.0f, V.a4[i].w);
        V.fw[i] = make_float4(0, 0, 0, 0);
        V.mw[i] = make_float4(0, 0, 0, 0);
      }
      if (what & FORCE_DRHO) reinterpret_cast<float*>(V.ab4 + i)[3] = 0.0f;
      if (thermal) reinterpret_cast<float*>(V.a4 + i)[3] = 0.0f;
    }
  }
  const Range fr = fluid_range(P, V);
  PARTICLE_LOOP(t, fr.count) {
    const int i = particle_at(fr, t);
    const float4 xpi = V.xp[i];
    const int ph = ph_of(xpi);
    if (!is_fluid(ph)) continue;
    const int pi_idx = phase_index(ph);
    const V3 xi = xyz(xpi);
    const float4 vTi = V.vT[i];
    const V3 vi = xyz(vTi);
    const float Ti = vTi.w;
    const float4 mri = V.mrps[i];
    const float mi = mri.x, rhoi = mri.y, pi = mri.z, sigmai = mri.w;
    const float4 nrmi = V.nrm[i];
    const float alpha_i_pc = nrmi.w;
    const float4 vti4 = V.vt[i];
    const float Vi = mi / rhoi;
    const float Vi2 = Vi * Vi;
    const float ci = sound_speed(P, ph, Ti);
    const float etai = P.mu[pi_idx] + (P.sps ? rhoi * V.nu_t[i] : 0.0f);
    const float alpha_i = ph == kVapor ? P.alpha_av_vap : P.alpha_av;
    // harmonic viscosity per neighbour phase (navier_stokes.cu:190-196),
    // evaluated once per particle when it does not vary per neighbour
    // (0 where eta_i + eta_j = 0: that term is skipped, and a zero term
    // added to a sum leaves it unchanged)
    // (two scalars picked by a select per pair: a small array indexed by the
    // neighbour's phase would live in local memory, a load on every pair's
    // dependent chain)
    float eta_pair0 = 0.0f, eta_pair1 = 0.0f;
    if (!P.sps) {
      auto harmonic = [&](float etaj) {
        const float eta_sum = etai + etaj;
        return eta_sum > 0.0f ? 2.0f * etai * etaj / eta_sum : 0.0f;
      };
      eta_pair0 = harmonic(P.mu[0] + 0.0f);
      eta_pair1 = harmonic(P.mu[1] + 0.0f);
    }

    // transport (SPH_kernels.cu:61-74)
    const bool do_T = (what & FORCE_TRANSPORT) && P.tvf && !(sigmai < P.tvf_sigma_min) &&
                      !(P.tvf_interface_only && !(alpha_i_pc > 0.0f));
    const float VT_i = 1.0f / sigmai;
    const float VT_i2 = VT_i * VT_i;
    const float mT_i = rhoi * VT_i;
    const float pb = P.tvf_factor * P.rho0[pi_idx] * ci * ci;
    V3 sumT{0, 0, 0};
    // momentum
    V3 force{0, 0, 0}, acc_av{0, 0, 0}, fwall{0, 0, 0}, mwall{0, 0, 0};
    const V3 dvi = xyz(vti4) - vi;
    // CSF (surface_tension.cu:131-136)
    V3 ni{0, 0, 0};
    bool do_C = false;
    if (what & FORCE_CSF) {
      ni = xyz(V.ns4[i]);
      do_C = norm2(ni) > 0.25f;
    }
    const float ciC = ph == kLiquid ? 1.0f : 0.0f;
    float num = 0.0f, den = 0.0f;
    V3 G{0, 0, 0};
    // Akinci
    const bool do_A = (what & FORCE_AKINCI) && ph == kLiquid;
    V3 accA{0, 0, 0};
    const float akc = P.support;
    const float psi = P.rho0[0] * P.vol0;
    // density rate
    const bool do_D = (what & FORCE_DRHO) != 0;
    const V3 veli = P.tvf ? xyz(vti4) : vi;
    float div = 0.0f, diff = 0.0f;
    // thermal: the harmonic conductivity per neighbour phase
    // (phase_change.cu:57-61), evaluated once per particle
    const float ki = P.k[pi_idx];
    const float k_pair0 = 4.0f * ki * P.k[0] / (ki + P.k[0]);
    const float k_pair1 = 4.0f * ki * P.k[1] / (ki + P.k[1]);
    float q = 0.0f;

    constexpr int kUnroll = (FORCES_UNROLL_HEAVY > 1 && WHAT >= 0 && (WHAT & (FORCE_CSF | FORCE_THERMAL)))
                                ? FORCES_UNROLL_HEAVY : 1;
    for_each_nbr<kUnroll>(P, V, i, xi, [&](int j, float4 xj, V3 rij, float r2) {
      if (j == i) return;
      const float r = sqrtf(r2);
      const float dW = kernel_dWdr(P, r);
      const bool separated = r > 1e-12f * h;
      const V3 gw = separated ? rij * (dW / r) : V3{0, 0, 0};  // == kernel_gradW
      const int phj = ph_of(xj);
      if (phj == kWall) {
        const float4 mrj = __ldg(V.mrps + j);
        const float4 vwj = __ldg(V.vwp + j);
        if (do_T) {
          float rho_w;
          if (ph == kVapor) {
            rho_w = (vwj.w - (P.p_bg - P.vapor_K)) / (P.gas_R * Ti);
          } else {
            const float ratio = (mrj.z - P.p_bg) / P.tait_B + 1.0f;
            rho_w = P.rho0[0] * powf(ratio > 0.5f ? ratio : 0.5f, inv_gamma);
          }
          const float Vj = rho_w > 0.0f ? VT_i * rhoi / rho_w : VT_i;
          sumT += gw * (VT_i2 + Vj * Vj);
        }
        if (what & FORCE_MOMENTUM) {
          const V3 f_before = force, a_before = acc_av;
          const float Vj = P.vol0;
          const float vsum = Vi2 + Vj * Vj;
          const float pw = ph == kVapor ? vwj.w : mrj.z;
          force -= gw * (vsum * 0.5f * (pi + pw));
          if (tvf_stress) force += vi * (0.5f * vsum * rhoi * dot(dvi, gw));
          if (r < r_guard && separated) {
            const float qg = 1.0f - r / r_guard;
            const V3 nn = rij / r;
            acc_av += nn * (4.0f * ci * ci * qg * qg / r_guard);
            const float vn = dot(vi, nn);
            if (vn < 0.0f && dt > 0.0f) acc_av -= nn * (qg * vn / dt);
          }
          if (P.no_slip) {
            const V3 vij = vi - xyz(vwj);
            if (separated) force += vij * (vsum * etai * dW / r);
            const float vr = dot(vij, rij);
            if (alpha_i > 0.0f && vr < 0.0f) {
              const float mu_ij = h * vr / (r2 + eta2);
              const float Pi = -alpha_i * ci * mu_ij / rhoi;
              acc_av -= gw * (rhoi * P.vol0 * Pi);
            }
          }
          const V3 dF = (force - f_before) + (acc_av - a_before) * mi;
          fwall += dF;
          mwall += cross(xyz(xj) - origin, dF);
        }
        if (do_A && r2 > 0.0f) accA -= (rij / r) * (P.akinci_beta * psi * akinci_adhesion(r, akc));
        if (do_D) div += P.vol0 * dot(veli, gw);
        if (thermal && iso_walls) {
          const float Tw = __ldg(V.vT + j).w;
          if (Ti != Tw) {  // equal temperatures: a zero term
            const float kij = 2.0f * ki;
            const float rgw = r * dW;
            q += Vi * P.vol0 * kij * (Ti - Tw) * rgw / (r2 + eta2);
          }
        }
        return;
      }
      // fluid neighbour
      const float4 mrj = __ldg(V.mrps + j);
      const float4 vTj = __ldg(V.vT + j);
      const float4 axj = __ldg(V.aux + j);  // {m_j / rho_j, 1 / sigma_j, c_j}
      const float mj = mrj.x, rhoj = mrj.y;
      if (do_T) {
        const float Vj = axj.y;
        sumT += gw * (VT_i2 + Vj * Vj);
      }
      const float Vj = axj.x;
      if (what & FORCE_MOMENTUM) {
        const float vsum = Vi2 + Vj * Vj;
        const float pt = (rhoj * pi + rhoi * mrj.z) / (rhoi + rhoj);
        force -= gw * (vsum * pt);
        if (tvf_stress) {
          const V3 vj = xyz(vTj);
          const V3 Ag = vi * (rhoi * dot(dvi, gw)) + vj * (rhoj * dot(xyz(__ldg(V.vt + j)) - vj, gw));
          force += Ag * (0.5f * vsum);
        }
        const V3 vij = vi - xyz(vTj);
        if (P.sps) {
          const float etaj = P.mu[phase_index(phj)] + rhoj * V.nu_t[j];
          const float eta_sum = etai + etaj;
          if (eta_sum > 0.0f && separated) {
            const float eta_ij = 2.0f * etai * etaj / eta_sum;
            force += vij * (vsum * eta_ij * dW / r);
          }
        } else {
          const float eta_ij = phj == kVapor ? eta_pair1 : eta_pair0;
          if (eta_ij != 0.0f && separated) force += vij * (vsum * eta_ij * dW / r);
        }
        if (alpha_i > 0.0f && phj == ph) {
          const float vr = dot(vij, rij);
          if (vr < 0.0f) {
            const float cj = axj.z;
            const float mu_ij = h * vr / (r2 + eta2);
            const float Pi = -alpha_i * 0.5f * (ci + cj) * mu_ij / (0.5f * (rhoi + rhoj));
            acc_av -= gw * (mj * Pi);
          }
        }
      }
      if (do_C) {
        const V3 gwC = separated ? gw : rij * (dW / r);  // the same product where gw is not zeroed
        const V3 nj = xyz(__ldg(V.ns4 + j));
        if (norm2(nj) > 0.25f) {
          num += Vj * dot(ni - nj, gwC);
          den += Vj * r * (-dW);
        }
        if (P.csf_balanced) {
          const float cj = phj == kLiquid ? 1.0f : 0.0f;
          G += gwC * ((Vi * Vi + Vj * Vj) * (rhoj * ciC + rhoi * cj) / (rhoi + rhoj));
        }
      }
      if (do_A && phj == kLiquid && r2 > 0.0f) {
        const V3 rhat = rij / r;
        const float K = 2.0f * P.rho0[0] / (rhoi + rhoj);
        const V3 f_coh = rhat * (-P.akinci_gamma * mi * mj * akinci_cohesion(r, akc));
        const V3 f_curv = (xyz(nrmi) - xyz(__ldg(V.nrm + j))) * (-P.akinci_gamma * mi);
        accA += (f_coh + f_curv) * (K / mi);
      }
      if (do_D) {
        const V3 velj = P.tvf ? xyz(__ldg(V.vt + j)) : xyz(vTj);
        div += Vj * dot(veli - velj, gw);
        if (phj == ph) diff += Vj * 2.0f * (rhoj - rhoi) * dot(-rij, gw) / (r2 + eta2);
      }
      // equal temperatures give a zero term that leaves q as it is
      if (thermal && Ti != vTj.w) {
        const float kij = phj == kVapor ? k_pair1 : k_pair0;
        const float rgw = r * dW;
        q += Vi * Vj * kij * (Ti - vTj.w) * rgw / (r2 + eta2);
      }
    });

    if constexpr (WHAT >= 0 && (WHAT & FORCE_TAPE)) {
      const int tn = V.tape_n;
      V.tape[i] = f4(force, q);
      V.tape[tn + i] = f4(sumT, num);
      V.tape[2 * tn + i] = make_float4(den, 0.0f, 0.0f, 0.0f);
    }
    V3 ab{0, 0, 0};
    if (what & FORCE_TRANSPORT) {
      if (do_T) ab = sumT * (-pb / mT_i);
      V.ab4[i] = f4(ab, V.ab4[i].w);
    }
    float4 a4 = V.a4[i];
    V3 acc = xyz(a4);
    if (what & FORCE_MOMENTUM) {
      const V3 grav = v3(dyn->fr.gravity[0], dyn->fr.gravity[1], dyn->fr.gravity[2]);
      acc = grav + force / mi + acc_av;
      if (dyn->fr.frame_rot) {
        const V3 omega = v3(dyn->fr.omega[0], dyn->fr.omega[1], dyn->fr.omega[2]);
        const V3 omega_dot = v3(dyn->fr.omega_dot[0], dyn->fr.omega_dot[1], dyn->fr.omega_dot[2]);
        const V3 rr = xi - origin;
        acc -= cross(omega_dot, rr) + cross(omega, cross(omega, rr)) + cross(omega, vi) * 2.0f;
      }
      V.fw[i] = f4(fwall, 0.0f);
      V.mw[i] = f4(mwall, 0.0f);
    }
    if (what & FORCE_CSF) {
      float4 ns4 = V.ns4[i];
      if (!do_C) {
        ns4.w = 0.0f;
      } else {
        const float kappa = den > 0.0f ? 3.0f * num / den : 0.0f;
        ns4.w = kappa;
        if (P.wetting_model != 0) acc += xyz(V.vwp[i]);
        if (P.csf_balanced) acc += G * (P.sigma * kappa / mi);
        else acc += xyz(nrmi) * (csf_coeff * kappa);
      }
      V.ns4[i] = ns4;
    }
    if (do_A) acc += accA;
    if (do_D) reinterpret_cast<float*>(V.ab4 + i)[3] = rhoi * div + P.delta_sph * h * P.c0 * diff;
    if (thermal) {
      q += P.heat_power * V.heat_w[i] * dyn->heat_inv_norm;
      a4.w = q / (mi * P.cp[pi_idx]);
    }
    V.a4[i] = f4(acc, a4.w);

    if ((what & FORCE_MAXIMA) && owned(own_lo, own_hi, n_sorted, i)) {
      vmax_l = fmaxf(vmax_l, norm(vi));
      const float rm = V.rmin[i];
      const float rr = rm > 0.05f * P.dx ? rm : 0.05f * P.dx;
      sr_l = fmaxf(sr_l, 0.5f * P.dx / rr);
      const float aa = norm(acc), bb = norm(ab);
      amax_l = fmaxf(amax_l, aa > bb ? aa : bb);
      if (ph == kVapor) tv_l = fmaxf(tv_l, Ti);
      if (P.sps) nut_l = fmaxf(nut_l, V.nu_t[i]);
    }
  }
  if (what & FORCE_MAXIMA) {
    vmax_l = warp_max(vmax_l);
    amax_l = warp_max(amax_l);
    tv_l = warp_max(tv_l);
    sr_l = warp_max(sr_l);
    nut_l = warp_max(nut_l);
    if ((threadIdx.x & 31) == 0) {
      atomic_max_pos(&dyn->v_max, vmax_l);
      atomic_max_pos(&dyn->a_max, amax_l);
      if (P.has_vapor) atomic_max_pos(&dyn->Tv_max, tv_l);
      atomic_max_pos(&dyn->spacing_ratio, sr_l);
      if (P.sps) atomic_max_pos(&dyn->nu_t_max, nut_l);
    }
  }
}

// Instances: the generic one and every step-path sub-pass set.
template __global__ void k_forces_t<-1>(Params, View, int);
template __global__ void k_forces_t<67>(Params, View, int);
template __global__ void k_forces_t<99>(Params, View, int);
template __global__ void k_forces_t<83>(Params, View, int);
template __global__ void k_forces_t<115>(Params, View, int);
template __global__ void k_forces_t<75>(Params, View, int);
template __global__ void k_forces_t<107>(Params, View, int);
template __global__ void k_forces_t<91>(Params, View, int);
template __global__ void k_forces_t<123>(Params, View, int);
template __global__ void k_forces_t<71>(Params, View, int);
template __global__ void k_forces_t<103>(Params, View, int);
template __global__ void k_forces_t<87>(Params, View, int);
template __global__ void k_forces_t<119>(Params, View, int);
// taped variants (FORCE_TAPE) of the sub-pass sets the adjoint covers
template __global__ void k_forces_t<323>(Params, View, int);
template __global__ void k_forces_t<355>(Params, View, int);
template __global__ void k_forces_t<327>(Params, View, int);
template __global__ void k_forces_t<359>(Params, View, int);

// Maxima only (CRYO_PASS_MAXIMA; sph_solver.cu:475-479), from the stored fields.
__global__ void __launch_bounds__(kBlock) k_maxima(Params P, View V) {
  DynState* dyn = V.dyn;
  const int n = dyn->n;
  const int own_lo = dyn->own_lo, own_hi = dyn->own_hi, n_sorted = dyn->n_sorted;
  float vmax_l = 0.0f, amax_l = 0.0f, tv_l = 0.0f, sr_l = 0.0f, nut_l = 0.0f;
  PARTICLE_LOOP(i, n) {
    const int ph = ph_of(V.xp[i]);
    if (!is_fluid(ph) || !owned(own_lo, own_hi, n_sorted, i)) continue;
    const float4 vT = V.vT[i];
    vmax_l = fmaxf(vmax_l, norm(xyz(vT)));
    const float rm = V.rmin[i];
    const float rr = rm > 0.05f * P.dx ? rm : 0.05f * P.dx;
    sr_l = fmaxf(sr_l, 0.5f * P.dx / rr);
    const float aa = norm(xyz(V.a4[i])), bb = norm(xyz(V.ab4[i]));
    amax_l = fmaxf(amax_l, aa > bb ? aa : bb);
    if (ph == kVapor) tv_l = fmaxf(tv_l, vT.w);
    if (P.sps) nut_l = fmaxf(nut_l, V.nu_t[i]);
  }
  vmax_l = warp_max(vmax_l);
  amax_l = warp_max(amax_l);
  tv_l = warp_max(tv_l);
  sr_l = warp_max(sr_l);
  nut_l = warp_max(nut_l);
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&dyn->v_max, vmax_l);
    atomic_max_pos(&dyn->a_max, amax_l);
    if (P.has_vapor) atomic_max_pos(&dyn->Tv_max, tv_l);
    atomic_max_pos(&dyn->spacing_ratio, sr_l);
    if (P.sps) atomic_max_pos(&dyn->nu_t_max, nut_l);
  }
}

// apply_particle_shifting, pass 1 (SPH_kernels.cu:113-152): shift into ns.
__global__ void __launch_bounds__(kBlock) k_shift_compute(Params P, View V) {
  DynState* dyn = V.dyn;
  const int n = dyn->n;
  const float mach = dyn->v_max / P.c0;
  const float h = P.h;
  const float w_dx = kernel_W(P, P.dx);
  const float coeff = P.shift_strength * mach * 4.0f * h * h;
  const float cap = 0.1f * P.dx;
  const int own_lo = V.dyn->own_lo, own_hi = V.dyn->own_hi, n_sorted = V.dyn->n_sorted;  // a slab skips its ghosts
  PARTICLE_LOOP(i, n) {
    if (!owned(own_lo, own_hi, n_sorted, i)) continue;
    const float kap = V.ns4[i].w;
    V.ns4[i] = make_float4(0.0f, 0.0f, 0.0f, kap);
    const float4 xpi = V.xp[i];
    const int ph = ph_of(xpi);
    const float sigmai = V.mrps[i].w;
    if (!is_fluid(ph) || sigmai < P.tvf_sigma_min) continue;
    V3 sum{0, 0, 0};
    for_each_nbr(P, V, i, xyz(xpi), [&](int j, float4 xj, V3 rij, float r2) {
      if (j == i) return;
      const int phj = ph_of(xj);
      if (phj == kDead) return;
      const float r = sqrtf(r2);
      const float Vj = phj == kWall ? 1.0f / sigmai : 1.0f / __ldg(V.mrps + j).w;
      const float qq = kernel_W(P, r) / w_dx;
      const float q2 = qq * qq;
      sum += kernel_gradW(P, rij, r) * (Vj * (1.0f + 0.2f * q2 * q2));
    });
    V3 dr = sum * (-coeff);
    const float4 nrmi = V.nrm[i];
    if (nrmi.w > 0.0f) {
      const float gm = norm(xyz(nrmi));
      if (gm > P.normal_eps) {
        const V3 nn = xyz(nrmi) / gm;
        dr -= nn * dot(dr, nn);
      } else {
        dr = V3{0, 0, 0};
      }
    }
    const float len = norm(dr);
    if (len > cap) dr = dr * (cap / len);
    V.ns4[i] = f4(dr, kap);
  }
}

// apply_particle_shifting, pass 2 (SPH_kernels.cu:154-159).
__global__ void __launch_bounds__(kBlock) k_shift_apply(Params P, View V) {
  const int n = V.dyn->n;
  const int own_lo = V.dyn->own_lo, own_hi = V.dyn->own_hi, n_sorted = V.dyn->n_sorted;  // a slab skips its ghosts
  PARTICLE_LOOP(i, n) {
    if (!owned(own_lo, own_hi, n_sorted, i)) continue;
    float4 xp = V.xp[i];
    if (!is_fluid(ph_of(xp))) continue;
    const V3 x = xyz(xp) + xyz(V.ns4[i]);
    xp.x = x.x;
    xp.y = x.y;
    xp.z = x.z;
    V.xp[i] = xp;
  }
}

// probe_liquid_pressure (sph_solver.cu:197-216)
__global__ void k_probe(Params P, View V, const float* __restrict__ pts, int np, float* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
    const V3 x = v3(pts[3 * k], pts[3 * k + 1], pts[3 * k + 2]);
    float num = 0.0f, den = 0.0f;
    for_each_neighbor(P, V.cell_begin, V.xp, x, [&](int j, float4 xj, V3, float r2) {
      if (ph_of(xj) != kLiquid) return;
      const float4 mr = __ldg(V.mrps + j);
      const float w = (mr.x / mr.y) * kernel_W(P, sqrtf(r2));
      num += mr.z * w;
      den += w;
    });
    out[k] = den > 0.0f ? num / den : __int_as_float(0x7fc00000);
  }
}

}  // namespace CRYO_FIELD_NS
}  // namespace cryo
