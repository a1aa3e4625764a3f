// cryo_adjoint.cu -- reverse passes of Solver::step (sph_solver.cu:511-533)
// for the differentiated window: the step's passes in reverse order, each the
// exact derivative of the forward kernel's arithmetic with the step's
// neighbour sets, phases and branch decisions held fixed.
//
// Forward kernels and the reference functions they restate:
//   k_kick_drift_keys  kick_drift (sph_solver.cu:20-34)
//   k_density          compute_density_summation + EOS (SPH_kernels.cu:6-34, navier_stokes.cu:5-14)
//   k_wall             compute_wall_boundary (navier_stokes.cu:16-69)
//   k_interface        compute_interface_fields (surface_tension.cu:5-85)
//   k_forces_t         transport, momentum, CSF, thermal (SPH_kernels.cu:56-104,
//                      navier_stokes.cu:121-245, surface_tension.cu:120-177, phase_change.cu:31-75)
//   k_kick             kick + phase_change_sources (sph_solver.cu:36-46, phase_change.cu:77-137)
//   k_pc_normalize     phase_change_normalize (phase_change.cu:139-172)
//   k_pc_apply         phase_change_apply (phase_change.cu:174-215)
//   k_rebalance1/2     rebalance_vapor_mass (phase_change.cu:217-268)
//   k_saturation       update_saturation (sph_solver.cu:586-607)
#include "cryo_adjoint.cuh"

namespace cryo {

#define PARTICLE_LOOP(i, n) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

namespace {

// F(r) = W'(r) / r and dF/dr of the smoothing kernel (SPH_kernels.cuh:34-64):
// grad W = r_vec F, W' = r F, W'' = F + r F'.
__device__ inline void kernel_F(const Params& P, float r, float& F, float& dF) {
  const float q = r * P.inv_h;
  if (q >= 2.0f) {
    F = 0.0f;
    dF = 0.0f;
    return;
  }
  const float ih2 = P.inv_h * P.inv_h, ih3 = ih2 * P.inv_h;
  if (P.ktype == CRYO_KERNEL_CUBIC) {
    if (q < 1.0f) {
      F = P.knorm * ih2 * (-3.0f + 2.25f * q);
      dF = P.knorm * ih3 * 2.25f;
    } else {
      const float t = 2.0f - q;
      F = -0.75f * P.knorm * ih2 * t * t / q;
      dF = 0.75f * P.knorm * ih3 * (2.0f * t * q + t * t) / (q * q);
    }
    return;
  }
  const float t = 1.0f - 0.5f * q;
  F = -5.0f * P.knorm * ih2 * t * t * t;
  dF = 7.5f * P.knorm * ih3 * t * t;
}

// Adjoint of grad W = r_vec F(r) with respect to r_vec, for upstream u.
__device__ inline V3 gradW_vjp(V3 rv, float r, float F, float dF, V3 u) {
  return u * F + rv * (dF * dot(u, rv) / r);
}

__device__ inline Reduce rows(const Adj& A, int row0) {
  return Reduce{A.partials + (size_t)row0 * A.max_chunks, A.ticket, A.max_chunks};
}
// Particle order of a gather's threads: the fluid particles' index list,
// then (with walls) the wall particles' list, so a warp runs one kind of
// loop; every particle (phase filtered in the body) without lists.
struct PhaseOrder {
  const int* f;
  const int* w;
  int nf, total;
};
__device__ inline PhaseOrder phase_order(const Params& P, const View& V, bool walls) {
  const int n = V.dyn->n;
  if (!P.use_lists) return PhaseOrder{nullptr, nullptr, n, n};
  const int nf = V.dyn->n_fluid_list;
  return PhaseOrder{V.fluid_idx, V.wall_idx, nf, walls ? nf + V.dyn->n_wall_list : nf};
}
__device__ inline int order_at(const PhaseOrder& o, int t) {
  if (!o.f) return t;
  return t < o.nf ? __ldg(o.f + t) : __ldg(o.w + (t - o.nf));
}

__device__ inline void add4(float4* p, V3 a, float w) {
  float4 v = *p;
  v.x += a.x;
  v.y += a.y;
  v.z += a.z;
  v.w += w;
  *p = v;
}
__device__ inline float4 zero4() { return make_float4(0.0f, 0.0f, 0.0f, 0.0f); }

// Temperature after the kick, as k_kick computes it (sph_solver.cu:43-44).
__device__ inline float kicked_T(const Adj& A, int i) {
  float T = A.vT1[i].w;
  if (A.dyn1->thermal_on) T += A.V.a4[i].w * A.dyn1->dt;
  return T;
}

// out_m of phase_change_sources before the normalisation (pc_source_one).
__device__ inline float source_out_m(const Params& P, int ph, float m, float T, float alpha, float Ts, float dt) {
  const int ii = phase_index(ph);
  if (m < P.merge_ratio * P.mref[ii]) return m;
  if (!(P.phase_change && alpha > 0.0f && dt > 0.0f)) return 0.0f;
  if (ph == kLiquid && T > Ts) {
    const float h_out = P.h_fg + P.cp[1] * (Ts - P.T_ref);
    const float latent = h_out - P.cp[0] * (Ts - P.T_ref);
    const float rate = P.lee_evap * m * alpha * (T - Ts) / Ts;
    float dm = rate * dt;
    const float dm_energy = m * P.cp[0] * (T - Ts) / latent;
    dm = dm < dm_energy ? dm : dm_energy;
    const float dm_cap = P.max_transfer_fraction * m;
    dm = dm < dm_cap ? dm : dm_cap;
    return dm > 0.0f ? dm : 0.0f;
  }
  if (ph == kVapor && T < Ts) {
    const float rate = P.lee_cond * m * alpha * (Ts - T) / Ts;
    float dm = rate * dt;
    float dm_cap = P.max_transfer_fraction * m;
    if (P.pc_density_limit > 0.0f && P.pc_density_limit * m < dm_cap) dm_cap = P.pc_density_limit * m;
    dm = dm < dm_cap ? dm : dm_cap;
    return dm > 0.0f ? dm : 0.0f;
  }
  return 0.0f;
}

// Adjoint of (out_m, out_h) of pc_source_one for upstream (omb, hb).
struct SourceBar {
  float m, T, alpha, Ts, lee_e, lee_c;
};
__device__ inline void source_adjoint(const Params& P, int ph, float m, float T, float alpha, float Ts, float dt,
                                      float omb, float hb, SourceBar& b) {
  const int ii = phase_index(ph);
  if (m < P.merge_ratio * P.mref[ii]) {  // merge: out = (m, h(T))
    b.m += omb;
    b.T += hb * P.cp[ii];
    return;
  }
  if (!(P.phase_change && alpha > 0.0f && dt > 0.0f)) return;
  if (ph == kLiquid && T > Ts) {
    const float h_out = P.h_fg + P.cp[1] * (Ts - P.T_ref);
    const float latent = h_out - P.cp[0] * (Ts - P.T_ref);
    const float rate = P.lee_evap * m * alpha * (T - Ts) / Ts;
    const float d_rate = rate * dt;
    const float d_en = m * P.cp[0] * (T - Ts) / latent;
    float dm = d_rate < d_en ? d_rate : d_en;
    int which = d_rate < d_en ? 0 : 1;
    const float cap = P.max_transfer_fraction * m;
    if (!(dm < cap)) which = 2;
    dm = dm < cap ? dm : cap;
    if (!(dm > 0.0f)) return;
    b.Ts += hb * P.cp[1];  // h_out = h_fg + cp_v (T_sat - T_ref)
    if (which == 0) {
      const float g = omb * dt;
      const float x = (T - Ts) / Ts;
      b.lee_e += g * m * alpha * x;
      b.m += g * P.lee_evap * alpha * x;
      b.alpha += g * P.lee_evap * m * x;
      const float k = g * P.lee_evap * m * alpha;
      b.T += k / Ts;
      b.Ts += -k * T / (Ts * Ts);
    } else if (which == 1) {
      b.m += omb * P.cp[0] * (T - Ts) / latent;
      b.T += omb * m * P.cp[0] / latent;
      b.Ts += omb * m * P.cp[0] * (-latent - (T - Ts) * (P.cp[1] - P.cp[0])) / (latent * latent);
    } else {
      b.m += omb * P.max_transfer_fraction;
    }
  } else if (ph == kVapor && T < Ts) {
    const float rate = P.lee_cond * m * alpha * (Ts - T) / Ts;
    const float d_rate = rate * dt;
    float cap = P.max_transfer_fraction * m, capf = P.max_transfer_fraction;
    if (P.pc_density_limit > 0.0f && P.pc_density_limit * m < cap) {
      cap = P.pc_density_limit * m;
      capf = P.pc_density_limit;
    }
    const int which = d_rate < cap ? 0 : 2;
    const float dm = d_rate < cap ? d_rate : cap;
    if (!(dm > 0.0f)) return;
    b.T += hb * P.cp[1];  // out_h = h_v(T)
    if (which == 0) {
      const float g = omb * dt;
      const float x = (Ts - T) / Ts;
      b.lee_c += g * m * alpha * x;
      b.m += g * P.lee_cond * alpha * x;
      b.alpha += g * P.lee_cond * m * x;
      const float k = g * P.lee_cond * m * alpha;
      b.T += -k / Ts;
      b.Ts += k * T / (Ts * Ts);
    } else {
      b.m += omb * capf;
    }
  }
}

// ------------------------------------------------------------ force pass
// One particle's values as the force pass reads them.  For a wall: p is
// the liquid-side wall pressure, p_wv the vapour-side one, v the ghost
// velocity.
struct FP {
  V3 x, v, ns;
  float T, m, rho, p, V, VT, c, p_wv;
  int ph;
};
// The pair's own particle i: its per-particle constants.
struct FI {
  FP f;
  float eta, av, ki, pb, mT, alpha;
  float eta_pair[2], k_pair[2];
  bool do_T, do_C;
};
// Upstream adjoints of particle i's force-pass sums.
struct FU {
  V3 f;   // of force (a / m)
  V3 av;  // of acc_av (= a)
  V3 sT;  // of sumT
  float num, den, q;
};
// Adjoints on one particle's force-pass inputs.
struct FA {
  V3 x, v, ns;
  float T, m, rho, p, V, VT, c, p_wv;
};

__device__ inline FP load_fluid(const Params& P, const Adj& A, int i, float4 xpi) {
  FP f;
  f.ph = ph_of(xpi);
  f.x = xyz(xpi);
  const float4 vT = __ldg(A.vT1 + i);
  f.v = xyz(vT);
  f.T = vT.w;
  const float4 mr = __ldg(A.V.mrps + i);
  f.m = __ldg(A.m1 + i);
  f.rho = mr.y;
  f.p = mr.z;
  f.V = f.m / f.rho;
  f.VT = 1.0f / mr.w;
  f.c = sound_speed(P, f.ph, f.T);
  f.ns = xyz(__ldg(A.ns1 + i));
  f.p_wv = 0.0f;
  return f;
}
__device__ inline FP load_wall(const Adj& A, int j, float4 xpj) {
  FP f{};
  f.ph = kWall;
  f.x = xyz(xpj);
  const float4 vw = __ldg(A.V.vwp + j);
  f.v = xyz(vw);
  f.p_wv = vw.w;
  f.p = __ldg(A.V.mrps + j).z;
  return f;
}
__device__ inline FI make_fi(const Params& P, const Adj& A, int i, const FP& f) {
  FI I;
  I.f = f;
  const int pi = phase_index(f.ph);
  I.eta = P.mu[pi];
  I.av = f.ph == kVapor ? P.alpha_av_vap : P.alpha_av;
  I.ki = P.k[pi];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const float eta_sum = I.eta + P.mu[q];
    I.eta_pair[q] = eta_sum > 0.0f ? 2.0f * I.eta * P.mu[q] / eta_sum : 0.0f;
    I.k_pair[q] = 4.0f * I.ki * P.k[q] / (I.ki + P.k[q]);
  }
  I.alpha = __ldg(A.V.nrm + i).w;
  const float sigma = __ldg(A.V.mrps + i).w;
  I.do_T = P.tvf && !(sigma < P.tvf_sigma_min) && !(P.tvf_interface_only && !(I.alpha > 0.0f));
  I.do_C = P.csf_active && norm2(f.ns) > 0.25f;
  I.pb = P.tvf_factor * P.rho0[pi] * f.c * f.c;
  I.mT = f.rho * f.VT;
  return I;
}
__device__ inline FU load_fu(const Adj& A, int i, float m) {
  FU U;
  const float4 u1 = __ldg(A.gU1 + i), u2 = __ldg(A.gU2 + i), u3 = __ldg(A.gU3 + i);
  U.av = xyz(u1);
  U.f = U.av / m;
  U.q = u1.w;
  U.sT = xyz(u2);
  U.num = u2.w;
  U.den = u3.x;
  return U;
}

// Derivative of the force-pass pair term (i, j) (k_forces_t, fluid i):
// OWN: with respect to i's inputs; otherwise to j's.  dFb: upstream of the
// pair's wall force increment dF (fw = sum dF, mw = sum (x_j - o) x dF).
template <bool OWN>
__device__ inline void forces_pair_adj(const Params& P, const FI& I, const FU& U, const FP& J, V3 rij, float r2,
                                       float dt, bool thermal, V3 dFb, FA& o) {
  const FP& Fi = I.f;
  const float h = P.h;
  const float eta2 = 0.01f * h * h;
  const float r = sqrtf(r2);
  if (!(r > 1e-12f * h)) return;  // coincident: every gradient term is zero
  float F, dF;
  kernel_F(P, r, F, dF);
  const float dW = r * F;
  const V3 gw = rij * F;
  V3 gwb{0, 0, 0}, rvb{0, 0, 0};
  float Fb = 0.0f, rb = 0.0f, r2b = 0.0f;
  if (J.ph == kWall) {
    if (I.do_T) {
      float rho_w, ratio = 0.0f;
      if (Fi.ph == kVapor) {
        rho_w = (J.p_wv - (P.p_bg - P.vapor_K)) / (P.gas_R * Fi.T);
      } else {
        ratio = (J.p - P.p_bg) / P.tait_B + 1.0f;
        rho_w = P.rho0[0] * powf(ratio > 0.5f ? ratio : 0.5f, 1.0f / P.tait_gamma);
      }
      const float Vw = rho_w > 0.0f ? I.f.VT * Fi.rho / rho_w : Fi.VT;
      gwb += U.sT * (Fi.VT * Fi.VT + Vw * Vw);
      const float s = dot(U.sT, gw);
      const float Vwb = 2.0f * Vw * s;
      if (OWN) o.VT += 2.0f * Fi.VT * s;
      if (rho_w > 0.0f) {
        if (OWN) {
          o.VT += Vwb * Fi.rho / rho_w;
          o.rho += Vwb * Fi.VT / rho_w;
        }
        const float rwb = -Vwb * Vw / rho_w;
        if (Fi.ph == kVapor) {
          if (OWN) o.T += -rwb * rho_w / Fi.T;
          else o.p_wv += rwb / (P.gas_R * Fi.T);
        } else if (ratio > 0.5f) {
          if (!OWN) o.p += rwb * rho_w / (P.tait_gamma * ratio * P.tait_B);
        }
      } else if (OWN) {
        o.VT += Vwb;
      }
    }
    const V3 Fp = U.f + dFb;          // force increments feed a (/ m) and dF
    const V3 Av = U.av + dFb * Fi.m;  // acc_av increments feed a and dF (x m)
    const float vsum = Fi.V * Fi.V + P.vol0 * P.vol0;
    const float pw = Fi.ph == kVapor ? J.p_wv : J.p;
    const float pa = 0.5f * (Fi.p + pw);
    gwb -= Fp * (vsum * pa);
    {
      const float s = -dot(Fp, gw);
      if (OWN) {
        o.V += 2.0f * Fi.V * s * pa;
        o.p += s * vsum * 0.5f;
      } else if (Fi.ph == kVapor) {
        o.p_wv += s * vsum * 0.5f;
      } else {
        o.p += s * vsum * 0.5f;
      }
    }
    V3 dacc{0, 0, 0};
    const float r_guard = 0.6f * P.dx;
    if (r < r_guard) {
      const float qg = 1.0f - r / r_guard;
      const V3 nn = rij / r;
      const float Ag = 4.0f * Fi.c * Fi.c * qg * qg / r_guard;
      dacc += nn * Ag;
      V3 nnb = Av * Ag;
      const float Agb = dot(Av, nn);
      if (OWN) o.c += Agb * 8.0f * Fi.c * qg * qg / r_guard;
      float qgb = Agb * 8.0f * Fi.c * Fi.c * qg / r_guard;
      const float vn = dot(Fi.v, nn);
      if (vn < 0.0f && dt > 0.0f) {
        const float B = qg * vn / dt;
        dacc -= nn * B;
        nnb -= Av * B;
        const float Bb = -dot(Av, nn);
        qgb += Bb * vn / dt;
        const float vnb = Bb * qg / dt;
        if (OWN) o.v += nn * vnb;
        nnb += Fi.v * vnb;
      }
      rb += -qgb / r_guard;
      rvb += nnb / r - rij * (dot(nnb, rij) / (r * r * r));
    }
    if (P.no_slip) {
      const V3 vij = Fi.v - J.v;
      {
        const float s = dot(Fp, vij);
        Fb += s * vsum * I.eta;
        const V3 vb = Fp * (vsum * I.eta * F);
        if (OWN) {
          o.V += 2.0f * Fi.V * s * I.eta * F;
          o.v += vb;
        } else {
          o.v -= vb;
        }
      }
      const float vr = dot(vij, rij);
      if (I.av > 0.0f && vr < 0.0f) {
        const float den = r2 + eta2;
        const float mu = h * vr / den;
        const float coef = -I.av * Fi.c * mu * P.vol0;  // rho_i vol0 Pi
        dacc -= gw * coef;
        gwb -= Av * coef;
        const float s = -dot(Av, gw);
        if (OWN) o.c += s * (-I.av * mu * P.vol0);
        const float mub = s * (-I.av * Fi.c * P.vol0);
        const float vrb = mub * h / den;
        r2b += -mub * mu / den;
        rvb += vij * vrb;
        if (OWN) o.v += rij * vrb;
        else o.v -= rij * vrb;
      }
    }
    if (OWN) o.m += dot(dFb, dacc);
  } else {
    // fluid neighbour
    if (I.do_T) {
      gwb += U.sT * (Fi.VT * Fi.VT + J.VT * J.VT);
      const float s = dot(U.sT, gw);
      o.VT += 2.0f * (OWN ? Fi.VT : J.VT) * s;
    }
    const float vsum = Fi.V * Fi.V + J.V * J.V;
    {
      const float D = Fi.rho + J.rho;
      const float pt = (J.rho * Fi.p + Fi.rho * J.p) / D;
      gwb -= U.f * (vsum * pt);
      const float s = -dot(U.f, gw);
      const float vsb = s * pt, ptb = s * vsum;
      if (OWN) {
        o.V += 2.0f * Fi.V * vsb;
        o.p += ptb * J.rho / D;
        o.rho += ptb * (J.p - pt) / D;
      } else {
        o.V += 2.0f * J.V * vsb;
        o.p += ptb * Fi.rho / D;
        o.rho += ptb * (Fi.p - pt) / D;
      }
    }
    const V3 vij = Fi.v - J.v;
    const float eta = I.eta_pair[phase_index(J.ph)];
    if (eta != 0.0f) {
      const float s = dot(U.f, vij);
      Fb += s * vsum * eta;
      const float vsb = s * eta * F;
      const V3 vb = U.f * (vsum * eta * F);
      if (OWN) {
        o.V += 2.0f * Fi.V * vsb;
        o.v += vb;
      } else {
        o.V += 2.0f * J.V * vsb;
        o.v -= vb;
      }
    }
    if (I.av > 0.0f && J.ph == Fi.ph) {
      const float vr = dot(vij, rij);
      if (vr < 0.0f) {
        const float den = r2 + eta2;
        const float mu = h * vr / den;
        const float cm = 0.5f * (Fi.c + J.c), rm = 0.5f * (Fi.rho + J.rho);
        const float Pi = -I.av * cm * mu / rm;
        gwb -= U.av * (J.m * Pi);
        const float s = -dot(U.av, gw);
        const float Pib = s * J.m;
        if (!OWN) o.m += s * Pi;
        o.c += 0.5f * Pib * (-I.av * mu / rm);
        o.rho += 0.5f * Pib * (-Pi / rm);
        const float mub = Pib * (-I.av * cm / rm);
        const float vrb = mub * h / den;
        r2b += -mub * mu / den;
        rvb += vij * vrb;
        if (OWN) o.v += rij * vrb;
        else o.v -= rij * vrb;
      }
    }
    if (I.do_C && norm2(J.ns) > 0.25f) {
      const V3 dn = Fi.ns - J.ns;
      gwb += dn * (U.num * J.V);
      const V3 nb = gw * (U.num * J.V);
      if (OWN) {
        o.ns += nb;
      } else {
        o.ns -= nb;
        o.V += U.num * dot(dn, gw) + U.den * r * (-dW);
      }
      rb += U.den * J.V * (-(dW + r * (F + r * dF)));
    }
    if (thermal) {
      const float kij = I.k_pair[phase_index(J.ph)];
      const float den = r2 + eta2;
      const float G = r2 * F / den;  // r W'(r) / (r^2 + eta^2)
      const float dT = Fi.T - J.T;
      const float qb = U.q;
      if (OWN) {
        o.V += qb * J.V * kij * dT * G;
        o.T += qb * Fi.V * J.V * kij * G;
      } else {
        o.V += qb * Fi.V * kij * dT * G;
        o.T -= qb * Fi.V * J.V * kij * G;
      }
      const float Gb = qb * Fi.V * J.V * kij * dT;
      r2b += Gb * (F / den - r2 * F / (den * den));
      rb += Gb * (r2 / den) * dF;
    }
  }
  rvb += gradW_vjp(rij, r, F, dF, gwb);
  rvb += rij * ((Fb * dF + rb) / r + 2.0f * r2b);
  if (OWN) o.x += rvb;
  else o.x -= rvb;
}

// A fluid particle's force-pass values from the records of
// k_adj_forces_local (no divisions at the use site).
struct FR {
  FP f;
  int bits;  // do_T | do_C << 1 | valid unit normal << 2
};
__device__ inline FR load_rec(const Adj& A, int i, float4 xpi) {
  FR r;
  r.f.ph = ph_of(xpi);
  r.f.x = xyz(xpi);
  r.f.v = xyz(__ldg(A.vT1 + i));
  r.f.ns = xyz(__ldg(A.ns1 + i));
  const float4 r1 = __ldg(A.R1 + i), r2 = __ldg(A.R2 + i);
  r.f.V = r1.x;
  r.f.VT = r1.y;
  r.f.c = r1.z;
  r.f.rho = r1.w;
  r.f.p = r2.x;
  r.f.T = r2.y;
  r.f.m = r2.z;
  r.f.p_wv = 0.0f;
  r.bits = __float_as_int(r2.w);
  return r;
}
// FI of a record (the fields the wall pairs use).
__device__ inline FI fi_of(const Params& P, const FR& r) {
  FI I;
  I.f = r.f;
  const int pi = phase_index(r.f.ph);
  I.eta = P.mu[pi];
  I.av = r.f.ph == kVapor ? P.alpha_av_vap : P.alpha_av;
  I.ki = P.k[pi];
  I.eta_pair[0] = I.eta_pair[1] = 0.0f;
  I.k_pair[0] = I.k_pair[1] = 0.0f;
  I.do_T = (r.bits & 1) != 0;
  I.do_C = (r.bits & 2) != 0;
  I.pb = 0.0f;
  I.mT = 0.0f;
  I.alpha = 0.0f;
  return I;
}

// Both directions of a fluid pair (k, l) of the force pass at once: the
// terms f(k, l) feeding k's outputs differentiated with respect to k's
// inputs, and the terms f(l, k) feeding l's outputs differentiated with
// respect to k's inputs.  The pair's pressure, viscous and conductive terms
// are equal and opposite, so both directions share one evaluation with the
// upstream adjoints combined (k's minus l's); artificial viscosity,
// transport velocity and curvature carry each side's own factors.
// eta, kc: the pair's harmonic viscosity and conductivity (symmetric).
__device__ inline void fluid_pair_both(const Params& P, const FR& K, const FU& Uk, const FR& L, const FU& Ul, V3 rkl,
                                       float r2, bool thermal, float eta, float kc, float av, FA& o) {
  const FP& a = K.f;
  const FP& b = L.f;
  const float h = P.h;
  const float eta2 = 0.01f * h * h;
  const float r = sqrtf(r2);
  if (!(r > 1e-12f * h)) return;
  const float ir = 1.0f / r;
  float F, dF;
  kernel_F(P, r, F, dF);
  const float dW = r * F;
  const V3 gw = rkl * F;  // grad W of (k, l); (l, k) has -gw
  V3 gwb{0, 0, 0}, rvb{0, 0, 0};
  float Fb = 0.0f, rb = 0.0f, r2b = 0.0f;
  // transport velocity: sumT_k += gw t (do_T_k), sumT_l -= gw t (do_T_l)
  {
    const bool tk = (K.bits & 1) != 0, tl = (L.bits & 1) != 0;
    if (tk || tl) {
      const V3 u = (tk ? Uk.sT : V3{0, 0, 0}) - (tl ? Ul.sT : V3{0, 0, 0});
      gwb += u * (a.VT * a.VT + b.VT * b.VT);
      o.VT += 2.0f * a.VT * dot(u, gw);
    }
  }
  const float vsum = a.V * a.V + b.V * b.V;
  const V3 du = Uk.f - Ul.f;  // force upstream, k's minus l's
  // pressure: force_k -= gw vsum pt, force_l += gw vsum pt
  {
    const float iD = 1.0f / (a.rho + b.rho);
    const float pt = (b.rho * a.p + a.rho * b.p) * iD;
    gwb -= du * (vsum * pt);
    const float s = -dot(du, gw);
    o.V += 2.0f * a.V * s * pt;
    const float ptb = s * vsum;
    o.p += ptb * b.rho * iD;
    o.rho += ptb * (b.p - pt) * iD;
  }
  const V3 vij = a.v - b.v;
  // viscosity: force_k += vij vsum eta F, force_l -= vij vsum eta F
  if (eta != 0.0f) {
    const float s = dot(du, vij);
    Fb += s * vsum * eta;
    o.V += 2.0f * a.V * s * eta * F;
    o.v += du * (vsum * eta * F);
  }
  const float iden = 1.0f / (r2 + eta2);
  // artificial viscosity (same phase, approaching): acc_k -= gw m_l Pi, acc_l += gw m_k Pi
  if (av > 0.0f && a.ph == b.ph) {
    const float vr = dot(vij, rkl);
    if (vr < 0.0f) {
      const float mu = h * vr * iden;
      const float cm = 0.5f * (a.c + b.c), irm = 2.0f / (a.rho + b.rho);
      const float Pi = -av * cm * mu * irm;
      const V3 w = Uk.av * b.m - Ul.av * a.m;
      gwb -= w * Pi;
      const float Pib = -dot(w, gw);
      o.m += Pi * dot(Ul.av, gw);
      o.c += 0.5f * Pib * (-av * mu * irm);
      o.rho += 0.5f * Pib * (-Pi * irm);
      const float mub = Pib * (-av * cm * irm);
      const float vrb = mub * h * iden;
      r2b += -mub * mu * iden;
      rvb += vij * vrb;
      o.v += rkl * vrb;
    }
  }
  // curvature: num_k += V_l dn.gw, den_k += V_l r (-dW) (do_C_k, valid n_l);
  //            num_l += V_k dn.gw, den_l += V_k r (-dW) (do_C_l, valid n_k)
  {
    const bool ck = (K.bits & 2) && (L.bits & 4), cl = (L.bits & 2) && (K.bits & 4);
    if (ck || cl) {
      const float an = ck ? Uk.num * b.V : 0.0f, bn = cl ? Ul.num * a.V : 0.0f;
      const V3 dn = a.ns - b.ns;
      gwb += dn * (an + bn);
      o.ns += gw * (an + bn);
      if (cl) o.V += Ul.num * dot(dn, gw) + Ul.den * r * (-dW);
      const float dd = (ck ? Uk.den * b.V : 0.0f) + (cl ? Ul.den * a.V : 0.0f);
      rb += dd * (-(dW + r * (F + r * dF)));
    }
  }
  // conduction: q_k += V_k V_l k (T_k - T_l) G, q_l -= the same
  if (thermal) {
    const float qd = Uk.q - Ul.q;
    const float G = r2 * F * iden;
    const float dT = a.T - b.T;
    o.V += qd * b.V * kc * dT * G;
    o.T += qd * a.V * b.V * kc * G;
    const float Gb = qd * a.V * b.V * kc * dT;
    r2b += Gb * (F * iden - r2 * F * iden * iden);
    rb += Gb * (r2 * iden) * dF;
  }
  rvb += gradW_vjp(rkl, r, F, dF, gwb);
  rvb += rkl * ((Fb * dF + rb) * ir + 2.0f * r2b);
  o.x += rvb;
}

// Rotation of the colour gradient toward the contact angle
// (surface_tension.cu:66-84): g' = normalized(nh (1 - b) + target b) |g|.
struct Rot {
  bool on;
  V3 g, wn;  // colour gradient and wall-normal sum before the rotation
  float ww;
};
__device__ inline void rotation_adjoint(const Params& P, const Rot& R, V3 gpb, V3& gb, V3& wnb, float& wwb,
                                        float& cosb, float& sinb) {
  gb = gpb;
  wnb = V3{0, 0, 0};
  wwb = 0.0f;
  if (!R.on) return;
  const float gmag = norm(R.g);
  const float wl = norm(R.wn);
  const V3 nw = wl > 1e-20f ? R.wn / wl : V3{0, 0, 0};
  const V3 nh = R.g / gmag;
  const float d = dot(nh, nw);
  const V3 t0 = nh - nw * d;
  const float tmag = norm(t0);
  const V3 t = t0 / tmag;
  const V3 target = nw * (-P.cos_theta) + t * P.sin_theta;
  const float bq = R.ww / P.wall_adhesion_weight;
  const float beta = clampf(bq, 0.0f, 1.0f);
  const V3 b0 = nh * (1.0f - beta) + target * beta;
  const float b0m = norm(b0);
  const V3 bl = b0m > 1e-20f ? b0 / b0m : V3{0, 0, 0};
  // g' = bl gmag
  const V3 blb = gpb * gmag;
  float gmagb = dot(gpb, bl);
  V3 b0b{0, 0, 0};
  if (b0m > 1e-20f) b0b = (blb - bl * dot(blb, bl)) / b0m;
  V3 nhb = b0b * (1.0f - beta);
  const V3 tgb = b0b * beta;
  const float betab = dot(b0b, target - nh);
  if (bq > 0.0f && bq < 1.0f) wwb = betab / P.wall_adhesion_weight;
  V3 nwb = tgb * (-P.cos_theta);
  cosb += -dot(tgb, nw);
  sinb += dot(tgb, t);
  const V3 tb = tgb * P.sin_theta;
  const V3 t0b = (tb - t * dot(tb, t)) / tmag;
  nhb += t0b;
  nwb -= t0b * d;
  const float db = -dot(t0b, nw);
  nhb += nw * db;
  nwb += nh * db;
  gb = (nhb - nh * dot(nhb, nh)) / gmag + nh * gmagb;
  if (wl > 1e-20f) wnb = (nwb - nw * dot(nwb, nw)) / wl;
}

}  // namespace

// ----------------------------------------------------------- saturation
// update_saturation (sph_solver.cu:586-607): the phase sums of the step's end
// state, then the factors d(objective)/d(m of a liquid particle) and
// d(objective)/d(m T of a vapour particle).
__global__ void __launch_bounds__(kBlock) k_adj_saturation_sums(Params P, Adj A) {
  __shared__ double sh[3 * kBlock / 32];
  const View& V = A.V;
  const DynState* d = V.dyn;
  const int n = d->n;
  const int nch = num_chunks(n);
  const Reduce R = rows(A, AR_SAT);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double s[3] = {0.0, 0.0, 0.0};
    if (i < n) {
      const int ph = ph_of(V.xp[i]);
      const double m = V.mrps[i].x;
      if (ph == kLiquid) s[0] = m;
      if (ph == kVapor) {
        s[1] = m;
        s[2] = m * V.vT[i].w;
      }
    }
    publish_chunk<3>(R, c, s, sh);
  }
  if (!last_block(A.ticket)) return;
  const double m_liq = block_sum_partials(R, 0, nch);
  const double m_vap = block_sum_partials(R, 1, nch);
  const double mT = block_sum_partials(R, 2, nch);
  if (threadIdx.x != 0) return;
  double cl = 0.0, ct = 0.0;
  if (P.thermo_closed && P.has_vapor) {
    const double v_u = d->fluid_volume0 - m_liq / P.f_rho_l;
    const double ratio = v_u > 0 && m_vap > 0 ? (mT / v_u) / ((double)P.f_rho_v * P.f_T_sat) : 0.0;
    if (isfinite(ratio) && ratio > 0) {
      const double p = d->p_ullage;
      const double Ts = d->T_sat;
      const double dTs_dp = Ts * Ts * ((double)P.f_R_gas / P.f_h_fg) / p;
      const double pb = A.glob[AG_P_OBJ] + A.glob[AG_TSAT_OUT] * dTs_dp;
      cl = pb * p / (v_u * P.f_rho_l);
      ct = pb * p / mT;
    }
  }
  A.glob[AG_C_LIQ] = cl;
  A.glob[AG_C_MT] = ct;
}

// ---------------------------------------------------------- rebalance
// rebalance_vapor_mass pass 2 (phase_change.cu:252-267) per vapour particle,
// after the saturation factors are added; stores the adjoints of the pass-1
// sums (dm, dH, dP).  Also clears the per-step adjoint components.
__global__ void __launch_bounds__(kBlock) k_adj_rebalance_local(Params P, Adj A) {
  const View& V = A.V;
  const int n = V.dyn->n;
  const double cl = A.glob[AG_C_LIQ], ct = A.glob[AG_C_MT];
  const bool reb = P.vapor_rebalance > 0.0f && P.has_vapor;
  const float beta = P.vapor_rebalance;
  PARTICLE_LOOP(i, n) {
    float4 ga = A.gA[i], gb = A.gB[i];
    ga.w = 0.0f;
    gb.w = 0.0f;
    A.gA[i] = ga;
    A.gB[i] = gb;
    A.gU1[i] = zero4();
    A.gU2[i] = zero4();
    const float4 xpi = V.xp[i];
    const int ph = ph_of(xpi);
    if (!is_fluid(ph)) {
      A.gX[i] = zero4();
      A.gV[i] = zero4();
      continue;
    }
    float4 gx = A.gX[i], gv = A.gV[i];
    const float m3 = V.mrps[i].x, T3 = V.vT[i].w;
    if (ph == kLiquid) {
      gx.w += (float)cl;
    } else {
      gx.w += (float)(ct * T3);
      gv.w += (float)(ct * m3);
    }
    if (reb && ph == kVapor) {
      const float m = A.m2[i];
      const float4 vT = A.vT2[i];
      const float hi = specific_enthalpy(P, kVapor, vT.w);
      const V3 vi = xyz(vT);
      float dm = 0.0f, dH = 0.0f;
      V3 dP{0, 0, 0};
      for_each_nbr(P, V, i, xyz(xpi), [&](int j, float4 xj, V3, float r2) {
        if (j == i || ph_of(xj) != kVapor) return;
        const float flow = beta * P.vol0 * kernel_W(P, sqrtf(r2)) * (__ldg(A.m2 + j) - m);
        dm += flow;
        if (flow > 0.0f) {
          const float4 vTj = __ldg(A.vT2 + j);
          dH += flow * specific_enthalpy(P, kVapor, vTj.w);
          dP += xyz(vTj) * flow;
        } else {
          dH += flow * hi;
          dP += vi * flow;
        }
      });
      if (dm != 0.0f) {
        const float mn = m + dm;
        const float H = m * hi + dH;
        const V3 vn = (vi * m + dP) / mn;
        const V3 vb = xyz(gv);
        const float hb = gv.w / P.cp[1];
        const float Hb = hb / mn;
        const float mnb = gx.w - hb * (H / mn) / mn - dot(vb, vn) / mn;
        A.gU1[i] = f4(vb / mn, mnb);                     // (dP, dm)
        A.gU2[i] = make_float4(Hb, 0.0f, 0.0f, 0.0f);    // dH
        gx.w = mnb + Hb * hi + dot(vb, vi) / mn;
        gv = f4(vb * (m / mn), Hb * m * P.cp[1]);
      }
    }
    A.gX[i] = gx;
    A.gV[i] = gv;
  }
}

// rebalance_vapor_mass pass 1 (phase_change.cu:223-250): the flow terms of
// every vapour pair, from both ends.
__global__ void __launch_bounds__(kBlock) k_adj_rebalance_gather(Params P, Adj A) {
  if (!(P.vapor_rebalance > 0.0f && P.has_vapor)) return;
  const View& V = A.V;
  const int n = V.dyn->n;
  const float bv = P.vapor_rebalance * P.vol0;
  const PhaseOrder ord = phase_order(P, V, false);
  PARTICLE_LOOP(t, ord.total) {
    const int k = order_at(ord, t);
    const float4 xpk = V.xp[k];
    if (ph_of(xpk) != kVapor) continue;
    const float mk = A.m2[k];
    const float4 vTk = A.vT2[k];
    const float hk = specific_enthalpy(P, kVapor, vTk.w);
    const float4 uk = A.gU1[k];
    const float dHk = A.gU2[k].x;
    V3 xb{0, 0, 0}, vb{0, 0, 0};
    float mb = 0.0f, Tb = 0.0f;
    for_each_nbr(P, V, k, xyz(xpk), [&](int l, float4 xl, V3 rkl, float r2) {
      if (l == k || ph_of(xl) != kVapor) return;
      const float r = sqrtf(r2);
      const float w = kernel_W(P, r);
      float F, dF;
      kernel_F(P, r, F, dF);
      const float ml = __ldg(A.m2 + l);
      const float4 vTl = __ldg(A.vT2 + l);
      const float hl = specific_enthalpy(P, kVapor, vTl.w);
      const float4 ul = __ldg(A.gU1 + l);
      const float dHl = __ldg(A.gU2 + l).x;
      {  // k's own sum over l
        const float flow = bv * w * (ml - mk);
        const bool from_l = flow > 0.0f;
        const float fb = uk.w + dHk * (from_l ? hl : hk) + dot(xyz(uk), from_l ? xyz(vTl) : xyz(vTk));
        xb += rkl * (fb * bv * (ml - mk) * F);
        mb -= fb * bv * w;
        if (!from_l) {
          Tb += dHk * flow * P.cp[1];
          vb += xyz(uk) * flow;
        }
      }
      {  // l's sum over k
        const float flow = bv * w * (mk - ml);
        const bool from_k = flow > 0.0f;
        const float fb = ul.w + dHl * (from_k ? hk : hl) + dot(xyz(ul), from_k ? xyz(vTk) : xyz(vTl));
        mb += fb * bv * w;
        xb += rkl * (fb * bv * (mk - ml) * F);
        if (from_k) {
          Tb += dHl * flow * P.cp[1];
          vb += xyz(ul) * flow;
        }
      }
    });
    add4(A.gX + k, xb, mb);
    add4(A.gV + k, vb, Tb);
  }
}

// ------------------------------------------------------- phase change
// phase_change_apply (phase_change.cu:174-215) per receiver: the enthalpy
// balance; stores the adjoints of its gathered sums (in_m, in_H) and of its
// own out_m / out_h.
__global__ void __launch_bounds__(kBlock) k_adj_apply_local(Params P, Adj A) {
  const View& V = A.V;
  const int n = V.dyn->n;
  PARTICLE_LOOP(i, n) {
    A.gU3[i] = zero4();
    const float4 xpi = V.xp[i];
    const int ph = ph_of(xpi);
    if (!is_fluid(ph)) continue;
    const int fl = fl_of(xpi);
    const int pi = phase_index(ph);
    const float m = A.m1[i];
    const float Vi = m / V.mrps[i].y;
    float in_m = 0.0f, in_H = 0.0f;
    if (!(fl & kDying)) {
      for_each_nbr(P, V, i, xyz(xpi), [&](int j, float4 xj, V3, float r2) {
        if (j == i || !(fl_of(xj) & kSource)) return;
        const float4 pcj = __ldg(A.pc2 + j);
        if (!(pcj.x > 0.0f)) return;
        const int target = (fl_of(xj) & kTargetVapor) ? kVapor : kLiquid;
        if (target != ph) return;
        const float share = pcj.x * Vi * kernel_W(P, sqrtf(r2)) / pcj.z;
        in_m += share;
        in_H += share * pcj.y;
      });
    }
    const float4 pci = A.pc2[i];
    const float om = pci.x;
    if ((fl & kDying) && om > 0.0f) {
      atomicOr(A.status, ADJ_TOPOLOGY);
      continue;
    }
    if (!(om > 0.0f) && !(in_m > 0.0f)) continue;
    const float m_new = m - om + in_m;
    const float T1 = kicked_T(A, i);
    const float hT = specific_enthalpy(P, ph, T1);
    const float H = m * hT - om * pci.y + in_H;
    float4 gx = A.gX[i], gv = A.gV[i];
    const float hb = gv.w / P.cp[pi];
    const float Hb = hb / m_new;
    const float mnb = gx.w - hb * (H / m_new) / m_new;
    gx.w = mnb + Hb * hT;
    gv.w = Hb * m * P.cp[pi];
    A.gX[i] = gx;
    A.gV[i] = gv;
    A.gC[i] = make_float4(-mnb - Hb * pci.y, -Hb * om, 0.0f, 0.0f);
    A.gU3[i] = make_float4(mnb, Hb, 0.0f, 0.0f);
  }
}

// The shares of phase_change_apply, from both ends: a receiver's volume and
// position, a source's out_m, out_h, w_norm and position.
__global__ void __launch_bounds__(kBlock) k_adj_apply_gather(Params P, Adj A) {
  const View& V = A.V;
  const int n = V.dyn->n;
  const PhaseOrder ord = phase_order(P, V, false);
  PARTICLE_LOOP(t, ord.total) {
    const int k = order_at(ord, t);
    const float4 xpk = V.xp[k];
    const int ph = ph_of(xpk);
    if (!is_fluid(ph)) continue;
    const int fl = fl_of(xpk);
    const float mk = A.m1[k], rk = V.mrps[k].y;
    const float Vk = mk / rk;
    const float4 uk = A.gU3[k];
    const float4 pck = A.pc2[k];
    const bool recv = !(fl & kDying) && (uk.x != 0.0f || uk.y != 0.0f);
    const bool src = (fl & kSource) && pck.x > 0.0f;
    if (!recv && !src) continue;
    const int target_k = (fl & kTargetVapor) ? kVapor : kLiquid;
    float Vb = 0.0f, omb = 0.0f, houtb = 0.0f, wnb = 0.0f;
    V3 xb{0, 0, 0};
    for_each_nbr(P, V, k, xyz(xpk), [&](int l, float4 xl, V3 rkl, float r2) {
      if (l == k) return;
      const int fll = fl_of(xl), phl = ph_of(xl);
      const float r = sqrtf(r2);
      if (recv && (fll & kSource)) {
        const float4 pcl = __ldg(A.pc2 + l);
        const int target_l = (fll & kTargetVapor) ? kVapor : kLiquid;
        if (pcl.x > 0.0f && target_l == ph) {
          float F, dF;
          kernel_F(P, r, F, dF);
          const float w = kernel_W(P, r);
          const float sb = uk.x + uk.y * pcl.y;
          Vb += sb * pcl.x * w / pcl.z;
          xb += rkl * (sb * pcl.x * Vk / pcl.z * F);
        }
      }
      if (src && phl == target_k && !(fll & kDying)) {
        const float4 ul = __ldg(A.gU3 + l);
        if (ul.x != 0.0f || ul.y != 0.0f) {
          float F, dF;
          kernel_F(P, r, F, dF);
          const float w = kernel_W(P, r);
          const float Vl = __ldg(A.m1 + l) / __ldg(A.V.mrps + l).y;
          const float share = pck.x * Vl * w / pck.z;
          const float sb = ul.x + ul.y * pck.y;
          omb += sb * Vl * w / pck.z;
          wnb -= sb * share / pck.z;
          houtb += ul.y * share;
          xb += rkl * (sb * pck.x * Vl / pck.z * F);
        }
      }
    });
    add4(A.gX + k, xb, Vb / rk);
    float4 gb = A.gB[k];
    gb.w -= Vb * Vk / rk;
    A.gB[k] = gb;
    float4 gc = A.gC[k];
    gc.x += omb;
    gc.y += houtb;
    gc.z += wnb;
    A.gC[k] = gc;
  }
}

// phase_change_normalize (phase_change.cu:139-172) per source: the density
// cap; stores the adjoints of w_sum and wr_max and the receiver that set
// wr_max.
__global__ void __launch_bounds__(kBlock) k_adj_normalize_local(Params P, Adj A) {
  const View& V = A.V;
  const int n = V.dyn->n;
  const float Ts = A.dyn1->T_sat, dt = A.dyn1->dt;
  PARTICLE_LOOP(i, n) {
    const float4 xpi = V.xp[i];
    const int fl = fl_of(xpi);
    A.argmax[i] = -1;
    if (!(fl & kSource)) continue;
    const int ph = ph_of(xpi);
    const int target = (fl & kTargetVapor) ? kVapor : kLiquid;
    float wsum = 0.0f, wr_max = 0.0f;
    int jmax = -1;
    for_each_nbr(P, V, i, xyz(xpi), [&](int j, float4 xj, V3, float r2) {
      if (j == i || ph_of(xj) != target || (fl_of(xj) & kDying)) return;
      const float w = kernel_W(P, sqrtf(r2));
      const float rhoj = __ldg(A.V.mrps + j).y;
      wsum += (__ldg(A.m1 + j) / rhoj) * w;
      const float wr = w / rhoj;
      if (wr > wr_max) {
        wr_max = wr;
        jmax = j;
      }
    });
    const float4 gc = A.gC[i];
    float omb = gc.x, wsb = gc.z, wrb = 0.0f;
    if (!(wsum > 0.0f)) {
      omb = 0.0f;
    } else if (target == kVapor && P.pc_density_limit > 0.0f && !(fl & kDying) && wr_max > 0.0f) {
      const float cap = P.pc_density_limit * wsum / wr_max;
      const float out = source_out_m(P, ph, A.m1[i], kicked_T(A, i), V.nrm[i].w, Ts, dt);
      if (out > cap) {
        wsb += omb * P.pc_density_limit / wr_max;
        wrb = -omb * cap / wr_max;
        omb = 0.0f;
      }
    }
    A.gC[i] = make_float4(omb, gc.y, wsb, wrb);
    A.argmax[i] = jmax;
  }
}

// The w_sum and wr_max terms of the normalisation, from both ends.
__global__ void __launch_bounds__(kBlock) k_adj_normalize_gather(Params P, Adj A) {
  const View& V = A.V;
  const int n = V.dyn->n;
  const PhaseOrder ord = phase_order(P, V, false);
  PARTICLE_LOOP(t, ord.total) {
    const int k = order_at(ord, t);
    const float4 xpk = V.xp[k];
    const int ph = ph_of(xpk);
    if (!is_fluid(ph)) continue;
    const int fl = fl_of(xpk);
    const bool src = (fl & kSource) != 0;
    const float4 gck = A.gC[k];
    const int amk = A.argmax[k];
    const int target_k = (fl & kTargetVapor) ? kVapor : kLiquid;
    const float mk = A.m1[k], rk = V.mrps[k].y;
    const float Vk = mk / rk;
    float Vb = 0.0f, rhob = 0.0f;
    V3 xb{0, 0, 0};
    for_each_nbr(P, V, k, xyz(xpk), [&](int l, float4 xl, V3 rkl, float r2) {
      if (l == k) return;
      const int fll = fl_of(xl), phl = ph_of(xl);
      const bool own = src && phl == target_k && !(fll & kDying);
      const bool cross = (fll & kSource) && !(fl & kDying) &&
                         ph == ((fll & kTargetVapor) ? kVapor : kLiquid);
      if (!own && !cross) return;
      const float r = sqrtf(r2);
      float F, dF;
      kernel_F(P, r, F, dF);
      if (own) {
        const float rl = __ldg(A.V.mrps + l).y;
        const float Vl = __ldg(A.m1 + l) / rl;
        xb += rkl * (gck.z * Vl * F);
        if (l == amk) xb += rkl * (gck.w * F / rl);
      }
      if (cross) {
        const float4 gcl = __ldg(A.gC + l);
        const float w = kernel_W(P, r);
        Vb += gcl.z * w;
        xb += rkl * (gcl.z * Vk * F);
        if (__ldg(A.argmax + l) == k) {
          rhob += gcl.w * (-w / (rk * rk));
          xb += rkl * (gcl.w * F / rk);
        }
      }
    });
    add4(A.gX + k, xb, Vb / rk);
    float4 gb = A.gB[k];
    gb.w += rhob - Vb * Vk / rk;
    A.gB[k] = gb;
  }
}

// ------------------------------------------------------------- kick
// phase_change_sources (phase_change.cu:77-137) and the kick
// (sph_solver.cu:36-46): v2 = v1 + a dt/2, T1 = T0 + dTdt dt.
__global__ void __launch_bounds__(kBlock) k_adj_kick_sources(Params P, Adj A) {
  __shared__ double sh[3 * kBlock / 32];
  const View& V = A.V;
  const int n = V.dyn->n;
  const int nch = num_chunks(n);
  const float dt = A.dyn1->dt, half = 0.5f * dt;
  const bool thermal = A.dyn1->thermal_on != 0;
  const float Ts = A.dyn1->T_sat;
  const bool do_src = P.cfg_phase_change && A.dyn1->phase_change_on;
  const Reduce R = rows(A, AR_SRC);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double s[3] = {0.0, 0.0, 0.0};
    if (i < n) {
      const float4 xpi = V.xp[i];
      const int ph = ph_of(xpi);
      if (is_fluid(ph)) {
        float4 gx = A.gX[i], gv = A.gV[i], ga = A.gA[i], gn = A.gN[i];
        const float T1 = kicked_T(A, i);
        SourceBar b{0, 0, 0, 0, 0, 0};
        if (do_src) {
          const float4 gc = A.gC[i];
          source_adjoint(P, ph, A.m1[i], T1, V.nrm[i].w, Ts, dt, gc.x, gc.y, b);
        }
        gx.w += b.m;
        gv.w += b.T;
        gn.w += b.alpha;
        ga.x += gv.x * half;
        ga.y += gv.y * half;
        ga.z += gv.z * half;
        if (thermal) ga.w += gv.w * dt;
        A.gX[i] = gx;
        A.gV[i] = gv;
        A.gA[i] = ga;
        A.gN[i] = gn;
        s[0] = b.Ts;
        s[1] = b.lee_e;
        s[2] = b.lee_c;
      }
    }
    publish_chunk<3>(R, c, s, sh);
  }
}

// ------------------------------------------------------------ forces
// Per fluid particle: the local part of the force pass's adjoint (a = g +
// force / m + acc_av + CSF, dTdt = q / (m cp), ab = sumT (-pb / mT)); stores
// the upstream coefficients its pairs need.
__global__ void __launch_bounds__(kBlock) k_adj_forces_local(Params P, Adj A) {
  __shared__ double sh[6 * kBlock / 32];
  const View& V = A.V;
  const DynState* d1 = A.dyn1;
  const int n = V.dyn->n;
  const int nch = num_chunks(n);
  const bool thermal = P.thermal && d1->thermal_on;
  const float csf_unit = 2.0f / (P.rho0[0] + P.rho0[1]);
  const float csf_coeff = P.sigma * csf_unit;
  const float hinv = d1->heat_inv_norm;
  const Reduce R = rows(A, AR_FORCE);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < n) {
      const float4 xpi = V.xp[i];
      const int ph = ph_of(xpi);
      if (is_fluid(ph)) {
        const FP f = load_fluid(P, A, i, xpi);
        const FI I = make_fi(P, A, i, f);
        // the forward pass's own sums (taped when the step was recomputed)
        const int tn = A.sums_n;
        const float4 s0 = A.sums[i], s1 = A.sums[tn + i];
        const V3 force = xyz(s0), sumT = xyz(s1);
        const float q = s0.w, num = s1.w, den = A.sums[2 * tn + i].x;
        const float4 ga = A.gA[i], gb = A.gB[i];
        const V3 ab = xyz(ga);
        const V3 abb = xyz(gb);
        float mb = -dot(ab, force) / (f.m * f.m);
        float Tb = 0.0f, rhob = 0.0f, VTb = 0.0f, cb = 0.0f;
        float4 gg = A.gG[i];
        float numb = 0.0f, denb = 0.0f, qb = 0.0f;
        V3 sTb{0, 0, 0};
        if (I.do_C) {
          const float kappa = den > 0.0f ? 3.0f * num / den : 0.0f;
          const V3 nrm = xyz(V.nrm[i]);
          gg.x += ab.x * csf_coeff * kappa;
          gg.y += ab.y * csf_coeff * kappa;
          gg.z += ab.z * csf_coeff * kappa;
          const float an = dot(ab, nrm);
          s[4] = (double)an * kappa * csf_unit;
          if (den > 0.0f) {
            const float kb = an * csf_coeff;
            numb = 3.0f * kb / den;
            denb = -3.0f * kb * num / (den * den);
          }
        }
        if (thermal) {
          const float cpi = P.cp[phase_index(ph)];
          const float hw = V.heat_w[i];
          const float qt = q + P.heat_power * hw * hinv;
          qb = ga.w / (f.m * cpi);
          mb += -ga.w * (qt / (f.m * cpi)) / f.m;
          gg.w += qb * P.heat_power * hinv;
          s[0] = (double)qb * P.heat_power * hw;
          s[5] = (double)qb * hw * hinv;
        }
        if (I.do_T) {
          sTb = abb * (-I.pb / I.mT);
          const float coefb = dot(abb, sumT);
          const float pbb = -coefb / I.mT;
          const float mTb = coefb * I.pb / (I.mT * I.mT);
          cb += pbb * 2.0f * P.tvf_factor * P.rho0[phase_index(ph)] * f.c;
          rhob += mTb * f.VT;
          VTb += mTb * f.rho;
        }
        s[1] = ab.x;
        s[2] = ab.y;
        s[3] = ab.z;
        V3 xb{0, 0, 0}, vb{0, 0, 0};
        if (d1->fr.frame_rot) {
          const V3 om = v3(d1->fr.omega[0], d1->fr.omega[1], d1->fr.omega[2]);
          const V3 omd = v3(d1->fr.omega_dot[0], d1->fr.omega_dot[1], d1->fr.omega_dot[2]);
          xb -= cross(ab, omd) + cross(cross(ab, om), om);
          vb -= cross(ab, om) * 2.0f;
        }
        if (ph == kVapor && f.T > 0.0f) Tb += cb * P.gas_R / (2.0f * f.c);
        A.gU1[i] = f4(ab, qb);
        A.gU2[i] = f4(sTb, numb);
        A.gU3[i] = make_float4(denb, 0.0f, 0.0f, 0.0f);
        const int bits = (I.do_T ? 1 : 0) | (I.do_C ? 2 : 0) | (norm2(f.ns) > 0.25f ? 4 : 0);
        A.R1[i] = make_float4(f.V, f.VT, f.c, f.rho);
        A.R2[i] = make_float4(f.p, f.T, f.m, __int_as_float(bits));
        A.gG[i] = gg;
        add4(A.gX + i, xb, mb);
        add4(A.gV + i, vb, Tb);
        float4 gbw = A.gB[i];
        gbw.w += rhob;
        A.gB[i] = gbw;
        float4 gp = A.gP[i];
        gp.y += -VTb * f.VT * f.VT;
        A.gP[i] = gp;
      } else {
        A.gU1[i] = zero4();
        A.gU2[i] = zero4();
        A.gU3[i] = zero4();
      }
    }
    publish_chunk<6>(R, c, s, sh);
  }
}

// Every force pair from both ends.  Fluid k: its own pairs (adjoints on k as
// i) and its fluid neighbours' pairs with k (k as j).  Wall k: its fluid
// neighbours' pairs with k (wall pressures and ghost velocity).
#ifndef ADJ_FORCES_MIN_BLOCKS
#define ADJ_FORCES_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(128, ADJ_FORCES_MIN_BLOCKS) k_adj_forces_gather(Params P, Adj A) {
  const View& V = A.V;
  const DynState* d1 = A.dyn1;
  const int n = V.dyn->n;
  const float dt = d1->dt;
  const bool thermal = P.thermal && d1->thermal_on;
  const V3 origin = v3(d1->fr.frame_origin[0], d1->fr.frame_origin[1], d1->fr.frame_origin[2]);
  // objective: sum over steps of dt (-sum fw) . seed_F + dt (-sum mw) . seed_M
  const float sdt = -dt;
  const V3 fwb = v3((float)A.glob[AG_FW], (float)A.glob[AG_FW + 1], (float)A.glob[AG_FW + 2]) * sdt;
  const V3 mwb = v3((float)A.glob[AG_MW], (float)A.glob[AG_MW + 1], (float)A.glob[AG_MW + 2]) * sdt;
  // harmonic viscosity and conductivity per phase pair (symmetric: index
  // = phase_k + phase_l), as navier_stokes.cu:190-196 and phase_change.cu:57-61
  float etp[3], kp[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int pa = q > 1 ? 1 : 0, pb = q > 0 ? 1 : 0;
    const float es = P.mu[pa] + P.mu[pb];
    etp[q] = es > 0.0f ? 2.0f * P.mu[pa] * P.mu[pb] / es : 0.0f;
    kp[q] = 4.0f * P.k[pa] * P.k[pb] / (P.k[pa] + P.k[pb]);
  }
  const PhaseOrder ord = phase_order(P, V, true);
  PARTICLE_LOOP(t, ord.total) {
    const int k = order_at(ord, t);
    const float4 xpk = V.xp[k];
    const int phk = ph_of(xpk);
    if (phk == kWall) {
      const FP W = load_wall(A, k, xpk);
      const V3 dFb = fwb + cross(mwb, W.x - origin);
      FA o{};
      for_each_nbr(P, V, k, W.x, [&](int l, float4 xl, V3 rkl, float r2) {
        if (!is_fluid(ph_of(xl))) return;
        const FR fl = load_rec(A, l, xl);
        const FI I = fi_of(P, fl);
        const FU U = load_fu(A, l, fl.f.m);
        forces_pair_adj<false>(P, I, U, W, -rkl, r2, dt, thermal, dFb, o);
      });
      float4 gp = A.gP[k];
      gp.x += o.p;
      gp.y += o.p_wv;
      A.gP[k] = gp;
      add4(A.gN + k, o.v, 0.0f);
      continue;
    }
    if (!is_fluid(phk)) continue;
    const FR rk = load_rec(A, k, xpk);
    const FI Ik = fi_of(P, rk);
    const FU Uk = load_fu(A, k, rk.f.m);
    const int pk = phase_index(phk);
    FA o{};
    for_each_nbr(P, V, k, rk.f.x, [&](int l, float4 xl, V3 rkl, float r2) {
      if (l == k) return;
      const int phl = ph_of(xl);
      if (phl == kWall) {
        const FP W = load_wall(A, l, xl);
        const V3 dFb = fwb + cross(mwb, W.x - origin);
        forces_pair_adj<true>(P, Ik, Uk, W, rkl, r2, dt, thermal, dFb, o);
        return;
      }
      if (!is_fluid(phl)) return;
      const FR rl = load_rec(A, l, xl);
      const FU Ul = load_fu(A, l, rl.f.m);
      const int q = pk + phase_index(phl);
      const float eta = q == 0 ? etp[0] : (q == 1 ? etp[1] : etp[2]);
      const float kc = q == 0 ? kp[0] : (q == 1 ? kp[1] : kp[2]);
      fluid_pair_both(P, rk, Uk, rl, Ul, rkl, r2, thermal, eta, kc, Ik.av, o);
    });
    // V = m / rho, VT = 1 / sigma, c(T)
    const FP& fk = rk.f;
    o.m += o.V / fk.rho;
    o.rho += -o.V * fk.V / fk.rho;
    float Tb = o.T;
    if (phk == kVapor && fk.T > 0.0f) Tb += o.c * P.gas_R / (2.0f * fk.c);
    add4(A.gX + k, o.x, o.m);
    add4(A.gV + k, o.v, Tb);
    float4 gb = A.gB[k];
    gb.w += o.rho;
    A.gB[k] = gb;
    float4 gp = A.gP[k];
    gp.x += o.p;
    gp.y += -o.VT * fk.VT * fk.VT;
    A.gP[k] = gp;
    add4(A.gN + k, o.ns, 0.0f);
  }
}

// --------------------------------------------------------- interface
// Per fluid particle: the sums of compute_interface_fields recomputed, then
// the adjoints of the unit normal, the contact-angle rotation and the colour
// fraction; stores the upstream coefficients of its pair sums.
__global__ void __launch_bounds__(kBlock) k_adj_interface_local(Params P, Adj A) {
  __shared__ double sh[2 * kBlock / 32];
  const View& V = A.V;
  const DynState* d1 = A.dyn1;
  const int n = V.dyn->n;
  const int nch = num_chunks(n);
  const bool write_ns = P.csf_active && !P.csf_smooth;
  const float hinv = d1->heat_inv_norm;
  const float hinvb = (float)A.glob[AG_HINV];
  const Reduce R = rows(A, AR_IFACE);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double s[2] = {0.0, 0.0};
    if (i < n) {
      const float4 xpi = V.xp[i];
      const int ph = ph_of(xpi);
      if (is_fluid(ph)) {
        // the forward pass's sums before the rotation (taped when the step was recomputed)
        const int tn = A.sums_n;
        const float4 t3 = A.sums[3 * tn + i], t4 = A.sums[4 * tn + i];
        const V3 gradc = xyz(t3), wall_n = xyz(t4);
        const float s_all = t3.w, s_other = t4.w, ww = A.sums[5 * tn + i].x;
        const float alpha = s_all > 0.0f ? s_other / s_all : 0.0f;
        const float4 gn = A.gN[i], gg = A.gG[i];
        // colour gradient after the rotation: nrm (forces) and ns (CSF)
        V3 gpb = xyz(gg);
        if (write_ns) {
          const V3 gp = xyz(V.nrm[i]);
          const float gm = norm(gp);
          if (gm > P.normal_eps) {
            const V3 ns = gp / gm;
            const V3 nsb = xyz(gn);
            gpb += (nsb - ns * dot(nsb, ns)) / gm;
          }
        }
        Rot rot{false, gradc, wall_n, ww};
        const float gmag = norm(gradc);
        if (P.wetting_model != 1 && ww > 0.0f && gmag > P.normal_eps) {
          const V3 nw = normalized(wall_n);
          const V3 nh = gradc / gmag;
          const V3 t = nh - nw * dot(nh, nw);
          rot.on = norm2(nw) > 0.0f && norm(t) > 1e-6f;
        }
        V3 gb, wnb;
        float wwb, cosb = 0.0f, sinb = 0.0f;
        rotation_adjoint(P, rot, gpb, gb, wnb, wwb, cosb, sinb);
        s[0] = cosb;
        s[1] = sinb;
        const float alb = gn.w;
        float s_allb = 0.0f, s_otherb = 0.0f;
        if (s_all > 0.0f) {
          s_otherb = alb / s_all;
          s_allb = -alb * alpha / s_all;
        }
        float hwb = gg.w;
        if (hinv > 0.0f) hwb += -hinvb * hinv * hinv;
        A.gU1[i] = f4(gb, s_allb);
        A.gU2[i] = f4(wnb, s_otherb);
        A.gU3[i] = make_float4(wwb, hwb, 0.0f, 0.0f);
      }
    }
    publish_chunk<2>(R, c, s, sh);
  }
}

// The pair sums of compute_interface_fields from both ends: positions and
// volumes of fluid particles, colour fractions of walls.
__global__ void __launch_bounds__(kBlock) k_adj_interface_gather(Params P, Adj A) {
  const View& V = A.V;
  const int n = V.dyn->n;
  const float w0 = kernel_W(P, 0.0f);
  const PhaseOrder ord = phase_order(P, V, true);
  PARTICLE_LOOP(t, ord.total) {
    const int k = order_at(ord, t);
    const float4 xpk = V.xp[k];
    const int phk = ph_of(xpk);
    const V3 xk = xyz(xpk);
    if (phk == kWall) {
      if (!P.wall_colour) continue;
      float ab = 0.0f;
      for_each_nbr(P, V, k, xk, [&](int l, float4 xl, V3 rkl, float r2) {
        if (!is_fluid(ph_of(xl))) return;
        const float r = sqrtf(r2);
        const V3 gw = kernel_gradW(P, -rkl, r);
        ab += dot(xyz(__ldg(A.gU1 + l)), gw) * P.vol0;
      });
      float4 gp = A.gP[k];
      gp.z += ab;
      A.gP[k] = gp;
      continue;
    }
    if (!is_fluid(phk)) continue;
    const float ck = phk == kLiquid ? 1.0f : 0.0f;
    const float4 u1 = A.gU1[k], u2 = A.gU2[k], u3 = A.gU3[k];
    const V3 gbk = xyz(u1), wnbk = xyz(u2);
    const float mk = A.m1[k], rk = V.mrps[k].y;
    const float Vk = mk / rk;
    float Vb = u1.w * w0;  // self term of s_all
    V3 xb{0, 0, 0};
    for_each_nbr(P, V, k, xk, [&](int l, float4 xl, V3 rkl, float r2) {
      if (l == k) return;
      const float r = sqrtf(r2);
      float F, dF;
      kernel_F(P, r, F, dF);
      const int phl = ph_of(xl);
      if (phl == kWall) {
        const float4 nl = __ldg(V.nrm + l);
        const float sw = u3.x + ((fl_of(xl) & kHeated) ? u3.y : 0.0f) + dot(wnbk, xyz(nl));
        xb += rkl * (sw * P.vol0 * F);
        if (P.wall_colour) xb += gradW_vjp(rkl, r, F, dF, gbk * (P.vol0 * (nl.w - ck)));
        return;
      }
      if (!is_fluid(phl)) return;
      const float w = kernel_W(P, r);
      const float Vl = __ldg(A.m1 + l) / __ldg(V.mrps + l).y;
      const float cl = phl == kLiquid ? 1.0f : 0.0f;
      // k's sums over l (s_all, s_other: V_l W; gradc: gw V_l (c_l - c_k)) and
      // l's sums over k (V_k W; -gw V_k (c_k - c_l)), sharing one evaluation
      const float sk = u1.w + (phl != phk ? u2.w : 0.0f);
      const float4 l1 = __ldg(A.gU1 + l);
      const float sl = l1.w + (phl != phk ? __ldg(A.gU2 + l).w : 0.0f);
      xb += rkl * ((sk * Vl + sl * Vk) * F);
      Vb += sl * w;
      if (cl != ck) {
        const V3 gl = xyz(l1);
        Vb += dot(gl, rkl) * (F * (cl - ck));  // grad W of (l, k) is -rkl F
        xb += gradW_vjp(rkl, r, F, dF, (gbk * Vl + gl * Vk) * (cl - ck));
      }
    });
    add4(A.gX + k, xb, Vb / rk);
    float4 gb = A.gB[k];
    gb.w -= Vb * Vk / rk;
    A.gB[k] = gb;
  }
}

// -------------------------------------------------------------- walls
// Per wall particle: compute_wall_boundary's sums recomputed, then the
// adjoints of those sums from the adjoints of p_wl, p_wv, alpha_w and vw.
__global__ void __launch_bounds__(kBlock) k_adj_wall_local(Params P, Adj A) {
  const View& V = A.V;
  const int n = V.dyn->n;
  const DynState* d1 = A.dyn1;
  const V3 g = v3(d1->fr.gravity[0], d1->fr.gravity[1], d1->fr.gravity[2]);
  PARTICLE_LOOP(i, n) {
    const float4 xpi = V.xp[i];
    if (ph_of(xpi) != kWall) continue;
    const V3 xi = xyz(xpi);
    float sw[2] = {0, 0}, sp[2] = {0, 0}, sgr[2] = {0, 0};
    V3 sv{0, 0, 0};
    for_each_nbr(P, V, i, xi, [&](int j, float4 xj, V3 rwf, float r2) {
      const int phj = ph_of(xj);
      if (!is_fluid(phj)) return;
      const float w = kernel_W(P, sqrtf(r2));
      const float4 mr = __ldg(V.mrps + j);
      const int k = phase_index(phj);
      sw[k] += w;
      sp[k] += mr.z * w;
      sgr[k] += dot(g, rwf) * mr.y * w;
      sv += xyz(__ldg(A.vT1 + j)) * w;
    });
    const float4 gp = A.gP[i];
    const V3 vwb = xyz(A.gN[i]);
    float Pb[2] = {0.0f, 0.0f};
    const bool h0 = sw[0] > 0.0f, h1 = sw[1] > 0.0f;
    if (h0 && h1) {
      Pb[0] = gp.x;
      Pb[1] = gp.y;
    } else if (h1) {
      Pb[1] = gp.x + gp.y;
    } else if (h0) {
      Pb[0] = gp.x + gp.y;
    }
    float swb[2] = {0, 0}, spb[2] = {0, 0}, sgb[2] = {0, 0};
    for (int k = 0; k < 2; ++k) {
      if (!(sw[k] > 0.0f)) continue;
      const float pw = (sp[k] + sgr[k]) / sw[k];
      spb[k] = Pb[k] / sw[k];
      sgb[k] = Pb[k] / sw[k];
      swb[k] = -Pb[k] * pw / sw[k];
    }
    const float swt = sw[0] + sw[1];
    V3 svb{0, 0, 0};
    if (swt > 0.0f) {
      const float ab = gp.z;
      swb[0] += ab * sw[1] / (swt * swt);
      swb[1] -= ab * sw[0] / (swt * swt);
      svb = vwb * (-1.0f / swt);
      const float swtb = dot(vwb, sv) / (swt * swt);
      swb[0] += swtb;
      swb[1] += swtb;
    }
    A.gU1[i] = make_float4(swb[0], swb[1], spb[0], spb[1]);
    A.gU2[i] = make_float4(sgb[0], sgb[1], 0.0f, 0.0f);
    A.gU3[i] = f4(svb, 0.0f);
  }
}

// Per fluid particle: its terms in the wall sums of its wall neighbours, then
// (every adjoint of its density, pressure and sigma now complete) the
// equation of state and rho = m sigma.
__global__ void __launch_bounds__(kBlock) k_adj_wall_gather(Params P, Adj A) {
  __shared__ double sh[3 * kBlock / 32];
  const View& V = A.V;
  const DynState* d1 = A.dyn1;
  const int n = V.dyn->n;
  const int nch = num_chunks(n);
  const V3 g = v3(d1->fr.gravity[0], d1->fr.gravity[1], d1->fr.gravity[2]);
  const Reduce R = rows(A, AR_WALL);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int k = c * kChunk + threadIdx.x;
    double s[3] = {0.0, 0.0, 0.0};
    if (k < n) {
      const float4 xpk = V.xp[k];
      const int ph = ph_of(xpk);
      if (is_fluid(ph)) {
        const int q = phase_index(ph);
        const float4 mr = V.mrps[k];
        const float4 vT = A.vT1[k];
        const V3 vk = xyz(vT);
        float pb = 0.0f, rhob = 0.0f;
        V3 xb{0, 0, 0}, vb{0, 0, 0}, gsum{0, 0, 0};
        for_each_nbr(P, V, k, xyz(xpk), [&](int l, float4 xl, V3 rkl, float r2) {
          if (ph_of(xl) != kWall) return;
          const float r = sqrtf(r2);
          const float w = kernel_W(P, r);
          float F, dF;
          kernel_F(P, r, F, dF);
          const float4 u1 = __ldg(A.gU1 + l), u2 = __ldg(A.gU2 + l), u3 = __ldg(A.gU3 + l);
          const float swb = q ? u1.y : u1.x, spb = q ? u1.w : u1.z, sgb = q ? u2.y : u2.x;
          const V3 rv = -rkl;  // wall - fluid
          const float grv = dot(g, rv);
          const float wb = swb + spb * mr.z + sgb * grv * mr.y + dot(xyz(u3), vk);
          pb += spb * w;
          rhob += sgb * grv * w;
          vb += xyz(u3) * w;
          xb += rkl * (wb * F) - g * (sgb * mr.y * w);
          gsum += rv * (sgb * mr.y * w);
        });
        s[0] = gsum.x;
        s[1] = gsum.y;
        s[2] = gsum.z;
        // EOS and rho = (m0 | m) sigma
        float4 gp = A.gP[k], gb = A.gB[k];
        float T = vT.w;
        float p_b = gp.x + pb;
        float rho_b = gb.w + rhob;
        float Tb = 0.0f, mb = 0.0f;
        if (ph == kVapor) {
          rho_b += p_b * P.gas_R * T;
          Tb += p_b * mr.y * P.gas_R;
        } else {
          const float ratio = mr.y / P.rho0[0];
          float dr;
          if (P.tait_gamma == 7.0f) {
            const float r2v = ratio * ratio;
            dr = 7.0f * r2v * r2v * r2v;
          } else {
            dr = P.tait_gamma * powf(ratio, P.tait_gamma - 1.0f);
          }
          rho_b += p_b * P.tait_B * dr / P.rho0[0];
        }
        float sig_b = gp.y;
        if (P.density_mode == CRYO_DENSITY_SUMMATION) {
          const float M = ph == kLiquid ? V.vt[k].w : A.m1[k];
          sig_b += rho_b * M;
          if (ph == kVapor) mb += rho_b * mr.w;
        }
        gp.x = p_b;
        gp.y = sig_b;
        gb.w = rho_b;
        A.gP[k] = gp;
        A.gB[k] = gb;
        add4(A.gX + k, xb, mb);
        add4(A.gV + k, vb, Tb);
      }
    }
    publish_chunk<3>(R, c, s, sh);
  }
}

// compute_density_summation (SPH_kernels.cu:6-34): sigma_i = sum_j W(r_ij),
// from both ends.
__global__ void __launch_bounds__(kBlock) k_adj_density_gather(Params P, Adj A) {
  const View& V = A.V;
  const int n = V.dyn->n;
  const PhaseOrder ord = phase_order(P, V, false);
  PARTICLE_LOOP(t, ord.total) {
    const int k = order_at(ord, t);
    const float4 xpk = V.xp[k];
    if (!is_fluid(ph_of(xpk))) continue;
    const float sk = A.gP[k].y;
    V3 xb{0, 0, 0};
    for_each_nbr(P, V, k, xyz(xpk), [&](int l, float4 xl, V3 rkl, float r2) {
      if (l == k) return;
      const float r = sqrtf(r2);
      float F, dF;
      kernel_F(P, r, F, dF);
      const float sl = is_fluid(ph_of(xl)) ? __ldg(A.gP + l).y : 0.0f;
      xb += rkl * ((sk + sl) * F);
    });
    add4(A.gX + k, xb, 0.0f);
  }
}

// kick_drift (sph_solver.cu:20-34) and the reorder gather
// (spatial_hash.cu:116-138): the adjoints of the previous step's end state,
// scattered to its sorted order.
__global__ void __launch_bounds__(kBlock) k_adj_drift_scatter(Params P, Adj A) {
  const View& V = A.V;
  const int n = V.dyn->n;
  const float dt = A.dyn1->dt, half = 0.5f * dt;
  PARTICLE_LOOP(i, n) {
    const uint32_t j = A.perm[i];
    if (!is_fluid(ph_of(V.xp[i]))) {
      A.prevX[j] = zero4();
      A.prevV[j] = zero4();
      A.prevA[j] = zero4();
      A.prevB[j] = zero4();
      continue;
    }
    const float4 gx = A.gX[i], gv = A.gV[i];
    const V3 vtb = xyz(gx) * dt;
    const V3 v1b = xyz(gv) + vtb;
    A.prevX[j] = gx;
    A.prevV[j] = f4(v1b, gv.w);
    A.prevA[j] = f4(v1b * half, 0.0f);
    A.prevB[j] = f4(P.tvf ? vtb * half : V3{0, 0, 0}, 0.0f);
  }
}

__global__ void __launch_bounds__(kBlock) k_adj_reduce(Adj A, AdjRows M) {
  // one block per row; the rows write distinct accumulators
  const int b = blockIdx.x;
  if (b >= M.count) return;
  const int nch = num_chunks(A.V.dyn->n);
  const double s = block_sum_partials(rows(A, M.row[b]), 0, nch);
  if (threadIdx.x == 0) A.glob[M.dst[b]] = M.accumulate[b] ? A.glob[M.dst[b]] + s : s;
}

__global__ void __launch_bounds__(kBlock) k_adj_objective(Params P, View V, Reduce R, double* obj) {
  __shared__ double sh[6 * kBlock / 32];
  const DynState* d = V.dyn;
  const int n = d->n;
  const int nch = num_chunks(n);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double s[6] = {0, 0, 0, 0, 0, 0};
    if (i < n && is_fluid(ph_of(V.xp[i]))) {
      const float4 fw = V.fw[i], mw = V.mw[i];
      s[0] = fw.x; s[1] = fw.y; s[2] = fw.z;
      s[3] = mw.x; s[4] = mw.y; s[5] = mw.z;
    }
    publish_chunk<6>(R, c, s, sh);
  }
  if (!last_block(R.ticket)) return;
  const double dt = d->dt;
  for (int k = 0; k < 6; ++k) {
    const double s = block_sum_partials(R, k, nch);
    if (threadIdx.x == 0) obj[k] += dt * (-s);
  }
}

__global__ void __launch_bounds__(kBlock) k_adj_snap_end(View V, const uint32_t* __restrict__ perm, AdjSlot S) {
  const int n = V.dyn->n;
  PARTICLE_LOOP(i, n) {
    S.xp[i] = V.xp[i];
    S.vT[i] = V.vT[i];
    S.vt[i] = V.vt[i];
    S.nrm[i] = V.nrm[i];
    S.mrps[i] = V.mrps[i];
    S.a4[i] = V.a4[i];
    S.vwp[i] = V.vwp[i];
    S.heat_w[i] = V.heat_w[i];
    S.perm[i] = perm[i];
    S.nbr_cnt[i] = V.nbr_cnt[i];
    if (V.fluid_idx) {  // valid up to the list lengths, which together are n
      S.fluid_idx[i] = V.fluid_idx[i];
      S.wall_idx[i] = V.wall_idx[i];
    }
  }
}

__global__ void k_adj_step_end(double* glob, double* grav_out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int k = 0; k < 3; ++k) grav_out[k] = glob[AG_GRAV + k];
  glob[AG_TSAT_OUT] = glob[AG_TSAT_IN];
  glob[AG_P_OBJ] = 0.0;
}

__global__ void __launch_bounds__(kBlock) k_adj_copy4(const float4* src, float4* dst, float* mdst, const float4* msrc,
                                                      const DynState* dyn) {
  const int n = dyn->n;
  PARTICLE_LOOP(i, n) {
    if (dst) dst[i] = src[i];
    if (mdst) mdst[i] = msrc[i].x;
  }
}

}  // namespace cryo
