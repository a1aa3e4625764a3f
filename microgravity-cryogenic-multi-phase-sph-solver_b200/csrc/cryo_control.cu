// cryo_control.cu -- device-resident step control: the adaptive time step,
// the manoeuvre frame, the lumped ullage model and the FP64 diagnostics.
// These replace host code of the reference (sph_solver.cu:244-268,482-504,
// 586-653) so that a whole step runs without a host round trip.
#include "cryo_kernels.cuh"

namespace cryo {

// ManeuverProfile::evaluate (sph_solver.cu:244-268)
__device__ void maneuver_evaluate(const View& V, int n, int rot, double t, V3& a, V3& w, V3& wd) {
  const double* tt = V.man_t;
  const float* acc = V.man_acc;
  const float* om = V.man_omega;
  auto A = [&](int k) { return v3(acc[3 * k], acc[3 * k + 1], acc[3 * k + 2]); };
  auto W = [&](int k) { return v3(om[3 * k], om[3 * k + 1], om[3 * k + 2]); };
  wd = V3{0, 0, 0};
  if (t <= tt[0] || n == 1) {
    a = A(0);
    w = rot ? W(0) : V3{0, 0, 0};
    return;
  }
  if (t >= tt[n - 1]) {
    a = A(n - 1);
    w = rot ? W(n - 1) : V3{0, 0, 0};
    return;
  }
  int lo = 0, hi = n;  // upper_bound
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (t < tt[mid]) hi = mid;
    else lo = mid + 1;
  }
  const int k = lo - 1;
  const double dt = tt[k + 1] - tt[k];
  const float f = (float)((t - tt[k]) / dt);
  a = A(k) * (1.0f - f) + A(k + 1) * f;
  if (rot) {
    w = W(k) * (1.0f - f) + W(k + 1) * f;
    wd = (W(k + 1) - W(k)) / (float)dt;
  } else {
    w = V3{0, 0, 0};
  }
}

// Solver::apply_frame (sph_solver.cu:660-667)
__device__ void apply_frame(DynState* d, V3 a, V3 w, V3 wd, const float* origin) {
  d->fr.frame_acc[0] = a.x; d->fr.frame_acc[1] = a.y; d->fr.frame_acc[2] = a.z;
  d->fr.gravity[0] = d->fr.cfg_gravity[0] - a.x;
  d->fr.gravity[1] = d->fr.cfg_gravity[1] - a.y;
  d->fr.gravity[2] = d->fr.cfg_gravity[2] - a.z;
  d->fr.omega[0] = w.x; d->fr.omega[1] = w.y; d->fr.omega[2] = w.z;
  d->fr.omega_dot[0] = wd.x; d->fr.omega_dot[1] = wd.y; d->fr.omega_dot[2] = wd.z;
  d->fr.frame_origin[0] = origin[0]; d->fr.frame_origin[1] = origin[1]; d->fr.frame_origin[2] = origin[2];
  d->fr.frame_rot = (norm2(w) > 0.0f || norm2(wd) > 0.0f) ? 1 : 0;
}

// Start of Solver::step (sph_solver.cu:513-522): the step size from the maxima
// of the previous rate evaluation, the frame at the new time level, and the
// maxima reset for this step's evaluation (BEGIN_STEP).  BEGIN_RATES only
// resets the maxima (a rate evaluation outside a step).
__global__ void k_begin_step(Params P, View V, int mode) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  DynState* d = V.dyn;
  if (mode == BEGIN_STEP) {
    const float dt = compute_dt(P, *d);
    d->dt = dt;
    if (d->fr.has_maneuver) {
      V3 a, w, wd;
      maneuver_evaluate(V, d->man_n, d->man_rot, d->time + (double)dt, a, w, wd);
      apply_frame(d, a, w, wd, d->man_origin);
    }
  }
  d->v_max = 0.0f;
  d->a_max = 0.0f;
  d->Tv_max = 0.0f;
  d->nu_t_max = 0.0f;
  d->spacing_ratio = 1.0f;
}

// The start of Solver::step fused with its kick_drift and hash keys (the
// step path, one launch instead of two): every block derives the step size
// itself from the previous evaluation's maxima -- compute_dt over the same
// scalars, so every block gets the same dt bit for bit -- and block 0 stores
// it and moves the manoeuvre frame to the new time level.  The maxima are
// reset later in the step (k_gather with reset_maxima), once no block of this
// kernel can still read them; the frame is not read here.
__global__ void __launch_bounds__(kBlock) k_begin_kick_drift_keys(Params P, View V, uint32_t* __restrict__ keys) {
  __shared__ float sdt;
  DynState* d = V.dyn;
  if (threadIdx.x == 0) {
    const float dt = compute_dt(P, *d);
    sdt = dt;
    if (blockIdx.x == 0) {
      d->dt = dt;
      if (d->fr.has_maneuver) {
        V3 a, w, wd;
        maneuver_evaluate(V, d->man_n, d->man_rot, d->time + (double)dt, a, w, wd);
        apply_frame(d, a, w, wd, d->man_origin);
      }
    }
  }
  __syncthreads();
  const float dt = sdt;
  const int n = d->n;
  const int continuity = P.density_mode == CRYO_DENSITY_CONTINUITY;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 xp = V.xp[i];
    const int ph = ph_of(xp);
    if (is_fluid(ph)) kick_drift_one(P, V, i, dt, continuity, P.tvf, xp);
    keys[i] = ph == kDead ? (uint32_t)P.num_cells : (uint32_t)cell_index(P, xyz(xp));
  }
}

// Solver::update_saturation (sph_solver.cu:586-607) with the phase inventory
// (sph_solver.cu:137-145) as one FP64 reduction; with end_of_step the clock
// advances (sph_solver.cu:530-532) and the relax damping is applied
// (scale_velocities, sph_solver.cu:716-717).
__global__ void __launch_bounds__(kBlock) k_saturation(Params P, View V, Reduce R, int end_of_step) {
  __shared__ double sh[3 * kBlock / 32];
  DynState* d = V.dyn;
  const int n = d->n;
  const int nch = num_chunks(n);
  const bool closed = P.thermo_closed && P.has_vapor;
  const bool damp = end_of_step && d->damp_after_step;
  const float damping = d->damping;
  const int own_lo = d->own_lo, own_hi = d->own_hi, n_sorted = d->n_sorted;
  if (closed || damp) {
    for (int c = blockIdx.x; c < nch; c += gridDim.x) {
      const int i = c * kChunk + threadIdx.x;
      double s[3] = {0.0, 0.0, 0.0};
      if (i < n) {
        const int ph = ph_of(V.xp[i]);
        const float4 vT = V.vT[i];
        if (closed && owned(own_lo, own_hi, n_sorted, i)) {
          const double m = V.mrps[i].x;
          if (ph == kLiquid) s[0] = m;
          if (ph == kVapor) {
            s[1] = m;
            s[2] = m * vT.w;
          }
        }
        if (damp && is_fluid(ph)) {
          V.vT[i] = f4(xyz(vT) * damping, vT.w);
          const float4 vt = V.vt[i];
          V.vt[i] = f4(xyz(vt) * damping, vt.w);
        }
      }
      if (closed) publish_chunk<3>(R, c, s, sh);
    }
  }
  const bool last = closed ? last_block(R.ticket) : (blockIdx.x == 0);
  if (!last) return;
  double m_liq = 0, m_vap = 0, mT_vap = 0;
  if (closed) {
    m_liq = block_sum_partials(R, 0, nch);
    m_vap = block_sum_partials(R, 1, nch);
    mT_vap = block_sum_partials(R, 2, nch);
  }
  if (threadIdx.x != 0) return;
  d->sat_sum[0] = m_liq;
  d->sat_sum[1] = m_vap;
  d->sat_sum[2] = mT_vap;
  if (!P.slab) saturation_update(P, d, closed, m_liq, m_vap, mT_vap);
  if (end_of_step) {
    d->time += (double)d->dt;
    d->step += 1;
    d->last_dt = (double)d->dt;
  }
}

// The closing kick (sph_solver.cu:36-46, k_kick without phase-change
// sources) fused with k_saturation's end of step, for steps where nothing runs
// between them (no particle shifting, no phase change, one context per
// tank): each thread kicks its particle and then adds it to the ullage sums
// and damps it, in the chunk order k_saturation uses, so the sums and the
// state equal the two launches' bit for bit.
__global__ void __launch_bounds__(kBlock) k_kick_saturation(Params P, View V, Reduce R) {
  __shared__ double sh[3 * kBlock / 32];
  DynState* d = V.dyn;
  const int n = d->n;
  const int nch = num_chunks(n);
  const float dt = d->dt;
  const float half = 0.5f * dt;
  const int thermal = d->thermal_on;
  const bool closed = P.thermo_closed && P.has_vapor;
  const bool damp = d->damp_after_step;
  const float damping = d->damping;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double s[3] = {0.0, 0.0, 0.0};
    if (i < n) {
      const int ph = ph_of(V.xp[i]);
      if (is_fluid(ph)) {
        float4 vT = V.vT[i];
        const float4 a4 = V.a4[i];
        V3 v = xyz(vT) + xyz(a4) * half;
        float T = vT.w;
        if (thermal) T += a4.w * dt;
        if (closed) {
          const double m = V.mrps[i].x;
          if (ph == kLiquid) s[0] = m;
          if (ph == kVapor) {
            s[1] = m;
            s[2] = m * T;
          }
        }
        if (damp) {
          v = v * damping;
          const float4 vt = V.vt[i];
          V.vt[i] = f4(xyz(vt) * damping, vt.w);
        }
        V.vT[i] = f4(v, T);
      }
    }
    if (closed) publish_chunk<3>(R, c, s, sh);
  }
  const bool last = closed ? last_block(R.ticket) : (blockIdx.x == 0);
  if (!last) return;
  double m_liq = 0, m_vap = 0, mT_vap = 0;
  if (closed) {
    m_liq = block_sum_partials(R, 0, nch);
    m_vap = block_sum_partials(R, 1, nch);
    mT_vap = block_sum_partials(R, 2, nch);
  }
  if (threadIdx.x != 0) return;
  if (thermal && d->heat_inv_norm > 0.0f) d->heat_input += (double)P.heat_power * (double)dt;
  d->sat_sum[0] = m_liq;
  d->sat_sum[1] = m_vap;
  d->sat_sum[2] = mT_vap;
  saturation_update(P, d, closed, m_liq, m_vap, mT_vap);
  d->time += (double)d->dt;
  d->step += 1;
  d->last_dt = (double)d->dt;
}

// Heat-weight normalisation on its own (sph_solver.cu:466-472), for
// operator-level calls.
__global__ void __launch_bounds__(kBlock) k_heat_norm(Params P, View V, Reduce R) {
  __shared__ double sh[kBlock / 32];
  DynState* d = V.dyn;
  const int n = d->n;
  const int nch = num_chunks(n);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double s[1] = {0.0};
    if (i < n && is_fluid(ph_of(V.xp[i]))) s[0] = (double)V.heat_w[i];
    publish_chunk<1>(R, c, s, sh);
  }
  if (last_block(R.ticket)) {
    const double S = block_sum_partials(R, 0, nch);
    if (threadIdx.x != 0) return;
    if (P.heat_power != 0.0f) {
      d->heat_inv_norm = S > 0 ? (float)(1.0 / S) : 0.0f;
    } else {
      d->heat_inv_norm = 0.0f;
    }
  }
}

// Solver::diagnostics (sph_solver.cu:609-653): every phase sum, count and
// maximum in one FP64 pass.  out[] layout:
//   0-2 counts L/V/W, 3-4 mass L/V, 5-6 KE L/V, 7-8 enthalpy L/V, 9-10 mT L/V,
//   11-13 m x (L), 14-16 m v (L), 17-19 sum fw (fluid), 20-22 sum mw (fluid),
//   23 max fluid speed, 24 max liquid T, 25-43 the scalar state (clock,
//   counters, ullage, frame)
// Two resident blocks per SM (at most 128 registers): a thread holds its four
// particles' records at once, and the 199 chunk blocks of a 200k-particle
// tank still run in one wave over the 148 SMs.
__global__ void __launch_bounds__(kBlock, 2) k_diagnostics(Params P, View V, Reduce R, double* __restrict__ out) {
  __shared__ double sh[23 * kBlock / 32];
  __shared__ float shmax[2][kBlock / 32];
  DynState* d = V.dyn;
  const int n = d->n;
  // chunks of kDiagPer * kChunk particles: each thread adds its kDiagPer
  // particles first, so a block reduction covers four times the particles
  constexpr int kDiagPer = 4;
  const int nch = (n + kDiagPer * kChunk - 1) / (kDiagPer * kChunk);
  const int own_lo = d->own_lo, own_hi = d->own_hi, n_sorted = d->n_sorted;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    double s[23];
#pragma unroll
    for (int k = 0; k < 23; ++k) s[k] = 0.0;
    float vmax = 0.0f, tmax = 0.0f;
    // the records of all kDiagPer particles are requested before any of them
    // is added, so the thread waits on one round trip instead of kDiagPer
    float4 xpu[kDiagPer], vTu[kDiagPer];
    float massu[kDiagPer];
    bool oku[kDiagPer];
#pragma unroll
    for (int u = 0; u < kDiagPer; ++u) {
      const int i = (c * kDiagPer + u) * kChunk + threadIdx.x;
      oku[u] = i < n && owned(own_lo, own_hi, n_sorted, i);
      xpu[u] = oku[u] ? V.xp[i] : make_float4(0, 0, 0, 0);
      vTu[u] = oku[u] ? V.vT[i] : make_float4(0, 0, 0, 0);
      massu[u] = oku[u] ? V.mrps[i].x : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < kDiagPer; ++u) {
      const int i = (c * kDiagPer + u) * kChunk + threadIdx.x;
      if (oku[u]) {
        const float4 xp = xpu[u];
        const int ph = ph_of(xp);
        const float4 vT = vTu[u];
        const double m = massu[u];
        if (ph == kLiquid || ph == kVapor) {
          // per-phase slots chosen by selects, not by a run-time index, so the
          // 23 sums stay in registers (an indexed store would put them in
          // local memory)
          const bool liq = ph == kLiquid;
          const double ke = 0.5 * m * (double)norm2(xyz(vT));
          const double H = m * (double)specific_enthalpy(P, ph, vT.w);
          const double mT = m * vT.w;
          s[0] += liq ? 1.0 : 0.0;
          s[1] += liq ? 0.0 : 1.0;
          s[3] += liq ? m : 0.0;
          s[4] += liq ? 0.0 : m;
          s[5] += liq ? ke : 0.0;
          s[6] += liq ? 0.0 : ke;
          s[7] += liq ? H : 0.0;
          s[8] += liq ? 0.0 : H;
          s[9] += liq ? mT : 0.0;
          s[10] += liq ? 0.0 : mT;
          const float4 fw = V.fw[i], mw = V.mw[i];
          s[17] += fw.x; s[18] += fw.y; s[19] += fw.z;
          s[20] += mw.x; s[21] += mw.y; s[22] += mw.z;
          vmax = fmaxf(vmax, norm(xyz(vT)));
          if (ph == kLiquid) {
            s[11] += m * xp.x; s[12] += m * xp.y; s[13] += m * xp.z;
            s[14] += m * vT.x; s[15] += m * vT.y; s[16] += m * vT.z;
            tmax = fmaxf(tmax, vT.w);
          }
        } else if (ph == kWall) {
          s[2] += 1.0;
        }
      }
    }
    publish_chunk<23>(R, c, s, sh);
    // chunk maxima (order-free)
    vmax = warp_max(vmax);
    tmax = warp_max(tmax);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
      shmax[0][warp] = vmax;
      shmax[1][warp] = tmax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      float a = 0.0f, b = 0.0f;
      for (int w = 0; w < kBlock / 32; ++w) {
        a = fmaxf(a, shmax[0][w]);
        b = fmaxf(b, shmax[1][w]);
      }
      R.partials[(size_t)23 * R.max_chunks + c] = a;
      R.partials[(size_t)24 * R.max_chunks + c] = b;
    }
    __syncthreads();
  }
  if (last_block(R.ticket)) {
    // the 23 sums spread over the block's warps, one warp per value
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int v = warp; v < 23; v += kBlock / 32) {
      const double s = warp_sum_partials(R, v, nch);
      if (lane == 0) out[v] = s;
    }
    __shared__ float wm[2][kBlock / 32];
    for (int v = 23; v < 25; ++v) {
      float mx = 0.0f;
      const double* p = R.partials + (size_t)v * R.max_chunks;
      for (int k = threadIdx.x; k < nch; k += blockDim.x) mx = fmaxf(mx, (float)__ldcg(p + k));
      mx = warp_max(mx);
      if ((threadIdx.x & 31) == 0) wm[v - 23][threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      float mx = 0.0f;
      for (int w = 0; w < kBlock / 32; ++w) mx = fmaxf(mx, wm[threadIdx.x][w]);
      out[23 + threadIdx.x] = mx;
    }
    if (threadIdx.x == 0) {  // the scalar state, so the host needs one copy
      out[25] = d->time; out[26] = (double)d->step; out[27] = d->last_dt; out[28] = d->n;
      out[29] = d->heat_input; out[30] = d->evaporated; out[31] = d->condensed; out[32] = d->vented;
      out[33] = d->vented_h; out[34] = d->T_sat; out[35] = d->p_ullage; out[36] = d->splits; out[37] = d->merges;
      for (int k = 0; k < 3; ++k) {
        out[38 + k] = d->fr.frame_acc[k];
        out[41 + k] = d->fr.omega[k];
      }
    }
  }
}

// Telemetry record pack (telemetry.cu:70-84): x, T, p, |v|, phase.
__global__ void __launch_bounds__(kBlock) k_telemetry_pack(View V, TelemetryRecord* __restrict__ out) {
  const int n = V.dyn->n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 xp = V.xp[i];
    const float4 vT = V.vT[i];
    TelemetryRecord r;
    r.x = xp.x;
    r.y = xp.y;
    r.z = xp.z;
    r.T = vT.w;
    r.p = V.mrps[i].z;
    r.speed = norm(xyz(vT));
    r.phase = (uint32_t)ph_of(xp);
    out[i] = r;
  }
}

}  // namespace cryo
