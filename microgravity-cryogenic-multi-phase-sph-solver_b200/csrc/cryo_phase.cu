// cryo_phase.cu -- integrator half-kicks and the phase-change stages
// (Solver::step / phase_change_step, sph_solver.cu:20-57,511-584;
// phase_change.cu:77-358).
#include "cryo_kernels.cuh"

namespace cryo {

#define PARTICLE_LOOP(i, n) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

__global__ void __launch_bounds__(kBlock) k_kick_drift(Params P, View V, int continuity, int tvf) {
  const DynState* dyn = V.dyn;
  const int n = dyn->n;
  const float dt = dyn->dt;
  PARTICLE_LOOP(i, n) {
    float4 xp = V.xp[i];
    if (is_fluid(ph_of(xp))) kick_drift_one(P, V, i, dt, continuity, tvf, xp);
  }
}

// phase_change_sources (phase_change.cu:77-137) for particle i.
__device__ inline void pc_source_one(const Params& P, const View& V, int i, float T_sat, float dt, float4 xp) {
  const int ph = ph_of(xp);
  int fl = fl_of(xp) & ~kScratchMask;
  float out_m = 0.0f, out_h = 0.0f;
  if (is_fluid(ph)) {
    const int ii = phase_index(ph);
    const float m = V.mrps[i].x;
    const float T = V.vT[i].w;
    if (m < P.merge_ratio * P.mref[ii]) {
      out_m = m;
      out_h = specific_enthalpy(P, ph, T);
      fl |= kSource | kDying;
      if (ph == kVapor) fl |= kTargetVapor;
    } else {
      const float alpha = V.nrm[i].w;
      if (P.phase_change && alpha > 0.0f && dt > 0.0f) {
        if (ph == kLiquid && T > T_sat) {
          const float h_out = P.h_fg + P.cp[1] * (T_sat - P.T_ref);
          const float latent = h_out - P.cp[0] * (T_sat - P.T_ref);
          const float rate = P.lee_evap * m * alpha * (T - T_sat) / T_sat;
          float dm = rate * dt;
          const float dm_energy = m * P.cp[0] * (T - T_sat) / latent;
          dm = dm < dm_energy ? dm : dm_energy;
          const float dm_cap = P.max_transfer_fraction * m;
          dm = dm < dm_cap ? dm : dm_cap;
          if (dm > 0.0f) {
            out_m = dm;
            out_h = h_out;
            fl |= kSource | kTargetVapor;
          }
        } else if (ph == kVapor && T < T_sat) {
          const float rate = P.lee_cond * m * alpha * (T_sat - T) / T_sat;
          float dm = rate * dt;
          float dm_cap = P.max_transfer_fraction * m;
          if (P.pc_density_limit > 0.0f && P.pc_density_limit * m < dm_cap) dm_cap = P.pc_density_limit * m;
          dm = dm < dm_cap ? dm : dm_cap;
          if (dm > 0.0f) {
            out_m = dm;
            out_h = specific_enthalpy(P, kVapor, T);
            fl |= kSource;
          }
        }
      }
    }
  }
  V.pc[i] = make_float4(out_m, out_h, 0.0f, V.pc[i].w);
  reinterpret_cast<float*>(V.xp + i)[3] = pack_pf(ph, fl);
}

// kick (sph_solver.cu:36-46).  flags & KICK_SOURCES: the phase-change sources
// of the same particle follow (they only read the particle's own kicked
// state; skipped while relax freezes phase change).  flags & KICK_HEAT: the
// heater energy is accumulated (sph_solver.cu:527).
__global__ void __launch_bounds__(kBlock) k_kick(Params P, View V, int flags) {
  DynState* dyn = V.dyn;
  const int sources = flags & KICK_SOURCES;
  const int n = dyn->n;
  const float dt = dyn->dt;
  const float half = 0.5f * dt;
  const int thermal = dyn->thermal_on;
  const float T_sat = dyn->T_sat;
  const bool do_src = sources && dyn->phase_change_on;
  PARTICLE_LOOP(i, n) {
    const float4 xp = V.xp[i];
    if (is_fluid(ph_of(xp))) {
      float4 vT = V.vT[i];
      const float4 a4 = V.a4[i];
      const V3 v = xyz(vT) + xyz(a4) * half;
      float T = vT.w;
      if (thermal) T += a4.w * dt;
      V.vT[i] = f4(v, T);
    }
    if (do_src) pc_source_one(P, V, i, T_sat, dt, xp);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && (flags & KICK_HEAT)) {
    if (thermal && dyn->heat_inv_norm > 0.0f) dyn->heat_input += (double)P.heat_power * (double)dt;
  }
}

__global__ void __launch_bounds__(kBlock) k_pc_sources(Params P, View V) {
  const DynState* dyn = V.dyn;
  const int n = dyn->n;
  PARTICLE_LOOP(i, n) pc_source_one(P, V, i, dyn->T_sat, dyn->dt, V.xp[i]);
}

// phase_change_normalize (phase_change.cu:139-172); with `sums` (step mode)
// the FP64 bookkeeping of sph_solver.cu:550-552 (sum_phase_change,
// count_merges) is reduced in the same pass and added to the cumulative
// counters.  Step mode is skipped while relax freezes phase change.
__global__ void __launch_bounds__(kBlock) k_pc_normalize(Params P, View V, Reduce R, int sums) {
  __shared__ double sh[3 * kBlock / 32];
  DynState* dyn = V.dyn;
  if (sums && !dyn->phase_change_on) return;
  const int n = dyn->n;
  const int nch = num_chunks(n);
  const int own_lo = dyn->own_lo, own_hi = dyn->own_hi, n_sorted = dyn->n_sorted;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double s[3] = {0.0, 0.0, 0.0};
    if (i < n && owned(own_lo, own_hi, n_sorted, i)) {  // a slab skips its ghosts
      const float4 xpi = V.xp[i];
      const int fl = fl_of(xpi);
      if (fl & kSource) {
        const int target = (fl & kTargetVapor) ? kVapor : kLiquid;
        float wsum = 0.0f, wr_max = 0.0f;
        for_each_nbr(P, V, i, xyz(xpi), [&](int j, float4 xj, V3, float r2) {
          if (j == i || ph_of(xj) != target || (fl_of(xj) & kDying)) return;
          const float w = kernel_W(P, sqrtf(r2));
          const float4 mr = __ldg(V.mrps + j);
          const float rhoj = mr.y;
          wsum += (mr.x / rhoj) * w;
          const float wr = w / rhoj;
          wr_max = wr > wr_max ? wr : wr_max;
        });
        float4 pc = V.pc[i];
        pc.z = wsum;
        if (!(wsum > 0.0f)) {
          pc.x = 0.0f;
        } else if (target == kVapor && P.pc_density_limit > 0.0f && !(fl & kDying) && wr_max > 0.0f) {
          const float cap = P.pc_density_limit * wsum / wr_max;
          if (pc.x > cap) pc.x = cap;
        }
        V.pc[i] = pc;
        if (!(fl & kDying)) {
          if (fl & kTargetVapor) s[0] = (double)pc.x;
          else s[1] = (double)pc.x;
        } else if (pc.x > 0.0f) {
          s[2] = 1.0;
        }
      }
    }
    if (sums) publish_chunk<3>(R, c, s, sh);
  }
  if (sums && last_block(R.ticket)) {
    const double ev = block_sum_partials(R, 0, nch);
    const double co = block_sum_partials(R, 1, nch);
    const double me = block_sum_partials(R, 2, nch);
    if (threadIdx.x == 0) {
      dyn->evaporated += ev;
      dyn->condensed += co;
      dyn->merges += (int)me;
    }
  }
}

// phase_change_apply (phase_change.cu:174-215)
__global__ void __launch_bounds__(kBlock) k_pc_apply(Params P, View V, int gated) {
  const DynState* dyn = V.dyn;
  if (gated && !dyn->phase_change_on) return;
  const int n = dyn->n;
  const int own_lo = dyn->own_lo, own_hi = dyn->own_hi, n_sorted = dyn->n_sorted;  // a slab skips its ghosts
  PARTICLE_LOOP(i, n) {
    if (!owned(own_lo, own_hi, n_sorted, i)) continue;
    const float4 xpi = V.xp[i];
    const int ph = ph_of(xpi);
    if (!is_fluid(ph)) continue;
    const int fl = fl_of(xpi);
    float4 mr = V.mrps[i];
    const float mi = mr.x;
    const float Vi = mi / mr.y;
    float in_m = 0.0f, in_H = 0.0f;
    if (!(fl & kDying)) {
      for_each_nbr(P, V, i, xyz(xpi), [&](int j, float4 xj, V3, float r2) {
        // only flagged sources carry out_m > 0 (pc_source_one), so the
        // others are passed over without reading their pc record
        if (j == i || !(fl_of(xj) & kSource)) return;
        const float4 pcj = __ldg(V.pc + j);
        const float om = pcj.x;
        if (!(om > 0.0f)) return;
        const int target = (fl_of(xj) & kTargetVapor) ? kVapor : kLiquid;
        if (target != ph) return;
        const float share = om * Vi * kernel_W(P, sqrtf(r2)) / pcj.z;
        in_m += share;
        in_H += share * pcj.y;
      });
    }
    const float4 pci = V.pc[i];
    const float om_i = pci.x;
    if ((fl & kDying) && om_i > 0.0f) {
      V.mrps[i].x = 0.0f;
      reinterpret_cast<float*>(V.xp + i)[3] = pack_pf(kDead, fl);
      continue;
    }
    if (!(om_i > 0.0f) && !(in_m > 0.0f)) continue;
    const float m_new = mi - om_i + in_m;
    float4 vT = V.vT[i];
    const float H_new = mi * specific_enthalpy(P, ph, vT.w) - om_i * pci.y + in_H;
    vT.w = temperature_from_enthalpy(P, ph, H_new / m_new);
    V.vT[i] = vT;
    V.mrps[i].x = m_new;
  }
}

// rebalance_vapor_mass, pass 1 (phase_change.cu:223-250).  The momentum
// exchange goes to ns (as in the reference).
__global__ void __launch_bounds__(kBlock) k_rebalance1(Params P, View V, int gated) {
  const DynState* dyn = V.dyn;
  if (gated && !dyn->phase_change_on) return;
  const int n = dyn->n;
  const float beta = P.vapor_rebalance;
  const int own_lo = dyn->own_lo, own_hi = dyn->own_hi, n_sorted = dyn->n_sorted;  // a slab skips its ghosts
  PARTICLE_LOOP(i, n) {
    if (!owned(own_lo, own_hi, n_sorted, i)) continue;
    const float4 xpi = V.xp[i];
    const float kap = V.ns4[i].w;
    const float wn = V.pc[i].z;
    if (ph_of(xpi) != kVapor) {
      V.pc[i] = make_float4(0.0f, 0.0f, wn, 0.0f);
      V.ns4[i] = make_float4(0.0f, 0.0f, 0.0f, kap);
      continue;
    }
    const float mi = V.mrps[i].x;
    const float4 vTi = V.vT[i];
    const float hi = specific_enthalpy(P, kVapor, vTi.w);
    const V3 vi = xyz(vTi);
    float dm = 0.0f, dH = 0.0f;
    V3 dP{0, 0, 0};
    for_each_nbr_pf(P, V, i, xyz(xpi), V.mrps, [&](int j, float4 xj, V3, float r2, const float4& mrj) {
      if (j == i || ph_of(xj) != kVapor) return;
      const float mj = mrj.x;
      // equal masses give flow = +0, and every sum below gains a zero that
      // leaves it as it is
      if (mj == mi) return;
      const float flow = beta * P.vol0 * kernel_W(P, sqrtf(r2)) * (mj - mi);
      const bool from_j = flow > 0.0f;
      dm += flow;
      if (from_j) {
        const float4 vTj = __ldg(V.vT + j);
        dH += flow * specific_enthalpy(P, kVapor, vTj.w);
        dP += xyz(vTj) * flow;
      } else {
        dH += flow * hi;
        dP += vi * flow;
      }
    });
    V.pc[i] = make_float4(dm, dH, wn, 0.0f);
    V.ns4[i] = f4(dP, kap);
  }
}

// rebalance_vapor_mass, pass 2 (phase_change.cu:252-267), then
// mark_heavy_particles (phase_change.cu:270-279) with the per-chunk counts of
// the split flags for the deterministic slot scan (cuda_utils.cuh:285-293).
__global__ void __launch_bounds__(kBlock) k_rebalance2_mark(Params P, View V, Reduce R, uint32_t* __restrict__ flag,
                                                            int rebalance, int gated) {
  __shared__ double sh[kBlock / 32];
  DynState* dyn = V.dyn;
  if (gated && !dyn->phase_change_on) return;
  const int n = dyn->n;
  const int nch = num_chunks(n);
  const int own_lo = dyn->own_lo, own_hi = dyn->own_hi, n_sorted = dyn->n_sorted;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double cnt[1] = {0.0};
    if (i < n) {
      const int ph = ph_of(V.xp[i]);
      float m = V.mrps[i].x;
      if (rebalance && ph == kVapor) {
        float4 pc = V.pc[i];
        const float dm = pc.x;
        if (dm != 0.0f) {
          const float m_new = m + dm;
          float4 vT = V.vT[i];
          const float H = m * specific_enthalpy(P, kVapor, vT.w) + pc.y;
          vT.w = temperature_from_enthalpy(P, kVapor, H / m_new);
          const V3 v = (xyz(vT) * m + xyz(V.ns4[i])) / m_new;
          V.vT[i] = f4(v, vT.w);
          V.vt[i] = f4(v, V.vt[i].w);
          V.mrps[i].x = m_new;
          pc.x = 0.0f;
          pc.y = 0.0f;
          V.pc[i] = pc;
          m = m_new;
        }
      }
      const uint32_t f =
          (is_fluid(ph) && m > P.split_ratio * P.mref[phase_index(ph)] && owned(own_lo, own_hi, n_sorted, i)) ? 1u : 0u;
      flag[i] = f;
      cnt[0] = (double)f;
    }
    publish_chunk<1>(R, c, cnt, sh);
  }
  if (last_block(R.ticket)) {
    // exclusive scan of the chunk counts (in place, exact in double)
    const double total = block_exclusive_scan(R, 0, nch);
    if (threadIdx.x == 0) {
      dyn->split_requested = (int)total;
      dyn->split_total = (int)total;  // the slabs replace it with the sum over slabs
    }
  }
}

// split_heavy_particles (phase_change.cu:281-335) + the bookkeeping of
// sph_solver.cu:568-576.  Slot k of a particle = exclusive prefix of the
// flags (chunk offset + in-chunk scan), independent of thread order.
__device__ inline uint32_t hash_u32(uint32_t x) {  // phase_change.cu:9-17
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}
__device__ inline float hash_unit(uint32_t x) { return (float)(hash_u32(x) & 0x00FFFFFFu) / (float)0x01000000u; }
__device__ inline V3 random_direction(uint32_t id, uint32_t seed) {  // phase_change.cu:22-27
  const float u = 2.0f * hash_unit(id * 2654435761u ^ seed) - 1.0f;
  const float phi = 2.0f * kPi * hash_unit(hash_u32(id + 0x9e3779b9u) ^ (seed * 747796405u));
  const float s = sqrtf(1.0f - u * u > 0.0f ? 1.0f - u * u : 0.0f);
  return V3{s * cos_cr(phi), s * sin_cr(phi), u};
}

__global__ void __launch_bounds__(kBlock) k_split(Params P, View V, Reduce R, const uint32_t* __restrict__ flag,
                                                  int gated) {
  __shared__ uint32_t warp_tot[kBlock / 32];
  DynState* dyn = V.dyn;
  if (gated && !dyn->phase_change_on) return;
  const int requested = dyn->split_requested;
  if (requested == 0) {
    // no split here; the ids other slabs hand out this step are still used
    if (blockIdx.x == 0 && threadIdx.x == 0) dyn->next_id += (uint32_t)dyn->split_total;
    return;
  }
  const int n = dyn->n;
  const int cap = dyn->capacity;
  const uint32_t seed = (uint32_t)dyn->step;
  const uint32_t id_base = dyn->next_id + dyn->id_offset;
  const int nch = num_chunks(n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    const uint32_t f = i < n ? flag[i] : 0u;
    // in-chunk exclusive scan
    uint32_t incl = f;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0;
    for (int w = 0; w < warp; ++w) wpre += warp_tot[w];
    __syncthreads();
    if (!f) continue;
    const uint32_t k = (uint32_t)__ldcg(R.partials + c) + wpre + incl - f;
    const int dst = n + (int)k;
    if (dst >= cap) continue;
    float4 xp = V.xp[i];
    const int ph = ph_of(xp);
    float4 mr = V.mrps[i];
    const float m = mr.x;
    const float vol = m / mr.y;
    V3 e = random_direction(V.id[i], seed);
    const V3 xi = xyz(xp);
    const float4 nrm = V.nrm[i];
    const V3 gc = xyz(nrm);
    const float gm = norm(gc);
    V3 xd;
    if (gm > P.normal_eps) {
      const V3 nn = gc / gm;
      const V3 t = e - nn * dot(e, nn);
      e = normalized(t - nn * 0.5f);
      xd = xi + e * (0.5f * cbrt_cr(vol));
    } else {
      const float delta = 0.25f * cbrt_cr(vol);
      xd = xi + e * delta;
      const V3 xn = xi - e * delta;
      xp.x = xn.x;
      xp.y = xn.y;
      xp.z = xn.z;
    }
    const int fl = fl_of(xp);
    V.xp[i] = xp;
    V.xp[dst] = f4(xd, pack_pf(ph, fl & ~kScratchMask));
    V.vT[dst] = V.vT[i];
    V.vt[dst] = V.vt[i];  // vt and m0 (w) -- m0 is halved below
    V.ab4[dst] = make_float4(V.ab4[i].x, V.ab4[i].y, V.ab4[i].z, V.ab4[dst].w);
    V.a4[dst] = make_float4(V.a4[i].x, V.a4[i].y, V.a4[i].z, 0.0f);  // dTdt[dst] = 0
    V.nrm[dst] = nrm;
    const float m0h = V.vt[i].w * 0.5f;
    V.vt[i].w = m0h;
    V.vt[dst].w = m0h;
    const float sig2 = mr.w * 2.0f;
    V.mrps[i] = make_float4(0.5f * m, mr.y, mr.z, sig2);
    V.mrps[dst] = make_float4(0.5f * m, mr.y, mr.z, sig2);
    V.id[dst] = id_base + k;
    V.pc[dst] = make_float4(0.0f, 0.0f, V.pc[dst].z, V.pc[dst].w);
    if (P.slab) {
      // The new half had no force pass: the whole tank's arrays hold whatever
      // an earlier particle left in this slot (and so does the reference),
      // which a slab cannot know; its slot counts as no wall force.
      V.fw[dst] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      V.mw[dst] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
  }
  if (last_block(R.ticket) && threadIdx.x == 0) {
    const long long room = (long long)cap - n;
    const int added = (int)((long long)requested < room ? requested : room);
    if (added < requested) dyn->status |= CRYO_DEV_SPLIT_DROPPED;
    dyn->n = n + added;
    dyn->next_id += (uint32_t)dyn->split_total;
    dyn->splits += added;
  }
}

// apply_venting (phase_change.cu:337-358) + the sums of sph_solver.cu:581-582.
__global__ void __launch_bounds__(kBlock) k_venting(Params P, View V, Reduce R, float relax, int gated) {
  __shared__ double sh[2 * kBlock / 32];
  DynState* dyn = V.dyn;
  if (gated && !dyn->phase_change_on) return;
  const int n = dyn->n;
  const int nch = num_chunks(n);
  const int own_lo = dyn->own_lo, own_hi = dyn->own_hi, n_sorted = dyn->n_sorted;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double s[2] = {0.0, 0.0};
    if (i < n) {
      const float wn = V.pc[i].z;
      float out_m = 0.0f, out_h = 0.0f;
      if (ph_of(V.xp[i]) == kVapor) {
        float4 mr = V.mrps[i];
        const float m = mr.x;
        const float vol = m / mr.y;
        const float target = P.rho0[1] * vol;
        if (m > target) {
          const float dm = relax * (m - target);
          out_m = dm;
          out_h = specific_enthalpy(P, kVapor, V.vT[i].w);
          if (P.density_mode == CRYO_DENSITY_CONTINUITY) mr.y *= (m - dm) / m;
          mr.x = m - dm;
          V.mrps[i] = mr;
        }
      }
      V.pc[i] = make_float4(out_m, out_h, wn, 0.0f);
      if (owned(own_lo, own_hi, n_sorted, i)) {
        s[0] = (double)out_m;
        s[1] = (double)out_m * (double)out_h;
      }
    }
    publish_chunk<2>(R, c, s, sh);
  }
  if (last_block(R.ticket)) {
    const double vm = block_sum_partials(R, 0, nch);
    const double vh = block_sum_partials(R, 1, nch);
    if (threadIdx.x == 0) {
      dyn->vented += vm;
      dyn->vented_h += vh;
    }
  }
}

// scale_velocities (sph_solver.cu:48-57); damp_velocities also scales v_max
// (sph_solver.cu:701-705).
__global__ void __launch_bounds__(kBlock) k_scale_velocities(View V, float factor, int scale_vmax) {
  DynState* dyn = V.dyn;
  const int n = dyn->n;
  PARTICLE_LOOP(i, n) {
    if (!is_fluid(ph_of(V.xp[i]))) continue;
    const float4 vT = V.vT[i];
    V.vT[i] = f4(xyz(vT) * factor, vT.w);
    const float4 vt = V.vt[i];
    V.vt[i] = f4(xyz(vt) * factor, vt.w);
  }
  if (scale_vmax && blockIdx.x == 0 && threadIdx.x == 0) dyn->v_max *= factor;
}

}  // namespace cryo
