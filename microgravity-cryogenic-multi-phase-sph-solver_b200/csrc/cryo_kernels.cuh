// cryo_kernels.cuh -- declarations of the device kernels (one definition file
// each: cryo_grid.cu, cryo_physics.cu, cryo_phase.cu, cryo_control.cu).
#pragma once

#include "cryo_common.cuh"

namespace cryo {

constexpr int RS_THREADS = 256;
#ifndef RS_TILE_KEYS
#define RS_TILE_KEYS 1024
#endif
constexpr int RS_TILE = RS_TILE_KEYS;  // keys per radix tile (RS_TILE / RS_THREADS per thread)
constexpr int RS_BITS = 8;
constexpr int RS_BINS = 1 << RS_BITS;
constexpr int RS_SCAN_THREADS = 256;

// Layout of the FP64 partials of one reduction: partials[v * max_chunks + c].
struct Reduce {
  double* partials;
  unsigned* ticket;
  int max_chunks;
};


// Last-block ticket: true in exactly one block, after every block of the grid
// has published its partials (each block fences before taking a ticket).
__device__ inline bool last_block(unsigned* ticket) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (is_last && threadIdx.x == 0) *ticket = 0u;  // ready for the next launch
  return is_last;
}
// Compensated two-sum accumulation (Neumaier).
__device__ inline void neumaier(double& s, double& c, double x) {
  const double t = s + x;
  c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
  s = t;
}
// (s, c) += (s2, c2) for compensated pairs: two-sum of the heads, the
// rounding error and both tails into the tail.
__device__ inline void neumaier_pair(double& s, double& c, double s2, double c2) {
  const double t = s + s2;
  c += (fabs(s) >= fabs(s2) ? (s - t) + s2 : (s2 - t) + s) + c2;
  s = t;
}
// Sum of value v over chunks [0, nchunks), computed by the whole (last) block
// in a fixed order that depends on nothing but nchunks: thread t sums chunks
// t, t + blockDim, ... (compensated), the 32 lanes of a warp combine in a
// fixed down-shift tree, and thread 0 combines the warps in order.  Every
// thread of the block must call it; the result is valid in thread 0.
// Compensated sum of p[k] for k = k0, k0 + step, ... below n, in that order;
// the loads go out kBatch at a time ahead of the additions, so a thread
// waits on one round trip per batch instead of one per element.
__device__ inline void strided_neumaier(const double* p, int k0, int step, int n, double& s, double& c) {
  constexpr int kBatch = 8;
  for (int kb = k0; kb < n; kb += kBatch * step) {
    double x[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int k = kb + u * step;
      x[u] = k < n ? __ldcg(p + k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u)
      if (kb + u * step < n) neumaier(s, c, x[u]);
  }
}
__device__ inline double block_sum_partials(const Reduce& R, int v, int nchunks) {
  __shared__ double ws[kBlock / 32], wc[kBlock / 32];
  double s = 0, c = 0;
  const double* p = R.partials + (size_t)v * R.max_chunks;
  strided_neumaier(p, threadIdx.x, blockDim.x, nchunks, s, c);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double s2 = __shfl_down_sync(0xffffffffu, s, o), c2 = __shfl_down_sync(0xffffffffu, c, o);
    neumaier_pair(s, c, s2, c2);  // lanes >= 32 - o combine garbage that lane 0 never sees
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    ws[warp] = s;
    wc[warp] = c;
  }
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0) {
    double S = ws[0], C = wc[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) neumaier_pair(S, C, ws[w], wc[w]);
    r = S + C;
  }
  __syncthreads();
  return r;
}
// Sum of value v over chunks [0, nchunks) by one warp, in a fixed order that
// depends on nothing but nchunks: lane l sums chunks l, l + 32, ...
// (compensated), then a fixed down-shift tree.  The result is valid in lane 0.
// Several warps of a block can each take their own values at once.
__device__ inline double warp_sum_partials(const Reduce& R, int v, int nchunks) {
  const int lane = threadIdx.x & 31;
  double s = 0, c = 0;
  const double* p = R.partials + (size_t)v * R.max_chunks;
  strided_neumaier(p, lane, 32, nchunks, s, c);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double s2 = __shfl_down_sync(0xffffffffu, s, o), c2 = __shfl_down_sync(0xffffffffu, c, o);
    neumaier_pair(s, c, s2, c2);
  }
  return s + c;
}
// In-place exclusive scan of the (integral) chunk values of row v by the whole
// block; returns the total (all threads).  Integral doubles add exactly, so
// the parallel order gives the serial result.
__device__ inline double block_exclusive_scan(const Reduce& R, int v, int nchunks) {
  __shared__ double wtot[kBlock / 32];
  __shared__ double total;
  double* p = R.partials + (size_t)v * R.max_chunks;
  const int per = (nchunks + blockDim.x - 1) / blockDim.x;
  const int lo = threadIdx.x * per, hi = min(lo + per, nchunks);
  double seg = 0;
  for (int k = lo; k < hi; ++k) seg += __ldcg(p + k);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double x = seg;  // inclusive scan over the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wtot[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    double run = 0;
    for (int w = 0; w < nw; ++w) {
      const double t = wtot[w];
      wtot[w] = run;
      run += t;
    }
    total = run;
  }
  __syncthreads();
  double run = wtot[warp] + (x - seg);
  for (int k = lo; k < hi; ++k) {
    const double y = __ldcg(p + k);
    p[k] = run;
    run += y;
  }
  const double t = total;
  __syncthreads();
  return t;
}
// Writes the block sums of NV values (one per thread each) for chunk c:
// every warp reduces its lanes, then lane k of warp 0 adds value k's warp
// sums in warp order (from 0.0, one after another) and stores it, so the
// values are finished side by side rather than one after another by one
// thread; each value's additions are the same either way.  `sh` must hold
// NV * (blockDim / 32) doubles; every thread of the block must call it.
template <int NV>
__device__ inline void publish_chunk(const Reduce& R, int c, double (&v)[NV], double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[k * nw + warp] = v[k];
  __syncthreads();
  if (warp == 0)
    for (int k = lane; k < NV; k += 32) {
      double s = 0;
      for (int w = 0; w < nw; ++w) s += sh[k * nw + w];
      R.partials[(size_t)k * R.max_chunks + c] = s;
    }
  __syncthreads();  // sh is free again
}
__device__ inline int num_chunks(int n) { return (n + kChunk - 1) / kChunk; }

// grid (cryo_grid.cu)
__global__ void k_keys(Params P, View V, uint32_t* keys);
__global__ void k_rs_upsweep(const uint32_t* keys, int shift, int bits, const DynState* dyn, uint32_t* hist);
__global__ void k_rs_scan(uint32_t* hist, const DynState* dyn);
__global__ void k_rs_downsweep(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, int shift,
                               int bits, const DynState* dyn, const uint32_t* hist);
__global__ void k_cells(Params P, const uint32_t* keys, DynState* dyn, int* cell_begin);
__global__ void k_gather(Params P, View src, View dst, const uint32_t* perm, Reduce R, int reset_maxima);
enum { LISTS_ONLY = 0, LISTS_PHASE = 1 };
__global__ void k_build_lists(Params P, View V, Reduce R, int mode);
__global__ void k_nbr_count(Params P, View V, int stored, int* counts);
__global__ void k_nbr_fill(Params P, View V, int stored, const long long* offsets, int* list);

// physics (cryo_physics.cu).  Fused rate pass; `what` selects the sub-passes (FORCE_* bits).
enum { FORCE_TRANSPORT = 1, FORCE_MOMENTUM = 2, FORCE_CSF = 4, FORCE_AKINCI = 8, FORCE_DRHO = 16,
       FORCE_THERMAL = 32, FORCE_MAXIMA = 64, FORCE_THERMAL_ALWAYS = 128,
       FORCE_TAPE = 256 };  // compile-time only: also store the sums into V.tape
// cryo_physics.cu is compiled twice.  namespace exact: the reference's IEEE
// single-precision operation sequence (no FMA contraction, IEEE division and
// square root), bit-identical to its CPU build.  namespace fast: the same
// source with FMA contraction and the approximate (2 ulp) division and square
// root, as the reference's own CUDA build contracts; fields then agree with
// the exact sequence to ~1e-6 relative per pass.  The neighbour lists, keys
// and sort are not in that file, so they stay bit-exact in both.
#define CRYO_FIELD_KERNELS                                                           \
  __global__ void k_density(Params P, View V, int fuse_eos);                        \
  __global__ void k_aux(Params P, View V);                                          \
  __global__ void k_normalize_masses(Params P, View V);                             \
  __global__ void k_eos(Params P, View V);                                          \
  __global__ void k_wall(Params P, View V);                                         \
  template <int TAPE>                                                               \
  __global__ void k_interface(Params P, View V, Reduce R, int heat_sum);            \
  __global__ void k_sps(Params P, View V);                                          \
  __global__ void k_smooth_normals(Params P, View V);                               \
  template <int WHAT>                                                               \
  __global__ void k_forces_t(Params P, View V, int what_rt);                        \
  __global__ void k_maxima(Params P, View V);                                       \
  __global__ void k_shift_compute(Params P, View V);                                \
  __global__ void k_shift_apply(Params P, View V);                                  \
  __global__ void k_probe(Params P, View V, const float* pts, int np, float* out);
namespace exact {
CRYO_FIELD_KERNELS
}
namespace fast {
CRYO_FIELD_KERNELS
}
// heat_sum of k_interface: 0 none, 1 when thermal is on (step), 2 always (operator call)
// TAPE: also store the sums into V.tape (the recomputation of a differentiated window).
constexpr int FORCE_BASE = FORCE_TRANSPORT | FORCE_MOMENTUM | FORCE_MAXIMA;
// Block shape of the force pass.  The pass is bound by the latency of each
// particle's neighbour chain, so what matters is how many particles are in
// flight at once.  Asking for 9 resident 64-thread blocks per SM makes the
// compiler fit 5 warps in each SM sub-partition's register file (96
// registers), 20 warps per SM: the 82k fluid particles of the dam break run
// in one wave.  A 112-register cap fits only 4 warps per sub-partition (16
// per SM) and needs two waves, 30 % slower there.
#ifndef FORCES_BLOCK
#define FORCES_BLOCK 64
#endif
#ifndef FORCES_MIN_BLOCKS
#define FORCES_MIN_BLOCKS 9
#endif
// The sub-pass sets with surface tension or heat need ~125 registers; at
// 8 blocks per SM (4 warps per sub-partition) they run without spilling.
#ifndef FORCES_MIN_BLOCKS_HEAVY
#define FORCES_MIN_BLOCKS_HEAVY 8
#endif
constexpr int forces_min_blocks(int what) {
  return (what >= 0 && (what & (FORCE_CSF | FORCE_THERMAL))) ? FORCES_MIN_BLOCKS_HEAVY : FORCES_MIN_BLOCKS;
}
// Neighbour-list build: candidate positions loaded per group, and the block
// count per SM the register cap keeps resident.
// Neighbour-loop unroll of the force-pass variants with surface tension or
// heat (the two-phase tanks): 2 takes the 4 M-particle LH2 sphere 3 % faster,
// no spills.
#ifndef FORCES_UNROLL_HEAVY
#define FORCES_UNROLL_HEAVY 2
#endif
#ifndef LIST_GROUP
#define LIST_GROUP 4
#endif
#ifndef LIST_MIN_BLOCKS
#define LIST_MIN_BLOCKS 4
#endif

// integrator + phase change (cryo_phase.cu)
__global__ void k_kick_drift(Params P, View V, int continuity, int tvf);
enum { KICK_SOURCES = 1, KICK_HEAT = 2 };
__global__ void k_kick(Params P, View V, int flags);
__global__ void k_pc_sources(Params P, View V);
__global__ void k_pc_normalize(Params P, View V, Reduce R, int sums);
__global__ void k_pc_apply(Params P, View V, int gated);
__global__ void k_rebalance1(Params P, View V, int gated);
__global__ void k_rebalance2_mark(Params P, View V, Reduce R, uint32_t* flag, int rebalance, int gated);
__global__ void k_split(Params P, View V, Reduce R, const uint32_t* flag, int gated);
__global__ void k_venting(Params P, View V, Reduce R, float relax, int gated);
__global__ void k_scale_velocities(View V, float factor, int scale_vmax);

// step control + reductions (cryo_control.cu)
enum { BEGIN_STEP = 0, BEGIN_RATES = 1 };
__global__ void k_begin_step(Params P, View V, int mode);
__global__ void k_heat_norm(Params P, View V, Reduce R);
// The ullage pressure and saturation temperature from the phase sums
// (sph_solver.cu:586-607).
__device__ inline void saturation_update(const Params& P, DynState* d, bool closed, double m_liq, double m_vap,
                                         double mT_vap) {
  bool done = false;
  if (closed) {
    if (!(d->fluid_volume0 > 0)) d->fluid_volume0 = m_liq / P.f_rho_l + m_vap / P.f_rho_v;
    const double v_ullage = d->fluid_volume0 - m_liq / P.f_rho_l;
    const double ratio = v_ullage > 0 && m_vap > 0 ? (mT_vap / v_ullage) / ((double)P.f_rho_v * P.f_T_sat) : 0.0;
    if (isfinite(ratio) && ratio > 0) {
      d->p_ullage = P.f_p_sat * ratio;
      // FluidProperties::saturation_temperature (fluid_properties.cpp:7-10)
      const float p = (float)d->p_ullage;
      const double inv_T = 1.0 / P.f_T_sat - ((double)P.f_R_gas / P.f_h_fg) * log((double)p / P.f_p_sat);
      d->T_sat = (float)(1.0 / inv_T);
      done = true;
    }
  }
  if (!done) {
    d->p_ullage = P.f_p_sat;
    d->T_sat = P.f_T_sat;
  }
}
__global__ void k_saturation(Params P, View V, Reduce R, int end_of_step);
__global__ void k_begin_kick_drift_keys(Params P, View V, uint32_t* keys);
__global__ void k_kick_saturation(Params P, View V, Reduce R);
__global__ void k_diagnostics(Params P, View V, Reduce R, double* out);

// Packed per-particle telemetry record (telemetry.hpp:28-31).
struct TelemetryRecord {
  float x, y, z, T, p, speed;
  uint32_t phase;
};
__global__ void k_telemetry_pack(View V, TelemetryRecord* out);

// Number of FP64 values per chunk of the diagnostics reduction.
constexpr int kDiagValues = 30;

// tank lattice generator (cryo_setup.cu)
constexpr int kGeomNodes = CRYO_GEOM_MAX_NODES;
// One geometry node with the offsets of its Translated ancestors, root first
// (applied to the query point in that order, as the nested sdf calls do).
struct GeomNode {
  int kind, a, b, nofs;
  double p[3];
  double ofs[kGeomNodes][3];
};
// Lattice nodes at ((i0 + i + 1/2) h, ...), i < nx, ...; band = wall_layers h.
// Slab decomposition of one tank (cryo_slab.cu).
__global__ void k_slab_bounds(Params P, View V, int zb, int ze);
__global__ void k_halo_pull(Params P, View dst, View src, int z);
__global__ void k_slab_heat(Params P, DynState* const* dyns, int nslabs, DynState* mine, int heat_mode);
__global__ void k_slab_split(DynState* const* dyns, int nslabs, int rank, DynState* mine);
__global__ void k_slab_end(Params P, DynState* const* dyns, int nslabs, DynState* mine, int saturation);
__global__ void k_slab_assemble(Params P, View dst, float4* a4_out, float4* ab4_out, View lo, View me, View up,
                                int has_lo, int has_up, int zb, int ze, int depth);
__global__ void k_slab_commit(View V, const float4* a4_in, const float4* ab4_in);

struct Lattice {
  int i0, j0, k0, nx, ny, nz;
  long long total;
  double h, band;
};
// Fill of the generated tank: key direction or centre, the liquid cut, the
// per-phase mass, density and temperature, the heater band.
struct FillDev {
  int mode, include_vapor, any_liquid;
  float g[3], c[3];
  double cut;
  float m_liq, m_vap, rho_liq, rho_vap, T_liq, T_vap, T_wall;
  double heater_zmin, heater_zmax;
};
__global__ void k_lattice_classify(const GeomNode* G, int ng, Lattice L, uint8_t* cls, uint32_t* cnt_f,
                                   uint32_t* cnt_w);
__global__ void k_scan_counts(uint32_t* cnt, int n, unsigned long long* total);
__global__ void k_lattice_scatter(Lattice L, const uint8_t* cls, const uint32_t* off_f, const uint32_t* off_w,
                                  long long* fluid_nodes, long long* wall_nodes);
__global__ void k_fill_keys(Lattice L, FillDev F, const long long* fluid_nodes, int nf, uint32_t* keys);
__global__ void k_key_digits(const uint32_t* keys, int n, uint32_t prefix, uint32_t mask, int shift,
                             unsigned int* hist);
__global__ void k_fill_split(Lattice L, FillDev F, const long long* fluid_nodes, int nf, uint8_t* liquid,
                             uint32_t* cnt_keep, uint32_t* cnt_liq);
__global__ void k_emit_walls(const GeomNode* G, int ng, Lattice L, FillDev F, const long long* wall_nodes, int nw,
                             View V);
__global__ void k_jitter_fluid(View V, int n, float amplitude, uint64_t seed);
__global__ void k_emit_fluid(Lattice L, FillDev F, const long long* fluid_nodes, int nf, const uint8_t* liquid,
                             const uint32_t* off_keep, int nw, View V);

}  // namespace cryo
