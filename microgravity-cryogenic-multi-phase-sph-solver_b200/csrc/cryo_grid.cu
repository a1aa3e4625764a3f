// cryo_grid.cu -- uniform-grid neighbour search on the GPU: integer cell keys,
// a stable LSD radix sort, the dense cell table and the reorder gather.
// Replaces SpatialHash::build / reorder_particles (spatial_hash.cu:48-138).
#include "cryo_kernels.cuh"

namespace cryo {

// Keys and the identity permutation (spatial_hash.cu:61-68): dead particles
// get the sentinel num_cells so they sort to the end.
__global__ void k_keys(Params P, View V, uint32_t* __restrict__ keys) {
  const int n = V.dyn->n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 xp = V.xp[i];
    keys[i] = ph_of(xp) == kDead ? (uint32_t)P.num_cells : (uint32_t)cell_index(P, xyz(xp));
  }
}

// ---------------------------------------------------------------- radix sort
// Stable LSD radix sort of (key, value) pairs, RS_BITS-wide digits.  One
// tile of RS_TILE keys per block; blocks beyond ceil(n / RS_TILE) exit, so the
// grid can be sized from the capacity and the key count stays on the device.
// Per pass: upsweep (digit histogram per tile), scan (digit-major, tile-minor
// exclusive scan), downsweep (stable in-tile ranking with warp match_any,
// scatter).  No atomics decide positions, so the permutation is unique.

__global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(const uint32_t* __restrict__ keys, int shift, int bits,
                                                           const DynState* __restrict__ dyn,
                                                           uint32_t* __restrict__ hist) {
  const int n = dyn->n;
  const int nt = (n + RS_TILE - 1) / RS_TILE;
  const int b = blockIdx.x;
  if (b >= nt) return;
  __shared__ uint32_t cnt[RS_BINS];
  for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) cnt[d] = 0;
  __syncthreads();
  const uint32_t mask = (1u << bits) - 1u;
  const int base = b * RS_TILE;
  for (int k = threadIdx.x; k < RS_TILE; k += blockDim.x) {
    const int idx = base + k;
    if (idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & mask], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) hist[d * nt + b] = cnt[d];
}

// Exclusive scan of hist[RS_BINS * nt] in place (one block).
__global__ void __launch_bounds__(1024) k_rs_scan(uint32_t* __restrict__ hist, const DynState* __restrict__ dyn) {
  const int n = dyn->n;
  const int nt = (n + RS_TILE - 1) / RS_TILE;
  const int total = RS_BINS * nt;
  const int per = (total + blockDim.x - 1) / blockDim.x;
  const int lo = threadIdx.x * per, hi = min(lo + per, total);
  uint32_t s = 0;
  for (int k = lo; k < hi; ++k) s += hist[k];
  __shared__ uint32_t warp_tot[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    warp_tot[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  uint32_t run = (incl - s) + (warp > 0 ? warp_tot[warp - 1] : 0);
  for (int k = lo; k < hi; ++k) {
    const uint32_t c = hist[k];
    hist[k] = run;
    run += c;
  }
}

__global__ void __launch_bounds__(RS_THREADS) k_rs_downsweep(const uint32_t* __restrict__ kin,
                                                             const uint32_t* __restrict__ vin,
                                                             uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                             int shift, int bits, const DynState* __restrict__ dyn,
                                                             const uint32_t* __restrict__ hist) {
  const int n = dyn->n;
  const int nt = (n + RS_TILE - 1) / RS_TILE;
  const int b = blockIdx.x;
  if (b >= nt) return;
  constexpr int kWarps = RS_THREADS / 32;
  constexpr int kPer = RS_TILE / kWarps / 32;  // keys per lane
  __shared__ uint32_t wcnt[kWarps][RS_BINS];
  for (int t = threadIdx.x; t < kWarps * RS_BINS; t += blockDim.x) (&wcnt[0][0])[t] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint32_t mask = (1u << bits) - 1u;
  const int wbase = b * RS_TILE + warp * (kPer * 32);
  uint32_t key[kPer], val[kPer], rank[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int idx = wbase + k * 32 + lane;
    const bool valid = idx < n;
    key[k] = valid ? kin[idx] : 0u;
    val[k] = valid ? (vin ? vin[idx] : (uint32_t)idx) : 0u;
    const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
    const uint32_t d = (key[k] >> shift) & mask;
    rank[k] = 0;
    if (valid) {
      const uint32_t peers = __match_any_sync(vmask, d);
      const uint32_t before = wcnt[warp][d];
      const int leader = __ffs(peers) - 1;
      rank[k] = before + __popc(peers & lt_mask);
      __syncwarp(vmask);
      if (lane == leader) wcnt[warp][d] = before + __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  // exclusive scan of the per-warp counts across warps, per digit
  for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) {
    uint32_t run = hist[d * nt + b];
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int idx = wbase + k * 32 + lane;
    if (idx < n) {
      const uint32_t d = (key[k] >> shift) & mask;
      const uint32_t pos = wcnt[warp][d] + rank[k];
      kout[pos] = key[k];
      vout[pos] = val[k];
    }
  }
}

// Dense cell table: cell_begin[c] = first sorted index with key >= c, for
// c in [0, num_cells]; cell_begin[num_cells] = number of live particles.
__global__ void k_cells(Params P, const uint32_t* __restrict__ keys, DynState* dyn, int* __restrict__ cell_begin) {
  const int n = dyn->n;
  const int nc = P.num_cells;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
    const int prev = i == 0 ? -1 : (int)min(keys[i - 1], (uint32_t)nc);
    const int cur = i < n ? (int)min(keys[i], (uint32_t)nc) : nc;
    for (int c = prev + 1; c <= cur; ++c) cell_begin[c] = i;
    if (prev < nc && cur >= nc) dyn->n_alive = i;
  }
}

// Reorder gather of the persistent arrays (spatial_hash.cu:116-138), fused
// into one pass: dst[i] = src[perm[i]] for i < n_alive; then n = n_alive.
__global__ void k_gather(View src, View dst, const uint32_t* __restrict__ perm) {
  DynState* dyn = src.dyn;
  const int na = dyn->n_alive;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
    const uint32_t j = perm[i];
    dst.xp[i] = src.xp[j];
    dst.vT[i] = src.vT[j];
    dst.vt[i] = src.vt[j];
    dst.nrm[i] = src.nrm[j];
    dst.mrps[i] = src.mrps[j];
    dst.id[i] = src.id[j];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) dyn->n = na;
}

// Neighbour list dump (test hook): counts, then the lists at given offsets.
__global__ void k_nbr_count(Params P, View V, int* __restrict__ counts) {
  const int n = V.dyn->n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = 0;
    for_each_neighbor(P, V.cell_begin, V.xp, xyz(V.xp[i]), [&](int, float4, V3, float) { ++c; });
    counts[i] = c;
  }
}
__global__ void k_nbr_fill(Params P, View V, const long long* __restrict__ offsets, int* __restrict__ list) {
  const int n = V.dyn->n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    long long o = offsets[i];
    for_each_neighbor(P, V.cell_begin, V.xp, xyz(V.xp[i]), [&](int j, float4, V3, float) { list[o++] = j; });
  }
}

}  // namespace cryo
