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

// Per digit (one block each): exclusive scan of the tile counts hist[d][*]
// in place and the digit total in hist_tot[d].  The downsweep adds the
// exclusive prefix of the digit totals.
__global__ void __launch_bounds__(RS_SCAN_THREADS) k_rs_scan(uint32_t* __restrict__ hist,
                                                              const DynState* __restrict__ dyn) {
  const int n = dyn->n;
  const int nt = (n + RS_TILE - 1) / RS_TILE;
  const int d = blockIdx.x;
  uint32_t* row = hist + (size_t)d * nt;
  const int per = (nt + blockDim.x - 1) / blockDim.x;
  const int lo = threadIdx.x * per, hi = min(lo + per, nt);
  uint32_t s = 0;
  for (int k = lo; k < hi; ++k) s += row[k];
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
    const uint32_t c = row[k];
    row[k] = run;
    run += c;
  }
  if (threadIdx.x == blockDim.x - 1) hist[(size_t)RS_BINS * nt + d] = run;  // digit total
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
  // digit offsets: exclusive scan of the digit totals (RS_BINS entries)
  __shared__ uint32_t dig[RS_BINS];
  for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) dig[d] = hist[(size_t)RS_BINS * nt + d];
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t carry = 0;
    for (int base = 0; base < RS_BINS; base += 32) {
      const uint32_t x = dig[base + threadIdx.x];
      uint32_t incl = x;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (threadIdx.x >= o) incl += t;
      }
      dig[base + threadIdx.x] = carry + incl - x;
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
  }
  __syncthreads();
  // exclusive scan of the per-warp counts across warps, per digit
  for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) {
    uint32_t run = dig[d] + hist[d * nt + b];
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
// One pass over the sorted keys (clamped to num_cells: dead particles carry
// that sentinel) instead of a binary search per cell: position i (0..n, with
// key[-1] = -1 and key[n] = num_cells) writes i to every cell in
// (key[i-1], key[i]], so each cell receives its lower bound exactly once.
// A run longer than 8 cells (the empty cells of padding layers or around a
// tank) is written by the whole warp together.
__global__ void k_cells(Params P, const uint32_t* __restrict__ keys, DynState* dyn, int* __restrict__ cell_begin) {
  const int n = dyn->n;
  const int nc = P.num_cells;
  const int lane = threadIdx.x & 31;
  // whole warps walk 32 positions at a time (a warp-uniform loop), so every
  // lane takes part in the ballots
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w * 32 <= n; w += warps) {
    const int i = w * 32 + lane;
    int lo = 0, hi = -1;  // cells lo..hi get i
    if (i <= n) {
      lo = (i == 0 ? -1 : (int)min(__ldg(keys + i - 1), (uint32_t)nc)) + 1;
      hi = i == n ? nc : (int)min(__ldg(keys + i), (uint32_t)nc);
    }
    const int len = hi - lo + 1;
    if (len > 0 && len <= 8) {
      for (int c = lo; c <= hi; ++c) cell_begin[c] = i;
      if (hi == nc) dyn->n_alive = i;
    }
    unsigned longs = __ballot_sync(0xffffffffu, len > 8);
    while (longs) {
      const int src = __ffs(longs) - 1;
      longs &= longs - 1u;
      const int rl = __shfl_sync(0xffffffffu, lo, src), rh = __shfl_sync(0xffffffffu, hi, src);
      const int ri = __shfl_sync(0xffffffffu, i, src);
      for (int c = rl + lane; c <= rh; c += 32) cell_begin[c] = ri;
      if (lane == src && rh == nc) dyn->n_alive = ri;
    }
  }
}

// Reorder gather of the persistent arrays (spatial_hash.cu:116-138), fused
// into one pass: dst[i] = src[perm[i]] for i < n_alive; then n = n_alive.
// Also counts the owned fluid and wall particles per chunk (every particle
// unless the context is one slab of a tank); the last block turns the counts
// into the chunk offsets of the ordered phase index lists (partials rows 0
// and 1) and their lengths.
__global__ void __launch_bounds__(kBlock) k_gather(Params P, View src, View dst, const uint32_t* __restrict__ perm,
                                                   Reduce R, int reset_maxima) {
  __shared__ double sh[2 * kBlock / 32];
  DynState* dyn = src.dyn;
  // the step's maxima start over for the force pass to come (the step size
  // was taken from them by the launch before the sort)
  if (reset_maxima && blockIdx.x == 0 && threadIdx.x == 0) {
    dyn->v_max = 0.0f;
    dyn->a_max = 0.0f;
    dyn->Tv_max = 0.0f;
    dyn->nu_t_max = 0.0f;
    dyn->spacing_ratio = 1.0f;
  }
  const int na = dyn->n_alive;
  const int nch = num_chunks(na);
  int own_lo, own_hi;
  owned_layers(P, src.cell_begin, own_lo, own_hi);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double cnt[2] = {0.0, 0.0};
    if (i < na) {
      const uint32_t j = perm[i];
      const float4 xp = src.xp[j];
      dst.xp[i] = xp;
      dst.vT[i] = src.vT[j];
      dst.vt[i] = src.vt[j];
      dst.nrm[i] = src.nrm[j];
      dst.mrps[i] = src.mrps[j];
      dst.id[i] = src.id[j];
      const int ph = ph_of(xp);
      const bool own = i >= own_lo && i < own_hi;
      if (is_fluid(ph) && own) cnt[0] = 1.0;
      else if (ph == kWall && own) cnt[1] = 1.0;
      if (P.use_lists && is_fluid(ph)) dst.cell_fluid[cell_index(P, xyz(xp))] = 1;
    }
    publish_chunk<2>(R, c, cnt, sh);
  }
  if (last_block(R.ticket)) {
    const double nf = block_exclusive_scan(R, 0, nch);
    const double nw = block_exclusive_scan(R, 1, nch);
    if (threadIdx.x == 0) {
      dyn->n_fluid_list = (int)nf;
      dyn->n_wall_list = (int)nw;
      dyn->n = na;
    }
  }
}

// Neighbour lists of every particle in the reference's iteration order
// (for_each_neighbor filtered by r^2 < support^2, self included), stored
// transposed so a warp reads consecutive words.  mode LISTS_PHASE also fills
// the ordered fluid / wall index lists from the gather's chunk offsets.
__global__ void __launch_bounds__(kBlock, LIST_MIN_BLOCKS) k_build_lists(Params P, View V, Reduce R, int mode) {
  __shared__ int wcnt[2][kBlock / 32];
  // each thread gathers a chunk of kNbrChunk entries here and stores it as
  // one full 32-byte sector (column per thread: no bank conflicts)
  __shared__ int stage[kNbrChunk][kBlock];
#pragma unroll
  for (int q = 0; q < kNbrChunk; ++q) stage[q][threadIdx.x] = 0;  // the unused tail of a last chunk
  DynState* dyn = V.dyn;
  const int n = dyn->n;
  const int nch = num_chunks(n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned overflow = 0;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    const bool valid = i < n;
    const float4 xpi = valid ? V.xp[i] : make_float4(0, 0, 0, 0);
    const int ph = valid ? ph_of(xpi) : kDead;
    if (mode != LISTS_ONLY) {
      // ordered phase lists of the owned particles: chunk offset + rank inside the chunk
      int own_lo, own_hi;
      owned_layers(P, V.cell_begin, own_lo, own_hi);
      const bool own = i >= own_lo && i < own_hi;
      const bool isf = valid && own && is_fluid(ph), isw = valid && own && ph == kWall;
      const unsigned bf = __ballot_sync(0xffffffffu, isf), bw = __ballot_sync(0xffffffffu, isw);
      if (lane == 0) {
        wcnt[0][warp] = __popc(bf);
        wcnt[1][warp] = __popc(bw);
      }
      __syncthreads();
      int pf = 0, pw = 0;
      for (int w = 0; w < warp; ++w) {
        pf += wcnt[0][w];
        pw += wcnt[1][w];
      }
      const unsigned lt = (1u << lane) - 1u;
      if (isf) V.fluid_idx[(int)__ldcg(R.partials + c) + pf + __popc(bf & lt)] = i;
      if (isw) V.wall_idx[(int)__ldcg(R.partials + R.max_chunks + c) + pw + __popc(bw & lt)] = i;
      __syncthreads();
    }
    if (!valid) continue;
    const V3 xi = xyz(xpi);
    int cnt = 0;
    const int t = threadIdx.x;
    int4* chunk = reinterpret_cast<int4*>(V.nbr + (size_t)i * kNbrChunk);
    const size_t cstride = (size_t)V.capacity * (kNbrChunk / 4);  // in int4
    auto store_chunk = [&](int q) {
      int4* dst = chunk + (size_t)q * cstride;
      dst[0] = make_int4(stage[0][t], stage[1][t], stage[2][t], stage[3][t]);
      dst[1] = make_int4(stage[4][t], stage[5][t], stage[6][t], stage[7][t]);
    };
    // A wall's list holds its fluid neighbours only: every pass that walks
    // a wall's neighbours (the wall boundary pass and its reverse) skips the
    // other walls, so the fluid entries in their order are all it needs;
    // rows of cells with no fluid are not scanned.
    const bool wall_i = ph == kWall;
    const CellWindow W(P, xi);
    for (int z = W.z0; z <= W.z1; ++z) {
      for (int y = W.y0; y <= W.y1; ++y) {
        // every row of the 27-cell block, whole: lanes in one cell then walk
        // the same ranges (dropping rows beyond the support radius, as the
        // cell scan does, saves candidates but splits the warp more)
        const int xs = W.x0, xe = W.x1;
        const int row = (z * P.ny + y) * P.nx;
        if (wall_i) {
          bool any = false;
          for (int x = xs; x <= xe; ++x) any |= V.cell_fluid[row + x] != 0;
          if (!any) continue;
        }
        const int s = __ldg(V.cell_begin + row + xs);
        const int e = __ldg(V.cell_begin + row + xe + 1);
        // candidates in groups of LIST_GROUP: all loads issued before the
        // tests, so a thread has that many positions in flight
        auto test = [&](const float4& xj, int j) {
          const V3 rij = xi - xyz(xj);
          const float r2 = norm2(rij);
          if (r2 < P.support2 && (!wall_i || is_fluid(ph_of(xj)))) {
            if (cnt < kMaxNbr) {
              stage[cnt & (kNbrChunk - 1)][t] = j;
              if ((cnt & (kNbrChunk - 1)) == kNbrChunk - 1) store_chunk(cnt / kNbrChunk);
            }
            ++cnt;
          }
        };
        int j = s;
        for (; j + LIST_GROUP <= e; j += LIST_GROUP) {
          float4 xg[LIST_GROUP];
#pragma unroll
          for (int u = 0; u < LIST_GROUP; ++u) xg[u] = __ldg(V.xp + j + u);
#pragma unroll
          for (int u = 0; u < LIST_GROUP; ++u) test(xg[u], j + u);
        }
        for (; j < e; ++j) test(__ldg(V.xp + j), j);
      }
    }
    if (cnt < kMaxNbr && (cnt & (kNbrChunk - 1)) != 0) store_chunk(cnt / kNbrChunk);  // partial last chunk
    V.nbr_cnt[i] = cnt;
    if (cnt > kMaxNbr) overflow = CRYO_DEV_NBR_OVERFLOW;
  }
  if (overflow) atomicOr(&dyn->status, overflow);
}

// Neighbour list dump (test hook): counts, then the lists at given offsets.
// stored = 0: the cell scan (every neighbour); 1: the lists of the last
// build, as the passes walk them (walls: their fluid neighbours only).
__global__ void k_nbr_count(Params P, View V, int stored, int* __restrict__ counts) {
  const int n = V.dyn->n;
  P.use_lists = stored;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = 0;
    for_each_nbr(P, V, i, xyz(V.xp[i]), [&](int, float4, V3, float) { ++c; });
    counts[i] = c;
  }
}
__global__ void k_nbr_fill(Params P, View V, int stored, const long long* __restrict__ offsets,
                           int* __restrict__ list) {
  const int n = V.dyn->n;
  P.use_lists = stored;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    long long o = offsets[i];
    for_each_nbr(P, V, i, xyz(V.xp[i]), [&](int j, float4, V3, float) { list[o++] = j; });
  }
}

}  // namespace cryo
