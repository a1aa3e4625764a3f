// cryo_slab.cu -- device side of the slab decomposition of one tank.
//
// A tank is cut into slabs of whole cell layers along z.  Cell keys are
// z-major (spatial_hash.hpp:22-32), so the particles of a range of layers are
// one contiguous range of a context's sorted order, and the tank's sorted
// order is the slabs' owned ranges one after another.  Each slab's context
// holds its owned layers plus ghost copies of the neighbouring slabs' layers:
//
//   * between steps every slab rebuilds its arrays from its owned particles
//     and the two layers of each neighbour that face it (refresh);
//   * during a step, after every pass whose outputs a later neighbour pass
//     reads, the ghost layer next to the slab (one cell, the whole support)
//     is copied from the slab that owns it (halo pull);
//   * sums and maxima are taken over owned particles only and combined over
//     the slabs in slab order where the step uses them.
//
// Ghost layers further out hold values computed from incomplete
// neighbourhoods; nothing owned reads them.  All copies are plain loads of
// the other context's memory (the same device, or a peer over NVLink).
#include "cryo_kernels.cuh"

namespace cryo {

// Sorted index range of cell layers [z0, z1) (clamped to the grid).
__device__ inline void layer_range(const Params& P, const int* cb, int z0, int z1, int& b, int& e) {
  const int L = P.nx * P.ny;
  z0 = z0 < 0 ? 0 : z0;
  z1 = z1 > P.nz ? P.nz : z1;
  if (z1 <= z0) {
    b = e = 0;
    return;
  }
  b = cb[z0 * L];
  e = cb[z1 * L];
}

// After a sort: the owned range of the slab of layers [zb, ze).
__global__ void k_slab_bounds(Params P, View V, int zb, int ze) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  DynState* d = V.dyn;
  int b, e;
  layer_range(P, V.cell_begin, zb, ze, b, e);
  d->own_lo = b;
  d->own_hi = e;
  d->n_sorted = d->n;
}

// Every per-particle array of a rate evaluation, particle j of src into
// particle i of dst.
__device__ inline void copy_all(const View& dst, int i, const View& src, int j) {
  dst.xp[i] = src.xp[j];
  dst.vT[i] = src.vT[j];
  dst.vt[i] = src.vt[j];
  dst.nrm[i] = src.nrm[j];
  dst.mrps[i] = src.mrps[j];
  dst.id[i] = src.id[j];
  dst.a4[i] = src.a4[j];
  dst.ab4[i] = src.ab4[j];
  dst.fw[i] = src.fw[j];
  dst.mw[i] = src.mw[j];
  dst.vwp[i] = src.vwp[j];
  dst.ns4[i] = src.ns4[j];
  dst.pc[i] = src.pc[j];
  dst.aux[i] = src.aux[j];
  dst.rmin[i] = src.rmin[j];
  dst.wall_w[i] = src.wall_w[j];
  dst.heat_w[i] = src.heat_w[j];
  dst.nu_t[i] = src.nu_t[j];
}

// Ghost layer z of dst := the same layer of src, the slab that owns it.  Both
// hold the same particles there in the same order; a count that differs is
// flagged and nothing is copied.
__global__ void __launch_bounds__(kBlock) k_halo_pull(Params P, View dst, View src, int z) {
  int db, de, sb, se;
  layer_range(P, dst.cell_begin, z, z + 1, db, de);
  layer_range(P, src.cell_begin, z, z + 1, sb, se);
  if (de - db != se - sb) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&dst.dyn->status, (unsigned)CRYO_DEV_SLAB_HALO);
    return;
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < de - db; k += gridDim.x * blockDim.x)
    copy_all(dst, db + k, src, sb + k);
}

// Heat-weight normalisation over every slab (sph_solver.cu:466-472): the
// owned sums added in slab order.  heat_mode is the pass's heat_sum switch.
__global__ void k_slab_heat(Params P, DynState* const* dyns, int nslabs, DynState* mine, int heat_mode) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double S = 0.0;
  for (int r = 0; r < nslabs; ++r) S += dyns[r]->heat_sum;
  if (heat_mode == 2 || mine->thermal_on)
    mine->heat_inv_norm = P.heat_power != 0.0f ? (S > 0 ? (float)(1.0 / S) : 0.0f) : 0.0f;
}

// New particle ids (phase_change.cu:281-335): this slab's splits take the ids
// after those of the slabs before it; every slab advances next_id by the
// total.
__global__ void k_slab_split(DynState* const* dyns, int nslabs, int rank, DynState* mine) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int prefix = 0, total = 0;
  for (int r = 0; r < nslabs; ++r) {
    const int q = dyns[r]->split_requested;
    if (r < rank) prefix += q;
    total += q;
  }
  mine->id_offset = (uint32_t)prefix;
  mine->split_total = total;
}

// The dt maxima over every slab (sph_solver.cu:475-479), after the force
// pass (particle shifting reads v_max in the same step) and at the end of a
// step; with `saturation` also the ullage state from the phase sums of every
// slab (sph_solver.cu:586-607).  Maxima are order-free; a slab that already
// took the maxima of the others holds the same values.
__global__ void k_slab_end(Params P, DynState* const* dyns, int nslabs, DynState* mine, int saturation) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double s[3] = {0.0, 0.0, 0.0};
  float vmax = 0.0f, amax = 0.0f, tv = 0.0f, nut = 0.0f, sr = 0.0f;
  for (int r = 0; r < nslabs; ++r) {
    const DynState* d = dyns[r];
    for (int k = 0; k < 3; ++k) s[k] += d->sat_sum[k];
    vmax = fmaxf(vmax, d->v_max);
    amax = fmaxf(amax, d->a_max);
    tv = fmaxf(tv, d->Tv_max);
    nut = fmaxf(nut, d->nu_t_max);
    sr = fmaxf(sr, d->spacing_ratio);
  }
  if (saturation) saturation_update(P, mine, P.thermo_closed && P.has_vapor, s[0], s[1], s[2]);
  mine->v_max = vmax;
  mine->a_max = amax;
  mine->Tv_max = tv;
  mine->nu_t_max = nut;
  mine->spacing_ratio = sr;
}

// Refresh between steps: dst (the slab's spare particle set, with a4 / ab4
// into a4_out / ab4_out) := [lower slab's top `depth` layers][own range]
// [upper slab's bottom `depth` layers][lower's split children][own split
// children][upper's split children].  Within any cell this keeps the order
// the whole tank's arrays have (sorted ranges in slab order, then the split
// children in slab order), so the next sort puts every particle where the
// whole tank's sort would.  The new count goes to dyn->n_next.
__global__ void __launch_bounds__(kBlock) k_slab_assemble(Params P, View dst, float4* a4_out, float4* ab4_out,
                                                          View lo, View me, View up, int has_lo, int has_up, int zb,
                                                          int ze, int depth) {
  int b[6], e[6];
  b[0] = e[0] = b[2] = e[2] = b[3] = e[3] = b[5] = e[5] = 0;
  if (has_lo) {
    layer_range(P, lo.cell_begin, zb - depth, zb, b[0], e[0]);
    b[3] = lo.dyn->n_sorted;
    e[3] = lo.dyn->n;
  }
  b[1] = me.dyn->own_lo;
  e[1] = me.dyn->own_hi;
  b[4] = me.dyn->n_sorted;
  e[4] = me.dyn->n;
  if (has_up) {
    layer_range(P, up.cell_begin, ze, ze + depth, b[2], e[2]);
    b[5] = up.dyn->n_sorted;
    e[5] = up.dyn->n;
  }
  int start[7];
  start[0] = 0;
  for (int s = 0; s < 6; ++s) start[s + 1] = start[s] + (e[s] > b[s] ? e[s] - b[s] : 0);
  const int total = start[6];
  if (total > dst.capacity) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&dst.dyn->status, (unsigned)CRYO_DEV_SLAB_CAPACITY);
    return;
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    int s = 0;
    while (k >= start[s + 1]) ++s;
    const View& src = (s == 0 || s == 3) ? lo : ((s == 2 || s == 5) ? up : me);
    const int j = b[s] + (k - start[s]);
    dst.xp[k] = src.xp[j];
    dst.vT[k] = src.vT[j];
    dst.vt[k] = src.vt[j];
    dst.nrm[k] = src.nrm[j];
    dst.mrps[k] = src.mrps[j];
    dst.id[k] = src.id[j];
    a4_out[k] = src.a4[j];
    ab4_out[k] = src.ab4[j];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) dst.dyn->n_next = total;
}

// The refreshed set becomes the slab's: a4 / ab4 back from the spare arrays
// and the new count.
__global__ void __launch_bounds__(kBlock) k_slab_commit(View V, const float4* a4_in, const float4* ab4_in) {
  DynState* d = V.dyn;
  if (d->status & CRYO_DEV_SLAB_CAPACITY) return;
  const int n = d->n_next;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    V.a4[k] = a4_in[k];
    V.ab4[k] = ab4_in[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d->n = n;
    d->n_alive = n;
  }
}

}  // namespace cryo
