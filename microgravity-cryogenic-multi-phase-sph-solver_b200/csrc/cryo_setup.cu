// cryo_setup.cu -- the tank lattice generator on the device
// (build_tank_particles, geometry.cpp:242-330): signed distances of the tank
// geometry at every lattice node, ordered compaction of wall and fluid nodes,
// the liquid/vapour split at an order statistic of the fill key, and the
// particles written into the solver's arrays.  The signed distances come from
// cryo_sdf.h, which the host generator evaluates too, so the particles are
// identical to the host's.
#include "cryo_kernels.cuh"
#include "cryo_sdf.h"

namespace cryo {

namespace {

// Geometry::sdf of the node tree (the analytic shapes and their CSG).  Nodes
// come children first; a primitive is evaluated at the query point shifted
// by the offsets of its Translated ancestors, root first, as nested calls to
// the host classes shift it.  The primitives are cryo_sdf.h's, which the host
// classes evaluate too.
__device__ double geom_sdf(const GeomNode* __restrict__ G, int ng, double x, double y, double z) {
  double val[kGeomNodes];
  for (int k = 0; k < ng; ++k) {
    const GeomNode& g = G[k];
    double v = 0.0;
    if (g.kind <= CRYO_GEOM_BOX) {
      double qx = x, qy = y, qz = z;
      for (int f = 0; f < g.nofs; ++f) {
        qx = qx - g.ofs[f][0];
        qy = qy - g.ofs[f][1];
        qz = qz - g.ofs[f][2];
      }
      switch (g.kind) {
        case CRYO_GEOM_CYLINDER: v = cryo_sdf::cylinder(qx, qy, qz, g.p[0], g.p[1]); break;
        case CRYO_GEOM_CAPSULE: v = cryo_sdf::capsule(qx, qy, qz, g.p[0], g.p[1]); break;
        case CRYO_GEOM_SPHERE: v = cryo_sdf::sphere(qx, qy, qz, g.p[0]); break;
        default: v = cryo_sdf::box(qx, qy, qz, g.p[0], g.p[1], g.p[2]); break;
      }
    } else if (g.kind == CRYO_GEOM_TRANSLATED) {
      v = val[g.a];
    } else if (g.kind == CRYO_GEOM_DIFFERENCE) {
      v = cryo_sdf::subtract(val[g.a], val[g.b]);
    } else {  // CRYO_GEOM_UNION
      v = cryo_sdf::unite(val[g.a], val[g.b]);
    }
    val[k] = v;
  }
  return val[ng - 1];
}

__device__ inline void node_xyz(const Lattice& L, long long t, double& x, double& y, double& z) {
  const long long nxy = (long long)L.nx * L.ny;
  const int k = (int)(t / nxy);
  const long long r = t - (long long)k * nxy;
  const int j = (int)(r / L.nx), i = (int)(r - (long long)j * L.nx);
  x = (L.i0 + i + 0.5) * L.h;
  y = (L.j0 + j + 0.5) * L.h;
  z = (L.k0 + k + 0.5) * L.h;
}

// Order-preserving unsigned image of a float key.
__device__ inline uint32_t float_order(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
// The fill key (geometry.cpp:309-313): dot(x, g) for a settled fill, the
// distance to the bubble centre otherwise, in single precision.
__device__ inline float fill_key(const FillDev& F, float px, float py, float pz) {
  if (F.mode == CRYO_FILL_SETTLED) return px * F.g[0] + py * F.g[1] + pz * F.g[2];
  const float dx = px - F.c[0], dy = py - F.c[1], dz = pz - F.c[2];
  return sqrtf(dx * dx + dy * dy + dz * dz);
}

}  // namespace

// Per node: 1 = fluid (sdf < 0), 2 = wall (sdf < band), 0 = outside; block b
// (one node per thread) counts its fluid and wall nodes.
__global__ void __launch_bounds__(kBlock) k_lattice_classify(const GeomNode* __restrict__ G, int ng, Lattice L,
                                                             uint8_t* __restrict__ cls, uint32_t* __restrict__ cnt_f,
                                                             uint32_t* __restrict__ cnt_w) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  if (t < L.total) {
    double x, y, z;
    node_xyz(L, t, x, y, z);
    const double d = geom_sdf(G, ng, x, y, z);
    c = d < 0 ? 1 : (d < L.band ? 2 : 0);
    cls[t] = (uint8_t)c;
  }
  const int nf = __syncthreads_count(c == 1), nw = __syncthreads_count(c == 2);
  if (threadIdx.x == 0) {
    cnt_f[blockIdx.x] = (uint32_t)nf;
    cnt_w[blockIdx.x] = (uint32_t)nw;
  }
}

// Exclusive scan of n block counts in place by one block of 1024 threads;
// *total = their sum.
__global__ void __launch_bounds__(1024) k_scan_counts(uint32_t* __restrict__ cnt, int n,
                                                      unsigned long long* __restrict__ total) {
  __shared__ unsigned long long wsum[32];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < n; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const unsigned long long v = i < n ? cnt[i] : 0ull;
    unsigned long long x = v;  // inclusive scan over the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      unsigned long long w = lane < nw ? wsum[lane] : 0ull;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      if (lane < nw) wsum[lane] = w;  // inclusive over the warps
    }
    __syncthreads();
    const unsigned long long before = carry + (warp > 0 ? wsum[warp - 1] : 0ull) + (x - v);
    if (i < n) cnt[i] = (uint32_t)before;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// Ordered compaction: the indices of the fluid and of the wall nodes in
// lattice order, at the block's offset plus the rank inside the block.
__global__ void __launch_bounds__(kBlock) k_lattice_scatter(Lattice L, const uint8_t* __restrict__ cls,
                                                            const uint32_t* __restrict__ off_f,
                                                            const uint32_t* __restrict__ off_w,
                                                            long long* __restrict__ fluid_nodes,
                                                            long long* __restrict__ wall_nodes) {
  __shared__ int wf[kBlock / 32], ww[kBlock / 32];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = t < L.total ? cls[t] : 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned bf = __ballot_sync(0xffffffffu, c == 1), bw = __ballot_sync(0xffffffffu, c == 2);
  if (lane == 0) {
    wf[warp] = __popc(bf);
    ww[warp] = __popc(bw);
  }
  __syncthreads();
  int pf = 0, pw = 0;
  for (int w = 0; w < warp; ++w) {
    pf += wf[w];
    pw += ww[w];
  }
  const unsigned lt = (1u << lane) - 1u;
  if (c == 1) fluid_nodes[off_f[blockIdx.x] + pf + __popc(bf & lt)] = t;
  if (c == 2) wall_nodes[off_w[blockIdx.x] + pw + __popc(bw & lt)] = t;
}

__global__ void __launch_bounds__(kBlock) k_fill_keys(Lattice L, FillDev F, const long long* __restrict__ fluid_nodes,
                                                      int nf, uint32_t* __restrict__ keys) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nf; q += gridDim.x * blockDim.x) {
    double x, y, z;
    node_xyz(L, fluid_nodes[q], x, y, z);
    keys[q] = float_order(fill_key(F, (float)x, (float)y, (float)z));
  }
}

// Histogram of the 8-bit digit at `shift` over the keys whose bits above it
// equal `prefix` (one pass of a radix selection of an order statistic).
__global__ void __launch_bounds__(kBlock) k_key_digits(const uint32_t* __restrict__ keys, int n, uint32_t prefix,
                                                       uint32_t mask, int shift, unsigned int* __restrict__ hist) {
  __shared__ unsigned int h[256];
  for (int k = threadIdx.x; k < 256; k += blockDim.x) h[k] = 0;
  __syncthreads();
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const uint32_t u = keys[q];
    if ((u & mask) == prefix) atomicAdd(&h[(u >> shift) & 0xffu], 1u);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 256; k += blockDim.x)
    if (h[k]) atomicAdd(&hist[k], h[k]);
}

// Liquid flag of each fluid node, key >= cut (geometry.cpp:318-321), and the
// per-block counts of the nodes kept (liquid, or vapour when it is
// included) and of the liquid ones.
__global__ void __launch_bounds__(kBlock) k_fill_split(Lattice L, FillDev F, const long long* __restrict__ fluid_nodes,
                                                       int nf, uint8_t* __restrict__ liquid,
                                                       uint32_t* __restrict__ cnt_keep, uint32_t* __restrict__ cnt_liq) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  int keep = 0, is_liq = 0;
  if (q < nf) {
    int liq = 1;
    if (F.mode != CRYO_FILL_FULL) {
      double x, y, z;
      node_xyz(L, fluid_nodes[q], x, y, z);
      liq = F.any_liquid && (double)fill_key(F, (float)x, (float)y, (float)z) >= F.cut;
    }
    liquid[q] = (uint8_t)liq;
    keep = liq || F.include_vapor;
    is_liq = liq;
  }
  const int k = __syncthreads_count(keep), l = __syncthreads_count(is_liq);
  if (threadIdx.x == 0) {
    cnt_keep[blockIdx.x] = (uint32_t)k;
    cnt_liq[blockIdx.x] = (uint32_t)l;
  }
}

// The particles in HostParticles::push order: walls [0, nw) in lattice
// order, then the kept fluid nodes in lattice order; id = position.
__global__ void __launch_bounds__(kBlock) k_emit_walls(const GeomNode* __restrict__ G, int ng, Lattice L, FillDev F,
                                                       const long long* __restrict__ wall_nodes, int nw, View V) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
    double x, y, z;
    node_xyz(L, wall_nodes[w], x, y, z);
    // Geometry::outward_normal: central differences at half a lattice step
    const double e = 0.5 * L.h;
    const double gx = geom_sdf(G, ng, x + e, y, z) - geom_sdf(G, ng, x - e, y, z);
    const double gy = geom_sdf(G, ng, x, y + e, z) - geom_sdf(G, ng, x, y - e, z);
    const double gz = geom_sdf(G, ng, x, y, z + e) - geom_sdf(G, ng, x, y, z - e);
    const double n = sqrt(gx * gx + gy * gy + gz * gz);
    float nx = 0.0f, ny = 0.0f, nz = 0.0f;
    if (!(n < 1e-300)) {
      nx = (float)(gx / n);
      ny = (float)(gy / n);
      nz = (float)(gz / n);
    }
    const bool heated = z >= F.heater_zmin && z <= F.heater_zmax;
    V.xp[w] = make_float4((float)x, (float)y, (float)z, pack_pf(kWall, heated ? kHeated : 0));
    V.vT[w] = make_float4(0.0f, 0.0f, 0.0f, F.T_wall);
    V.vt[w] = make_float4(0.0f, 0.0f, 0.0f, F.m_liq);
    V.nrm[w] = make_float4(-nx, -ny, -nz, 0.0f);
    V.mrps[w] = make_float4(F.m_liq, F.rho_liq, 0.0f, 0.0f);
    V.id[w] = (uint32_t)w;
  }
}
__global__ void __launch_bounds__(kBlock) k_emit_fluid(Lattice L, FillDev F, const long long* __restrict__ fluid_nodes,
                                                       int nf, const uint8_t* __restrict__ liquid,
                                                       const uint32_t* __restrict__ off_keep, int nw, View V) {
  __shared__ int wk[kBlock / 32];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int liq = q < nf ? liquid[q] : 0;
  const int keep = q < nf && (liq || F.include_vapor);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned b = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) wk[warp] = __popc(b);
  __syncthreads();
  int p = 0;
  for (int w = 0; w < warp; ++w) p += wk[w];
  if (!keep) return;
  const int o = nw + (int)off_keep[blockIdx.x] + p + __popc(b & ((1u << lane) - 1u));
  double x, y, z;
  node_xyz(L, fluid_nodes[q], x, y, z);
  const float m = liq ? F.m_liq : F.m_vap, rho = liq ? F.rho_liq : F.rho_vap, T = liq ? F.T_liq : F.T_vap;
  V.xp[o] = make_float4((float)x, (float)y, (float)z, pack_pf(liq ? kLiquid : kVapor, 0));
  V.vT[o] = make_float4(0.0f, 0.0f, 0.0f, T);
  V.vt[o] = make_float4(0.0f, 0.0f, 0.0f, m);
  V.nrm[o] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  V.mrps[o] = make_float4(m, rho, 0.0f, 0.0f);
  V.id[o] = (uint32_t)o;
}

// Seeded jitter of the fluid lattice (liquid and vapour; walls stay on the
// lattice): every coordinate moves by amplitude * (2u - 1), u uniform in
// [0, 1) with 24 bits, drawn by a counter-based generator from (seed,
// particle id, axis): the SplitMix64 output function (S. Vigna, "Further
// scramblings of Marsaglia's xorshift generators", 2017) of
// seed + (3 id + axis + 1) * 0x9E3779B97F4A7C15.  The draw depends on the
// id, not on the slot, so it is the same whatever order the particles are in,
// and a host restatement (cryo_cabi.jitter_offsets) reproduces it bit for bit.
__device__ inline float jitter_unit(uint64_t seed, uint32_t id, int axis) {
  uint64_t z = seed + (3ull * id + (uint64_t)axis + 1ull) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (float)(uint32_t)(z >> 40) * (1.0f / 16777216.0f);
}
__global__ void __launch_bounds__(kBlock) k_jitter_fluid(View V, int n, float amplitude, uint64_t seed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 xp = V.xp[i];
    if (!is_fluid(ph_of(xp))) continue;
    const uint32_t id = V.id[i];
    xp.x = xp.x + amplitude * (2.0f * jitter_unit(seed, id, 0) - 1.0f);
    xp.y = xp.y + amplitude * (2.0f * jitter_unit(seed, id, 1) - 1.0f);
    xp.z = xp.z + amplitude * (2.0f * jitter_unit(seed, id, 2) - 1.0f);
    V.xp[i] = xp;
  }
}

}  // namespace cryo
