// cryo_common.cuh -- shared device definitions of the B200 hot path.
//
// Arithmetic: the library is compiled with -fmad=false (no FMA contraction),
// IEEE division and square root, and every expression keeps the evaluation
// order of the CryoSPH reference (paths below are inside that project).  The
// single-precision field arithmetic is therefore the same IEEE operation
// sequence as the reference's CPU build; only libm calls (powf, cosf, sinf,
// cbrtf, log) can differ in the last place.
//
// Data layout (cell-sorted structure of arrays, one slot per particle):
//   persistent, permuted by the reorder gather (two copies, ping-pong):
//     xp   float4  x, y, z, bits(phase | flags << 8)
//     vT   float4  velocity, temperature
//     vt   float4  transport velocity, reference mass m0
//     nrm  float4  normal / colour gradient, alpha (opposite-phase fraction)
//     mrps float4  mass, density, pressure, sigma (number density)
//     id   u32
//   scratch, not permuted (as in the reference, particle_system.hpp:52-72):
//     a4 {a, dTdt}  ab4 {ab, drho}  fw  mw  vwp {vw, p_wv}  ns4 {ns, kappa}
//     pc {out_m, out_h, w_norm, -}  rmin  wall_w  heat_w  nu_t
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cryosph_b200.h"

namespace cryo {

constexpr int kLiquid = 0, kVapor = 1, kWall = 2, kDead = 3;
constexpr int kHeated = 1, kSource = 2, kTargetVapor = 4, kDying = 8, kScratchMask = 2 | 4 | 8;
constexpr float kPi = 3.14159265358979323846f;
constexpr int kBlock = 256;      // threads per block of the particle kernels
constexpr int kChunk = kBlock;   // particles per reduction partial (fixed tree, tank-local)

__host__ __device__ inline bool is_fluid(int ph) { return ph <= kVapor; }
__host__ __device__ inline int phase_index(int ph) { return ph == kVapor ? 1 : 0; }

// ------------------------------------------------------------ vectors
// cuda_utils.cuh:85-108 of the reference; float3 with the same operation order.
struct V3 {
  float x, y, z;
};
__host__ __device__ inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ inline V3& operator+=(V3& a, V3 b) {
  a.x += b.x; a.y += b.y; a.z += b.z;
  return a;
}
__host__ __device__ inline V3& operator-=(V3& a, V3 b) {
  a.x -= b.x; a.y -= b.y; a.z -= b.z;
  return a;
}
__host__ __device__ inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ inline float norm2(V3 a) { return dot(a, a); }
__host__ __device__ inline float norm(V3 a) { return sqrtf(dot(a, a)); }
__host__ __device__ inline V3 normalized(V3 a) {
  const float n = norm(a);
  return n > 1e-20f ? a / n : V3{0, 0, 0};
}
__host__ __device__ inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
__host__ __device__ inline V3 xyz(float4 a) { return {a.x, a.y, a.z}; }
__host__ __device__ inline float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// xp.w packs phase (bits 0-7) and flags (bits 8-15) as integer bits.
__device__ inline int ph_of(float4 xp) { return __float_as_int(xp.w) & 0xff; }
__device__ inline int fl_of(float4 xp) { return (__float_as_int(xp.w) >> 8) & 0xff; }
__host__ __device__ inline float pack_pf(int phase, int flags) {
#if defined(__CUDA_ARCH__)
  return __int_as_float((phase & 0xff) | ((flags & 0xff) << 8));
#else
  union { int i; float f; } u;
  u.i = (phase & 0xff) | ((flags & 0xff) << 8);
  return u.f;
#endif
}

// ------------------------------------------------------------ params
// SimParams (sim_params.cuh:20-95) + KernelParams (SPH_kernels.cuh:15-31) + the
// grid view (spatial_hash.hpp:14-20).  Passed by value to every kernel; the
// values that change during a step live in DynState instead.
struct Params {
  // kernel
  int ktype;
  float h, inv_h, support, knorm;
  float dx, vol0, support2;
  float rho0[2], mu[2], k[2], cp[2], mref[2];
  float c0, tait_B, tait_gamma, p_bg, gas_R, vapor_K;
  int clamp_neg;
  float alpha_av, alpha_av_vap, delta_sph;
  int density_mode, no_slip, sps, tvf, tvf_stress, tvf_interface_only;
  float tvf_factor, tvf_sigma_min, shift_strength, smagorinsky_cs;
  int st_model;
  float sigma, cos_theta, sin_theta, normal_eps, wall_adhesion_weight;
  int wetting_model, wall_colour, csf_smooth, csf_balanced;
  float akinci_gamma, akinci_beta;
  int thermal, phase_change, wall_bc;
  float T_wall, T_ref, h_fg, lee_evap, lee_cond, max_transfer_fraction, vapor_rebalance;
  float pc_density_limit, merge_ratio, split_ratio, heat_power;
  // solver-level switches (SolverConfig fields used inside the step)
  int cfg_phase_change, thermo_closed, has_vapor, csf_active;
  float vent_relaxation;
  // dt limits (sph_solver.cu:482-504)
  float cfl, viscous_number, force_number, capillary_number, thermal_number, dt_max, dt_min, fixed_dt;
  // fluid constants for the ullage model
  float f_rho_l, f_rho_v, f_T_sat, f_p_sat, f_R_gas, f_h_fg;
  // grid
  float ox, oy, oz, inv_cell, cell;
  int nx, ny, nz, num_cells, key_bits;
  // neighbour lists (0: every pass scans the 27 cells)
  int use_lists;
  // 1: this context is one slab of a decomposed tank; the heat normalisation
  // and the ullage state come from the slabs' combined sums
  int slab;
  // cell layers [slab_z0, slab_z1) this context owns (0, nz: the whole tank);
  // the phase index lists hold only the owned particles
  int slab_z0, slab_z1;
};

// Capacity of the per-particle neighbour list; a particle with more
// in-support neighbours falls back to the 27-cell scan.
constexpr int kMaxNbr = 128;
constexpr int kNbrChunk = 8;  // list entries per 32-byte chunk (kMaxNbr is a multiple)

// Device-resident scalar block: everything the host used to keep between
// kernel launches (dt, frame state, maxima, FP64 bookkeeping, counts).
struct DynState {
  // particle counts
  int n;              // current particle count (incl. dead until the next build)
  int n_alive;
  int capacity;
  uint32_t next_id;
  // clock
  double time, last_dt;
  long long step;
  float dt;           // dt of the current step (SimParams::dt)
  // frame (SimParams gravity/omega..., sph_solver.cu:660-667); one contiguous
  // block so the host can replace it with a single asynchronous copy
  struct Frame {
    float gravity[3], omega[3], omega_dot[3], frame_origin[3], frame_acc[3];
    int frame_rot;
    float cfg_gravity[3];
    int has_maneuver;
  } fr;
  // thermodynamics
  float T_sat, heat_inv_norm;
  double p_ullage, fluid_volume0, heat_input;
  // maxima of the last rate evaluation (float bits, atomicMax-able for >= 0)
  float v_max, a_max, Tv_max, nu_t_max, spacing_ratio;
  // cumulative bookkeeping
  double evaporated, condensed, vented, vented_h;
  int merges, splits;
  int n_fluid_list, n_wall_list;  // lengths of the phase index lists
  unsigned status;    // CRYO_DEV_* guard bits
  int split_requested;
  // relax / damping applied after the step (0 = none)
  int damp_after_step;
  float damping;
  int thermal_on;     // SimParams::thermal (relax turns it off)
  int phase_change_on;  // SolverConfig::phase_change (relax turns it off)
  // maneuver
  int man_n, man_rot;
  float man_origin[3];
  // slab decomposition: the sorted range this context owns (0, INT_MAX when
  // it holds the whole tank), the sorted count (split children follow it),
  // and the owned sums the slabs combine
  int own_lo, own_hi, n_sorted;
  uint32_t id_offset;  // this slab's offset into the step's new split ids
  int split_total;     // splits requested by every slab this step
  double heat_sum;     // owned heat weights
  double sat_sum[3];   // owned liquid mass, vapour mass, vapour m T
  int n_next;          // particle count of a refreshed slab
};

// Particle i counts towards this context's global sums and maxima: inside
// its owned sorted range, or a split child appended after the sorted count.
__device__ inline bool owned(int own_lo, int own_hi, int n_sorted, int i) {
  return (i >= own_lo && i < own_hi) || i >= n_sorted;
}


// Solver::compute_dt (sph_solver.cu:482-504); host and device share it so the
// host's next_dt() and the device step agree bit for bit.
__host__ __device__ inline float compute_dt(const Params& P, const DynState& d) {
  if (P.fixed_dt > 0.0f) return P.fixed_dt;
  const float h = P.h;
  float c_max = P.c0;
  auto mx = [](float a, float b) { return (a < b) ? b : a; };  // std::max
  auto mn = [](float a, float b) { return (b < a) ? b : a; };  // std::min
  if (P.has_vapor) c_max = mx(c_max, sqrtf(P.gas_R * mx(d.Tv_max, P.T_ref)));
  float dt = P.cfl * h / ((c_max + d.v_max) * mx(1.0f, d.spacing_ratio));
  const float nu = mx(P.mu[0] / P.rho0[0], P.mu[1] / P.rho0[1]) + d.nu_t_max;
  if (nu > 0.0f) dt = mn(dt, P.viscous_number * h * h / nu);
  if (d.a_max > 0.0f) dt = mn(dt, P.force_number * sqrtf(h / d.a_max));
  if (P.sigma > 0.0f) {
    const float rho_avg = 0.5f * (P.rho0[0] + (P.has_vapor ? P.rho0[1] : P.rho0[0]));
    dt = mn(dt, P.capillary_number * sqrtf(rho_avg * h * h * h / (2.0f * kPi * P.sigma)));
  }
  if (d.thermal_on) {
    float alpha = P.k[0] / (P.rho0[0] * P.cp[0]);
    if (P.has_vapor) alpha = mx(alpha, P.k[1] / (P.rho0[1] * P.cp[1]));
    if (alpha > 0.0f) dt = mn(dt, P.thermal_number * h * h / alpha);
  }
  return dt < P.dt_min ? P.dt_min : (P.dt_max < dt ? P.dt_max : dt);  // std::clamp
}

// Pointers a kernel may touch (the current persistent copy + scratch).
struct View {
  float4 *xp, *vT, *vt, *nrm, *mrps;
  uint32_t* id;
  float4 *a4, *ab4, *fw, *mw, *vwp, *ns4, *pc;
  float *rmin, *wall_w, *heat_w, *nu_t;
  // per fluid particle {m/rho, 1/sigma, sound speed, 0}: the neighbour
  // passes' per-pair volume factors, evaluated once per particle with the
  // same operations (written by the density pass, valid until the kick)
  float4* aux;
  const int* cell_begin;  // dense cell prefix table, num_cells + 1 entries
  uint8_t* cell_fluid;    // per cell: 1 if a fluid particle was sorted into it (lists mode)
  DynState* dyn;
  // maneuver table
  const double* man_t;
  const float* man_acc;
  const float* man_omega;
  // reduction workspace
  double* partials;   // per-chunk FP64 partials
  unsigned* counters; // last-block tickets
  int capacity;
  // neighbour lists, in chunks of kNbrChunk: the k-th in-support neighbour
  // of i (reference iteration order) is nbr[((k / 8) * capacity + i) * 8 +
  // k % 8], so one particle's chunk is one 32-byte sector and a warp's
  // chunks are contiguous; nbr_cnt[i] = count (> kMaxNbr: overflow)
  int* nbr;
  int* nbr_cnt;
  // ordered phase index lists (built after each reorder)
  int* fluid_idx;
  int* wall_idx;
  // Only while a differentiated window is recomputed (null otherwise): the
  // force and interface sums the reverse sweep reads, 6 arrays of tape_n
  // records (force pass: rows 0-2, interface pass: rows 3-5).
  float4* tape;
  int tape_n;
};

// --------------------------------------------------------- SPH kernels
// Single-precision pow, cos, sin and cbrt as the reference's CPU build gets
// them: from the C library, which returns the correctly rounded value for
// nearly every argument (all but ~2e-4 of the powf and ~1e-2 of the cosf /
// sinf arguments these passes see; cbrtf misses more often).  These device
// versions take the correctly rounded value from the double-precision
// function (CUDA's single-precision versions are within 2 ulp).  The force
// pass keeps CUDA's powf for the transport-velocity wall volume: the double
// code inlined there cost the whole pass 20 % (registers), and that path
// matched the library no less often in the runs compared.
__host__ __device__ inline float pow_cr(float x, float y) {
#ifdef __CUDA_ARCH__
  return (float)pow((double)x, (double)y);
#else
  return powf(x, y);
#endif
}
__device__ inline float cos_cr(float x) { return (float)cos((double)x); }
__device__ inline float sin_cr(float x) { return (float)sin((double)x); }
__device__ inline float cbrt_cr(float x) { return (float)cbrt((double)x); }

// kernel_W / kernel_dWdr / kernel_gradW (SPH_kernels.cuh:34-64)
__host__ __device__ inline float kernel_W(const Params& P, float r) {
  const float q = r * P.inv_h;
  if (q >= 2.0f) return 0.0f;
  if (P.ktype == CRYO_KERNEL_CUBIC) {
    if (q < 1.0f) return P.knorm * (1.0f - 1.5f * q * q + 0.75f * q * q * q);
    const float t = 2.0f - q;
    return P.knorm * 0.25f * t * t * t;
  }
  const float t = 1.0f - 0.5f * q;
  const float t2 = t * t;
  return P.knorm * t2 * t2 * (2.0f * q + 1.0f);
}
__host__ __device__ inline float kernel_dWdr(const Params& P, float r) {
  const float q = r * P.inv_h;
  if (q >= 2.0f) return 0.0f;
  if (P.ktype == CRYO_KERNEL_CUBIC) {
    if (q < 1.0f) return P.knorm * P.inv_h * (-3.0f * q + 2.25f * q * q);
    const float t = 2.0f - q;
    return P.knorm * P.inv_h * -0.75f * t * t;
  }
  const float t = 1.0f - 0.5f * q;
  return P.knorm * P.inv_h * -5.0f * q * t * t * t;
}
__device__ inline V3 kernel_gradW(const Params& P, V3 rij, float r) {
  if (r <= 1e-12f * P.h) return V3{0, 0, 0};
  return rij * (kernel_dWdr(P, r) / r);
}
// Akinci splines (SPH_kernels.cuh:69-86)
__host__ __device__ inline float akinci_cohesion(float r, float c) {
  if (r >= c || r <= 0.0f) return 0.0f;
  const float c3 = c * c * c;
  const float c9 = c3 * c3 * c3;
  const float coeff = 32.0f / (kPi * c9);
  const float t = (c - r);
  const float base = t * t * t * r * r * r;
  if (2.0f * r > c) return coeff * base;
  return coeff * (2.0f * base - c3 * c3 / 64.0f);
}
__host__ __device__ inline float akinci_adhesion(float r, float c) {
  if (r >= c || 2.0f * r <= c) return 0.0f;
  const float arg = -4.0f * r * r / c + 6.0f * r - 2.0f * c;
  if (arg <= 0.0f) return 0.0f;
  return 0.007f / pow_cr(c, 3.25f) * pow_cr(arg, 0.25f);
}

// EOS and enthalpy (sim_params.cuh:100-135)
__device__ inline float eos_pressure(const Params& P, int ph, float rho, float T) {
  float p;
  if (ph == kVapor) {
    p = rho * P.gas_R * T + (P.p_bg - P.vapor_K);
  } else {
    // IEEE division in either field arithmetic: the Tait form takes 1 off
    // ratio^7, so a last-place error of the ratio would be amplified by
    // 7 / (ratio^7 - 1) in the pressure of a liquid near rest
    const float ratio = __fdiv_rn(rho, P.rho0[0]);
    float r_g;
    if (P.tait_gamma == 7.0f) {
      const float r2 = ratio * ratio;
      r_g = r2 * r2 * r2 * ratio;
    } else {
      r_g = pow_cr(ratio, P.tait_gamma);
    }
    p = P.tait_B * (r_g - 1.0f) + P.p_bg;
  }
  return (P.clamp_neg && p < 0.0f) ? 0.0f : p;
}
__device__ inline float sound_speed(const Params& P, int ph, float T) {
  if (ph == kVapor) return sqrtf(P.gas_R * (T > 0.0f ? T : 0.0f));
  return P.c0;
}
__device__ inline float specific_enthalpy(const Params& P, int ph, float T) {
  return ph == kVapor ? P.h_fg + P.cp[1] * (T - P.T_ref) : P.cp[0] * (T - P.T_ref);
}
__device__ inline float temperature_from_enthalpy(const Params& P, int ph, float h) {
  return ph == kVapor ? P.T_ref + (h - P.h_fg) / P.cp[1] : P.T_ref + h / P.cp[0];
}

// ------------------------------------------------------- grid helpers
// float -> int as the reference's static_cast<int> executes on x86-64
// (cvttss2si): NaN and out-of-range values give INT_MIN.
__device__ inline int to_int_trunc(float f) {
  return (f >= 2147483648.0f || f < -2147483648.0f || f != f) ? (int)0x80000000 : __float2int_rz(f);
}
// grid_cell_coords (spatial_hash.hpp:22-26)
__device__ inline void cell_coords(const Params& P, V3 p, int& cx, int& cy, int& cz) {
  cx = min(max(to_int_trunc(floorf((p.x - P.ox) * P.inv_cell)), 0), P.nx - 1);
  cy = min(max(to_int_trunc(floorf((p.y - P.oy) * P.inv_cell)), 0), P.ny - 1);
  cz = min(max(to_int_trunc(floorf((p.z - P.oz) * P.inv_cell)), 0), P.nz - 1);
}
__device__ inline int cell_index(const Params& P, V3 p) {
  int cx, cy, cz;
  cell_coords(P, p, cx, cy, cz);
  return (cz * P.ny + cy) * P.nx + cx;
}

// The 27-cell visit of particle position xi, narrowed without changing what
// it finds: a (y, z) row of cells whose slab lies beyond the support radius
// is skipped, and a row's side cells (x -+ 1) are dropped likewise.  Gaps
// are measured to the faces of xi's own cell, pulled in by a margin that
// covers the rounding of the cell index (1e-3 of a cell plus 1e-6 per cell
// of grid extent), so every particle within the support is still visited;
// particles clamped into a boundary cell from outside the grid lie beyond
// the face too.  Visit order and accepted set equal the full scan's.
struct CellWindow {
  int cx, cy, cz, x0, x1, y0, y1, z0, z1;
  float glo[3], ghi[3];  // gaps from xi to its own cell's faces, less the margin
  __device__ CellWindow(const Params& P, V3 xi) {
    cell_coords(P, xi, cx, cy, cz);
    z0 = cz > 0 ? cz - 1 : 0; z1 = cz < P.nz - 1 ? cz + 1 : cz;
    y0 = cy > 0 ? cy - 1 : 0; y1 = cy < P.ny - 1 ? cy + 1 : cy;
    x0 = cx > 0 ? cx - 1 : 0; x1 = cx < P.nx - 1 ? cx + 1 : cx;
    const float eps = P.cell * (1e-3f + 1e-6f * (float)(P.nx + P.ny + P.nz));
    const float o[3] = {P.ox, P.oy, P.oz}, x[3] = {xi.x, xi.y, xi.z};
    const int c[3] = {cx, cy, cz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float face = o[a] + (float)c[a] * P.cell;
      glo[a] = fmaxf(x[a] - face - eps, 0.0f);
      ghi[a] = fmaxf(face + P.cell - x[a] - eps, 0.0f);
    }
  }
  // Cells [xs, xe] of row (y, z) that can hold a neighbour; false: none.
  __device__ bool row(const Params& P, int y, int z, int& xs, int& xe) const {
    const float gy = y < cy ? glo[1] : (y > cy ? ghi[1] : 0.0f);
    const float gz = z < cz ? glo[2] : (z > cz ? ghi[2] : 0.0f);
    const float g2 = gy * gy + gz * gz;
    if (g2 >= P.support2) return false;
    xs = x0;
    xe = x1;
    if (x0 < cx && glo[0] * glo[0] + g2 >= P.support2) xs = cx;
    if (x1 > cx && ghi[0] * ghi[0] + g2 >= P.support2) xe = cx;
    return true;
  }
};

// Neighbour iteration (spatial_hash.hpp:37-56).  Cells are key-sorted, so the
// three x-neighbouring cells of one (y, z) row are one contiguous index range;
// the 27-cell visit becomes at most 9 ranges in the reference's z, y, x, j
// order (CellWindow drops the parts that cannot hold a neighbour).
// f(j, xj, rij, r2) is called for every j with r2 < support^2 (self included),
// r2 evaluated as ((dx*dx + dy*dy) + dz*dz) exactly as norm2() does.
template <class F>
__device__ inline void for_each_neighbor(const Params& P, const int* __restrict__ cell_begin,
                                         const float4* __restrict__ xp, V3 xi, F&& f) {
  const CellWindow W(P, xi);
  for (int z = W.z0; z <= W.z1; ++z) {
    for (int y = W.y0; y <= W.y1; ++y) {
      int xs, xe;
      if (!W.row(P, y, z, xs, xe)) continue;
      const int row = (z * P.ny + y) * P.nx;
      const int s = __ldg(cell_begin + row + xs);
      const int e = __ldg(cell_begin + row + xe + 1);
      for (int j = s; j < e; ++j) {
        const float4 xj = __ldg(xp + j);
        const V3 rij = xi - xyz(xj);
        const float r2 = norm2(rij);
        if (r2 >= P.support2) continue;
        f(j, xj, rij, r2);
      }
    }
  }
}

// Neighbour iteration of particle i through its list (same j order and the
// same r2 bits as for_each_neighbor); falls back to the scan on overflow or
// when lists are off.
// UNROLL = 2 lets the compiler interleave two neighbours' work (the
// heaviest force-pass variants gain from it at a million particles).
template <int UNROLL = 1, class F>
__device__ inline void for_each_nbr(const Params& P, const View& V, int i, V3 xi, F&& f) {
  const int c = P.use_lists ? __ldg(V.nbr_cnt + i) : kMaxNbr + 1;
  if (c <= kMaxNbr) {
    // the list is read 4 indices (16 bytes) at a time, the next 4 already in
    // flight; the next neighbour's position is in flight while the current
    // one is processed
    const int4* __restrict__ base = reinterpret_cast<const int4*>(V.nbr + (size_t)i * kNbrChunk);
    const size_t cstride = (size_t)V.capacity * (kNbrChunk / 4);  // chunk stride in int4
    auto quad = [&](int q) { return __ldg(base + (size_t)(q >> 1) * cstride + (q & 1)); };
    int4 cur = c > 0 ? quad(0) : make_int4(0, 0, 0, 0);
    int4 nxt = c > 4 ? quad(1) : make_int4(0, 0, 0, 0);
    int jn = cur.x;
    float4 xn = c > 0 ? __ldg(V.xp + jn) : make_float4(0, 0, 0, 0);
#pragma unroll UNROLL
    for (int k = 0; k < c; ++k) {
      const int j = jn;
      const float4 xj = xn;
      cur.x = cur.y; cur.y = cur.z; cur.z = cur.w;
      if (((k + 1) & 3) == 0) {
        cur = nxt;
        if (k + 5 < c) nxt = quad(((k + 1) >> 2) + 1);
      }
      if (k + 1 < c) {
        jn = cur.x;
        xn = __ldg(V.xp + jn);
      }
      const V3 rij = xi - xyz(xj);
      const float r2 = norm2(rij);
      f(j, xj, rij, r2);
    }
  } else {
    for_each_neighbor(P, V.cell_begin, V.xp, xi, f);
  }
}

// for_each_nbr for passes with little work per neighbour: the loop takes
// each loaded quad of indices whole (its four entries at fixed positions, no
// shifting), with one reload test per four neighbours; the next neighbour's
// position is in flight while the current one is processed, as in
// for_each_nbr, and the order and the r2 bits are the same.
template <class F>
__device__ inline void for_each_nbr_quads(const Params& P, const View& V, int i, V3 xi, F&& f) {
  const int c = P.use_lists ? __ldg(V.nbr_cnt + i) : kMaxNbr + 1;
  if (c <= kMaxNbr) {
    const int4* __restrict__ base = reinterpret_cast<const int4*>(V.nbr + (size_t)i * kNbrChunk);
    const size_t cstride = (size_t)V.capacity * (kNbrChunk / 4);
    auto quad = [&](int q) { return __ldg(base + (size_t)(q >> 1) * cstride + (q & 1)); };
    int4 cur = c > 0 ? quad(0) : make_int4(0, 0, 0, 0);
    int4 nxt = c > 4 ? quad(1) : make_int4(0, 0, 0, 0);
    float4 xn = c > 0 ? __ldg(V.xp + cur.x) : make_float4(0, 0, 0, 0);
    for (int k0 = 0; k0 < c; k0 += 4) {
      const int js[4] = {cur.x, cur.y, cur.z, cur.w};
      const int next0 = nxt.x;  // the first entry of the next quad
      cur = nxt;
      if (k0 + 8 < c) nxt = quad((k0 >> 2) + 2);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (k0 + u < c) {
          const int j = js[u];
          const float4 xj = xn;
          if (k0 + u + 1 < c) xn = __ldg(V.xp + (u < 3 ? js[u + 1] : next0));
          const V3 rij = xi - xyz(xj);
          const float r2 = norm2(rij);
          f(j, xj, rij, r2);
        }
      }
    }
  } else {
    for_each_neighbor(P, V.cell_begin, V.xp, xi, f);
  }
}

// for_each_nbr that also brings each neighbour's record of `A` (one float4
// per particle) along with its position, one neighbour ahead, so that load
// is in flight while the previous neighbour is processed: f(j, xj, rij, r2, aj).
template <class F>
__device__ inline void for_each_nbr_pf(const Params& P, const View& V, int i, V3 xi,
                                       const float4* __restrict__ A, F&& f) {
  const int c = P.use_lists ? __ldg(V.nbr_cnt + i) : kMaxNbr + 1;
  if (c <= kMaxNbr) {
    const int4* __restrict__ base = reinterpret_cast<const int4*>(V.nbr + (size_t)i * kNbrChunk);
    const size_t cstride = (size_t)V.capacity * (kNbrChunk / 4);
    auto quad = [&](int q) { return __ldg(base + (size_t)(q >> 1) * cstride + (q & 1)); };
    int4 cur = c > 0 ? quad(0) : make_int4(0, 0, 0, 0);
    int4 nxt = c > 4 ? quad(1) : make_int4(0, 0, 0, 0);
    int jn = cur.x;
    float4 xn = c > 0 ? __ldg(V.xp + jn) : make_float4(0, 0, 0, 0);
    float4 an = c > 0 ? __ldg(A + jn) : make_float4(0, 0, 0, 0);
    for (int k = 0; k < c; ++k) {
      const int j = jn;
      const float4 xj = xn, aj = an;
      cur.x = cur.y; cur.y = cur.z; cur.z = cur.w;
      if (((k + 1) & 3) == 0) {
        cur = nxt;
        if (k + 5 < c) nxt = quad(((k + 1) >> 2) + 1);
      }
      if (k + 1 < c) {
        jn = cur.x;
        xn = __ldg(V.xp + jn);
        an = __ldg(A + jn);
      }
      const V3 rij = xi - xyz(xj);
      const float r2 = norm2(rij);
      f(j, xj, rij, r2, aj);
    }
  } else {
    for_each_neighbor(P, V.cell_begin, V.xp, xi,
                      [&](int j, float4 xj, V3 rij, float r2) { f(j, xj, rij, r2, __ldg(A + j)); });
  }
}

// The particles a pass visits: with lists, an ordered phase index list
// (fluid or wall); otherwise every particle (the pass filters by phase).
struct Range {
  const int* idx;
  int count;
};
__device__ inline int particle_at(const Range& r, int t) { return r.idx ? __ldg(r.idx + t) : t; }
// Sorted index range of the owned cell layers (after the cell table is built).
__device__ inline void owned_layers(const Params& P, const int* cell_begin, int& lo, int& hi) {
  const int L = P.nx * P.ny;
  lo = __ldg(cell_begin + P.slab_z0 * L);
  hi = __ldg(cell_begin + P.slab_z1 * L);
}
__device__ inline Range fluid_range(const Params& P, const View& V) {
  return P.use_lists ? Range{V.fluid_idx, V.dyn->n_fluid_list} : Range{nullptr, V.dyn->n};
}
__device__ inline Range wall_range(const Params& P, const View& V) {
  return P.use_lists ? Range{V.wall_idx, V.dyn->n_wall_list} : Range{nullptr, V.dyn->n};
}

// Same iteration, every candidate (no distance filter); for passes whose
// filter order matters only for speed.
template <class F>
__device__ inline void for_each_candidate(const Params& P, const int* __restrict__ cell_begin, V3 xi, F&& f) {
  int cx, cy, cz;
  cell_coords(P, xi, cx, cy, cz);
  const int z0 = cz > 0 ? cz - 1 : 0, z1 = cz < P.nz - 1 ? cz + 1 : cz;
  const int y0 = cy > 0 ? cy - 1 : 0, y1 = cy < P.ny - 1 ? cy + 1 : cy;
  const int x0 = cx > 0 ? cx - 1 : 0, x1 = cx < P.nx - 1 ? cx + 1 : cx;
  for (int z = z0; z <= z1; ++z)
    for (int y = y0; y <= y1; ++y) {
      const int row = (z * P.ny + y) * P.nx;
      const int s = __ldg(cell_begin + row + x0);
      const int e = __ldg(cell_begin + row + x1 + 1);
      for (int j = s; j < e; ++j) f(j);
    }
}

// ------------------------------------------------------- reductions
// Warp / block sums in a fixed tree (deterministic).
__device__ inline double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
// kick_drift (sph_solver.cu:20-34)
__device__ inline void kick_drift_one(const Params& P, const View& V, int i, float dt, int continuity, int tvf,
                                      float4& xp) {
  const float half = 0.5f * dt;
  float4 vT = V.vT[i];
  const V3 v = xyz(vT) + xyz(V.a4[i]) * half;
  V.vT[i] = f4(v, vT.w);
  float4 vt4 = V.vt[i];
  const V3 vt = tvf ? v + xyz(V.ab4[i]) * half : v;
  V.vt[i] = f4(vt, vt4.w);
  const V3 x = xyz(xp) + vt * dt;
  xp.x = x.x;
  xp.y = x.y;
  xp.z = x.z;
  V.xp[i] = xp;
  if (continuity) {
    float* mr = reinterpret_cast<float*>(V.mrps + i);
    mr[1] += V.ab4[i].w * dt;
  }
}

// atomicMax on non-negative floats through their (order-preserving) bits.
__device__ inline void atomic_max_pos(float* addr, float v) {
  if (v > 0.0f) atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

// Neumaier-compensated sequential sum of a double array (fixed order).
__device__ inline double compensated_sum(const double* a, int n, int stride) {
  double s = 0, c = 0;
  for (int k = 0; k < n; ++k) {
    const double x = a[(size_t)k * stride];
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  return s + c;
}

}  // namespace cryo
