/*
 * cryo_oracle.c -- plain-C restatement of the CryoSPH per-step particle hot
 * path (TEST INFRASTRUCTURE ONLY; see cryo_oracle.h).
 *
 * Every function restates one reference function; the citation in front of it
 * names the file:line it follows (paths inside the CryoSPH-CUDA project).  The
 * arithmetic keeps the reference's single-precision evaluation order and is
 * compiled with -ffp-contract=off, so with one OpenMP thread on the reference
 * side the two agree bit for bit.  Loops run serially in index order, which
 * equals the reference's parallel_for because no pass reads what another
 * iteration of the same pass writes.
 */
#include "cryo_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef float real;
typedef struct { real x, y, z; } V3;

static const real kPi = (real)3.14159265358979323846;

/* ------------------------------------------------------------ Vec3 ops
 * cuda_utils.cuh:85-108 */
static inline V3 v3(real x, real y, real z) { V3 r = {x, y, z}; return r; }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vneg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline V3 vmul(V3 a, real s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vdiv(V3 a, real s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline real vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 vcross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline real vnorm2(V3 a) { return vdot(a, a); }
static inline real vnorm(V3 a) { return sqrtf(vdot(a, a)); }
static inline V3 vnormalized(V3 a) {
  const real n = vnorm(a);
  return n > (real)1e-20 ? vdiv(a, n) : v3(0, 0, 0);
}
static inline real clampf(real v, real lo, real hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline real maxf(real a, real b) { return (a < b) ? b : a; } /* std::max */
static inline real minf(real a, real b) { return (b < a) ? b : a; } /* std::min */

enum { LIQ = 0, VAP = 1, WALL = 2, DEAD = 3 };
enum { F_HEATED = 1, F_SOURCE = 2, F_TVAP = 4, F_DYING = 8, F_SCRATCH = 2 | 4 | 8 };
static inline int is_fluid(unsigned char ph) { return ph <= VAP; }
static inline int phase_index(unsigned char ph) { return ph == VAP ? 1 : 0; }

/* -------------------------------------------------------------- kernels
 * SPH_kernels.cuh:14-64 */
typedef struct { int type; real h, inv_h, support, norm; } KParams;

static KParams kparams_make(int t, real h) { /* SPH_kernels.cuh:21-30 */
  KParams k;
  k.type = t;
  k.h = h;
  k.inv_h = (real)1 / h;
  k.support = (real)2 * h;
  const real h3 = h * h * h;
  k.norm = (t == CRYO_KERNEL_CUBIC) ? (real)1 / (kPi * h3) : (real)21 / ((real)16 * kPi * h3);
  return k;
}

static real kernel_W(const KParams* k, real r) { /* SPH_kernels.cuh:34-45 */
  const real q = r * k->inv_h;
  if (q >= (real)2) return 0;
  if (k->type == CRYO_KERNEL_CUBIC) {
    if (q < (real)1) return k->norm * ((real)1 - (real)1.5 * q * q + (real)0.75 * q * q * q);
    const real t = (real)2 - q;
    return k->norm * (real)0.25 * t * t * t;
  }
  const real t = (real)1 - (real)0.5 * q;
  const real t2 = t * t;
  return k->norm * t2 * t2 * ((real)2 * q + (real)1);
}

static real kernel_dWdr(const KParams* k, real r) { /* SPH_kernels.cuh:48-58 */
  const real q = r * k->inv_h;
  if (q >= (real)2) return 0;
  if (k->type == CRYO_KERNEL_CUBIC) {
    if (q < (real)1) return k->norm * k->inv_h * ((real)-3 * q + (real)2.25 * q * q);
    const real t = (real)2 - q;
    return k->norm * k->inv_h * (real)-0.75 * t * t;
  }
  const real t = (real)1 - (real)0.5 * q;
  return k->norm * k->inv_h * (real)-5 * q * t * t * t;
}

static V3 kernel_gradW(const KParams* k, V3 rij, real r) { /* SPH_kernels.cuh:61-64 */
  if (r <= (real)1e-12 * k->h) return v3(0, 0, 0);
  return vmul(rij, kernel_dWdr(k, r) / r);
}

static real akinci_cohesion(real r, real c) { /* SPH_kernels.cuh:69-78 */
  if (r >= c || r <= (real)0) return 0;
  const real c3 = c * c * c;
  const real c9 = c3 * c3 * c3;
  const real coeff = (real)32 / (kPi * c9);
  const real t = (c - r);
  const real base = t * t * t * r * r * r;
  if ((real)2 * r > c) return coeff * base;
  return coeff * ((real)2 * base - c3 * c3 / (real)64);
}

static real akinci_adhesion(real r, real c) { /* SPH_kernels.cuh:81-86 */
  if (r >= c || (real)2 * r <= c) return 0;
  const real arg = (real)-4 * r * r / c + (real)6 * r - (real)2 * c;
  if (arg <= (real)0) return 0;
  return (real)0.007 / powf(c, (real)3.25) * powf(arg, (real)0.25);
}

/* ---------------------------------------------------------- parameters
 * sim_params.cuh:20-95 */
typedef struct {
  KParams kernel;
  real dx, vol0, support2;
  real rho0[2], mu[2], k[2], cp[2], mref[2];
  real c0, tait_B, tait_gamma, p_bg, gas_R, vapor_K;
  int clamp_negative_pressure;
  V3 gravity;
  int frame_rot;
  V3 omega, omega_dot, frame_origin;
  real alpha_av, alpha_av_vap, delta_sph;
  int density_mode, no_slip, sps, tvf, tvf_stress;
  real tvf_factor, tvf_sigma_min, shift_strength;
  int tvf_interface_only;
  real smagorinsky_cs;
  int st_model;
  real sigma, cos_theta, sin_theta, normal_eps, wall_adhesion_weight;
  int wetting_model, wall_colour, csf_smooth_normals, csf_balanced;
  real akinci_gamma, akinci_beta;
  int thermal, phase_change, wall_bc;
  real T_wall, T_ref, T_sat, h_fg, lee_evap, lee_cond, max_transfer_fraction, vapor_rebalance;
  real pc_density_limit, merge_ratio, split_ratio, heat_power, heat_inv_norm, dt;
} Params;

/* sim_params.cuh:100-121 */
static real eos_pressure(const Params* P, unsigned char ph, real rho, real T) {
  real p;
  if (ph == VAP) {
    p = rho * P->gas_R * T + (P->p_bg - P->vapor_K);
  } else {
    const real ratio = rho / P->rho0[0];
    real r_g;
    if (P->tait_gamma == (real)7) {
      const real r2 = ratio * ratio;
      r_g = r2 * r2 * r2 * ratio;
    } else {
      r_g = powf(ratio, P->tait_gamma);
    }
    p = P->tait_B * (r_g - (real)1) + P->p_bg;
  }
  return (P->clamp_negative_pressure && p < (real)0) ? (real)0 : p;
}
/* sim_params.cuh:124-127 */
static real sound_speed(const Params* P, unsigned char ph, real T) {
  if (ph == VAP) return sqrtf(P->gas_R * (T > (real)0 ? T : (real)0));
  return P->c0;
}
/* sim_params.cuh:129-135 */
static real specific_enthalpy(const Params* P, unsigned char ph, real T) {
  return ph == VAP ? P->h_fg + P->cp[1] * (T - P->T_ref) : P->cp[0] * (T - P->T_ref);
}
static real temperature_from_enthalpy(const Params* P, unsigned char ph, real h) {
  return ph == VAP ? P->T_ref + (h - P->h_fg) / P->cp[1] : P->T_ref + h / P->cp[0];
}

/* ----------------------------------------------------------- state */
typedef struct {
  /* persistent (particle_system.hpp:40-51) */
  V3 *x, *v, *vt, *nrm;
  real *m, *m0, *rho, *T;
  unsigned char *phase, *flags;
  unsigned *id;
  /* scratch (particle_system.hpp:52-72) */
  V3 *a, *ab, *fw, *mw, *ns, *vw;
  real *p, *drho, *dTdt, *sigma, *kappa, *nu_t, *alpha, *wall_w, *heat_w, *out_m, *out_h, *w_norm, *rmin, *p_wv;
  int n, capacity;
  unsigned next_id;
} Particles;

typedef struct {
  V3 origin;
  real cell, inv_cell;
  int nx, ny, nz, num_cells;
  int *cell_start, *cell_end;
  unsigned *keys, *perm;
  int keys_n;
} Grid;

typedef struct {
  int n;
  double* time;
  V3* acc;
  V3* omega; /* NULL when the table has no angular velocity */
  V3 origin;
} Maneuver;

typedef struct {
  cryo_config_t cfg;
  cryo_fluid_t fluid;
  Params P;
  Particles ps;
  Grid grid;
  unsigned *split_flag, *split_offset;
  int split_cap;
  int initialized, has_vapor;
  double time;
  long long step;
  double last_dt;
  real char_length;
  real v_max, a_max, Tv_max, nu_t_max, spacing_ratio;
  double heat_input, evaporated, condensed, vented, vented_h, p_ullage;
  int has_maneuver;
  Maneuver man;
  V3 frame_acc;
  double fluid_volume0;
  int splits, merges;
  real pass_dt;
  char err[256];
} Oracle;

#define ALLOC(p, n) ((p) = calloc((size_t)((n) > 0 ? (n) : 1), sizeof(*(p))))
#define GROW(p, n, keep)                                                         \
  do {                                                                           \
    void* q__ = calloc((size_t)((n) > 0 ? (n) : 1), sizeof(*(p)));                \
    if ((keep) > 0) memcpy(q__, (p), (size_t)(keep) * sizeof(*(p)));             \
    free(p);                                                                     \
    (p) = q__;                                                                   \
  } while (0)

static void ps_free(Particles* s) {
  free(s->x); free(s->v); free(s->vt); free(s->nrm); free(s->m); free(s->m0); free(s->rho); free(s->T);
  free(s->phase); free(s->flags); free(s->id);
  free(s->a); free(s->ab); free(s->fw); free(s->mw); free(s->ns); free(s->vw);
  free(s->p); free(s->drho); free(s->dTdt); free(s->sigma); free(s->kappa); free(s->nu_t); free(s->alpha);
  free(s->wall_w); free(s->heat_w); free(s->out_m); free(s->out_h); free(s->w_norm); free(s->rmin); free(s->p_wv);
  memset(s, 0, sizeof(*s));
}

/* ParticleSystem::allocate (particle_system.cpp:60-64) */
static void ps_allocate(Particles* s, int cap) {
  ps_free(s);
  ALLOC(s->x, cap); ALLOC(s->v, cap); ALLOC(s->vt, cap); ALLOC(s->nrm, cap);
  ALLOC(s->m, cap); ALLOC(s->m0, cap); ALLOC(s->rho, cap); ALLOC(s->T, cap);
  ALLOC(s->phase, cap); ALLOC(s->flags, cap); ALLOC(s->id, cap);
  ALLOC(s->a, cap); ALLOC(s->ab, cap); ALLOC(s->fw, cap); ALLOC(s->mw, cap); ALLOC(s->ns, cap); ALLOC(s->vw, cap);
  ALLOC(s->p, cap); ALLOC(s->drho, cap); ALLOC(s->dTdt, cap); ALLOC(s->sigma, cap); ALLOC(s->kappa, cap);
  ALLOC(s->nu_t, cap); ALLOC(s->alpha, cap); ALLOC(s->wall_w, cap); ALLOC(s->heat_w, cap);
  ALLOC(s->out_m, cap); ALLOC(s->out_h, cap); ALLOC(s->w_norm, cap); ALLOC(s->rmin, cap); ALLOC(s->p_wv, cap);
  s->capacity = cap;
  s->n = 0;
}

/* ParticleSystem::grow (particle_system.cpp:66-71) */
static void ps_grow(Particles* s, int cap) {
  if (cap <= s->capacity) return;
  const int k = s->n;
  GROW(s->x, cap, k); GROW(s->v, cap, k); GROW(s->vt, cap, k); GROW(s->nrm, cap, k);
  GROW(s->m, cap, k); GROW(s->m0, cap, k); GROW(s->rho, cap, k); GROW(s->T, cap, k);
  GROW(s->phase, cap, k); GROW(s->flags, cap, k); GROW(s->id, cap, k);
  GROW(s->a, cap, k); GROW(s->ab, cap, k); GROW(s->fw, cap, k); GROW(s->mw, cap, k); GROW(s->ns, cap, k);
  GROW(s->vw, cap, k); GROW(s->p, cap, k); GROW(s->drho, cap, k); GROW(s->dTdt, cap, k); GROW(s->sigma, cap, k);
  GROW(s->kappa, cap, k); GROW(s->nu_t, cap, k); GROW(s->alpha, cap, k); GROW(s->wall_w, cap, k);
  GROW(s->heat_w, cap, k); GROW(s->out_m, cap, k); GROW(s->out_h, cap, k); GROW(s->w_norm, cap, k);
  GROW(s->rmin, cap, k); GROW(s->p_wv, cap, k);
  s->capacity = cap;
}

/* --------------------------------------------------------------- grid */
/* spatial_hash.hpp:22-26 */
static void cell_coords(const Grid* g, V3 p, int* cx, int* cy, int* cz) {
  *cx = clampi((int)floorf((p.x - g->origin.x) * g->inv_cell), 0, g->nx - 1);
  *cy = clampi((int)floorf((p.y - g->origin.y) * g->inv_cell), 0, g->ny - 1);
  *cz = clampi((int)floorf((p.z - g->origin.z) * g->inv_cell), 0, g->nz - 1);
}
/* spatial_hash.hpp:28-32 */
static int cell_index(const Grid* g, V3 p) {
  int cx, cy, cz;
  cell_coords(g, p, &cx, &cy, &cz);
  return (cz * g->ny + cy) * g->nx + cx;
}

/* Neighbour iteration of spatial_hash.hpp:37-56: 27 cells in z, y, x order
 * (clipped at the grid), j ascending inside a cell.  Written as a macro so
 * each pass keeps its loop body inline, like the reference's lambdas. */
#define FOR_EACH_NEIGHBOR(G, P, J, ...)                                         \
  do {                                                                           \
    int cx__, cy__, cz__;                                                        \
    cell_coords((G), (P), &cx__, &cy__, &cz__);                                  \
    const int z0__ = cz__ > 0 ? cz__ - 1 : 0, z1__ = cz__ < (G)->nz - 1 ? cz__ + 1 : cz__; \
    const int y0__ = cy__ > 0 ? cy__ - 1 : 0, y1__ = cy__ < (G)->ny - 1 ? cy__ + 1 : cy__; \
    const int x0__ = cx__ > 0 ? cx__ - 1 : 0, x1__ = cx__ < (G)->nx - 1 ? cx__ + 1 : cx__; \
    for (int z__ = z0__; z__ <= z1__; ++z__)                                     \
      for (int y__ = y0__; y__ <= y1__; ++y__) {                                 \
        const int row__ = (z__ * (G)->ny + y__) * (G)->nx;                       \
        for (int x__ = x0__; x__ <= x1__; ++x__) {                               \
          const int c__ = row__ + x__;                                           \
          const int s__ = (G)->cell_start[c__];                                  \
          if (s__ < 0) continue;                                                 \
          const int e__ = (G)->cell_end[c__];                                    \
          for (int J = s__; J < e__; ++J) { __VA_ARGS__ }                               \
        }                                                                        \
      }                                                                          \
  } while (0)

/* SpatialHash::configure (spatial_hash.cu:15-30) */
static int grid_configure(Oracle* o, V3 lo, V3 hi, real cell) {
  Grid* g = &o->grid;
  if (!(cell > 0)) { snprintf(o->err, sizeof o->err, "SpatialHash: cell size must be positive"); return CRYO_EINVAL; }
  g->cell = cell;
  g->origin = vsub(lo, v3(cell, cell, cell));
  const V3 ext = vsub(hi, lo);
  g->nx = (int)ceilf(ext.x / cell) + 2; if (g->nx < 1) g->nx = 1;
  g->ny = (int)ceilf(ext.y / cell) + 2; if (g->ny < 1) g->ny = 1;
  g->nz = (int)ceilf(ext.z / cell) + 2; if (g->nz < 1) g->nz = 1;
  const long long cells = (long long)g->nx * g->ny * g->nz;
  if (cells > 400000000LL) {
    snprintf(o->err, sizeof o->err, "SpatialHash: grid too large; increase the cell size");
    return CRYO_ERUNTIME;
  }
  g->num_cells = (int)cells;
  free(g->cell_start); free(g->cell_end);
  ALLOC(g->cell_start, g->num_cells + 1);
  ALLOC(g->cell_end, g->num_cells + 1);
  g->inv_cell = (real)1 / g->cell; /* SpatialHash::view (spatial_hash.cu:36-46) */
  return CRYO_OK;
}

/* gather_into + reorder_particles (spatial_hash.cu:116-138): only the 11
 * persistent arrays are permuted; scratch arrays keep their slots. */
#define GATHER(arr, T)                                                   \
  do {                                                                   \
    T* tmp__ = malloc((size_t)(n_new > 0 ? n_new : 1) * sizeof(T));      \
    for (int i = 0; i < n_new; ++i) tmp__[i] = s->arr[perm[i]];          \
    memcpy(s->arr, tmp__, (size_t)n_new * sizeof(T));                   \
    free(tmp__);                                                         \
  } while (0)
static void reorder_particles(Particles* s, const unsigned* perm, int n_new) {
  GATHER(x, V3); GATHER(v, V3); GATHER(vt, V3); GATHER(nrm, V3);
  GATHER(m, real); GATHER(m0, real); GATHER(rho, real); GATHER(T, real);
  GATHER(phase, unsigned char); GATHER(flags, unsigned char); GATHER(id, unsigned);
}

/* SpatialHash::build, CPU counting-sort branch (spatial_hash.cu:48-114).
 * Returns the number of removed (dead) particles. */
static int grid_build(Oracle* o) {
  Grid* g = &o->grid;
  Particles* s = &o->ps;
  const int n = s->n;
  if (g->keys_n < s->capacity) {
    free(g->keys); free(g->perm);
    ALLOC(g->keys, s->capacity);
    ALLOC(g->perm, s->capacity);
    g->keys_n = s->capacity;
  }
  const int sentinel = g->num_cells;
  for (int i = 0; i < n; ++i) {
    g->keys[i] = s->phase[i] == DEAD ? (unsigned)sentinel : (unsigned)cell_index(g, s->x[i]);
    g->perm[i] = (unsigned)i;
  }
  int* counts = calloc((size_t)g->num_cells + 2, sizeof(int));
  for (int i = 0; i < n; ++i) ++counts[g->keys[i] + 1];
  for (int c = 0; c <= g->num_cells; ++c) counts[c + 1] += counts[c];
  for (int c = 0; c < g->num_cells; ++c) {
    const int st = counts[c], e = counts[c + 1];
    g->cell_start[c] = (e > st) ? st : -1;
    g->cell_end[c] = (e > st) ? e : -1;
  }
  const int n_alive = counts[g->num_cells];
  unsigned* sorted = malloc((size_t)(n > 0 ? n : 1) * sizeof(unsigned));
  for (int i = 0; i < n; ++i) sorted[counts[g->keys[i]]++] = (unsigned)i;
  memcpy(g->perm, sorted, (size_t)n * sizeof(unsigned));
  free(sorted);
  free(counts);
  /* sorted keys, for inspection */
  unsigned* k2 = malloc((size_t)(n > 0 ? n : 1) * sizeof(unsigned));
  for (int i = 0; i < n; ++i) k2[i] = g->keys[g->perm[i]];
  memcpy(g->keys, k2, (size_t)n * sizeof(unsigned));
  free(k2);
  reorder_particles(s, g->perm, n_alive);
  s->n = n_alive;
  return n - n_alive;
}

/* ---------------------------------------------------------- physics */
/* compute_density_summation (SPH_kernels.cu:6-34) */
static void density_summation(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph)) {
      s->sigma[i] = (real)1 / P->vol0;
      s->rmin[i] = P->kernel.support;
      continue;
    }
    const V3 xi = s->x[i];
    real sum = 0, r2min = P->support2;
    FOR_EACH_NEIGHBOR(g, xi, j, {
      const real r2 = vnorm2(vsub(xi, s->x[j]));
      if (r2 >= P->support2) continue;
      sum += kernel_W(&P->kernel, sqrtf(r2));
      if (j != i && r2 < r2min) r2min = r2;
    });
    s->sigma[i] = sum;
    s->rmin[i] = sqrtf(r2min);
    if (P->density_mode == CRYO_DENSITY_SUMMATION) s->rho[i] = (ph == LIQ ? s->m0[i] : s->m[i]) * sum;
  }
}

/* normalize_initial_masses (SPH_kernels.cu:36-54) */
static void normalize_initial_masses(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    if (!is_fluid(s->phase[i])) continue;
    const V3 xi = s->x[i];
    real sum = 0;
    FOR_EACH_NEIGHBOR(g, xi, j, {
      const real r2 = vnorm2(vsub(xi, s->x[j]));
      if (r2 < P->support2) sum += kernel_W(&P->kernel, sqrtf(r2));
    });
    if (sum > (real)0) {
      s->m[i] = s->rho[i] / sum;
      s->m0[i] = s->m[i];
    }
  }
}

/* compute_transport_acceleration (SPH_kernels.cu:56-104) */
static void transport_acceleration(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph) || !P->tvf || s->sigma[i] < P->tvf_sigma_min ||
        (P->tvf_interface_only && !(s->alpha[i] > (real)0))) {
      s->ab[i] = v3(0, 0, 0);
      continue;
    }
    const V3 xi = s->x[i];
    const real rhoi = s->rho[i];
    const real Vi = (real)1 / s->sigma[i];
    const real Vi2 = Vi * Vi;
    const real mi = rhoi * Vi;
    const real ci = sound_speed(P, ph, s->T[i]);
    const real pb = P->tvf_factor * P->rho0[phase_index(ph)] * ci * ci;
    const real inv_gamma = (real)1 / P->tait_gamma;
    V3 sum = v3(0, 0, 0);
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i) continue;
      const V3 rij = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rij);
      if (r2 >= P->support2) continue;
      const unsigned char phj = s->phase[j];
      real Vj;
      if (phj == WALL) {
        real rho_w;
        if (ph == VAP) {
          rho_w = (s->p_wv[j] - (P->p_bg - P->vapor_K)) / (P->gas_R * s->T[i]);
        } else {
          const real ratio = (s->p[j] - P->p_bg) / P->tait_B + (real)1;
          rho_w = P->rho0[0] * powf(ratio > (real)0.5 ? ratio : (real)0.5, inv_gamma);
        }
        Vj = rho_w > (real)0 ? Vi * rhoi / rho_w : Vi;
      } else {
        Vj = (real)1 / s->sigma[j];
      }
      sum = vadd(sum, vmul(kernel_gradW(&P->kernel, rij, sqrtf(r2)), Vi2 + Vj * Vj));
    });
    s->ab[i] = vmul(sum, -pb / mi);
  }
}

/* apply_particle_shifting (SPH_kernels.cu:106-160) */
static void particle_shifting(Oracle* o, real mach) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  const real h = P->kernel.h;
  const real w_dx = kernel_W(&P->kernel, P->dx);
  const real coeff = P->shift_strength * mach * (real)4 * h * h;
  const real cap = (real)0.1 * P->dx;
  for (int i = 0; i < s->n; ++i) {
    s->ns[i] = v3(0, 0, 0);
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph) || s->sigma[i] < P->tvf_sigma_min) continue;
    const V3 xi = s->x[i];
    V3 sum = v3(0, 0, 0);
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i) continue;
      const unsigned char phj = s->phase[j];
      if (phj == DEAD) continue;
      const V3 rij = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rij);
      if (r2 >= P->support2) continue;
      const real r = sqrtf(r2);
      const real Vj = phj == WALL ? (real)1 / s->sigma[i] : (real)1 / s->sigma[j];
      const real q = kernel_W(&P->kernel, r) / w_dx;
      const real q2 = q * q;
      sum = vadd(sum, vmul(kernel_gradW(&P->kernel, rij, r), Vj * ((real)1 + (real)0.2 * q2 * q2)));
    });
    V3 dr = vmul(sum, -coeff);
    if (s->alpha[i] > (real)0) {
      const real gm = vnorm(s->nrm[i]);
      if (gm > P->normal_eps) {
        const V3 nn = vdiv(s->nrm[i], gm);
        dr = vsub(dr, vmul(nn, vdot(dr, nn)));
      } else {
        dr = v3(0, 0, 0);
      }
    }
    const real len = vnorm(dr);
    if (len > cap) dr = vmul(dr, cap / len);
    s->ns[i] = dr;
  }
  for (int i = 0; i < s->n; ++i)
    if (is_fluid(s->phase[i])) s->x[i] = vadd(s->x[i], s->ns[i]);
}

/* compute_density_rate (SPH_kernels.cu:162-203) */
static void density_rate(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph)) { s->drho[i] = 0; continue; }
    const V3 xi = s->x[i];
    const V3* vel = P->tvf ? s->vt : s->v;
    const V3 vi = vel[i];
    const real rhoi = s->rho[i];
    const real h = P->kernel.h;
    const real eta2 = (real)0.01 * h * h;
    real div = 0, diff = 0;
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i) continue;
      const V3 rij = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rij);
      if (r2 >= P->support2) continue;
      const real r = sqrtf(r2);
      const V3 gw = kernel_gradW(&P->kernel, rij, r);
      const unsigned char phj = s->phase[j];
      if (phj == WALL) {
        div += P->vol0 * vdot(vi, gw);
        continue;
      }
      const real Vj = s->m[j] / s->rho[j];
      div += Vj * vdot(vsub(vi, vel[j]), gw);
      if (phj == ph) diff += Vj * (real)2 * (s->rho[j] - rhoi) * vdot(vneg(rij), gw) / (r2 + eta2);
    });
    s->drho[i] = rhoi * div + P->delta_sph * h * P->c0 * diff;
  }
}

/* compute_equation_of_state (navier_stokes.cu:5-14) */
static void equation_of_state(Oracle* o) {
  Particles* s = &o->ps;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (is_fluid(ph)) s->p[i] = eos_pressure(&o->P, ph, s->rho[i], s->T[i]);
  }
}

/* compute_wall_boundary (navier_stokes.cu:16-69) */
static void wall_boundary(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    if (s->phase[i] != WALL) continue;
    const V3 xi = s->x[i];
    real sw[2] = {0, 0}, sp[2] = {0, 0}, sgr[2] = {0, 0};
    real srho = 0;
    V3 sv = v3(0, 0, 0);
    FOR_EACH_NEIGHBOR(g, xi, j, {
      const unsigned char phj = s->phase[j];
      if (!is_fluid(phj)) continue;
      const V3 rwf = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rwf);
      if (r2 >= P->support2) continue;
      const real w = kernel_W(&P->kernel, sqrtf(r2));
      const real rhoj = s->rho[j];
      const int k = phase_index(phj);
      sw[k] += w;
      sp[k] += s->p[j] * w;
      sgr[k] += vdot(P->gravity, rwf) * rhoj * w;
      srho += rhoj * w;
      sv = vadd(sv, vmul(s->v[j], w));
    });
    real pw[2];
    for (int k = 0; k < 2; ++k) {
      pw[k] = sw[k] > (real)0 ? (sp[k] + sgr[k]) / sw[k] : P->p_bg;
      if (P->clamp_negative_pressure && pw[k] < (real)0) pw[k] = 0;
    }
    if (!(sw[0] > (real)0) && sw[1] > (real)0) pw[0] = pw[1];
    if (!(sw[1] > (real)0) && sw[0] > (real)0) pw[1] = pw[0];
    s->p[i] = pw[0];
    s->p_wv[i] = pw[1];
    s->alpha[i] = (sw[0] + sw[1]) > (real)0 ? sw[0] / (sw[0] + sw[1]) : (real)0;
    const real swt = sw[0] + sw[1];
    if (swt > (real)0) {
      s->rho[i] = srho / swt;
      s->vw[i] = vmul(sv, (real)-1 / swt);
    } else {
      s->rho[i] = P->rho0[0];
      s->vw[i] = v3(0, 0, 0);
    }
    s->a[i] = v3(0, 0, 0);
  }
}

/* compute_sps_viscosity (navier_stokes.cu:71-119) */
static void sps_viscosity(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph)) { s->nu_t[i] = 0; continue; }
    const V3 xi = s->x[i];
    const V3 vi = s->v[i];
    real L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i) continue;
      const V3 rij = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rij);
      if (r2 >= P->support2) continue;
      const V3 gw = kernel_gradW(&P->kernel, rij, sqrtf(r2));
      const unsigned char phj = s->phase[j];
      V3 vj;
      real Vj;
      if (phj == WALL) {
        if (!P->no_slip) continue;
        vj = s->vw[j];
        Vj = P->vol0;
      } else {
        vj = s->v[j];
        Vj = s->m[j] / s->rho[j];
      }
      const V3 dv = vmul(vsub(vj, vi), Vj);
      const real dvc[3] = {dv.x, dv.y, dv.z};
      const real gwc[3] = {gw.x, gw.y, gw.z};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) L[a][b] += dvc[a] * gwc[b];
    });
    real ss = 0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        const real sab = (real)0.5 * (L[a][b] + L[b][a]);
        ss += sab * sab;
      }
    const real smag = sqrtf((real)2 * ss);
    const real l = P->smagorinsky_cs * P->dx;
    s->nu_t[i] = l * l * smag;
  }
}

/* compute_momentum (navier_stokes.cu:121-245) */
static void momentum(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph)) {
      s->a[i] = v3(0, 0, 0);
      s->fw[i] = v3(0, 0, 0);
      s->mw[i] = v3(0, 0, 0);
      continue;
    }
    const int pi_idx = phase_index(ph);
    const V3 xi = s->x[i];
    const V3 vi = s->v[i];
    const real mi = s->m[i];
    const real rhoi = s->rho[i];
    const real Vi = mi / rhoi;
    const real Vi2 = Vi * Vi;
    const real pi = s->p[i];
    const real ci = sound_speed(P, ph, s->T[i]);
    const real etai = P->mu[pi_idx] + (P->sps ? rhoi * s->nu_t[i] : (real)0);
    const real alpha_i = ph == VAP ? P->alpha_av_vap : P->alpha_av;
    const real h = P->kernel.h;
    const real eta2 = (real)0.01 * h * h;
    V3 force = v3(0, 0, 0);
    V3 acc_av = v3(0, 0, 0);
    const real r_guard = (real)0.6 * P->dx;
    const int tvf_stress = P->tvf && P->tvf_stress;
    const V3 dvi = vsub(s->vt[i], vi);
    V3 fwall = v3(0, 0, 0), mwall = v3(0, 0, 0);
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i) continue;
      const V3 rij = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rij);
      if (r2 >= P->support2) continue;
      const real r = sqrtf(r2);
      const real dW = kernel_dWdr(&P->kernel, r);
      const int separated = r > (real)1e-12 * h;
      const V3 gw = separated ? vmul(rij, dW / r) : v3(0, 0, 0);
      const unsigned char phj = s->phase[j];
      if (phj == WALL) {
        const V3 f_before = force, a_before = acc_av;
        const real Vj = P->vol0;
        const real vsum = Vi2 + Vj * Vj;
        const real pw = ph == VAP ? s->p_wv[j] : s->p[j];
        force = vsub(force, vmul(gw, vsum * (real)0.5 * (pi + pw)));
        if (tvf_stress) force = vadd(force, vmul(vi, (real)0.5 * vsum * rhoi * vdot(dvi, gw)));
        if (r < r_guard && separated) {
          const real q = (real)1 - r / r_guard;
          const V3 nn = vdiv(rij, r);
          acc_av = vadd(acc_av, vmul(nn, (real)4 * ci * ci * q * q / r_guard));
          const real vn = vdot(vi, nn);
          if (vn < (real)0 && P->dt > (real)0) acc_av = vsub(acc_av, vmul(nn, q * vn / P->dt));
        }
        if (P->no_slip) {
          const V3 vij = vsub(vi, s->vw[j]);
          if (separated) force = vadd(force, vmul(vij, vsum * etai * dW / r));
          const real vr = vdot(vij, rij);
          if (alpha_i > (real)0 && vr < (real)0) {
            const real mu_ij = h * vr / (r2 + eta2);
            const real Pi = -alpha_i * ci * mu_ij / rhoi;
            acc_av = vsub(acc_av, vmul(gw, rhoi * P->vol0 * Pi));
          }
        }
        const V3 dF = vadd(vsub(force, f_before), vmul(vsub(acc_av, a_before), mi));
        fwall = vadd(fwall, dF);
        mwall = vadd(mwall, vcross(vsub(s->x[j], P->frame_origin), dF));
        continue;
      }
      const real mj = s->m[j];
      const real rhoj = s->rho[j];
      const real Vj = mj / rhoj;
      const real vsum = Vi2 + Vj * Vj;
      const real pt = (rhoj * pi + rhoi * s->p[j]) / (rhoi + rhoj);
      force = vsub(force, vmul(gw, vsum * pt));
      if (tvf_stress) {
        const V3 vj = s->v[j];
        const V3 Ag = vadd(vmul(vi, rhoi * vdot(dvi, gw)), vmul(vj, rhoj * vdot(vsub(s->vt[j], vj), gw)));
        force = vadd(force, vmul(Ag, (real)0.5 * vsum));
      }
      const V3 vij = vsub(vi, s->v[j]);
      const real etaj = P->mu[phase_index(phj)] + (P->sps ? rhoj * s->nu_t[j] : (real)0);
      const real eta_sum = etai + etaj;
      if (eta_sum > (real)0 && separated) {
        const real eta_ij = (real)2 * etai * etaj / eta_sum;
        force = vadd(force, vmul(vij, vsum * eta_ij * dW / r));
      }
      if (alpha_i > (real)0 && phj == ph) {
        const real vr = vdot(vij, rij);
        if (vr < (real)0) {
          const real cj = sound_speed(P, phj, s->T[j]);
          const real mu_ij = h * vr / (r2 + eta2);
          const real Pi = -alpha_i * (real)0.5 * (ci + cj) * mu_ij / ((real)0.5 * (rhoi + rhoj));
          acc_av = vsub(acc_av, vmul(gw, mj * Pi));
        }
      }
    });
    V3 acc = vadd(vadd(P->gravity, vdiv(force, mi)), acc_av);
    if (P->frame_rot) {
      const V3 r = vsub(xi, P->frame_origin);
      acc = vsub(acc, vadd(vadd(vcross(P->omega_dot, r), vcross(P->omega, vcross(P->omega, r))),
                           vmul(vcross(P->omega, vi), (real)2)));
    }
    s->a[i] = acc;
    s->fw[i] = fwall;
    s->mw[i] = mwall;
  }
}

/* compute_interface_fields (surface_tension.cu:5-85) */
static void interface_fields(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph)) continue;
    const V3 xi = s->x[i];
    const real ci = ph == LIQ ? (real)1 : (real)0;
    V3 gradc = v3(0, 0, 0), wall_n = v3(0, 0, 0), akn = v3(0, 0, 0), gradphi = v3(0, 0, 0);
    real s_all = 0, s_other = 0, ww = 0, hw = 0;
    FOR_EACH_NEIGHBOR(g, xi, j, {
      const V3 rij = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rij);
      if (r2 >= P->support2) continue;
      const real r = sqrtf(r2);
      const real w = kernel_W(&P->kernel, r);
      const unsigned char phj = s->phase[j];
      if (phj == WALL) {
        const real vw = P->vol0 * w;
        ww += vw;
        if (s->flags[j] & F_HEATED) hw += vw;
        wall_n = vadd(wall_n, vmul(s->nrm[j], vw));
        gradphi = vadd(gradphi, vmul(kernel_gradW(&P->kernel, rij, r), P->vol0));
        if (P->wall_colour)
          gradc = vadd(gradc, vmul(kernel_gradW(&P->kernel, rij, r), P->vol0 * (s->alpha[j] - ci)));
        continue;
      }
      const real Vj = s->m[j] / s->rho[j];
      s_all += Vj * w;
      if (phj != ph) s_other += Vj * w;
      if (j == i) continue;
      const V3 gw = kernel_gradW(&P->kernel, rij, r);
      const real cj = phj == LIQ ? (real)1 : (real)0;
      gradc = vadd(gradc, vmul(gw, Vj * (cj - ci)));
      if (phj == LIQ) akn = vadd(akn, vmul(gw, Vj));
    });
    s->alpha[i] = s_all > (real)0 ? s_other / s_all : (real)0;
    s->wall_w[i] = ww;
    s->heat_w[i] = hw;
    if (P->st_model == CRYO_ST_AKINCI) {
      s->nrm[i] = ph == LIQ ? vmul(akn, -P->kernel.h) : v3(0, 0, 0);
      continue;
    }
    const real gmag = vnorm(gradc);
    s->vw[i] = v3(0, 0, 0);
    if (P->wetting_model != 0 && ww > (real)0 && gmag > P->normal_eps && vnorm2(wall_n) > (real)0) {
      const V3 nw = vnormalized(wall_n);
      const V3 nh = vdiv(gradc, gmag);
      const V3 tan_in = vsub(nh, vmul(nw, vdot(nh, nw)));
      const real tm = vnorm(tan_in);
      if (tm > (real)1e-6) {
        const real cos_d = -vdot(nh, nw);
        const real delta_w = (real)2 * vnorm(gradphi);
        const real coeff = (real)2 * P->sigma / (P->rho0[0] + P->rho0[1]);
        s->vw[i] = vmul(tan_in, -(P->cos_theta - cos_d) * coeff * gmag * delta_w / tm);
      }
    }
    if (P->wetting_model != 1 && ww > (real)0 && gmag > P->normal_eps) {
      const V3 nw = vnormalized(wall_n);
      const V3 nh = vdiv(gradc, gmag);
      V3 t = vsub(nh, vmul(nw, vdot(nh, nw)));
      const real tmag = vnorm(t);
      if (vnorm2(nw) > (real)0 && tmag > (real)1e-6) {
        t = vdiv(t, tmag);
        const V3 target = vadd(vmul(nw, -P->cos_theta), vmul(t, P->sin_theta));
        const real beta = clampf(ww / P->wall_adhesion_weight, (real)0, (real)1);
        const V3 blended = vnormalized(vadd(vmul(nh, (real)1 - beta), vmul(target, beta)));
        gradc = vmul(blended, gmag);
      }
    }
    s->nrm[i] = gradc;
  }
}

/* smooth_interface_normals (surface_tension.cu:87-118) */
static void smooth_normals(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    if (!is_fluid(s->phase[i])) continue;
    const V3 gi = s->nrm[i];
    const real gmag = vnorm(gi);
    if (!(gmag > P->normal_eps)) { s->ns[i] = v3(0, 0, 0); continue; }
    if (!P->csf_smooth_normals) { s->ns[i] = vdiv(gi, gmag); continue; }
    const V3 xi = s->x[i];
    V3 acc = v3(0, 0, 0);
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (!is_fluid(s->phase[j])) continue;
      const V3 gj = s->nrm[j];
      const real gjm = vnorm(gj);
      if (!(gjm > P->normal_eps)) continue;
      const real r2 = vnorm2(vsub(xi, s->x[j]));
      if (r2 >= P->support2) continue;
      acc = vadd(acc, vmul(gj, (s->m[j] / s->rho[j]) * kernel_W(&P->kernel, sqrtf(r2)) / gjm));
    });
    s->ns[i] = vnormalized(acc);
  }
}

/* apply_csf_surface_tension (surface_tension.cu:120-177) */
static void csf_surface_tension(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  const real coeff = (real)2 * P->sigma / (P->rho0[0] + P->rho0[1]);
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph)) continue;
    const V3 ni = s->ns[i];
    if (!(vnorm2(ni) > (real)0.25)) { s->kappa[i] = 0; continue; }
    const V3 xi = s->x[i];
    const real rhoi = s->rho[i];
    const real mi = s->m[i];
    const real Vi = mi / rhoi;
    const real ci = ph == LIQ ? (real)1 : (real)0;
    real num = 0, den = 0;
    V3 G = v3(0, 0, 0);
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i) continue;
      const unsigned char phj = s->phase[j];
      if (!is_fluid(phj)) continue;
      const V3 rij = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rij);
      if (r2 >= P->support2) continue;
      const real r = sqrtf(r2);
      const real dW = kernel_dWdr(&P->kernel, r);
      const V3 gw = vmul(rij, dW / r);
      const real rhoj = s->rho[j];
      const real Vj = s->m[j] / rhoj;
      const V3 nj = s->ns[j];
      if (vnorm2(nj) > (real)0.25) {
        num += Vj * vdot(vsub(ni, nj), gw);
        den += Vj * r * (-dW);
      }
      if (P->csf_balanced) {
        const real cj = phj == LIQ ? (real)1 : (real)0;
        G = vadd(G, vmul(gw, (Vi * Vi + Vj * Vj) * (rhoj * ci + rhoi * cj) / (rhoi + rhoj)));
      }
    });
    const real kappa = den > (real)0 ? (real)3 * num / den : (real)0;
    s->kappa[i] = kappa;
    if (P->wetting_model != 0) s->a[i] = vadd(s->a[i], s->vw[i]);
    if (P->csf_balanced) s->a[i] = vadd(s->a[i], vmul(G, P->sigma * kappa / mi));
    else s->a[i] = vadd(s->a[i], vmul(s->nrm[i], coeff * kappa));
  }
}

/* apply_akinci_surface_tension (surface_tension.cu:179-213) */
static void akinci_surface_tension(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    if (s->phase[i] != LIQ) continue;
    const V3 xi = s->x[i];
    const V3 ni = s->nrm[i];
    const real mi = s->m[i];
    const real rhoi = s->rho[i];
    const real c = P->kernel.support;
    const real rho0 = P->rho0[0];
    const real psi = rho0 * P->vol0;
    V3 acc = v3(0, 0, 0);
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i) continue;
      const V3 rij = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rij);
      if (r2 >= c * c || r2 <= (real)0) continue;
      const real r = sqrtf(r2);
      const V3 rhat = vdiv(rij, r);
      const unsigned char phj = s->phase[j];
      if (phj == LIQ) {
        const real K = (real)2 * rho0 / (rhoi + s->rho[j]);
        const V3 f_coh = vmul(rhat, -P->akinci_gamma * mi * s->m[j] * akinci_cohesion(r, c));
        const V3 f_curv = vmul(vsub(ni, s->nrm[j]), -P->akinci_gamma * mi);
        acc = vadd(acc, vmul(vadd(f_coh, f_curv), K / mi));
      } else if (phj == WALL) {
        acc = vsub(acc, vmul(rhat, P->akinci_beta * psi * akinci_adhesion(r, c)));
      }
    });
    s->a[i] = vadd(s->a[i], acc);
  }
}

/* compute_thermal_rates (phase_change.cu:31-75) */
static void thermal_rates(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph)) { s->dTdt[i] = 0; continue; }
    const int ii = phase_index(ph);
    const V3 xi = s->x[i];
    const real Ti = s->T[i];
    const real mi = s->m[i];
    const real Vi = mi / s->rho[i];
    const real ki = P->k[ii];
    const real eta2 = (real)0.01 * P->kernel.h * P->kernel.h;
    const int iso = P->wall_bc == CRYO_WALL_ISOTHERMAL;
    real q = 0;
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i) continue;
      const unsigned char phj = s->phase[j];
      real Vj, kij;
      if (phj == WALL) {
        if (!iso) continue;
        Vj = P->vol0;
        kij = (real)2 * ki;
      } else {
        const real kj = P->k[phase_index(phj)];
        Vj = s->m[j] / s->rho[j];
        kij = (real)4 * ki * kj / (ki + kj);
      }
      const V3 rij = vsub(xi, s->x[j]);
      const real r2 = vnorm2(rij);
      if (r2 >= P->support2) continue;
      const real r = sqrtf(r2);
      const real rgw = r * kernel_dWdr(&P->kernel, r);
      q += Vi * Vj * kij * (Ti - s->T[j]) * rgw / (r2 + eta2);
    });
    q += P->heat_power * s->heat_w[i] * P->heat_inv_norm;
    s->dTdt[i] = q / (mi * P->cp[ii]);
  }
}

/* phase_change_sources (phase_change.cu:77-137) */
static void pc_sources(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    unsigned char fl = (unsigned char)(s->flags[i] & ~F_SCRATCH);
    s->out_m[i] = 0;
    s->out_h[i] = 0;
    s->w_norm[i] = 0;
    if (!is_fluid(ph)) { s->flags[i] = fl; continue; }
    const int ii = phase_index(ph);
    const real m = s->m[i];
    const real T = s->T[i];
    if (m < P->merge_ratio * P->mref[ii]) {
      s->out_m[i] = m;
      s->out_h[i] = specific_enthalpy(P, ph, T);
      fl |= F_SOURCE | F_DYING;
      if (ph == VAP) fl |= F_TVAP;
      s->flags[i] = fl;
      continue;
    }
    const real alpha = s->alpha[i];
    if (P->phase_change && alpha > (real)0 && P->dt > (real)0) {
      if (ph == LIQ && T > P->T_sat) {
        const real h_out = P->h_fg + P->cp[1] * (P->T_sat - P->T_ref);
        const real latent = h_out - P->cp[0] * (P->T_sat - P->T_ref);
        const real rate = P->lee_evap * m * alpha * (T - P->T_sat) / P->T_sat;
        real dm = rate * P->dt;
        const real dm_energy = m * P->cp[0] * (T - P->T_sat) / latent;
        dm = dm < dm_energy ? dm : dm_energy;
        const real dm_cap = P->max_transfer_fraction * m;
        dm = dm < dm_cap ? dm : dm_cap;
        if (dm > (real)0) {
          s->out_m[i] = dm;
          s->out_h[i] = h_out;
          fl |= F_SOURCE | F_TVAP;
        }
      } else if (ph == VAP && T < P->T_sat) {
        const real rate = P->lee_cond * m * alpha * (P->T_sat - T) / P->T_sat;
        real dm = rate * P->dt;
        real dm_cap = P->max_transfer_fraction * m;
        if (P->pc_density_limit > (real)0 && P->pc_density_limit * m < dm_cap) dm_cap = P->pc_density_limit * m;
        dm = dm < dm_cap ? dm : dm_cap;
        if (dm > (real)0) {
          s->out_m[i] = dm;
          s->out_h[i] = specific_enthalpy(P, VAP, T);
          fl |= F_SOURCE;
        }
      }
    }
    s->flags[i] = fl;
  }
}

/* phase_change_normalize (phase_change.cu:139-172) */
static void pc_normalize(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char fl = s->flags[i];
    if (!(fl & F_SOURCE)) continue;
    const unsigned char target = (fl & F_TVAP) ? VAP : LIQ;
    const V3 xi = s->x[i];
    real wsum = 0, wr_max = 0;
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i || s->phase[j] != target || (s->flags[j] & F_DYING)) continue;
      const real r2 = vnorm2(vsub(xi, s->x[j]));
      if (r2 >= P->support2) continue;
      const real w = kernel_W(&P->kernel, sqrtf(r2));
      const real rhoj = s->rho[j];
      wsum += (s->m[j] / rhoj) * w;
      const real wr = w / rhoj;
      wr_max = wr > wr_max ? wr : wr_max;
    });
    s->w_norm[i] = wsum;
    if (!(wsum > (real)0)) { s->out_m[i] = 0; continue; }
    if (target == VAP && P->pc_density_limit > (real)0 && !(fl & F_DYING) && wr_max > (real)0) {
      const real cap = P->pc_density_limit * wsum / wr_max;
      if (s->out_m[i] > cap) s->out_m[i] = cap;
    }
  }
}

/* phase_change_apply (phase_change.cu:174-215) */
static void pc_apply(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    if (!is_fluid(ph)) continue;
    const unsigned char fl = s->flags[i];
    const real mi = s->m[i];
    const real Vi = mi / s->rho[i];
    const V3 xi = s->x[i];
    real in_m = 0, in_H = 0;
    if (!(fl & F_DYING)) {
      FOR_EACH_NEIGHBOR(g, xi, j, {
        if (j == i) continue;
        const real om = s->out_m[j];
        if (!(om > (real)0)) continue;
        const unsigned char target = (s->flags[j] & F_TVAP) ? VAP : LIQ;
        if (target != ph) continue;
        const real r2 = vnorm2(vsub(xi, s->x[j]));
        if (r2 >= P->support2) continue;
        const real share = om * Vi * kernel_W(&P->kernel, sqrtf(r2)) / s->w_norm[j];
        in_m += share;
        in_H += share * s->out_h[j];
      });
    }
    const real om_i = s->out_m[i];
    if ((fl & F_DYING) && om_i > (real)0) {
      s->m[i] = 0;
      s->phase[i] = DEAD;
      continue;
    }
    if (!(om_i > (real)0) && !(in_m > (real)0)) continue;
    const real m_new = mi - om_i + in_m;
    const real H_new = mi * specific_enthalpy(P, ph, s->T[i]) - om_i * s->out_h[i] + in_H;
    s->T[i] = temperature_from_enthalpy(P, ph, H_new / m_new);
    s->m[i] = m_new;
  }
}

/* rebalance_vapor_mass (phase_change.cu:217-268) */
static void rebalance_vapor(Oracle* o) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  const real beta = P->vapor_rebalance;
  for (int i = 0; i < s->n; ++i) {
    s->out_m[i] = 0;
    s->out_h[i] = 0;
    s->ns[i] = v3(0, 0, 0);
    if (s->phase[i] != VAP) continue;
    const V3 xi = s->x[i];
    const real mi = s->m[i];
    const real hi = specific_enthalpy(P, VAP, s->T[i]);
    const V3 vi = s->v[i];
    real dm = 0, dH = 0;
    V3 dP = v3(0, 0, 0);
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (j == i || s->phase[j] != VAP) continue;
      const real r2 = vnorm2(vsub(xi, s->x[j]));
      if (r2 >= P->support2) continue;
      const real flow = beta * P->vol0 * kernel_W(&P->kernel, sqrtf(r2)) * (s->m[j] - mi);
      const int from_j = flow > (real)0;
      dm += flow;
      dH += flow * (from_j ? specific_enthalpy(P, VAP, s->T[j]) : hi);
      dP = vadd(dP, vmul(from_j ? s->v[j] : vi, flow));
    });
    s->out_m[i] = dm;
    s->out_h[i] = dH;
    s->ns[i] = dP;
  }
  for (int i = 0; i < s->n; ++i) {
    if (s->phase[i] != VAP) continue;
    const real dm = s->out_m[i];
    if (dm == (real)0) continue;
    const real m = s->m[i];
    const real m_new = m + dm;
    const real H = m * specific_enthalpy(P, VAP, s->T[i]) + s->out_h[i];
    s->T[i] = temperature_from_enthalpy(P, VAP, H / m_new);
    s->v[i] = vdiv(vadd(vmul(s->v[i], m), s->ns[i]), m_new);
    s->vt[i] = s->v[i];
    s->m[i] = m_new;
    s->out_m[i] = 0;
    s->out_h[i] = 0;
  }
}

/* hash_u32 / hash_unit / random_direction (phase_change.cu:7-27) */
static unsigned hash_u32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}
static real hash_unit(unsigned x) { return (real)(hash_u32(x) & 0x00FFFFFFu) / (real)0x01000000u; }
static V3 random_direction(unsigned id, unsigned seed) {
  const real u = (real)2 * hash_unit(id * 2654435761u ^ seed) - (real)1;
  const real phi = (real)2 * kPi * hash_unit(hash_u32(id + 0x9e3779b9u) ^ (seed * 747796405u));
  const real sq = sqrtf((real)1 - u * u > (real)0 ? (real)1 - u * u : (real)0);
  return v3(sq * cosf(phi), sq * sinf(phi), u);
}

/* mark_heavy_particles (phase_change.cu:270-279) */
static void mark_heavy(Oracle* o, unsigned* flag) {
  const Particles* s = &o->ps;
  const Params* P = &o->P;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char ph = s->phase[i];
    flag[i] = (is_fluid(ph) && s->m[i] > P->split_ratio * P->mref[phase_index(ph)]) ? 1u : 0u;
  }
}

/* split_heavy_particles (phase_change.cu:281-335) */
static void split_heavy(Oracle* o, const unsigned* flag, const unsigned* offset, unsigned id_base, unsigned seed) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  const int n = s->n;
  for (int i = 0; i < n; ++i) {
    if (!flag[i]) continue;
    const unsigned char ph = s->phase[i];
    const real m = s->m[i];
    const unsigned k = offset[i];
    const int dst = n + (int)k;
    if (dst >= s->capacity) continue;
    const real vol = m / s->rho[i];
    V3 e = random_direction(s->id[i], seed);
    const V3 xi = s->x[i];
    const V3 gc = s->nrm[i];
    const real gm = vnorm(gc);
    if (gm > P->normal_eps) {
      const V3 nn = vdiv(gc, gm);
      const V3 t = vsub(e, vmul(nn, vdot(e, nn)));
      e = vnormalized(vsub(t, vmul(nn, (real)0.5)));
      s->x[dst] = vadd(xi, vmul(e, (real)0.5 * cbrtf(vol)));
    } else {
      const real delta = (real)0.25 * cbrtf(vol);
      s->x[dst] = vadd(xi, vmul(e, delta));
      s->x[i] = vsub(xi, vmul(e, delta));
    }
    s->v[dst] = s->v[i];
    s->vt[dst] = s->vt[i];
    s->ab[dst] = s->ab[i];
    s->a[dst] = s->a[i];
    s->nrm[dst] = s->nrm[i];
    s->m[dst] = (real)0.5 * m;
    s->m0[i] *= (real)0.5;
    s->m0[dst] = s->m0[i];
    s->m[i] = (real)0.5 * m;
    s->rho[dst] = s->rho[i];
    s->T[dst] = s->T[i];
    s->phase[dst] = ph;
    s->flags[dst] = (unsigned char)(s->flags[i] & ~F_SCRATCH);
    s->id[dst] = id_base + k;
    s->p[dst] = s->p[i];
    s->sigma[i] *= (real)2;
    s->sigma[dst] = s->sigma[i];
    s->dTdt[dst] = 0;
    s->out_m[dst] = 0;
    s->out_h[dst] = 0;
  }
}

/* apply_venting (phase_change.cu:337-358) */
static void venting(Oracle* o, real relax) {
  Particles* s = &o->ps;
  const Params* P = &o->P;
  for (int i = 0; i < s->n; ++i) {
    s->out_m[i] = 0;
    s->out_h[i] = 0;
    if (s->phase[i] != VAP) continue;
    const real m = s->m[i];
    const real vol = m / s->rho[i];
    const real target = P->rho0[1] * vol;
    if (!(m > target)) continue;
    const real dm = relax * (m - target);
    s->out_m[i] = dm;
    s->out_h[i] = specific_enthalpy(P, VAP, s->T[i]);
    if (P->density_mode == CRYO_DENSITY_CONTINUITY) s->rho[i] *= (m - dm) / m;
    s->m[i] = m - dm;
  }
}

/* --------------------------------------------- solver_detail helpers
 * sph_solver.cu:20-179 */
static void kick_drift(Oracle* o, real dt, int continuity, int tvf) { /* :20-34 */
  Particles* s = &o->ps;
  const real half = (real)0.5 * dt;
  for (int i = 0; i < s->n; ++i) {
    if (!is_fluid(s->phase[i])) continue;
    const V3 v = vadd(s->v[i], vmul(s->a[i], half));
    s->v[i] = v;
    const V3 vt = tvf ? vadd(v, vmul(s->ab[i], half)) : v;
    s->vt[i] = vt;
    s->x[i] = vadd(s->x[i], vmul(vt, dt));
    if (continuity) s->rho[i] += s->drho[i] * dt;
  }
}
static void kick(Oracle* o, real dt, int thermal) { /* :36-46 */
  Particles* s = &o->ps;
  const real half = (real)0.5 * dt;
  for (int i = 0; i < s->n; ++i) {
    if (!is_fluid(s->phase[i])) continue;
    s->v[i] = vadd(s->v[i], vmul(s->a[i], half));
    if (thermal) s->T[i] += s->dTdt[i] * dt;
  }
}
static void scale_velocities(Oracle* o, real f) { /* :48-57 */
  Particles* s = &o->ps;
  for (int i = 0; i < s->n; ++i) {
    if (!is_fluid(s->phase[i])) continue;
    s->v[i] = vmul(s->v[i], f);
    s->vt[i] = vmul(s->vt[i], f);
  }
}
/* reduce_max with the OpenMP semantics: acc = v > acc ? v : acc */
static real max_spacing_ratio(Oracle* o) { /* :62-71 */
  const Particles* s = &o->ps;
  const real dx = o->P.dx;
  real acc = 1;
  for (int i = 0; i < s->n; ++i) {
    real v = 0;
    if (is_fluid(s->phase[i])) {
      const real r = s->rmin[i] > (real)0.05 * dx ? s->rmin[i] : (real)0.05 * dx;
      v = (real)0.5 * dx / r;
    }
    acc = v > acc ? v : acc;
  }
  return acc;
}
static real max_fluid_speed(Oracle* o) { /* :73-76 */
  const Particles* s = &o->ps;
  real acc = 0;
  for (int i = 0; i < s->n; ++i) {
    const real v = is_fluid(s->phase[i]) ? vnorm(s->v[i]) : (real)0;
    acc = v > acc ? v : acc;
  }
  return acc;
}
static real max_fluid_accel(Oracle* o) { /* :78-89 */
  const Particles* s = &o->ps;
  real acc = 0;
  for (int i = 0; i < s->n; ++i) {
    real v = 0;
    if (is_fluid(s->phase[i])) {
      const real a = vnorm(s->a[i]), b = vnorm(s->ab[i]);
      v = a > b ? a : b;
    }
    acc = v > acc ? v : acc;
  }
  return acc;
}
static real max_phase_T(Oracle* o, unsigned char ph) { /* :91-94, :176-179 */
  const Particles* s = &o->ps;
  real acc = 0;
  for (int i = 0; i < s->n; ++i) {
    const real v = s->phase[i] == ph ? s->T[i] : (real)0;
    acc = v > acc ? v : acc;
  }
  return acc;
}
static real max_eddy_viscosity(Oracle* o) { /* :96-99 */
  const Particles* s = &o->ps;
  real acc = 0;
  for (int i = 0; i < s->n; ++i) {
    const real v = is_fluid(s->phase[i]) ? s->nu_t[i] : (real)0;
    acc = v > acc ? v : acc;
  }
  return acc;
}
static double sum_heat_weight(Oracle* o) { /* :101-104 */
  const Particles* s = &o->ps;
  double acc = 0;
  for (int i = 0; i < s->n; ++i) acc += is_fluid(s->phase[i]) ? (double)s->heat_w[i] : 0.0;
  return 0.0 + acc;
}
static double sum_phase_change(Oracle* o, int evaporation) { /* :108-118 */
  const Particles* s = &o->ps;
  double acc = 0;
  for (int i = 0; i < s->n; ++i) {
    const unsigned char fl = s->flags[i];
    double v = 0;
    if ((fl & F_SOURCE) && !(fl & F_DYING)) {
      const int to_vapor = (fl & F_TVAP) != 0;
      v = to_vapor == evaporation ? (double)s->out_m[i] : 0.0;
    }
    acc += v;
  }
  return 0.0 + acc;
}
static int count_merges(Oracle* o) { /* :120-124 */
  const Particles* s = &o->ps;
  int acc = 0;
  for (int i = 0; i < s->n; ++i) acc += ((s->flags[i] & F_DYING) && s->out_m[i] > (real)0) ? 1 : 0;
  return acc;
}
static double sum_out_mass(Oracle* o) { /* :126-128 */
  const Particles* s = &o->ps;
  double acc = 0;
  for (int i = 0; i < s->n; ++i) acc += (double)s->out_m[i];
  return 0.0 + acc;
}
static double sum_out_enthalpy(Oracle* o) { /* :130-133 */
  const Particles* s = &o->ps;
  double acc = 0;
  for (int i = 0; i < s->n; ++i) acc += (double)s->out_m[i] * (double)s->out_h[i];
  return 0.0 + acc;
}
static int count_phase(Oracle* o, unsigned char ph) { /* :147-149 */
  const Particles* s = &o->ps;
  int acc = 0;
  for (int i = 0; i < s->n; ++i) acc += s->phase[i] == ph ? 1 : 0;
  return acc;
}
/* phase_sum (sph_solver.cu:151-174) */
static double phase_sum(Oracle* o, unsigned char ph, int what) {
  const Particles* s = &o->ps;
  const Params* P = &o->P;
  double acc = 0;
  for (int i = 0; i < s->n; ++i) {
    double v = 0;
    if (s->phase[i] == ph) {
      const double m = s->m[i];
      switch (what) {
        case 0: v = m; break;
        case 1: v = m * s->T[i]; break;
        case 2: v = 0.5 * m * (double)vnorm2(s->v[i]); break;
        case 3: v = m * s->x[i].x; break;
        case 4: v = m * s->x[i].y; break;
        case 5: v = m * s->x[i].z; break;
        case 6: v = m * s->v[i].x; break;
        case 7: v = m * s->v[i].y; break;
        case 8: v = m * s->v[i].z; break;
        case 9: v = m * (double)specific_enthalpy(P, ph, s->T[i]); break;
        default: v = 0.0;
      }
    }
    acc += v;
  }
  return 0.0 + acc;
}
/* sum_fluid_vec3 (sph_solver.cu:219-232) */
static V3 sum_fluid_vec3(Oracle* o, const V3* f) {
  const Particles* s = &o->ps;
  double c[3];
  for (int k = 0; k < 3; ++k) {
    double acc = 0;
    for (int i = 0; i < s->n; ++i) {
      double v = 0;
      if (is_fluid(s->phase[i])) v = k == 0 ? (double)f[i].x : (k == 1 ? (double)f[i].y : (double)f[i].z);
      acc += v;
    }
    c[k] = 0.0 + acc;
  }
  return v3((real)c[0], (real)c[1], (real)c[2]);
}

/* FluidProperties::saturation_temperature (fluid_properties.cpp:7-10) */
static real saturation_temperature(const cryo_fluid_t* f, real p) {
  const double inv_T = 1.0 / f->T_sat - ((double)f->R_gas / f->h_fg) * log((double)p / f->p_sat);
  return (real)(1.0 / inv_T);
}
static real saturation_pressure(const cryo_fluid_t* f, real T) { /* :12-14 */
  return (real)(f->p_sat * exp((double)f->h_fg / f->R_gas * (1.0 / f->T_sat - 1.0 / (double)T)));
}

/* Fowler radial moment (sph_solver.cu:181-193) */
static double radial_moment4(int adhesion, double c) {
  const int n = 2000;
  const double hstep = c / n;
  double acc = 0;
  for (int k = 0; k <= n; ++k) {
    const double r = k * hstep;
    const double w = (k == 0 || k == n) ? 1.0 : (k % 2 ? 4.0 : 2.0);
    const double f = adhesion ? (double)akinci_adhesion((real)r, (real)c) : (double)akinci_cohesion((real)r, (real)c);
    acc += w * r * r * r * r * f;
  }
  return acc * hstep / 3.0;
}

/* ManeuverProfile::evaluate (sph_solver.cu:244-268) */
static void maneuver_evaluate(const Maneuver* mp, double t, V3* a, V3* omega, V3* omega_dot) {
  const int n = mp->n;
  const int rot = mp->omega != NULL;
  *omega_dot = v3(0, 0, 0);
  if (t <= mp->time[0] || n == 1) {
    *a = mp->acc[0];
    *omega = rot ? mp->omega[0] : v3(0, 0, 0);
    return;
  }
  if (t >= mp->time[n - 1]) {
    *a = mp->acc[n - 1];
    *omega = rot ? mp->omega[n - 1] : v3(0, 0, 0);
    return;
  }
  int ub = 0; /* upper_bound */
  while (ub < n && !(t < mp->time[ub])) ++ub;
  const int k = ub - 1;
  const double dt = mp->time[k + 1] - mp->time[k];
  const real f = (real)((t - mp->time[k]) / dt);
  *a = vadd(vmul(mp->acc[k], (real)1 - f), vmul(mp->acc[k + 1], f));
  if (rot) {
    *omega = vadd(vmul(mp->omega[k], (real)1 - f), vmul(mp->omega[k + 1], f));
    *omega_dot = vdiv(vsub(mp->omega[k + 1], mp->omega[k]), (real)dt);
  } else {
    *omega = v3(0, 0, 0);
  }
}

/* ------------------------------------------------------ Solver methods */
/* Solver::init_params (sph_solver.cu:292-405) */
static void init_params(Oracle* o) {
  const cryo_config_t* c = &o->cfg;
  const cryo_fluid_t* fl = &o->fluid;
  Params* P = &o->P;
  const real dx = c->dx;
  const real h = c->h_factor * dx;
  P->kernel = kparams_make(c->kernel, h);
  P->dx = dx;
  P->support2 = P->kernel.support * P->kernel.support;
  {
    double sigma0 = 0;
    const int r = (int)ceilf(P->kernel.support / dx);
    for (int k = -r; k <= r; ++k)
      for (int j = -r; j <= r; ++j)
        for (int i = -r; i <= r; ++i) sigma0 += kernel_W(&P->kernel, dx * sqrtf((real)(i * i + j * j + k * k)));
    P->vol0 = (real)(1.0 / sigma0);
  }
  P->rho0[0] = fl->rho_liquid;
  P->rho0[1] = fl->rho_vapor;
  P->mu[0] = fl->mu_liquid;
  P->mu[1] = fl->mu_vapor;
  P->k[0] = fl->k_liquid * c->conductivity_scale;
  P->k[1] = fl->k_vapor * c->conductivity_scale;
  P->cp[0] = fl->cp_liquid;
  P->cp[1] = fl->cp_vapor;
  P->mref[0] = P->rho0[0] * P->vol0;
  P->mref[1] = P->rho0[1] * P->vol0;

  const int st_on = c->surface_tension != CRYO_ST_NONE;
  const V3 cg = v3(c->gravity[0], c->gravity[1], c->gravity[2]);
  const real gmag = vnorm(cg);
  real vref = c->velocity_scale;
  if (!(vref > 0)) {
    vref = sqrtf(gmag * o->char_length);
    if (st_on) vref = maxf(vref, sqrtf(fl->sigma / (fl->rho_liquid * h)));
    vref = maxf(vref, (real)1e-3);
  }
  P->c0 = c->sound_speed > 0 ? c->sound_speed : (real)10 * vref;
  P->tait_gamma = c->tait_gamma;
  P->tait_B = P->rho0[0] * P->c0 * P->c0 / P->tait_gamma;
  P->p_bg = c->background_pressure >= 0 ? c->background_pressure
                                        : (o->has_vapor ? (real)0.1 * P->rho0[1] * P->c0 * P->c0 : (real)0);
  P->vapor_K = c->vapor_stiffness > 0 ? c->vapor_stiffness : (o->has_vapor ? P->rho0[1] * P->c0 * P->c0 : P->p_bg);
  P->gas_R = P->vapor_K > 0 ? P->vapor_K / (P->rho0[1] * fl->T_sat) : fl->R_gas;
  P->clamp_negative_pressure = c->clamp_negative_pressure ? 1 : 0;

  P->gravity = vsub(cg, o->frame_acc);
  P->alpha_av = c->artificial_viscosity;
  P->alpha_av_vap = c->artificial_viscosity_vapor;
  P->delta_sph = c->delta_sph;
  P->density_mode = c->density_mode;
  P->no_slip = c->no_slip ? 1 : 0;
  P->sps = c->sps_turbulence ? 1 : 0;
  P->smagorinsky_cs = c->smagorinsky_cs;
  P->tvf = c->transport_velocity ? 1 : 0;
  P->tvf_stress = c->transport_stress ? 1 : 0;
  P->tvf_factor = c->transport_background_factor;
  P->tvf_interface_only = c->transport_interface_only ? 1 : 0;
  P->shift_strength = c->particle_shifting ? c->shifting_strength : (real)0;
  P->tvf_sigma_min = o->has_vapor ? (real)0 : (real)0.95 / P->vol0;

  P->st_model = c->surface_tension;
  P->sigma = st_on ? fl->sigma : (real)0;
  const real theta = c->contact_angle_deg * kPi / (real)180;
  P->cos_theta = cosf(theta);
  P->sin_theta = sinf(theta);
  P->wall_adhesion_weight = c->contact_angle_wall_weight;
  P->wall_colour = c->wall_colour ? 1 : 0;
  P->wetting_model = c->wetting_model;
  P->csf_smooth_normals = c->csf_smooth_normals ? 1 : 0;
  P->csf_balanced = c->csf_balanced ? 1 : 0;
  P->normal_eps = (real)0.1 / h;
  {
    const double sup = P->kernel.support;
    const double i_coh = radial_moment4(0, sup);
    const double i_adh = radial_moment4(1, sup);
    const double rho = fl->rho_liquid;
    const double gamma = c->akinci_gamma >= 0
                             ? (double)c->akinci_gamma
                             : (i_coh > 0 ? 8.0 * fl->sigma / ((double)kPi * rho * rho * i_coh) : 0.0);
    P->akinci_gamma = (real)gamma;
    P->akinci_beta = c->akinci_beta >= 0
                         ? c->akinci_beta
                         : (real)(i_adh > 0 ? gamma * (i_coh / i_adh) * 0.5 * (1.0 + (double)P->cos_theta) : 0.0);
  }
  P->thermal = c->thermal ? 1 : 0;
  P->phase_change = c->phase_change ? 1 : 0;
  P->wall_bc = c->wall_thermal_bc;
  P->T_wall = fl->T_sat;
  P->T_ref = fl->T_sat;
  P->T_sat = fl->T_sat;
  P->h_fg = fl->h_fg;
  P->lee_evap = c->lee_evaporation;
  P->lee_cond = c->lee_condensation;
  P->max_transfer_fraction = c->max_transfer_fraction;
  P->pc_density_limit = c->phase_change_density_limit;
  P->vapor_rebalance = c->vapor_mass_rebalance;
  P->merge_ratio = c->merge_ratio;
  P->split_ratio = c->split_ratio;
  P->heat_power = c->heater_power;
  P->heat_inv_norm = 0;
  P->dt = 0;
}

/* Solver::evaluate_rates (sph_solver.cu:449-480) */
static void evaluate_rates(Oracle* o) {
  density_summation(o);
  equation_of_state(o);
  wall_boundary(o);
  interface_fields(o);
  transport_acceleration(o);
  if (o->P.sps) sps_viscosity(o);
  momentum(o);
  if (o->cfg.surface_tension == CRYO_ST_CSF && o->has_vapor) {
    smooth_normals(o);
    csf_surface_tension(o);
  } else if (o->cfg.surface_tension == CRYO_ST_AKINCI) {
    akinci_surface_tension(o);
  }
  if (o->cfg.density_mode == CRYO_DENSITY_CONTINUITY) density_rate(o);
  if (o->P.thermal) {
    if (o->P.heat_power != (real)0) {
      const double S = sum_heat_weight(o);
      o->P.heat_inv_norm = S > 0 ? (real)(1.0 / S) : (real)0;
    } else {
      o->P.heat_inv_norm = 0;
    }
    thermal_rates(o);
  }
  o->v_max = max_fluid_speed(o);
  o->spacing_ratio = max_spacing_ratio(o);
  o->a_max = max_fluid_accel(o);
  o->Tv_max = o->has_vapor ? max_phase_T(o, VAP) : (real)0;
  o->nu_t_max = o->P.sps ? max_eddy_viscosity(o) : (real)0;
}

/* Solver::compute_dt (sph_solver.cu:482-504) */
static real compute_dt(const Oracle* o) {
  const cryo_config_t* c = &o->cfg;
  const Params* P = &o->P;
  if (c->fixed_dt > 0) return c->fixed_dt;
  const real h = P->kernel.h;
  real c_max = P->c0;
  if (o->has_vapor) c_max = maxf(c_max, sqrtf(P->gas_R * maxf(o->Tv_max, P->T_ref)));
  real dt = c->cfl * h / ((c_max + o->v_max) * maxf((real)1, o->spacing_ratio));
  const real nu = maxf(P->mu[0] / P->rho0[0], P->mu[1] / P->rho0[1]) + o->nu_t_max;
  if (nu > 0) dt = minf(dt, c->viscous_number * h * h / nu);
  if (o->a_max > 0) dt = minf(dt, c->force_number * sqrtf(h / o->a_max));
  if (P->sigma > 0) {
    const real rho_avg = (real)0.5 * (P->rho0[0] + (o->has_vapor ? P->rho0[1] : P->rho0[0]));
    dt = minf(dt, c->capillary_number * sqrtf(rho_avg * h * h * h / ((real)2 * kPi * P->sigma)));
  }
  if (P->thermal) {
    real alpha = P->k[0] / (P->rho0[0] * P->cp[0]);
    if (o->has_vapor) alpha = maxf(alpha, P->k[1] / (P->rho0[1] * P->cp[1]));
    if (alpha > 0) dt = minf(dt, c->thermal_number * h * h / alpha);
  }
  /* std::clamp(dt, dt_min, dt_max) */
  return dt < c->dt_min ? c->dt_min : (c->dt_max < dt ? c->dt_max : dt);
}

/* Solver::update_saturation (sph_solver.cu:586-607) */
static void update_saturation(Oracle* o) {
  if (o->cfg.thermo_mode == CRYO_THERMO_CLOSED && o->has_vapor) {
    const double m_liq = phase_sum(o, LIQ, 0);
    const double m_vap = phase_sum(o, VAP, 0);
    const double mT_vap = phase_sum(o, VAP, 1);
    if (!(o->fluid_volume0 > 0)) o->fluid_volume0 = m_liq / o->fluid.rho_liquid + m_vap / o->fluid.rho_vapor;
    const double v_ullage = o->fluid_volume0 - m_liq / o->fluid.rho_liquid;
    const double ratio =
        v_ullage > 0 && m_vap > 0 ? (mT_vap / v_ullage) / ((double)o->fluid.rho_vapor * o->fluid.T_sat) : 0.0;
    if (isfinite(ratio) && ratio > 0) {
      o->p_ullage = o->fluid.p_sat * ratio;
      o->P.T_sat = saturation_temperature(&o->fluid, (real)o->p_ullage);
      return;
    }
  }
  o->p_ullage = o->fluid.p_sat;
  o->P.T_sat = o->fluid.T_sat;
}

/* Solver::phase_change_step (sph_solver.cu:545-584) */
static void phase_change_step(Oracle* o) {
  pc_sources(o);
  pc_normalize(o);
  o->evaporated += sum_phase_change(o, 1);
  o->condensed += sum_phase_change(o, 0);
  o->merges += count_merges(o);
  pc_apply(o);
  if (o->P.vapor_rebalance > (real)0 && o->has_vapor) rebalance_vapor(o);
  if ((long long)o->ps.n * 4 > (long long)o->ps.capacity * 3) ps_grow(&o->ps, o->ps.capacity * 3 / 2 + 1024);
  if (o->split_cap < o->ps.capacity) {
    free(o->split_flag); free(o->split_offset);
    ALLOC(o->split_flag, o->ps.capacity);
    ALLOC(o->split_offset, o->ps.capacity);
    o->split_cap = o->ps.capacity;
  }
  mark_heavy(o, o->split_flag);
  unsigned requested = 0;
  for (int i = 0; i < o->ps.n; ++i) { /* exclusive_scan, CPU branch (cuda_utils.cuh:341-349) */
    const unsigned v = o->split_flag[i];
    o->split_offset[i] = requested;
    requested += v;
  }
  if (requested > 0) {
    split_heavy(o, o->split_flag, o->split_offset, o->ps.next_id, (unsigned)o->step);
    const long long room = (long long)o->ps.capacity - o->ps.n;
    const long long added = (long long)requested < room ? (long long)requested : room;
    o->ps.n += (int)added;
    o->ps.next_id += requested;
    o->splits += (int)added;
  }
  if (o->cfg.thermo_mode == CRYO_THERMO_VENTED && o->has_vapor) {
    venting(o, o->cfg.vent_relaxation);
    o->vented += sum_out_mass(o);
    o->vented_h += sum_out_enthalpy(o);
  }
}

/* Solver::ensure_initialized (sph_solver.cu:439-447) */
static int ensure_initialized(Oracle* o) {
  if (o->initialized) return CRYO_OK;
  if (o->ps.n == 0) { snprintf(o->err, sizeof o->err, "Solver: no particles loaded"); return CRYO_ERUNTIME; }
  grid_build(o);
  if (o->cfg.normalize_initial_masses) normalize_initial_masses(o);
  evaluate_rates(o);
  update_saturation(o);
  o->initialized = 1;
  return CRYO_OK;
}

/* Solver::apply_frame (sph_solver.cu:660-667) */
static void apply_frame(Oracle* o, V3 a, V3 w, V3 wdot, V3 origin) {
  o->frame_acc = a;
  o->P.gravity = vsub(v3(o->cfg.gravity[0], o->cfg.gravity[1], o->cfg.gravity[2]), a);
  o->P.omega = w;
  o->P.omega_dot = wdot;
  o->P.frame_origin = origin;
  o->P.frame_rot = (vnorm2(w) > (real)0 || vnorm2(wdot) > (real)0) ? 1 : 0;
}

/* Solver::step (sph_solver.cu:511-533) */
static int solver_step(Oracle* o) {
  int rc = ensure_initialized(o);
  if (rc) return rc;
  const real dt = compute_dt(o);
  o->P.dt = dt;
  kick_drift(o, dt, o->cfg.density_mode == CRYO_DENSITY_CONTINUITY, o->P.tvf);
  grid_build(o);
  if (o->has_maneuver) {
    V3 a, w, wd;
    maneuver_evaluate(&o->man, o->time + dt, &a, &w, &wd);
    apply_frame(o, a, w, wd, o->man.origin);
  }
  evaluate_rates(o);
  kick(o, dt, o->P.thermal);
  if (o->P.shift_strength > (real)0) particle_shifting(o, o->v_max / o->P.c0);
  if (o->P.thermal && o->P.heat_inv_norm > 0) o->heat_input += (double)o->P.heat_power * dt;
  if (o->cfg.phase_change) phase_change_step(o);
  update_saturation(o);
  o->time += dt;
  ++o->step;
  o->last_dt = dt;
  return CRYO_OK;
}

/* ------------------------------------------------------------- C API */
int orc_real_size(void) { return (int)sizeof(real); }
void orc_set_threads(int n) { (void)n; }
int orc_get_threads(void) { return 1; }

/* Solver::Solver (sph_solver.cu:273-279) */
void* orc_create(const cryo_config_t* cfg, const cryo_fluid_t* fluid, char* err, int errlen) {
  if (!(cfg->dx > 0)) {
    if (err) snprintf(err, (size_t)errlen, "SolverConfig.dx must be > 0");
    return NULL;
  }
  if (cfg->contact_angle_deg < 0 || cfg->contact_angle_deg > 180) {
    if (err) snprintf(err, (size_t)errlen, "contact angle must be within [0, 180] degrees");
    return NULL;
  }
  Oracle* o = calloc(1, sizeof(Oracle));
  o->cfg = *cfg;
  o->fluid = *fluid;
  o->p_ullage = fluid->p_sat;
  o->spacing_ratio = 1;
  return o;
}

void orc_destroy(void* h) {
  Oracle* o = h;
  if (!o) return;
  ps_free(&o->ps);
  free(o->grid.cell_start); free(o->grid.cell_end); free(o->grid.keys); free(o->grid.perm);
  free(o->split_flag); free(o->split_offset);
  free(o->man.time); free(o->man.acc); free(o->man.omega);
  free(o);
}

const char* orc_last_error(void* h) { return ((Oracle*)h)->err; }

/* Solver::set_particles (sph_solver.cu:407-428) + ParticleSystem::upload
 * (particle_system.cpp:73-93) */
int orc_set_particles(void* h, const cryo_host_particles_t* p, const float* lo, const float* hi) {
  Oracle* o = h;
  const int n = p->n;
  if (n == 0) { snprintf(o->err, sizeof o->err, "Solver::set_particles: no particles"); return CRYO_EINVAL; }
  o->has_vapor = 0;
  for (int i = 0; i < n; ++i)
    if (p->phase[i] == VAP) o->has_vapor = 1;
  if (o->has_vapor && o->cfg.surface_tension == CRYO_ST_AKINCI) {
    snprintf(o->err, sizeof o->err,
             "Solver: the Akinci surface-tension model is a free-surface (liquid-only) model; use CSF when vapour "
             "particles are present (FillSpec.include_vapor = false for Akinci runs)");
    return CRYO_EINVAL;
  }
  const V3 ext = vsub(v3(hi[0], hi[1], hi[2]), v3(lo[0], lo[1], lo[2]));
  o->char_length = maxf(maxf(ext.x, ext.y), ext.z);
  /* std::max({a, b, c}) returns the first largest */
  {
    real m = ext.x;
    if (m < ext.y) m = ext.y;
    if (m < ext.z) m = ext.z;
    o->char_length = m;
  }
  init_params(o);
  {
    long long cap2 = (long long)((double)n * 2.0);
    long long cap = cap2 > (long long)n + 1024 ? cap2 : (long long)n + 1024;
    if (cap > o->ps.capacity) ps_allocate(&o->ps, (int)cap);
  }
  Particles* s = &o->ps;
  for (int i = 0; i < n; ++i) {
    s->x[i] = v3(p->x[3 * i], p->x[3 * i + 1], p->x[3 * i + 2]);
    s->v[i] = p->v ? v3(p->v[3 * i], p->v[3 * i + 1], p->v[3 * i + 2]) : v3(0, 0, 0);
    s->vt[i] = s->v[i];
    s->nrm[i] = p->nrm ? v3(p->nrm[3 * i], p->nrm[3 * i + 1], p->nrm[3 * i + 2]) : v3(0, 0, 0);
    s->m[i] = p->m[i];
    s->m0[i] = p->m[i];
    s->rho[i] = p->rho[i];
    s->T[i] = p->T[i];
    s->phase[i] = p->phase[i];
    s->flags[i] = p->flags ? p->flags[i] : 0;
    s->id[i] = p->id ? p->id[i] : (unsigned)i;
  }
  const int cap = s->capacity;
  memset(s->a, 0, (size_t)cap * sizeof(V3)); memset(s->ab, 0, (size_t)cap * sizeof(V3));
  memset(s->ns, 0, (size_t)cap * sizeof(V3)); memset(s->vw, 0, (size_t)cap * sizeof(V3));
  memset(s->fw, 0, (size_t)cap * sizeof(V3)); memset(s->mw, 0, (size_t)cap * sizeof(V3));
  memset(s->p, 0, (size_t)cap * sizeof(real)); memset(s->drho, 0, (size_t)cap * sizeof(real));
  memset(s->dTdt, 0, (size_t)cap * sizeof(real)); memset(s->sigma, 0, (size_t)cap * sizeof(real));
  memset(s->kappa, 0, (size_t)cap * sizeof(real)); memset(s->nu_t, 0, (size_t)cap * sizeof(real));
  memset(s->alpha, 0, (size_t)cap * sizeof(real)); memset(s->wall_w, 0, (size_t)cap * sizeof(real));
  memset(s->heat_w, 0, (size_t)cap * sizeof(real)); memset(s->out_m, 0, (size_t)cap * sizeof(real));
  memset(s->out_h, 0, (size_t)cap * sizeof(real)); memset(s->w_norm, 0, (size_t)cap * sizeof(real));
  memset(s->p_wv, 0, (size_t)cap * sizeof(real));
  s->n = n;
  s->next_id = 0;
  for (int i = 0; i < n; ++i)
    if (s->id[i] + 1 > s->next_id) s->next_id = s->id[i] + 1;
  int rc = grid_configure(o, v3(lo[0], lo[1], lo[2]), v3(hi[0], hi[1], hi[2]), o->P.kernel.support);
  if (rc) return rc;
  o->initialized = 0;
  o->time = 0;
  o->step = 0;
  o->last_dt = 0;
  o->heat_input = o->evaporated = o->condensed = o->vented = o->vented_h = 0;
  o->splits = o->merges = 0;
  o->p_ullage = o->fluid.p_sat;
  o->fluid_volume0 = 0;
  return CRYO_OK;
}

int orc_step(void* h, long long n) {
  Oracle* o = h;
  for (long long k = 0; k < n; ++k) {
    int rc = solver_step(o);
    if (rc) return rc;
  }
  return CRYO_OK;
}

int orc_run_until(void* h, double t_end) {
  Oracle* o = h;
  while (o->time < t_end) {
    int rc = solver_step(o);
    if (rc) return rc;
  }
  return CRYO_OK;
}

/* Solver::relax (sph_solver.cu:707-736) */
int orc_relax(void* h, double duration, float damping) {
  Oracle* o = h;
  int rc = ensure_initialized(o);
  if (rc) return rc;
  const int thermal = o->P.thermal;
  const int phase_change = o->cfg.phase_change;
  o->P.thermal = 0;
  o->cfg.phase_change = 0;
  const double t_end = o->time + duration;
  while (o->time < t_end) {
    rc = solver_step(o);
    if (rc) break;
    scale_velocities(o, damping);
  }
  o->P.thermal = thermal;
  o->cfg.phase_change = phase_change;
  if (rc) return rc;
  scale_velocities(o, 0);
  o->time = 0;
  o->step = 0;
  o->last_dt = 0;
  o->heat_input = o->evaporated = o->condensed = o->vented = o->vented_h = 0;
  o->splits = o->merges = 0;
  evaluate_rates(o);
  update_saturation(o);
  return CRYO_OK;
}

int orc_next_dt(void* h, double* dt) {
  Oracle* o = h;
  int rc = ensure_initialized(o);
  if (rc) return rc;
  *dt = compute_dt(o);
  return CRYO_OK;
}

int orc_time(void* h, double* t, long long* step, double* last_dt) {
  Oracle* o = h;
  *t = o->time;
  *step = o->step;
  *last_dt = o->last_dt;
  return CRYO_OK;
}

int orc_num_particles(void* h) { return ((Oracle*)h)->ps.n; }

/* Solver::diagnostics (sph_solver.cu:609-653) */
int orc_diagnostics(void* h, cryo_diagnostics_t* d) {
  Oracle* o = h;
  int rc = ensure_initialized(o);
  if (rc) return rc;
  memset(d, 0, sizeof(*d));
  d->time = o->time;
  d->step = o->step;
  d->dt = o->last_dt;
  d->n_total = o->ps.n;
  d->n_liquid = count_phase(o, LIQ);
  d->n_vapor = count_phase(o, VAP);
  d->n_wall = count_phase(o, WALL);
  d->mass_liquid = phase_sum(o, LIQ, 0);
  d->mass_vapor = phase_sum(o, VAP, 0);
  d->mass_total = d->mass_liquid + d->mass_vapor;
  d->kinetic_energy = phase_sum(o, LIQ, 2) + phase_sum(o, VAP, 2);
  d->enthalpy = phase_sum(o, LIQ, 9) + phase_sum(o, VAP, 9);
  d->heat_input = o->heat_input;
  d->evaporated_mass = o->evaporated;
  d->condensed_mass = o->condensed;
  d->vented_mass = o->vented;
  d->vented_enthalpy = o->vented_h;
  d->T_sat = o->P.T_sat;
  d->p_ullage = o->p_ullage;
  d->max_speed = max_fluid_speed(o);
  if (d->mass_liquid > 0) {
    d->T_liquid_mean = phase_sum(o, LIQ, 1) / d->mass_liquid;
    d->T_liquid_max = max_phase_T(o, LIQ);
    d->liquid_com[0] = (float)(phase_sum(o, LIQ, 3) / d->mass_liquid);
    d->liquid_com[1] = (float)(phase_sum(o, LIQ, 4) / d->mass_liquid);
    d->liquid_com[2] = (float)(phase_sum(o, LIQ, 5) / d->mass_liquid);
    d->liquid_momentum[0] = (float)phase_sum(o, LIQ, 6);
    d->liquid_momentum[1] = (float)phase_sum(o, LIQ, 7);
    d->liquid_momentum[2] = (float)phase_sum(o, LIQ, 8);
  }
  if (d->mass_vapor > 0) d->T_vapor_mean = phase_sum(o, VAP, 1) / d->mass_vapor;
  d->splits = o->splits;
  d->merges = o->merges;
  const V3 f = vneg(sum_fluid_vec3(o, o->ps.fw));
  const V3 m = vneg(sum_fluid_vec3(o, o->ps.mw));
  d->slosh_force[0] = f.x; d->slosh_force[1] = f.y; d->slosh_force[2] = f.z;
  d->slosh_moment[0] = m.x; d->slosh_moment[1] = m.y; d->slosh_moment[2] = m.z;
  d->frame_acceleration[0] = o->frame_acc.x;
  d->frame_acceleration[1] = o->frame_acc.y;
  d->frame_acceleration[2] = o->frame_acc.z;
  d->frame_angular_velocity[0] = o->P.omega.x;
  d->frame_angular_velocity[1] = o->P.omega.y;
  d->frame_angular_velocity[2] = o->P.omega.z;
  return CRYO_OK;
}

static void* field_ptr(Oracle* o, int field, size_t* elem) {
  Particles* s = &o->ps;
  *elem = sizeof(real);
  switch (field) {
    case CRYO_F_X: *elem = sizeof(V3); return s->x;
    case CRYO_F_V: *elem = sizeof(V3); return s->v;
    case CRYO_F_VT: *elem = sizeof(V3); return s->vt;
    case CRYO_F_NRM: *elem = sizeof(V3); return s->nrm;
    case CRYO_F_M: return s->m;
    case CRYO_F_M0: return s->m0;
    case CRYO_F_RHO: return s->rho;
    case CRYO_F_T: return s->T;
    case CRYO_F_PHASE: *elem = 1; return s->phase;
    case CRYO_F_FLAGS: *elem = 1; return s->flags;
    case CRYO_F_ID: *elem = 4; return s->id;
    case CRYO_F_A: *elem = sizeof(V3); return s->a;
    case CRYO_F_AB: *elem = sizeof(V3); return s->ab;
    case CRYO_F_FW: *elem = sizeof(V3); return s->fw;
    case CRYO_F_MW: *elem = sizeof(V3); return s->mw;
    case CRYO_F_NS: *elem = sizeof(V3); return s->ns;
    case CRYO_F_VW: *elem = sizeof(V3); return s->vw;
    case CRYO_F_P: return s->p;
    case CRYO_F_DRHO: return s->drho;
    case CRYO_F_DTDT: return s->dTdt;
    case CRYO_F_SIGMA: return s->sigma;
    case CRYO_F_KAPPA: return s->kappa;
    case CRYO_F_NU_T: return s->nu_t;
    case CRYO_F_ALPHA: return s->alpha;
    case CRYO_F_WALL_W: return s->wall_w;
    case CRYO_F_HEAT_W: return s->heat_w;
    case CRYO_F_OUT_M: return s->out_m;
    case CRYO_F_OUT_H: return s->out_h;
    case CRYO_F_W_NORM: return s->w_norm;
    case CRYO_F_RMIN: return s->rmin;
    case CRYO_F_P_WV: return s->p_wv;
    default: return NULL;
  }
}

int orc_get_field(void* h, int field, void* out) {
  Oracle* o = h;
  size_t elem;
  void* p = field_ptr(o, field, &elem);
  if (!p) { snprintf(o->err, sizeof o->err, "unknown field"); return CRYO_EINVAL; }
  memcpy(out, p, elem * (size_t)o->ps.n);
  return CRYO_OK;
}

int orc_set_field(void* h, int field, const void* in) {
  Oracle* o = h;
  size_t elem;
  void* p = field_ptr(o, field, &elem);
  if (!p) { snprintf(o->err, sizeof o->err, "unknown field"); return CRYO_EINVAL; }
  memcpy(p, in, elem * (size_t)o->ps.n);
  return CRYO_OK;
}

int orc_params(void* h, float* c0, float* hsm, float* vol0, float* support2, float* T_sat, float* dt,
               float* heat_inv_norm) {
  Oracle* o = h;
  *c0 = o->P.c0;
  *hsm = o->P.kernel.h;
  *vol0 = o->P.vol0;
  *support2 = o->P.support2;
  *T_sat = o->P.T_sat;
  *dt = o->P.dt;
  *heat_inv_norm = o->P.heat_inv_norm;
  return CRYO_OK;
}

int orc_scalars(void* h, double* out) {
  Oracle* o = h;
  out[0] = o->p_ullage;
  out[1] = o->fluid_volume0;
  out[2] = o->v_max;
  out[3] = o->a_max;
  out[4] = o->Tv_max;
  out[5] = o->spacing_ratio;
  out[6] = o->nu_t_max;
  out[7] = o->heat_input;
  return CRYO_OK;
}

int orc_set_gravity(void* h, const float* g) { /* sph_solver.cu:655-658 */
  Oracle* o = h;
  o->cfg.gravity[0] = g[0]; o->cfg.gravity[1] = g[1]; o->cfg.gravity[2] = g[2];
  o->P.gravity = vsub(v3(g[0], g[1], g[2]), o->frame_acc);
  return CRYO_OK;
}

int orc_set_frame_motion(void* h, const float* a, const float* w, const float* wd, const float* og) {
  Oracle* o = h; /* sph_solver.cu:669-672 */
  o->has_maneuver = 0;
  apply_frame(o, v3(a[0], a[1], a[2]), v3(w[0], w[1], w[2]), v3(wd[0], wd[1], wd[2]), v3(og[0], og[1], og[2]));
  return CRYO_OK;
}

int orc_set_maneuver(void* h, int n, const double* t, const float* acc, const float* omega, const float* og) {
  Oracle* o = h; /* ManeuverProfile::validate (sph_solver.cu:234-242) + set_maneuver (:674-681) */
  if (n <= 0) { snprintf(o->err, sizeof o->err, "ManeuverProfile: empty time table"); return CRYO_EINVAL; }
  for (int k = 1; k < n; ++k)
    if (!(t[k] > t[k - 1])) {
      snprintf(o->err, sizeof o->err, "ManeuverProfile: time must be strictly increasing");
      return CRYO_EINVAL;
    }
  free(o->man.time); free(o->man.acc); free(o->man.omega);
  o->man.n = n;
  o->man.time = malloc((size_t)n * sizeof(double));
  o->man.acc = malloc((size_t)n * sizeof(V3));
  o->man.omega = omega ? malloc((size_t)n * sizeof(V3)) : NULL;
  for (int k = 0; k < n; ++k) {
    o->man.time[k] = t[k];
    o->man.acc[k] = v3(acc[3 * k], acc[3 * k + 1], acc[3 * k + 2]);
    if (omega) o->man.omega[k] = v3(omega[3 * k], omega[3 * k + 1], omega[3 * k + 2]);
  }
  o->man.origin = og ? v3(og[0], og[1], og[2]) : v3(0, 0, 0);
  o->has_maneuver = 1;
  V3 a, w, wd;
  maneuver_evaluate(&o->man, o->time, &a, &w, &wd);
  apply_frame(o, a, w, wd, o->man.origin);
  return CRYO_OK;
}

int orc_clear_frame_motion(void* h) { /* sph_solver.cu:683-686 */
  Oracle* o = h;
  o->has_maneuver = 0;
  apply_frame(o, v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0));
  return CRYO_OK;
}

int orc_set_heater_power(void* h, float w) { /* sph_solver.cu:688-691 */
  Oracle* o = h;
  o->cfg.heater_power = w;
  o->P.heat_power = w;
  return CRYO_OK;
}

int orc_set_contact_angle(void* h, float deg) { /* sph_solver.cu:693-699 */
  Oracle* o = h;
  if (deg < 0 || deg > 180) {
    snprintf(o->err, sizeof o->err, "contact angle must be within [0, 180] degrees");
    return CRYO_EINVAL;
  }
  o->cfg.contact_angle_deg = deg;
  const real theta = deg * kPi / (real)180;
  o->P.cos_theta = cosf(theta);
  o->P.sin_theta = sinf(theta);
  return CRYO_OK;
}

int orc_damp_velocities(void* h, float f) { /* sph_solver.cu:701-705 */
  Oracle* o = h;
  scale_velocities(o, f);
  o->v_max *= f;
  return CRYO_OK;
}

/* probe_liquid_pressure (sph_solver.cu:197-216) + Solver::probe_pressure (:738-748) */
int orc_probe_pressure(void* h, const float* pts, int np, float* out) {
  Oracle* o = h;
  int rc = ensure_initialized(o);
  if (rc) return rc;
  const Particles* s = &o->ps;
  const Params* P = &o->P;
  const Grid* g = &o->grid;
  for (int k = 0; k < np; ++k) {
    const V3 x = v3(pts[3 * k], pts[3 * k + 1], pts[3 * k + 2]);
    real num = 0, den = 0;
    FOR_EACH_NEIGHBOR(g, x, j, {
      if (s->phase[j] != LIQ) continue;
      const real r2 = vnorm2(vsub(x, s->x[j]));
      if (r2 >= P->support2) continue;
      const real w = (s->m[j] / s->rho[j]) * kernel_W(&P->kernel, sqrtf(r2));
      num += s->p[j] * w;
      den += w;
    });
    out[k] = den > (real)0 ? num / den : NAN;
  }
  return CRYO_OK;
}

int orc_set_dt(void* h, float dt) {
  ((Oracle*)h)->pass_dt = dt;
  return CRYO_OK;
}

/* Operator hooks with the semantics of the reference free functions. */
int orc_pass(void* h, int pass) {
  Oracle* o = h;
  o->P.dt = o->pass_dt;
  switch (pass) {
    case CRYO_PASS_KICK_DRIFT:
      kick_drift(o, o->P.dt, o->cfg.density_mode == CRYO_DENSITY_CONTINUITY, o->P.tvf);
      break;
    case CRYO_PASS_GRID_BUILD: grid_build(o); break;
    case CRYO_PASS_DENSITY: density_summation(o); break;
    case CRYO_PASS_NORMALIZE_MASSES: normalize_initial_masses(o); break;
    case CRYO_PASS_EOS: equation_of_state(o); break;
    case CRYO_PASS_WALL_BOUNDARY: wall_boundary(o); break;
    case CRYO_PASS_INTERFACE: interface_fields(o); break;
    case CRYO_PASS_TRANSPORT: transport_acceleration(o); break;
    case CRYO_PASS_SPS: sps_viscosity(o); break;
    case CRYO_PASS_MOMENTUM: momentum(o); break;
    case CRYO_PASS_SMOOTH_NORMALS: smooth_normals(o); break;
    case CRYO_PASS_CSF: csf_surface_tension(o); break;
    case CRYO_PASS_AKINCI: akinci_surface_tension(o); break;
    case CRYO_PASS_DENSITY_RATE: density_rate(o); break;
    case CRYO_PASS_THERMAL:
      if (o->P.heat_power != (real)0) {
        const double S = sum_heat_weight(o);
        o->P.heat_inv_norm = S > 0 ? (real)(1.0 / S) : (real)0;
      } else {
        o->P.heat_inv_norm = 0;
      }
      thermal_rates(o);
      break;
    case CRYO_PASS_MAXIMA:
      o->v_max = max_fluid_speed(o);
      o->spacing_ratio = max_spacing_ratio(o);
      o->a_max = max_fluid_accel(o);
      o->Tv_max = o->has_vapor ? max_phase_T(o, VAP) : (real)0;
      o->nu_t_max = o->P.sps ? max_eddy_viscosity(o) : (real)0;
      break;
    case CRYO_PASS_KICK: kick(o, o->P.dt, o->P.thermal); break;
    case CRYO_PASS_SHIFTING: particle_shifting(o, o->v_max / o->P.c0); break;
    case CRYO_PASS_PC_SOURCES: pc_sources(o); break;
    case CRYO_PASS_PC_NORMALIZE: pc_normalize(o); break;
    case CRYO_PASS_PC_APPLY: pc_apply(o); break;
    case CRYO_PASS_REBALANCE: rebalance_vapor(o); break;
    case CRYO_PASS_VENTING: venting(o, o->cfg.vent_relaxation); break;
    case CRYO_PASS_SATURATION: update_saturation(o); break;
    default: snprintf(o->err, sizeof o->err, "pass not exposed by the oracle"); return CRYO_EINVAL;
  }
  return CRYO_OK;
}

int orc_grid_info(void* h, int* num_cells, int* nx, int* ny, int* nz, float* origin, float* inv_cell) {
  Oracle* o = h;
  *num_cells = o->grid.num_cells;
  *nx = o->grid.nx; *ny = o->grid.ny; *nz = o->grid.nz;
  origin[0] = o->grid.origin.x; origin[1] = o->grid.origin.y; origin[2] = o->grid.origin.z;
  *inv_cell = o->grid.inv_cell;
  return CRYO_OK;
}

int orc_grid_tables(void* h, int32_t* cs, int32_t* ce) {
  Oracle* o = h;
  memcpy(cs, o->grid.cell_start, (size_t)o->grid.num_cells * sizeof(int));
  memcpy(ce, o->grid.cell_end, (size_t)o->grid.num_cells * sizeof(int));
  return CRYO_OK;
}

int orc_grid_sort(void* h, uint32_t* keys, uint32_t* perm) {
  Oracle* o = h;
  const int n = o->grid.keys_n < o->ps.n ? o->grid.keys_n : o->ps.n;
  memcpy(keys, o->grid.keys, (size_t)n * sizeof(unsigned));
  memcpy(perm, o->grid.perm, (size_t)n * sizeof(unsigned));
  return CRYO_OK;
}

int orc_neighbor_lists(void* h, int32_t* counts, int32_t* list, long long cap, long long* total) {
  Oracle* o = h;
  const Particles* s = &o->ps;
  const Grid* g = &o->grid;
  long long t = 0;
  for (int i = 0; i < s->n; ++i) {
    const V3 xi = s->x[i];
    int c = 0;
    FOR_EACH_NEIGHBOR(g, xi, j, {
      if (vnorm2(vsub(xi, s->x[j])) < o->P.support2) {
        if (list && t < cap) list[t] = j;
        ++t;
        ++c;
      }
    });
    counts[i] = c;
  }
  *total = t;
  return CRYO_OK;
}

/* exported for the tests of the host helpers */
float orc_saturation_temperature(const cryo_fluid_t* f, float p) { return saturation_temperature(f, p); }
float orc_saturation_pressure(const cryo_fluid_t* f, float T) { return saturation_pressure(f, T); }
