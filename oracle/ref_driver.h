/*
 * ref_driver.h -- C ABI over the CryoSPH-CUDA reference built for the CPU
 * (OpenMP backend) from its own sources (see oracle/Makefile).  TEST
 * INFRASTRUCTURE ONLY: used by tests/, the smoke check and bench.py's CPU
 * baseline to pin the oracle restatement and to time the reference.  Nothing
 * in the product links or loads it.
 *
 * The same header serves the FP32 build (libcryoref.so) and the FP64 build
 * (libcryoref64.so, CRYOSPH_DOUBLE_PRECISION); ref_real_size() tells which.
 */
#ifndef CRYOSPH_REF_DRIVER_H
#define CRYOSPH_REF_DRIVER_H

#include "../include/cryosph_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Geometry description shared by the oracle and the tests: a node list whose
 * last entry is the root.  Kinds follow geometry.hpp:37-140. */
enum {
  REF_GEOM_CYLINDER = 0, /* p = {R, H}          */
  REF_GEOM_CAPSULE = 1,  /* p = {R, L}          */
  REF_GEOM_SPHERE = 2,   /* p = {R}             */
  REF_GEOM_BOX = 3,      /* p = {lx, ly, lz}    */
  REF_GEOM_TRANSLATED = 4, /* a, p = {ox, oy, oz} */
  REF_GEOM_DIFFERENCE = 5, /* a - b              */
  REF_GEOM_UNION = 6       /* a U b              */
};
typedef struct ref_geom_node {
  int kind;
  int a, b;
  double p[3];
} ref_geom_node_t;

/* FillSpec (geometry.hpp:166-181). NaN temperatures mean T_sat. */
typedef struct ref_fill {
  int mode;
  double fill_fraction;
  float settle_direction[3];
  float bubble_center[3];
  int include_vapor;
  int wall_layers;
  float T_liquid, T_vapor, T_wall;
  double heater_zmin, heater_zmax;
} ref_fill_t;

int ref_real_size(void);
void ref_set_threads(int n);
int ref_get_threads(void);

void* ref_create(const cryo_config_t* cfg, const cryo_fluid_t* fluid, char* err, int errlen);
void ref_destroy(void* h);
const char* ref_last_error(void* h);

int ref_set_particles(void* h, const cryo_host_particles_t* p, const float* lo, const float* hi);
int ref_build_tank(void* h, const ref_geom_node_t* nodes, int n_nodes, const ref_fill_t* fill);
/* Lattice generator only (build_tank_particles, geometry.cpp:242-330).  The
 * arrays are malloc'ed by the driver; release with ref_free_particles. */
int ref_tank_particles(const ref_geom_node_t* nodes, int n_nodes, const cryo_fluid_t* fluid, float dx,
                       const ref_fill_t* fill, cryo_host_particles_out_t* out);
void ref_free_particles(cryo_host_particles_out_t* out);
/* Domain padding used by Solver::build_tank (sph_solver.cu:430-437). */
int ref_tank_domain(const ref_geom_node_t* nodes, int n_nodes, float dx, int wall_layers, float* lo, float* hi);
double ref_geom_sdf(const ref_geom_node_t* nodes, int n_nodes, double x, double y, double z);

int ref_step(void* h, long long n);
int ref_run_until(void* h, double t_end);
int ref_relax(void* h, double duration, float damping);
int ref_next_dt(void* h, double* dt);
int ref_time(void* h, double* t, long long* step, double* last_dt);
int ref_num_particles(void* h);
int ref_diagnostics(void* h, cryo_diagnostics_t* d);
/* Field CRYO_F_* in the build's real type (vectors: 3 reals per particle;
 * phase/flags: u8; id: u32). */
int ref_get_field(void* h, int field, void* out);
int ref_params(void* h, float* c0, float* hsm, float* vol0, float* support2, float* T_sat, float* dt,
               float* heat_inv_norm);

int ref_set_gravity(void* h, const float* g);
int ref_set_frame_motion(void* h, const float* a, const float* w, const float* wd, const float* o);
int ref_set_maneuver(void* h, int n, const double* t, const float* acc, const float* omega, const float* o);
int ref_clear_frame_motion(void* h);
int ref_set_heater_power(void* h, float w);
int ref_set_contact_angle(void* h, float deg);
int ref_damp_velocities(void* h, float f);
int ref_probe_pressure(void* h, const float* pts, int np, float* out);

/* Operator-level hooks: run one reference free function (CRYO_PASS_*) on the
 * solver's current state, with SimParams::dt = the value given to ref_set_dt. */
int ref_pass(void* h, int pass);
int ref_set_dt(void* h, float dt);
/* Grid tables of the last build: nx,ny,nz, origin, cell_start/end (num_cells). */
int ref_grid_info(void* h, int* num_cells, int* nx, int* ny, int* nz, float* origin, float* inv_cell);
int ref_grid_tables(void* h, int32_t* cell_start, int32_t* cell_end);
/* Neighbour lists of the current state in for_each_neighbor order, r^2 < support^2. */
int ref_neighbor_lists(void* h, int32_t* counts, int32_t* list, long long cap, long long* total);
/* SpatialHash::neighbor_stats (spatial_hash.cu:140-171). */
int ref_neighbor_stats(void* h, float radius, int32_t* counts, uint64_t* id_sums);

#ifdef __cplusplus
}
#endif
#endif
