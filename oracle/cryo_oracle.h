/*
 * cryo_oracle.h -- plain-C restatement of the CryoSPH per-step particle hot
 * path.  TEST INFRASTRUCTURE ONLY: it is the checker the CUDA path is compared
 * against (tests/, the smoke check and bench.py's CPU baseline); the product
 * never links or loads it.
 *
 * Parity pinned: the tests run it next to the reference's own CPU build
 * (oracle/_ref) on identical inputs with one OpenMP thread and require
 * bit-identical particle state and diagnostics (tests/test_oracle_vs_ref.py),
 * and against committed golden vectors made by that build
 * (tests/golden/make_golden.py).
 *
 * Surface: the same functions as ref_driver.h with the prefix orc_ instead of
 * ref_ (minus the lattice generator), plus orc_set_field to inject state.
 */
#ifndef CRYOSPH_ORACLE_H
#define CRYOSPH_ORACLE_H

#include "../include/cryosph_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

int orc_real_size(void);
void orc_set_threads(int n);
int orc_get_threads(void);
void* orc_create(const cryo_config_t* cfg, const cryo_fluid_t* fluid, char* err, int errlen);
void orc_destroy(void* h);
const char* orc_last_error(void* h);
int orc_set_particles(void* h, const cryo_host_particles_t* p, const float* lo, const float* hi);
int orc_step(void* h, long long n);
int orc_run_until(void* h, double t_end);
int orc_relax(void* h, double duration, float damping);
int orc_next_dt(void* h, double* dt);
int orc_time(void* h, double* t, long long* step, double* last_dt);
int orc_num_particles(void* h);
int orc_diagnostics(void* h, cryo_diagnostics_t* d);
int orc_get_field(void* h, int field, void* out);
int orc_set_field(void* h, int field, const void* in);
int orc_params(void* h, float* c0, float* hsm, float* vol0, float* support2, float* T_sat, float* dt,
               float* heat_inv_norm);
int orc_set_gravity(void* h, const float* g);
int orc_set_frame_motion(void* h, const float* a, const float* w, const float* wd, const float* o);
int orc_set_maneuver(void* h, int n, const double* t, const float* acc, const float* omega, const float* o);
int orc_clear_frame_motion(void* h);
int orc_set_heater_power(void* h, float w);
int orc_set_contact_angle(void* h, float deg);
int orc_damp_velocities(void* h, float f);
int orc_probe_pressure(void* h, const float* pts, int np, float* out);
int orc_pass(void* h, int pass);
int orc_set_dt(void* h, float dt);
int orc_grid_info(void* h, int* num_cells, int* nx, int* ny, int* nz, float* origin, float* inv_cell);
int orc_grid_tables(void* h, int32_t* cell_start, int32_t* cell_end);
/* keys (sorted) and gather permutation of the last grid build (n entries). */
int orc_grid_sort(void* h, uint32_t* keys, uint32_t* perm);
int orc_neighbor_lists(void* h, int32_t* counts, int32_t* list, long long cap, long long* total);
/* Dynamic scalars: p_ullage, fluid_volume0, v_max, a_max, Tv_max, spacing ratio. */
int orc_scalars(void* h, double* out8);

#ifdef __cplusplus
}
#endif
#endif
