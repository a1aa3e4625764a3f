/*
 * cryosph_b200.h -- C ABI of the B200-native per-step particle hot path of the
 * CryoSPH multiphase SPH solver (weakly-compressible liquid/vapour SPH with
 * CSF surface tension, heat conduction and Lee phase change).
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (CRYO_OK == 0) and never throws.  cryo_last_error() gives the message of the
 * last failure on a context.  Host arrays are copied; device memory is owned by
 * the context.  All work of a context is ordered on one CUDA stream.
 *
 * Reference interfaces replaced (paths inside the CryoSPH-CUDA project):
 *   include/cryosph/solvers/sph_solver.hpp:20-91    SolverConfig      -> cryo_config_t
 *   include/cryosph/physics/fluid_properties.hpp:11  FluidProperties   -> cryo_fluid_t
 *   include/cryosph/solvers/sph_solver.hpp:108-132  Diagnostics       -> cryo_diagnostics_t
 *   include/cryosph/solvers/sph_solver.hpp:134-232  Solver            -> cryo_ctx + cryo_* below
 *   include/cryosph/core/spatial_hash.hpp:62-92     SpatialHash/reorder -> cryo_grid_build
 *   include/cryosph/physics/SPH_kernels.cuh:95-113  density passes    -> cryo_pass(...)
 *   include/cryosph/physics/navier_stokes.cuh:13-23 momentum passes   -> cryo_pass(...)
 *   include/cryosph/physics/surface_tension.cuh:14-25 ST passes       -> cryo_pass(...)
 *   include/cryosph/physics/phase_change.cuh:15-46  thermal/PC passes -> cryo_pass(...)
 */
#ifndef CRYOSPH_B200_H
#define CRYOSPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CRYO_ABI_VERSION 1

/* ---------------------------------------------------------------- status */
enum {
  CRYO_OK = 0,
  CRYO_EINVAL = 1,   /* maps to std::invalid_argument / ValueError           */
  CRYO_ERANGE = 2,   /* maps to std::out_of_range                            */
  CRYO_ERUNTIME = 3, /* maps to std::runtime_error                           */
  CRYO_ECUDA = 4,    /* CUDA runtime failure (also std::runtime_error)       */
  CRYO_EDEVICE = 5   /* a device-side guard tripped (status word non-zero)   */
};

/* Device-side guard bits reported through cryo_device_status(). */
enum {
  CRYO_DEV_NBR_OVERFLOW = 1u << 0, /* neighbour list capacity exceeded (scan fallback used) */
  CRYO_DEV_SPLIT_DROPPED = 1u << 1,/* split halves dropped: capacity exhausted */
  CRYO_DEV_NONFINITE = 1u << 2,    /* NaN/Inf seen in a dt maximum */
  CRYO_DEV_BAD_CELL = 1u << 3,     /* a cell index fell outside the grid table */
  CRYO_DEV_SLAB_HALO = 1u << 4,    /* a slab and its neighbour hold different ghost layers */
  CRYO_DEV_SLAB_CAPACITY = 1u << 5 /* a refreshed slab did not fit its capacity */
};

/* ------------------------------------------------------------- enums */
/* Values equal the reference enums (sim_params.cuh:12-18, SPH_kernels.cuh:12,
 * geometry.hpp:160-164, particle_system.hpp:13-18). */
enum { CRYO_KERNEL_CUBIC = 0, CRYO_KERNEL_WENDLAND_C2 = 1 };
enum { CRYO_DENSITY_SUMMATION = 0, CRYO_DENSITY_CONTINUITY = 1 };
enum { CRYO_ST_NONE = 0, CRYO_ST_CSF = 1, CRYO_ST_AKINCI = 2 };
enum { CRYO_WALL_ADIABATIC = 0, CRYO_WALL_ISOTHERMAL = 1 };
enum { CRYO_THERMO_VENTED = 0, CRYO_THERMO_CLOSED = 1 };
enum { CRYO_WET_NORMAL_ROTATION = 0, CRYO_WET_CONTACT_LINE_FORCE = 1, CRYO_WET_BOTH = 2 };
enum { CRYO_LIQUID = 0, CRYO_VAPOR = 1, CRYO_WALL = 2, CRYO_DEAD = 3 };
enum { CRYO_FLAG_HEATED = 1, CRYO_FLAG_SOURCE = 2, CRYO_FLAG_TARGET_VAPOR = 4, CRYO_FLAG_DYING = 8 };
enum { CRYO_FLUID_CUSTOM = 0, CRYO_FLUID_LH2 = 1, CRYO_FLUID_LN2 = 2, CRYO_FLUID_LOX = 3,
       CRYO_FLUID_LCH4 = 4, CRYO_FLUID_H2O = 5 };

/* ------------------------------------------------------------ structs */
/* FluidProperties (fluid_properties.hpp:11-38), SI units. */
typedef struct cryo_fluid {
  float rho_liquid, rho_vapor, mu_liquid, mu_vapor, k_liquid, k_vapor;
  float cp_liquid, cp_vapor, sigma, h_fg, T_sat, p_sat, R_gas;
} cryo_fluid_t;

/* SolverConfig (sph_solver.hpp:20-91), field for field; booleans are int. */
typedef struct cryo_config {
  float dx, h_factor;
  int kernel, density_mode, normalize_initial_masses;
  float gravity[3];
  float velocity_scale, sound_speed, tait_gamma, background_pressure, vapor_stiffness;
  int clamp_negative_pressure;
  int transport_velocity;
  float transport_background_factor;
  int transport_stress, transport_interface_only;
  int particle_shifting;
  float shifting_strength;
  float artificial_viscosity, artificial_viscosity_vapor, delta_sph;
  int no_slip, sps_turbulence;
  float smagorinsky_cs;
  int surface_tension;
  float contact_angle_deg, contact_angle_wall_weight;
  int wall_colour, wetting_model, csf_smooth_normals, csf_balanced;
  float akinci_gamma, akinci_beta;
  int thermal, phase_change, wall_thermal_bc;
  float heater_power, conductivity_scale, lee_evaporation, lee_condensation;
  int thermo_mode;
  float vent_relaxation, merge_ratio, split_ratio, max_transfer_fraction;
  float phase_change_density_limit, vapor_mass_rebalance;
  float cfl, viscous_number, force_number, capillary_number, thermal_number;
  float dt_max, dt_min, fixed_dt;
} cryo_config_t;

/* Diagnostics (sph_solver.hpp:108-132). */
typedef struct cryo_diagnostics {
  double time;
  long long step;
  double dt;
  int n_total, n_liquid, n_vapor, n_wall;
  double mass_liquid, mass_vapor, mass_total;
  double kinetic_energy, enthalpy, heat_input;
  double evaporated_mass, condensed_mass, vented_mass, vented_enthalpy;
  double T_sat, p_ullage, max_speed;
  double T_liquid_mean, T_liquid_max, T_vapor_mean;
  float liquid_com[3], liquid_momentum[3];
  int splits, merges;
  float slosh_force[3], slosh_moment[3];
  float frame_acceleration[3], frame_angular_velocity[3];
} cryo_diagnostics_t;

/* Host particle arrays (HostParticles, particle_system.hpp:76-90).  Vectors are
 * packed xyz float triples (n*3 floats).  NULL v / nrm / flags / id mean zero
 * (ids default to 0..n-1). */
typedef struct cryo_host_particles {
  int n;
  const float* x;
  const float* v;
  const float* nrm;
  const float* m;
  const float* rho;
  const float* T;
  const uint8_t* phase;
  const uint8_t* flags;
  const uint32_t* id;
} cryo_host_particles_t;

/* Writable variant for downloads (caller allocates n entries per array). */
typedef struct cryo_host_particles_out {
  int n;
  float* x;
  float* v;
  float* nrm;
  float* m;
  float* rho;
  float* T;
  uint8_t* phase;
  uint8_t* flags;
  uint32_t* id;
} cryo_host_particles_out_t;

/* Per-particle fields that can be read back (ParticleView members,
 * particle_system.hpp:37-73).  Vector fields have 3 floats per particle. */
enum {
  CRYO_F_X = 0, CRYO_F_V, CRYO_F_VT, CRYO_F_NRM, CRYO_F_M, CRYO_F_M0, CRYO_F_RHO, CRYO_F_T,
  CRYO_F_PHASE, CRYO_F_FLAGS, CRYO_F_ID,
  CRYO_F_A, CRYO_F_AB, CRYO_F_FW, CRYO_F_MW, CRYO_F_NS, CRYO_F_VW,
  CRYO_F_P, CRYO_F_DRHO, CRYO_F_DTDT, CRYO_F_SIGMA, CRYO_F_KAPPA, CRYO_F_NU_T, CRYO_F_ALPHA,
  CRYO_F_WALL_W, CRYO_F_HEAT_W, CRYO_F_OUT_M, CRYO_F_OUT_H, CRYO_F_W_NORM, CRYO_F_RMIN,
  CRYO_F_P_WV,
  CRYO_F_COUNT
};

/* Individual operator passes (the reference's physics free functions). */
enum {
  CRYO_PASS_KICK_DRIFT = 0,      /* sph_solver.cu:20-34             */
  CRYO_PASS_GRID_BUILD,          /* spatial_hash.cu:48-114          */
  CRYO_PASS_DENSITY,             /* SPH_kernels.cu:6-34             */
  CRYO_PASS_NORMALIZE_MASSES,    /* SPH_kernels.cu:36-54            */
  CRYO_PASS_EOS,                 /* navier_stokes.cu:5-14           */
  CRYO_PASS_WALL_BOUNDARY,       /* navier_stokes.cu:16-69          */
  CRYO_PASS_INTERFACE,           /* surface_tension.cu:5-85         */
  CRYO_PASS_TRANSPORT,           /* SPH_kernels.cu:56-104           */
  CRYO_PASS_SPS,                 /* navier_stokes.cu:71-119         */
  CRYO_PASS_MOMENTUM,            /* navier_stokes.cu:121-245        */
  CRYO_PASS_SMOOTH_NORMALS,      /* surface_tension.cu:87-118       */
  CRYO_PASS_CSF,                 /* surface_tension.cu:120-177      */
  CRYO_PASS_AKINCI,              /* surface_tension.cu:179-213      */
  CRYO_PASS_DENSITY_RATE,        /* SPH_kernels.cu:162-203          */
  CRYO_PASS_THERMAL,             /* phase_change.cu:31-75 (+ heat-weight sum, sph_solver.cu:466-473) */
  CRYO_PASS_MAXIMA,              /* sph_solver.cu:475-479           */
  CRYO_PASS_KICK,                /* sph_solver.cu:36-46             */
  CRYO_PASS_SHIFTING,            /* SPH_kernels.cu:106-160          */
  CRYO_PASS_PC_SOURCES,          /* phase_change.cu:77-137          */
  CRYO_PASS_PC_NORMALIZE,        /* phase_change.cu:139-172 (+ sums, sph_solver.cu:550-552) */
  CRYO_PASS_PC_APPLY,            /* phase_change.cu:174-215         */
  CRYO_PASS_REBALANCE,           /* phase_change.cu:217-268         */
  CRYO_PASS_SPLIT,               /* phase_change.cu:270-335, sph_solver.cu:556-576 */
  CRYO_PASS_VENTING,             /* phase_change.cu:337-358, sph_solver.cu:578-583 */
  CRYO_PASS_SATURATION,          /* sph_solver.cu:586-607           */
  CRYO_PASS_COUNT
};

typedef struct cryo_ctx cryo_ctx;
typedef struct cryo_ensemble cryo_ensemble;
typedef struct cryo_slabs cryo_slabs;

/* Tank geometry for the device lattice generator (geometry.hpp:22-130):
 * a tree of nodes, children before parents, the last node the root.
 *   CYLINDER p = {R, H}  CAPSULE p = {R, L}  SPHERE p = {R}  BOX p = {lx, ly, lz}
 *   TRANSLATED a = child, p = offset   DIFFERENCE / UNION a, b = children
 * (mesh tanks have no device form: the host generator builds them). */
enum { CRYO_GEOM_CYLINDER = 0, CRYO_GEOM_CAPSULE = 1, CRYO_GEOM_SPHERE = 2, CRYO_GEOM_BOX = 3,
       CRYO_GEOM_TRANSLATED = 4, CRYO_GEOM_DIFFERENCE = 5, CRYO_GEOM_UNION = 6 };
#define CRYO_GEOM_MAX_NODES 32
typedef struct cryo_geom_node {
  int kind, a, b;
  double p[3];
} cryo_geom_node_t;
/* FillSpec (geometry.hpp:162-176); NaN temperatures mean T_sat. */
enum { CRYO_FILL_SETTLED = 0, CRYO_FILL_CENTRAL_BUBBLE = 1, CRYO_FILL_FULL = 2 };
typedef struct cryo_fill {
  int mode;
  double fill_fraction;
  float settle_direction[3];
  float bubble_center[3];
  int include_vapor;
  int wall_layers;
  float T_liquid, T_vapor, T_wall;
  double heater_zmin, heater_zmax;
} cryo_fill_t;

/* ----------------------------------------------------------- defaults */
/* Default SolverConfig values (sph_solver.hpp:20-91). */
void cryo_config_default(cryo_config_t* cfg);
/* Fluid presets (fluid_properties.cpp:16-79); which = CRYO_FLUID_*. */
int cryo_fluid_preset(int which, cryo_fluid_t* out);
/* Clausius-Clapeyron (fluid_properties.cpp:7-14). */
float cryo_saturation_temperature(const cryo_fluid_t* f, float p);
float cryo_saturation_pressure(const cryo_fluid_t* f, float T);
int cryo_abi_version(void);

/* ------------------------------------------------------------ context */
/* Solver::Solver (sph_solver.cu:273-279): validates dx > 0 and the contact
 * angle in [0,180]; creates the blocking stream on `device`. */
int cryo_create(const cryo_config_t* cfg, const cryo_fluid_t* fluid, int device, cryo_ctx** out);
void cryo_destroy(cryo_ctx* ctx);
const char* cryo_last_error(const cryo_ctx* ctx);
/* Device name string, "NAME (sm_XY)" (cuda_utils.cpp:70-76). */
int cryo_device_name(int device, char* buf, int buflen);
int cryo_device_count(void);
/* The context's CUDA stream (cudaStream_t) as an integer handle. */
uintptr_t cryo_stream(const cryo_ctx* ctx);

/* Solver::set_particles (sph_solver.cu:407-428).  domain_lo/hi: float[3]. */
int cryo_set_particles(cryo_ctx* ctx, const cryo_host_particles_t* p, const float* domain_lo,
                       const float* domain_hi);
/* The same particle set with each float column given as float or as double
 * (no counterpart in the reference, whose upload takes one element type).
 * Callers holding double-precision arrays (NumPy's default) pass them as
 * they are: each value is rounded to float, as a C cast rounds it, while the
 * copy threads move it into the transfer buffer, so no converted copy of the
 * caller's arrays is made.  x / v / nrm hold n*3 values, m / rho / T n values;
 * the matching *_f64 flag is 1 for double, 0 for float. */
typedef struct cryo_host_columns {
  int n;
  const void* x;
  const void* v;
  const void* nrm;
  const void* m;
  const void* rho;
  const void* T;
  int x_f64, v_f64, nrm_f64, m_f64, rho_f64, T_f64;
  const uint8_t* phase;
  const uint8_t* flags;
  const uint32_t* id;
} cryo_host_columns_t;
int cryo_set_particles_columns(cryo_ctx* ctx, const cryo_host_columns_t* p, const float* domain_lo,
                               const float* domain_hi);

/* Solver::build_tank (sph_solver.cu:430-437) with the lattice generated on
 * the device: build_tank_particles (geometry.cpp:242-330) evaluated per
 * lattice node (signed distances in double, the host generator's operations
 * in its order, so the particles are identical), ordered compaction of walls
 * and fluid, the liquid/vapour split at an order statistic of the fill key,
 * and the particles written straight into the solver's arrays.  bounds_lo/hi:
 * the geometry's AABB (Geometry::bounds); the domain is padded by
 * (wall_layers + 1) dx as build_tank does. */
int cryo_build_tank(cryo_ctx* ctx, const cryo_geom_node_t* nodes, int n_nodes, const cryo_fill_t* fill,
                    const float* bounds_lo, const float* bounds_hi);

/* Seeded jitter of the fluid lattice on the device (no counterpart in the
 * reference, whose inputs are jittered on the host): before the first step,
 * every liquid and vapour coordinate moves by amplitude * (2u - 1) with u a
 * 24-bit uniform in [0, 1) drawn from (seed, particle id, axis) by the
 * SplitMix64 output function, so the result does not depend on particle
 * order and can be restated on the host bit for bit; walls stay on the
 * lattice.  CRYO_EINVAL once the solver has stepped. */
int cryo_jitter_fluid(cryo_ctx* ctx, float amplitude, unsigned long long seed);

/* Solver::step / run_steps / run_until / relax / next_dt (sph_solver.cu:506-543,707-736). */
int cryo_step(cryo_ctx* ctx);
int cryo_run_steps(cryo_ctx* ctx, long long n);
int cryo_run_until(cryo_ctx* ctx, double t_end);
int cryo_relax(cryo_ctx* ctx, double duration, float damping);
int cryo_next_dt(cryo_ctx* ctx, double* dt);
/* Blocks until all submitted work finished; then refreshes the host mirror. */
int cryo_synchronize(cryo_ctx* ctx);

/* Clock and counters (sph_solver.hpp:155-158). */
int cryo_time(cryo_ctx* ctx, double* t, long long* step, double* last_dt);
int cryo_num_particles(cryo_ctx* ctx, int* n);
int cryo_capacity(cryo_ctx* ctx, int* capacity);

/* Solver::diagnostics (sph_solver.cu:609-653). */
int cryo_diagnostics(cryo_ctx* ctx, cryo_diagnostics_t* out);
/* The same record without blocking the caller (no counterpart in the
 * reference): request enqueues the reduction of the current state and its
 * copy into a pinned slot on the solver's stream; fetch returns the oldest
 * pending result in request order (*got = 1), waiting for it when wait != 0,
 * else *got = 0 while it is not ready or nothing is pending.  At most 8
 * requests pending (EINVAL beyond).  A control loop requests after each step
 * and fetches the previous step's record while the next step runs. */
int cryo_diagnostics_request(cryo_ctx* ctx);
int cryo_diagnostics_fetch(cryo_ctx* ctx, cryo_diagnostics_t* out, int wait, int* got);

/* Solver::particles (persistent arrays).  out->n must be >= the particle count;
 * on return out->n holds the count. */
int cryo_download(cryo_ctx* ctx, cryo_host_particles_out_t* out);
/* Output frames packed on the device from the current state (no counterpart
 * as entry points in the reference; they carry what its write_vtk and
 * make_frame + write_json_frame write, io.cpp:52-142).
 *
 * cryo_frame_vtk: the binary payload of the legacy VTK polydata file, every
 * word big-endian, in file order: POINTS (3 floats per particle), VERTICES
 * (the int pair 1, i), SCALARS temperature, mass, density, phase, pressure
 * (1 float each), VECTORS velocity (3 floats): CRYO_VTK_WORDS_PER_PARTICLE
 * 32-bit words per particle.  `out` (cap bytes) may be null to query the
 * particle count (*count). */
#define CRYO_VTK_WORDS_PER_PARTICLE 13
int cryo_frame_vtk(cryo_ctx* ctx, void* out, size_t cap, int* count);
/* cryo_frame_viewer: the viewer frame of write_json (TelemetryFrame,
 * telemetry.hpp:16-25): particles in state order, walls left out unless
 * include_walls; position (3 floats), temperature, pressure, speed (|v|),
 * phase.  Each array holds `cap` >= the particle count entries; *count gets
 * the number written. */
int cryo_frame_viewer(cryo_ctx* ctx, int include_walls, float* position, float* temperature, float* pressure,
                      float* speed, uint8_t* phase, int cap, int* count);

/* One per-particle field (CRYO_F_*) into a host buffer of `cap` bytes.
 * Vector fields: 3 floats per particle; phase/flags: uint8; id: uint32. */
int cryo_get_field(cryo_ctx* ctx, int field, void* host_out, size_t cap);
/* Overwrites one per-particle field of the current particles (same layout as
 * cryo_get_field, `bytes` must match the particle count).  Test and
 * checkpoint helper: the DeviceArray::upload of ParticleSystem fields
 * (cuda_utils.cuh:214-217). */
int cryo_set_field(cryo_ctx* ctx, int field, const void* host_in, size_t bytes);

/* Run-time controls (sph_solver.cu:655-705). */
int cryo_set_gravity(cryo_ctx* ctx, const float* g3);
int cryo_set_frame_motion(cryo_ctx* ctx, const float* acc3, const float* omega3, const float* omega_dot3,
                          const float* origin3);
/* ManeuverProfile (sph_solver.hpp:96-105): n knots, times strictly increasing,
 * acc n*3, omega n*3 or NULL. */
int cryo_set_maneuver(cryo_ctx* ctx, int n, const double* time, const float* acc, const float* omega,
                      const float* origin3);
int cryo_clear_frame_motion(cryo_ctx* ctx);
int cryo_set_heater_power(cryo_ctx* ctx, float watts);
int cryo_set_contact_angle(cryo_ctx* ctx, float degrees);
int cryo_damp_velocities(cryo_ctx* ctx, float factor);
/* ManeuverProfile::evaluate (sph_solver.cu:244-268), host helper. */
int cryo_maneuver_evaluate(int n, const double* time, const float* acc, const float* omega, double t,
                           float* a3, float* w3, float* wdot3);

/* Field arithmetic of the neighbour passes (no counterpart in the
 * reference's API; its two builds differ exactly this way).  EXACT (the
 * default): the reference's IEEE single-precision operation sequence, no FMA
 * contraction, IEEE division and square root -- fields bit-identical to its
 * CPU build.  FAST: the same passes with FMA contraction and approximate
 * (2 ulp) division and square root, as the reference's own CUDA build
 * contracts; every pass's fields stay within 1e-5 (normwise, relative) of
 * EXACT.  Keys, sort and neighbour lists are bit-exact in both.  The
 * differentiated window (cryo_adj_*) needs EXACT. */
enum { CRYO_ARITH_EXACT = 0, CRYO_ARITH_FAST = 1 };
int cryo_set_field_arithmetic(cryo_ctx* ctx, int mode);
int cryo_field_arithmetic(cryo_ctx* ctx, int* mode);

/* Solver::probe_pressure (sph_solver.cu:738-748): np points (np*3 floats). */
int cryo_probe_pressure(cryo_ctx* ctx, const float* points, int np, float* out);

/* Solver::probe_pressure without device allocation; no counterpart in the
   reference. For callers that must not allocate device memory once running
   (a control loop probing pressure every cycle under a fixed memory budget,
   where a pool allocation can fail or stall once the particle arena has
   filled the device). Points and results go through one fixed device array
   per device of CRYO_PROBE_STATIC_MAX points; more points return CRYO_ERANGE.
   The context must be initialised first (one step, or one cryo_probe_pressure
   call): an uninitialised context returns CRYO_EINVAL, since initialising it
   may allocate. Calls whose GPU work overlapped would race on the shared
   array, so calls are serialised by a process-wide lock and return only once
   their stream has finished, on error too. Same results as
   cryo_probe_pressure. */
#define CRYO_PROBE_STATIC_MAX 16384
int cryo_probe_pressure_noalloc(cryo_ctx* ctx, const float* points, int np, float* out);

/* Derived parameters (the SimParams scalars the Python API exposes). */
int cryo_sound_speed(cryo_ctx* ctx, float* c0);
int cryo_smoothing_length(cryo_ctx* ctx, float* h);

/* ------------------------------------------------ operator-level access */
/* Runs one operator pass on the current state, exactly as the reference's
 * free function of the same name would (see CRYO_PASS_*).  Used to check
 * parity pass by pass.  Requires set_particles. */
int cryo_pass(cryo_ctx* ctx, int pass);
/* Cell-sorted grid tables after the last grid build.  keys/perm: n entries
 * (sorted key, gather permutation); cell_start/cell_end: num_cells entries. */
int cryo_grid_info(cryo_ctx* ctx, int* num_cells, int* nx, int* ny, int* nz, float* origin3, float* cell);
int cryo_grid_tables(cryo_ctx* ctx, uint32_t* keys, uint32_t* perm, int32_t* cell_start, int32_t* cell_end);
/* Neighbour list of every particle in reference iteration order
 * (spatial_hash.hpp:37-56 filtered by r^2 < (2h)^2, self included):
 * counts[n], and the indices concatenated into list (capacity `cap`). */
int cryo_neighbor_lists(cryo_ctx* ctx, int32_t* counts, int32_t* list, long long cap, long long* total);
/* The same from the stored neighbour lists the passes walk (the last grid
 * build's): fluid particles' lists as above, walls' lists hold their fluid
 * neighbours only.  EINVAL when lists are off or no grid build ran since the
 * load. */
int cryo_stored_neighbor_lists(cryo_ctx* ctx, int32_t* counts, int32_t* list, long long cap, long long* total);
/* Sets the step size used by the next pass calls (SimParams::dt). */
int cryo_set_pass_dt(cryo_ctx* ctx, float dt);
/* Device guard word (CRYO_DEV_* bits), cleared on read. */
int cryo_device_status(cryo_ctx* ctx, unsigned* status);

/* Full-state checkpoint (persistent arrays + scalar block) in a host blob. */
int cryo_state_size(cryo_ctx* ctx, size_t* bytes);
int cryo_save_state(cryo_ctx* ctx, void* blob, size_t cap);
int cryo_load_state(cryo_ctx* ctx, const void* blob, size_t bytes);

/* ------------------------------------------------------------ telemetry
 * TelemetryStream (telemetry.hpp:13-70, telemetry.cu:27-127): a non-blocking
 * capture of x, T, p, |v| and phase.  mode 0 = AsyncCopy (device staging +
 * pinned host buffer on a copy stream), 1 = ZeroCopy (kernel writes mapped
 * pinned memory).  request returns *accepted = 0 while a frame is pending. */
int cryo_telemetry_configure(cryo_ctx* ctx, int mode);
int cryo_telemetry_mode(cryo_ctx* ctx, int* mode);
int cryo_telemetry_request(cryo_ctx* ctx, int* accepted);
int cryo_telemetry_ready(cryo_ctx* ctx, int* ready);
int cryo_telemetry_pending(cryo_ctx* ctx, int* pending);
/* Waits for the pending frame.  *got = 0 when nothing was requested.  Arrays
 * must hold *n entries (query with positions == NULL first: returns n only). */
int cryo_telemetry_fetch(cryo_ctx* ctx, int* got, double* time, long long* step, int* n, float* position,
                         float* temperature, float* pressure, float* speed, uint8_t* phase);

/* ------------------------------------------------------------ profiling
 * With profiling on, steps run as individual launches bracketed by CUDA
 * events and the device time of every kernel is accumulated per kernel name. */
int cryo_set_profiling(cryo_ctx* ctx, int enable);
/* Kernel count and names/totals: names is a buffer of count*64 chars. */
int cryo_kernel_times(cryo_ctx* ctx, int* count, char* names, double* total_ms, long long* launches);
/* Number of kernel launches one step issues with the current settings. */
int cryo_kernels_per_step(cryo_ctx* ctx, int* launches);

/* Execution mode: 1 = capture each step as a CUDA graph and replay it (default),
 * 0 = launch the kernels one by one. */
int cryo_set_graph_mode(cryo_ctx* ctx, int enable);
/* Neighbour iteration: 1 = per-step neighbour lists (default), 0 = scan the
 * 27 cells in every pass. */
int cryo_set_neighbor_mode(cryo_ctx* ctx, int use_lists);

/* ------------------------------------------------------------ ensembles
 * Batched stepping of independent tanks; no counterpart in the reference
 * (its perf_scaling.cpp steps one Solver at a time).  Each member keeps its
 * own context; an ensemble step advances every member by one of its own
 * steps.  One graph launch holds `steps_per_launch` such steps, the members
 * spread over `chains` concurrent branches (0 = one branch per member).  A
 * member's results are bit-identical to stepping it alone with
 * cryo_run_steps.  Members must live on the ensemble's device and belong to
 * one ensemble at a time; destroying a member removes it.  The member's own
 * entry points stay usable between ensemble calls (the ensemble orders its
 * stream against theirs). */
int cryo_ensemble_create(int device, cryo_ensemble** out);
void cryo_ensemble_destroy(cryo_ensemble* ens);
const char* cryo_ensemble_last_error(const cryo_ensemble* ens);
int cryo_ensemble_add(cryo_ensemble* ens, cryo_ctx* tank);
int cryo_ensemble_remove(cryo_ensemble* ens, cryo_ctx* tank);
int cryo_ensemble_size(cryo_ensemble* ens, int* tanks);
int cryo_ensemble_set_chains(cryo_ensemble* ens, int chains);
/* Branches in use (chains clipped to the member count). */
int cryo_ensemble_chains(cryo_ensemble* ens, int* chains);
/* Steps per graph launch: 1, 2, 4, 8 or 16 (runs of other lengths end with
 * single-step launches). */
int cryo_ensemble_set_steps_per_launch(cryo_ensemble* ens, int steps);
int cryo_ensemble_steps_per_launch(cryo_ensemble* ens, int* steps);
/* n ensemble steps (Solver::run_steps of every member, sph_solver.cu:535-538). */
int cryo_ensemble_run_steps(cryo_ensemble* ens, long long n);
/* Device time per ensemble step over `steps` steps rounded up to whole
 * launches, after one untimed launch; all of these steps advance the members
 * (their step counters tell how many). */
int cryo_ensemble_step_time(cryo_ensemble* ens, int steps, float* ms_per_step);
/* Autotuner: times every pair of branch count (chain_candidates; NULL: the
 * member count halved down to 1) and steps per launch (launch_candidates;
 * NULL: the current one) with cryo_ensemble_step_time and keeps the
 * fastest.  The timed steps advance the members. */
int cryo_ensemble_tune(cryo_ensemble* ens, const int* chain_candidates, int nchain, const int* launch_candidates,
                       int nlaunch, int steps, int* best_chains, int* best_steps_per_launch,
                       float* best_ms_per_step);
/* The members' tile: particles per thread of their grid-stride kernels
 * inside the ensemble's graphs (1 to 64; 1 = one thread per particle, as a
 * member stepped alone).  Results do not depend on it.  cryo_ensemble_tune_tiles
 * runs cryo_ensemble_tune for every tile candidate (NULL: the current tile)
 * and keeps the fastest branch count, steps per launch and tile. */
int cryo_ensemble_set_tile(cryo_ensemble* ens, int particles_per_thread);
int cryo_ensemble_tile(cryo_ensemble* ens, int* particles_per_thread);
int cryo_ensemble_tune_tiles(cryo_ensemble* ens, const int* chain_candidates, int nchain,
                             const int* launch_candidates, int nlaunch, const int* tile_candidates, int ntile,
                             int steps, int* best_chains, int* best_steps_per_launch, int* best_tile,
                             float* best_ms_per_step);
/* Kernel launches per ensemble step inside the step graphs. */
int cryo_ensemble_launches_per_step(cryo_ensemble* ens, int* launches);
int cryo_ensemble_synchronize(cryo_ensemble* ens);
uintptr_t cryo_ensemble_stream(const cryo_ensemble* ens);

/* ------------------------------------------------------------------------
 * Slab decomposition of one tank (no counterpart in the reference, whose
 * Solver runs one tank on one device).  The tank is cut along z into slabs
 * of whole cell layers; slab r is a context on devices[r] (NULL: all on
 * device 0; slabs may share a device).  Every slab holds its own layers and
 * ghost copies of its neighbours' facing layers; between passes the ghost
 * layer next to each slab is copied from the slab that owns it (plain loads
 * of the neighbour's memory, peer access over NVLink between devices), and
 * sums and maxima are taken over owned particles and combined in slab order.
 * Particle results equal the one-context run's: the slabs' sorted orders are
 * the whole tank's, cut at layer boundaries.  FP64 sums are added per slab,
 * so the diagnostics' sums may differ from the one-context run's in the
 * last bits.  The slabs' contexts are private; the group is stepped
 * through these entry points only (no step graphs, relax, manoeuvres or
 * differentiated windows). */
/* Layer partition (host only): slab r gets layers [z_begin[r], z_begin[r+1])
 * (z_begin has nslabs + 1 entries), each at least min_layers thick, cut
 * where the running particle count crosses r / nslabs of the total. */
int cryo_slab_partition(const long long* layer_counts, int nz, int nslabs, int min_layers, int* z_begin);
int cryo_slabs_create(const cryo_config_t* cfg, const cryo_fluid_t* fluid, int nslabs, const int* devices,
                      cryo_slabs** out);
void cryo_slabs_destroy(cryo_slabs* s);
const char* cryo_slabs_last_error(const cryo_slabs* s);
int cryo_slabs_count(cryo_slabs* s, int* nslabs);
/* Solver::set_particles of the whole tank (sph_solver.cu:407-428). */
int cryo_slabs_set_particles(cryo_slabs* s, const cryo_host_particles_t* p, const float* lo, const float* hi);
/* Graph mode (default 1): the group's step (every slab's refresh and step,
 * their exchange points as graph edges) is captured once as one CUDA graph
 * rooted on slab 0's stream and replayed, with no host barrier inside a
 * step; 0: one host thread per slab enqueues every step.  cryo_slabs_graph_mode
 * reports 0 (off), 1 (steps replay the graph) or 2 (on, but the runtime
 * refused the capture, e.g. across devices that cannot share a graph: the
 * steps run as in mode 0). */
int cryo_slabs_set_graph_mode(cryo_slabs* s, int enable);
int cryo_slabs_graph_mode(cryo_slabs* s, int* mode);
/* Solver::run_steps (sph_solver.cu:535-538) of the whole tank. */
int cryo_slabs_run_steps(cryo_slabs* s, long long n);
int cryo_slabs_num_particles(cryo_slabs* s, int* n);
/* Solver::particles of the whole tank, in the order the one-context run's
 * arrays have (out->n as in cryo_download). */
int cryo_slabs_download(cryo_slabs* s, cryo_host_particles_out_t* out);
/* Solver::diagnostics (sph_solver.cu:609-653) of the whole tank. */
int cryo_slabs_diagnostics(cryo_slabs* s, cryo_diagnostics_t* out);
/* z_begin (nslabs + 1 entries), owned[r] = particles slab r owns, held[r] =
 * particles its context holds (owned + ghosts); owned / held may be NULL. */
int cryo_slabs_layout(cryo_slabs* s, int* z_begin, int* owned, int* held);

/* ------------------------------------------------------------------------
 * Differentiated window (no counterpart in the reference).  cryo_adj_forward
 * runs `steps` ordinary steps from the current state, keeps a state
 * checkpoint every `checkpoint_every` steps and returns the objectives
 *   objectives[0..2] = sum over the steps of dt * slosh_force
 *                      (slosh_force = -sum fw, sph_solver.cu:219-232, 640)
 *   objectives[3..5] = sum over the steps of dt * slosh_moment (-sum mw)
 *   objectives[6]    = p_ullage after the last step (sph_solver.cu:586-607).
 * cryo_adj_backward takes seed[7] = d(loss)/d(objectives) and returns the
 * gradients of that loss, computed by the hand-written reverse passes of
 * every step (segments recomputed from the checkpoints):
 *   grads[0] surface tension coefficient (FluidProperties::sigma)
 *   grads[1] contact angle, per degree (SolverConfig::contact_angle_deg)
 *   grads[2] lee_evaporation, grads[3] lee_condensation, grads[4] heater_power
 *   frame_acc_grads[3 * k + c] (optional) = d(loss)/d(frame acceleration c
 *   of step k), the acceleration the manoeuvre gives at the end of step k.
 * The neighbour sets, phases and branch decisions of each step are held
 * fixed (the derivative of the step as it ran); particles may not split,
 * merge or die inside the window.  The solver's state after the backward is
 * the window's final state.  Requires fixed_dt, a pinned sound speed
 * (sound_speed or velocity_scale > 0), summation density, the default
 * CSF/normal-rotation surface tension or none, adiabatic walls, a closed tank
 * when phase change has vapour, no SPS, shifting or transport stress; other
 * configurations return CRYO_EINVAL. */
#define CRYO_ADJ_OBJECTIVES 7
#define CRYO_ADJ_PARAMS 5
int cryo_adj_forward(cryo_ctx* ctx, long long steps, int checkpoint_every, double* objectives);
int cryo_adj_backward(cryo_ctx* ctx, const double* seed, double* grads, double* frame_acc_grads);
/* Final-state adjoint seeds and initial-state adjoints (verification hooks):
 * which 0 x, 1 v, 2 T, 3 m, 4 a, 5 ab; 3 or 1 floats per particle, in the
 * window's final (seed) or initial (gradient) particle order. */
int cryo_adj_seed_state(cryo_ctx* ctx, int which, const float* data, size_t count);
int cryo_adj_state_gradient(cryo_ctx* ctx, int which, float* out, size_t count);
/* Device bytes held by the window (checkpoints, tape, adjoints). */
int cryo_adj_memory(cryo_ctx* ctx, size_t* bytes);
int cryo_adj_release(cryo_ctx* ctx);
/* Parameter setters for differentiated runs (the reference fixes these at
 * construction: FluidProperties::sigma, SolverConfig::lee_*). */
int cryo_set_surface_tension(cryo_ctx* ctx, float sigma);
int cryo_set_lee_coefficients(cryo_ctx* ctx, float evaporation, float condensation);

#ifdef __cplusplus
}
#endif

#endif /* CRYOSPH_B200_H */
