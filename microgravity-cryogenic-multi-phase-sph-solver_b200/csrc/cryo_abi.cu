// cryo_abi.cu -- the solver's entry points: the context's parameter lowering
// (Solver::init_params), the step orchestration, loading, fields, probes,
// passes, checkpoints, telemetry and profiling (the extern "C" functions of
// cryosph_b200.h not in cryo_ensemble.cu, cryo_adj_abi.cu or
// cryo_slab_abi.cu).
#include "cryo_ctx.cuh"

namespace cryo {
thread_local std::string g_create_error;
}  // namespace cryo

// -------------------------------------------------------------------------
// Solver::init_params (sph_solver.cu:292-405), host single precision in the
// reference's order (the host compiler emits no FMA on x86-64 by default and
// the build passes -ffp-contract=off).
void cryo_ctx::init_params() {
  const cryo_config_t& c = cfg;
  Params& p = P;
  const float dx = c.dx;
  const float h = c.h_factor * dx;
  p.ktype = c.kernel;
  p.h = h;
  p.inv_h = 1.0f / h;
  p.support = 2.0f * h;
  {
    const float h3 = h * h * h;
    p.knorm = (c.kernel == CRYO_KERNEL_CUBIC) ? 1.0f / (kPi * h3) : 21.0f / (16.0f * kPi * h3);
  }
  p.dx = dx;
  p.support2 = p.support * p.support;
  {
    double sigma0 = 0;
    const int r = (int)std::ceil(p.support / dx);
    for (int k = -r; k <= r; ++k)
      for (int j = -r; j <= r; ++j)
        for (int i = -r; i <= r; ++i) sigma0 += kernel_W(p, dx * std::sqrt((float)(i * i + j * j + k * k)));
    p.vol0 = (float)(1.0 / sigma0);
  }
  p.rho0[0] = fluid.rho_liquid;
  p.rho0[1] = fluid.rho_vapor;
  p.mu[0] = fluid.mu_liquid;
  p.mu[1] = fluid.mu_vapor;
  p.k[0] = fluid.k_liquid * c.conductivity_scale;
  p.k[1] = fluid.k_vapor * c.conductivity_scale;
  p.cp[0] = fluid.cp_liquid;
  p.cp[1] = fluid.cp_vapor;
  p.mref[0] = p.rho0[0] * p.vol0;
  p.mref[1] = p.rho0[1] * p.vol0;

  const bool st_on = c.surface_tension != CRYO_ST_NONE;
  const V3 cg = v3(c.gravity[0], c.gravity[1], c.gravity[2]);
  const float g = norm(cg);
  float vref = c.velocity_scale;
  auto mx = [](float a, float b) { return (a < b) ? b : a; };
  if (!(vref > 0)) {
    vref = std::sqrt(g * char_length);
    if (st_on) vref = mx(vref, std::sqrt(fluid.sigma / (fluid.rho_liquid * h)));
    vref = mx(vref, 1e-3f);
  }
  p.c0 = c.sound_speed > 0 ? c.sound_speed : 10.0f * vref;
  p.tait_gamma = c.tait_gamma;
  p.tait_B = p.rho0[0] * p.c0 * p.c0 / p.tait_gamma;
  p.p_bg = c.background_pressure >= 0 ? c.background_pressure
                                      : (has_vapor ? 0.1f * p.rho0[1] * p.c0 * p.c0 : 0.0f);
  p.vapor_K = c.vapor_stiffness > 0 ? c.vapor_stiffness : (has_vapor ? p.rho0[1] * p.c0 * p.c0 : p.p_bg);
  p.gas_R = p.vapor_K > 0 ? p.vapor_K / (p.rho0[1] * fluid.T_sat) : fluid.R_gas;
  p.clamp_neg = c.clamp_negative_pressure ? 1 : 0;

  p.alpha_av = c.artificial_viscosity;
  p.alpha_av_vap = c.artificial_viscosity_vapor;
  p.delta_sph = c.delta_sph;
  p.density_mode = c.density_mode;
  p.no_slip = c.no_slip ? 1 : 0;
  p.sps = c.sps_turbulence ? 1 : 0;
  p.smagorinsky_cs = c.smagorinsky_cs;
  p.tvf = c.transport_velocity ? 1 : 0;
  p.tvf_stress = c.transport_stress ? 1 : 0;
  p.tvf_factor = c.transport_background_factor;
  p.tvf_interface_only = c.transport_interface_only ? 1 : 0;
  p.shift_strength = c.particle_shifting ? c.shifting_strength : 0.0f;
  p.tvf_sigma_min = has_vapor ? 0.0f : 0.95f / p.vol0;

  p.st_model = c.surface_tension;
  p.sigma = st_on ? fluid.sigma : 0.0f;
  const float theta = c.contact_angle_deg * kPi / 180.0f;
  p.cos_theta = std::cos(theta);
  p.sin_theta = std::sin(theta);
  p.wall_adhesion_weight = c.contact_angle_wall_weight;
  p.wall_colour = c.wall_colour ? 1 : 0;
  p.wetting_model = c.wetting_model;
  p.csf_smooth = c.csf_smooth_normals ? 1 : 0;
  p.csf_balanced = c.csf_balanced ? 1 : 0;
  p.normal_eps = 0.1f / h;
  {
    // Akinci strengths (sph_solver.cu:372-386), Simpson rule of
    // radial_moment4 (sph_solver.cu:181-193)
    const double sup = p.support;
    auto moment = [&](bool adh) {
      const int nn = 2000;
      const double hs = sup / nn;
      double acc = 0;
      for (int k = 0; k <= nn; ++k) {
        const double r = k * hs;
        const double w = (k == 0 || k == nn) ? 1.0 : (k % 2 ? 4.0 : 2.0);
        const double f = adh ? (double)akinci_adhesion((float)r, (float)sup) : (double)akinci_cohesion((float)r, (float)sup);
        acc += w * r * r * r * r * f;
      }
      return acc * hs / 3.0;
    };
    const double i_coh = moment(false), i_adh = moment(true);
    const double rho = fluid.rho_liquid;
    const double gamma = c.akinci_gamma >= 0
                             ? (double)c.akinci_gamma
                             : (i_coh > 0 ? 8.0 * fluid.sigma / ((double)kPi * rho * rho * i_coh) : 0.0);
    p.akinci_gamma = (float)gamma;
    p.akinci_beta = c.akinci_beta >= 0
                        ? c.akinci_beta
                        : (float)(i_adh > 0 ? gamma * (i_coh / i_adh) * 0.5 * (1.0 + (double)p.cos_theta) : 0.0);
  }
  p.thermal = c.thermal ? 1 : 0;
  p.phase_change = c.phase_change ? 1 : 0;
  p.wall_bc = c.wall_thermal_bc;
  p.T_wall = fluid.T_sat;
  p.T_ref = fluid.T_sat;
  p.h_fg = fluid.h_fg;
  p.lee_evap = c.lee_evaporation;
  p.lee_cond = c.lee_condensation;
  p.max_transfer_fraction = c.max_transfer_fraction;
  p.pc_density_limit = c.phase_change_density_limit;
  p.vapor_rebalance = c.vapor_mass_rebalance;
  p.merge_ratio = c.merge_ratio;
  p.split_ratio = c.split_ratio;
  p.heat_power = c.heater_power;

  p.cfg_phase_change = c.phase_change ? 1 : 0;
  p.thermo_closed = c.thermo_mode == CRYO_THERMO_CLOSED ? 1 : 0;
  p.has_vapor = has_vapor ? 1 : 0;
  p.csf_active = (c.surface_tension == CRYO_ST_CSF && has_vapor) ? 1 : 0;
  p.vent_relaxation = c.vent_relaxation;
  p.cfl = c.cfl;
  p.viscous_number = c.viscous_number;
  p.force_number = c.force_number;
  p.capillary_number = c.capillary_number;
  p.thermal_number = c.thermal_number;
  p.dt_max = c.dt_max;
  p.dt_min = c.dt_min;
  p.fixed_dt = c.fixed_dt;
  p.f_rho_l = fluid.rho_liquid;
  p.f_rho_v = fluid.rho_vapor;
  p.f_T_sat = fluid.T_sat;
  p.f_p_sat = fluid.p_sat;
  p.f_R_gas = fluid.R_gas;
  p.f_h_fg = fluid.h_fg;
  p.use_lists = use_lists ? 1 : 0;
  p.slab = slab_group ? 1 : 0;
}

// SpatialHash::configure (spatial_hash.cu:15-30) + view() (:36-46)
void cryo_ctx::configure_grid(const float* lo, const float* hi) {
  const float cell = P.support;
  if (!(cell > 0)) throw std::invalid_argument("SpatialHash: cell size must be positive");
  P.cell = cell;
  P.ox = lo[0] - cell;
  P.oy = lo[1] - cell;
  P.oz = lo[2] - cell;
  const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
  P.nx = std::max(1, (int)std::ceil(ex / cell) + 2);
  P.ny = std::max(1, (int)std::ceil(ey / cell) + 2);
  P.nz = std::max(1, (int)std::ceil(ez / cell) + 2);
  const long long cells = (long long)P.nx * P.ny * P.nz;
  if (cells > 400000000LL) throw std::runtime_error("SpatialHash: grid too large; increase the cell size");
  P.num_cells = (int)cells;
  P.slab_z0 = 0;
  P.slab_z1 = P.nz;
  P.inv_cell = 1.0f / cell;
  int bits = 0;
  while (bits < 32 && ((uint64_t)1 << bits) <= (uint64_t)P.num_cells) ++bits;  // sentinel fits
  P.key_bits = std::max(bits, 1);
  if (cell_cap < P.num_cells + 2) {
    if (cell_begin) CK(cudaFree(cell_begin));
    if (cell_fluid) CK(cudaFree(cell_fluid));
    CK(cudaMalloc(&cell_begin, (size_t)(P.num_cells + 2) * sizeof(int)));
    CK(cudaMalloc(&cell_fluid, (size_t)(P.num_cells + 2)));
    cell_cap = P.num_cells + 2;
  }
  CK(cudaMemsetAsync(cell_begin, 0, (size_t)(P.num_cells + 2) * sizeof(int), stream));
}

// Keys of the current positions in keys_a, then sort, cell table and gather
// (SpatialHash::build, spatial_hash.cu:48-114).  Flips `cur`.
void cryo_ctx::grid_build(int src) {
  const int G = grid_blocks();
  LAUNCH(k_keys, G, kBlock, P, view(src), keys_a);
  sort_and_gather(src, LISTS_PHASE);
}

// Radix sort of keys_a, cell table, reorder gather into the other set and
// (with lists on) the neighbour / phase lists of the new order.
void cryo_ctx::sort_and_gather(int src, int list_mode, bool reset_maxima) {
  const int G = grid_blocks();
  const int tiles = (capacity + RS_TILE - 1) / RS_TILE;
  const uint32_t* kin = keys_a;
  const uint32_t* vin = nullptr;
  uint32_t* kout = keys_b;
  uint32_t* vout = vals_b;
  for (int shift = 0; shift < P.key_bits; shift += RS_BITS) {
    const int bits = std::min(RS_BITS, P.key_bits - shift);
    LAUNCH(k_rs_upsweep, tiles, RS_THREADS, kin, shift, bits, dyn, hist);
    LAUNCH(k_rs_scan, RS_BINS, RS_SCAN_THREADS, hist, dyn);
    LAUNCH(k_rs_downsweep, tiles, RS_THREADS, kin, vin, kout, vout, shift, bits, dyn, hist);
    kin = kout;
    vin = vout;
    kout = (kout == keys_b) ? keys_a : keys_b;
    vout = (vout == vals_b) ? vals_a : vals_b;
  }
  sorted_keys = kin;
  sorted_perm = vin;
  LAUNCH(k_cells, G, kBlock, P, kin, dyn, cell_begin);
  if (P.use_lists) CK(cudaMemsetAsync(cell_fluid, 0, (size_t)P.num_cells, stream));
  LAUNCH(k_gather, G, kBlock, P, view(src), view(1 - src), vin, reduce(), reset_maxima ? 1 : 0);
  if (P.use_lists) {
    LAUNCH(k_build_lists, G, kBlock, P, view(1 - src), reduce(), list_mode);
    lists_built = true;
  }
}

// Solver::evaluate_rates (sph_solver.cu:449-480) on set s.  density_done:
// the density/EOS pass already ran inside the list build.
void cryo_ctx::evaluate_rates(int s, bool maxima_reset, bool density_done, bool tape) {
  const int G = grid_blocks();
  const View V = view(s);
  if (maxima_reset) LAUNCH(k_begin_step, 1, 1, P, V, BEGIN_RATES);
  if (!density_done) {
    FIELD_LAUNCH(k_density, G, kBlock, P, V, 1);
    slab_point(SLAB_HALO, s);
  }
  FIELD_LAUNCH(k_wall, G, kBlock, P, V);
  slab_point(SLAB_HALO, s);
  if (tape) FIELD_LAUNCH(k_interface<1>, G, kBlock, P, V, reduce(), P.thermal ? 1 : 0);
  else FIELD_LAUNCH(k_interface<0>, G, kBlock, P, V, reduce(), P.thermal ? 1 : 0);
  slab_point(P.thermal ? SLAB_HEAT : SLAB_HALO, s);
  if (P.sps) {
    FIELD_LAUNCH(k_sps, G, kBlock, P, V);
    slab_point(SLAB_HALO, s);
  }
  if (P.csf_active && P.csf_smooth) {
    FIELD_LAUNCH(k_smooth_normals, G, kBlock, P, V);
    slab_point(SLAB_HALO, s);
  }
  const int GF = forces_blocks();
  int what = FORCE_TRANSPORT | FORCE_MOMENTUM | FORCE_MAXIMA;
  if (P.csf_active) what |= FORCE_CSF;
  if (P.st_model == CRYO_ST_AKINCI) what |= FORCE_AKINCI;
  if (P.density_mode == CRYO_DENSITY_CONTINUITY) what |= FORCE_DRHO;
  if (P.thermal) what |= FORCE_THERMAL;
  if (tape) {  // the recomputation of a differentiated window: variants that also store their sums
    switch (what) {
      case FORCE_BASE: FIELD_LAUNCH(k_forces_t<FORCE_BASE | FORCE_TAPE>, GF, FORCES_BLOCK, P, V, what); break;
      case FORCE_BASE | FORCE_THERMAL:
        FIELD_LAUNCH(k_forces_t<FORCE_BASE | FORCE_THERMAL | FORCE_TAPE>, GF, FORCES_BLOCK, P, V, what);
        break;
      case FORCE_BASE | FORCE_CSF: FIELD_LAUNCH(k_forces_t<FORCE_BASE | FORCE_CSF | FORCE_TAPE>, GF, FORCES_BLOCK, P, V, what); break;
      case FORCE_BASE | FORCE_CSF | FORCE_THERMAL:
        FIELD_LAUNCH(k_forces_t<FORCE_BASE | FORCE_CSF | FORCE_THERMAL | FORCE_TAPE>, GF, FORCES_BLOCK, P, V, what);
        break;
      default: throw std::runtime_error("internal: no taped force pass for this configuration");
    }
    return;
  }
  switch (what) {
#define FORCES_CASE(W) \
  case W: FIELD_LAUNCH(k_forces_t<W>, GF, FORCES_BLOCK, P, V, W); break;
    FORCES_CASE(FORCE_BASE)
    FORCES_CASE(FORCE_BASE | FORCE_THERMAL)
    FORCES_CASE(FORCE_BASE | FORCE_DRHO)
    FORCES_CASE(FORCE_BASE | FORCE_DRHO | FORCE_THERMAL)
    FORCES_CASE(FORCE_BASE | FORCE_AKINCI)
    FORCES_CASE(FORCE_BASE | FORCE_AKINCI | FORCE_THERMAL)
    FORCES_CASE(FORCE_BASE | FORCE_AKINCI | FORCE_DRHO)
    FORCES_CASE(FORCE_BASE | FORCE_AKINCI | FORCE_DRHO | FORCE_THERMAL)
    FORCES_CASE(FORCE_BASE | FORCE_CSF)
    FORCES_CASE(FORCE_BASE | FORCE_CSF | FORCE_THERMAL)
    FORCES_CASE(FORCE_BASE | FORCE_CSF | FORCE_DRHO)
    FORCES_CASE(FORCE_BASE | FORCE_CSF | FORCE_DRHO | FORCE_THERMAL)
#undef FORCES_CASE
    default: FIELD_LAUNCH(k_forces_t<-1>, GF, FORCES_BLOCK, P, V, what);
  }
  slab_point(SLAB_FORCES, s);
}

// One Solver::step (sph_solver.cu:511-533) starting from set s; all device
// side.  With a tape (the reverse sweep's recomputation) the values the later
// stages overwrite are copied out as they are produced.
void cryo_ctx::enqueue_step(int s, const StepTape* tape) {
  const int G = grid_blocks();
  // the sums tape is visible to view() for this step only, also if a launch throws
  struct TapeScope {
    cryo_ctx* c;
    ~TapeScope() {
      if (c) {
        c->tape_sums = nullptr;
        c->tape_n = 0;
      }
    }
  } scope{tape ? this : nullptr};
  if (tape) {
    tape_sums = tape->sums;
    tape_n = tape->n;
  }
  // the step size, the frame and the kick-drift in one launch; the maxima
  // are reset by the gather
  LAUNCH(k_begin_kick_drift_keys, G, kBlock, P, view(s), keys_a);
  sort_and_gather(s, LISTS_PHASE, true);
  const int d = 1 - s;
  const View V = view(d);
  slab_point(SLAB_SORTED, d);
  evaluate_rates(d, false, false, tape != nullptr);
  if (tape) {
    LAUNCH(k_adj_copy4, G, kBlock, V.vT, tape->vT1, tape->m1, V.mrps, dyn);
    LAUNCH(k_adj_copy4, G, kBlock, V.ns4, tape->ns1, nullptr, nullptr, dyn);
    CK(cudaMemcpyAsync(tape->dyn1, dyn, sizeof(DynState), cudaMemcpyDeviceToDevice, stream));
  }
  if (!P.cfg_phase_change && !(P.shift_strength > 0.0f) && !slab_group) {
    // nothing runs between the closing kick and the end of the step
    LAUNCH(k_kick_saturation, G, kBlock, P, V, reduce());
    return;
  }
  LAUNCH(k_kick, G, kBlock, P, V, (P.cfg_phase_change ? KICK_SOURCES : 0) | KICK_HEAT);
  slab_point(SLAB_HALO, d);
  if (P.shift_strength > 0.0f) {
    FIELD_LAUNCH(k_shift_compute, G, kBlock, P, V);
    slab_point(SLAB_HALO, d);
    FIELD_LAUNCH(k_shift_apply, G, kBlock, P, V);
    slab_point(SLAB_HALO, d);
    // the phase-change passes search around the shifted positions
    // (old cell table), as for_each_neighbor does in the reference
    if (P.use_lists) LAUNCH(k_build_lists, G, kBlock, P, V, reduce(), LISTS_ONLY);
  }
  if (P.cfg_phase_change) {
    const Reduce R = reduce();
    LAUNCH(k_pc_normalize, G, kBlock, P, V, R, 1);
    slab_point(SLAB_HALO, d);
    if (tape) LAUNCH(k_adj_copy4, G, kBlock, V.pc, tape->pc2, nullptr, nullptr, dyn);
    LAUNCH(k_pc_apply, G, kBlock, P, V, 1);
    slab_point(SLAB_HALO, d);
    if (tape) LAUNCH(k_adj_copy4, G, kBlock, V.vT, tape->vT2, tape->m2, V.mrps, dyn);
    const bool reb = P.vapor_rebalance > 0.0f && has_vapor;
    if (reb) {
      LAUNCH(k_rebalance1, G, kBlock, P, V, 1);
      slab_point(SLAB_HALO, d);
    }
    LAUNCH(k_rebalance2_mark, G, kBlock, P, V, R, split_flag, reb ? 1 : 0, 1);
    slab_point(SLAB_SPLIT, d);
    LAUNCH(k_split, G, kBlock, P, V, R, split_flag, 1);
    if (cfg.thermo_mode == CRYO_THERMO_VENTED && has_vapor) {
      LAUNCH(k_venting, G, kBlock, P, V, R, cfg.vent_relaxation, 1);
    }
  }
  LAUNCH(k_saturation, G, kBlock, P, V, reduce(), 1);
  slab_point(SLAB_END, d);
}

void cryo_ctx::launch_step() {
  const int s = cur;
  if (profiling) {
    const long long c0 = launch_counter;
    enqueue_step(s);
    step_launches = (int)(launch_counter - c0);
    collect_marks();
    cur = 1 - s;
    return;
  }
  if (graph_mode) {
    if (!graph_valid[s]) {
      if (graph[s]) CK(cudaGraphExecDestroy(graph[s]));
      graph[s] = nullptr;
      cudaGraph_t g = nullptr;
      size_grids();
      CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      try {
        const long long c0 = launch_counter;
        enqueue_step(s);
        step_launches = (int)(launch_counter - c0);
      } catch (...) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      CK(cudaStreamEndCapture(stream, &g));
      CK(cudaGraphInstantiate(&graph[s], g, 0));
      CK(cudaGraphDestroy(g));
      graph_valid[s] = true;
    }
    CK(cudaGraphLaunch(graph[s], stream));
  } else {
    const long long c0 = launch_counter;
    enqueue_step(s);
    step_launches = (int)(launch_counter - c0);
  }
  cur = 1 - s;
}

// Solver::ensure_initialized (sph_solver.cu:439-447)
void cryo_ctx::ensure_initialized() {
  if (initialized) return;
  if (!has_particles) throw std::runtime_error("Solver: no particles loaded");
  size_grids();
  grid_build(cur);
  cur = 1 - cur;
  slab_point(SLAB_SORTED, cur);
  const int G = grid_blocks();
  if (cfg.normalize_initial_masses) {
    FIELD_LAUNCH(k_normalize_masses, G, kBlock, P, view(cur));
    slab_point(SLAB_HALO, cur);
  }
  evaluate_rates(cur, true, false);
  LAUNCH(k_saturation, G, kBlock, P, view(cur), reduce(), 0);
  slab_point(SLAB_END, cur);
  initialized = true;
}

// Head-room for splits (sph_solver.cu:556-560), checked between steps.
void cryo_ctx::check_capacity() {
  pull();
  if ((long long)hdyn->n * 4 > (long long)capacity * 3) allocate(capacity * 3 / 2 + 1024);
  if (grid_span > 0 && hdyn->n > span()) invalidate_graphs();
}

void cryo_ctx::run_steps(long long n) {
  ensure_initialized();
  // Particles appear (splits) or leave (merges, deaths) only through the
  // phase change; without it the count is fixed, so the steps return without
  // a round trip and the host mirror is refreshed by the next call that reads it.
  const bool count_can_change = P.cfg_phase_change != 0;
  for (long long k = 0; k < n; ++k) {
    launch_step();
    if (count_can_change && (k & 15) == 15) check_capacity();
  }
  if (count_can_change) check_capacity();
}

// Solver::run_until (sph_solver.cu:540-543): the steps are issued in batches
// that cannot pass t_end (each step is at most dt_max), then one at a time.
void cryo_ctx::run_until(double t_end) {
  ensure_initialized();
  pull();
  while (hdyn->time < t_end) {
    const double bound = cfg.fixed_dt > 0 ? (double)cfg.fixed_dt : (double)cfg.dt_max;
    long long k = (long long)std::floor((t_end - hdyn->time) / bound);
    k = std::max(1LL, std::min(k, 64LL));
    for (long long s = 0; s < k; ++s) launch_step();
    check_capacity();  // pulls the clock
  }
}

// ---------------------------------------------------------------------------
namespace {

void fluid_from(int which, cryo_fluid_t* f) {
  // FluidProperties presets (fluid_properties.cpp:16-79); custom = the
  // struct defaults (fluid_properties.hpp:12-24).
  auto put = [&](float rl, float rv, float ml, float mv, float kl, float kv, float cl, float cv, float s, float hfg,
                 float ts, float ps, float R) {
    *f = cryo_fluid_t{rl, rv, ml, mv, kl, kv, cl, cv, s, hfg, ts, ps, R};
  };
  switch (which) {
    case CRYO_FLUID_LH2: put(70.85f, 1.338f, 1.33e-5f, 1.11e-6f, 0.1034f, 0.0166f, 9770.f, 12200.f, 1.93e-3f, 445.6e3f, 20.37f, 101325.f, 4124.2f); break;
    case CRYO_FLUID_LN2: put(806.1f, 4.61f, 1.61e-4f, 5.4e-6f, 0.1446f, 0.0074f, 2042.f, 1123.f, 8.85e-3f, 199.2e3f, 77.36f, 101325.f, 296.8f); break;
    case CRYO_FLUID_LOX: put(1141.f, 4.47f, 1.96e-4f, 6.9e-6f, 0.152f, 0.0084f, 1699.f, 972.f, 13.2e-3f, 213.1e3f, 90.19f, 101325.f, 259.8f); break;
    case CRYO_FLUID_LCH4: put(422.4f, 1.816f, 1.17e-4f, 4.4e-6f, 0.184f, 0.0119f, 3481.f, 2218.f, 13.4e-3f, 510.8e3f, 111.67f, 101325.f, 518.3f); break;
    case CRYO_FLUID_H2O: put(998.2f, 0.598f, 1.0e-3f, 1.23e-5f, 0.598f, 0.0248f, 4182.f, 2080.f, 0.0728f, 2.257e6f, 373.15f, 101325.f, 461.5f); break;
    case CRYO_FLUID_CUSTOM: put(1000.f, 1.f, 1e-3f, 1e-5f, 0.6f, 0.025f, 4180.f, 2000.f, 0.072f, 2.26e6f, 373.15f, 101325.f, 461.5f); break;
    default: throw std::invalid_argument("unknown fluid preset");
  }
}

// Field access: (array, component offset in floats, components, element stride in bytes).
struct FieldLoc {
  void* base;
  int offset;   // in 4-byte words inside the element
  int comps;    // 1 or 3
  int stride;   // element size in bytes
  int kind;     // 0 float, 1 u8 phase, 2 u8 flags, 3 u32
};

FieldLoc locate(cryo_ctx* c, int field) {
  const Persist& s = c->set[c->cur];
  switch (field) {
    case CRYO_F_X: return {s.xp, 0, 3, 16, 0};
    case CRYO_F_V: return {s.vT, 0, 3, 16, 0};
    case CRYO_F_VT: return {s.vt, 0, 3, 16, 0};
    case CRYO_F_NRM: return {s.nrm, 0, 3, 16, 0};
    case CRYO_F_M: return {s.mrps, 0, 1, 16, 0};
    case CRYO_F_M0: return {s.vt, 3, 1, 16, 0};
    case CRYO_F_RHO: return {s.mrps, 1, 1, 16, 0};
    case CRYO_F_T: return {s.vT, 3, 1, 16, 0};
    case CRYO_F_PHASE: return {s.xp, 3, 1, 16, 1};
    case CRYO_F_FLAGS: return {s.xp, 3, 1, 16, 2};
    case CRYO_F_ID: return {s.id, 0, 1, 4, 3};
    case CRYO_F_A: return {c->a4, 0, 3, 16, 0};
    case CRYO_F_AB: return {c->ab4, 0, 3, 16, 0};
    case CRYO_F_FW: return {c->fw, 0, 3, 16, 0};
    case CRYO_F_MW: return {c->mw, 0, 3, 16, 0};
    case CRYO_F_NS: return {c->ns4, 0, 3, 16, 0};
    case CRYO_F_VW: return {c->vwp, 0, 3, 16, 0};
    case CRYO_F_P: return {s.mrps, 2, 1, 16, 0};
    case CRYO_F_DRHO: return {c->ab4, 3, 1, 16, 0};
    case CRYO_F_DTDT: return {c->a4, 3, 1, 16, 0};
    case CRYO_F_SIGMA: return {s.mrps, 3, 1, 16, 0};
    case CRYO_F_KAPPA: return {c->ns4, 3, 1, 16, 0};
    case CRYO_F_NU_T: return {c->nu_t, 0, 1, 4, 0};
    case CRYO_F_ALPHA: return {s.nrm, 3, 1, 16, 0};
    case CRYO_F_WALL_W: return {c->wall_w, 0, 1, 4, 0};
    case CRYO_F_HEAT_W: return {c->heat_w, 0, 1, 4, 0};
    case CRYO_F_OUT_M: return {c->pc, 0, 1, 16, 0};
    case CRYO_F_OUT_H: return {c->pc, 1, 1, 16, 0};
    case CRYO_F_W_NORM: return {c->pc, 2, 1, 16, 0};
    case CRYO_F_RMIN: return {c->rmin, 0, 1, 4, 0};
    case CRYO_F_P_WV: return {c->vwp, 3, 1, 16, 0};
    default: throw std::invalid_argument("unknown field");
  }
}

size_t field_bytes(const FieldLoc& f, int n) {
  if (f.kind == 1 || f.kind == 2) return (size_t)n;
  return (size_t)n * 4 * f.comps;
}

}  // namespace

// ===========================================================================
extern "C" {

int cryo_abi_version(void) { return CRYO_ABI_VERSION; }

// SolverConfig defaults (sph_solver.hpp:20-91)
void cryo_config_default(cryo_config_t* c) {
  std::memset(c, 0, sizeof(*c));
  c->dx = 0.005f; c->h_factor = 1.3f; c->kernel = CRYO_KERNEL_WENDLAND_C2;
  c->density_mode = CRYO_DENSITY_SUMMATION; c->normalize_initial_masses = 1;
  c->gravity[0] = 0; c->gravity[1] = 0; c->gravity[2] = -9.81f;
  c->velocity_scale = 0; c->sound_speed = 0; c->tait_gamma = 7; c->background_pressure = -1;
  c->vapor_stiffness = -1; c->clamp_negative_pressure = 0;
  c->transport_velocity = 1; c->transport_background_factor = 2.0f; c->transport_stress = 0;
  c->transport_interface_only = 1; c->particle_shifting = 0; c->shifting_strength = 0.25f;
  c->artificial_viscosity = 0.02f; c->artificial_viscosity_vapor = 0.2f; c->delta_sph = 0.1f;
  c->no_slip = 1; c->sps_turbulence = 0; c->smagorinsky_cs = 0.12f;
  c->surface_tension = CRYO_ST_CSF; c->contact_angle_deg = 90; c->contact_angle_wall_weight = 0.01f;
  c->wall_colour = 1; c->wetting_model = CRYO_WET_NORMAL_ROTATION; c->csf_smooth_normals = 0;
  c->csf_balanced = 0; c->akinci_gamma = -1; c->akinci_beta = -1;
  c->thermal = 1; c->phase_change = 1; c->wall_thermal_bc = CRYO_WALL_ADIABATIC; c->heater_power = 0;
  c->conductivity_scale = 1; c->lee_evaporation = 10; c->lee_condensation = 10;
  c->thermo_mode = CRYO_THERMO_VENTED; c->vent_relaxation = 0.02f; c->merge_ratio = 0.3f; c->split_ratio = 2.0f;
  c->max_transfer_fraction = 0.25f; c->phase_change_density_limit = 0.01f; c->vapor_mass_rebalance = 1.0f;
  c->cfl = 0.25f; c->viscous_number = 0.125f; c->force_number = 0.25f; c->capillary_number = 0.25f;
  c->thermal_number = 0.1f; c->dt_max = 1e-2f; c->dt_min = 1e-9f; c->fixed_dt = 0;
}

int cryo_fluid_preset(int which, cryo_fluid_t* out) {
  return guard(nullptr, [&] { fluid_from(which, out); });
}

// FluidProperties::saturation_temperature / _pressure (fluid_properties.cpp:7-14)
float cryo_saturation_temperature(const cryo_fluid_t* f, float p) {
  const double inv_T = 1.0 / f->T_sat - ((double)f->R_gas / f->h_fg) * std::log((double)p / f->p_sat);
  return (float)(1.0 / inv_T);
}
float cryo_saturation_pressure(const cryo_fluid_t* f, float T) {
  return (float)(f->p_sat * std::exp((double)f->h_fg / f->R_gas * (1.0 / f->T_sat - 1.0 / (double)T)));
}

int cryo_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int cryo_device_name(int device, char* buf, int buflen) {
  return guard(nullptr, [&] {
    cudaDeviceProp prop{};
    CK(cudaGetDeviceProperties(&prop, device));
    const std::string s = std::string(prop.name) + " (sm_" + std::to_string(prop.major) + std::to_string(prop.minor) + ")";
    if (buf && buflen > 0) {
      std::strncpy(buf, s.c_str(), (size_t)buflen - 1);
      buf[buflen - 1] = 0;
    }
  });
}

// Solver::Solver (sph_solver.cu:273-279)
int cryo_create(const cryo_config_t* cfg, const cryo_fluid_t* fluid, int device, cryo_ctx** out) {
  *out = nullptr;
  cryo_ctx* c = nullptr;
  const int rc = guard(nullptr, [&] {
    if (!(cfg->dx > 0)) throw std::invalid_argument("SolverConfig.dx must be > 0");
    if (cfg->contact_angle_deg < 0 || cfg->contact_angle_deg > 180)
      throw std::invalid_argument("contact angle must be within [0, 180] degrees");
    c = new cryo_ctx;
    try {
      c->cfg = *cfg;
      c->fluid = *fluid;
      c->device = device;
      CK(cudaSetDevice(device));
      int sms = 0;
      if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
        c->sm_count = sms;
      CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault));
      CK(cudaMalloc(&c->dyn, sizeof(DynState)));
      CK(cudaMallocHost(&c->hdyn, sizeof(DynState)));
      CK(cudaMallocHost(&c->diag_host, 64 * sizeof(double)));
      CK(cudaMallocHost(&c->frame_ring, cryo_ctx::kFrameSlots * sizeof(DynState::Frame)));
      for (int k = 0; k < cryo_ctx::kFrameSlots; ++k)
        CK(cudaEventCreateWithFlags(&c->frame_ev[k], cudaEventDisableTiming));
      std::memset(c->hdyn, 0, sizeof(DynState));
      set3(c->hframe.cfg_gravity, cfg->gravity);
      set3(c->hframe.gravity, cfg->gravity);
      c->hdyn->p_ullage = fluid->p_sat;
      c->hdyn->spacing_ratio = 1.0f;
      c->hdyn->T_sat = fluid->T_sat;
      set_whole_tank(*c->hdyn);
      c->push();
    } catch (...) {
      delete c;
      c = nullptr;
      throw;
    }
  });
  *out = c;
  return rc;
}

void cryo_destroy(cryo_ctx* ctx) { delete ctx; }

const char* cryo_last_error(const cryo_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

uintptr_t cryo_stream(const cryo_ctx* ctx) { return reinterpret_cast<uintptr_t>(ctx->stream); }

// Solver::set_particles (sph_solver.cu:407-428) + ParticleSystem::upload
// (particle_system.cpp:73-93) + SpatialHash::configure.
// Set-up shared by set_particles and build_tank (sph_solver.cu:407-428 and
// ParticleSystem::upload, particle_system.cpp:73-93): checks, parameters,
// capacity and grid for n particles, then (finish_load) the clean scratch and
// the reset scalar block once the particles are in set[0].
void cryo_ctx::begin_load(int n, bool vap, const float* lo, const float* hi) {
  if (vap && cfg.surface_tension == CRYO_ST_AKINCI)
    throw std::invalid_argument(
        "Solver: the Akinci surface-tension model is a free-surface (liquid-only) model; use CSF when vapour "
        "particles are present (FillSpec.include_vapor = false for Akinci runs)");
  sync();
  // What the step graphs captured: the parameter block (by value), the arena
  // and cell-table addresses, and the launch grids sized for the count.
  const Params old_P = P;
  const void* old_arena = arena.base;
  const int* old_cells = cell_begin;
  const int old_n = loaded_n;
  has_vapor = vap;
  lists_built = false;
  const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
  float cl = ex;
  if (cl < ey) cl = ey;
  if (cl < ez) cl = ez;
  this->char_length = cl;
  this->init_params();
  {
    const long long cap2 = (long long)((double)n * 2.0);
    const long long cap = std::max(cap2, (long long)n + 1024);
    if (cap > (long long)std::numeric_limits<int>::max() / 2) throw std::out_of_range("particle count too large");
    if (cap > this->capacity) {
      this->arena.release();
      this->capacity = 0;
      this->allocate((int)cap);
    }
  }
  this->configure_grid(lo, hi);
  // A reload with the same count, parameters, grid and storage (an
  // optimisation or restart loop) keeps the captured step graphs: every
  // argument they hold is unchanged, so its first step replays instead of
  // capturing again.  Anything else drops them.
  const bool same = n == old_n && old_arena == arena.base && old_cells == cell_begin &&
                    std::memcmp(&old_P, &P, sizeof(Params)) == 0;
  if (!same) this->invalidate_graphs();
  loaded_n = n;
  cur = 0;
}

void cryo_ctx::finish_load(int n, uint32_t next_id) {
  cryo_ctx* c = this;
  // scratch fields start clean (particle_system.cpp:85-88)
  const size_t cap = (size_t)c->capacity;
  for (float4* a : {c->a4, c->ab4, c->fw, c->mw, c->vwp, c->ns4, c->pc})
    CK(cudaMemsetAsync(a, 0, cap * 16, c->stream));
  for (float* a : {c->wall_w, c->heat_w, c->nu_t}) CK(cudaMemsetAsync(a, 0, cap * 4, c->stream));
  // scalar block: keep the frame state, reset the rest (sph_solver.cu:419-427)
  c->pull();
  DynState& d = *c->hdyn;
  d.n = n;
  d.n_alive = n;
  d.capacity = c->capacity;
  d.next_id = next_id;
  d.time = 0;
  d.last_dt = 0;
  d.step = 0;
  d.dt = 0;
  DynState::Frame& f = c->man_active ? d.fr : c->hframe;
  set3(f.cfg_gravity, c->cfg.gravity);
  for (int k = 0; k < 3; ++k) f.gravity[k] = c->cfg.gravity[k] - f.frame_acc[k];
  d.T_sat = c->fluid.T_sat;
  d.heat_inv_norm = 0;
  d.p_ullage = c->fluid.p_sat;
  d.fluid_volume0 = 0;
  d.heat_input = 0;
  d.v_max = d.a_max = d.Tv_max = d.nu_t_max = 0;
  d.spacing_ratio = 1.0f;
  d.evaporated = d.condensed = d.vented = d.vented_h = 0;
  d.merges = d.splits = 0;
  d.status = 0;
  d.split_requested = 0;
  d.damp_after_step = 0;
  d.damping = 1.0f;
  d.thermal_on = c->P.thermal;
  d.phase_change_on = c->cfg.phase_change ? 1 : 0;
  set_whole_tank(d);
  c->push();
  c->has_particles = true;
  c->initialized = false;
}

// Seeded jitter of the loaded fluid lattice on the device (k_jitter_fluid):
// before the first step, every liquid and vapour coordinate moves by a
// uniform offset in [-amplitude, amplitude) drawn from (seed, id, axis).
int cryo_jitter_fluid(cryo_ctx* c, float amplitude, unsigned long long seed) {
  return guard(c, [&] {
    if (!c->has_particles) throw std::invalid_argument("cryo_jitter_fluid: no particles loaded");
    if (c->initialized)
      throw std::invalid_argument("cryo_jitter_fluid: the solver has stepped; jitter the lattice before the first step");
    if (!(amplitude >= 0.0f) || !std::isfinite(amplitude))
      throw std::invalid_argument("cryo_jitter_fluid: the amplitude must be finite and >= 0");
    c->pull();
    const int n = c->hdyn->n;
    if (n == 0 || amplitude == 0.0f) return;
    const int G = std::max(1, std::min((n + kBlock - 1) / kBlock, c->sm_count * 8));
    k_jitter_fluid<<<G, kBlock, 0, c->stream>>>(c->view(c->cur), n, amplitude, (uint64_t)seed);
    LAUNCH_CHECK();
    c->sync();
  });
}

// Solver::build_tank with the lattice generated on the device (see
// cryo_setup.cu).  The lattice range, the liquid cut and the particle
// constants follow build_tank_particles (geometry.cpp:242-330) operation for
// operation; the domain is build_tank's (sph_solver.cu:430-437).
int cryo_build_tank(cryo_ctx* c, const cryo_geom_node_t* nodes, int n_nodes, const cryo_fill_t* fill,
                    const float* blo, const float* bhi) {
  return guard(c, [&] {
    const float dxf = c->cfg.dx;
    if (!(dxf > 0)) throw std::invalid_argument("build_tank_particles: dx must be > 0");
    if (fill->wall_layers < 1) throw std::invalid_argument("build_tank_particles: wall_layers must be >= 1");
    if (fill->fill_fraction < 0 || fill->fill_fraction > 1)
      throw std::invalid_argument("build_tank_particles: fill_fraction must be in [0, 1]");
    if (n_nodes < 1 || n_nodes > kGeomNodes)
      throw std::invalid_argument("build_tank: geometry needs 1 to " + std::to_string(kGeomNodes) + " nodes");
    // the node tree: children before parents, one parent each, root last
    std::vector<int> parent(n_nodes, -1);
    for (int k = 0; k < n_nodes; ++k) {
      const cryo_geom_node_t& g = nodes[k];
      if (g.kind < CRYO_GEOM_CYLINDER || g.kind > CRYO_GEOM_UNION) throw std::invalid_argument("build_tank: bad node");
      const int nch = g.kind == CRYO_GEOM_TRANSLATED ? 1 : (g.kind >= CRYO_GEOM_DIFFERENCE ? 2 : 0);
      for (int q = 0; q < nch; ++q) {
        const int ch = q == 0 ? g.a : g.b;
        if (ch < 0 || ch >= k || parent[ch] >= 0) throw std::invalid_argument("build_tank: the nodes are not a tree");
        parent[ch] = k;
      }
    }
    for (int k = 0; k + 1 < n_nodes; ++k)
      if (parent[k] < 0) throw std::invalid_argument("build_tank: every node but the last needs a parent");
    std::vector<GeomNode> prog(n_nodes);
    for (int k = 0; k < n_nodes; ++k) {
      GeomNode& g = prog[k];
      std::memset(&g, 0, sizeof(g));
      g.kind = nodes[k].kind;
      g.a = nodes[k].a;
      g.b = nodes[k].b;
      for (int q = 0; q < 3; ++q) g.p[q] = nodes[k].p[q];
      std::vector<int> chain;  // Translated ancestors, nearest first
      for (int u = parent[k]; u >= 0; u = parent[u])
        if (nodes[u].kind == CRYO_GEOM_TRANSLATED) chain.push_back(u);
      g.nofs = (int)chain.size();
      for (int f = 0; f < g.nofs; ++f)  // root first
        for (int q = 0; q < 3; ++q) g.ofs[f][q] = nodes[chain[g.nofs - 1 - f]].p[q];
    }
    // lattice (geometry.cpp:255-271)
    const double h = dxf;
    const double band = fill->wall_layers * h;
    Lattice L{};
    L.i0 = static_cast<int>(std::floor((blo[0] - band) / h)) - 1;
    L.j0 = static_cast<int>(std::floor((blo[1] - band) / h)) - 1;
    L.k0 = static_cast<int>(std::floor((blo[2] - band) / h)) - 1;
    const int i1 = static_cast<int>(std::ceil((bhi[0] + band) / h)) + 1;
    const int j1 = static_cast<int>(std::ceil((bhi[1] + band) / h)) + 1;
    const int k1 = static_cast<int>(std::ceil((bhi[2] + band) / h)) + 1;
    L.nx = i1 - L.i0;
    L.ny = j1 - L.j0;
    L.nz = k1 - L.k0;
    L.total = static_cast<long long>(L.nx) * L.ny * L.nz;
    L.h = h;
    L.band = band;
    if (L.total > 400'000'000LL) throw std::runtime_error("build_tank_particles: lattice too large, increase dx");
    // particle constants (geometry.cpp:281-285)
    const cryo_fluid_t& fl = c->fluid;
    const float vol = dxf * dxf * dxf;
    FillDev F{};
    F.mode = fill->mode;
    F.include_vapor = fill->include_vapor ? 1 : 0;
    F.m_liq = fl.rho_liquid * vol;
    F.m_vap = fl.rho_vapor * vol;
    F.rho_liq = fl.rho_liquid;
    F.rho_vap = fl.rho_vapor;
    F.T_liq = std::isnan(fill->T_liquid) ? fl.T_sat : fill->T_liquid;
    F.T_vap = std::isnan(fill->T_vapor) ? fl.T_sat : fill->T_vapor;
    F.T_wall = std::isnan(fill->T_wall) ? fl.T_sat : fill->T_wall;
    F.heater_zmin = fill->heater_zmin;
    F.heater_zmax = fill->heater_zmax;
    {  // normalized(settle_direction) (geometry.cpp:17-21, eps 1e-20)
      const float* d = fill->settle_direction;
      const float nn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      for (int q = 0; q < 3; ++q) F.g[q] = nn > 1e-20f ? d[q] / nn : 0.0f;
      for (int q = 0; q < 3; ++q) F.c[q] = fill->bubble_center[q];
    }
    c->sync();
    cudaStream_t st = c->stream;
    const long long nb_ll = (L.total + kBlock - 1) / kBlock;
    const int nb = (int)nb_ll;
    // device scratch of the set-up (freed at the end of the call)
    std::vector<void*> tmp;
    auto take = [&](size_t bytes) {
      void* q = nullptr;
      CK(cudaMallocAsync(&q, std::max<size_t>(bytes, 16), st));
      tmp.push_back(q);
      return q;
    };
    auto release = [&] {
      for (void* q : tmp) cudaFreeAsync(q, st);
      tmp.clear();
    };
    try {
      GeomNode* dG = static_cast<GeomNode*>(take(sizeof(GeomNode) * n_nodes));
      uint8_t* cls = static_cast<uint8_t*>(take((size_t)L.total));
      uint32_t* cnt_f = static_cast<uint32_t*>(take(sizeof(uint32_t) * nb));
      uint32_t* cnt_w = static_cast<uint32_t*>(take(sizeof(uint32_t) * nb));
      unsigned long long* tot = static_cast<unsigned long long*>(take(4 * sizeof(unsigned long long)));
      unsigned long long htot[4] = {0, 0, 0, 0};
      CK(cudaMemcpyAsync(dG, prog.data(), sizeof(GeomNode) * n_nodes, cudaMemcpyHostToDevice, st));
      k_lattice_classify<<<nb, kBlock, 0, st>>>(dG, n_nodes, L, cls, cnt_f, cnt_w);
      LAUNCH_CHECK();
      k_scan_counts<<<1, 1024, 0, st>>>(cnt_f, nb, tot);
      LAUNCH_CHECK();
      k_scan_counts<<<1, 1024, 0, st>>>(cnt_w, nb, tot + 1);
      LAUNCH_CHECK();
      CK(cudaMemcpyAsync(htot, tot, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
      c->sync();
      const long long nf = (long long)htot[0], nw = (long long)htot[1];
      if (nf == 0) throw std::runtime_error("build_tank_particles: no fluid particles; dx too large?");
      if (nf + nw > (long long)std::numeric_limits<int>::max() / 4) throw std::out_of_range("particle count too large");
      long long* fluid_nodes = static_cast<long long*>(take(sizeof(long long) * nf));
      long long* wall_nodes = static_cast<long long*>(take(sizeof(long long) * std::max(nw, 1LL)));
      k_lattice_scatter<<<nb, kBlock, 0, st>>>(L, cls, cnt_f, cnt_w, fluid_nodes, wall_nodes);
      LAUNCH_CHECK();
      // liquid cut: the n_liq-th largest fill key (geometry.cpp:308-323)
      const int nfi = (int)nf;
      const int gb = std::max(1, std::min((nfi + kBlock - 1) / kBlock, c->sm_count * 8));
      F.any_liquid = 1;
      if (fill->mode != CRYO_FILL_FULL) {
        const long long n_liq = std::llround(fill->fill_fraction * static_cast<double>(nf));
        if (n_liq <= 0) {
          F.any_liquid = 0;
        } else {
          uint32_t* keys = static_cast<uint32_t*>(take(sizeof(uint32_t) * nf));
          unsigned int* hist = static_cast<unsigned int*>(take(256 * sizeof(unsigned int)));
          k_fill_keys<<<gb, kBlock, 0, st>>>(L, F, fluid_nodes, nfi, keys);
          LAUNCH_CHECK();
          long long r = nf - n_liq;  // rank from the smallest
          uint32_t prefix = 0, mask = 0;
          unsigned int hh[256];
          for (int shift = 24; shift >= 0; shift -= 8) {
            CK(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned int), st));
            k_key_digits<<<gb, kBlock, 0, st>>>(keys, nfi, prefix, mask, shift, hist);
            LAUNCH_CHECK();
            CK(cudaMemcpyAsync(hh, hist, sizeof(hh), cudaMemcpyDeviceToHost, st));
            c->sync();
            int d = 0;
            for (; d < 255; ++d) {
              if (r < (long long)hh[d]) break;
              r -= hh[d];
            }
            prefix |= (uint32_t)d << shift;
            mask |= 0xffu << shift;
          }
          const uint32_t bits = (prefix & 0x80000000u) ? (prefix & 0x7fffffffu) : ~prefix;
          float kf;
          std::memcpy(&kf, &bits, sizeof(kf));
          F.cut = static_cast<double>(kf) - 1e-6 * h;
        }
      }
      uint8_t* liquid = static_cast<uint8_t*>(take((size_t)nf));
      const int nbf = (nfi + kBlock - 1) / kBlock;
      uint32_t* cnt_keep = static_cast<uint32_t*>(take(sizeof(uint32_t) * nbf));
      uint32_t* cnt_liq = static_cast<uint32_t*>(take(sizeof(uint32_t) * nbf));
      k_fill_split<<<nbf, kBlock, 0, st>>>(L, F, fluid_nodes, nfi, liquid, cnt_keep, cnt_liq);
      LAUNCH_CHECK();
      k_scan_counts<<<1, 1024, 0, st>>>(cnt_keep, nbf, tot + 2);
      LAUNCH_CHECK();
      k_scan_counts<<<1, 1024, 0, st>>>(cnt_liq, nbf, tot + 3);
      LAUNCH_CHECK();
      CK(cudaMemcpyAsync(htot, tot, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
      c->sync();
      const int kept = (int)htot[2], n_liquid = (int)htot[3];
      const int n = (int)nw + kept;
      const bool vapor = kept > n_liquid;
      float lo[3], hi[3];  // build_tank's domain (sph_solver.cu:433-435)
      const float pad = (fill->wall_layers + 1) * dxf;
      for (int q = 0; q < 3; ++q) {
        lo[q] = blo[q] - pad;
        hi[q] = bhi[q] + pad;
      }
      c->begin_load(n, vapor, lo, hi);
      const View V = c->view(0);
      const int gw = std::max(1, std::min((int)((nw + kBlock - 1) / kBlock), c->sm_count * 8));
      if (nw > 0) {
        k_emit_walls<<<gw, kBlock, 0, st>>>(dG, n_nodes, L, F, wall_nodes, (int)nw, V);
        LAUNCH_CHECK();
      }
      k_emit_fluid<<<nbf, kBlock, 0, st>>>(L, F, fluid_nodes, nfi, liquid, cnt_keep, (int)nw, V);
      LAUNCH_CHECK();
      c->finish_load(n, (uint32_t)n);
      release();
      c->sync();
    } catch (...) {
      release();
      throw;
    }
  });
}

int cryo_step(cryo_ctx* c) {
  return guard(c, [&] {
    c->ensure_initialized();
    c->launch_step();
  });
}

int cryo_run_steps(cryo_ctx* c, long long n) {
  return guard(c, [&] {
    c->run_steps(n);
    c->sync();
  });
}

int cryo_run_until(cryo_ctx* c, double t_end) {
  return guard(c, [&] {
    c->run_until(t_end);
    c->sync();
  });
}

// Solver::relax (sph_solver.cu:707-736)
int cryo_relax(cryo_ctx* c, double duration, float damping) {
  return guard(c, [&] {
    c->ensure_initialized();
    c->pull();
    const int thermal = c->hdyn->thermal_on;
    const int pc_on = c->hdyn->phase_change_on;
    c->hdyn->thermal_on = 0;
    c->hdyn->phase_change_on = 0;
    c->hdyn->damp_after_step = 1;
    c->hdyn->damping = damping;
    c->push();
    const double t_end = c->hdyn->time + duration;
    auto restore = [&] {
      c->pull();
      c->hdyn->thermal_on = thermal;
      c->hdyn->phase_change_on = pc_on;
      c->hdyn->damp_after_step = 0;
      c->push();
    };
    try {
      c->run_until(t_end);
    } catch (...) {
      restore();
      throw;
    }
    restore();
    const int G = c->grid_blocks();
    k_scale_velocities<<<G, kBlock, 0, c->stream>>>(c->view(c->cur), 0.0f, 0);
    LAUNCH_CHECK();
    c->pull();
    DynState& d = *c->hdyn;
    d.time = 0;
    d.step = 0;
    d.last_dt = 0;
    d.heat_input = d.evaporated = d.condensed = d.vented = d.vented_h = 0;
    d.splits = d.merges = 0;
    c->push();
    c->evaluate_rates(c->cur, true, false);
    k_saturation<<<G, kBlock, 0, c->stream>>>(c->P, c->view(c->cur), c->reduce(), 0);
    LAUNCH_CHECK();
    c->sync();
  });
}

int cryo_next_dt(cryo_ctx* c, double* dt) {
  return guard(c, [&] {
    c->ensure_initialized();
    c->pull();
    *dt = compute_dt(c->P, *c->hdyn);
  });
}

int cryo_synchronize(cryo_ctx* c) {
  return guard(c, [&] { c->pull(); });
}

int cryo_time(cryo_ctx* c, double* t, long long* step, double* last_dt) {
  return guard(c, [&] {
    c->pull();
    *t = c->hdyn->time;
    *step = c->hdyn->step;
    *last_dt = c->hdyn->last_dt;
  });
}

int cryo_num_particles(cryo_ctx* c, int* n) {
  return guard(c, [&] {
    c->pull();
    *n = c->has_particles ? c->hdyn->n : 0;
  });
}

int cryo_capacity(cryo_ctx* c, int* cap) {
  return guard(c, [&] { *cap = c->capacity; });
}

// Solver::diagnostics (sph_solver.cu:609-653): one reduction kernel and one
// device-to-host copy.

int cryo_diagnostics(cryo_ctx* c, cryo_diagnostics_t* o) {
  return guard(c, [&] {
    c->ensure_initialized();
    const int G = c->grid_blocks();
    k_diagnostics<<<G, kBlock, 0, c->stream>>>(c->P, c->view(c->cur), c->reduce(), c->diag_out);
    LAUNCH_CHECK();
    double* v = c->diag_host;
    CK(cudaMemcpyAsync(v, c->diag_out, 44 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    diag_fill(v, o);
  });
}

int cryo_diagnostics_request(cryo_ctx* c) {
  return guard(c, [&] {
    c->ensure_initialized();
    if (c->diag_head - c->diag_tail >= cryo_ctx::kDiagSlots)
      throw std::invalid_argument("cryo_diagnostics_request: " + std::to_string(cryo_ctx::kDiagSlots) +
                                  " requests are pending; fetch one first");
    if (!c->diag_ring) {
      CK(cudaMallocHost(&c->diag_ring, (size_t)cryo_ctx::kDiagSlots * 64 * sizeof(double)));
      for (int k = 0; k < cryo_ctx::kDiagSlots; ++k)
        CK(cudaEventCreateWithFlags(&c->diag_ev[k], cudaEventDisableTiming));
    }
    const int slot = (int)(c->diag_head % cryo_ctx::kDiagSlots);
    const int G = c->grid_blocks();
    k_diagnostics<<<G, kBlock, 0, c->stream>>>(c->P, c->view(c->cur), c->reduce(), c->diag_out);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(c->diag_ring + (size_t)slot * 64, c->diag_out, 44 * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaEventRecord(c->diag_ev[slot], c->stream));
    ++c->diag_head;
  });
}

int cryo_diagnostics_fetch(cryo_ctx* c, cryo_diagnostics_t* o, int wait, int* got) {
  return guard(c, [&] {
    *got = 0;
    if (c->diag_tail == c->diag_head) return;
    const int slot = (int)(c->diag_tail % cryo_ctx::kDiagSlots);
    if (wait) {
      CK(cudaEventSynchronize(c->diag_ev[slot]));
    } else {
      const cudaError_t e = cudaEventQuery(c->diag_ev[slot]);
      if (e == cudaErrorNotReady) {
        (void)cudaGetLastError();
        return;
      }
      CK(e);
    }
    diag_fill(c->diag_ring + (size_t)slot * 64, o);
    ++c->diag_tail;
    *got = 1;
  });
}

// The Diagnostics record from the k_diagnostics output row.
}  // extern "C"
void cryo::diag_fill(const double* v, cryo_diagnostics_t* o) {
  std::memset(o, 0, sizeof(*o));
  o->time = v[25];
  o->step = (long long)v[26];
  o->dt = v[27];
  o->n_total = (int)v[28];
  o->n_liquid = (int)v[0];
  o->n_vapor = (int)v[1];
  o->n_wall = (int)v[2];
  o->mass_liquid = v[3];
  o->mass_vapor = v[4];
  o->mass_total = o->mass_liquid + o->mass_vapor;
  o->kinetic_energy = v[5] + v[6];
  o->enthalpy = v[7] + v[8];
  o->heat_input = v[29];
  o->evaporated_mass = v[30];
  o->condensed_mass = v[31];
  o->vented_mass = v[32];
  o->vented_enthalpy = v[33];
  o->T_sat = v[34];
  o->p_ullage = v[35];
  o->max_speed = (double)(float)v[23];
  if (o->mass_liquid > 0) {
    o->T_liquid_mean = v[9] / o->mass_liquid;
    o->T_liquid_max = (double)(float)v[24];
    for (int k = 0; k < 3; ++k) {
      o->liquid_com[k] = (float)(v[11 + k] / o->mass_liquid);
      o->liquid_momentum[k] = (float)v[14 + k];
    }
  }
  if (o->mass_vapor > 0) o->T_vapor_mean = v[10] / o->mass_vapor;
  o->splits = (int)v[36];
  o->merges = (int)v[37];
  for (int k = 0; k < 3; ++k) {
    o->slosh_force[k] = -(float)v[17 + k];
    o->slosh_moment[k] = -(float)v[20 + k];
    o->frame_acceleration[k] = (float)v[38 + k];
    o->frame_angular_velocity[k] = (float)v[41 + k];
  }
}
extern "C" {

int cryo_get_field(cryo_ctx* c, int field, void* out, size_t cap) {
  return guard(c, [&] {
    c->pull();
    const int n = c->has_particles ? c->hdyn->n : 0;
    const FieldLoc f = locate(c, field);
    if (cap < field_bytes(f, n)) throw std::out_of_range("cryo_get_field: buffer too small");
    if (n == 0) return;
    std::vector<char> raw((size_t)n * f.stride);
    CK(cudaMemcpyAsync(raw.data(), f.base, raw.size(), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    for (int i = 0; i < n; ++i) {
      const char* e = raw.data() + (size_t)i * f.stride;
      if (f.kind == 0) {
        std::memcpy(static_cast<float*>(out) + (size_t)i * f.comps, e + 4 * f.offset, 4 * f.comps);
      } else if (f.kind == 3) {
        std::memcpy(static_cast<uint32_t*>(out) + i, e, 4);
      } else {
        int bits;
        std::memcpy(&bits, e + 4 * f.offset, 4);
        static_cast<uint8_t*>(out)[i] = (uint8_t)(f.kind == 1 ? (bits & 0xff) : ((bits >> 8) & 0xff));
      }
    }
  });
}

int cryo_set_field(cryo_ctx* c, int field, const void* in, size_t bytes) {
  return guard(c, [&] {
    c->pull();
    const int n = c->has_particles ? c->hdyn->n : 0;
    const FieldLoc f = locate(c, field);
    if (bytes != field_bytes(f, n)) throw std::invalid_argument("cryo_set_field: size does not match the particle count");
    if (n == 0) return;
    std::vector<char> raw((size_t)n * f.stride);
    CK(cudaMemcpyAsync(raw.data(), f.base, raw.size(), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    for (int i = 0; i < n; ++i) {
      char* e = raw.data() + (size_t)i * f.stride;
      if (f.kind == 0) {
        std::memcpy(e + 4 * f.offset, static_cast<const float*>(in) + (size_t)i * f.comps, 4 * f.comps);
      } else if (f.kind == 3) {
        std::memcpy(e, static_cast<const uint32_t*>(in) + i, 4);
      } else {
        int bits;
        std::memcpy(&bits, e + 4 * f.offset, 4);
        const int v = static_cast<const uint8_t*>(in)[i];
        bits = f.kind == 1 ? ((bits & ~0xff) | v) : ((bits & ~0xff00) | (v << 8));
        std::memcpy(e + 4 * f.offset, &bits, 4);
      }
    }
    CK(cudaMemcpyAsync(f.base, raw.data(), raw.size(), cudaMemcpyHostToDevice, c->stream));
    c->sync();
  });
}


// Solver::set_gravity (sph_solver.cu:655-658)
int cryo_set_gravity(cryo_ctx* c, const float* g) {
  return guard(c, [&] {
    set3(c->cfg.gravity, g);
    if (c->man_active) c->pull();  // the device holds the manoeuvre's frame
    set3(c->hframe.cfg_gravity, g);
    for (int k = 0; k < 3; ++k) c->hframe.gravity[k] = g[k] - c->hframe.frame_acc[k];
    c->push_frame();
  });
}

namespace {
void host_apply_frame(DynState::Frame& f, const float* a, const float* w, const float* wd, const float* o) {
  set3(f.frame_acc, a);
  for (int k = 0; k < 3; ++k) f.gravity[k] = f.cfg_gravity[k] - a[k];
  set3(f.omega, w);
  set3(f.omega_dot, wd);
  set3(f.frame_origin, o);
  const float n1 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  const float n2 = wd[0] * wd[0] + wd[1] * wd[1] + wd[2] * wd[2];
  f.frame_rot = (n1 > 0.0f || n2 > 0.0f) ? 1 : 0;
}

// ManeuverProfile::evaluate (sph_solver.cu:244-268), host
void host_maneuver(int n, const double* t, const float* acc, const float* om, double tq, float* a, float* w,
                   float* wd) {
  wd[0] = wd[1] = wd[2] = 0;
  if (tq <= t[0] || n == 1) {
    set3(a, acc);
    if (om) set3(w, om); else w[0] = w[1] = w[2] = 0;
    return;
  }
  if (tq >= t[n - 1]) {
    set3(a, acc + 3 * (n - 1));
    if (om) set3(w, om + 3 * (n - 1)); else w[0] = w[1] = w[2] = 0;
    return;
  }
  const int k = (int)(std::upper_bound(t, t + n, tq) - t) - 1;
  const double dt = t[k + 1] - t[k];
  const float f = (float)((tq - t[k]) / dt);
  for (int q = 0; q < 3; ++q) a[q] = acc[3 * k + q] * (1.0f - f) + acc[3 * (k + 1) + q] * f;
  if (om) {
    for (int q = 0; q < 3; ++q) {
      w[q] = om[3 * k + q] * (1.0f - f) + om[3 * (k + 1) + q] * f;
      wd[q] = (om[3 * (k + 1) + q] - om[3 * k + q]) / (float)dt;
    }
  } else {
    w[0] = w[1] = w[2] = 0;
  }
}
}  // namespace

// Solver::set_frame_motion (sph_solver.cu:669-672)
int cryo_set_frame_motion(cryo_ctx* c, const float* a, const float* w, const float* wd, const float* o) {
  return guard(c, [&] {
    if (c->man_active) c->pull();
    c->man_active = false;
    c->hframe.has_maneuver = 0;
    host_apply_frame(c->hframe, a, w, wd, o);
    c->push_frame();
  });
}

// ManeuverProfile::validate + Solver::set_maneuver (sph_solver.cu:234-242,674-681)
int cryo_set_maneuver(cryo_ctx* c, int n, const double* t, const float* acc, const float* omega,
                      const float* origin) {
  return guard(c, [&] {
    if (n <= 0) throw std::invalid_argument("ManeuverProfile: empty time table");
    for (int k = 1; k < n; ++k)
      if (!(t[k] > t[k - 1])) throw std::invalid_argument("ManeuverProfile: time must be strictly increasing");
    c->sync();
    if (n > c->man_cap) {
      if (c->man_t) CK(cudaFree(c->man_t));
      if (c->man_acc) CK(cudaFree(c->man_acc));
      if (c->man_omega) CK(cudaFree(c->man_omega));
      CK(cudaMalloc(&c->man_t, n * sizeof(double)));
      CK(cudaMalloc(&c->man_acc, n * 3 * sizeof(float)));
      CK(cudaMalloc(&c->man_omega, n * 3 * sizeof(float)));
      c->man_cap = n;
      c->invalidate_graphs();
    }
    CK(cudaMemcpyAsync(c->man_t, t, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->man_acc, acc, n * 3 * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    if (omega) CK(cudaMemcpyAsync(c->man_omega, omega, n * 3 * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    c->pull();
    DynState& d = *c->hdyn;
    c->hframe = c->man_active ? d.fr : c->hframe;
    c->man_active = true;
    c->hframe.has_maneuver = 1;
    d.man_n = n;
    d.man_rot = omega ? 1 : 0;
    const float zero[3] = {0, 0, 0};
    set3(d.man_origin, origin ? origin : zero);
    float a[3], w[3], wd[3];
    host_maneuver(n, t, acc, omega, d.time, a, w, wd);
    host_apply_frame(c->hframe, a, w, wd, d.man_origin);
    d.fr = c->hframe;
    c->push();
  });
}

int cryo_maneuver_evaluate(int n, const double* t, const float* acc, const float* omega, double tq, float* a,
                           float* w, float* wd) {
  return guard(nullptr, [&] {
    if (n <= 0) throw std::invalid_argument("ManeuverProfile: empty time table");
    host_maneuver(n, t, acc, omega, tq, a, w, wd);
  });
}

// Solver::clear_frame_motion (sph_solver.cu:683-686)
int cryo_clear_frame_motion(cryo_ctx* c) {
  return guard(c, [&] {
    if (c->man_active) c->pull();
    c->man_active = false;
    c->hframe.has_maneuver = 0;
    const float z[3] = {0, 0, 0};
    host_apply_frame(c->hframe, z, z, z, z);
    c->push_frame();
  });
}

// Solver::set_heater_power (sph_solver.cu:688-691)
int cryo_set_heater_power(cryo_ctx* c, float watts) {
  return guard(c, [&] {
    c->sync();
    c->cfg.heater_power = watts;
    c->P.heat_power = watts;
    c->invalidate_graphs();
  });
}

// Solver::set_contact_angle (sph_solver.cu:693-699)
int cryo_set_contact_angle(cryo_ctx* c, float degrees) {
  return guard(c, [&] {
    if (degrees < 0 || degrees > 180) throw std::invalid_argument("contact angle must be within [0, 180] degrees");
    c->sync();
    c->cfg.contact_angle_deg = degrees;
    const float theta = degrees * kPi / 180.0f;
    c->P.cos_theta = std::cos(theta);
    c->P.sin_theta = std::sin(theta);
    c->invalidate_graphs();
  });
}

// Solver::damp_velocities (sph_solver.cu:701-705)
int cryo_damp_velocities(cryo_ctx* c, float factor) {
  return guard(c, [&] {
    if (!c->has_particles) return;
    k_scale_velocities<<<c->grid_blocks(), kBlock, 0, c->stream>>>(c->view(c->cur), factor, 1);
    LAUNCH_CHECK();
    c->sync();
  });
}

// Solver::probe_pressure (sph_solver.cu:738-748)
int cryo_probe_pressure(cryo_ctx* c, const float* pts, int np, float* out) {
  return guard(c, [&] {
    c->ensure_initialized();
    if (np <= 0) return;
    float* d = nullptr;
    CK(cudaMallocAsync(&d, (size_t)np * 4 * sizeof(float), c->stream));
    CK(cudaMemcpyAsync(d, pts, (size_t)np * 3 * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    const int blocks = std::max(1, std::min((np + 127) / 128, c->sm_count * 8));
    FIELD_KERNEL(c, k_probe)<<<blocks, 128, 0, c->stream>>>(c->P, c->view(c->cur), d, np, d + 3 * (size_t)np);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(out, d + 3 * (size_t)np, (size_t)np * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaFreeAsync(d, c->stream));
    c->sync();
  });
}

// Solver::probe_pressure without device allocation. cryo_probe_pressure
// takes its point/result buffer from the stream-ordered pool on every call;
// this variant stages through one fixed array per device instead. It is for
// callers that must not allocate device memory once running: a monitoring or
// control loop that probes tank pressure every cycle under a fixed memory
// budget, where a pool allocation can fail or stall once the particle arena
// has filled the device. The context must already be initialised (stepped
// once, or probed once through cryo_probe_pressure): initialisation sizes the
// cell tables, which may allocate, so an uninitialised context is refused
// with CRYO_EINVAL instead. The array's device address is looked up on every
// call (cudaGetSymbolAddress with the context's device current; it allocates
// nothing), so no address outlives a device reset. The array is shared by
// every context on the device: calls whose GPU work overlapped would race on
// it, so calls hold a process-wide lock, and the lock is released only after
// the call's stream has drained, on the error paths too. Nothing in the array
// has to start at zero: each call writes the points it reads and a result for
// every point before copying the results back.
namespace {
__device__ __align__(256) float g_probe_scratch[4 * CRYO_PROBE_STATIC_MAX];  // xyz per point, then results
std::mutex g_probe_scratch_mu;
// Waits for the stream when it goes out of scope (declared after the lock, so
// it runs first): a failed copy or launch cannot leave work that still uses
// the shared array behind a released lock.
struct DrainOnExit {
  cudaStream_t s;
  ~DrainOnExit() { cudaStreamSynchronize(s); }
};
}  // namespace

int cryo_probe_pressure_noalloc(cryo_ctx* c, const float* pts, int np, float* out) {
  return guard(c, [&] {
    if (np > CRYO_PROBE_STATIC_MAX)
      throw std::out_of_range("cryo_probe_pressure_noalloc: " + std::to_string(np) +
                              " points exceed the fixed scratch of " + std::to_string(CRYO_PROBE_STATIC_MAX) +
                              " points; split the call or use cryo_probe_pressure");
    if (!c->initialized)
      throw std::invalid_argument(
          "cryo_probe_pressure_noalloc: the context is not initialised (its first step or an allocating "
          "probe sizes the cell tables); step once or call cryo_probe_pressure first");
    if (np <= 0) return;
    std::lock_guard<std::mutex> lock(g_probe_scratch_mu);
    DrainOnExit drain{c->stream};
    float* d = nullptr;
    {
      int prev = 0;
      CK(cudaGetDevice(&prev));
      CK(cudaSetDevice(c->device));
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_probe_scratch);
      CK(cudaSetDevice(prev));
      CK(e);
      d = static_cast<float*>(p);
    }
    CK(cudaMemcpyAsync(d, pts, (size_t)np * 3 * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    const int blocks = std::max(1, std::min((np + 127) / 128, c->sm_count * 8));
    FIELD_KERNEL(c, k_probe)<<<blocks, 128, 0, c->stream>>>(c->P, c->view(c->cur), d, np, d + 3 * (size_t)np);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(out, d + 3 * (size_t)np, (size_t)np * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    c->sync();
  });
}

int cryo_sound_speed(cryo_ctx* c, float* c0) {
  return guard(c, [&] { *c0 = c->P.c0; });
}
int cryo_smoothing_length(cryo_ctx* c, float* h) {
  return guard(c, [&] { *h = c->P.h; });
}

int cryo_set_pass_dt(cryo_ctx* c, float dt) {
  return guard(c, [&] {
    c->pass_dt = dt;
    c->pull();
    c->hdyn->dt = dt;
    c->push();
  });
}

// Operator-level calls: one reference free function on the current state.
int cryo_pass(cryo_ctx* c, int pass) {
  return guard(c, [&] {
    if (!c->has_particles) throw std::runtime_error("Solver: no particles loaded");
    const int G = c->grid_blocks();
    const View V = c->view(c->cur);
    const Reduce R = c->reduce();
    cudaStream_t st = c->stream;
    const Params& P = c->P;
    switch (pass) {  // passes that read View::aux get it from the current fields
      case CRYO_PASS_INTERFACE: case CRYO_PASS_TRANSPORT: case CRYO_PASS_SPS: case CRYO_PASS_MOMENTUM:
      case CRYO_PASS_CSF: case CRYO_PASS_AKINCI: case CRYO_PASS_DENSITY_RATE: case CRYO_PASS_THERMAL:
        FIELD_KERNEL(c, k_aux)<<<G, kBlock, 0, st>>>(P, V);
        LAUNCH_CHECK();
        break;
      default: break;
    }
    switch (pass) {
      case CRYO_PASS_KICK_DRIFT:
        k_kick_drift<<<G, kBlock, 0, st>>>(P, V, P.density_mode == CRYO_DENSITY_CONTINUITY, P.tvf);
        break;
      case CRYO_PASS_GRID_BUILD:
        c->grid_build(c->cur);
        c->cur = 1 - c->cur;
        break;
      case CRYO_PASS_DENSITY: FIELD_KERNEL(c, k_density)<<<G, kBlock, 0, st>>>(P, V, 0); break;
      case CRYO_PASS_NORMALIZE_MASSES: FIELD_KERNEL(c, k_normalize_masses)<<<G, kBlock, 0, st>>>(P, V); break;
      case CRYO_PASS_EOS: FIELD_KERNEL(c, k_eos)<<<G, kBlock, 0, st>>>(P, V); break;
      case CRYO_PASS_WALL_BOUNDARY: FIELD_KERNEL(c, k_wall)<<<G, kBlock, 0, st>>>(P, V); break;
      case CRYO_PASS_INTERFACE: FIELD_KERNEL(c, k_interface<0>)<<<G, kBlock, 0, st>>>(P, V, R, 0); break;
      case CRYO_PASS_TRANSPORT: FIELD_KERNEL(c, k_forces_t<-1>)<<<c->forces_blocks(), FORCES_BLOCK, 0, st>>>(P, V, FORCE_TRANSPORT); break;
      case CRYO_PASS_SPS: FIELD_KERNEL(c, k_sps)<<<G, kBlock, 0, st>>>(P, V); break;
      case CRYO_PASS_MOMENTUM: FIELD_KERNEL(c, k_forces_t<-1>)<<<c->forces_blocks(), FORCES_BLOCK, 0, st>>>(P, V, FORCE_MOMENTUM); break;
      case CRYO_PASS_SMOOTH_NORMALS: FIELD_KERNEL(c, k_smooth_normals)<<<G, kBlock, 0, st>>>(P, V); break;
      case CRYO_PASS_CSF: FIELD_KERNEL(c, k_forces_t<-1>)<<<c->forces_blocks(), FORCES_BLOCK, 0, st>>>(P, V, FORCE_CSF); break;
      case CRYO_PASS_AKINCI: FIELD_KERNEL(c, k_forces_t<-1>)<<<c->forces_blocks(), FORCES_BLOCK, 0, st>>>(P, V, FORCE_AKINCI); break;
      case CRYO_PASS_DENSITY_RATE: FIELD_KERNEL(c, k_forces_t<-1>)<<<c->forces_blocks(), FORCES_BLOCK, 0, st>>>(P, V, FORCE_DRHO); break;
      case CRYO_PASS_THERMAL:
        k_heat_norm<<<G, kBlock, 0, st>>>(P, V, R);
        LAUNCH_CHECK();
        FIELD_KERNEL(c, k_forces_t<-1>)<<<c->forces_blocks(), FORCES_BLOCK, 0, st>>>(P, V, FORCE_THERMAL_ALWAYS);
        break;
      case CRYO_PASS_MAXIMA:
        k_begin_step<<<1, 1, 0, st>>>(P, V, BEGIN_RATES);
        LAUNCH_CHECK();
        FIELD_KERNEL(c, k_maxima)<<<G, kBlock, 0, st>>>(P, V);
        break;
      case CRYO_PASS_KICK: k_kick<<<G, kBlock, 0, st>>>(P, V, 0); break;
      case CRYO_PASS_SHIFTING:
        FIELD_KERNEL(c, k_shift_compute)<<<G, kBlock, 0, st>>>(P, V);
        LAUNCH_CHECK();
        FIELD_KERNEL(c, k_shift_apply)<<<G, kBlock, 0, st>>>(P, V);
        LAUNCH_CHECK();
        if (P.use_lists) k_build_lists<<<G, kBlock, 0, st>>>(P, V, R, LISTS_ONLY);
        break;
      case CRYO_PASS_PC_SOURCES: k_pc_sources<<<G, kBlock, 0, st>>>(P, V); break;
      case CRYO_PASS_PC_NORMALIZE: k_pc_normalize<<<G, kBlock, 0, st>>>(P, V, R, 0); break;
      case CRYO_PASS_PC_APPLY: k_pc_apply<<<G, kBlock, 0, st>>>(P, V, 0); break;
      case CRYO_PASS_REBALANCE:
        k_rebalance1<<<G, kBlock, 0, st>>>(P, V, 0);
        LAUNCH_CHECK();
        k_rebalance2_mark<<<G, kBlock, 0, st>>>(P, V, R, c->split_flag, 1, 0);
        break;
      case CRYO_PASS_SPLIT:
        k_rebalance2_mark<<<G, kBlock, 0, st>>>(P, V, R, c->split_flag, 0, 0);
        LAUNCH_CHECK();
        k_split<<<G, kBlock, 0, st>>>(P, V, R, c->split_flag, 0);
        break;
      case CRYO_PASS_VENTING: k_venting<<<G, kBlock, 0, st>>>(P, V, R, c->cfg.vent_relaxation, 0); break;
      case CRYO_PASS_SATURATION: k_saturation<<<G, kBlock, 0, st>>>(P, V, R, 0); break;
      default: throw std::invalid_argument("unknown pass");
    }
    LAUNCH_CHECK();
    c->sync();
  });
}

int cryo_grid_info(cryo_ctx* c, int* num_cells, int* nx, int* ny, int* nz, float* origin, float* cell) {
  return guard(c, [&] {
    *num_cells = c->P.num_cells;
    *nx = c->P.nx; *ny = c->P.ny; *nz = c->P.nz;
    origin[0] = c->P.ox; origin[1] = c->P.oy; origin[2] = c->P.oz;
    *cell = c->P.cell;
  });
}

// Tables of the last grid build: the sorted keys and permutation, and the
// reference's cell_start / cell_end (-1 for empty cells, spatial_hash.cu:79-91)
// derived from the dense cell table.
int cryo_grid_tables(cryo_ctx* c, uint32_t* keys, uint32_t* perm, int32_t* cs, int32_t* ce) {
  return guard(c, [&] {
    c->pull();
    const int nc = c->P.num_cells;
    if (keys || perm) {
      if (!c->sorted_keys) throw std::runtime_error("no grid build yet");
      if (keys) CK(cudaMemcpyAsync(keys, c->sorted_keys, (size_t)c->hdyn->n_alive * 4, cudaMemcpyDeviceToHost, c->stream));
      if (perm) CK(cudaMemcpyAsync(perm, c->sorted_perm, (size_t)c->hdyn->n_alive * 4, cudaMemcpyDeviceToHost, c->stream));
    }
    if (cs || ce) {
      std::vector<int> b(nc + 1);
      CK(cudaMemcpyAsync(b.data(), c->cell_begin, (size_t)(nc + 1) * 4, cudaMemcpyDeviceToHost, c->stream));
      c->sync();
      for (int k = 0; k < nc; ++k) {
        const bool nonempty = b[k + 1] > b[k];
        if (cs) cs[k] = nonempty ? b[k] : -1;
        if (ce) ce[k] = nonempty ? b[k + 1] : -1;
      }
    }
    c->sync();
  });
}

static void neighbor_dump(cryo_ctx* c, int stored, int32_t* counts, int32_t* list, long long cap, long long* total) {
  c->pull();
  const int n = c->hdyn->n;
  int* dcount = nullptr;
  CK(cudaMallocAsync(&dcount, (size_t)std::max(n, 1) * sizeof(int), c->stream));
  k_nbr_count<<<c->grid_blocks(), kBlock, 0, c->stream>>>(c->P, c->view(c->cur), stored, dcount);
  LAUNCH_CHECK();
  CK(cudaMemcpyAsync(counts, dcount, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  c->sync();
  std::vector<long long> off(n);
  long long t = 0;
  for (int i = 0; i < n; ++i) {
    off[i] = t;
    t += counts[i];
  }
  *total = t;
  if (list && cap >= t && t > 0) {
    long long* doff = nullptr;
    int* dlist = nullptr;
    CK(cudaMallocAsync(&doff, (size_t)n * sizeof(long long), c->stream));
    CK(cudaMallocAsync(&dlist, (size_t)t * sizeof(int), c->stream));
    CK(cudaMemcpyAsync(doff, off.data(), (size_t)n * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    k_nbr_fill<<<c->grid_blocks(), kBlock, 0, c->stream>>>(c->P, c->view(c->cur), stored, doff, dlist);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(list, dlist, (size_t)t * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaFreeAsync(doff, c->stream));
    CK(cudaFreeAsync(dlist, c->stream));
  }
  CK(cudaFreeAsync(dcount, c->stream));
  c->sync();
}

int cryo_neighbor_lists(cryo_ctx* c, int32_t* counts, int32_t* list, long long cap, long long* total) {
  return guard(c, [&] { neighbor_dump(c, 0, counts, list, cap, total); });
}

int cryo_stored_neighbor_lists(cryo_ctx* c, int32_t* counts, int32_t* list, long long cap, long long* total) {
  return guard(c, [&] {
    if (!c->P.use_lists || !c->lists_built)
      throw std::invalid_argument("no neighbour lists: lists are off or no grid build ran since the load");
    neighbor_dump(c, 1, counts, list, cap, total);
  });
}

int cryo_device_status(cryo_ctx* c, unsigned* status) {
  return guard(c, [&] {
    c->pull();
    *status = c->hdyn->status;
    c->hdyn->status = 0;
    c->push();
  });
}

// ------------------------------------------------------------- checkpoints
namespace {
struct Blob {
  uint32_t magic, version;
  int n, capacity, num_cells;
  int initialized, has_vapor;
  DynState dyn;
};
const int kCkptArrays16 = 12;  // xp vT vt nrm mrps | a4 ab4 fw mw vwp ns4 pc
const int kCkptArrays4 = 5;    // id | rmin wall_w heat_w nu_t
}  // namespace

int cryo_state_size(cryo_ctx* c, size_t* bytes) {
  return guard(c, [&] {
    c->pull();
    const size_t n = (size_t)c->hdyn->n;
    *bytes = sizeof(Blob) + n * (16 * kCkptArrays16 + 4 * kCkptArrays4) + (size_t)(c->P.num_cells + 1) * 4;
  });
}

int cryo_save_state(cryo_ctx* c, void* blob, size_t cap) {
  return guard(c, [&] {
    c->pull();
    const size_t n = (size_t)c->hdyn->n;
    const size_t cells = (size_t)(c->P.num_cells + 1) * 4;
    const size_t need = sizeof(Blob) + n * (16 * kCkptArrays16 + 4 * kCkptArrays4) + cells;
    if (cap < need) throw std::out_of_range("cryo_save_state: buffer too small");
    Blob h{0x43525953u, 1u, (int)n, c->capacity, c->P.num_cells, c->initialized ? 1 : 0, c->has_vapor ? 1 : 0,
           *c->hdyn};
    char* p = static_cast<char*>(blob);
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    const Persist& s = c->set[c->cur];
    const void* a16[kCkptArrays16] = {s.xp, s.vT, s.vt, s.nrm, s.mrps, c->a4, c->ab4, c->fw, c->mw, c->vwp, c->ns4, c->pc};
    const void* a4[kCkptArrays4] = {s.id, c->rmin, c->wall_w, c->heat_w, c->nu_t};
    for (const void* a : a16) {
      CK(cudaMemcpyAsync(p, a, n * 16, cudaMemcpyDeviceToHost, c->stream));
      p += n * 16;
    }
    for (const void* a : a4) {
      CK(cudaMemcpyAsync(p, a, n * 4, cudaMemcpyDeviceToHost, c->stream));
      p += n * 4;
    }
    CK(cudaMemcpyAsync(p, c->cell_begin, cells, cudaMemcpyDeviceToHost, c->stream));
    c->sync();
  });
}

int cryo_load_state(cryo_ctx* c, const void* blob, size_t bytes) {
  return guard(c, [&] {
    if (bytes < sizeof(Blob)) throw std::invalid_argument("cryo_load_state: blob too small");
    Blob h;
    std::memcpy(&h, blob, sizeof(h));
    if (h.magic != 0x43525953u || h.version != 1u) throw std::invalid_argument("cryo_load_state: not a state blob");
    const size_t n = (size_t)h.n;
    if (!c->has_particles) throw std::runtime_error("cryo_load_state: call set_particles first (grid and parameters)");
    if (h.num_cells != c->P.num_cells) throw std::invalid_argument("cryo_load_state: grid does not match");
    const size_t cells = (size_t)(h.num_cells + 1) * 4;
    if (bytes != sizeof(Blob) + n * (16 * kCkptArrays16 + 4 * kCkptArrays4) + cells)
      throw std::invalid_argument("cryo_load_state: blob size mismatch");
    c->sync();
    if ((int)n > c->capacity || h.capacity > c->capacity) c->allocate(std::max((int)n, h.capacity));
    const char* p = static_cast<const char*>(blob) + sizeof(Blob);
    const Persist& s = c->set[c->cur];
    void* a16[kCkptArrays16] = {s.xp, s.vT, s.vt, s.nrm, s.mrps, c->a4, c->ab4, c->fw, c->mw, c->vwp, c->ns4, c->pc};
    void* a4[kCkptArrays4] = {s.id, c->rmin, c->wall_w, c->heat_w, c->nu_t};
    for (void* a : a16) {
      CK(cudaMemcpyAsync(a, p, n * 16, cudaMemcpyHostToDevice, c->stream));
      p += n * 16;
    }
    for (void* a : a4) {
      CK(cudaMemcpyAsync(a, p, n * 4, cudaMemcpyHostToDevice, c->stream));
      p += n * 4;
    }
    *c->hdyn = h.dyn;
    c->hdyn->capacity = c->capacity;
    c->man_active = c->hdyn->fr.has_maneuver != 0;
    c->hframe = c->hdyn->fr;
    c->push();
    c->initialized = h.initialized != 0;
    c->has_vapor = h.has_vapor != 0;
    c->lists_built = false;
    CK(cudaMemcpyAsync(c->cell_begin, p, cells, cudaMemcpyHostToDevice, c->stream));
    c->sync();
  });
}

int cryo_set_profiling(cryo_ctx* c, int enable) {
  return guard(c, [&] {
    c->sync();
    c->profiling = enable != 0;
    c->prof_names.clear();
    c->prof_ms.clear();
    c->prof_count.clear();
    c->marks.clear();
    c->event_used = 0;
  });
}

int cryo_kernel_times(cryo_ctx* c, int* count, char* names, double* total_ms, long long* launches) {
  return guard(c, [&] {
    const int k = (int)c->prof_names.size();
    if (names) {
      const int cap = *count;
      for (int i = 0; i < k && i < cap; ++i) {
        std::strncpy(names + 64 * i, c->prof_names[i].c_str(), 63);
        names[64 * i + 63] = 0;
        if (total_ms) total_ms[i] = c->prof_ms[i];
        if (launches) launches[i] = c->prof_count[i];
      }
    }
    *count = k;
  });
}

int cryo_kernels_per_step(cryo_ctx* c, int* launches) {
  return guard(c, [&] { *launches = c->step_launches; });
}

// TelemetryStream::configure (telemetry.cu:27-55)
int cryo_telemetry_configure(cryo_ctx* c, int mode) {
  return guard(c, [&] {
    if (mode != 0 && mode != 1) throw std::invalid_argument("telemetry mode must be AsyncCopy (0) or ZeroCopy (1)");
    c->sync();
    c->telemetry_release();
    c->tele_mode = mode;
    const size_t cap = (size_t)std::max(c->capacity, 1);
    const size_t bytes = cap * sizeof(TelemetryRecord);
    if (mode == 1) {
      if (cudaHostAlloc(&c->tele_host, bytes, cudaHostAllocMapped) == cudaSuccess &&
          cudaHostGetDevicePointer(&c->tele_host_dev, c->tele_host, 0) == cudaSuccess) {
      } else {
        cudaGetLastError();
        if (c->tele_host) cudaFreeHost(c->tele_host);
        c->tele_host = c->tele_host_dev = nullptr;
        c->tele_mode = 0;  // platform without mapped pinned memory
      }
    }
    if (c->tele_mode == 0) {
      CK(cudaHostAlloc(&c->tele_host, bytes, cudaHostAllocDefault));
      CK(cudaMalloc(&c->tele_stage, bytes));
      CK(cudaStreamCreateWithFlags(&c->tele_stream, cudaStreamNonBlocking));
    }
    CK(cudaEventCreateWithFlags(&c->tele_computed, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->tele_landed, cudaEventDisableTiming));
    c->tele_cap = cap;
  });
}

int cryo_telemetry_mode(cryo_ctx* c, int* mode) {
  return guard(c, [&] { *mode = c->tele_mode; });
}

// TelemetryStream::request (telemetry.cu:57-96) + Solver::request_telemetry
int cryo_telemetry_request(cryo_ctx* c, int* accepted) {
  return guard(c, [&] {
    *accepted = 0;
    c->ensure_initialized();
    c->pull();
    const int n = c->hdyn->n;
    if (!c->tele_host || (size_t)std::max(c->capacity, 1) != c->tele_cap) cryo_telemetry_configure(c, c->tele_mode);
    if (c->tele_pending || (size_t)n > c->tele_cap) return;
    TelemetryRecord* dst = c->tele_mode == 1 ? c->tele_host_dev : c->tele_stage;
    k_telemetry_pack<<<c->grid_blocks(), kBlock, 0, c->stream>>>(c->view(c->cur), dst);
    LAUNCH_CHECK();
    CK(cudaEventRecord(c->tele_computed, c->stream));
    if (c->tele_mode == 0) {
      CK(cudaStreamWaitEvent(c->tele_stream, c->tele_computed, 0));
      CK(cudaMemcpyAsync(c->tele_host, c->tele_stage, (size_t)n * sizeof(TelemetryRecord), cudaMemcpyDeviceToHost,
                         c->tele_stream));
      CK(cudaEventRecord(c->tele_landed, c->tele_stream));
    }
    c->tele_pending = true;
    c->tele_time = c->hdyn->time;
    c->tele_step = c->hdyn->step;
    c->tele_n = n;
    *accepted = 1;
  });
}

int cryo_telemetry_ready(cryo_ctx* c, int* ready) {
  return guard(c, [&] {
    if (!c->tele_pending) {
      *ready = 1;
      return;
    }
    const cudaError_t st = cudaEventQuery(c->tele_mode == 1 ? c->tele_computed : c->tele_landed);
    if (st == cudaSuccess) *ready = 1;
    else if (st == cudaErrorNotReady) *ready = 0;
    else CK(st);
  });
}

int cryo_telemetry_pending(cryo_ctx* c, int* pending) {
  return guard(c, [&] { *pending = c->tele_pending ? 1 : 0; });
}

// TelemetryStream::fetch (telemetry.cu:104-127)
int cryo_telemetry_fetch(cryo_ctx* c, int* got, double* time, long long* step, int* n, float* position,
                         float* temperature, float* pressure, float* speed, uint8_t* phase) {
  return guard(c, [&] {
    *got = 0;
    if (!c->tele_pending) return;
    *n = c->tele_n;
    if (!position) return;
    CK(cudaEventSynchronize(c->tele_mode == 1 ? c->tele_computed : c->tele_landed));
    c->tele_pending = false;
    *got = 1;
    *time = c->tele_time;
    *step = c->tele_step;
    for (int i = 0; i < c->tele_n; ++i) {
      const TelemetryRecord& r = c->tele_host[i];
      position[3 * i] = r.x;
      position[3 * i + 1] = r.y;
      position[3 * i + 2] = r.z;
      if (temperature) temperature[i] = r.T;
      if (pressure) pressure[i] = r.p;
      if (speed) speed[i] = r.speed;
      if (phase) phase[i] = (uint8_t)r.phase;
    }
  });
}

int cryo_set_graph_mode(cryo_ctx* c, int enable) {
  return guard(c, [&] {
    c->sync();
    c->graph_mode = enable != 0;
    c->invalidate_graphs();
  });
}

int cryo_set_field_arithmetic(cryo_ctx* c, int mode) {
  return guard(c, [&] {
    if (mode != CRYO_ARITH_EXACT && mode != CRYO_ARITH_FAST)
      throw std::invalid_argument("cryo_set_field_arithmetic: mode must be CRYO_ARITH_EXACT or CRYO_ARITH_FAST");
    c->sync();
    c->fast_fields = mode == CRYO_ARITH_FAST;
    c->invalidate_graphs();
  });
}

int cryo_field_arithmetic(cryo_ctx* c, int* mode) {
  return guard(c, [&] { *mode = c->fast_fields ? CRYO_ARITH_FAST : CRYO_ARITH_EXACT; });
}

int cryo_set_neighbor_mode(cryo_ctx* c, int use_lists) {
  return guard(c, [&] {
    c->sync();
    c->use_lists = use_lists != 0;
    c->P.use_lists = c->use_lists ? 1 : 0;
    c->lists_built = false;
    c->invalidate_graphs();
  });
}


}  // extern "C"
