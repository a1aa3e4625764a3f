// solver.cpp -- cryosph::Solver over the C ABI.  Each method is one cryo_*
// call; status codes come back as the reference's exception types
// (CRYO_EINVAL -> std::invalid_argument, CRYO_ERANGE -> std::out_of_range,
// otherwise std::runtime_error).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <stdexcept>

#include "cryosph.hpp"

namespace cryosph {

namespace {
void raise(int rc, const char* msg) {
  const std::string m = msg ? msg : "";
  switch (rc) {
    case CRYO_OK: return;
    case CRYO_EINVAL: throw std::invalid_argument(m);
    case CRYO_ERANGE: throw std::out_of_range(m);
    default: throw std::runtime_error(m);
  }
}
void put3(float* d, Vec3 v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; }
Vec3 get3(const float* s) { return Vec3{s[0], s[1], s[2]}; }
}  // namespace

// ----------------------------------------------------------- fluids
// fluid_properties.cpp:7-14
real FluidProperties::saturation_temperature(real p) const {
  const cryo_fluid_t f = to_c();
  return cryo_saturation_temperature(&f, p);
}
real FluidProperties::saturation_pressure(real T) const {
  const cryo_fluid_t f = to_c();
  return cryo_saturation_pressure(&f, T);
}
cryo_fluid_t FluidProperties::to_c() const {
  return cryo_fluid_t{rho_liquid, rho_vapor, mu_liquid, mu_vapor, k_liquid, k_vapor, cp_liquid,
                      cp_vapor,   sigma,     h_fg,      T_sat,    p_sat,   R_gas};
}
namespace {
FluidProperties preset(int which, const char* name) {
  cryo_fluid_t f{};
  raise(cryo_fluid_preset(which, &f), "unknown fluid preset");
  FluidProperties p;
  p.name = name;
  p.rho_liquid = f.rho_liquid; p.rho_vapor = f.rho_vapor; p.mu_liquid = f.mu_liquid; p.mu_vapor = f.mu_vapor;
  p.k_liquid = f.k_liquid; p.k_vapor = f.k_vapor; p.cp_liquid = f.cp_liquid; p.cp_vapor = f.cp_vapor;
  p.sigma = f.sigma; p.h_fg = f.h_fg; p.T_sat = f.T_sat; p.p_sat = f.p_sat; p.R_gas = f.R_gas;
  return p;
}
}  // namespace
FluidProperties FluidProperties::liquid_hydrogen() { return preset(CRYO_FLUID_LH2, "LH2"); }
FluidProperties FluidProperties::liquid_nitrogen() { return preset(CRYO_FLUID_LN2, "LN2"); }
FluidProperties FluidProperties::liquid_oxygen() { return preset(CRYO_FLUID_LOX, "LOX"); }
FluidProperties FluidProperties::liquid_methane() { return preset(CRYO_FLUID_LCH4, "LCH4"); }
FluidProperties FluidProperties::water() { return preset(CRYO_FLUID_H2O, "H2O"); }

cryo_config_t SolverConfig::to_c() const {
  cryo_config_t c{};
  c.dx = dx; c.h_factor = h_factor; c.kernel = static_cast<int>(kernel);
  c.density_mode = static_cast<int>(density_mode); c.normalize_initial_masses = normalize_initial_masses;
  put3(c.gravity, gravity);
  c.velocity_scale = velocity_scale; c.sound_speed = sound_speed; c.tait_gamma = tait_gamma;
  c.background_pressure = background_pressure; c.vapor_stiffness = vapor_stiffness;
  c.clamp_negative_pressure = clamp_negative_pressure; c.transport_velocity = transport_velocity;
  c.transport_background_factor = transport_background_factor; c.transport_stress = transport_stress;
  c.transport_interface_only = transport_interface_only; c.particle_shifting = particle_shifting;
  c.shifting_strength = shifting_strength; c.artificial_viscosity = artificial_viscosity;
  c.artificial_viscosity_vapor = artificial_viscosity_vapor; c.delta_sph = delta_sph; c.no_slip = no_slip;
  c.sps_turbulence = sps_turbulence; c.smagorinsky_cs = smagorinsky_cs;
  c.surface_tension = static_cast<int>(surface_tension); c.contact_angle_deg = contact_angle_deg;
  c.contact_angle_wall_weight = contact_angle_wall_weight; c.wall_colour = wall_colour;
  c.wetting_model = static_cast<int>(wetting_model); c.csf_smooth_normals = csf_smooth_normals;
  c.csf_balanced = csf_balanced; c.akinci_gamma = akinci_gamma; c.akinci_beta = akinci_beta;
  c.thermal = thermal; c.phase_change = phase_change; c.wall_thermal_bc = static_cast<int>(wall_thermal_bc);
  c.heater_power = heater_power; c.conductivity_scale = conductivity_scale; c.lee_evaporation = lee_evaporation;
  c.lee_condensation = lee_condensation; c.thermo_mode = static_cast<int>(thermo_mode);
  c.vent_relaxation = vent_relaxation; c.merge_ratio = merge_ratio; c.split_ratio = split_ratio;
  c.max_transfer_fraction = max_transfer_fraction; c.phase_change_density_limit = phase_change_density_limit;
  c.vapor_mass_rebalance = vapor_mass_rebalance; c.cfl = cfl; c.viscous_number = viscous_number;
  c.force_number = force_number; c.capillary_number = capillary_number; c.thermal_number = thermal_number;
  c.dt_max = dt_max; c.dt_min = dt_min; c.fixed_dt = fixed_dt;
  return c;
}

// ------------------------------------------------------------ maneuver
// ManeuverProfile::validate / evaluate (sph_solver.cu:234-268)
void ManeuverProfile::validate() const {
  if (time.empty()) throw std::invalid_argument("ManeuverProfile: empty time table");
  if (acceleration.size() != time.size())
    throw std::invalid_argument("ManeuverProfile: acceleration must have one entry per time");
  if (!angular_velocity.empty() && angular_velocity.size() != time.size())
    throw std::invalid_argument("ManeuverProfile: angular_velocity must be empty or have one entry per time");
  for (std::size_t k = 1; k < time.size(); ++k)
    if (!(time[k] > time[k - 1])) throw std::invalid_argument("ManeuverProfile: time must be strictly increasing");
}
void ManeuverProfile::evaluate(double t, Vec3& a, Vec3& omega, Vec3& omega_dot) const {
  std::vector<float> acc(3 * time.size()), om;
  for (std::size_t k = 0; k < time.size(); ++k) put3(acc.data() + 3 * k, acceleration[k]);
  if (!angular_velocity.empty()) {
    om.resize(3 * time.size());
    for (std::size_t k = 0; k < time.size(); ++k) put3(om.data() + 3 * k, angular_velocity[k]);
  }
  float A[3], W[3], WD[3];
  raise(cryo_maneuver_evaluate(static_cast<int>(time.size()), time.data(), acc.data(), om.empty() ? nullptr : om.data(),
                               t, A, W, WD),
        "ManeuverProfile: empty time table");
  a = get3(A);
  omega = get3(W);
  omega_dot = get3(WD);
}

// -------------------------------------------------------------- solver
Solver::Solver(const SolverConfig& config, const FluidProperties& fluid, int device) : cfg_(config), fluid_(fluid) {
  const cryo_config_t c = cfg_.to_c();
  const cryo_fluid_t f = fluid_.to_c();
  const int rc = cryo_create(&c, &f, device, &ctx_);
  if (rc) raise(rc, cryo_last_error(nullptr));
}

Solver::~Solver() { cryo_destroy(ctx_); }

void Solver::check(int rc) const {
  if (rc) raise(rc, cryo_last_error(ctx_));
}

// HostParticles as the C ABI's structure of arrays: Vec3 is three packed
// floats, so the vectors are passed in place.
static_assert(sizeof(Vec3) == 3 * sizeof(float) && sizeof(real) == sizeof(float), "Vec3 must be three floats");
static cryo_host_particles_t soa_view(const HostParticles& hp) {
  auto f3 = [](const std::vector<Vec3>& v) { return const_cast<float*>(reinterpret_cast<const float*>(v.data())); };
  return cryo_host_particles_t{static_cast<int>(hp.size()),
                               f3(hp.x),
                               f3(hp.v),
                               f3(hp.nrm),
                               const_cast<float*>(hp.m.data()),
                               const_cast<float*>(hp.rho.data()),
                               const_cast<float*>(hp.T.data()),
                               const_cast<std::uint8_t*>(hp.phase.data()),
                               const_cast<std::uint8_t*>(hp.flags.data()),
                               const_cast<std::uint32_t*>(hp.id.data())};
}
static void domain_floats(const AABB& d, float* lo, float* hi) {
  put3(lo, d.lo);
  put3(hi, d.hi);
}
// Resizes `h` to n particles and points `out` at its arrays.
static cryo_host_particles_out_t soa_sink(HostParticles& h, std::size_t n) {
  h.x.resize(n); h.v.resize(n); h.nrm.resize(n); h.m.resize(n); h.rho.resize(n); h.T.resize(n);
  h.phase.resize(n); h.flags.resize(n); h.id.resize(n);
  return cryo_host_particles_out_t{static_cast<int>(n), reinterpret_cast<float*>(h.x.data()),
                                   reinterpret_cast<float*>(h.v.data()), reinterpret_cast<float*>(h.nrm.data()),
                                   h.m.data(), h.rho.data(), h.T.data(), h.phase.data(), h.flags.data(), h.id.data()};
}

void Solver::set_particles(const HostParticles& hp, const AABB& domain) { set_particles(soa_view(hp), domain); }

void Solver::set_particles(const cryo_host_particles_t& p, const AABB& domain) {
  float lo[3], hi[3];
  domain_floats(domain, lo, hi);
  check(cryo_set_particles(ctx_, &p, lo, hi));
}

void Solver::set_particles(const cryo_host_columns_t& p, const AABB& domain) {
  float lo[3], hi[3];
  domain_floats(domain, lo, hi);
  check(cryo_set_particles_columns(ctx_, &p, lo, hi));
}

void Solver::download(cryo_host_particles_out_t& out) const { check(cryo_download(ctx_, &out)); }

// Solver::build_tank (sph_solver.cu:430-437)
void Solver::build_tank(const Geometry& geometry, const FillSpec& fill, bool on_device) {
  std::vector<cryo_geom_node_t> nodes;
  if (on_device && geometry.emit_nodes(nodes) >= 0 && nodes.size() <= CRYO_GEOM_MAX_NODES) {
    // the lattice generated on the GPU (identical particles; mesh tanks and
    // larger trees take the host generator below)
    cryo_fill_t f{};
    f.mode = static_cast<int>(fill.mode);
    f.fill_fraction = fill.fill_fraction;
    put3(f.settle_direction, fill.settle_direction);
    put3(f.bubble_center, fill.bubble_center);
    f.include_vapor = fill.include_vapor ? 1 : 0;
    f.wall_layers = fill.wall_layers;
    f.T_liquid = fill.T_liquid;
    f.T_vapor = fill.T_vapor;
    f.T_wall = fill.T_wall;
    f.heater_zmin = fill.heater_zmin;
    f.heater_zmax = fill.heater_zmax;
    const AABB b = geometry.bounds();
    float lo[3], hi[3];
    put3(lo, b.lo);
    put3(hi, b.hi);
    check(cryo_build_tank(ctx_, nodes.data(), static_cast<int>(nodes.size()), &f, lo, hi));
    return;
  }
  const HostParticles hp = build_tank_particles(geometry, fluid_, cfg_.dx, fill);
  AABB dom = geometry.bounds();
  const real pad = (fill.wall_layers + 1) * cfg_.dx;
  dom.lo = dom.lo - Vec3{pad, pad, pad};
  dom.hi = dom.hi + Vec3{pad, pad, pad};
  set_particles(hp, dom);
}

void Solver::step() { check(cryo_step(ctx_)); }
void Solver::run_steps(long long n) { check(cryo_run_steps(ctx_, n)); }
void Solver::run_until(double t_end) { check(cryo_run_until(ctx_, t_end)); }

double Solver::time() const {
  double t, dt;
  long long s;
  check(cryo_time(ctx_, &t, &s, &dt));
  return t;
}
long long Solver::step_count() const {
  double t, dt;
  long long s;
  check(cryo_time(ctx_, &t, &s, &dt));
  return s;
}
double Solver::last_dt() const {
  double t, dt;
  long long s;
  check(cryo_time(ctx_, &t, &s, &dt));
  return dt;
}
double Solver::next_dt() {
  double dt = 0;
  check(cryo_next_dt(ctx_, &dt));
  return dt;
}

static Diagnostics to_diagnostics(const cryo_diagnostics_t& d) {
  Diagnostics o;
  o.time = d.time; o.step = d.step; o.dt = d.dt;
  o.n_total = d.n_total; o.n_liquid = d.n_liquid; o.n_vapor = d.n_vapor; o.n_wall = d.n_wall;
  o.mass_liquid = d.mass_liquid; o.mass_vapor = d.mass_vapor; o.mass_total = d.mass_total;
  o.kinetic_energy = d.kinetic_energy; o.enthalpy = d.enthalpy; o.heat_input = d.heat_input;
  o.evaporated_mass = d.evaporated_mass; o.condensed_mass = d.condensed_mass;
  o.vented_mass = d.vented_mass; o.vented_enthalpy = d.vented_enthalpy;
  o.T_sat = d.T_sat; o.p_ullage = d.p_ullage; o.max_speed = d.max_speed;
  o.T_liquid_mean = d.T_liquid_mean; o.T_liquid_max = d.T_liquid_max; o.T_vapor_mean = d.T_vapor_mean;
  o.liquid_com = get3(d.liquid_com); o.liquid_momentum = get3(d.liquid_momentum);
  o.splits = d.splits; o.merges = d.merges;
  o.slosh_force = get3(d.slosh_force); o.slosh_moment = get3(d.slosh_moment);
  o.frame_acceleration = get3(d.frame_acceleration); o.frame_angular_velocity = get3(d.frame_angular_velocity);
  return o;
}

Diagnostics Solver::diagnostics() {
  cryo_diagnostics_t d{};
  check(cryo_diagnostics(ctx_, &d));
  return to_diagnostics(d);
}

void Solver::request_diagnostics() { check(cryo_diagnostics_request(ctx_)); }

bool Solver::fetch_diagnostics(Diagnostics& out, bool wait) {
  cryo_diagnostics_t d{};
  int got = 0;
  check(cryo_diagnostics_fetch(ctx_, &d, wait ? 1 : 0, &got));
  if (got) out = to_diagnostics(d);
  return got != 0;
}

HostParticles Solver::particles() const {
  HostParticles h;
  cryo_host_particles_out_t o = soa_sink(h, num_particles());
  download(o);
  return h;
}

std::vector<real> Solver::field(int f) const {
  const std::size_t n = num_particles();
  const bool vec = f == CRYO_F_X || f == CRYO_F_V || f == CRYO_F_VT || f == CRYO_F_NRM || f == CRYO_F_A ||
                   f == CRYO_F_AB || f == CRYO_F_FW || f == CRYO_F_MW || f == CRYO_F_NS || f == CRYO_F_VW;
  std::vector<real> out(vec ? 3 * n : n);
  check(cryo_get_field(ctx_, f, out.data(), out.size() * sizeof(real)));
  return out;
}
std::vector<real> Solver::pressure() const { return field(CRYO_F_P); }
std::vector<real> Solver::curvature() const { return field(CRYO_F_KAPPA); }

std::size_t Solver::num_particles() const {
  int n = 0;
  check(cryo_num_particles(ctx_, &n));
  return static_cast<std::size_t>(n);
}

void Solver::set_gravity(Vec3 g) {
  cfg_.gravity = g;
  float a[3];
  put3(a, g);
  check(cryo_set_gravity(ctx_, a));
}
void Solver::set_frame_motion(Vec3 acceleration, Vec3 angular_velocity, Vec3 angular_acceleration, Vec3 origin) {
  float a[3], w[3], wd[3], o[3];
  put3(a, acceleration); put3(w, angular_velocity); put3(wd, angular_acceleration); put3(o, origin);
  check(cryo_set_frame_motion(ctx_, a, w, wd, o));
}
void Solver::set_maneuver(const ManeuverProfile& p) {
  p.validate();
  std::vector<float> acc(3 * p.time.size()), om;
  for (std::size_t k = 0; k < p.time.size(); ++k) put3(acc.data() + 3 * k, p.acceleration[k]);
  if (!p.angular_velocity.empty()) {
    om.resize(3 * p.time.size());
    for (std::size_t k = 0; k < p.time.size(); ++k) put3(om.data() + 3 * k, p.angular_velocity[k]);
  }
  float o[3];
  put3(o, p.origin);
  check(cryo_set_maneuver(ctx_, static_cast<int>(p.time.size()), p.time.data(), acc.data(),
                          om.empty() ? nullptr : om.data(), o));
}
void Solver::clear_frame_motion() { check(cryo_clear_frame_motion(ctx_)); }
void Solver::set_heater_power(real watts) {
  cfg_.heater_power = watts;
  check(cryo_set_heater_power(ctx_, watts));
}
void Solver::set_contact_angle(real degrees) {
  check(cryo_set_contact_angle(ctx_, degrees));
  cfg_.contact_angle_deg = degrees;
}
void Solver::set_surface_tension(real sigma) {
  check(cryo_set_surface_tension(ctx_, sigma));
  fluid_.sigma = sigma;
}
void Solver::set_lee_coefficients(real evaporation, real condensation) {
  check(cryo_set_lee_coefficients(ctx_, evaporation, condensation));
  cfg_.lee_evaporation = evaporation;
  cfg_.lee_condensation = condensation;
}
std::array<double, 7> Solver::adjoint_forward(long long steps, int checkpoint_every) {
  std::array<double, 7> obj{};
  check(cryo_adj_forward(ctx_, steps, checkpoint_every, obj.data()));
  adj_steps_ = steps;
  return obj;
}
Solver::AdjointGradients Solver::adjoint_backward(const std::array<double, 7>& seed) {
  AdjointGradients g;
  double p[CRYO_ADJ_PARAMS] = {0};
  g.frame_acceleration.assign(static_cast<std::size_t>(adj_steps_) * 3, 0.0);
  check(cryo_adj_backward(ctx_, seed.data(), p, g.frame_acceleration.data()));
  g.sigma = p[0];
  g.contact_angle = p[1];
  g.lee_evaporation = p[2];
  g.lee_condensation = p[3];
  g.heater_power = p[4];
  return g;
}
std::size_t Solver::adjoint_memory() const {
  std::size_t b = 0;
  check(cryo_adj_memory(ctx_, &b));
  return b;
}
void Solver::adjoint_release() { check(cryo_adj_release(ctx_)); }
void Solver::damp_velocities(real factor) { check(cryo_damp_velocities(ctx_, factor)); }
void Solver::relax(double duration, real damping) { check(cryo_relax(ctx_, duration, damping)); }

real Solver::sound_speed() const {
  float c = 0;
  check(cryo_sound_speed(ctx_, &c));
  return c;
}
real Solver::smoothing_length() const {
  float h = 0;
  check(cryo_smoothing_length(ctx_, &h));
  return h;
}
std::string Solver::device() const { return device_name(0); }

void Solver::configure_telemetry(TelemetryMode mode) { check(cryo_telemetry_configure(ctx_, static_cast<int>(mode))); }
TelemetryMode Solver::telemetry_mode() const {
  int m = 0;
  check(cryo_telemetry_mode(ctx_, &m));
  return static_cast<TelemetryMode>(m);
}
bool Solver::request_telemetry() {
  int ok = 0;
  check(cryo_telemetry_request(ctx_, &ok));
  return ok != 0;
}
bool Solver::telemetry_ready() const {
  int r = 0;
  check(cryo_telemetry_ready(ctx_, &r));
  return r != 0;
}
bool Solver::telemetry_pending() const {
  int p = 0;
  check(cryo_telemetry_pending(ctx_, &p));
  return p != 0;
}
bool Solver::fetch_telemetry(TelemetryFrame& f) {
  int got = 0, n = 0;
  double t = 0;
  long long s = 0;
  check(cryo_telemetry_fetch(ctx_, &got, &t, &s, &n, nullptr, nullptr, nullptr, nullptr, nullptr));
  if (n == 0 && !telemetry_pending()) return false;
  f.position.resize(3 * static_cast<std::size_t>(n));
  f.temperature.resize(n); f.pressure.resize(n); f.speed.resize(n); f.phase.resize(n);
  check(cryo_telemetry_fetch(ctx_, &got, &t, &s, &n, f.position.data(), f.temperature.data(), f.pressure.data(),
                             f.speed.data(), f.phase.data()));
  if (!got) return false;
  f.time = t;
  f.step = s;
  f.n = n;
  return true;
}

std::vector<real> Solver::probe_pressure(const std::vector<Vec3>& points) {
  std::vector<float> p(3 * points.size()), out(points.size());
  for (std::size_t k = 0; k < points.size(); ++k) put3(p.data() + 3 * k, points[k]);
  if (!points.empty()) check(cryo_probe_pressure(ctx_, p.data(), static_cast<int>(points.size()), out.data()));
  return out;
}

std::uintptr_t Solver::stream_handle() const { return cryo_stream(ctx_); }
void Solver::set_graph_mode(bool on) { check(cryo_set_graph_mode(ctx_, on ? 1 : 0)); }
void Solver::jitter_fluid(real amplitude, std::uint64_t seed) {
  check(cryo_jitter_fluid(ctx_, amplitude, static_cast<unsigned long long>(seed)));
}
void Solver::set_field_arithmetic(FieldArithmetic mode) { check(cryo_set_field_arithmetic(ctx_, static_cast<int>(mode))); }
FieldArithmetic Solver::field_arithmetic() const {
  int m = 0;
  check(cryo_field_arithmetic(ctx_, &m));
  return static_cast<FieldArithmetic>(m);
}

std::vector<std::uint8_t> Solver::save_state() const {
  std::size_t bytes = 0;
  check(cryo_state_size(ctx_, &bytes));
  std::vector<std::uint8_t> blob(bytes);
  check(cryo_save_state(ctx_, blob.data(), blob.size()));
  return blob;
}
void Solver::load_state(const std::vector<std::uint8_t>& blob) {
  check(cryo_load_state(ctx_, blob.data(), blob.size()));
}

// ------------------------------------------------------------------ Ensemble
Ensemble::Ensemble(int device) {
  const int rc = cryo_ensemble_create(device, &e_);
  if (rc) raise(rc, cryo_ensemble_last_error(nullptr));
}
Ensemble::~Ensemble() { cryo_ensemble_destroy(e_); }
void Ensemble::check(int rc) const {
  if (rc) raise(rc, cryo_ensemble_last_error(e_));
}
void Ensemble::add(Solver& tank) {
  check(cryo_ensemble_add(e_, tank.handle()));
  tanks_.push_back(&tank);
}
void Ensemble::remove(Solver& tank) {
  check(cryo_ensemble_remove(e_, tank.handle()));
  tanks_.erase(std::remove(tanks_.begin(), tanks_.end(), &tank), tanks_.end());
}
std::size_t Ensemble::size() const { return tanks_.size(); }
void Ensemble::run_steps(long long n) { check(cryo_ensemble_run_steps(e_, n)); }
void Ensemble::set_chains(int chains) { check(cryo_ensemble_set_chains(e_, chains)); }
int Ensemble::chains() const {
  int k = 0;
  check(cryo_ensemble_chains(e_, &k));
  return k;
}
void Ensemble::set_steps_per_launch(int steps) { check(cryo_ensemble_set_steps_per_launch(e_, steps)); }
int Ensemble::steps_per_launch() const {
  int k = 0;
  check(cryo_ensemble_steps_per_launch(e_, &k));
  return k;
}
std::tuple<int, int, float> Ensemble::tune(const std::vector<int>& chain_candidates,
                                           const std::vector<int>& launch_candidates, int steps,
                                           const std::vector<int>& tile_candidates) {
  int best = 0, per = 0, tile = 0;
  float ms = 0.0f;
  auto ptr = [](const std::vector<int>& v) { return v.empty() ? nullptr : v.data(); };
  check(cryo_ensemble_tune_tiles(e_, ptr(chain_candidates), static_cast<int>(chain_candidates.size()),
                                 ptr(launch_candidates), static_cast<int>(launch_candidates.size()),
                                 ptr(tile_candidates), static_cast<int>(tile_candidates.size()), steps, &best, &per,
                                 &tile, &ms));
  return {best, per, ms};
}
void Ensemble::set_tile(int particles_per_thread) { check(cryo_ensemble_set_tile(e_, particles_per_thread)); }
int Ensemble::tile() const {
  int k = 0;
  check(cryo_ensemble_tile(e_, &k));
  return k;
}
float Ensemble::step_time(int steps) {
  float ms = 0.0f;
  check(cryo_ensemble_step_time(e_, steps, &ms));
  return ms;
}
int Ensemble::launches_per_step() const {
  int k = 0;
  check(cryo_ensemble_launches_per_step(e_, &k));
  return k;
}
std::uintptr_t Ensemble::stream_handle() const { return cryo_ensemble_stream(e_); }
std::vector<Diagnostics> Ensemble::diagnostics() {
  std::vector<Diagnostics> out;
  out.reserve(tanks_.size());
  for (Solver* t : tanks_) out.push_back(t->diagnostics());
  return out;
}

std::string device_name(int device) {
  char buf[256] = {0};
  if (cryo_device_name(device, buf, sizeof(buf)) != CRYO_OK) return "no CUDA device";
  return buf;
}
int device_count() { return cryo_device_count(); }

// ------------------------------------------------------------------ slabs
SlabSolver::SlabSolver(const SolverConfig& config, const FluidProperties& fluid, int slabs,
                       const std::vector<int>& devices)
    : cfg_(config), fluid_(fluid), slabs_(slabs) {
  if (!devices.empty() && static_cast<int>(devices.size()) != slabs)
    throw std::invalid_argument("SlabSolver: one device per slab");
  const cryo_config_t c = cfg_.to_c();
  const cryo_fluid_t f = fluid_.to_c();
  const int rc = cryo_slabs_create(&c, &f, slabs, devices.empty() ? nullptr : devices.data(), &s_);
  if (rc) raise(rc, cryo_slabs_last_error(nullptr));
}

SlabSolver::~SlabSolver() { cryo_slabs_destroy(s_); }

void SlabSolver::check(int rc) const {
  if (rc) raise(rc, cryo_slabs_last_error(s_));
}

void SlabSolver::set_particles(const HostParticles& hp, const AABB& domain) { set_particles(soa_view(hp), domain); }

void SlabSolver::set_particles(const cryo_host_particles_t& p, const AABB& domain) {
  float lo[3], hi[3];
  domain_floats(domain, lo, hi);
  check(cryo_slabs_set_particles(s_, &p, lo, hi));
}

void SlabSolver::download(cryo_host_particles_out_t& out) const { check(cryo_slabs_download(s_, &out)); }

// Solver::build_tank (sph_solver.cu:430-437) with the host generator.
void SlabSolver::build_tank(const Geometry& geometry, const FillSpec& fill) {
  const HostParticles hp = build_tank_particles(geometry, fluid_, cfg_.dx, fill);
  AABB dom = geometry.bounds();
  const real pad = (fill.wall_layers + 1) * cfg_.dx;
  dom.lo = dom.lo - Vec3{pad, pad, pad};
  dom.hi = dom.hi + Vec3{pad, pad, pad};
  set_particles(hp, dom);
}

void SlabSolver::run_steps(long long n) { check(cryo_slabs_run_steps(s_, n)); }

void SlabSolver::set_graph_mode(bool on) { check(cryo_slabs_set_graph_mode(s_, on ? 1 : 0)); }

int SlabSolver::graph_mode() const {
  int m = 0;
  check(cryo_slabs_graph_mode(s_, &m));
  return m;
}

Diagnostics SlabSolver::diagnostics() {
  cryo_diagnostics_t d{};
  check(cryo_slabs_diagnostics(s_, &d));
  return to_diagnostics(d);
}

std::size_t SlabSolver::num_particles() const {
  int n = 0;
  check(cryo_slabs_num_particles(s_, &n));
  return static_cast<std::size_t>(n);
}

HostParticles SlabSolver::particles() const {
  HostParticles h;
  cryo_host_particles_out_t o = soa_sink(h, num_particles());
  download(o);
  return h;
}

std::tuple<std::vector<int>, std::vector<int>, std::vector<int>> SlabSolver::layout() const {
  std::vector<int> zb(slabs_ + 1), owned(slabs_), held(slabs_);
  check(cryo_slabs_layout(s_, zb.data(), owned.data(), held.data()));
  return {zb, owned, held};
}

}  // namespace cryosph
