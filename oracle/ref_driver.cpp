// ref_driver.cpp -- C ABI over the CryoSPH-CUDA reference's CPU build.
// TEST INFRASTRUCTURE ONLY (see ref_driver.h).  Compiled by oracle/Makefile
// against the reference headers; links the reference's own objects.
#include "ref_driver.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#if defined(_OPENMP)
#include <omp.h>
#endif

#include "cryosph/core/geometry.hpp"
#include "cryosph/core/spatial_hash.hpp"
#include "cryosph/physics/SPH_kernels.cuh"
#include "cryosph/physics/navier_stokes.cuh"
#include "cryosph/physics/phase_change.cuh"
#include "cryosph/physics/surface_tension.cuh"
#include "cryosph/solvers/sph_solver.hpp"

using namespace cryosph;

// Helpers with external linkage inside sph_solver.cu (namespace solver_detail).
namespace cryosph {
namespace solver_detail {
void kick_drift(ParticleView pv, real dt, int continuity, int tvf, stream_t s);
void kick(ParticleView pv, real dt, int thermal, stream_t s);
double sum_heat_weight(ParticleView pv, stream_t s);
real max_spacing_ratio(ParticleView pv, real dx, stream_t s);
real max_fluid_speed(ParticleView pv, stream_t s);
real max_fluid_accel(ParticleView pv, stream_t s);
real max_vapor_temperature(ParticleView pv, stream_t s);
}  // namespace solver_detail
}  // namespace cryosph

namespace {

struct Handle {
  std::unique_ptr<Solver> solver;
  std::string err;
  float pass_dt = 0;
  // maxima of the last CRYO_PASS_MAXIMA hook
  float v_max = 0, a_max = 0, Tv_max = 0, spacing = 1;
};

Vec3 v3(const float* p) { return Vec3{real(p[0]), real(p[1]), real(p[2])}; }

SolverConfig to_cfg(const cryo_config_t& c) {
  SolverConfig s;
  s.dx = c.dx;
  s.h_factor = c.h_factor;
  s.kernel = static_cast<KernelType>(c.kernel);
  s.density_mode = static_cast<DensityMode>(c.density_mode);
  s.normalize_initial_masses = c.normalize_initial_masses != 0;
  s.gravity = v3(c.gravity);
  s.velocity_scale = c.velocity_scale;
  s.sound_speed = c.sound_speed;
  s.tait_gamma = c.tait_gamma;
  s.background_pressure = c.background_pressure;
  s.vapor_stiffness = c.vapor_stiffness;
  s.clamp_negative_pressure = c.clamp_negative_pressure != 0;
  s.transport_velocity = c.transport_velocity != 0;
  s.transport_background_factor = c.transport_background_factor;
  s.transport_stress = c.transport_stress != 0;
  s.transport_interface_only = c.transport_interface_only != 0;
  s.particle_shifting = c.particle_shifting != 0;
  s.shifting_strength = c.shifting_strength;
  s.artificial_viscosity = c.artificial_viscosity;
  s.artificial_viscosity_vapor = c.artificial_viscosity_vapor;
  s.delta_sph = c.delta_sph;
  s.no_slip = c.no_slip != 0;
  s.sps_turbulence = c.sps_turbulence != 0;
  s.smagorinsky_cs = c.smagorinsky_cs;
  s.surface_tension = static_cast<SurfaceTensionModel>(c.surface_tension);
  s.contact_angle_deg = c.contact_angle_deg;
  s.contact_angle_wall_weight = c.contact_angle_wall_weight;
  s.wall_colour = c.wall_colour != 0;
  s.wetting_model = static_cast<WettingModel>(c.wetting_model);
  s.csf_smooth_normals = c.csf_smooth_normals != 0;
  s.csf_balanced = c.csf_balanced != 0;
  s.akinci_gamma = c.akinci_gamma;
  s.akinci_beta = c.akinci_beta;
  s.thermal = c.thermal != 0;
  s.phase_change = c.phase_change != 0;
  s.wall_thermal_bc = static_cast<WallThermalBC>(c.wall_thermal_bc);
  s.heater_power = c.heater_power;
  s.conductivity_scale = c.conductivity_scale;
  s.lee_evaporation = c.lee_evaporation;
  s.lee_condensation = c.lee_condensation;
  s.thermo_mode = static_cast<TankThermoMode>(c.thermo_mode);
  s.vent_relaxation = c.vent_relaxation;
  s.merge_ratio = c.merge_ratio;
  s.split_ratio = c.split_ratio;
  s.max_transfer_fraction = c.max_transfer_fraction;
  s.phase_change_density_limit = c.phase_change_density_limit;
  s.vapor_mass_rebalance = c.vapor_mass_rebalance;
  s.cfl = c.cfl;
  s.viscous_number = c.viscous_number;
  s.force_number = c.force_number;
  s.capillary_number = c.capillary_number;
  s.thermal_number = c.thermal_number;
  s.dt_max = c.dt_max;
  s.dt_min = c.dt_min;
  s.fixed_dt = c.fixed_dt;
  return s;
}

FluidProperties to_fluid(const cryo_fluid_t& f) {
  FluidProperties p;
  p.name = "custom";
  p.rho_liquid = f.rho_liquid;
  p.rho_vapor = f.rho_vapor;
  p.mu_liquid = f.mu_liquid;
  p.mu_vapor = f.mu_vapor;
  p.k_liquid = f.k_liquid;
  p.k_vapor = f.k_vapor;
  p.cp_liquid = f.cp_liquid;
  p.cp_vapor = f.cp_vapor;
  p.sigma = f.sigma;
  p.h_fg = f.h_fg;
  p.T_sat = f.T_sat;
  p.p_sat = f.p_sat;
  p.R_gas = f.R_gas;
  return p;
}

std::shared_ptr<const Geometry> make_geom(const ref_geom_node_t* nodes, int n, int idx) {
  if (idx < 0 || idx >= n) throw std::invalid_argument("geometry node index out of range");
  const ref_geom_node_t& g = nodes[idx];
  switch (g.kind) {
    case REF_GEOM_CYLINDER: return std::make_shared<CylinderTank>(g.p[0], g.p[1]);
    case REF_GEOM_CAPSULE: return std::make_shared<CapsuleTank>(g.p[0], g.p[1]);
    case REF_GEOM_SPHERE: return std::make_shared<SphereTank>(g.p[0]);
    case REF_GEOM_BOX: return std::make_shared<BoxTank>(g.p[0], g.p[1], g.p[2]);
    case REF_GEOM_TRANSLATED:
      return std::make_shared<Translated>(make_geom(nodes, n, g.a),
                                          Vec3{real(g.p[0]), real(g.p[1]), real(g.p[2])});
    case REF_GEOM_DIFFERENCE: return std::make_shared<Difference>(make_geom(nodes, n, g.a), make_geom(nodes, n, g.b));
    case REF_GEOM_UNION: return std::make_shared<Union>(make_geom(nodes, n, g.a), make_geom(nodes, n, g.b));
    default: throw std::invalid_argument("unknown geometry kind");
  }
}

FillSpec to_fill(const ref_fill_t& f) {
  FillSpec s;
  s.mode = static_cast<FillMode>(f.mode);
  s.fill_fraction = f.fill_fraction;
  s.settle_direction = v3(f.settle_direction);
  s.bubble_center = v3(f.bubble_center);
  s.include_vapor = f.include_vapor != 0;
  s.wall_layers = f.wall_layers;
  s.T_liquid = f.T_liquid;
  s.T_vapor = f.T_vapor;
  s.T_wall = f.T_wall;
  s.heater_zmin = f.heater_zmin;
  s.heater_zmax = f.heater_zmax;
  return s;
}

HostParticles to_host(const cryo_host_particles_t& p) {
  HostParticles hp;
  hp.reserve(static_cast<std::size_t>(p.n));
  for (int i = 0; i < p.n; ++i) {
    const Vec3 x = v3(p.x + 3 * i);
    const Vec3 v = p.v ? v3(p.v + 3 * i) : Vec3{0, 0, 0};
    const Vec3 nn = p.nrm ? v3(p.nrm + 3 * i) : Vec3{0, 0, 0};
    hp.push(x, v, p.m[i], p.rho[i], p.T[i], static_cast<Phase>(p.phase[i]), nn, p.flags ? p.flags[i] : 0);
    if (p.id) hp.id.back() = p.id[i];
  }
  return hp;
}

template <class F>
int guard(Handle* h, F&& f) {
  try {
    f();
    return CRYO_OK;
  } catch (const std::invalid_argument& e) {
    if (h) h->err = e.what();
    return CRYO_EINVAL;
  } catch (const std::out_of_range& e) {
    if (h) h->err = e.what();
    return CRYO_ERANGE;
  } catch (const std::exception& e) {
    if (h) h->err = e.what();
    return CRYO_ERUNTIME;
  }
}

template <class T, class U>
void copy_out(const DeviceArray<T>& a, int n, U* out) {
  const std::vector<T> v = a.to_host(static_cast<std::size_t>(n));
  std::memcpy(out, v.data(), v.size() * sizeof(T));
}

void fill_out(const HostParticles& hp, cryo_host_particles_out_t* out) {
  const int n = static_cast<int>(hp.size());
  out->n = n;
  const std::size_t nn = static_cast<std::size_t>(n > 0 ? n : 1);
  out->x = static_cast<float*>(std::malloc(nn * 3 * sizeof(float)));
  out->v = static_cast<float*>(std::malloc(nn * 3 * sizeof(float)));
  out->nrm = static_cast<float*>(std::malloc(nn * 3 * sizeof(float)));
  out->m = static_cast<float*>(std::malloc(nn * sizeof(float)));
  out->rho = static_cast<float*>(std::malloc(nn * sizeof(float)));
  out->T = static_cast<float*>(std::malloc(nn * sizeof(float)));
  out->phase = static_cast<uint8_t*>(std::malloc(nn));
  out->flags = static_cast<uint8_t*>(std::malloc(nn));
  out->id = static_cast<uint32_t*>(std::malloc(nn * sizeof(uint32_t)));
  for (int i = 0; i < n; ++i) {
    const std::size_t k = static_cast<std::size_t>(i);
    out->x[3 * k] = float(hp.x[k].x); out->x[3 * k + 1] = float(hp.x[k].y); out->x[3 * k + 2] = float(hp.x[k].z);
    out->v[3 * k] = float(hp.v[k].x); out->v[3 * k + 1] = float(hp.v[k].y); out->v[3 * k + 2] = float(hp.v[k].z);
    out->nrm[3 * k] = float(hp.nrm[k].x); out->nrm[3 * k + 1] = float(hp.nrm[k].y); out->nrm[3 * k + 2] = float(hp.nrm[k].z);
    out->m[k] = float(hp.m[k]);
    out->rho[k] = float(hp.rho[k]);
    out->T[k] = float(hp.T[k]);
    out->phase[k] = hp.phase[k];
    out->flags[k] = hp.flags[k];
    out->id[k] = hp.id[k];
  }
}

SimParams& mut_params(Solver& s) { return const_cast<SimParams&>(s.params()); }

}  // namespace

extern "C" {

int ref_real_size(void) { return static_cast<int>(sizeof(real)); }

void ref_set_threads(int n) {
#if defined(_OPENMP)
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int ref_get_threads(void) {
#if defined(_OPENMP)
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void* ref_create(const cryo_config_t* cfg, const cryo_fluid_t* fluid, char* err, int errlen) {
  try {
    auto* h = new Handle;
    h->solver = std::make_unique<Solver>(to_cfg(*cfg), to_fluid(*fluid));
    return h;
  } catch (const std::exception& e) {
    if (err && errlen > 0) {
      std::strncpy(err, e.what(), static_cast<std::size_t>(errlen - 1));
      err[errlen - 1] = 0;
    }
    return nullptr;
  }
}

void ref_destroy(void* h) { delete static_cast<Handle*>(h); }
const char* ref_last_error(void* h) { return static_cast<Handle*>(h)->err.c_str(); }

int ref_set_particles(void* hv, const cryo_host_particles_t* p, const float* lo, const float* hi) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->set_particles(to_host(*p), AABB{v3(lo), v3(hi)}); });
}

int ref_build_tank(void* hv, const ref_geom_node_t* nodes, int n_nodes, const ref_fill_t* fill) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->build_tank(*make_geom(nodes, n_nodes, n_nodes - 1), to_fill(*fill)); });
}

int ref_tank_particles(const ref_geom_node_t* nodes, int n_nodes, const cryo_fluid_t* fluid, float dx,
                       const ref_fill_t* fill, cryo_host_particles_out_t* out) {
  return guard(nullptr, [&] {
    const HostParticles hp =
        build_tank_particles(*make_geom(nodes, n_nodes, n_nodes - 1), to_fluid(*fluid), dx, to_fill(*fill));
    fill_out(hp, out);
  });
}

void ref_free_particles(cryo_host_particles_out_t* o) {
  std::free(o->x); std::free(o->v); std::free(o->nrm); std::free(o->m); std::free(o->rho);
  std::free(o->T); std::free(o->phase); std::free(o->flags); std::free(o->id);
  std::memset(o, 0, sizeof(*o));
}

int ref_tank_domain(const ref_geom_node_t* nodes, int n_nodes, float dx, int wall_layers, float* lo, float* hi) {
  return guard(nullptr, [&] {
    AABB dom = make_geom(nodes, n_nodes, n_nodes - 1)->bounds();
    const real pad = (wall_layers + 1) * real(dx);
    dom.lo = dom.lo - Vec3{pad, pad, pad};
    dom.hi = dom.hi + Vec3{pad, pad, pad};
    lo[0] = float(dom.lo.x); lo[1] = float(dom.lo.y); lo[2] = float(dom.lo.z);
    hi[0] = float(dom.hi.x); hi[1] = float(dom.hi.y); hi[2] = float(dom.hi.z);
  });
}

double ref_geom_sdf(const ref_geom_node_t* nodes, int n_nodes, double x, double y, double z) {
  return make_geom(nodes, n_nodes, n_nodes - 1)->sdf(x, y, z);
}

int ref_step(void* hv, long long n) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->run_steps(n); });
}
int ref_run_until(void* hv, double t) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->run_until(t); });
}
int ref_relax(void* hv, double d, float damping) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->relax(d, damping); });
}
int ref_next_dt(void* hv, double* dt) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { *dt = h->solver->next_dt(); });
}
int ref_time(void* hv, double* t, long long* step, double* last_dt) {
  auto* h = static_cast<Handle*>(hv);
  *t = h->solver->time();
  *step = h->solver->step_count();
  *last_dt = h->solver->last_dt();
  return CRYO_OK;
}
int ref_num_particles(void* hv) { return static_cast<int>(static_cast<Handle*>(hv)->solver->num_particles()); }

int ref_diagnostics(void* hv, cryo_diagnostics_t* o) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] {
    const Diagnostics d = h->solver->diagnostics();
    std::memset(o, 0, sizeof(*o));
    o->time = d.time; o->step = d.step; o->dt = d.dt;
    o->n_total = d.n_total; o->n_liquid = d.n_liquid; o->n_vapor = d.n_vapor; o->n_wall = d.n_wall;
    o->mass_liquid = d.mass_liquid; o->mass_vapor = d.mass_vapor; o->mass_total = d.mass_total;
    o->kinetic_energy = d.kinetic_energy; o->enthalpy = d.enthalpy; o->heat_input = d.heat_input;
    o->evaporated_mass = d.evaporated_mass; o->condensed_mass = d.condensed_mass;
    o->vented_mass = d.vented_mass; o->vented_enthalpy = d.vented_enthalpy;
    o->T_sat = d.T_sat; o->p_ullage = d.p_ullage; o->max_speed = d.max_speed;
    o->T_liquid_mean = d.T_liquid_mean; o->T_liquid_max = d.T_liquid_max; o->T_vapor_mean = d.T_vapor_mean;
    auto put = [](float* dst, Vec3 v) { dst[0] = float(v.x); dst[1] = float(v.y); dst[2] = float(v.z); };
    put(o->liquid_com, d.liquid_com);
    put(o->liquid_momentum, d.liquid_momentum);
    o->splits = d.splits; o->merges = d.merges;
    put(o->slosh_force, d.slosh_force);
    put(o->slosh_moment, d.slosh_moment);
    put(o->frame_acceleration, d.frame_acceleration);
    put(o->frame_angular_velocity, d.frame_angular_velocity);
  });
}

int ref_get_field(void* hv, int field, void* out) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] {
    ParticleSystem& ps = h->solver->particle_system();
    const int n = static_cast<int>(ps.size());
    switch (field) {
      case CRYO_F_X: copy_out(ps.x, n, static_cast<char*>(out)); break;
      case CRYO_F_V: copy_out(ps.v, n, static_cast<char*>(out)); break;
      case CRYO_F_VT: copy_out(ps.vt, n, static_cast<char*>(out)); break;
      case CRYO_F_NRM: copy_out(ps.nrm, n, static_cast<char*>(out)); break;
      case CRYO_F_M: copy_out(ps.m, n, static_cast<char*>(out)); break;
      case CRYO_F_M0: copy_out(ps.m0, n, static_cast<char*>(out)); break;
      case CRYO_F_RHO: copy_out(ps.rho, n, static_cast<char*>(out)); break;
      case CRYO_F_T: copy_out(ps.T, n, static_cast<char*>(out)); break;
      case CRYO_F_PHASE: copy_out(ps.phase, n, static_cast<char*>(out)); break;
      case CRYO_F_FLAGS: copy_out(ps.flags, n, static_cast<char*>(out)); break;
      case CRYO_F_ID: copy_out(ps.id, n, static_cast<char*>(out)); break;
      case CRYO_F_A: copy_out(ps.a, n, static_cast<char*>(out)); break;
      case CRYO_F_AB: copy_out(ps.ab, n, static_cast<char*>(out)); break;
      case CRYO_F_FW: copy_out(ps.fw, n, static_cast<char*>(out)); break;
      case CRYO_F_MW: copy_out(ps.mw, n, static_cast<char*>(out)); break;
      case CRYO_F_NS: copy_out(ps.ns, n, static_cast<char*>(out)); break;
      case CRYO_F_VW: copy_out(ps.vw, n, static_cast<char*>(out)); break;
      case CRYO_F_P: copy_out(ps.p, n, static_cast<char*>(out)); break;
      case CRYO_F_DRHO: copy_out(ps.drho, n, static_cast<char*>(out)); break;
      case CRYO_F_DTDT: copy_out(ps.dTdt, n, static_cast<char*>(out)); break;
      case CRYO_F_SIGMA: copy_out(ps.sigma, n, static_cast<char*>(out)); break;
      case CRYO_F_KAPPA: copy_out(ps.kappa, n, static_cast<char*>(out)); break;
      case CRYO_F_NU_T: copy_out(ps.nu_t, n, static_cast<char*>(out)); break;
      case CRYO_F_ALPHA: copy_out(ps.alpha, n, static_cast<char*>(out)); break;
      case CRYO_F_WALL_W: copy_out(ps.wall_w, n, static_cast<char*>(out)); break;
      case CRYO_F_HEAT_W: copy_out(ps.heat_w, n, static_cast<char*>(out)); break;
      case CRYO_F_OUT_M: copy_out(ps.out_m, n, static_cast<char*>(out)); break;
      case CRYO_F_OUT_H: copy_out(ps.out_h, n, static_cast<char*>(out)); break;
      case CRYO_F_W_NORM: copy_out(ps.w_norm, n, static_cast<char*>(out)); break;
      case CRYO_F_RMIN: copy_out(ps.rmin, n, static_cast<char*>(out)); break;
      case CRYO_F_P_WV: copy_out(ps.p_wv, n, static_cast<char*>(out)); break;
      default: throw std::invalid_argument("unknown field");
    }
  });
}

int ref_params(void* hv, float* c0, float* hsm, float* vol0, float* support2, float* T_sat, float* dt,
               float* heat_inv_norm) {
  auto* h = static_cast<Handle*>(hv);
  const SimParams& P = h->solver->params();
  *c0 = float(P.c0);
  *hsm = float(P.kernel.h);
  *vol0 = float(P.vol0);
  *support2 = float(P.support2);
  *T_sat = float(P.T_sat);
  *dt = float(P.dt);
  *heat_inv_norm = float(P.heat_inv_norm);
  return CRYO_OK;
}

int ref_set_gravity(void* hv, const float* g) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->set_gravity(v3(g)); });
}
int ref_set_frame_motion(void* hv, const float* a, const float* w, const float* wd, const float* o) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->set_frame_motion(v3(a), v3(w), v3(wd), v3(o)); });
}
int ref_set_maneuver(void* hv, int n, const double* t, const float* acc, const float* omega, const float* o) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] {
    ManeuverProfile p;
    p.time.assign(t, t + n);
    for (int k = 0; k < n; ++k) p.acceleration.push_back(v3(acc + 3 * k));
    if (omega)
      for (int k = 0; k < n; ++k) p.angular_velocity.push_back(v3(omega + 3 * k));
    p.origin = o ? v3(o) : Vec3{0, 0, 0};
    h->solver->set_maneuver(p);
  });
}
int ref_clear_frame_motion(void* hv) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->clear_frame_motion(); });
}
int ref_set_heater_power(void* hv, float w) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->set_heater_power(w); });
}
int ref_set_contact_angle(void* hv, float deg) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->set_contact_angle(deg); });
}
int ref_damp_velocities(void* hv, float f) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] { h->solver->damp_velocities(f); });
}
int ref_probe_pressure(void* hv, const float* pts, int np, float* out) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] {
    std::vector<Vec3> v(static_cast<std::size_t>(np));
    for (int k = 0; k < np; ++k) v[static_cast<std::size_t>(k)] = v3(pts + 3 * k);
    const std::vector<real> r = h->solver->probe_pressure(v);
    for (int k = 0; k < np; ++k) out[k] = float(r[static_cast<std::size_t>(k)]);
  });
}

int ref_set_dt(void* hv, float dt) {
  auto* h = static_cast<Handle*>(hv);
  h->pass_dt = dt;
  return CRYO_OK;
}

int ref_pass(void* hv, int pass) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] {
    Solver& s = *h->solver;
    SimParams& P = mut_params(s);
    P.dt = h->pass_dt;
    ParticleSystem& ps = s.particle_system();
    SpatialHash& grid = s.grid();
    const stream_t st = s.stream();
    const SolverConfig& c = s.config();
    ParticleView pv = ps.view();
    const GridView gv = grid.view();
    switch (pass) {
      case CRYO_PASS_KICK_DRIFT:
        solver_detail::kick_drift(pv, P.dt, c.density_mode == DensityMode::Continuity, P.tvf, st);
        break;
      case CRYO_PASS_GRID_BUILD: grid.build(ps, st); break;
      case CRYO_PASS_DENSITY: compute_density_summation(pv, gv, P, st); break;
      case CRYO_PASS_NORMALIZE_MASSES: normalize_initial_masses(pv, gv, P, st); break;
      case CRYO_PASS_EOS: compute_equation_of_state(pv, P, st); break;
      case CRYO_PASS_WALL_BOUNDARY: compute_wall_boundary(pv, gv, P, st); break;
      case CRYO_PASS_INTERFACE: compute_interface_fields(pv, gv, P, st); break;
      case CRYO_PASS_TRANSPORT: compute_transport_acceleration(pv, gv, P, st); break;
      case CRYO_PASS_SPS: compute_sps_viscosity(pv, gv, P, st); break;
      case CRYO_PASS_MOMENTUM: compute_momentum(pv, gv, P, st); break;
      case CRYO_PASS_SMOOTH_NORMALS: smooth_interface_normals(pv, gv, P, st); break;
      case CRYO_PASS_CSF: apply_csf_surface_tension(pv, gv, P, st); break;
      case CRYO_PASS_AKINCI: apply_akinci_surface_tension(pv, gv, P, st); break;
      case CRYO_PASS_DENSITY_RATE: compute_density_rate(pv, gv, P, st); break;
      case CRYO_PASS_THERMAL: {
        if (P.heat_power != real(0)) {
          const double S = solver_detail::sum_heat_weight(pv, st);
          P.heat_inv_norm = S > 0 ? static_cast<real>(1.0 / S) : real(0);
        } else {
          P.heat_inv_norm = 0;
        }
        compute_thermal_rates(pv, gv, P, st);
        break;
      }
      case CRYO_PASS_KICK: solver_detail::kick(pv, P.dt, P.thermal, st); break;
      case CRYO_PASS_PC_SOURCES: phase_change_sources(pv, P, st); break;
      case CRYO_PASS_PC_NORMALIZE: phase_change_normalize(pv, gv, P, st); break;
      case CRYO_PASS_PC_APPLY: phase_change_apply(pv, gv, P, st); break;
      case CRYO_PASS_REBALANCE: rebalance_vapor_mass(pv, gv, P, st); break;
      default: throw std::invalid_argument("pass not exposed by the reference driver");
    }
  });
}

int ref_grid_info(void* hv, int* num_cells, int* nx, int* ny, int* nz, float* origin, float* inv_cell) {
  auto* h = static_cast<Handle*>(hv);
  const GridView g = h->solver->grid().view();
  *num_cells = h->solver->grid().num_cells();
  *nx = g.nx; *ny = g.ny; *nz = g.nz;
  origin[0] = float(g.origin.x); origin[1] = float(g.origin.y); origin[2] = float(g.origin.z);
  *inv_cell = float(g.inv_cell);
  return CRYO_OK;
}

int ref_grid_tables(void* hv, int32_t* cs, int32_t* ce) {
  auto* h = static_cast<Handle*>(hv);
  const GridView g = h->solver->grid().view();
  const int nc = h->solver->grid().num_cells();
  std::memcpy(cs, g.cell_start, static_cast<std::size_t>(nc) * sizeof(int));
  std::memcpy(ce, g.cell_end, static_cast<std::size_t>(nc) * sizeof(int));
  return CRYO_OK;
}

int ref_neighbor_lists(void* hv, int32_t* counts, int32_t* list, long long cap, long long* total) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] {
    ParticleSystem& ps = h->solver->particle_system();
    const GridView g = h->solver->grid().view();
    const real s2 = h->solver->params().support2;
    const int n = static_cast<int>(ps.size());
    const Vec3* x = ps.x.data();
    long long t = 0;
    for (int i = 0; i < n; ++i) {
      const Vec3 xi = x[i];
      int c = 0;
      for_each_neighbor(g, xi, [&](int j) {
        if (norm2(xi - x[j]) < s2) {
          if (list && t < cap) list[t] = j;
          ++t;
          ++c;
        }
      });
      counts[i] = c;
    }
    *total = t;
  });
}

int ref_neighbor_stats(void* hv, float radius, int32_t* counts, uint64_t* id_sums) {
  auto* h = static_cast<Handle*>(hv);
  return guard(h, [&] {
    std::vector<int> c;
    std::vector<std::uint64_t> s;
    h->solver->grid().neighbor_stats(h->solver->particle_system(), radius, c, s, h->solver->stream());
    std::memcpy(counts, c.data(), c.size() * sizeof(int));
    std::memcpy(id_sums, s.data(), s.size() * sizeof(std::uint64_t));
  });
}

}  // extern "C"
