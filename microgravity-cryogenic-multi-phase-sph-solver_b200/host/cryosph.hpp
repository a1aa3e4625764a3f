// cryosph.hpp -- the C++ API of the B200 solver.  Same names, fields, defaults
// and exceptions as the reference's public headers (include/cryosph/...), so
// code written against cryosph::Solver compiles against this; the work is done
// by libcryosph_b200.so through the C ABI (include/cryosph_b200.h).
#pragma once

#include <array>
#include <cstdint>
#include <limits>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "cryosph_b200.h"

namespace cryosph {

using real = float;  // the FP32 build of the reference (cuda_utils.cuh:51-55)
inline constexpr real kPi = real(3.14159265358979323846);

// Vec3 (cuda_utils.cuh:85-108)
struct Vec3 {
  real x, y, z;
};
inline Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator-(Vec3 a) { return {-a.x, -a.y, -a.z}; }
inline Vec3 operator*(Vec3 a, real s) { return {a.x * s, a.y * s, a.z * s}; }
inline Vec3 operator/(Vec3 a, real s) { return {a.x / s, a.y / s, a.z / s}; }
inline real dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline real norm2(Vec3 a) { return dot(a, a); }
real norm(Vec3 a);
Vec3 normalized(Vec3 a, real eps = real(1e-20));

// particle_system.hpp:13-34
enum class Phase : std::uint8_t { Liquid = 0, Vapor = 1, Wall = 2, Dead = 3 };
inline constexpr std::uint8_t kLiquid = 0, kVapor = 1, kWall = 2, kDead = 3;
namespace pflag {
inline constexpr std::uint8_t Heated = 1u << 0;
inline constexpr std::uint8_t Source = 1u << 1;
inline constexpr std::uint8_t TargetVapor = 1u << 2;
inline constexpr std::uint8_t Dying = 1u << 3;
inline constexpr std::uint8_t ScratchMask = Source | TargetVapor | Dying;
}  // namespace pflag

// HostParticles (particle_system.hpp:76-90)
struct HostParticles {
  std::vector<Vec3> x, v, nrm;
  std::vector<real> m, rho, T;
  std::vector<std::uint8_t> phase, flags;
  std::vector<std::uint32_t> id;
  std::size_t size() const { return x.size(); }
  void reserve(std::size_t n);
  void clear();
  std::size_t push(Vec3 pos, Vec3 vel, real mass, real density, real temperature, Phase ph, Vec3 normal = {0, 0, 0},
                   std::uint8_t flag = 0);
  void append(const HostParticles& other);
};

// enums (sim_params.cuh:12-18, SPH_kernels.cuh:12, geometry.hpp:160-164, telemetry.hpp:13)
enum class KernelType : int { CubicSpline = 0, WendlandC2 = 1 };
enum class DensityMode : int { Summation = 0, Continuity = 1 };
enum class SurfaceTensionModel : int { None = 0, CSF = 1, Akinci = 2 };
enum class WallThermalBC : int { Adiabatic = 0, Isothermal = 1 };
enum class TankThermoMode : int { Vented = 0, Closed = 1 };
enum class WettingModel : int { NormalRotation = 0, ContactLineForce = 1, Both = 2 };
enum class TelemetryMode : int { AsyncCopy = 0, ZeroCopy = 1 };

// FluidProperties (fluid_properties.hpp:11-38)
struct FluidProperties {
  std::string name = "custom";
  real rho_liquid = 1000, rho_vapor = 1, mu_liquid = real(1e-3), mu_vapor = real(1e-5);
  real k_liquid = real(0.6), k_vapor = real(0.025), cp_liquid = 4180, cp_vapor = 2000;
  real sigma = real(0.072), h_fg = real(2.26e6), T_sat = real(373.15), p_sat = 101325, R_gas = real(461.5);
  real saturation_temperature(real p) const;
  real saturation_pressure(real T) const;
  static FluidProperties liquid_hydrogen();
  static FluidProperties liquid_nitrogen();
  static FluidProperties liquid_oxygen();
  static FluidProperties liquid_methane();
  static FluidProperties water();
  cryo_fluid_t to_c() const;
};

// SolverConfig (sph_solver.hpp:20-91)
struct SolverConfig {
  real dx = real(0.005), h_factor = real(1.3);
  KernelType kernel = KernelType::WendlandC2;
  DensityMode density_mode = DensityMode::Summation;
  bool normalize_initial_masses = true;
  Vec3 gravity{0, 0, real(-9.81)};
  real velocity_scale = 0, sound_speed = 0, tait_gamma = 7, background_pressure = -1, vapor_stiffness = -1;
  bool clamp_negative_pressure = false;
  bool transport_velocity = true;
  real transport_background_factor = real(2.0);
  bool transport_stress = false, transport_interface_only = true;
  bool particle_shifting = false;
  real shifting_strength = real(0.25);
  real artificial_viscosity = real(0.02), artificial_viscosity_vapor = real(0.2), delta_sph = real(0.1);
  bool no_slip = true, sps_turbulence = false;
  real smagorinsky_cs = real(0.12);
  SurfaceTensionModel surface_tension = SurfaceTensionModel::CSF;
  real contact_angle_deg = 90, contact_angle_wall_weight = real(0.01);
  bool wall_colour = true;
  WettingModel wetting_model = WettingModel::NormalRotation;
  bool csf_smooth_normals = false, csf_balanced = false;
  real akinci_gamma = -1, akinci_beta = -1;
  bool thermal = true, phase_change = true;
  WallThermalBC wall_thermal_bc = WallThermalBC::Adiabatic;
  real heater_power = 0, conductivity_scale = 1, lee_evaporation = 10, lee_condensation = 10;
  TankThermoMode thermo_mode = TankThermoMode::Vented;
  real vent_relaxation = real(0.02), merge_ratio = real(0.3), split_ratio = real(2.0);
  real max_transfer_fraction = real(0.25), phase_change_density_limit = real(0.01), vapor_mass_rebalance = real(1.0);
  real cfl = real(0.25), viscous_number = real(0.125), force_number = real(0.25), capillary_number = real(0.25);
  real thermal_number = real(0.1), dt_max = real(1e-2), dt_min = real(1e-9), fixed_dt = 0;
  cryo_config_t to_c() const;
};

// ManeuverProfile (sph_solver.hpp:96-105)
struct ManeuverProfile {
  std::vector<double> time;
  std::vector<Vec3> acceleration;
  std::vector<Vec3> angular_velocity;
  Vec3 origin{0, 0, 0};
  void evaluate(double t, Vec3& a, Vec3& omega, Vec3& omega_dot) const;
  void validate() const;
};

// Diagnostics (sph_solver.hpp:108-132)
struct Diagnostics {
  double time = 0;
  long long step = 0;
  double dt = 0;
  int n_total = 0, n_liquid = 0, n_vapor = 0, n_wall = 0;
  double mass_liquid = 0, mass_vapor = 0, mass_total = 0, kinetic_energy = 0, enthalpy = 0, heat_input = 0;
  double evaporated_mass = 0, condensed_mass = 0, vented_mass = 0, vented_enthalpy = 0;
  double T_sat = 0, p_ullage = 0, max_speed = 0, T_liquid_mean = 0, T_liquid_max = 0, T_vapor_mean = 0;
  Vec3 liquid_com{0, 0, 0}, liquid_momentum{0, 0, 0};
  int splits = 0, merges = 0;
  Vec3 slosh_force{0, 0, 0}, slosh_moment{0, 0, 0}, frame_acceleration{0, 0, 0}, frame_angular_velocity{0, 0, 0};
};

// TelemetryFrame (telemetry.hpp:16-25)
struct TelemetryFrame {
  double time = 0;
  long long step = 0;
  int n = 0;
  std::vector<float> position, temperature, pressure, speed;
  std::vector<std::uint8_t> phase;
};

// ------------------------------------------------------------- geometry
// geometry.hpp:17-183
struct AABB {
  Vec3 lo{0, 0, 0};
  Vec3 hi{0, 0, 0};
};

class Geometry {
 public:
  virtual ~Geometry() = default;
  virtual double sdf(double x, double y, double z) const = 0;
  virtual AABB bounds() const = 0;
  virtual std::string name() const = 0;
  virtual double volume() const { return -1.0; }
  Vec3 outward_normal(double x, double y, double z, double eps) const;
  // Appends this geometry's node tree for the device lattice generator
  // (children first) and returns the root's index; -1: no device form.
  virtual int emit_nodes(std::vector<cryo_geom_node_t>& out) const { (void)out; return -1; }
};

class CylinderTank final : public Geometry {
 public:
  int emit_nodes(std::vector<cryo_geom_node_t>& out) const override;
  CylinderTank(double radius, double height);
  double sdf(double x, double y, double z) const override;
  AABB bounds() const override;
  std::string name() const override { return "cylinder"; }
  double volume() const override;
  double radius() const { return R_; }
  double height() const { return H_; }

 private:
  double R_, H_;
};

class CapsuleTank final : public Geometry {
 public:
  int emit_nodes(std::vector<cryo_geom_node_t>& out) const override;
  CapsuleTank(double radius, double length);
  double sdf(double x, double y, double z) const override;
  AABB bounds() const override;
  std::string name() const override { return "capsule"; }
  double volume() const override;

 private:
  double R_, L_;
};

class SphereTank final : public Geometry {
 public:
  int emit_nodes(std::vector<cryo_geom_node_t>& out) const override;
  explicit SphereTank(double radius);
  double sdf(double x, double y, double z) const override;
  AABB bounds() const override;
  std::string name() const override { return "sphere"; }
  double volume() const override;

 private:
  double R_;
};

class BoxTank final : public Geometry {
 public:
  int emit_nodes(std::vector<cryo_geom_node_t>& out) const override;
  BoxTank(double lx, double ly, double lz);
  double sdf(double x, double y, double z) const override;
  AABB bounds() const override;
  std::string name() const override { return "box"; }
  double volume() const override;

 private:
  double hx_, hy_, hz_;
};

class Translated final : public Geometry {
 public:
  int emit_nodes(std::vector<cryo_geom_node_t>& out) const override;
  Translated(std::shared_ptr<const Geometry> g, Vec3 offset);
  double sdf(double x, double y, double z) const override;
  AABB bounds() const override;
  std::string name() const override { return "translated(" + g_->name() + ")"; }
  double volume() const override { return g_->volume(); }

 private:
  std::shared_ptr<const Geometry> g_;
  double ox_, oy_, oz_;
};

class Difference final : public Geometry {
 public:
  int emit_nodes(std::vector<cryo_geom_node_t>& out) const override;
  Difference(std::shared_ptr<const Geometry> a, std::shared_ptr<const Geometry> b);
  double sdf(double x, double y, double z) const override;
  AABB bounds() const override { return a_->bounds(); }
  std::string name() const override { return "difference(" + a_->name() + ", " + b_->name() + ")"; }

 private:
  std::shared_ptr<const Geometry> a_, b_;
};

class Union final : public Geometry {
 public:
  int emit_nodes(std::vector<cryo_geom_node_t>& out) const override;
  Union(std::shared_ptr<const Geometry> a, std::shared_ptr<const Geometry> b);
  double sdf(double x, double y, double z) const override;
  AABB bounds() const override;
  std::string name() const override { return "union(" + a_->name() + ", " + b_->name() + ")"; }

 private:
  std::shared_ptr<const Geometry> a_, b_;
};

class MeshTank final : public Geometry {
 public:
  MeshTank(const std::string& obj_path, double scale = 1.0, Vec3 offset = {0, 0, 0});
  MeshTank(std::vector<std::array<double, 3>> vertices, std::vector<std::array<int, 3>> triangles);
  double sdf(double x, double y, double z) const override;
  AABB bounds() const override;
  std::string name() const override { return "mesh"; }
  double volume() const override;
  std::size_t num_triangles() const { return tris_.size(); }
  double winding_number(double x, double y, double z) const;

 private:
  void finalize();
  std::vector<std::array<double, 3>> verts_;
  std::vector<std::array<int, 3>> tris_;
  AABB box_;
};

void load_obj(const std::string& path, std::vector<std::array<double, 3>>& vertices,
              std::vector<std::array<int, 3>>& triangles);

enum class FillMode : int { Settled = 0, CentralBubble = 1, Full = 2 };
enum class FieldArithmetic : int { Exact = CRYO_ARITH_EXACT, Fast = CRYO_ARITH_FAST };

struct FillSpec {
  FillMode mode = FillMode::Settled;
  double fill_fraction = 0.5;
  Vec3 settle_direction{0, 0, -1};
  Vec3 bubble_center{0, 0, 0};
  bool include_vapor = true;
  int wall_layers = 3;
  real T_liquid = std::numeric_limits<real>::quiet_NaN();
  real T_vapor = std::numeric_limits<real>::quiet_NaN();
  real T_wall = std::numeric_limits<real>::quiet_NaN();
  double heater_zmin = -std::numeric_limits<double>::infinity();
  double heater_zmax = std::numeric_limits<double>::infinity();
};

HostParticles build_tank_particles(const Geometry& geo, const FluidProperties& fluid, real dx, const FillSpec& fill);
HostParticles make_block(Vec3 lo, Vec3 hi, real dx, Phase phase, real density, real temperature);

// ------------------------------------------------------------------ I/O
// io.hpp:13-22
void write_vtk(const std::string& path, const HostParticles& particles, const std::vector<real>& pressure = {});
void write_json_frame(const std::string& path, const TelemetryFrame& frame, bool include_walls = true);
TelemetryFrame make_frame(const HostParticles& particles, const std::vector<real>& pressure, double time,
                          long long step);

// --------------------------------------------------------------- solver
// Solver (sph_solver.hpp:134-232) over a cryo_ctx.
class Solver {
 public:
  Solver(const SolverConfig& config, const FluidProperties& fluid, int device = 0);
  ~Solver();
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;

  void set_particles(const HostParticles& particles, const AABB& domain);
  // the same from caller-owned arrays in the C ABI's layout (no host copy)
  void set_particles(const cryo_host_particles_t& particles, const AABB& domain);
  // Columns of floats or doubles (cryo_set_particles_columns): doubles are
  // rounded to float while they are copied into the transfer buffer.
  void set_particles(const cryo_host_columns_t& particles, const AABB& domain);
  // on_device: generate the lattice on the GPU where the geometry has a
  // device form (the particles are the same as the host generator's)
  void build_tank(const Geometry& geometry, const FillSpec& fill, bool on_device = true);

  void step();
  void run_steps(long long n);
  void run_until(double t_end);

  double time() const;
  long long step_count() const;
  double last_dt() const;
  double next_dt();

  Diagnostics diagnostics();
  // Non-blocking diagnostics: request after a step, fetch in request order
  // (false while the oldest result is not ready and wait is false, or when
  // nothing is pending).
  void request_diagnostics();
  bool fetch_diagnostics(Diagnostics& out, bool wait = true);
  HostParticles particles() const;
  // particles() into caller-owned arrays (out.n >= num_particles())
  void download(cryo_host_particles_out_t& out) const;
  std::vector<real> pressure() const;
  std::vector<real> curvature() const;
  std::vector<real> field(int cryo_field) const;
  std::size_t num_particles() const;

  void set_gravity(Vec3 g);
  void set_frame_motion(Vec3 acceleration, Vec3 angular_velocity, Vec3 angular_acceleration, Vec3 origin);
  void set_maneuver(const ManeuverProfile& profile);
  void clear_frame_motion();
  void set_heater_power(real watts);
  void set_contact_angle(real degrees);
  void damp_velocities(real factor);
  void relax(double duration, real damping = real(0.98));

  const SolverConfig& config() const noexcept { return cfg_; }
  const FluidProperties& fluid() const noexcept { return fluid_; }
  real sound_speed() const;
  real smoothing_length() const;
  std::string device() const;

  // telemetry (TelemetryStream through the solver, sph_solver.hpp:183-189)
  void configure_telemetry(TelemetryMode mode);
  TelemetryMode telemetry_mode() const;
  bool request_telemetry();
  bool telemetry_ready() const;
  bool telemetry_pending() const;
  bool fetch_telemetry(TelemetryFrame& out);

  std::vector<real> probe_pressure(const std::vector<Vec3>& points);

  // write_vtk(path, particles(), pressure()) and write_json_frame(path,
  // make_frame(...)) of the reference, with the payload packed on the device
  void write_vtk(const std::string& path) const;
  void write_json(const std::string& path, bool include_walls = false) const;

  // B200 extensions
  cryo_ctx* handle() const noexcept { return ctx_; }
  std::uintptr_t stream_handle() const;
  void set_graph_mode(bool on);
  // Seeded uniform jitter of the fluid lattice on the device, before the
  // first step (walls stay on the lattice; cryo_jitter_fluid).
  void jitter_fluid(real amplitude, std::uint64_t seed);
  // Exact: the reference's IEEE operation sequence in the neighbour passes
  // (bit-identical to its CPU build); Fast: contracted, within 1e-5 of it.
  void set_field_arithmetic(FieldArithmetic mode);
  FieldArithmetic field_arithmetic() const;
  std::vector<std::uint8_t> save_state() const;
  void load_state(const std::vector<std::uint8_t>& blob);

  // Differentiated window (cryo_adj_*): objectives of `steps` steps from the
  // current state, then the gradients of seed . objectives by the reverse
  // passes (include/cryosph_b200.h describes both).
  std::array<double, 7> adjoint_forward(long long steps, int checkpoint_every = 20);
  struct AdjointGradients {
    double sigma = 0, contact_angle = 0, lee_evaporation = 0, lee_condensation = 0, heater_power = 0;
    std::vector<double> frame_acceleration;  // 3 per step
  };
  AdjointGradients adjoint_backward(const std::array<double, 7>& seed);
  std::size_t adjoint_memory() const;
  void adjoint_release();
  void set_surface_tension(real sigma);
  void set_lee_coefficients(real evaporation, real condensation);

 private:
  void check(int rc) const;
  SolverConfig cfg_;
  FluidProperties fluid_;
  cryo_ctx* ctx_ = nullptr;
  long long adj_steps_ = 0;
};

// Batched stepping of independent tanks (no counterpart in the reference):
// one ensemble step advances every member Solver by one of its own steps in a
// single graph launch; each member's results equal stepping it alone.
class Ensemble {
 public:
  explicit Ensemble(int device = 0);
  ~Ensemble();
  Ensemble(const Ensemble&) = delete;
  Ensemble& operator=(const Ensemble&) = delete;

  void add(Solver& tank);
  void remove(Solver& tank);
  std::size_t size() const;
  void run_steps(long long n);
  void set_chains(int chains);  // concurrent branches; 0 = one per member
  int chains() const;
  void set_steps_per_launch(int steps);  // 1, 2, 4, 8 or 16
  int steps_per_launch() const;
  // Times `steps` steps per (branch count, steps per launch) candidate and
  // keeps the fastest; returns (branches, steps per launch, ms per step).
  // The timed steps advance the members.
  // Times `steps` steps per (branch count, steps per launch, tile) candidate
  // and keeps the fastest; returns (branches, steps per launch, ms per step).
  std::tuple<int, int, float> tune(const std::vector<int>& chain_candidates, const std::vector<int>& launch_candidates,
                                   int steps, const std::vector<int>& tile_candidates = {});
  void set_tile(int particles_per_thread);  // particles per thread of the members' kernels (1..64)
  int tile() const;
  float step_time(int steps);
  int launches_per_step() const;
  std::uintptr_t stream_handle() const;
  std::vector<Diagnostics> diagnostics();

 private:
  void check(int rc) const;
  cryo_ensemble* e_ = nullptr;
  std::vector<Solver*> tanks_;
};

// One tank cut along z into slabs of cell layers, each slab a context on its
// own device (or several on one device), halo layers exchanged between
// passes (no counterpart in the reference).  The particles equal a Solver's
// over the same steps, in the same order.
class SlabSolver {
 public:
  SlabSolver(const SolverConfig& config, const FluidProperties& fluid, int slabs,
             const std::vector<int>& devices = {});
  ~SlabSolver();
  SlabSolver(const SlabSolver&) = delete;
  SlabSolver& operator=(const SlabSolver&) = delete;

  void set_particles(const HostParticles& particles, const AABB& domain);
  void set_particles(const cryo_host_particles_t& particles, const AABB& domain);
  void build_tank(const Geometry& geometry, const FillSpec& fill);  // the host lattice generator
  void step() { run_steps(1); }
  void run_steps(long long n);
  Diagnostics diagnostics();
  HostParticles particles() const;
  void download(cryo_host_particles_out_t& out) const;
  std::size_t num_particles() const;
  int slabs() const noexcept { return slabs_; }
  // 1 (default): the group's step is one captured CUDA graph; 0: host
  // threads per slab.  graph_mode() reports 0, 1, or 2 (on, capture refused).
  void set_graph_mode(bool on);
  int graph_mode() const;
  // cell-layer boundaries (slabs + 1 entries), then per slab the particles
  // it owns and the particles its context holds (owned + ghost copies)
  std::tuple<std::vector<int>, std::vector<int>, std::vector<int>> layout() const;
  const SolverConfig& config() const noexcept { return cfg_; }

 private:
  void check(int rc) const;
  SolverConfig cfg_;
  FluidProperties fluid_;
  cryo_slabs* s_ = nullptr;
  int slabs_ = 0;
};

std::string device_name(int device = 0);
int device_count();

}  // namespace cryosph
