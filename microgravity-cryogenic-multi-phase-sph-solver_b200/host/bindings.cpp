// bindings.cpp -- Python module `CryoSPH` with the reference's Python API
// (src/python/bindings.cpp:133-499): the same classes, attribute names,
// argument names and defaults; arrays cross as NumPy copies; step / run_steps /
// run_until / relax release the GIL; std::invalid_argument -> ValueError.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <cstring>
#include <string>
#include <vector>

#include "cryosph.hpp"

namespace py = pybind11;
using namespace cryosph;

namespace {

using Triple = std::array<double, 3>;
using F64 = py::array_t<double, py::array::c_style | py::array::forcecast>;
using F32 = py::array_t<float, py::array::c_style | py::array::forcecast>;
using U8 = py::array_t<std::uint8_t, py::array::c_style | py::array::forcecast>;
using U32 = py::array_t<std::uint32_t, py::array::c_style | py::array::forcecast>;

Vec3 vec(const Triple& t) { return {static_cast<real>(t[0]), static_cast<real>(t[1]), static_cast<real>(t[2])}; }
py::tuple triple(Vec3 v) { return py::make_tuple(static_cast<double>(v.x), static_cast<double>(v.y), static_cast<double>(v.z)); }

// A NumPy array of the given shape filled from `src` (element count = the shape's product).
template <class T>
py::array_t<T> numpy_copy(const T* src, std::initializer_list<py::ssize_t> shape) {
  py::array_t<T> out{std::vector<py::ssize_t>(shape)};
  if (out.size() > 0) std::memcpy(out.mutable_data(), src, static_cast<std::size_t>(out.size()) * sizeof(T));
  return out;
}
template <class T>
py::array_t<T> numpy_copy(const std::vector<T>& v) {
  return numpy_copy(v.data(), {static_cast<py::ssize_t>(v.size())});
}

// One input column of a particle set, converted to the solver's element type
// by NumPy: n rows of `width` values ((n, 3) for vectors, n values otherwise).
template <class Arr>
Arr column(py::handle src, py::ssize_t n, int width, const char* name) {
  Arr a = py::cast<Arr>(src);
  const bool ok = width == 3 ? (a.ndim() == 2 && a.shape(0) == n && a.shape(1) == 3) : a.size() == n;
  if (!ok)
    throw std::invalid_argument(std::string(name) + (width == 3 ? ": expected an array of shape (N, 3)"
                                                                : ": expected N values (one per particle)"));
  return a;
}

// One float column of a particle set: a C-contiguous float64 array is kept
// as it is (the upload rounds each value while copying it into the transfer
// buffer), anything else becomes float32 through NumPy.
struct FloatColumn {
  py::array arr;
  bool f64 = false;
  bool present = false;
};
FloatColumn float_column(py::handle src, py::ssize_t n, int width, const char* name) {
  FloatColumn c;
  c.present = true;
  if (py::isinstance<py::array_t<double, py::array::c_style>>(src)) {
    c.arr = py::reinterpret_borrow<py::array>(src);
    c.f64 = true;
  } else {
    c.arr = py::cast<F32>(src);
  }
  const bool ok = width == 3 ? (c.arr.ndim() == 2 && (n < 0 || c.arr.shape(0) == n) && c.arr.shape(1) == 3)
                             : c.arr.size() == n;
  if (!ok)
    throw std::invalid_argument(std::string(name) + (width == 3 ? ": expected an array of shape (N, 3)"
                                                                : ": expected N values (one per particle)"));
  return c;
}

// The particle set a caller hands over; columns() gives the C ABI's typed
// columns over it (float or double per column, absent columns null), view()
// the all-float structure of arrays (double columns converted by NumPy).
struct ParticleColumns {
  FloatColumn x, v, nrm, m, rho, T;
  U8 phase, flags;
  bool has_flags = false;
  py::ssize_t n = 0;
  mutable std::vector<F32> f32_copies;

  ParticleColumns(py::handle position, py::handle mass, py::handle density, py::handle temperature,
                  py::handle phase_in, py::handle velocity, py::handle normal, py::handle flags_in) {
    x = float_column(position, -1, 3, "position");
    n = x.arr.shape(0);
    m = float_column(mass, n, 1, "mass");
    rho = float_column(density, n, 1, "density");
    T = float_column(temperature, n, 1, "temperature");
    phase = column<U8>(phase_in, n, 1, "phase");
    const std::uint8_t* ph = phase.data();
    for (py::ssize_t i = 0; i < n; ++i)
      if (ph[i] > kWall) throw std::invalid_argument("phase: values must be 0 (liquid), 1 (vapour) or 2 (wall)");
    if (!velocity.is_none()) v = float_column(velocity, n, 3, "velocity");
    if (!normal.is_none()) nrm = float_column(normal, n, 3, "normal");
    if ((has_flags = !flags_in.is_none())) flags = column<U8>(flags_in, n, 1, "flags");
  }
  cryo_host_columns_t columns() const {
    auto d = [](const FloatColumn& c) { return c.present ? c.arr.data() : nullptr; };
    return cryo_host_columns_t{static_cast<int>(n), d(x), d(v), d(nrm), d(m), d(rho), d(T),
                               x.f64, v.f64, nrm.f64, m.f64, rho.f64, T.f64,
                               phase.data(), has_flags ? flags.data() : nullptr, nullptr};
  }
  cryo_host_particles_t view() const {
    auto f = [&](const FloatColumn& c) -> const float* {
      if (!c.present) return nullptr;
      if (!c.f64) return static_cast<const float*>(c.arr.data());
      f32_copies.push_back(py::cast<F32>(c.arr));
      return f32_copies.back().data();
    };
    return cryo_host_particles_t{static_cast<int>(n), f(x), f(v), f(nrm), f(m), f(rho), f(T), phase.data(),
                                 has_flags ? flags.data() : nullptr, nullptr};
  }
};

// The state of a solver (anything with num_particles() and download()) as
// the reference's dict of NumPy arrays, filled in place by one download.
template <class S>
py::dict state_dict(const S& s) {
  const auto n = static_cast<py::ssize_t>(s.num_particles());
  py::array_t<real> x({n, py::ssize_t{3}}), v({n, py::ssize_t{3}}), nrm({n, py::ssize_t{3}});
  py::array_t<real> m(n), rho(n), T(n);
  py::array_t<std::uint8_t> phase(n), flags(n);
  py::array_t<std::uint32_t> id(n);
  cryo_host_particles_out_t o{static_cast<int>(n), x.mutable_data(), v.mutable_data(), nrm.mutable_data(),
                              m.mutable_data(), rho.mutable_data(), T.mutable_data(), phase.mutable_data(),
                              flags.mutable_data(), id.mutable_data()};
  {
    py::gil_scoped_release nogil;
    s.download(o);
  }
  py::dict d;
  d["position"] = x;
  d["velocity"] = v;
  d["normal"] = nrm;
  d["mass"] = m;
  d["density"] = rho;
  d["temperature"] = T;
  d["phase"] = phase;
  d["flags"] = flags;
  d["id"] = id;
  return d;
}

// Host particles (the generators' output) as the same dict.
py::dict host_dict(const HostParticles& hp) {
  const auto n = static_cast<py::ssize_t>(hp.size());
  auto vecs = [n](const std::vector<Vec3>& a) { return numpy_copy(reinterpret_cast<const real*>(a.data()), {n, 3}); };
  py::dict d;
  d["position"] = vecs(hp.x);
  d["velocity"] = vecs(hp.v);
  d["normal"] = vecs(hp.nrm);
  d["mass"] = numpy_copy(hp.m);
  d["density"] = numpy_copy(hp.rho);
  d["temperature"] = numpy_copy(hp.T);
  d["phase"] = numpy_copy(hp.phase);
  d["flags"] = numpy_copy(hp.flags);
  d["id"] = numpy_copy(hp.id);
  return d;
}

// The reverse, for the host writers: a particles dict into HostParticles.
HostParticles host_particles_of(const py::dict& d) {
  const ParticleColumns c(d["position"], d["mass"], d["density"], d["temperature"], d["phase"],
                          d.contains("velocity") ? py::handle(d["velocity"]) : py::handle(py::none()),
                          d.contains("normal") ? py::handle(d["normal"]) : py::handle(py::none()),
                          d.contains("flags") ? py::handle(d["flags"]) : py::handle(py::none()));
  const auto n = static_cast<std::size_t>(c.n);
  const cryo_host_particles_t f = c.view();  // float columns
  HostParticles hp;
  auto vecs = [n](std::vector<Vec3>& dst, const float* a) {
    dst.assign(n, Vec3{0, 0, 0});
    if (a && n) std::memcpy(dst.data(), a, 12 * n);
  };
  vecs(hp.x, f.x);
  vecs(hp.v, f.v);
  vecs(hp.nrm, f.nrm);
  hp.m.assign(f.m, f.m + n);
  hp.rho.assign(f.rho, f.rho + n);
  hp.T.assign(f.T, f.T + n);
  hp.phase.assign(c.phase.data(), c.phase.data() + n);
  hp.flags = c.has_flags ? std::vector<std::uint8_t>(c.flags.data(), c.flags.data() + n) : std::vector<std::uint8_t>(n, 0);
  hp.id.resize(n);
  for (std::size_t i = 0; i < n; ++i) hp.id[i] = static_cast<std::uint32_t>(i);
  if (d.contains("id")) {
    const U32 id = column<U32>(d["id"], c.n, 1, "id");
    std::memcpy(hp.id.data(), id.data(), 4 * n);
  }
  return hp;
}

py::dict frame_dict(const TelemetryFrame& f) {
  py::dict d;
  d["time"] = f.time;
  d["step"] = f.step;
  d["position"] = numpy_copy(f.position.data(), {static_cast<py::ssize_t>(f.n), 3});
  d["temperature"] = numpy_copy(f.temperature);
  d["pressure"] = numpy_copy(f.pressure);
  d["speed"] = numpy_copy(f.speed);
  d["phase"] = numpy_copy(f.phase);
  return d;
}

// Rows of a (count, 3) array as Vec3 (manoeuvre tables).
std::vector<Vec3> vec_rows(const F64& a, std::size_t count, const char* what) {
  if (a.ndim() != 2 || a.shape(1) != 3 || static_cast<std::size_t>(a.shape(0)) != count)
    throw std::invalid_argument(std::string(what) + ": expected an array of shape (len(time), 3)");
  std::vector<Vec3> out;
  out.reserve(count);
  const double* p = a.data();
  for (std::size_t k = 0; k < count; ++k, p += 3) out.push_back(Vec3{static_cast<real>(p[0]), static_cast<real>(p[1]), static_cast<real>(p[2])});
  return out;
}

}  // namespace

PYBIND11_MODULE(CryoSPH, m) {
  m.doc() = "CryoSPH (B200): GPU multiphase SPH for cryogenic propellant management in microgravity";
  m.attr("__version__") = "0.2.0";
  m.attr("cuda_backend") = true;
  m.attr("double_precision") = false;
  m.def("device_name", []() { return device_name(0); }, "Name of the compute device used by the solver.");
  m.def("device_count", &device_count, "Number of CUDA devices.");

  py::enum_<Phase>(m, "Phase").value("Liquid", Phase::Liquid).value("Vapor", Phase::Vapor).value("Wall", Phase::Wall);
  py::enum_<KernelType>(m, "KernelType")
      .value("CubicSpline", KernelType::CubicSpline)
      .value("WendlandC2", KernelType::WendlandC2);
  py::enum_<DensityMode>(m, "DensityMode")
      .value("Summation", DensityMode::Summation)
      .value("Continuity", DensityMode::Continuity);
  py::enum_<SurfaceTensionModel>(m, "SurfaceTensionModel")
      .value("NoTension", SurfaceTensionModel::None)
      .value("CSF", SurfaceTensionModel::CSF)
      .value("Akinci", SurfaceTensionModel::Akinci);
  py::enum_<WallThermalBC>(m, "WallThermalBC")
      .value("Adiabatic", WallThermalBC::Adiabatic)
      .value("Isothermal", WallThermalBC::Isothermal);
  py::enum_<TankThermoMode>(m, "TankThermoMode")
      .value("Vented", TankThermoMode::Vented)
      .value("Closed", TankThermoMode::Closed);
  py::enum_<FillMode>(m, "FillMode")
      .value("Settled", FillMode::Settled)
      .value("CentralBubble", FillMode::CentralBubble)
      .value("Full", FillMode::Full);
  py::enum_<WettingModel>(m, "WettingModel")
      .value("NormalRotation", WettingModel::NormalRotation)
      .value("ContactLineForce", WettingModel::ContactLineForce)
      .value("Both", WettingModel::Both);
  py::enum_<FieldArithmetic>(m, "FieldArithmetic")
      .value("Exact", FieldArithmetic::Exact)
      .value("Fast", FieldArithmetic::Fast);
  py::enum_<TelemetryMode>(m, "TelemetryMode")
      .value("AsyncCopy", TelemetryMode::AsyncCopy)
      .value("ZeroCopy", TelemetryMode::ZeroCopy);

  py::class_<FluidProperties>(m, "FluidProperties", "Saturated liquid/vapour property set (SI units).")
      .def(py::init<>())
      .def_readwrite("name", &FluidProperties::name)
      .def_readwrite("rho_liquid", &FluidProperties::rho_liquid)
      .def_readwrite("rho_vapor", &FluidProperties::rho_vapor)
      .def_readwrite("mu_liquid", &FluidProperties::mu_liquid)
      .def_readwrite("mu_vapor", &FluidProperties::mu_vapor)
      .def_readwrite("k_liquid", &FluidProperties::k_liquid)
      .def_readwrite("k_vapor", &FluidProperties::k_vapor)
      .def_readwrite("cp_liquid", &FluidProperties::cp_liquid)
      .def_readwrite("cp_vapor", &FluidProperties::cp_vapor)
      .def_readwrite("sigma", &FluidProperties::sigma)
      .def_readwrite("h_fg", &FluidProperties::h_fg)
      .def_readwrite("T_sat", &FluidProperties::T_sat)
      .def_readwrite("p_sat", &FluidProperties::p_sat)
      .def_readwrite("R_gas", &FluidProperties::R_gas)
      .def("saturation_temperature", &FluidProperties::saturation_temperature, py::arg("p"))
      .def("saturation_pressure", &FluidProperties::saturation_pressure, py::arg("T"))
      .def_static("liquid_hydrogen", &FluidProperties::liquid_hydrogen)
      .def_static("liquid_nitrogen", &FluidProperties::liquid_nitrogen)
      .def_static("liquid_oxygen", &FluidProperties::liquid_oxygen)
      .def_static("liquid_methane", &FluidProperties::liquid_methane)
      .def_static("water", &FluidProperties::water)
      .def("__repr__", [](const FluidProperties& f) {
        return "<FluidProperties " + f.name + " rho_l=" + std::to_string(f.rho_liquid) +
               " rho_v=" + std::to_string(f.rho_vapor) + " T_sat=" + std::to_string(f.T_sat) + ">";
      });

  py::class_<Geometry, std::shared_ptr<Geometry>>(m, "Geometry", "Tank geometry given by a signed distance function.")
      .def("sdf", &Geometry::sdf, py::arg("x"), py::arg("y"), py::arg("z"))
      .def("volume", &Geometry::volume)
      .def_property_readonly("name", &Geometry::name)
      .def_property_readonly("bounds", [](const Geometry& g) {
        const AABB b = g.bounds();
        return std::make_pair(triple(b.lo), triple(b.hi));
      });
  py::class_<CylinderTank, Geometry, std::shared_ptr<CylinderTank>>(m, "CylinderTank")
      .def(py::init<double, double>(), py::arg("radius"), py::arg("height"));
  py::class_<CapsuleTank, Geometry, std::shared_ptr<CapsuleTank>>(m, "CapsuleTank")
      .def(py::init<double, double>(), py::arg("radius"), py::arg("length"));
  py::class_<SphereTank, Geometry, std::shared_ptr<SphereTank>>(m, "SphereTank")
      .def(py::init<double>(), py::arg("radius"));
  py::class_<BoxTank, Geometry, std::shared_ptr<BoxTank>>(m, "BoxTank")
      .def(py::init<double, double, double>(), py::arg("lx"), py::arg("ly"), py::arg("lz"));
  py::class_<Translated, Geometry, std::shared_ptr<Translated>>(m, "Translated", "Geometry shifted by a constant offset.")
      .def(py::init([](std::shared_ptr<Geometry> g, const Triple& o) { return std::make_shared<Translated>(g, vec(o)); }),
           py::arg("geometry"), py::arg("offset"));
  py::class_<Difference, Geometry, std::shared_ptr<Difference>>(
      m, "Difference", "Fluid domain of `a` minus the solid `b` (obstacles, baffles, PMD vanes).")
      .def(py::init<std::shared_ptr<const Geometry>, std::shared_ptr<const Geometry>>(), py::arg("a"), py::arg("b"));
  py::class_<Union, Geometry, std::shared_ptr<Union>>(m, "Union", "Fluid domain of `a` united with `b`.")
      .def(py::init<std::shared_ptr<const Geometry>, std::shared_ptr<const Geometry>>(), py::arg("a"), py::arg("b"));
  py::class_<MeshTank, Geometry, std::shared_ptr<MeshTank>>(m, "MeshTank")
      .def(py::init([](const std::string& path, double scale, const Triple& offset) {
             return std::make_shared<MeshTank>(path, scale, vec(offset));
           }),
           py::arg("obj_path"), py::arg("scale") = 1.0, py::arg("offset") = Triple{0, 0, 0})
      .def_property_readonly("num_triangles", &MeshTank::num_triangles)
      .def("winding_number", &MeshTank::winding_number, py::arg("x"), py::arg("y"), py::arg("z"));

  py::class_<FillSpec>(m, "FillSpec", "How the generator fills a tank with liquid and vapour.")
      .def(py::init<>())
      .def_readwrite("mode", &FillSpec::mode)
      .def_readwrite("fill_fraction", &FillSpec::fill_fraction)
      .def_property(
          "settle_direction", [](const FillSpec& f) { return triple(f.settle_direction); },
          [](FillSpec& f, const Triple& t) { f.settle_direction = vec(t); })
      .def_property(
          "bubble_center", [](const FillSpec& f) { return triple(f.bubble_center); },
          [](FillSpec& f, const Triple& t) { f.bubble_center = vec(t); })
      .def_readwrite("include_vapor", &FillSpec::include_vapor)
      .def_readwrite("wall_layers", &FillSpec::wall_layers)
      .def_readwrite("T_liquid", &FillSpec::T_liquid)
      .def_readwrite("T_vapor", &FillSpec::T_vapor)
      .def_readwrite("T_wall", &FillSpec::T_wall)
      .def_readwrite("heater_zmin", &FillSpec::heater_zmin)
      .def_readwrite("heater_zmax", &FillSpec::heater_zmax);

  // Host-side generator access (no device needed): the particles build_tank
  // would load, and the domain it would pad (sph_solver.cu:430-437).
  m.def(
      "tank_particles",
      [](const Geometry& g, const FluidProperties& f, real dx, const FillSpec& fill) {
        return host_dict(build_tank_particles(g, f, dx, fill));
      },
      py::arg("geometry"), py::arg("fluid"), py::arg("dx"), py::arg("fill") = FillSpec{},
      "Lattice particles of a filled tank (walls first, then fluid) as a dict of NumPy arrays.");
  m.def(
      "tank_domain",
      [](const Geometry& g, real dx, int wall_layers) {
        AABB dom = g.bounds();
        const real pad = (wall_layers + 1) * dx;
        return std::make_pair(triple(dom.lo - Vec3{pad, pad, pad}), triple(dom.hi + Vec3{pad, pad, pad}));
      },
      py::arg("geometry"), py::arg("dx"), py::arg("wall_layers") = 3);
  m.def(
      "make_block",
      [](const Triple& lo, const Triple& hi, real dx, Phase phase, real density, real temperature) {
        return host_dict(make_block(vec(lo), vec(hi), dx, phase, density, temperature));
      },
      py::arg("lo"), py::arg("hi"), py::arg("dx"), py::arg("phase"), py::arg("density"), py::arg("temperature"));

  // The writers of io.hpp:13-22 for host particle dicts (no device needed;
  // Solver.write_vtk / write_json write the same files from the device).
  m.def(
      "write_vtk",
      [](const std::string& path, const py::dict& particles, py::object pressure) {
        const HostParticles hp = host_particles_of(particles);
        std::vector<real> p;
        if (!pressure.is_none()) {
          const F32 a = column<F32>(pressure, static_cast<py::ssize_t>(hp.size()), 1, "pressure");
          p.assign(a.data(), a.data() + a.size());
        }
        write_vtk(path, hp, p);
      },
      py::arg("path"), py::arg("particles"), py::arg("pressure") = py::none(),
      "Legacy binary VTK polydata of a particle dict (pressure scalars when given).");
  m.def(
      "make_frame",
      [](const py::dict& particles, py::object pressure, double time, long long step) {
        const HostParticles hp = host_particles_of(particles);
        std::vector<real> p;
        if (!pressure.is_none()) {
          const F32 a = column<F32>(pressure, static_cast<py::ssize_t>(hp.size()), 1, "pressure");
          p.assign(a.data(), a.data() + a.size());
        }
        return frame_dict(make_frame(hp, p, time, step));
      },
      py::arg("particles"), py::arg("pressure") = py::none(), py::arg("time") = 0.0, py::arg("step") = 0,
      "The viewer frame of a particle dict (as fetch_telemetry returns it).");
  m.def(
      "write_json_frame",
      [](const std::string& path, const py::dict& frame, bool include_walls) {
        TelemetryFrame f;
        f.time = frame["time"].cast<double>();
        f.step = frame["step"].cast<long long>();
        const F32 pos = py::cast<F32>(frame["position"]);
        f.n = static_cast<int>(pos.size() / 3);
        const py::ssize_t n = f.n;
        f.position.assign(pos.data(), pos.data() + 3 * n);
        auto col = [&](const char* k) {
          const F32 a = column<F32>(frame[k], n, 1, k);
          return std::vector<float>(a.data(), a.data() + n);
        };
        f.temperature = col("temperature");
        f.pressure = col("pressure");
        f.speed = col("speed");
        const U8 ph = column<U8>(frame["phase"], n, 1, "phase");
        f.phase.assign(ph.data(), ph.data() + n);
        write_json_frame(path, f, include_walls);
      },
      py::arg("path"), py::arg("frame"), py::arg("include_walls") = true,
      "The viewer's JSON frame file of a frame dict (walls left out unless include_walls).");

  py::class_<SolverConfig> cfg(m, "SolverConfig", "Solver parameters (the reference's SolverConfig).");
  cfg.def(py::init<>())
      .def_property(
          "gravity", [](const SolverConfig& c) { return triple(c.gravity); },
          [](SolverConfig& c, const Triple& t) { c.gravity = vec(t); });
#define CRYO_RW(field) cfg.def_readwrite(#field, &SolverConfig::field)
  CRYO_RW(dx); CRYO_RW(h_factor); CRYO_RW(kernel); CRYO_RW(density_mode); CRYO_RW(normalize_initial_masses);
  CRYO_RW(velocity_scale); CRYO_RW(sound_speed); CRYO_RW(tait_gamma); CRYO_RW(background_pressure);
  CRYO_RW(vapor_stiffness); CRYO_RW(clamp_negative_pressure); CRYO_RW(transport_velocity);
  CRYO_RW(transport_background_factor); CRYO_RW(transport_stress); CRYO_RW(transport_interface_only);
  CRYO_RW(particle_shifting); CRYO_RW(shifting_strength); CRYO_RW(artificial_viscosity);
  CRYO_RW(artificial_viscosity_vapor); CRYO_RW(delta_sph); CRYO_RW(no_slip); CRYO_RW(sps_turbulence);
  CRYO_RW(smagorinsky_cs); CRYO_RW(surface_tension); CRYO_RW(contact_angle_deg); CRYO_RW(contact_angle_wall_weight);
  CRYO_RW(wall_colour); CRYO_RW(wetting_model); CRYO_RW(csf_smooth_normals); CRYO_RW(csf_balanced);
  CRYO_RW(akinci_gamma); CRYO_RW(akinci_beta); CRYO_RW(thermal); CRYO_RW(phase_change); CRYO_RW(wall_thermal_bc);
  CRYO_RW(heater_power); CRYO_RW(conductivity_scale); CRYO_RW(lee_evaporation); CRYO_RW(lee_condensation);
  CRYO_RW(thermo_mode); CRYO_RW(vent_relaxation); CRYO_RW(merge_ratio); CRYO_RW(split_ratio);
  CRYO_RW(max_transfer_fraction); CRYO_RW(phase_change_density_limit); CRYO_RW(vapor_mass_rebalance);
  CRYO_RW(cfl); CRYO_RW(viscous_number); CRYO_RW(force_number); CRYO_RW(capillary_number); CRYO_RW(thermal_number);
  CRYO_RW(dt_max); CRYO_RW(dt_min); CRYO_RW(fixed_dt);
#undef CRYO_RW

  py::class_<Diagnostics> diag(m, "Diagnostics", "Global state summary returned by Solver.diagnostics().");
#define CRYO_RO(field) diag.def_readonly(#field, &Diagnostics::field)
  CRYO_RO(time); CRYO_RO(step); CRYO_RO(dt); CRYO_RO(n_total); CRYO_RO(n_liquid); CRYO_RO(n_vapor); CRYO_RO(n_wall);
  CRYO_RO(mass_liquid); CRYO_RO(mass_vapor); CRYO_RO(mass_total); CRYO_RO(kinetic_energy); CRYO_RO(enthalpy);
  CRYO_RO(heat_input); CRYO_RO(evaporated_mass); CRYO_RO(condensed_mass); CRYO_RO(vented_mass);
  CRYO_RO(vented_enthalpy); CRYO_RO(T_sat); CRYO_RO(p_ullage); CRYO_RO(max_speed); CRYO_RO(T_liquid_mean);
  CRYO_RO(T_liquid_max); CRYO_RO(T_vapor_mean); CRYO_RO(splits); CRYO_RO(merges);
#undef CRYO_RO
  diag.def_property_readonly("liquid_com", [](const Diagnostics& d) { return triple(d.liquid_com); })
      .def_property_readonly("slosh_force", [](const Diagnostics& d) { return triple(d.slosh_force); })
      .def_property_readonly("slosh_moment", [](const Diagnostics& d) { return triple(d.slosh_moment); })
      .def_property_readonly("frame_acceleration", [](const Diagnostics& d) { return triple(d.frame_acceleration); })
      .def_property_readonly("frame_angular_velocity",
                             [](const Diagnostics& d) { return triple(d.frame_angular_velocity); })
      .def_property_readonly("liquid_momentum", [](const Diagnostics& d) { return triple(d.liquid_momentum); })
      .def("as_dict", [](const Diagnostics& d) {
        py::dict r;
        py::object self = py::cast(d);
        for (const char* k :
             {"time", "step", "dt", "n_total", "n_liquid", "n_vapor", "n_wall", "mass_liquid", "mass_vapor",
              "mass_total", "kinetic_energy", "enthalpy", "heat_input", "evaporated_mass", "condensed_mass",
              "vented_mass", "vented_enthalpy", "T_sat", "p_ullage", "max_speed", "T_liquid_mean", "T_liquid_max",
              "T_vapor_mean", "splits", "merges", "liquid_com", "liquid_momentum", "slosh_force", "slosh_moment",
              "frame_acceleration", "frame_angular_velocity"})
          r[k] = self.attr(k);
        return r;
      });

  py::class_<ManeuverProfile>(m, "ManeuverProfile",
                              "Prescribed tank motion (tank frame): piecewise-linear acceleration and angular velocity.")
      .def(py::init([](std::vector<double> time, F64 acc, py::object omega, const Triple& origin) {
             ManeuverProfile p;
             p.time = std::move(time);
             p.acceleration = vec_rows(acc, p.time.size(), "acceleration");
             if (!omega.is_none()) p.angular_velocity = vec_rows(omega.cast<F64>(), p.time.size(), "angular_velocity");
             p.origin = vec(origin);
             p.validate();
             return p;
           }),
           py::arg("time"), py::arg("acceleration"), py::arg("angular_velocity") = py::none(),
           py::arg("origin") = Triple{0, 0, 0})
      .def(
          "evaluate",
          [](const ManeuverProfile& p, double t) {
            Vec3 a, w, wd;
            p.evaluate(t, a, w, wd);
            return py::make_tuple(triple(a), triple(w), triple(wd));
          },
          py::arg("t"), "Returns (acceleration, angular_velocity, angular_acceleration) at time t.");

  py::class_<Solver>(m, "Solver", "Weakly-compressible multiphase SPH solver (B200).")
      .def(py::init<const SolverConfig&, const FluidProperties&, int>(), py::arg("config"), py::arg("fluid"),
           py::arg("device") = 0)
      .def(
          "build_tank", [](Solver& s, const Geometry& g, const FillSpec& f, bool on_device) { s.build_tank(g, f, on_device); },
          py::arg("geometry"), py::arg("fill") = FillSpec{}, py::arg("on_device") = true,
          "Generates wall/liquid/vapour particles for a tank (on the GPU for analytic and CSG tanks).")
      .def(
          "set_particles",
          [](Solver& s, py::object position, py::object mass, py::object density, py::object temperature,
             py::object phase, const Triple& domain_lo, const Triple& domain_hi, py::object velocity,
             py::object normal, py::object flags) {
            const ParticleColumns cols(position, mass, density, temperature, phase, velocity, normal, flags);
            const cryo_host_columns_t view = cols.columns();
            py::gil_scoped_release nogil;
            s.set_particles(view, AABB{vec(domain_lo), vec(domain_hi)});
          },
          py::arg("position"), py::arg("mass"), py::arg("density"), py::arg("temperature"), py::arg("phase"),
          py::arg("domain_lo"), py::arg("domain_hi"), py::arg("velocity") = py::none(), py::arg("normal") = py::none(),
          py::arg("flags") = py::none(), "Loads a custom particle set (arrays of length N; position (N,3)).")
      .def("step", &Solver::step, py::call_guard<py::gil_scoped_release>())
      .def("run_steps", &Solver::run_steps, py::arg("n"), py::call_guard<py::gil_scoped_release>())
      .def("run_until", &Solver::run_until, py::arg("t_end"), py::call_guard<py::gil_scoped_release>())
      .def("relax", &Solver::relax, py::arg("duration"), py::arg("damping") = real(0.98),
           py::call_guard<py::gil_scoped_release>())
      .def("next_dt", &Solver::next_dt)
      .def("diagnostics", &Solver::diagnostics)
      .def("request_diagnostics", &Solver::request_diagnostics,
           "Enqueues the diagnostics of the current state without waiting (fetch them with fetch_diagnostics).")
      .def(
          "fetch_diagnostics",
          [](Solver& s, bool wait) -> py::object {
            Diagnostics d;
            bool got;
            {
              py::gil_scoped_release nogil;
              got = s.fetch_diagnostics(d, wait);
            }
            return got ? py::cast(d) : py::none();
          },
          py::arg("wait") = true,
          "The oldest requested diagnostics, in request order; None while not ready (wait=False) or when none is "
          "pending.")
      .def(
          "particles", [](const Solver& s) { return state_dict(s); },
          "Copies the particle state into a dict of NumPy arrays.")
      .def("pressure", [](const Solver& s) { return numpy_copy(s.pressure()); })
      .def("curvature", [](const Solver& s) { return numpy_copy(s.curvature()); })
      .def_property_readonly("time", &Solver::time)
      .def_property_readonly("step_count", &Solver::step_count)
      .def_property_readonly("last_dt", &Solver::last_dt)
      .def_property_readonly("num_particles", &Solver::num_particles)
      .def_property_readonly("device", &Solver::device)
      .def_property_readonly("config", &Solver::config)
      .def_property_readonly("fluid", &Solver::fluid)
      .def_property_readonly("sound_speed", &Solver::sound_speed)
      .def_property_readonly("smoothing_length", &Solver::smoothing_length)
      .def("set_gravity", [](Solver& s, const Triple& g) { s.set_gravity(vec(g)); }, py::arg("g"))
      .def("set_heater_power", &Solver::set_heater_power, py::arg("watts"))
      .def(
          "set_frame_motion",
          [](Solver& s, const Triple& acc, const Triple& w, const Triple& wdot, const Triple& origin) {
            s.set_frame_motion(vec(acc), vec(w), vec(wdot), vec(origin));
          },
          py::arg("acceleration") = Triple{0, 0, 0}, py::arg("angular_velocity") = Triple{0, 0, 0},
          py::arg("angular_acceleration") = Triple{0, 0, 0}, py::arg("origin") = Triple{0, 0, 0},
          "Constant tank-frame motion: linear acceleration of the tank, angular velocity and acceleration.")
      .def("set_maneuver", &Solver::set_maneuver, py::arg("profile"))
      .def("clear_frame_motion", &Solver::clear_frame_motion)
      .def("set_contact_angle", &Solver::set_contact_angle, py::arg("degrees"))
      .def("set_surface_tension", &Solver::set_surface_tension, py::arg("sigma"),
           "Surface tension coefficient (FluidProperties.sigma) for the following steps.")
      .def("set_lee_coefficients", &Solver::set_lee_coefficients, py::arg("evaporation"), py::arg("condensation"))
      .def(
          "adjoint_forward",
          [](Solver& s, long long steps, int checkpoint_every) {
            std::array<double, 7> o;
            {
              py::gil_scoped_release nogil;
              o = s.adjoint_forward(steps, checkpoint_every);
            }
            py::array_t<double> out(7);
            std::memcpy(out.mutable_data(), o.data(), sizeof(o));
            return out;
          },
          py::arg("steps"), py::arg("checkpoint_every") = 20,
          "Runs `steps` steps keeping checkpoints; returns [time-integrated slosh force (3), time-integrated "
          "slosh moment (3), final ullage pressure].")
      .def(
          "adjoint_backward",
          [](Solver& s, const std::array<double, 7>& seed) {
            Solver::AdjointGradients g;
            {
              py::gil_scoped_release nogil;
              g = s.adjoint_backward(seed);
            }
            const py::ssize_t steps = static_cast<py::ssize_t>(g.frame_acceleration.size() / 3);
            py::array_t<double> fa({steps, py::ssize_t{3}});
            if (steps) std::memcpy(fa.mutable_data(), g.frame_acceleration.data(), g.frame_acceleration.size() * 8);
            py::dict d;
            d["sigma"] = g.sigma;
            d["contact_angle"] = g.contact_angle;
            d["lee_evaporation"] = g.lee_evaporation;
            d["lee_condensation"] = g.lee_condensation;
            d["heater_power"] = g.heater_power;
            d["frame_acceleration"] = fa;
            return d;
          },
          py::arg("seed"),
          "Gradients of seed . objectives of the last adjoint_forward window (hand-written reverse passes).")
      .def_property_readonly("adjoint_memory", &Solver::adjoint_memory)
      .def("adjoint_release", &Solver::adjoint_release)
      .def("damp_velocities", &Solver::damp_velocities, py::arg("factor"))
      .def(
          "configure_telemetry", [](Solver& s, TelemetryMode mode) { s.configure_telemetry(mode); }, py::arg("mode"),
          "Selects AsyncCopy (pinned DMA) or ZeroCopy (mapped host memory) telemetry.")
      .def_property_readonly("telemetry_mode", &Solver::telemetry_mode)
      .def(
          "probe_pressure",
          [](Solver& s, const F32& pts) {
            if (pts.ndim() != 2 || pts.shape(1) != 3) throw std::invalid_argument("points: expected an array of shape (N, 3)");
            const auto* p = reinterpret_cast<const Vec3*>(pts.data());
            return numpy_copy(s.probe_pressure(std::vector<Vec3>(p, p + pts.shape(0))));
          },
          py::arg("points"), "Virtual pressure sensors: Shepard-weighted liquid pressure at each point; NaN where dry.")
      .def("request_telemetry", &Solver::request_telemetry,
           "Enqueues a non-blocking capture of the current state; returns False if one is pending.")
      .def("telemetry_ready", &Solver::telemetry_ready)
      .def(
          "fetch_telemetry",
          [](Solver& s) -> py::object {
            TelemetryFrame f;
            bool ok;
            {
              py::gil_scoped_release release;
              ok = s.fetch_telemetry(f);
            }
            if (!ok) return py::none();
            return frame_dict(f);
          },
          "Waits for the pending capture and returns it as a dict (None if nothing was requested).")
      .def("write_vtk", &Solver::write_vtk, py::arg("path"),
           "Legacy binary VTK polydata of the state (payload packed on the device).")
      .def("write_json", &Solver::write_json, py::arg("path"), py::arg("include_walls") = false,
           "Viewer frame as JSON (walls dropped on the device unless include_walls).")
      // B200 extensions
      .def_property_readonly("stream_handle", &Solver::stream_handle, "The solver's CUDA stream (cudaStream_t).")
      .def_property_readonly(
          "handle", [](const Solver& s) { return reinterpret_cast<std::uintptr_t>(s.handle()); },
          "The cryo_ctx* behind this solver, for direct C-ABI calls (include/cryosph_b200.h).")
      .def_property("field_arithmetic", &Solver::field_arithmetic, &Solver::set_field_arithmetic,
                    "Exact (default): the reference's IEEE operation sequence in the neighbour passes, bit-identical "
                    "to its CPU build; Fast: FMA contraction and approximate division / square root, within 1e-5.")
      .def("jitter_fluid", &Solver::jitter_fluid, py::arg("amplitude"), py::arg("seed"),
           "Moves every liquid and vapour particle by a seeded uniform offset in [-amplitude, amplitude) per axis, "
           "on the device, before the first step (cryo_cabi.jitter_offsets restates it on the host).")
      .def("set_graph_mode", &Solver::set_graph_mode, py::arg("enabled"),
           "Replay each step as a captured CUDA graph (default) or launch kernels one by one.")
      .def(
          "save_state", [](const Solver& s) { auto b = s.save_state(); return py::bytes(reinterpret_cast<const char*>(b.data()), b.size()); },
          "Full device state (persistent + scratch arrays, clock, counters) as bytes.")
      .def(
          "load_state",
          [](Solver& s, py::bytes blob) {
            const std::string str = blob;
            s.load_state(std::vector<std::uint8_t>(str.begin(), str.end()));
          },
          py::arg("state"))
      .def(
          "field",
          [](const Solver& s, int f) {
            auto v = s.field(f);
            return numpy_copy(v);
          },
          py::arg("field"), "Raw per-particle field (cryosph_b200.h CRYO_F_*).");

  // Batched stepping (B200 extension): members stay ordinary Solvers.
  py::class_<Ensemble>(m, "Ensemble",
                       "Independent tanks advanced together: one graph launch per ensemble step, each member's "
                       "results identical to stepping it alone.")
      .def(py::init<int>(), py::arg("device") = 0)
      .def(
          "add", [](Ensemble& e, Solver& s) { e.add(s); }, py::arg("solver"), py::keep_alive<1, 2>(),
          "Adds a Solver with particles loaded (kept alive by the ensemble).")
      .def("remove", &Ensemble::remove, py::arg("solver"))
      .def("__len__", &Ensemble::size)
      .def("run_steps", &Ensemble::run_steps, py::arg("n"), py::call_guard<py::gil_scoped_release>(),
           "Advances every member by n of its own steps.")
      .def_property("chains", &Ensemble::chains, &Ensemble::set_chains,
                    "Concurrent branches the members are spread over (0 = one per member).")
      .def_property("steps_per_launch", &Ensemble::steps_per_launch, &Ensemble::set_steps_per_launch,
                    "Ensemble steps per graph launch (1, 2, 4, 8 or 16).")
      .def(
          "tune",
          [](Ensemble& e, std::vector<int> chains, std::vector<int> steps_per_launch, int steps,
             std::vector<int> tiles) {
            py::gil_scoped_release nogil;
            return e.tune(chains, steps_per_launch, steps, tiles);
          },
          py::arg("chains") = std::vector<int>{}, py::arg("steps_per_launch") = std::vector<int>{},
          py::arg("steps") = 3, py::arg("tiles") = std::vector<int>{},
          "Autotunes branch count, steps per launch and the members' tile (particles per thread) by timing "
          "`steps` steps per candidate (these steps advance the members); returns (branches, steps per launch, "
          "ms per step).")
      .def_property("tile", &Ensemble::tile, &Ensemble::set_tile,
                    "Particles per thread of the members' grid-stride kernels inside the ensemble (results do not "
                    "depend on it).")
      .def("step_time", &Ensemble::step_time, py::arg("steps"), py::call_guard<py::gil_scoped_release>(),
           "Device ms per ensemble step over `steps` steps (which advance the members).")
      .def_property_readonly("launches_per_step", &Ensemble::launches_per_step)
      .def_property_readonly("stream_handle", &Ensemble::stream_handle)
      .def("diagnostics", &Ensemble::diagnostics, "Diagnostics of every member, in insertion order.");

  // One tank over several slabs (B200 extension).
  py::class_<SlabSolver>(m, "SlabSolver",
                         "One tank cut along z into slabs of cell layers, each slab a context on its own device "
                         "(or several on one); the particles equal a Solver's over the same steps.")
      .def(py::init<const SolverConfig&, const FluidProperties&, int, const std::vector<int>&>(), py::arg("config"),
           py::arg("fluid"), py::arg("slabs") = 2, py::arg("devices") = std::vector<int>{})
      .def("build_tank", &SlabSolver::build_tank, py::arg("geometry"), py::arg("fill") = FillSpec{},
           "Generates the tank's particles (host generator) and cuts them into the slabs.")
      .def(
          "set_particles",
          [](SlabSolver& s, py::object position, py::object mass, py::object density, py::object temperature,
             py::object phase, const Triple& domain_lo, const Triple& domain_hi, py::object velocity,
             py::object normal, py::object flags) {
            const ParticleColumns cols(position, mass, density, temperature, phase, velocity, normal, flags);
            const cryo_host_particles_t view = cols.view();
            py::gil_scoped_release nogil;
            s.set_particles(view, AABB{vec(domain_lo), vec(domain_hi)});
          },
          py::arg("position"), py::arg("mass"), py::arg("density"), py::arg("temperature"), py::arg("phase"),
          py::arg("domain_lo"), py::arg("domain_hi"), py::arg("velocity") = py::none(), py::arg("normal") = py::none(),
          py::arg("flags") = py::none(), "Loads the whole tank's particles (as Solver.set_particles).")
      .def("step", &SlabSolver::step, py::call_guard<py::gil_scoped_release>())
      .def("run_steps", &SlabSolver::run_steps, py::arg("n"), py::call_guard<py::gil_scoped_release>())
      .def("diagnostics", &SlabSolver::diagnostics)
      .def(
          "particles", [](const SlabSolver& s) { return state_dict(s); },
          "The whole tank's particles, in the order a Solver's arrays have.")
      .def_property_readonly("num_particles", &SlabSolver::num_particles)
      .def_property_readonly("slabs", &SlabSolver::slabs)
      .def_property(
          "graph_mode", &SlabSolver::graph_mode, [](SlabSolver& s, bool on) { s.set_graph_mode(on); },
          "True (default): every step replays one captured CUDA graph of all slabs; False: host threads per slab. "
          "Reads 0 (off), 1 (graph) or 2 (on, but the capture was refused and the steps run without it).")
      .def(
          "layout",
          [](const SlabSolver& s) {
            auto [zb, owned, held] = s.layout();
            py::dict d;
            d["z_begin"] = zb;
            d["owned"] = owned;
            d["held"] = held;
            return d;
          },
          "Cell-layer boundaries and the particles each slab owns and holds (owned + ghost copies).");
}
