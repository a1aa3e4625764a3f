// geometry.cpp -- tank geometries on the host and the host lattice generator.
//
// Analytic shapes and their CSG evaluate the signed distances of
// csrc/cryo_sdf.h, the same functions the device generator (cryo_setup.cu)
// evaluates, and emit the node tree that generator takes.  The host
// generator below follows the device's formulation: classify every lattice
// node, compact wall and fluid nodes in lattice order, place the liquid cut
// at an order statistic of the fill key, emit walls then fluid.  It serves
// the geometries without a device form (triangle meshes, CSG over a mesh)
// and tank_particles(); both generators give the particles of the
// reference's build_tank_particles (geometry.cpp:242-330), bit for bit.
//
// Triangle meshes: distances from a point-triangle query written here (the
// plane projection when it falls inside the triangle, else the nearest of
// the three edges), the sign from the generalized winding number (solid
// angles by the formula of Van Oosterom and Strackee, IEEE Trans. Biomed.
// Eng. 30 (1983) 125-126), and a Wavefront OBJ reader.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <stdexcept>

#include "../csrc/cryo_sdf.h"
#include "cryosph.hpp"

namespace cryosph {

real norm(Vec3 a) { return std::sqrt(dot(a, a)); }
Vec3 normalized(Vec3 a, real eps) {
  const real n = norm(a);
  if (n > eps) return a / n;
  return Vec3{0, 0, 0};
}

Vec3 Geometry::outward_normal(double x, double y, double z, double eps) const {
  const double g[3] = {sdf(x + eps, y, z) - sdf(x - eps, y, z), sdf(x, y + eps, z) - sdf(x, y - eps, z),
                       sdf(x, y, z + eps) - sdf(x, y, z - eps)};
  const double len = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  if (len < 1e-300) return Vec3{0, 0, 0};
  return Vec3{static_cast<real>(g[0] / len), static_cast<real>(g[1] / len), static_cast<real>(g[2] / len)};
}

namespace {

constexpr double kPiD = 3.14159265358979323846;

Vec3 v3(double x, double y, double z) { return {static_cast<real>(x), static_cast<real>(y), static_cast<real>(z)}; }

// One node of the device generator's tree; returns its index.
int add_node(std::vector<cryo_geom_node_t>& out, int kind, int a, int b, double p0, double p1, double p2) {
  cryo_geom_node_t node{};
  node.kind = kind;
  node.a = a;
  node.b = b;
  node.p[0] = p0;
  node.p[1] = p1;
  node.p[2] = p2;
  out.push_back(node);
  return static_cast<int>(out.size()) - 1;
}

void require(bool ok, const char* what) {
  if (!ok) throw std::invalid_argument(what);
}

}  // namespace

// ------------------------------------------------------------ analytic shapes
CylinderTank::CylinderTank(double radius, double height) : R_(radius), H_(height) {
  require(radius > 0 && height > 0, "CylinderTank: radius and height must be > 0");
}
double CylinderTank::sdf(double x, double y, double z) const { return cryo_sdf::cylinder(x, y, z, R_, H_); }
AABB CylinderTank::bounds() const { return {v3(-R_, -R_, -0.5 * H_), v3(R_, R_, 0.5 * H_)}; }
double CylinderTank::volume() const { return kPiD * R_ * R_ * H_; }
int CylinderTank::emit_nodes(std::vector<cryo_geom_node_t>& out) const {
  return add_node(out, CRYO_GEOM_CYLINDER, -1, -1, R_, H_, 0.0);
}

CapsuleTank::CapsuleTank(double radius, double length) : R_(radius), L_(length) {
  require(radius > 0 && length >= 0, "CapsuleTank: radius must be > 0 and length >= 0");
}
double CapsuleTank::sdf(double x, double y, double z) const { return cryo_sdf::capsule(x, y, z, R_, L_); }
AABB CapsuleTank::bounds() const { return {v3(-R_, -R_, -(0.5 * L_ + R_)), v3(R_, R_, 0.5 * L_ + R_)}; }
double CapsuleTank::volume() const { return kPiD * R_ * R_ * L_ + 4.0 / 3.0 * kPiD * R_ * R_ * R_; }
int CapsuleTank::emit_nodes(std::vector<cryo_geom_node_t>& out) const {
  return add_node(out, CRYO_GEOM_CAPSULE, -1, -1, R_, L_, 0.0);
}

SphereTank::SphereTank(double radius) : R_(radius) { require(radius > 0, "SphereTank: radius must be > 0"); }
double SphereTank::sdf(double x, double y, double z) const { return cryo_sdf::sphere(x, y, z, R_); }
AABB SphereTank::bounds() const { return {v3(-R_, -R_, -R_), v3(R_, R_, R_)}; }
double SphereTank::volume() const { return 4.0 / 3.0 * kPiD * R_ * R_ * R_; }
int SphereTank::emit_nodes(std::vector<cryo_geom_node_t>& out) const {
  return add_node(out, CRYO_GEOM_SPHERE, -1, -1, R_, 0.0, 0.0);
}

// The box keeps its half sides; 2 * half is the side exactly.
BoxTank::BoxTank(double lx, double ly, double lz) : hx_(0.5 * lx), hy_(0.5 * ly), hz_(0.5 * lz) {
  require(lx > 0 && ly > 0 && lz > 0, "BoxTank: side lengths must be > 0");
}
double BoxTank::sdf(double x, double y, double z) const {
  return cryo_sdf::box(x, y, z, 2.0 * hx_, 2.0 * hy_, 2.0 * hz_);
}
AABB BoxTank::bounds() const { return {v3(-hx_, -hy_, -hz_), v3(hx_, hy_, hz_)}; }
double BoxTank::volume() const { return 8.0 * hx_ * hy_ * hz_; }
int BoxTank::emit_nodes(std::vector<cryo_geom_node_t>& out) const {
  return add_node(out, CRYO_GEOM_BOX, -1, -1, 2.0 * hx_, 2.0 * hy_, 2.0 * hz_);
}

// --------------------------------------------------------------------- CSG
Translated::Translated(std::shared_ptr<const Geometry> g, Vec3 offset)
    : g_(std::move(g)), ox_(offset.x), oy_(offset.y), oz_(offset.z) {
  require(g_ != nullptr, "Translated: null geometry");
}
double Translated::sdf(double x, double y, double z) const { return g_->sdf(x - ox_, y - oy_, z - oz_); }
AABB Translated::bounds() const {
  const AABB b = g_->bounds();
  const Vec3 shift = v3(ox_, oy_, oz_);
  return {b.lo + shift, b.hi + shift};
}
int Translated::emit_nodes(std::vector<cryo_geom_node_t>& out) const {
  const int child = g_->emit_nodes(out);
  if (child < 0) return -1;
  return add_node(out, CRYO_GEOM_TRANSLATED, child, -1, ox_, oy_, oz_);
}

Difference::Difference(std::shared_ptr<const Geometry> a, std::shared_ptr<const Geometry> b)
    : a_(std::move(a)), b_(std::move(b)) {
  require(a_ && b_, "Difference: null geometry");
}
double Difference::sdf(double x, double y, double z) const {
  return cryo_sdf::subtract(a_->sdf(x, y, z), b_->sdf(x, y, z));
}
int Difference::emit_nodes(std::vector<cryo_geom_node_t>& out) const {
  const int a = a_->emit_nodes(out);
  if (a < 0) return -1;
  const int b = b_->emit_nodes(out);
  if (b < 0) return -1;
  return add_node(out, CRYO_GEOM_DIFFERENCE, a, b, 0.0, 0.0, 0.0);
}

Union::Union(std::shared_ptr<const Geometry> a, std::shared_ptr<const Geometry> b) : a_(std::move(a)), b_(std::move(b)) {
  require(a_ && b_, "Union: null geometry");
}
double Union::sdf(double x, double y, double z) const { return cryo_sdf::unite(a_->sdf(x, y, z), b_->sdf(x, y, z)); }
AABB Union::bounds() const {
  const AABB p = a_->bounds(), q = b_->bounds();
  return {Vec3{std::min(p.lo.x, q.lo.x), std::min(p.lo.y, q.lo.y), std::min(p.lo.z, q.lo.z)},
          Vec3{std::max(p.hi.x, q.hi.x), std::max(p.hi.y, q.hi.y), std::max(p.hi.z, q.hi.z)}};
}
int Union::emit_nodes(std::vector<cryo_geom_node_t>& out) const {
  const int a = a_->emit_nodes(out);
  if (a < 0) return -1;
  const int b = b_->emit_nodes(out);
  if (b < 0) return -1;
  return add_node(out, CRYO_GEOM_UNION, a, b, 0.0, 0.0, 0.0);
}

// ----------------------------------------------------------- triangle meshes
namespace {

struct P3 {
  double x, y, z;
};
P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
double dotp(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
P3 crossp(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
P3 at(const std::array<double, 3>& v) { return {v[0], v[1], v[2]}; }

// Squared distance from p to the segment [a, b].
double segment_dist2(P3 p, P3 a, P3 b) {
  const P3 ab = sub(b, a), ap = sub(p, a);
  const double len2 = dotp(ab, ab);
  double t = len2 > 0 ? dotp(ap, ab) / len2 : 0.0;
  t = t < 0 ? 0.0 : (t > 1 ? 1.0 : t);
  const P3 d = {ap.x - ab.x * t, ap.y - ab.y * t, ap.z - ab.z * t};
  return dotp(d, d);
}

// Squared distance from p to the triangle abc: the plane distance when p
// projects inside the triangle (p on the inner side of all three edges),
// otherwise the nearest edge.
double triangle_dist2(P3 p, P3 a, P3 b, P3 c) {
  const P3 n = crossp(sub(b, a), sub(c, a));
  const double n2 = dotp(n, n);
  if (n2 > 0) {
    const bool inside = dotp(crossp(sub(b, a), sub(p, a)), n) >= 0 && dotp(crossp(sub(c, b), sub(p, b)), n) >= 0 &&
                        dotp(crossp(sub(a, c), sub(p, c)), n) >= 0;
    if (inside) {
      const double h = dotp(sub(p, a), n);
      return h * h / n2;
    }
  }
  return std::min(segment_dist2(p, a, b), std::min(segment_dist2(p, b, c), segment_dist2(p, c, a)));
}

const char* skip_blanks(const char* s) {
  while (*s == ' ' || *s == '\t' || *s == '\r') ++s;
  return s;
}

}  // namespace

// Wavefront OBJ: "v x y z" vertices and "f i j k ..." faces (1-based or
// negative relative indices, "i/t/n" forms; polygons fanned from the first
// corner).  Other records are ignored.
void load_obj(const std::string& path, std::vector<std::array<double, 3>>& vertices,
              std::vector<std::array<int, 3>>& triangles) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("load_obj: cannot read '" + path + "'");
  vertices.clear();
  triangles.clear();
  std::string line;
  long lineno = 0;
  auto fail = [&](const char* what) {
    throw std::runtime_error("load_obj: " + std::string(what) + " at line " + std::to_string(lineno) + " of '" +
                             path + "'");
  };
  std::vector<int> corners;
  while (std::getline(in, line)) {
    ++lineno;
    const char* s = skip_blanks(line.c_str());
    if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
      std::array<double, 3> v{};
      const char* q = s + 1;
      for (double& c : v) {
        char* end = nullptr;
        c = std::strtod(q, &end);
        if (end == q) fail("malformed vertex");
        q = end;
      }
      vertices.push_back(v);
    } else if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
      corners.clear();
      const char* q = skip_blanks(s + 1);
      while (*q) {
        char* end = nullptr;
        const long k = std::strtol(q, &end, 10);
        if (end == q) fail("malformed face");
        const long idx = k > 0 ? k - 1 : static_cast<long>(vertices.size()) + k;
        if (k == 0 || idx < 0 || idx >= static_cast<long>(vertices.size())) fail("face index out of range");
        corners.push_back(static_cast<int>(idx));
        q = end;
        while (*q && !std::isspace(static_cast<unsigned char>(*q))) ++q;  // "/t/n"
        q = skip_blanks(q);
      }
      for (std::size_t t = 2; t < corners.size(); ++t) triangles.push_back({corners[0], corners[t - 1], corners[t]});
    }
  }
  if (triangles.empty()) throw std::runtime_error("load_obj: '" + path + "' holds no faces");
}

MeshTank::MeshTank(const std::string& obj_path, double scale, Vec3 offset) {
  load_obj(obj_path, verts_, tris_);
  const double o[3] = {offset.x, offset.y, offset.z};
  for (auto& v : verts_)
    for (int k = 0; k < 3; ++k) v[k] = v[k] * scale + o[k];
  finalize();
}

MeshTank::MeshTank(std::vector<std::array<double, 3>> vertices, std::vector<std::array<int, 3>> triangles)
    : verts_(std::move(vertices)), tris_(std::move(triangles)) {
  const int nv = static_cast<int>(verts_.size());
  for (const auto& t : tris_)
    require(std::all_of(t.begin(), t.end(), [nv](int k) { return k >= 0 && k < nv; }),
            "MeshTank: triangle index out of range");
  finalize();
}

void MeshTank::finalize() {
  require(!verts_.empty() && !tris_.empty(), "MeshTank: the mesh has no triangles");
  std::array<double, 3> lo = verts_[0], hi = verts_[0];
  for (const auto& v : verts_)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], v[k]);
      hi[k] = std::max(hi[k], v[k]);
    }
  box_ = {v3(lo[0], lo[1], lo[2]), v3(hi[0], hi[1], hi[2])};
}

double MeshTank::winding_number(double x, double y, double z) const {
  const P3 p{x, y, z};
  double solid = 0;
  for (const auto& t : tris_) {
    const P3 a = sub(at(verts_[t[0]]), p), b = sub(at(verts_[t[1]]), p), c = sub(at(verts_[t[2]]), p);
    const double la = std::sqrt(dotp(a, a)), lb = std::sqrt(dotp(b, b)), lc = std::sqrt(dotp(c, c));
    const double triple = dotp(a, crossp(b, c));
    const double denom = la * lb * lc + dotp(a, b) * lc + dotp(b, c) * la + dotp(c, a) * lb;
    solid += 2.0 * std::atan2(triple, denom);
  }
  return solid / (4.0 * kPiD);
}

double MeshTank::sdf(double x, double y, double z) const {
  const P3 p{x, y, z};
  double best = HUGE_VAL;
  for (const auto& t : tris_) best = std::min(best, triangle_dist2(p, at(verts_[t[0]]), at(verts_[t[1]]), at(verts_[t[2]])));
  const double dist = std::sqrt(best);
  return std::fabs(winding_number(x, y, z)) > 0.5 ? -dist : dist;
}

AABB MeshTank::bounds() const { return box_; }

double MeshTank::volume() const {
  double six = 0;  // signed tetrahedra against the origin
  for (const auto& t : tris_) six += dotp(at(verts_[t[0]]), crossp(at(verts_[t[1]]), at(verts_[t[2]])));
  return std::fabs(six) / 6.0;
}

// --------------------------------------------------------- lattice generator
HostParticles build_tank_particles(const Geometry& geo, const FluidProperties& fluid, real dx, const FillSpec& fill) {
  require(dx > 0, "build_tank_particles: dx must be > 0");
  require(fill.wall_layers >= 1, "build_tank_particles: wall_layers must be >= 1");
  require(fill.fill_fraction >= 0 && fill.fill_fraction <= 1, "build_tank_particles: fill_fraction must be in [0, 1]");
  // Lattice nodes at ((i + 1/2) h, (j + 1/2) h, (k + 1/2) h) over the tank's
  // box padded by the wall band and one node.
  const double h = dx, band = fill.wall_layers * h;
  const AABB b = geo.bounds();
  const int lo[3] = {static_cast<int>(std::floor((b.lo.x - band) / h)) - 1,
                     static_cast<int>(std::floor((b.lo.y - band) / h)) - 1,
                     static_cast<int>(std::floor((b.lo.z - band) / h)) - 1};
  const int hi[3] = {static_cast<int>(std::ceil((b.hi.x + band) / h)) + 1,
                     static_cast<int>(std::ceil((b.hi.y + band) / h)) + 1,
                     static_cast<int>(std::ceil((b.hi.z + band) / h)) + 1};
  const long long nx = hi[0] - lo[0], ny = hi[1] - lo[1], nz = hi[2] - lo[2];
  const long long total = nx * ny * nz;
  if (total > 400'000'000LL) throw std::runtime_error("build_tank_particles: lattice too large, increase dx");
  auto coord = [&](long long t, double& x, double& y, double& z) {
    const long long i = t % nx, j = (t / nx) % ny, k = t / (nx * ny);
    x = (lo[0] + static_cast<int>(i) + 0.5) * h;
    y = (lo[1] + static_cast<int>(j) + 0.5) * h;
    z = (lo[2] + static_cast<int>(k) + 0.5) * h;
  };

  // 1. classify: 1 fluid (sdf < 0), 2 wall (0 <= sdf < band), 0 outside
  std::vector<std::uint8_t> cls(static_cast<std::size_t>(total));
#pragma omp parallel for schedule(dynamic, 4096)
  for (long long t = 0; t < total; ++t) {
    double x, y, z;
    coord(t, x, y, z);
    const double d = geo.sdf(x, y, z);
    cls[static_cast<std::size_t>(t)] = d < 0 ? 1 : (d < band ? 2 : 0);
  }
  // 2. ordered compaction of the wall and fluid nodes
  std::vector<long long> walls, fluid_nodes;
  for (long long t = 0; t < total; ++t) {
    const std::uint8_t c = cls[static_cast<std::size_t>(t)];
    if (c == 1) fluid_nodes.push_back(t);
    else if (c == 2) walls.push_back(t);
  }
  if (fluid_nodes.empty()) throw std::runtime_error("build_tank_particles: no fluid nodes inside the tank; is dx too large?");

  // 3. liquid cut: the n_liq-th largest fill key, less a hair (whole planes
  //    or shells of equal keys stay together)
  const std::size_t nf = fluid_nodes.size();
  auto node_point = [&](long long t) {
    double x, y, z;
    coord(t, x, y, z);
    return v3(x, y, z);
  };
  std::vector<std::uint8_t> liquid(nf, 1);
  if (fill.mode != FillMode::Full) {
    const Vec3 g = normalized(fill.settle_direction);
    std::vector<double> key(nf);
    for (std::size_t q = 0; q < nf; ++q) {
      const Vec3 p = node_point(fluid_nodes[q]);
      key[q] = fill.mode == FillMode::Settled ? static_cast<double>(dot(p, g))
                                              : static_cast<double>(norm(p - fill.bubble_center));
    }
    const auto n_liq = static_cast<std::size_t>(std::llround(fill.fill_fraction * static_cast<double>(nf)));
    if (n_liq == 0) {
      std::fill(liquid.begin(), liquid.end(), 0);
    } else {
      std::vector<double> sorted(key);
      std::nth_element(sorted.begin(), sorted.begin() + static_cast<std::ptrdiff_t>(n_liq - 1), sorted.end(),
                       std::greater<double>());
      const double cut = sorted[n_liq - 1] - 1e-6 * h;
      for (std::size_t q = 0; q < nf; ++q) liquid[q] = key[q] >= cut ? 1 : 0;
    }
  }

  // 4. emit: walls (normal = -grad sdf, heated inside the z band), then fluid
  const auto T_of = [&](real given) { return std::isnan(given) ? fluid.T_sat : given; };
  const real vol = dx * dx * dx;
  const real m_liq = fluid.rho_liquid * vol, m_vap = fluid.rho_vapor * vol;
  std::vector<Vec3> wall_normal(walls.size());
#pragma omp parallel for schedule(dynamic, 256)
  for (long long w = 0; w < static_cast<long long>(walls.size()); ++w) {
    double x, y, z;
    coord(walls[static_cast<std::size_t>(w)], x, y, z);
    wall_normal[static_cast<std::size_t>(w)] = -geo.outward_normal(x, y, z, 0.5 * h);
  }
  HostParticles out;
  out.reserve(walls.size() + nf);
  for (std::size_t w = 0; w < walls.size(); ++w) {
    double x, y, z;
    coord(walls[w], x, y, z);
    const bool heated = z >= fill.heater_zmin && z <= fill.heater_zmax;
    out.push(v3(x, y, z), {0, 0, 0}, m_liq, fluid.rho_liquid, T_of(fill.T_wall), Phase::Wall, wall_normal[w],
             heated ? pflag::Heated : std::uint8_t{0});
  }
  for (std::size_t q = 0; q < nf; ++q) {
    const Vec3 p = node_point(fluid_nodes[q]);
    if (liquid[q]) out.push(p, {0, 0, 0}, m_liq, fluid.rho_liquid, T_of(fill.T_liquid), Phase::Liquid);
    else if (fill.include_vapor) out.push(p, {0, 0, 0}, m_vap, fluid.rho_vapor, T_of(fill.T_vapor), Phase::Vapor);
  }
  return out;
}

// make_block (geometry.cpp:332-346 of the reference): whole lattice cells of
// the box [lo, hi), nodes at lo + (i + 1/2) dx, the reference's 1e-4 slack on
// the cell count.
HostParticles make_block(Vec3 lo, Vec3 hi, real dx, Phase phase, real density, real temperature) {
  auto cells = [dx](real a, real b) { return std::max(0, static_cast<int>(std::floor((b - a) / dx + real(1e-4)))); };
  const int n[3] = {cells(lo.x, hi.x), cells(lo.y, hi.y), cells(lo.z, hi.z)};
  const real mass = density * dx * dx * dx;
  HostParticles out;
  out.reserve(static_cast<std::size_t>(n[0]) * n[1] * n[2]);
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i)
        out.push(Vec3{lo.x + (i + real(0.5)) * dx, lo.y + (j + real(0.5)) * dx, lo.z + (k + real(0.5)) * dx}, {0, 0, 0},
                 mass, density, temperature, phase);
  return out;
}

// ------------------------------------------------------------ HostParticles
void HostParticles::reserve(std::size_t n) {
  x.reserve(n); v.reserve(n); nrm.reserve(n); m.reserve(n); rho.reserve(n); T.reserve(n);
  phase.reserve(n); flags.reserve(n); id.reserve(n);
}
void HostParticles::clear() { *this = HostParticles{}; }
std::size_t HostParticles::push(Vec3 pos, Vec3 vel, real mass, real density, real temperature, Phase ph, Vec3 normal,
                                std::uint8_t flag) {
  const std::size_t k = x.size();
  x.push_back(pos); v.push_back(vel); nrm.push_back(normal);
  m.push_back(mass); rho.push_back(density); T.push_back(temperature);
  phase.push_back(static_cast<std::uint8_t>(ph)); flags.push_back(flag);
  id.push_back(static_cast<std::uint32_t>(k));
  return k;
}
void HostParticles::append(const HostParticles& o) {
  const auto offset = static_cast<std::uint32_t>(size());
  auto cat = [](auto& dst, const auto& src) { dst.insert(dst.end(), src.begin(), src.end()); };
  cat(x, o.x); cat(v, o.v); cat(nrm, o.nrm); cat(m, o.m); cat(rho, o.rho); cat(T, o.T);
  cat(phase, o.phase); cat(flags, o.flags);
  for (std::uint32_t k : o.id) id.push_back(offset + k);
}

}  // namespace cryosph
