// cryo_sdf.h -- signed distances of the analytic tank shapes (negative inside
// the fluid), shared by the host geometry classes (host/geometry.cpp) and the
// device lattice generator (cryo_setup.cu), so both classify every lattice
// node from the same double-precision arithmetic.
//
// The shapes are those of the reference's geometry.cpp (CylinderTank,
// CapsuleTank, SphereTank, BoxTank; the box by its full side lengths) and
// each formula keeps that file's operation order, with std::max, std::min
// and std::clamp restated here with their tie rules (max(a, b) returns a
// when they compare equal; min(a, b) likewise), so host and device results
// agree with the reference's to the last bit.  Compiles as C++ and CUDA.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define CRYO_HD __host__ __device__
#else
#define CRYO_HD
#endif

namespace cryo_sdf {

CRYO_HD inline double dmax(double a, double b) { return (a < b) ? b : a; }
CRYO_HD inline double dmin(double a, double b) { return (b < a) ? b : a; }
CRYO_HD inline double dclamp(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

// Finite cylinder about the z axis, radius R, height H, centred at the origin.
CRYO_HD inline double cylinder(double x, double y, double z, double R, double H) {
  const double radial = sqrt(x * x + y * y) - R;
  const double axial = fabs(z) - 0.5 * H;
  const double er = dmax(radial, 0.0), ea = dmax(axial, 0.0);
  return dmin(dmax(radial, axial), 0.0) + sqrt(er * er + ea * ea);
}

// Capsule: a cylinder of length L along z capped by hemispheres of radius R.
CRYO_HD inline double capsule(double x, double y, double z, double R, double L) {
  const double half = 0.5 * L;
  const double dz = z - dclamp(z, -half, half);
  return sqrt(x * x + y * y + dz * dz) - R;
}

CRYO_HD inline double sphere(double x, double y, double z, double R) { return sqrt(x * x + y * y + z * z) - R; }

// Axis-aligned box of side lengths lx, ly, lz centred at the origin.
CRYO_HD inline double box(double x, double y, double z, double lx, double ly, double lz) {
  const double bx = fabs(x) - 0.5 * lx, by = fabs(y) - 0.5 * ly, bz = fabs(z) - 0.5 * lz;
  const double ox = dmax(bx, 0.0), oy = dmax(by, 0.0), oz = dmax(bz, 0.0);
  return sqrt(ox * ox + oy * oy + oz * oz) + dmin(dmax(dmax(bx, by), bz), 0.0);
}

// CSG of two signed distances: the fluid of a without b, and of a or b.
CRYO_HD inline double subtract(double a, double b) { return dmax(a, -b); }
CRYO_HD inline double unite(double a, double b) { return dmin(a, b); }

}  // namespace cryo_sdf
