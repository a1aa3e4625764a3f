// cryo_adjoint.cuh -- reverse (adjoint) passes of one Solver::step
// (sph_solver.cu:511-533) with the neighbour topology of the step frozen.
//
// The reverse of a step reads the step as it was recomputed from the
// segment's checkpoint: the arrays the rate passes left (positions and
// phases, density, pressure and sigma, normals and colour fraction, wall
// fields, accelerations, heater weights, the neighbour lists), copied at the
// end of the step (AdjSlot), the values the later stages overwrite, copied
// as they were produced, and the sums of the force and interface passes.
//
// Every adjoint is held per particle in the step's sorted order.  A pair
// term f(i, j) that feeds particle i's output is differentiated twice: with
// respect to i's inputs in i's own thread, and with respect to j's inputs in
// j's thread, which visits i as its own neighbour (the lists are symmetric:
// r^2 of (i, j) and (j, i) are the same float).  No atomics; every adjoint
// is a deterministic gather.  Global adjoints (parameters, gravity, the
// saturation temperature) go through fixed-tree FP64 chunk partials.
#pragma once

#include "cryo_kernels.cuh"

namespace cryo {

// FP64 accumulators of the reverse sweep (Adj::glob).
enum AdjGlobal {
  AG_TSAT_IN = 0,   // adjoint of the T_sat this step's sources read (the previous step's output)
  AG_HINV = 1,      // adjoint of heat_inv_norm (this step)
  AG_GRAV = 2,      // 2..4: adjoint of the effective gravity (this step)
  AG_SIGMA = 5,     // surface tension coefficient (window total)
  AG_COS = 6,       // cos(contact angle)
  AG_SIN = 7,       // sin(contact angle)
  AG_LEE_E = 8,     // Lee evaporation coefficient
  AG_LEE_C = 9,     // Lee condensation coefficient
  AG_HEAT = 10,     // heater power
  AG_TSAT_OUT = 11, // upstream adjoint of this step's output T_sat
  AG_P_OBJ = 12,    // upstream adjoint of this step's output ullage pressure
  AG_FW = 13,       // 13..15: seed of the time-integrated slosh force (-sum dt fw)
  AG_MW = 16,       // 16..18: seed of the time-integrated slosh moment (-sum dt mw)
  AG_C_LIQ = 19,    // saturation: d(objective)/d(liquid mass of a particle)
  AG_C_MT = 20,     // saturation: d(objective)/d(m T of a vapour particle)
  AG_COUNT = 24
};
// Rows of the chunk partials: each kernel with global terms owns its rows.
enum AdjRow {
  AR_SRC = 0,    // 0..2: k_adj_kick_sources (tsat, lee_e, lee_c)
  AR_FORCE = 3,  // 3..8: k_adj_forces_local (hinv, g x3, sigma, heat)
  AR_IFACE = 9,  // 9..10: k_adj_interface_local (cos, sin)
  AR_WALL = 11,  // 11..13: k_adj_wall_gather (g x3)
  AR_SAT = 14,   // 14..16: k_adj_saturation_sums (m_liq, m_vap, mT_vap)
  AR_COUNT = 17
};

// The arrays of one recomputed step that the reverse sweep reads, as they
// stand at the end of the step (positions and phase flags, v and T, m0,
// normals and colour fraction, mass / density / pressure / sigma,
// accelerations, wall fields, heater weights), plus the step's permutation,
// neighbour lists (kNbrChunk-entry chunks with chunk stride n), cell table
// and scalar block.
struct AdjSlot {
  float4 *xp, *vT, *vt, *nrm, *mrps, *a4, *vwp;
  float* heat_w;
  uint32_t* perm;
  int* nbr_cnt;
  int* nbr;
  int* cell_begin;
  int *fluid_idx, *wall_idx;  // the step's ordered phase index lists
  DynState* dyn;
};

struct Adj {
  // forward values: the live sorted set of the recomputed step ...
  View V;
  // ... and the one-step tape
  const float4* vT1;  // (v, T) at the rate evaluation
  const float* m1;    // mass at the rate evaluation
  const float4* ns1;  // (unit normal, kappa) of the rate evaluation
  const float4* pc2;  // (out_m, out_h, w_norm) after the normalisation
  const float4* vT2;  // (v, T) after the phase-change apply
  const float* m2;    // mass after the phase-change apply
  const DynState* dyn1;  // scalar block at the rate evaluation
  const float4* sums;    // force-pass sums (rows 0-2) and interface sums (rows 3-5), sums_n records each
  int sums_n;
  // adjoints (sorted order of the step)
  float4* gX;  // (x, m)         carried between steps
  float4* gV;  // (v, T)         carried
  float4* gA;  // (a, dTdt)      a carried, dTdt per step
  float4* gB;  // (ab, rho)      ab carried, rho per step
  float4* gP;  // fluid (p, sigma, -, -); wall (p_wl, p_wv, alpha_w, -)
  float4* gN;  // fluid (ns, alpha); wall (vw, -)
  float4* gG;  // fluid (nrm, heat_w)
  float4* gC;  // sources (out_m, out_h, w_norm | w_sum, wr_max)
  float4* gU1; // per-particle upstream coefficients of the gather passes
  float4* gU2;
  float4* gU3;
  float4* R1;  // fluid particles' force-pass values: (V, 1/sigma, c, rho)
  float4* R2;  // ... (p, T, m, flags: do_T | do_C << 1 | valid unit normal << 2)
  int* argmax;     // sources: index of the receiver that set wr_max
  float4* prevX;   // scatter targets (the previous step's sorted order)
  float4* prevV;
  float4* prevA;
  float4* prevB;
  const uint32_t* perm;  // this step's reorder: sorted slot -> previous slot
  double* glob;
  double* partials;
  unsigned* ticket;
  int max_chunks;
  unsigned* status;  // ADJ_* bits
};

enum { ADJ_TOPOLOGY = 1u };  // a particle died or was born inside the window

__global__ void k_adj_saturation_sums(Params P, Adj A);
__global__ void k_adj_rebalance_local(Params P, Adj A);
__global__ void k_adj_rebalance_gather(Params P, Adj A);
__global__ void k_adj_apply_local(Params P, Adj A);
__global__ void k_adj_apply_gather(Params P, Adj A);
__global__ void k_adj_normalize_local(Params P, Adj A);
__global__ void k_adj_normalize_gather(Params P, Adj A);
__global__ void k_adj_kick_sources(Params P, Adj A);
__global__ void k_adj_forces_local(Params P, Adj A);
__global__ void k_adj_forces_gather(Params P, Adj A);
__global__ void k_adj_interface_local(Params P, Adj A);
__global__ void k_adj_interface_gather(Params P, Adj A);
__global__ void k_adj_wall_local(Params P, Adj A);
__global__ void k_adj_wall_gather(Params P, Adj A);
__global__ void k_adj_density_gather(Params P, Adj A);
__global__ void k_adj_drift_scatter(Params P, Adj A);
// glob[dst[b]] (+)= sum of partial row row[b], b < count; one block per row.
struct AdjRows {
  int count;
  int row[12], dst[12], accumulate[12];
};
__global__ void k_adj_reduce(Adj A, AdjRows M);
// Objective of the forward window: obj[0..2] += dt * (-sum fw), obj[3..5] +=
// dt * (-sum mw) over fluid particles (the slosh force and moment of
// sph_solver.cu:219-232 and :640-641, integrated in time).
__global__ void k_adj_objective(Params P, View V, Reduce R, double* obj);
// End-of-step copy of the arrays of AdjSlot (the lists are copied apart).
__global__ void k_adj_snap_end(View V, const uint32_t* perm, AdjSlot S);
// End of one reverse step: the step's gravity adjoint out, the T_sat adjoint
// carried to the previous step, the ullage-pressure seed consumed.
__global__ void k_adj_step_end(double* glob, double* grav_out);
// Tape snapshot of a float4 array (and optionally the mass component).
__global__ void k_adj_copy4(const float4* src, float4* dst, float* mdst, const float4* msrc, const DynState* dyn);

}  // namespace cryo
