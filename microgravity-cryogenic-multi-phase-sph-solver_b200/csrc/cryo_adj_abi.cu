// cryo_adj_abi.cu -- the differentiated window's driver (checkpoints,
// segment recomputation, the reverse sweep over cryo_adjoint.cu's passes)
// and its extern "C" entry points (cryo_adj_*).
#include "cryo_ctx.cuh"

// ---------------------------------------------------------------------------
// Differentiated window (no counterpart in the reference).  The forward run
// steps as usual (step graphs), keeps a state checkpoint every `every` steps
// and integrates the slosh force and moment.  The backward sweep takes the
// segments from the last: it restores the segment's checkpoint, re-runs the
// segment keeping every step's start state, then for each step from the last
// restores its start state, recomputes it eagerly with the one-step tape and
// runs the reverse passes (cryo_adjoint.cu).  At the end the window's final
// state is restored, so the solver continues as if only the forward had run.
namespace {

struct AdjSnap {
  char* base = nullptr;
  int cur = 0;
};

}  // namespace

struct AdjWindow {
  int n = 0, every = 20, cap = 0;
  long long steps = 0;
  bool recorded = false;
  int splits0 = 0, merges0 = 0;
  char* arena = nullptr;
  size_t bytes = 0, snap_bytes = 0;
  std::vector<AdjSnap> ckpt;  // start of every segment + the window's end
  // one per step of a segment: the step's tape and its end-of-step arrays
  struct Slot {
    StepTape tape;
    AdjSlot end;
  };
  std::vector<Slot> slots;
  size_t slot_bytes = 0;
  float4 *cX[2]{}, *cV[2]{}, *cA[2]{}, *cB[2]{};
  float4 *gP = nullptr, *gN = nullptr, *gG = nullptr, *gC = nullptr, *gU1 = nullptr, *gU2 = nullptr,
         *gU3 = nullptr, *R1 = nullptr, *R2 = nullptr;
  int* argmax = nullptr;
  double *glob = nullptr, *partials = nullptr, *obj = nullptr, *ggrav = nullptr;
  unsigned *ticket = nullptr, *status = nullptr;
  int max_chunks = 0;
  int q = 0;
  // final-state seeds (float4 per particle, final order): x|m, v|T, a, ab
  std::vector<float4> seed[4];
};

void adj_free(AdjWindow* w) {
  if (!w) return;
  if (w->arena) cudaFree(w->arena);
  delete w;
}

namespace {

constexpr int kSnap16 = 7;  // xp, vT, vt, nrm, mrps, a4, ab4

size_t r256(size_t b) { return (b + 255) & ~size_t(255); }

size_t snap_size(int n) { return kSnap16 * r256((size_t)n * 16) + r256((size_t)n * 4) + r256(sizeof(DynState)); }

void snap_save(cryo_ctx* c, AdjWindow& W, AdjSnap& S) {
  const size_t n = (size_t)W.n;
  const Persist& p = c->set[c->cur];
  const void* src[kSnap16] = {p.xp, p.vT, p.vt, p.nrm, p.mrps, c->a4, c->ab4};
  char* q = S.base;
  for (const void* a : src) {
    CK(cudaMemcpyAsync(q, a, n * 16, cudaMemcpyDeviceToDevice, c->stream));
    q += r256(n * 16);
  }
  CK(cudaMemcpyAsync(q, p.id, n * 4, cudaMemcpyDeviceToDevice, c->stream));
  q += r256(n * 4);
  CK(cudaMemcpyAsync(q, c->dyn, sizeof(DynState), cudaMemcpyDeviceToDevice, c->stream));
  S.cur = c->cur;
}

void snap_load(cryo_ctx* c, AdjWindow& W, const AdjSnap& S) {
  const size_t n = (size_t)W.n;
  c->cur = S.cur;
  const Persist& p = c->set[c->cur];
  void* dst[kSnap16] = {p.xp, p.vT, p.vt, p.nrm, p.mrps, c->a4, c->ab4};
  const char* q = S.base;
  for (void* a : dst) {
    CK(cudaMemcpyAsync(a, q, n * 16, cudaMemcpyDeviceToDevice, c->stream));
    q += r256(n * 16);
  }
  CK(cudaMemcpyAsync(p.id, q, n * 4, cudaMemcpyDeviceToDevice, c->stream));
  q += r256(n * 4);
  CK(cudaMemcpyAsync(c->dyn, q, sizeof(DynState), cudaMemcpyDeviceToDevice, c->stream));
}

// The configurations the reverse passes cover.
void adj_check_config(const cryo_ctx* c) {
  const cryo_config_t& g = c->cfg;
  const Params& P = c->P;
  auto no = [](const char* what) { throw std::invalid_argument(std::string("adjoint: not supported: ") + what); };
  if (c->fast_fields) no("the fast field arithmetic (the reverse passes differentiate the exact sequence)");
  if (!(P.fixed_dt > 0.0f)) no("adaptive time step (set fixed_dt)");
  if (!(g.sound_speed > 0 || g.velocity_scale > 0)) no("sound speed derived from the surface tension (set sound_speed)");
  if (P.density_mode != CRYO_DENSITY_SUMMATION) no("continuity density");
  if (P.sps) no("SPS turbulence");
  if (P.shift_strength > 0.0f) no("particle shifting");
  if (P.tvf_stress) no("transport-velocity stress");
  if (P.st_model == CRYO_ST_AKINCI) no("Akinci surface tension");
  if (P.csf_smooth || P.csf_balanced) no("smoothed or balanced CSF");
  if (P.wetting_model != 0) no("contact-line force wetting");
  if (P.wall_bc != CRYO_WALL_ADIABATIC) no("isothermal walls");
  if (P.clamp_neg) no("negative-pressure clamp");
  if (g.thermo_mode == CRYO_THERMO_VENTED && c->has_vapor && P.cfg_phase_change) no("vented tank");
}

// Device bytes of one segment slot: the tape and end-of-step arrays of one
// step, every per-particle array sized by the capacity.
size_t slot_size(int cap, int num_cells) {
  const size_t c16 = r256((size_t)cap * 16), c4 = r256((size_t)cap * 4);
  return 4 * c16 + 2 * c4 + r256(sizeof(DynState))  // mid-step tape
         + 6 * c16                                   // force / interface sums
         + 7 * c16 + c4                              // xp vT vt nrm mrps a4 vwp, heat_w
         + 4 * c4                                    // perm, list counts, phase index lists
         + r256((size_t)cap * 4 * kMaxNbr)           // lists
         + r256((size_t)(num_cells + 1) * 4) + r256(sizeof(DynState));
}

void adj_alloc(cryo_ctx* c, AdjWindow& W, long long steps, int every) {
  // snapshots hold the window's n particles; the tape and the adjoints are
  // sized by the capacity, which every kernel's particle count stays within
  const int n = W.cap;
  const long long nck = (steps + every - 1) / every + 1;
  const int nslot = (int)std::min<long long>(every, steps);
  W.snap_bytes = snap_size(W.n);
  W.slot_bytes = slot_size(n, c->P.num_cells);
  const size_t n16 = r256((size_t)n * 16), n4 = r256((size_t)n * 4);
  W.max_chunks = n / kChunk + 2;
  size_t t = (size_t)nck * W.snap_bytes + (size_t)nslot * W.slot_bytes;
  t += 8 * n16 + 9 * n16 + n4;                                // adjoints, force-pass records
  t += r256(AG_COUNT * 8) + r256((size_t)AR_COUNT * W.max_chunks * 8) + r256(8 * 8) + r256((size_t)steps * 3 * 8);
  t += r256(64) + r256(64);
  if (W.arena && W.bytes >= t) {
    // reuse
  } else {
    if (W.arena) CK(cudaFree(W.arena));
    W.arena = nullptr;
    W.bytes = 0;
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    if (t > free_b)
      throw std::invalid_argument("adjoint: the window needs " + std::to_string(t >> 20) + " MiB of device memory, " +
                                  std::to_string(free_b >> 20) +
                                  " MiB are free; use a smaller checkpoint interval (one segment of steps is held "
                                  "at a time) or a shorter window");
    CK(cudaMalloc(&W.arena, t));
    W.bytes = t;
  }
  char* p = W.arena;
  auto take = [&](size_t b) {
    char* r = p;
    p += r256(b);
    return r;
  };
  W.ckpt.assign((size_t)nck, AdjSnap{});
  for (auto& s : W.ckpt) s.base = take(W.snap_bytes);
  W.slots.assign((size_t)nslot, AdjWindow::Slot{});
  for (auto& sl : W.slots) {
    StepTape& tp = sl.tape;
    tp.vT1 = (float4*)take(n16);
    tp.ns1 = (float4*)take(n16);
    tp.pc2 = (float4*)take(n16);
    tp.vT2 = (float4*)take(n16);
    tp.m1 = (float*)take(n4);
    tp.m2 = (float*)take(n4);
    tp.dyn1 = (DynState*)take(sizeof(DynState));
    tp.sums = (float4*)take(6 * (size_t)n * 16);
    tp.n = n;
    AdjSlot& e = sl.end;
    e.xp = (float4*)take(n16);
    e.vT = (float4*)take(n16);
    e.vt = (float4*)take(n16);
    e.nrm = (float4*)take(n16);
    e.mrps = (float4*)take(n16);
    e.a4 = (float4*)take(n16);
    e.vwp = (float4*)take(n16);
    e.heat_w = (float*)take(n4);
    e.perm = (uint32_t*)take(n4);
    e.nbr_cnt = (int*)take(n4);
    e.fluid_idx = (int*)take(n4);
    e.wall_idx = (int*)take(n4);
    e.nbr = (int*)take((size_t)n * 4 * kMaxNbr);
    e.cell_begin = (int*)take((size_t)(c->P.num_cells + 1) * 4);
    e.dyn = (DynState*)take(sizeof(DynState));
  }
  for (int k = 0; k < 2; ++k) {
    W.cX[k] = (float4*)take(n16);
    W.cV[k] = (float4*)take(n16);
    W.cA[k] = (float4*)take(n16);
    W.cB[k] = (float4*)take(n16);
  }
  W.gP = (float4*)take(n16);
  W.gN = (float4*)take(n16);
  W.gG = (float4*)take(n16);
  W.gC = (float4*)take(n16);
  W.gU1 = (float4*)take(n16);
  W.gU2 = (float4*)take(n16);
  W.gU3 = (float4*)take(n16);
  W.R1 = (float4*)take(n16);
  W.R2 = (float4*)take(n16);
  W.argmax = (int*)take(n4);
  W.glob = (double*)take(AG_COUNT * 8);
  W.partials = (double*)take((size_t)AR_COUNT * W.max_chunks * 8);
  W.obj = (double*)take(8 * 8);
  W.ggrav = (double*)take((size_t)steps * 3 * 8);
  W.ticket = (unsigned*)take(64);
  W.status = (unsigned*)take(64);
  if ((size_t)(p - W.arena) > W.bytes) throw std::runtime_error("internal: adjoint arena overflow");
  CK(cudaMemsetAsync(W.ticket, 0, 64, c->stream));
  CK(cudaMemsetAsync(W.status, 0, 64, c->stream));
  W.steps = steps;
  W.every = every;
}

#define ALAUNCH(c, K, G, B, ...)                      \
  do {                                                \
    ++(c)->launch_counter;                            \
    K<<<(G), (B), 0, (c)->stream>>>(__VA_ARGS__);     \
    LAUNCH_CHECK();                                   \
  } while (0)

// End-of-step copies into a slot: the per-particle arrays by one kernel, the
// lists (chunk rows of n entries), the cell table and the scalar block by
// copies.
void adj_snap_end(cryo_ctx* c, AdjWindow& W, AdjWindow::Slot& sl) {
  const View V = c->view(c->cur);
  ALAUNCH(c, k_adj_snap_end, c->grid_blocks(), kBlock, V, c->sorted_perm, sl.end);
  const size_t row = (size_t)W.n * kNbrChunk * 4;  // bytes of one chunk row of the n particles
  const size_t pitch = (size_t)c->capacity * kNbrChunk * 4, dpitch = (size_t)W.cap * kNbrChunk * 4;
  if (W.n > 0)
    CK(cudaMemcpy2DAsync(sl.end.nbr, dpitch, c->nbr, pitch, row, kMaxNbr / kNbrChunk, cudaMemcpyDeviceToDevice,
                         c->stream));
  CK(cudaMemcpyAsync(sl.end.cell_begin, c->cell_begin, (size_t)(c->P.num_cells + 1) * 4, cudaMemcpyDeviceToDevice,
                     c->stream));
  CK(cudaMemcpyAsync(sl.end.dyn, c->dyn, sizeof(DynState), cudaMemcpyDeviceToDevice, c->stream));
}

// The arrays of a recomputed step (slot) through View, as the reverse
// kernels read them; the list chunk stride is the capacity the slot was
// sized by.
View slot_view(const AdjWindow& W, const AdjWindow::Slot& sl) {
  View V{};
  const AdjSlot& e = sl.end;
  V.xp = e.xp;
  V.vT = e.vT;
  V.vt = e.vt;
  V.nrm = e.nrm;
  V.mrps = e.mrps;
  V.a4 = e.a4;
  V.vwp = e.vwp;
  V.heat_w = e.heat_w;
  V.cell_begin = e.cell_begin;
  V.dyn = e.dyn;
  V.capacity = W.cap;
  V.nbr = e.nbr;
  V.nbr_cnt = e.nbr_cnt;
  V.fluid_idx = e.fluid_idx;
  V.wall_idx = e.wall_idx;
  return V;
}

void adj_reverse_step(cryo_ctx* c, AdjWindow& W, long long k, const AdjWindow::Slot& sl) {
  const Params& P = c->P;
  Adj A{};
  A.V = slot_view(W, sl);
  A.vT1 = sl.tape.vT1;
  A.m1 = sl.tape.m1;
  A.ns1 = sl.tape.ns1;
  A.pc2 = sl.tape.pc2;
  A.vT2 = sl.tape.vT2;
  A.m2 = sl.tape.m2;
  A.dyn1 = sl.tape.dyn1;
  A.sums = sl.tape.sums;
  A.sums_n = sl.tape.n;
  A.gX = W.cX[W.q];
  A.gV = W.cV[W.q];
  A.gA = W.cA[W.q];
  A.gB = W.cB[W.q];
  A.prevX = W.cX[1 - W.q];
  A.prevV = W.cV[1 - W.q];
  A.prevA = W.cA[1 - W.q];
  A.prevB = W.cB[1 - W.q];
  A.gP = W.gP;
  A.gN = W.gN;
  A.gG = W.gG;
  A.gC = W.gC;
  A.gU1 = W.gU1;
  A.gU2 = W.gU2;
  A.gU3 = W.gU3;
  A.R1 = W.R1;
  A.R2 = W.R2;
  A.argmax = W.argmax;
  A.perm = sl.end.perm;
  A.glob = W.glob;
  A.partials = W.partials;
  A.ticket = W.ticket;
  A.max_chunks = W.max_chunks;
  A.status = W.status;
  const size_t n16 = (size_t)W.n * 16;
  for (float4* a : {W.gP, W.gN, W.gG, W.gC, W.gU1, W.gU2, W.gU3}) CK(cudaMemsetAsync(a, 0, n16, c->stream));
  const int G = c->grid_blocks();
  const int GF = std::max(1, std::min((W.n + 127) / 128, c->sm_count * 16));
  ALAUNCH(c, k_adj_saturation_sums, G, kBlock, P, A);
  ALAUNCH(c, k_adj_rebalance_local, G, kBlock, P, A);
  if (P.cfg_phase_change) {
    ALAUNCH(c, k_adj_rebalance_gather, G, kBlock, P, A);
    ALAUNCH(c, k_adj_apply_local, G, kBlock, P, A);
    ALAUNCH(c, k_adj_apply_gather, G, kBlock, P, A);
    ALAUNCH(c, k_adj_normalize_local, G, kBlock, P, A);
    ALAUNCH(c, k_adj_normalize_gather, G, kBlock, P, A);
  }
  ALAUNCH(c, k_adj_kick_sources, G, kBlock, P, A);
  ALAUNCH(c, k_adj_forces_local, G, kBlock, P, A);
  {
    // heater-norm and gravity adjoints of this step (set), sigma and heater (summed)
    const AdjRows M{6, {AR_FORCE, AR_FORCE + 1, AR_FORCE + 2, AR_FORCE + 3, AR_FORCE + 4, AR_FORCE + 5},
                    {AG_HINV, AG_GRAV, AG_GRAV + 1, AG_GRAV + 2, AG_SIGMA, AG_HEAT}, {0, 0, 0, 0, 1, 1}};
    ALAUNCH(c, k_adj_reduce, M.count, kBlock, A, M);
  }
  ALAUNCH(c, k_adj_forces_gather, GF, 128, P, A);
  ALAUNCH(c, k_adj_interface_local, G, kBlock, P, A);
  ALAUNCH(c, k_adj_interface_gather, G, kBlock, P, A);
  ALAUNCH(c, k_adj_wall_local, G, kBlock, P, A);
  ALAUNCH(c, k_adj_wall_gather, G, kBlock, P, A);
  ALAUNCH(c, k_adj_density_gather, G, kBlock, P, A);
  {
    // T_sat adjoint of this step's input (set); Lee, contact angle (summed); wall part of gravity (added)
    const AdjRows M{8,
                    {AR_SRC, AR_SRC + 1, AR_SRC + 2, AR_IFACE, AR_IFACE + 1, AR_WALL, AR_WALL + 1, AR_WALL + 2},
                    {AG_TSAT_IN, AG_LEE_E, AG_LEE_C, AG_COS, AG_SIN, AG_GRAV, AG_GRAV + 1, AG_GRAV + 2},
                    {0, 1, 1, 1, 1, 1, 1, 1}};
    ALAUNCH(c, k_adj_reduce, M.count, kBlock, A, M);
  }
  ALAUNCH(c, k_adj_drift_scatter, G, kBlock, P, A);
  ALAUNCH(c, k_adj_step_end, 1, 32, W.glob, W.ggrav + 3 * k);
  W.q = 1 - W.q;
}

AdjWindow& adj_window(cryo_ctx* c) {
  if (!c->adj || !c->adj->recorded) throw std::runtime_error("adjoint: no recorded window (call cryo_adj_forward)");
  return *c->adj;
}

}  // namespace

extern "C" {

int cryo_set_surface_tension(cryo_ctx* c, float sigma) {
  return guard(c, [&] {
    if (!(sigma >= 0)) throw std::invalid_argument("surface tension must be >= 0");
    c->sync();
    c->fluid.sigma = sigma;
    c->P.sigma = c->cfg.surface_tension != CRYO_ST_NONE ? sigma : 0.0f;
    c->invalidate_graphs();
  });
}

int cryo_set_lee_coefficients(cryo_ctx* c, float evaporation, float condensation) {
  return guard(c, [&] {
    if (!(evaporation >= 0 && condensation >= 0)) throw std::invalid_argument("Lee coefficients must be >= 0");
    c->sync();
    c->cfg.lee_evaporation = evaporation;
    c->cfg.lee_condensation = condensation;
    c->P.lee_evap = evaporation;
    c->P.lee_cond = condensation;
    c->invalidate_graphs();
  });
}

int cryo_adj_forward(cryo_ctx* c, long long steps, int every, double* objectives) {
  return guard(c, [&] {
    if (steps < 1) throw std::invalid_argument("adjoint: steps must be >= 1");
    if (every < 1) throw std::invalid_argument("adjoint: checkpoint interval must be >= 1");
    adj_check_config(c);
    c->ensure_initialized();
    c->pull();
    if (!c->adj) c->adj = new AdjWindow;
    AdjWindow& W = *c->adj;
    W.recorded = false;
    W.n = c->hdyn->n;
    W.cap = c->capacity;
    W.splits0 = c->hdyn->splits;
    W.merges0 = c->hdyn->merges;
    adj_alloc(c, W, steps, every);
    CK(cudaMemsetAsync(W.obj, 0, 8 * 8, c->stream));
    for (long long k = 0; k < steps; ++k) {
      if (k % every == 0) snap_save(c, W, W.ckpt[(size_t)(k / every)]);
      c->launch_step();
      const View V = c->view(c->cur);
      ALAUNCH(c, k_adj_objective, c->grid_blocks(), kBlock, c->P, V, c->reduce(), W.obj);
    }
    snap_save(c, W, W.ckpt.back());
    double obj[6];
    CK(cudaMemcpyAsync(obj, W.obj, sizeof(obj), cudaMemcpyDeviceToHost, c->stream));
    c->pull();
    if (c->hdyn->n != W.n || c->hdyn->splits != W.splits0 || c->hdyn->merges != W.merges0)
      throw std::runtime_error("adjoint: particles split, merged or died inside the window (topology must stay fixed)");
    for (int k = 0; k < 6; ++k) objectives[k] = obj[k];
    objectives[6] = c->hdyn->p_ullage;
    for (auto& v : W.seed) v.clear();
    W.recorded = true;
  });
}

// Seeds of the final state's adjoint (tests): which 0 x, 1 v, 2 T, 3 m, 4 a,
// 5 ab; 3 or 1 floats per particle in the window's final order.
int cryo_adj_seed_state(cryo_ctx* c, int which, const float* data, size_t count) {
  return guard(c, [&] {
    AdjWindow& W = adj_window(c);
    if (which < 0 || which > 5) throw std::invalid_argument("adjoint: unknown state field");
    const int comps = (which == 2 || which == 3) ? 1 : 3;
    if (count != (size_t)W.n * comps) throw std::invalid_argument("adjoint: seed size mismatch");
    const int slot = which == 0 || which == 3 ? 0 : (which == 1 || which == 2 ? 1 : which - 2);
    std::vector<float4>& s = W.seed[slot];
    if (s.empty()) s.assign((size_t)W.n, make_float4(0, 0, 0, 0));
    for (int i = 0; i < W.n; ++i) {
      if (comps == 3) {
        s[i].x = data[3 * i];
        s[i].y = data[3 * i + 1];
        s[i].z = data[3 * i + 2];
      } else {
        s[i].w = data[i];
      }
    }
  });
}

int cryo_adj_backward(cryo_ctx* c, const double* seed, double* grads, double* frame_grads) {
  return guard(c, [&] {
    AdjWindow& W = adj_window(c);
    double g[AG_COUNT] = {0};
    for (int k = 0; k < 3; ++k) {
      g[AG_FW + k] = seed[k];
      g[AG_MW + k] = seed[3 + k];
    }
    g[AG_P_OBJ] = seed[6];
    CK(cudaMemcpyAsync(W.glob, g, sizeof(g), cudaMemcpyHostToDevice, c->stream));
    const size_t n16 = (size_t)W.n * 16;
    for (int k = 0; k < 2; ++k)
      for (float4* a : {W.cX[k], W.cV[k], W.cA[k], W.cB[k]}) CK(cudaMemsetAsync(a, 0, n16, c->stream));
    W.q = 0;
    float4* dst[4] = {W.cX[0], W.cV[0], W.cA[0], W.cB[0]};
    for (int k = 0; k < 4; ++k)
      if (!W.seed[k].empty()) CK(cudaMemcpyAsync(dst[k], W.seed[k].data(), n16, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(W.status, 0, 4, c->stream));
    c->sync();  // the pageable sources above are free again
    const long long nseg = (W.steps + W.every - 1) / W.every;
    for (long long sg = nseg - 1; sg >= 0; --sg) {
      const long long k0 = sg * W.every, k1 = std::min(W.steps, k0 + W.every);
      // recompute the segment once, keeping what each step's reverse reads
      snap_load(c, W, W.ckpt[(size_t)sg]);
      for (long long k = k0; k < k1; ++k) {
        AdjWindow::Slot& sl = W.slots[(size_t)(k - k0)];
        const int s = c->cur;
        c->enqueue_step(s, &sl.tape);
        c->cur = 1 - s;
        adj_snap_end(c, W, sl);
      }
      for (long long k = k1 - 1; k >= k0; --k) adj_reverse_step(c, W, k, W.slots[(size_t)(k - k0)]);
    }
    snap_load(c, W, W.ckpt.back());
    unsigned status = 0;
    std::vector<double> gg((size_t)W.steps * 3);
    CK(cudaMemcpyAsync(g, W.glob, sizeof(g), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&status, W.status, 4, cudaMemcpyDeviceToHost, c->stream));
    if (frame_grads) CK(cudaMemcpyAsync(gg.data(), W.ggrav, gg.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    c->pull();
    if (status & ADJ_TOPOLOGY) throw std::runtime_error("adjoint: a particle died inside the window");
    const double deg = (double)kPi / 180.0;
    grads[0] = g[AG_SIGMA];
    grads[1] = (-(double)c->P.sin_theta * g[AG_COS] + (double)c->P.cos_theta * g[AG_SIN]) * deg;
    grads[2] = g[AG_LEE_E];
    grads[3] = g[AG_LEE_C];
    grads[4] = g[AG_HEAT];
    if (frame_grads)
      for (size_t k = 0; k < gg.size(); ++k) frame_grads[k] = -gg[k];  // gravity = g - a_frame
  });
}

// Adjoint of the window's initial state (after cryo_adj_backward): which as
// in cryo_adj_seed_state, in the order of the state the window started from.
int cryo_adj_state_gradient(cryo_ctx* c, int which, float* out, size_t count) {
  return guard(c, [&] {
    AdjWindow& W = adj_window(c);
    if (which < 0 || which > 5) throw std::invalid_argument("adjoint: unknown state field");
    const int comps = (which == 2 || which == 3) ? 1 : 3;
    if (count != (size_t)W.n * comps) throw std::invalid_argument("adjoint: output size mismatch");
    const float4* src[6] = {W.cX[W.q], W.cV[W.q], W.cV[W.q], W.cX[W.q], W.cA[W.q], W.cB[W.q]};
    std::vector<float4> h((size_t)W.n);
    CK(cudaMemcpyAsync(h.data(), src[which], (size_t)W.n * 16, cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    for (int i = 0; i < W.n; ++i) {
      if (comps == 3) {
        out[3 * i] = h[i].x;
        out[3 * i + 1] = h[i].y;
        out[3 * i + 2] = h[i].z;
      } else {
        out[i] = h[i].w;
      }
    }
  });
}

int cryo_adj_memory(cryo_ctx* c, size_t* bytes) {
  return guard(c, [&] { *bytes = c->adj ? c->adj->bytes : 0; });
}

int cryo_adj_release(cryo_ctx* c) {
  return guard(c, [&] {
    c->sync();
    adj_free(c->adj);
    c->adj = nullptr;
  });
}

}  // extern "C"

