// cryo_ctx.cuh -- the host-side context behind every extern "C" entry point
// of cryosph_b200.h: device memory (one arena per context), the stream, the
// step graphs and the device-resident scalar block, plus the error mapping
// shared by the entry-point files (cryo_abi.cu: the solver; cryo_ensemble.cu:
// batched tanks; cryo_adj_abi.cu: the differentiated window; cryo_slab_abi.cu:
// one tank over several slabs).
//
// Nothing throws across the ABI: each entry point runs inside guard(), which
// maps exceptions to status codes the way the reference's exceptions map to
// Python (invalid_argument -> CRYO_EINVAL, out_of_range -> CRYO_ERANGE,
// runtime_error -> CRYO_ERUNTIME, CUDA failures -> CRYO_ECUDA).
#pragma once
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "cryo_adjoint.cuh"

using namespace cryo;

namespace cryo {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& m) : std::runtime_error(m) {}
};

#define CK(expr)                                                                                 \
  do {                                                                                           \
    const cudaError_t e__ = (expr);                                                              \
    if (e__ != cudaSuccess)                                                                      \
      throw CudaError(std::string("CUDA error '") + cudaGetErrorString(e__) + "' at " #expr);   \
  } while (0)

#define LAUNCH_CHECK() CK(cudaGetLastError())

// Kernel launch inside a cryo_ctx member: counted, and bracketed by events
// when profiling is on.
#define LAUNCH(K, G, B, ...)                     \
  do {                                           \
    this->before_launch(#K);                     \
    K<<<(G), (B), 0, this->stream>>>(__VA_ARGS__); \
    LAUNCH_CHECK();                              \
    this->after_launch();                        \
  } while (0)

// A kernel of cryo_physics.cu in the context's field arithmetic (exact: the
// reference's IEEE sequence; fast: contracted, see cryo_kernels.cuh).
#define FIELD_KERNEL(ctx, K) ((ctx)->fast_fields ? &fast::K : &exact::K)
#define FIELD_LAUNCH(K, G, B, ...)                  \
  do {                                              \
    if (this->fast_fields)                          \
      LAUNCH(fast::K, G, B, __VA_ARGS__);           \
    else                                            \
      LAUNCH(exact::K, G, B, __VA_ARGS__);          \
  } while (0)

struct Persist {
  float4 *xp = nullptr, *vT = nullptr, *vt = nullptr, *nrm = nullptr, *mrps = nullptr;
  uint32_t* id = nullptr;
};

// One device allocation carved into 256-byte aligned arrays.
struct Arena {
  char* base = nullptr;
  size_t size = 0, used = 0;
  void release() {
    if (base) cudaFree(base);
    base = nullptr;
    size = used = 0;
  }
  template <class T>
  T* take(size_t n) {
    const size_t bytes = (n * sizeof(T) + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + used);
    used += bytes;
    return p;
  }
};

inline size_t particle_bytes(size_t cap) {
  const size_t a = 256;
  auto r = [&](size_t b) { return (b + a - 1) / a * a; };
  size_t t = 0;
  for (int s = 0; s < 2; ++s) t += 5 * r(cap * 16) + r(cap * 4);    // persistent sets
  t += 8 * r(cap * 16) + 4 * r(cap * 4);                            // scratch
  t += 5 * r(cap * 4);                                              // sort keys/vals, split flags
  const size_t tiles = (cap + RS_TILE - 1) / RS_TILE + 1;
  t += r((tiles + 1) * RS_BINS * 4);                                // radix histogram + digit totals
  const size_t chunks = cap / kChunk + 2;
  t += r(chunks * 32 * 8);                                          // reduction partials
  t += r(64 * 8) + r(64);                                           // diagnostics out, tickets
  t += r(cap * 4 * (size_t)kMaxNbr) + 3 * r(cap * 4);              // neighbour lists, counts, phase lists
  return t;
}

}  // namespace cryo

void ensemble_detach(cryo_ensemble* e, cryo_ctx* c);
struct AdjWindow;
struct SlabGroup;
// Where a slab of a decomposed tank meets its neighbours inside a step:
// after a sort (its owned range), after a pass a later neighbour pass reads
// (the ghost layers), after the heat weights (also the heat normalisation),
// after the force pass (also the dt maxima), after the split marks (the
// split ids) and at the end (ullage and maxima).
enum SlabPoint { SLAB_SORTED, SLAB_HALO, SLAB_HEAT, SLAB_FORCES, SLAB_SPLIT, SLAB_END };
void adj_free(AdjWindow* w);

// Where a step recomputed for the reverse sweep leaves the values its later
// stages overwrite (cryo_adjoint.cuh, Adj).
struct StepTape {
  float4 *vT1, *ns1, *pc2, *vT2;
  float *m1, *m2;
  DynState* dyn1;
  float4* sums;  // View::tape for the taped force / interface variants
  int n;
};

// A context that holds the whole tank owns every particle.
inline void set_whole_tank(DynState& d) {
  d.own_lo = 0;
  d.own_hi = std::numeric_limits<int>::max();
  d.n_sorted = std::numeric_limits<int>::max();
  d.id_offset = 0;
  d.split_total = 0;
}

struct cryo_ctx {
  cryo_config_t cfg{};
  cryo_fluid_t fluid{};
  Params P{};
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  std::string err;

  // particle storage
  int capacity = 0;
  Arena arena;
  Persist set[2];
  int cur = 0;
  float4 *a4 = nullptr, *ab4 = nullptr, *fw = nullptr, *mw = nullptr, *vwp = nullptr, *ns4 = nullptr,
         *pc = nullptr, *aux = nullptr;
  float *rmin = nullptr, *wall_w = nullptr, *heat_w = nullptr, *nu_t = nullptr;
  uint32_t *keys_a = nullptr, *keys_b = nullptr, *vals_a = nullptr, *vals_b = nullptr, *split_flag = nullptr;
  uint32_t* hist = nullptr;
  int *nbr = nullptr, *nbr_cnt = nullptr, *fluid_idx = nullptr, *wall_idx = nullptr;
  double* partials = nullptr;
  int max_chunks = 0;
  double* diag_out = nullptr;
  unsigned* ticket = nullptr;
  const uint32_t* sorted_keys = nullptr;  // of the last grid build
  const uint32_t* sorted_perm = nullptr;
  int last_sort_n = 0;

  // grid
  int* cell_begin = nullptr;
  uint8_t* cell_fluid = nullptr;  // 1: a fluid particle was sorted into the cell
  int cell_cap = 0;

  // scalar block
  DynState* dyn = nullptr;   // device
  DynState* hdyn = nullptr;  // pinned host mirror
  double* diag_host = nullptr;  // pinned, 64 doubles
  // Non-blocking diagnostics (cryo_diagnostics_request / _fetch): a FIFO of
  // pinned result rows, each completed by an event on the stream.
  static constexpr int kDiagSlots = 8;
  double* diag_ring = nullptr;  // pinned, kDiagSlots rows of 64 doubles (made on first request)
  cudaEvent_t diag_ev[kDiagSlots] = {};
  long long diag_head = 0, diag_tail = 0;  // requests made, results fetched
  // Host-owned frame state (authoritative unless a manoeuvre table drives the
  // frame on the device); updates go out through a ring of pinned slots.
  DynState::Frame hframe{};
  bool man_active = false;
  static constexpr int kFrameSlots = 16;
  DynState::Frame* frame_ring = nullptr;
  cudaEvent_t frame_ev[kFrameSlots] = {};
  int frame_next = 0;

  // maneuver table (device)
  double* man_t = nullptr;
  float* man_acc = nullptr;
  float* man_omega = nullptr;
  int man_cap = 0;
  // host copy of the table (for host-side evaluation at set time)
  std::vector<double> h_man_t;
  std::vector<float> h_man_acc, h_man_omega;

  // solver state on the host side
  bool has_particles = false, initialized = false, has_vapor = false;
  bool lists_built = false;  // the neighbour lists of the current particles exist
  int loaded_n = -1;  // particle count of the last set_particles / build_tank
  float char_length = 0;
  float pass_dt = 0;

  // batched stepping: the ensemble this tank belongs to (if any), an event
  // for ordering its stream against the ensemble's, and a counter bumped
  // whenever the step graphs are invalidated (the ensemble then rebuilds)
  cryo_ensemble* ensemble = nullptr;
  cudaEvent_t ens_ev = nullptr;
  unsigned long long generation = 0;

  // slab decomposition: the group this context is one slab of (null: it
  // holds the whole tank)
  SlabGroup* slab_group = nullptr;
  int slab_rank = 0;
  void slab_point(int what, int set);

  // execution
  bool graph_mode = true;
  bool graph_valid[2] = {false, false};
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  bool use_lists = true;
  bool fast_fields = false;  // field arithmetic of the neighbour passes (cryo_set_field_arithmetic)

  // launch accounting / profiling
  long long launch_counter = 0;
  int step_launches = 0;
  bool profiling = false;
  struct Mark { cudaEvent_t a, b; int kernel; };
  std::vector<Mark> marks;
  std::vector<cudaEvent_t> event_pool;
  size_t event_used = 0;
  std::vector<std::string> prof_names;
  std::vector<double> prof_ms;
  std::vector<long long> prof_count;
  int prof_current = -1;

  // telemetry (TelemetryStream, telemetry.cu)
  int tele_mode = 0;
  size_t tele_cap = 0;
  TelemetryRecord* tele_host = nullptr;
  TelemetryRecord* tele_host_dev = nullptr;
  TelemetryRecord* tele_stage = nullptr;
  cudaStream_t tele_stream = nullptr;
  cudaEvent_t tele_computed = nullptr, tele_landed = nullptr;
  bool tele_pending = false;
  double tele_time = 0;
  long long tele_step = 0;
  int tele_n = 0;

  // host <-> device particle transfers and output frames (cryo_io.cu): a
  // device and a pinned host buffer of the same size, grown on demand
  char* io_dev = nullptr;
  char* io_host = nullptr;
  size_t io_cap = 0;
  void io_reserve(size_t bytes);

  // differentiated window (cryo_adj_*), and the sums tape of the step being
  // recomputed for it (View::tape; null otherwise)
  AdjWindow* adj = nullptr;
  float4* tape_sums = nullptr;
  int tape_n = 0;

  cudaEvent_t next_event() {
    if (event_used == event_pool.size()) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      event_pool.push_back(e);
    }
    return event_pool[event_used++];
  }
  void before_launch(const char* raw) {
    ++launch_counter;
    if (!profiling) return;
    std::string name(raw);
    const size_t lt = name.find('<');
    if (lt != std::string::npos) name = name.substr(0, lt);
    const size_t ns = name.rfind("::");
    if (ns != std::string::npos) name = name.substr(ns + 2);
    if (name == "k_forces_t") name = "k_forces";
    int k = 0;
    while (k < (int)prof_names.size() && prof_names[k] != name) ++k;
    if (k == (int)prof_names.size()) {
      prof_names.push_back(name);
      prof_ms.push_back(0.0);
      prof_count.push_back(0);
    }
    Mark m{next_event(), next_event(), k};
    CK(cudaEventRecord(m.a, stream));
    marks.push_back(m);
  }
  void after_launch() {
    if (!profiling) return;
    CK(cudaEventRecord(marks.back().b, stream));
  }
  void collect_marks() {
    if (marks.empty()) return;
    CK(cudaStreamSynchronize(stream));
    for (const Mark& m : marks) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, m.a, m.b));
      prof_ms[m.kernel] += ms;
      prof_count[m.kernel] += 1;
    }
    marks.clear();
    event_used = 0;
  }
  void telemetry_release() {
    if (tele_pending) {
      cudaEventSynchronize(tele_mode == 1 ? tele_computed : tele_landed);
      tele_pending = false;
    }
    if (tele_host) cudaFreeHost(tele_host);
    if (tele_stage) cudaFree(tele_stage);
    if (tele_stream) cudaStreamDestroy(tele_stream);
    if (tele_computed) cudaEventDestroy(tele_computed);
    if (tele_landed) cudaEventDestroy(tele_landed);
    tele_host = tele_host_dev = tele_stage = nullptr;
    tele_stream = nullptr;
    tele_computed = tele_landed = nullptr;
    tele_cap = 0;
  }

  ~cryo_ctx() {
    if (ensemble) ensemble_detach(ensemble, this);
    if (adj) {
      if (stream) cudaStreamSynchronize(stream);
      adj_free(adj);
    }
    if (ens_ev) cudaEventDestroy(ens_ev);
    telemetry_release();
    if (io_dev || io_host) {
      if (stream) cudaStreamSynchronize(stream);
      if (io_dev) cudaFree(io_dev);
      if (io_host) cudaFreeHost(io_host);
    }
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    for (int k = 0; k < 2; ++k)
      if (graph[k]) cudaGraphExecDestroy(graph[k]);
    if (stream) cudaStreamSynchronize(stream);
    arena.release();
    if (cell_begin) cudaFree(cell_begin);
    if (cell_fluid) cudaFree(cell_fluid);
    if (dyn) cudaFree(dyn);
    if (hdyn) cudaFreeHost(hdyn);
    if (diag_host) cudaFreeHost(diag_host);
    if (diag_ring) cudaFreeHost(diag_ring);
    for (cudaEvent_t e : diag_ev)
      if (e) cudaEventDestroy(e);
    if (frame_ring) cudaFreeHost(frame_ring);
    for (cudaEvent_t e : frame_ev)
      if (e) cudaEventDestroy(e);
    if (man_t) cudaFree(man_t);
    if (man_acc) cudaFree(man_acc);
    if (man_omega) cudaFree(man_omega);
    if (stream) cudaStreamDestroy(stream);
  }

  // ------------------------------------------------------------ helpers
  View view(int s) const {
    View V{};
    V.xp = set[s].xp; V.vT = set[s].vT; V.vt = set[s].vt; V.nrm = set[s].nrm; V.mrps = set[s].mrps;
    V.id = set[s].id;
    V.a4 = a4; V.ab4 = ab4; V.fw = fw; V.mw = mw; V.vwp = vwp; V.ns4 = ns4; V.pc = pc;
    V.rmin = rmin; V.wall_w = wall_w; V.heat_w = heat_w; V.nu_t = nu_t;
    V.aux = aux;
    V.cell_begin = cell_begin;
    V.cell_fluid = cell_fluid;
    V.dyn = dyn;
    V.man_t = man_t; V.man_acc = man_acc; V.man_omega = man_omega;
    V.partials = partials;
    V.counters = ticket;
    V.capacity = capacity;
    V.nbr = nbr;
    V.nbr_cnt = nbr_cnt;
    V.fluid_idx = fluid_idx;
    V.wall_idx = wall_idx;
    V.tape = tape_sums;
    V.tape_n = tape_n;
    return V;
  }
  Reduce reduce() const { return Reduce{partials, ticket, max_chunks}; }
  // Particles the launch grids are sized for (0: the capacity).  Every step
  // kernel loops over its particles with a grid stride, so any grid gives
  // the same results; a grid sized for the capacity (up to twice the count)
  // only adds blocks that find no particle.
  int grid_span = 0;
  int span() const { return grid_span > 0 ? std::min(grid_span, capacity) : capacity; }
  // the particle count last read plus head-room for splits; check_capacity
  // drops the graphs when the count outgrows it
  void size_grids() { grid_span = std::max(1, std::min(capacity, hdyn->n + hdyn->n / 8 + 1024)); }
  // Particles per thread of the grid-stride kernels (1: one thread per
  // particle).  Any value gives the same results; an ensemble's autotuner
  // picks it for the members' kernels (coarser grids of many small tanks
  // running side by side).
  int grid_tile = 1;
  int grid_blocks() const {
    const int per_block = kBlock * grid_tile;
    const int need = (span() + per_block - 1) / per_block;
    return std::max(1, std::min(need, sm_count * 8));
  }
  // force pass: one thread per particle (times the tile) up to two
  // full-occupancy waves
  int forces_blocks() const {
    const int per_block = FORCES_BLOCK * grid_tile;
    const int need = (span() + per_block - 1) / per_block;
    return std::max(1, std::min(need, sm_count * (2048 / FORCES_BLOCK) * 2));
  }
  void invalidate_graphs() {
    ++generation;
    for (int k = 0; k < 2; ++k) {
      if (graph[k]) cudaGraphExecDestroy(graph[k]);
      graph[k] = nullptr;
      graph_valid[k] = false;
    }
  }
  void sync() { CK(cudaStreamSynchronize(stream)); }
  void pull() {  // device scalar block -> host mirror
    CK(cudaMemcpyAsync(hdyn, dyn, sizeof(DynState), cudaMemcpyDeviceToHost, stream));
    sync();
    if (man_active) hframe = hdyn->fr;
  }
  void push() {  // host mirror -> device scalar block
    if (!man_active) hdyn->fr = hframe;
    CK(cudaMemcpyAsync(dyn, hdyn, sizeof(DynState), cudaMemcpyHostToDevice, stream));
    sync();
  }
  // Sends the host frame state without synchronising: the copy reads a
  // pinned ring slot that is not reused until its previous copy completed.
  void push_frame() {
    const int k = frame_next;
    frame_next = (frame_next + 1) % kFrameSlots;
    CK(cudaEventSynchronize(frame_ev[k]));
    frame_ring[k] = hframe;
    CK(cudaMemcpyAsync(&dyn->fr, frame_ring + k, sizeof(DynState::Frame), cudaMemcpyHostToDevice, stream));
    CK(cudaEventRecord(frame_ev[k], stream));
  }

  // -------------------------------------------------------- allocation
  void allocate(int cap) {
    sync();
    invalidate_graphs();
    Arena a;
    a.size = particle_bytes((size_t)cap);
    CK(cudaMalloc(&a.base, a.size));
    CK(cudaMemsetAsync(a.base, 0, a.size, stream));
    Persist ns[2];
    for (int s = 0; s < 2; ++s) {
      ns[s].xp = a.take<float4>(cap); ns[s].vT = a.take<float4>(cap); ns[s].vt = a.take<float4>(cap);
      ns[s].nrm = a.take<float4>(cap); ns[s].mrps = a.take<float4>(cap); ns[s].id = a.take<uint32_t>(cap);
    }
    float4* na4 = a.take<float4>(cap); float4* nab4 = a.take<float4>(cap); float4* nfw = a.take<float4>(cap);
    float4* nmw = a.take<float4>(cap); float4* nvwp = a.take<float4>(cap); float4* nns4 = a.take<float4>(cap);
    float4* npc = a.take<float4>(cap);
    float4* naux = a.take<float4>(cap);
    float* nrmin = a.take<float>(cap); float* nwall = a.take<float>(cap); float* nheat = a.take<float>(cap);
    float* nnut = a.take<float>(cap);
    uint32_t* nka = a.take<uint32_t>(cap); uint32_t* nkb = a.take<uint32_t>(cap);
    uint32_t* nva = a.take<uint32_t>(cap); uint32_t* nvb = a.take<uint32_t>(cap);
    uint32_t* nsf = a.take<uint32_t>(cap);
    const size_t tiles = (size_t)(cap + RS_TILE - 1) / RS_TILE + 1;
    uint32_t* nhist = a.take<uint32_t>(tiles * RS_BINS + RS_BINS);
    const int nchunks = cap / kChunk + 2;
    double* npart = a.take<double>((size_t)nchunks * 32);
    double* ndiag = a.take<double>(64);
    unsigned* ntick = a.take<unsigned>(64);
    int* nnbr = a.take<int>((size_t)cap * kMaxNbr);
    int* nnc = a.take<int>(cap);
    int* nfi = a.take<int>(cap);
    int* nwi = a.take<int>(cap);
    if (a.used > a.size) throw std::runtime_error("internal: arena overflow");
    // keep the first n particles of every array (ParticleSystem::grow,
    // particle_system.cpp:66-71)
    if (arena.base && capacity > 0) {
      pull();
      const size_t keep = (size_t)std::min(hdyn->n, cap);
      auto cp = [&](void* dst, const void* src, size_t elem) {
        if (keep) CK(cudaMemcpyAsync(dst, src, keep * elem, cudaMemcpyDeviceToDevice, stream));
      };
      for (int s = 0; s < 2; ++s) {
        cp(ns[s].xp, set[s].xp, 16); cp(ns[s].vT, set[s].vT, 16); cp(ns[s].vt, set[s].vt, 16);
        cp(ns[s].nrm, set[s].nrm, 16); cp(ns[s].mrps, set[s].mrps, 16); cp(ns[s].id, set[s].id, 4);
      }
      cp(na4, a4, 16); cp(nab4, ab4, 16); cp(nfw, fw, 16); cp(nmw, mw, 16); cp(nvwp, vwp, 16); cp(nns4, ns4, 16);
      cp(npc, pc, 16); cp(naux, aux, 16); cp(nrmin, rmin, 4); cp(nwall, wall_w, 4); cp(nheat, heat_w, 4); cp(nnut, nu_t, 4);
      sync();
    }
    arena.release();
    arena = a;
    set[0] = ns[0]; set[1] = ns[1];
    a4 = na4; ab4 = nab4; fw = nfw; mw = nmw; vwp = nvwp; ns4 = nns4; pc = npc; aux = naux;
    rmin = nrmin; wall_w = nwall; heat_w = nheat; nu_t = nnut;
    keys_a = nka; keys_b = nkb; vals_a = nva; vals_b = nvb; split_flag = nsf;
    hist = nhist; partials = npart; max_chunks = nchunks; diag_out = ndiag; ticket = ntick;
    nbr = nnbr; nbr_cnt = nnc; fluid_idx = nfi; wall_idx = nwi;
    lists_built = false;
    sorted_keys = nullptr;
    sorted_perm = nullptr;
    capacity = cap;
    if (hdyn) {
      pull();
      hdyn->capacity = cap;
      push();
    }
  }

  // --------------------------------------------------- parameter lowering
  void init_params();
  void configure_grid(const float* lo, const float* hi);
  void begin_load(int n, bool vapor, const float* lo, const float* hi);
  void finish_load(int n, uint32_t next_id);

  // ------------------------------------------------------ step pieces
  void grid_build(int src);               // keys of current positions, sort, cells, gather, lists
  void sort_and_gather(int src, int list_mode, bool reset_maxima = false);  // after keys_a holds the keys
  void evaluate_rates(int s, bool maxima_reset, bool density_done, bool tape = false);
  void enqueue_step(int s, const StepTape* tape = nullptr);
  void launch_step();
  void ensure_initialized();
  void check_capacity();
  void run_steps(long long n);
  void run_until(double t_end);
};

namespace cryo {
// Message of the last failed create call on this thread (no context to hold it).
extern thread_local std::string g_create_error;
// cryo_diagnostics_t from the diagnostics reduction's FP64 values (cryo_abi.cu).
void diag_fill(const double* v, cryo_diagnostics_t* o);

template <class F>
inline int guard(cryo_ctx* ctx, F&& f) {
  try {
    f();
    return CRYO_OK;
  } catch (const std::invalid_argument& e) {
    if (ctx) ctx->err = e.what(); else g_create_error = e.what();
    return CRYO_EINVAL;
  } catch (const std::out_of_range& e) {
    if (ctx) ctx->err = e.what(); else g_create_error = e.what();
    return CRYO_ERANGE;
  } catch (const CudaError& e) {
    if (ctx) ctx->err = e.what(); else g_create_error = e.what();
    return CRYO_ECUDA;
  } catch (const std::exception& e) {
    if (ctx) ctx->err = e.what(); else g_create_error = e.what();
    return CRYO_ERUNTIME;
  }
}

inline void set3(float* d, const float* s) { d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; }

}  // namespace cryo

