// cryo_slab_abi.cu -- one tank over several slabs: the slab group (one
// context per slab, host threads meeting at the exchange points) and its
// extern "C" entry points (cryo_slab_partition, cryo_slabs_*).
#include "cryo_ctx.cuh"

// ===========================================================================
// Slab decomposition of one tank (no counterpart in the reference; the device
// side and the ownership rules are in cryo_slab.cu).  Each slab is a context
// on its own device (or several on one device).  One host thread per slab
// enqueues that slab's step; the threads meet at every SlabPoint (a host
// barrier), so each slab's stream can wait on its neighbours' events before
// it reads their memory, and they wait on its events before they overwrite
// what it read.  No kernel waits on another slab's kernel.
//
// In graph mode (the default) that enqueue runs once, under stream capture:
// slab 0's stream forks into every other slab's stream, the exchange points
// become graph edges between the slabs' kernels, and every stream joins back
// into slab 0's.  The steps then replay that one graph, with no host thread
// or barrier inside a step.  A group whose capture the runtime refuses (for
// instance across devices that cannot share one graph) steps without it.
namespace {

class HostBarrier {
 public:
  explicit HostBarrier(int n) : count_(n) {}
  // Blocks until every thread arrived; throws when another thread gave up.
  void wait() {
    std::unique_lock<std::mutex> lk(m_);
    if (broken_) throw std::runtime_error("slabs: another slab failed");
    const unsigned g = gen_;
    if (++waiting_ == count_) {
      waiting_ = 0;
      ++gen_;
      cv_.notify_all();
      return;
    }
    cv_.wait(lk, [&] { return gen_ != g || broken_; });
    if (gen_ == g) throw std::runtime_error("slabs: another slab failed");
  }
  void fail() {
    std::lock_guard<std::mutex> lk(m_);
    broken_ = true;
    cv_.notify_all();
  }
  void reset() {
    std::lock_guard<std::mutex> lk(m_);
    broken_ = false;
    waiting_ = 0;
  }

 private:
  std::mutex m_;
  std::condition_variable cv_;
  int count_, waiting_ = 0;
  unsigned gen_ = 0;
  bool broken_ = false;
};

}  // namespace

struct SlabGroup {
  // Neighbour layers copied in between steps.  A particle moves far less
  // than a layer (2h) per step, so the ghost layer next to a slab after the
  // drift holds only particles that were in the two layers before it.
  static constexpr int kRefreshLayers = 2;
  std::vector<cryo_ctx*> slabs;
  std::vector<int> zb;          // slab r owns cell layers [zb[r], zb[r + 1])
  std::vector<View> live;       // each slab's live arrays at the current point
  std::vector<cudaEvent_t> ev_a, ev_b;
  std::vector<DynState**> dyn_table;  // per slab, on its device: every slab's scalar block
  std::vector<float4*> spare;         // per slab: a4 / ab4 of a refresh (2 x capacity)
  std::vector<int> spare_cap;
  HostBarrier barrier;
  // the captured group step (graph mode)
  bool graph_mode = true;
  bool graph_refused = false;  // the runtime refused the capture: eager steps
  cudaGraphExec_t gexec = nullptr;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  std::vector<unsigned long long> graph_gen;  // each slab's graph generation at capture
  std::vector<float4*> graph_spare;
  std::vector<int> graph_cur;

  explicit SlabGroup(int n) : barrier(n) {}
  int count() const { return (int)slabs.size(); }

  // A pass's outputs are complete on every slab: pull the ghost layers next
  // to this slab from their owners, then combine what `what` needs.
  void point(int r, int what, int set) {
    cryo_ctx* c = slabs[r];
    if (what == SLAB_SORTED) {
      k_slab_bounds<<<1, 1, 0, c->stream>>>(c->P, c->view(set), zb[r], zb[r + 1]);
      CK(cudaGetLastError());
      return;
    }
    const int R = count();
    const bool every = what != SLAB_HALO;  // the combines read every slab
    live[r] = c->view(set);
    CK(cudaEventRecord(ev_a[r], c->stream));
    barrier.wait();
    for (int q = 0; q < R; ++q)
      if (q != r && (every || q == r - 1 || q == r + 1)) CK(cudaStreamWaitEvent(c->stream, ev_a[q], 0));
    if (what == SLAB_HALO || what == SLAB_HEAT || what == SLAB_FORCES) {
      const int G = std::max(1, c->sm_count * 2);
      if (r > 0) k_halo_pull<<<G, kBlock, 0, c->stream>>>(c->P, live[r], live[r - 1], zb[r] - 1);
      if (r + 1 < R) k_halo_pull<<<G, kBlock, 0, c->stream>>>(c->P, live[r], live[r + 1], zb[r + 1]);
    }
    if (what == SLAB_HEAT) k_slab_heat<<<1, 1, 0, c->stream>>>(c->P, dyn_table[r], R, c->dyn, 1);
    if (what == SLAB_SPLIT) k_slab_split<<<1, 1, 0, c->stream>>>(dyn_table[r], R, r, c->dyn);
    if (what == SLAB_FORCES) k_slab_end<<<1, 1, 0, c->stream>>>(c->P, dyn_table[r], R, c->dyn, 0);
    if (what == SLAB_END) k_slab_end<<<1, 1, 0, c->stream>>>(c->P, dyn_table[r], R, c->dyn, 1);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ev_b[r], c->stream));
    barrier.wait();
    for (int q = 0; q < R; ++q)
      if (q != r && (every || q == r - 1 || q == r + 1)) CK(cudaStreamWaitEvent(c->stream, ev_b[q], 0));
  }

  // Between steps: rebuild this slab's arrays from its owned particles and
  // the layers of its neighbours that face it (cryo_slab.cu, k_slab_assemble).
  void refresh(int r) {
    cryo_ctx* c = slabs[r];
    const int R = count();
    live[r] = c->view(c->cur);
    CK(cudaEventRecord(ev_a[r], c->stream));
    barrier.wait();
    if (r > 0) CK(cudaStreamWaitEvent(c->stream, ev_a[r - 1], 0));
    if (r + 1 < R) CK(cudaStreamWaitEvent(c->stream, ev_a[r + 1], 0));
    const View dst = c->view(1 - c->cur);
    const View& lo = r > 0 ? live[r - 1] : live[r];
    const View& up = r + 1 < R ? live[r + 1] : live[r];
    float4* a4 = spare[r];
    float4* ab4 = spare[r] + spare_cap[r];
    const int G = c->grid_blocks();
    k_slab_assemble<<<G, kBlock, 0, c->stream>>>(c->P, dst, a4, ab4, lo, live[r], up, r > 0 ? 1 : 0,
                                                  r + 1 < R ? 1 : 0, zb[r], zb[r + 1], kRefreshLayers);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ev_b[r], c->stream));
    barrier.wait();
    if (r > 0) CK(cudaStreamWaitEvent(c->stream, ev_b[r - 1], 0));
    if (r + 1 < R) CK(cudaStreamWaitEvent(c->stream, ev_b[r + 1], 0));
    k_slab_commit<<<G, kBlock, 0, c->stream>>>(dst, a4, ab4);
    CK(cudaGetLastError());
    c->cur = 1 - c->cur;
  }

  // Runs body(r) for every slab in its own thread; the first failure is
  // rethrown after every thread has ended.  sync: wait for the streams
  // afterwards (not while they are being captured).
  template <class F>
  void lockstep(F&& body, bool sync = true) {
    barrier.reset();
    const int R = count();
    std::vector<std::exception_ptr> errs(R);
    std::vector<std::thread> th;
    th.reserve(R);
    for (int r = 0; r < R; ++r)
      th.emplace_back([&, r] {
        try {
          CK(cudaSetDevice(slabs[r]->device));
          body(r);
        } catch (...) {
          errs[r] = std::current_exception();
          barrier.fail();
        }
      });
    for (auto& t : th) t.join();
    if (sync)
      for (cryo_ctx* c : slabs) cudaStreamSynchronize(c->stream);
    // a real error first, not another thread's "another slab failed"
    for (int pass = 0; pass < 2; ++pass)
      for (int r = 0; r < R; ++r) {
        if (!errs[r]) continue;
        try {
          std::rethrow_exception(errs[r]);
        } catch (const std::runtime_error& e) {
          if (pass == 0 && std::string(e.what()).rfind("slabs: another slab failed", 0) == 0) continue;
          throw;
        }
      }
  }

  // Guard words, capacity head-room and spare arrays between step batches.
  void check() {
    unsigned bad = 0;
    for (cryo_ctx* c : slabs) {
      CK(cudaSetDevice(c->device));
      c->pull();
      bad |= c->hdyn->status & (CRYO_DEV_SLAB_HALO | CRYO_DEV_SLAB_CAPACITY);
    }
    if (bad & CRYO_DEV_SLAB_HALO)
      throw std::runtime_error("slabs: a slab and its neighbour hold different ghost layers (a particle moved "
                               "more than a cell layer in one step?)");
    if (bad & CRYO_DEV_SLAB_CAPACITY) throw std::runtime_error("slabs: a refreshed slab did not fit its capacity");
    for (int r = 0; r < count(); ++r) {
      cryo_ctx* c = slabs[r];
      CK(cudaSetDevice(c->device));
      c->check_capacity();
      if (spare_cap[r] < c->capacity) alloc_spare(r);
    }
  }
  void alloc_spare(int r) {
    cryo_ctx* c = slabs[r];
    CK(cudaSetDevice(c->device));
    if (spare[r]) CK(cudaFree(spare[r]));
    spare[r] = nullptr;
    CK(cudaMalloc(&spare[r], (size_t)2 * c->capacity * sizeof(float4)));
    spare_cap[r] = c->capacity;
  }

  void initialize() {
    bool need = false;
    for (cryo_ctx* c : slabs) need |= !c->initialized;
    if (!need) return;
    lockstep([&](int r) { slabs[r]->ensure_initialized(); });
    check();
  }

  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
  }
  // The captured step is valid while no slab re-allocated or re-sized its
  // grids (its graph generation) and the spare arrays and buffer parities
  // are those of the capture.
  bool graph_current() const {
    if (!gexec) return false;
    for (int r = 0; r < count(); ++r)
      if (slabs[r]->generation != graph_gen[r] || spare[r] != graph_spare[r] || slabs[r]->cur != graph_cur[r])
        return false;
    return true;
  }
  // One step of every slab (refresh + step) captured into one graph rooted
  // on slab 0's stream.  Returns false when the runtime refused the capture.
  bool capture() {
    drop_graph();
    const int R = count();
    for (cryo_ctx* c : slabs) c->size_grids();
    if (!ev_fork) CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    if ((int)ev_join.size() != R) {
      ev_join.assign(R, nullptr);
      for (int r = 0; r < R; ++r) {
        CK(cudaSetDevice(slabs[r]->device));
        CK(cudaEventCreateWithFlags(&ev_join[r], cudaEventDisableTiming));
      }
    }
    std::vector<unsigned long long> gen(R);
    std::vector<int> cur(R);
    for (int r = 0; r < R; ++r) {
      gen[r] = slabs[r]->generation;
      cur[r] = slabs[r]->cur;
    }
    cryo_ctx* c0 = slabs[0];
    CK(cudaSetDevice(c0->device));
    CK(cudaStreamSynchronize(c0->stream));
    CK(cudaStreamBeginCapture(c0->stream, cudaStreamCaptureModeRelaxed));
    cudaGraph_t g = nullptr;
    try {
      CK(cudaEventRecord(ev_fork, c0->stream));
      for (int r = 1; r < R; ++r) {
        CK(cudaSetDevice(slabs[r]->device));
        CK(cudaStreamWaitEvent(slabs[r]->stream, ev_fork, 0));
      }
      lockstep([&](int r) {
        refresh(r);
        slabs[r]->launch_step();
      }, false);
      for (int r = 1; r < R; ++r) {
        CK(cudaSetDevice(slabs[r]->device));
        CK(cudaEventRecord(ev_join[r], slabs[r]->stream));
        CK(cudaSetDevice(c0->device));
        CK(cudaStreamWaitEvent(c0->stream, ev_join[r], 0));
      }
      CK(cudaSetDevice(c0->device));
      CK(cudaStreamEndCapture(c0->stream, &g));
      CK(cudaGraphInstantiate(&gexec, g, 0));
      CK(cudaGraphDestroy(g));
    } catch (...) {
      cudaSetDevice(c0->device);
      cudaGraph_t bad = nullptr;
      cudaStreamEndCapture(c0->stream, &bad);
      if (bad) cudaGraphDestroy(bad);
      if (g) cudaGraphDestroy(g);
      gexec = nullptr;
      (void)cudaGetLastError();
      // the capture enqueued nothing; the host side of the step (buffer
      // parities) is put back
      for (int r = 0; r < R; ++r) slabs[r]->cur = cur[r];
      try {
        throw;
      } catch (const CudaError&) {
        return false;  // refused by the runtime: the group steps without a graph
      }
    }
    // the capture only recorded the step: the parities it flipped are the
    // ones the replay flips, and every step returns them to these values
    for (int r = 0; r < R; ++r) slabs[r]->cur = cur[r];
    graph_gen = gen;
    graph_spare = spare;
    graph_cur = cur;
    return true;
  }

  void run(long long n) {
    initialize();
    while (n > 0) {
      const int k = (int)std::min<long long>(n, 16);
      bool done = false;
      if (graph_mode && !graph_refused) {
        if (!graph_current() && !capture()) graph_refused = true;
        if (!graph_refused) {
          cryo_ctx* c0 = slabs[0];
          CK(cudaSetDevice(c0->device));
          for (int q = 0; q < k; ++q) CK(cudaGraphLaunch(gexec, c0->stream));
          CK(cudaStreamSynchronize(c0->stream));
          done = true;
        }
      }
      if (!done)
        lockstep([&](int r) {
          for (int q = 0; q < k; ++q) {
            refresh(r);
            slabs[r]->launch_step();
          }
        });
      check();
      n -= k;
    }
  }

  ~SlabGroup() {  // also after a failed create: slabs not made yet are null
    for (cryo_ctx* c : slabs)
      if (c && c->stream) cudaStreamSynchronize(c->stream);
    drop_graph();
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (cudaEvent_t e : ev_join)
      if (e) cudaEventDestroy(e);
    for (size_t r = 0; r < slabs.size(); ++r) {
      if (r < spare.size() && spare[r]) cudaFree(spare[r]);
      if (r < dyn_table.size() && dyn_table[r]) cudaFree(dyn_table[r]);
      if (r < ev_a.size() && ev_a[r]) cudaEventDestroy(ev_a[r]);
      if (r < ev_b.size() && ev_b[r]) cudaEventDestroy(ev_b[r]);
    }
    for (cryo_ctx* c : slabs) delete c;
  }
};

void cryo_ctx::slab_point(int what, int set) {
  if (slab_group) slab_group->point(slab_rank, what, set);
}

struct cryo_slabs {
  SlabGroup* g = nullptr;
  std::string err;
  ~cryo_slabs() { delete g; }
};

namespace {

template <class F>
int slab_guard(cryo_slabs* s, F&& f) {
  try {
    f();
    return CRYO_OK;
  } catch (const std::invalid_argument& e) {
    s->err = e.what();
    return CRYO_EINVAL;
  } catch (const std::out_of_range& e) {
    s->err = e.what();
    return CRYO_ERANGE;
  } catch (const CudaError& e) {
    s->err = e.what();
    return CRYO_ECUDA;
  } catch (const std::exception& e) {
    s->err = e.what();
    return CRYO_ERUNTIME;
  }
}

// Cell layer of a position, with the device's cell_coords operations.
int host_layer(const Params& P, float z) {
  const float f = std::floor((z - P.oz) * P.inv_cell);
  const int cz = (f >= 2147483648.0f || f < -2147483648.0f || f != f) ? std::numeric_limits<int>::min() : (int)f;
  return std::min(std::max(cz, 0), P.nz - 1);
}

}  // namespace

extern "C" {

// Slab boundaries: layers [z_begin[r], z_begin[r+1]) to slab r, each slab at
// least min_layers thick, the cuts where the running particle count crosses
// r / nslabs of the total.
int cryo_slab_partition(const long long* layer_counts, int nz, int nslabs, int min_layers, int* z_begin) {
  if (nslabs < 1 || min_layers < 1 || nz < 1 || (long long)nslabs * min_layers > nz || !layer_counts || !z_begin)
    return CRYO_EINVAL;
  long long total = 0;
  for (int z = 0; z < nz; ++z) {
    if (layer_counts[z] < 0) return CRYO_EINVAL;
    total += layer_counts[z];
  }
  z_begin[0] = 0;
  z_begin[nslabs] = nz;
  long long before = 0;  // particles in layers [0, cut)
  int cut = 0;
  for (int r = 1; r < nslabs; ++r) {
    const long long target = (total * r + nslabs / 2) / nslabs;
    const int lo = z_begin[r - 1] + min_layers;    // the slab before keeps min_layers
    const int hi = nz - (nslabs - r) * min_layers;  // and so can every slab after
    while (cut < lo) before += layer_counts[cut++];
    while (cut < hi && before + layer_counts[cut] <= target) before += layer_counts[cut++];
    z_begin[r] = cut;
  }
  return CRYO_OK;
}

int cryo_slabs_create(const cryo_config_t* cfg, const cryo_fluid_t* fluid, int nslabs, const int* devices,
                      cryo_slabs** out) {
  *out = nullptr;
  if (nslabs < 1) {
    g_create_error = "slabs: need at least one slab";
    return CRYO_EINVAL;
  }
  cryo_slabs* S = new cryo_slabs;
  const int rc = slab_guard(S, [&] {
    S->g = new SlabGroup(nslabs);
    SlabGroup& G = *S->g;
    G.slabs.assign(nslabs, nullptr);
    G.live.resize(nslabs);
    G.ev_a.assign(nslabs, nullptr);
    G.ev_b.assign(nslabs, nullptr);
    G.dyn_table.assign(nslabs, nullptr);
    G.spare.assign(nslabs, nullptr);
    G.spare_cap.assign(nslabs, 0);
    for (int r = 0; r < nslabs; ++r) {
      const int dev = devices ? devices[r] : 0;
      cryo_ctx* c = nullptr;
      if (cryo_create(cfg, fluid, dev, &c) != CRYO_OK) throw std::invalid_argument(g_create_error);
      G.slabs[r] = c;
      c->slab_group = &G;
      c->slab_rank = r;
      c->graph_mode = false;  // the slabs' steps meet on the host between passes
      CK(cudaEventCreateWithFlags(&G.ev_a[r], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&G.ev_b[r], cudaEventDisableTiming));
    }
    // neighbours on other devices read each other's memory
    for (int r = 0; r + 1 < nslabs; ++r) {
      const int a = G.slabs[r]->device, b = G.slabs[r + 1]->device;
      if (a == b) continue;
      for (const auto& pr : {std::make_pair(a, b), std::make_pair(b, a)}) {
        int can = 0;
        CK(cudaDeviceCanAccessPeer(&can, pr.first, pr.second));
        if (!can) throw std::runtime_error("slabs: devices " + std::to_string(pr.first) + " and " +
                                           std::to_string(pr.second) + " cannot reach each other's memory");
        CK(cudaSetDevice(pr.first));
        const cudaError_t e = cudaDeviceEnablePeerAccess(pr.second, 0);
        if (e == cudaErrorPeerAccessAlreadyEnabled) (void)cudaGetLastError();
        else CK(e);
      }
    }
    std::vector<DynState*> table(nslabs);
    for (int r = 0; r < nslabs; ++r) table[r] = G.slabs[r]->dyn;
    for (int r = 0; r < nslabs; ++r) {
      CK(cudaSetDevice(G.slabs[r]->device));
      CK(cudaMalloc(&G.dyn_table[r], nslabs * sizeof(DynState*)));
      CK(cudaMemcpy(G.dyn_table[r], table.data(), nslabs * sizeof(DynState*), cudaMemcpyHostToDevice));
    }
  });
  if (rc != CRYO_OK) {
    g_create_error = S->err;
    delete S;
    return rc;
  }
  *out = S;
  return CRYO_OK;
}

void cryo_slabs_destroy(cryo_slabs* s) { delete s; }

const char* cryo_slabs_last_error(const cryo_slabs* s) { return s ? s->err.c_str() : g_create_error.c_str(); }

int cryo_slabs_count(cryo_slabs* s, int* nslabs) {
  return slab_guard(s, [&] { *nslabs = s->g->count(); });
}

// Solver::set_particles of the whole tank (sph_solver.cu:407-428), cut into
// the slabs: slab r receives, in input order, the particles of its layers and
// of kRefreshLayers layers on either side.
int cryo_slabs_set_particles(cryo_slabs* s, const cryo_host_particles_t* p, const float* lo, const float* hi) {
  return slab_guard(s, [&] {
    SlabGroup& G = *s->g;
    G.drop_graph();
    const int n = p->n;
    if (n <= 0) throw std::invalid_argument("Solver::set_particles: no particles");
    bool vap = false;
    for (int i = 0; i < n; ++i) vap |= p->phase[i] == CRYO_VAPOR;
    uint32_t next_id = 0;
    for (int i = 0; i < n; ++i) next_id = std::max(next_id, (p->id ? p->id[i] : (uint32_t)i) + 1);
    const int R = G.count();
    cryo_ctx* c0 = G.slabs[0];
    CK(cudaSetDevice(c0->device));
    c0->begin_load(1, vap, lo, hi);  // the grid the whole tank has
    const Params P0 = c0->P;
    std::vector<int> layer(n);
    std::vector<long long> counts(P0.nz, 0);
    for (int i = 0; i < n; ++i) {
      layer[i] = host_layer(P0, p->x[3 * i + 2]);
      ++counts[layer[i]];
    }
    G.zb.assign(R + 1, 0);
    if (cryo_slab_partition(counts.data(), P0.nz, R, SlabGroup::kRefreshLayers, G.zb.data()) != CRYO_OK)
      throw std::invalid_argument("slabs: the tank has " + std::to_string(P0.nz) + " cell layers, fewer than " +
                                  std::to_string(SlabGroup::kRefreshLayers) + " per slab");
    for (int r = 0; r < R; ++r) {
      long long own = 0;
      for (int z = G.zb[r]; z < G.zb[r + 1]; ++z) own += counts[z];
      if (own == 0) throw std::invalid_argument("slabs: slab " + std::to_string(r) + " would hold no particle");
    }
    for (int r = 0; r < R; ++r) {
      cryo_ctx* c = G.slabs[r];
      CK(cudaSetDevice(c->device));
      const int z0 = G.zb[r] - SlabGroup::kRefreshLayers, z1 = G.zb[r + 1] + SlabGroup::kRefreshLayers;
      std::vector<int> idx;
      for (int i = 0; i < n; ++i)
        if (layer[i] >= z0 && layer[i] < z1) idx.push_back(i);
      const int m = (int)idx.size();
      c->begin_load(std::max(m, 1), vap, lo, hi);
      c->P.slab_z0 = G.zb[r];  // the passes run over owned particles only
      c->P.slab_z1 = G.zb[r + 1];
      std::vector<float4> xp(m), vT(m), vt(m), nrm(m), mrps(m);
      std::vector<uint32_t> id(m);
      for (int k = 0; k < m; ++k) {
        const int i = idx[k];
        const float* x = p->x + 3 * i;
        const float v0 = p->v ? p->v[3 * i] : 0.f, v1 = p->v ? p->v[3 * i + 1] : 0.f, v2 = p->v ? p->v[3 * i + 2] : 0.f;
        xp[k] = make_float4(x[0], x[1], x[2], pack_pf(p->phase[i], p->flags ? p->flags[i] : 0));
        vT[k] = make_float4(v0, v1, v2, p->T[i]);
        vt[k] = make_float4(v0, v1, v2, p->m[i]);
        nrm[k] = p->nrm ? make_float4(p->nrm[3 * i], p->nrm[3 * i + 1], p->nrm[3 * i + 2], 0.f)
                        : make_float4(0.f, 0.f, 0.f, 0.f);
        mrps[k] = make_float4(p->m[i], p->rho[i], 0.f, 0.f);
        id[k] = p->id ? p->id[i] : (uint32_t)i;
      }
      const Persist& st = c->set[0];
      if (m > 0) {
        CK(cudaMemcpyAsync(st.xp, xp.data(), (size_t)m * 16, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(st.vT, vT.data(), (size_t)m * 16, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(st.vt, vt.data(), (size_t)m * 16, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(st.nrm, nrm.data(), (size_t)m * 16, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(st.mrps, mrps.data(), (size_t)m * 16, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(st.id, id.data(), (size_t)m * 4, cudaMemcpyHostToDevice, c->stream));
      }
      c->finish_load(m, next_id);
      G.alloc_spare(r);
    }
  });
}

int cryo_slabs_layout(cryo_slabs* s, int* z_begin, int* owned, int* held) {
  return slab_guard(s, [&] {
    SlabGroup& G = *s->g;
    if (!z_begin) throw std::invalid_argument("cryo_slabs_layout: z_begin is required");
    if (G.zb.empty()) throw std::runtime_error("slabs: no particles loaded");
    G.initialize();
    for (int r = 0; r <= G.count(); ++r) z_begin[r] = G.zb[r];
    for (int r = 0; r < G.count(); ++r) {
      cryo_ctx* c = G.slabs[r];
      CK(cudaSetDevice(c->device));
      c->pull();
      const DynState& d = *c->hdyn;
      if (owned) owned[r] = (d.own_hi - d.own_lo) + (d.n - d.n_sorted);
      if (held) held[r] = d.n;
    }
  });
}

int cryo_slabs_set_graph_mode(cryo_slabs* s, int enable) {
  return slab_guard(s, [&] {
    SlabGroup& G = *s->g;
    for (cryo_ctx* c : G.slabs) {
      CK(cudaSetDevice(c->device));
      CK(cudaStreamSynchronize(c->stream));
    }
    G.graph_mode = enable != 0;
    G.graph_refused = false;
    G.drop_graph();
  });
}

int cryo_slabs_graph_mode(cryo_slabs* s, int* mode) {
  return slab_guard(s, [&] {
    const SlabGroup& G = *s->g;
    *mode = !G.graph_mode ? 0 : (G.graph_refused ? 2 : 1);
  });
}

int cryo_slabs_run_steps(cryo_slabs* s, long long n) {
  return slab_guard(s, [&] {
    if (s->g->zb.empty()) throw std::runtime_error("Solver: no particles loaded");
    s->g->run(n);
  });
}

int cryo_slabs_num_particles(cryo_slabs* s, int* n) {
  return slab_guard(s, [&] {
    SlabGroup& G = *s->g;
    if (G.zb.empty()) throw std::runtime_error("Solver: no particles loaded");
    G.initialize();
    long long t = 0;
    for (cryo_ctx* c : G.slabs) {
      CK(cudaSetDevice(c->device));
      c->pull();
      const DynState& d = *c->hdyn;
      t += (d.own_hi - d.own_lo) + (d.n - d.n_sorted);
    }
    *n = (int)t;
  });
}

// Solver::particles of the whole tank: every slab's owned sorted range in slab
// order, then every slab's split children in slab order -- the order the whole
// tank's own arrays have.
int cryo_slabs_download(cryo_slabs* s, cryo_host_particles_out_t* o) {
  return slab_guard(s, [&] {
    SlabGroup& G = *s->g;
    if (G.zb.empty()) throw std::runtime_error("Solver: no particles loaded");
    G.initialize();
    const int R = G.count();
    struct Part {
      std::vector<float> x, v, nrm, m, rho, T;
      std::vector<uint8_t> phase, flags;
      std::vector<uint32_t> id;
      int n, lo, hi, ns;
    };
    std::vector<Part> parts(R);
    long long total = 0;
    for (int r = 0; r < R; ++r) {
      cryo_ctx* c = G.slabs[r];
      CK(cudaSetDevice(c->device));
      c->pull();
      Part& q = parts[r];
      q.n = c->hdyn->n;
      q.lo = c->hdyn->own_lo;
      q.hi = c->hdyn->own_hi;
      q.ns = c->hdyn->n_sorted;
      q.x.resize(3 * (size_t)q.n); q.v.resize(3 * (size_t)q.n); q.nrm.resize(3 * (size_t)q.n);
      q.m.resize(q.n); q.rho.resize(q.n); q.T.resize(q.n);
      q.phase.resize(q.n); q.flags.resize(q.n); q.id.resize(q.n);
      cryo_host_particles_out_t t{q.n, q.x.data(), q.v.data(), q.nrm.data(), q.m.data(), q.rho.data(),
                                  q.T.data(), q.phase.data(), q.flags.data(), q.id.data()};
      if (cryo_download(c, &t) != CRYO_OK) throw std::runtime_error(c->err);
      total += (q.hi - q.lo) + (q.n - q.ns);
    }
    if (o->n < total) {
      o->n = (int)total;
      throw std::out_of_range("cryo_slabs_download: arrays too small");
    }
    o->n = (int)total;
    long long k = 0;
    auto put = [&](const Part& q, int i) {
      for (int a = 0; a < 3; ++a) {
        if (o->x) o->x[3 * k + a] = q.x[3 * (size_t)i + a];
        if (o->v) o->v[3 * k + a] = q.v[3 * (size_t)i + a];
        if (o->nrm) o->nrm[3 * k + a] = q.nrm[3 * (size_t)i + a];
      }
      if (o->m) o->m[k] = q.m[i];
      if (o->rho) o->rho[k] = q.rho[i];
      if (o->T) o->T[k] = q.T[i];
      if (o->phase) o->phase[k] = q.phase[i];
      if (o->flags) o->flags[k] = q.flags[i];
      if (o->id) o->id[k] = q.id[i];
      ++k;
    };
    for (const Part& q : parts)
      for (int i = q.lo; i < q.hi; ++i) put(q, i);
    for (const Part& q : parts)
      for (int i = q.ns; i < q.n; ++i) put(q, i);
  });
}

// Solver::diagnostics of the whole tank: each slab's owned sums (added in
// slab order), maxima over the slabs, the shared scalar state of slab 0 and
// the per-slab counters added up.
int cryo_slabs_diagnostics(cryo_slabs* s, cryo_diagnostics_t* out) {
  return slab_guard(s, [&] {
    SlabGroup& G = *s->g;
    if (G.zb.empty()) throw std::runtime_error("Solver: no particles loaded");
    G.initialize();
    double v[44];
    long long owned = 0;
    for (int r = 0; r < G.count(); ++r) {
      cryo_ctx* c = G.slabs[r];
      CK(cudaSetDevice(c->device));
      k_diagnostics<<<c->grid_blocks(), kBlock, 0, c->stream>>>(c->P, c->view(c->cur), c->reduce(), c->diag_out);
      CK(cudaGetLastError());
      double* h = c->diag_host;
      CK(cudaMemcpyAsync(h, c->diag_out, 44 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      c->pull();  // also waits for the copy
      owned += (c->hdyn->own_hi - c->hdyn->own_lo) + (c->hdyn->n - c->hdyn->n_sorted);
      if (r == 0) {
        std::memcpy(v, h, sizeof(v));
        continue;
      }
      for (int k = 0; k < 23; ++k) v[k] += h[k];
      for (int k = 23; k < 25; ++k) v[k] = std::max(v[k], h[k]);
      for (int k : {30, 31, 32, 33, 36, 37}) v[k] += h[k];
    }
    v[28] = (double)owned;
    diag_fill(v, out);
  });
}

}  // extern "C"

