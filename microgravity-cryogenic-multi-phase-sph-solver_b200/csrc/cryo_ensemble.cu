// cryo_ensemble.cu -- batched stepping of independent tanks: the ensemble
// (one graph launch advances every member by its own steps) and its extern
// "C" entry points (cryo_ensemble_*).
#include "cryo_ctx.cuh"

// ---------------------------------------------------------------------------
// Batched stepping of independent tanks (no counterpart in the reference).
// Each tank keeps its own context: arena, stream, parameters and step
// sequence.  A graph launch holds `per_launch` consecutive steps of every
// tank, each tank's steps a chain of that tank's own kernels, spread over
// `chains` concurrent branches (tanks assigned longest-processing-time first
// by particle count; one branch per tank by default).  Tanks far too small
// to fill the GPU alone then run side by side, and several steps per launch
// spare the drain at every launch boundary.  Every tank runs exactly the
// kernels, launch shapes and arguments of its own step graph, so its results
// are those of stepping it alone, bit for bit.
struct cryo_ensemble {
  struct Graphs {  // one launch shape: `steps` steps from either parity
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int steps = 0;
    void drop() {
      for (int k = 0; k < 2; ++k) {
        if (exec[k]) cudaGraphExecDestroy(exec[k]);
        exec[k] = nullptr;
      }
      steps = 0;
    }
  };
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr, t0 = nullptr, t1 = nullptr;
  std::vector<cryo_ctx*> tanks;
  int chains = 0;      // 0: one branch per tank
  int per_launch = 1;  // steps per graph launch (divides 16)
  int tile = 1;        // particles per thread of the members' grid-stride kernels
  int built_tile = 0;
  Graphs multi, single;
  std::vector<int> built_cur;  // each tank's ping-pong parity when the graphs were built
  std::vector<unsigned long long> built_gen;
  int built_chains = -1;
  int phase = 0;  // steps taken since the build, mod 2
  int step_launches = 0;
  long long steps_run = 0;
  std::string err;

  ~cryo_ensemble() {
    if (stream) cudaStreamSynchronize(stream);
    drop();
    for (cryo_ctx* c : tanks) c->ensemble = nullptr;
    for (cudaEvent_t e : {fork, done, t0, t1})
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
  void drop() {
    multi.drop();
    single.drop();
    built_chains = -1;
  }
  int branches() const {
    const int t = (int)tanks.size();
    return chains <= 0 ? t : std::min(chains, t);
  }
  bool valid() const {
    if (built_chains != branches() || multi.steps != per_launch || built_tile != tile) return false;
    for (size_t t = 0; t < tanks.size(); ++t)
      if (tanks[t]->generation != built_gen[t] || tanks[t]->cur != ((built_cur[t] + phase) & 1)) return false;
    return true;
  }
  // Tanks per branch: largest first, each to the least-loaded branch.
  std::vector<std::vector<int>> plan() const {
    const int k = branches();
    std::vector<int> order(tanks.size());
    for (size_t t = 0; t < tanks.size(); ++t) order[t] = (int)t;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return tanks[a]->hdyn->n > tanks[b]->hdyn->n; });
    std::vector<std::vector<int>> out(k);
    std::vector<long long> load(k, 0);
    for (int t : order) {
      int best = 0;
      for (int b = 1; b < k; ++b)
        if (load[b] < load[best]) best = b;
      out[best].push_back(t);
      load[best] += std::max(tanks[t]->hdyn->n, 1);
    }
    return out;
  }
  // `steps` steps of every tank starting at parity offset q, as one graph.
  void capture(int q, int steps, const std::vector<std::vector<int>>& branches_plan, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    int launches = 0;
    try {
      CK(cudaEventRecord(fork, stream));
      for (const auto& br : branches_plan) {
        cudaEvent_t prev = fork;
        for (int t : br) {
          cryo_ctx* c = tanks[t];
          CK(cudaStreamWaitEvent(c->stream, prev, 0));
          // the member's kernels at the ensemble's tile (its own step graphs keep theirs)
          struct TileScope {
            cryo_ctx* c;
            int saved;
            ~TileScope() { c->grid_tile = saved; }
          } scope{c, c->grid_tile};
          c->grid_tile = tile;
          for (int k = 0; k < steps; ++k) {
            const long long c0 = c->launch_counter;
            c->enqueue_step((built_cur[t] + q + k) & 1);
            launches += (int)(c->launch_counter - c0);
          }
          CK(cudaEventRecord(c->ens_ev, c->stream));
          prev = c->ens_ev;
        }
      }
      for (cryo_ctx* c : tanks) CK(cudaStreamWaitEvent(stream, c->ens_ev, 0));
    } catch (...) {
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CK(cudaStreamEndCapture(stream, &g));
    const cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    step_launches = launches / std::max(steps, 1);
  }
  // Graphs for both start parities (a run can reach either before a launch).
  void build_shape(Graphs& gr, int steps, const std::vector<std::vector<int>>& pl) {
    gr.drop();
    capture(0, steps, pl, &gr.exec[0]);
    capture(1, steps, pl, &gr.exec[1]);
    gr.steps = steps;
  }
  void build() {
    drop();
    leave();
    for (cryo_ctx* c : tanks) {  // particle counts for the plan and the launch grids
      c->pull();
      c->size_grids();
    }
    enter();
    built_cur.resize(tanks.size());
    built_gen.resize(tanks.size());
    for (size_t t = 0; t < tanks.size(); ++t) {
      built_cur[t] = tanks[t]->cur;
      built_gen[t] = tanks[t]->generation;
    }
    phase = 0;
    const auto pl = plan();
    build_shape(multi, per_launch, pl);
    if (per_launch > 1) build_shape(single, 1, pl);
    built_chains = branches();
    built_tile = tile;
  }
  // tank streams -> ensemble stream, and back
  void enter() {
    for (cryo_ctx* c : tanks) {
      CK(cudaEventRecord(c->ens_ev, c->stream));
      CK(cudaStreamWaitEvent(stream, c->ens_ev, 0));
    }
  }
  void leave() {
    CK(cudaEventRecord(done, stream));
    for (cryo_ctx* c : tanks) CK(cudaStreamWaitEvent(c->stream, done, 0));
  }
  void prepare() {
    for (cryo_ctx* c : tanks) {
      if (c->profiling) throw std::invalid_argument("ensemble: a tank has per-kernel profiling on");
      c->ensure_initialized();
    }
  }
  // One launch of `steps` (per_launch or 1) steps of every tank.
  void launch(int steps) {
    const Graphs& gr = (steps == per_launch) ? multi : single;
    CK(cudaGraphLaunch(gr.exec[phase], stream));
    phase = (phase + steps) & 1;
    for (cryo_ctx* c : tanks) c->cur = (c->cur + steps) & 1;
    steps_run += steps;
  }
  // Head-room for splits, per tank, between steps (sph_solver.cu:556-560).
  void check_capacity() {
    leave();
    for (cryo_ctx* c : tanks) c->check_capacity();
  }
  void run(long long n) {
    if (tanks.empty() || n <= 0) return;
    prepare();
    enter();
    long long since_check = 0;
    while (n > 0) {
      if (!valid()) build();
      const int k = n >= per_launch ? per_launch : 1;
      launch(k);
      n -= k;
      since_check += k;
      if (since_check >= 16 && n > 0) {
        check_capacity();
        enter();
        since_check = 0;
      }
    }
    check_capacity();
  }
  // Device time per step over `steps` steps (rounded up to whole launches)
  // with the current shape, after one untimed launch that also builds it.
  float time_steps(int steps) {
    run(per_launch);
    enter();
    if (!valid()) build();
    const int launches = std::max(1, (steps + per_launch - 1) / per_launch);
    CK(cudaEventRecord(t0, stream));
    for (int k = 0; k < launches; ++k) launch(per_launch);
    CK(cudaEventRecord(t1, stream));
    check_capacity();
    CK(cudaEventSynchronize(t1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, t0, t1));
    return ms / (float)(launches * per_launch);
  }
};

void ensemble_detach(cryo_ensemble* e, cryo_ctx* c) {
  cudaStreamSynchronize(e->stream);
  e->drop();
  e->tanks.erase(std::remove(e->tanks.begin(), e->tanks.end(), c), e->tanks.end());
  c->ensemble = nullptr;
}

namespace {
template <class F>
int eguard(cryo_ensemble* e, F&& f) {
  try {
    f();
    return CRYO_OK;
  } catch (const std::invalid_argument& x) {
    if (e) e->err = x.what(); else g_create_error = x.what();
    return CRYO_EINVAL;
  } catch (const std::out_of_range& x) {
    if (e) e->err = x.what(); else g_create_error = x.what();
    return CRYO_ERANGE;
  } catch (const CudaError& x) {
    if (e) e->err = x.what(); else g_create_error = x.what();
    return CRYO_ECUDA;
  } catch (const std::exception& x) {
    if (e) e->err = x.what(); else g_create_error = x.what();
    return CRYO_ERUNTIME;
  }
}
}  // namespace
extern "C" {

int cryo_ensemble_create(int device, cryo_ensemble** out) {
  *out = nullptr;
  cryo_ensemble* e = nullptr;
  const int rc = eguard(nullptr, [&] {
    e = new cryo_ensemble;
    try {
      e->device = device;
      CK(cudaSetDevice(device));
      CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamDefault));
      CK(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming));
      CK(cudaEventCreate(&e->t0));
      CK(cudaEventCreate(&e->t1));
    } catch (...) {
      delete e;
      e = nullptr;
      throw;
    }
  });
  *out = e;
  return rc;
}

void cryo_ensemble_destroy(cryo_ensemble* e) { delete e; }

const char* cryo_ensemble_last_error(const cryo_ensemble* e) { return e ? e->err.c_str() : g_create_error.c_str(); }

int cryo_ensemble_add(cryo_ensemble* e, cryo_ctx* c) {
  return eguard(e, [&] {
    if (!c) throw std::invalid_argument("ensemble: null tank");
    if (c->ensemble) throw std::invalid_argument("ensemble: the tank already belongs to an ensemble");
    if (c->device != e->device) throw std::invalid_argument("ensemble: the tank lives on another device");
    if (!c->has_particles) throw std::invalid_argument("ensemble: the tank has no particles");
    if (!c->ens_ev) CK(cudaEventCreateWithFlags(&c->ens_ev, cudaEventDisableTiming));
    CK(cudaStreamSynchronize(e->stream));
    e->drop();
    e->tanks.push_back(c);
    c->ensemble = e;
  });
}

int cryo_ensemble_remove(cryo_ensemble* e, cryo_ctx* c) {
  return eguard(e, [&] {
    if (!c || c->ensemble != e) throw std::invalid_argument("ensemble: the tank is not a member");
    ensemble_detach(e, c);
  });
}

int cryo_ensemble_size(cryo_ensemble* e, int* tanks) {
  return eguard(e, [&] { *tanks = (int)e->tanks.size(); });
}

int cryo_ensemble_set_chains(cryo_ensemble* e, int chains) {
  return eguard(e, [&] {
    if (chains < 0) throw std::invalid_argument("ensemble: chains must be >= 0");
    e->chains = chains;
  });
}

int cryo_ensemble_chains(cryo_ensemble* e, int* chains) {
  return eguard(e, [&] { *chains = e->branches(); });
}

int cryo_ensemble_set_steps_per_launch(cryo_ensemble* e, int steps) {
  return eguard(e, [&] {
    if (steps < 1 || steps > 16 || (16 % steps) != 0)
      throw std::invalid_argument("ensemble: steps per launch must be 1, 2, 4, 8 or 16");
    e->per_launch = steps;
  });
}

int cryo_ensemble_steps_per_launch(cryo_ensemble* e, int* steps) {
  return eguard(e, [&] { *steps = e->per_launch; });
}

int cryo_ensemble_run_steps(cryo_ensemble* e, long long n) {
  return eguard(e, [&] { e->run(n); });
}

int cryo_ensemble_step_time(cryo_ensemble* e, int steps, float* ms_per_step) {
  return eguard(e, [&] {
    if (steps <= 0) throw std::invalid_argument("ensemble: steps must be > 0");
    *ms_per_step = e->tanks.empty() ? 0.0f : e->time_steps(steps);
  });
}

int cryo_ensemble_set_tile(cryo_ensemble* e, int particles_per_thread) {
  return eguard(e, [&] {
    if (particles_per_thread < 1 || particles_per_thread > 64)
      throw std::invalid_argument("ensemble: the tile must be 1 to 64 particles per thread");
    e->tile = particles_per_thread;
  });
}

int cryo_ensemble_tile(cryo_ensemble* e, int* particles_per_thread) {
  return eguard(e, [&] { *particles_per_thread = e->tile; });
}

// The tuner of cryo_ensemble_tune over a third axis: the members' tile
// (particles per thread of their grid-stride kernels).
int cryo_ensemble_tune_tiles(cryo_ensemble* e, const int* chain_candidates, int nchain, const int* launch_candidates,
                             int nlaunch, const int* tile_candidates, int ntile, int steps, int* best_chains,
                             int* best_steps_per_launch, int* best_tile, float* best_ms) {
  return eguard(e, [&] {
    std::vector<int> tc;
    if (tile_candidates && ntile > 0) tc.assign(tile_candidates, tile_candidates + ntile);
    else tc.push_back(e->tile);
    for (int k : tc)
      if (k < 1 || k > 64) throw std::invalid_argument("ensemble: tiles must be 1 to 64 particles per thread");
    int bc = 0, bl = 1, bt = tc[0];
    float bm = 0.0f;
    bool any = false;
    for (int k : tc) {
      e->tile = k;
      int c = 0, l = 1;
      float ms = 0.0f;
      const int rc = cryo_ensemble_tune(e, chain_candidates, nchain, launch_candidates, nlaunch, steps, &c, &l, &ms);
      if (rc != CRYO_OK) throw std::runtime_error(e->err);
      if (!any || ms < bm) {
        any = true;
        bc = c; bl = l; bt = k; bm = ms;
      }
    }
    e->chains = bc;
    e->per_launch = bl;
    e->tile = bt;
    if (best_chains) *best_chains = bc;
    if (best_steps_per_launch) *best_steps_per_launch = bl;
    if (best_tile) *best_tile = bt;
    if (best_ms) *best_ms = bm;
  });
}

int cryo_ensemble_tune(cryo_ensemble* e, const int* chain_candidates, int nchain, const int* launch_candidates,
                       int nlaunch, int steps, int* best_chains, int* best_steps_per_launch, float* best_ms) {
  return eguard(e, [&] {
    if (steps <= 0) throw std::invalid_argument("ensemble: steps must be > 0");
    const int t = (int)e->tanks.size();
    if (t == 0) throw std::invalid_argument("ensemble: no tanks");
    std::vector<int> cc, lc;
    if (chain_candidates && nchain > 0) cc.assign(chain_candidates, chain_candidates + nchain);
    else for (int k = t; k >= 1; k /= 2) cc.push_back(k);
    if (launch_candidates && nlaunch > 0) lc.assign(launch_candidates, launch_candidates + nlaunch);
    else lc.push_back(e->per_launch);
    for (int k : cc)
      if (k < 0) throw std::invalid_argument("ensemble: chain counts must be >= 0");
    for (int k : lc)
      if (k < 1 || k > 16 || (16 % k) != 0)
        throw std::invalid_argument("ensemble: steps per launch must be 1, 2, 4, 8 or 16");
    int best_c = -1, best_l = 1;
    float best_t = 0.0f;
    for (int l : lc)
      for (int k : cc) {
        e->chains = k;
        e->per_launch = l;
        const float ms = e->time_steps(steps);
        if (best_c < 0 || ms < best_t) {
          best_c = k;
          best_l = l;
          best_t = ms;
        }
      }
    e->chains = best_c;
    e->per_launch = best_l;
    if (best_chains) *best_chains = best_c;
    if (best_steps_per_launch) *best_steps_per_launch = best_l;
    if (best_ms) *best_ms = best_t;
  });
}

int cryo_ensemble_launches_per_step(cryo_ensemble* e, int* launches) {
  return eguard(e, [&] { *launches = e->step_launches; });
}

int cryo_ensemble_synchronize(cryo_ensemble* e) {
  return eguard(e, [&] { CK(cudaStreamSynchronize(e->stream)); });
}

uintptr_t cryo_ensemble_stream(const cryo_ensemble* e) { return reinterpret_cast<uintptr_t>(e->stream); }

}  // extern "C"

