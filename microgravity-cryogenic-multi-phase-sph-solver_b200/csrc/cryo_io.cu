// cryo_io.cu -- particle transfers between host arrays and the cell-sorted
// device state, and the output frames, packed on the device.
//
// Host arrays cross in the structure-of-arrays layout of
// cryo_host_particles_t (x, v, nrm: 3 floats per particle; m, rho, T; id;
// phase, flags).  An upload copies the caller's arrays into one pinned host
// buffer, moves it with a single asynchronous copy and builds the float4
// records of the persistent state on the device (k_load_pack); a download
// runs the reverse (k_unload).  The buffers are the context's and grow on
// demand, so a reload of the same size allocates nothing.
//
// Frames (Solver::write_vtk / write_json of the reference, io.cpp:52-142 and
// telemetry.hpp:16-25): the device writes the file's binary payload -- the
// sections of a legacy VTK polydata file, byte-swapped to big-endian -- or
// the viewer's compacted arrays (walls left out on request, particle order
// kept); the host only adds the text framing (host/io.cpp).
#include "cryo_ctx.cuh"

namespace cryo {

// Offsets of the SoA sections inside one transfer buffer (256-byte aligned).
struct IoLayout {
  size_t x, v, nrm, m, rho, T, id, phase, flags, bytes;
};
inline IoLayout io_layout(size_t n) {
  auto r = [](size_t b) { return (b + 255) & ~size_t(255); };
  IoLayout L{};
  size_t o = 0;
  L.x = o; o += r(12 * n);
  L.v = o; o += r(12 * n);
  L.nrm = o; o += r(12 * n);
  L.m = o; o += r(4 * n);
  L.rho = o; o += r(4 * n);
  L.T = o; o += r(4 * n);
  L.id = o; o += r(4 * n);
  L.phase = o; o += r(n);
  L.flags = o; o += r(n);
  L.bytes = o;
  return L;
}

struct IoArrays {
  float *x, *v, *nrm, *m, *rho, *T;
  uint32_t* id;
  uint8_t *phase, *flags;
};
inline IoArrays io_arrays(char* base, const IoLayout& L) {
  return IoArrays{reinterpret_cast<float*>(base + L.x),   reinterpret_cast<float*>(base + L.v),
                  reinterpret_cast<float*>(base + L.nrm), reinterpret_cast<float*>(base + L.m),
                  reinterpret_cast<float*>(base + L.rho), reinterpret_cast<float*>(base + L.T),
                  reinterpret_cast<uint32_t*>(base + L.id), reinterpret_cast<uint8_t*>(base + L.phase),
                  reinterpret_cast<uint8_t*>(base + L.flags)};
}

// Which optional arrays an upload carries.
enum { IO_V = 1, IO_NRM = 2, IO_FLAGS = 4, IO_ID = 8 };

// Persistent records from the SoA upload (ParticleSystem::upload,
// particle_system.cpp:73-93): the transport velocity starts at v, m0 at m,
// the pressure and number density at 0; absent ids are the slot numbers.
__global__ void __launch_bounds__(kBlock) k_load_pack(int n, IoArrays a, int have, View V) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float m = a.m[i];
    float3 v = make_float3(0.f, 0.f, 0.f);
    if (have & IO_V) v = make_float3(a.v[3 * i], a.v[3 * i + 1], a.v[3 * i + 2]);
    V.xp[i] = make_float4(a.x[3 * i], a.x[3 * i + 1], a.x[3 * i + 2],
                          pack_pf(a.phase[i], (have & IO_FLAGS) ? a.flags[i] : 0));
    V.vT[i] = make_float4(v.x, v.y, v.z, a.T[i]);
    V.vt[i] = make_float4(v.x, v.y, v.z, m);
    V.nrm[i] = (have & IO_NRM) ? make_float4(a.nrm[3 * i], a.nrm[3 * i + 1], a.nrm[3 * i + 2], 0.f)
                               : make_float4(0.f, 0.f, 0.f, 0.f);
    V.mrps[i] = make_float4(m, a.rho[i], 0.f, 0.f);
    V.id[i] = (have & IO_ID) ? a.id[i] : (uint32_t)i;
  }
}

// The reverse: SoA arrays of the current persistent state (Solver::particles).
__global__ void __launch_bounds__(kBlock) k_unload(int n, View V, IoArrays a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 xp = V.xp[i], vT = V.vT[i], nr = V.nrm[i], mr = V.mrps[i];
    a.x[3 * i] = xp.x; a.x[3 * i + 1] = xp.y; a.x[3 * i + 2] = xp.z;
    a.v[3 * i] = vT.x; a.v[3 * i + 1] = vT.y; a.v[3 * i + 2] = vT.z;
    a.nrm[3 * i] = nr.x; a.nrm[3 * i + 1] = nr.y; a.nrm[3 * i + 2] = nr.z;
    a.m[i] = mr.x;
    a.rho[i] = mr.y;
    a.T[i] = vT.w;
    a.id[i] = V.id[i];
    a.phase[i] = (uint8_t)ph_of(xp);
    a.flags[i] = (uint8_t)fl_of(xp);
  }
}

// Big-endian 32-bit word (legacy VTK binary data is big-endian).
__device__ inline uint32_t be32(uint32_t w) { return __byte_perm(w, 0u, 0x0123); }
__device__ inline uint32_t be32f(float f) { return be32(__float_as_uint(f)); }

// The binary payload of the VTK file, section after section: POINTS (3
// words), VERTICES (the pair 1, i), SCALARS temperature, mass, density,
// phase, pressure (1 word each), VECTORS velocity (3 words).
__global__ void __launch_bounds__(kBlock) k_frame_vtk(int n, View V, uint32_t* __restrict__ out) {
  uint32_t* pts = out;
  uint32_t* verts = out + 3 * (size_t)n;
  uint32_t* temp = out + 5 * (size_t)n;
  uint32_t* mass = temp + n;
  uint32_t* dens = mass + n;
  uint32_t* phase = dens + n;
  uint32_t* pres = phase + n;
  uint32_t* vel = pres + n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 xp = V.xp[i], vT = V.vT[i], mr = V.mrps[i];
    pts[3 * i] = be32f(xp.x);
    pts[3 * i + 1] = be32f(xp.y);
    pts[3 * i + 2] = be32f(xp.z);
    verts[2 * i] = be32(1u);
    verts[2 * i + 1] = be32((uint32_t)i);
    temp[i] = be32f(vT.w);
    mass[i] = be32f(mr.x);
    dens[i] = be32f(mr.y);
    phase[i] = be32f((float)ph_of(xp));
    pres[i] = be32f(mr.z);
    vel[3 * i] = be32f(vT.x);
    vel[3 * i + 1] = be32f(vT.y);
    vel[3 * i + 2] = be32f(vT.z);
  }
}

// Viewer frame, pass 1: kept particles per chunk, then (last block) the
// exclusive scan of the chunk counts and the total.
__global__ void __launch_bounds__(kBlock) k_frame_count(int n, View V, Reduce R, int include_walls, int* total) {
  __shared__ double sh[kBlock / 32];
  const int nch = num_chunks(n);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    double cnt[1] = {0.0};
    if (i < n) cnt[0] = (include_walls || ph_of(V.xp[i]) != kWall) ? 1.0 : 0.0;
    publish_chunk<1>(R, c, cnt, sh);
  }
  if (last_block(R.ticket)) {
    const double t = block_exclusive_scan(R, 0, nch);
    if (threadIdx.x == 0) *total = (int)t;
  }
}

// Viewer frame, pass 2: each kept particle's slot = its chunk's offset plus
// its rank inside the chunk, so the order is the state's.
__global__ void __launch_bounds__(kBlock) k_frame_viewer(int n, View V, Reduce R, int include_walls,
                                                         float* __restrict__ pos, float* __restrict__ temp,
                                                         float* __restrict__ pres, float* __restrict__ speed,
                                                         uint8_t* __restrict__ phase) {
  __shared__ uint32_t warp_tot[kBlock / 32];
  const int nch = num_chunks(n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int i = c * kChunk + threadIdx.x;
    float4 xp = make_float4(0.f, 0.f, 0.f, 0.f);
    bool keep = false;
    if (i < n) {
      xp = V.xp[i];
      keep = include_walls || ph_of(xp) != kWall;
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_tot[warp] = __popc(ballot);
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += warp_tot[w];
    __syncthreads();
    if (!keep) continue;
    const int k = (int)__ldcg(R.partials + c) + (int)before + __popc(ballot & ((1u << lane) - 1u));
    const float4 vT = V.vT[i];
    pos[3 * k] = xp.x;
    pos[3 * k + 1] = xp.y;
    pos[3 * k + 2] = xp.z;
    temp[k] = vT.w;
    pres[k] = V.mrps[i].z;
    speed[k] = norm(xyz(vT));
    phase[k] = (uint8_t)ph_of(xp);
  }
}

}  // namespace cryo

// ------------------------------------------------------------- host side
namespace {

// Host copies between the caller's arrays and the pinned transfer buffer,
// cut into pieces of at most 1 MiB (of the destination) and spread over up to
// 8 host threads (one thread copies a few GB/s; the DMA engine moves far
// more).  A job with f64 set reads doubles and writes them rounded to float
// (bytes counts the float destination).
struct HostCopy {
  void* dst;
  const void* src;
  size_t bytes;
  bool f64 = false;
};
void copy_piece(const HostCopy& p) {
  if (!p.f64) {
    std::memcpy(p.dst, p.src, p.bytes);
    return;
  }
  float* d = static_cast<float*>(p.dst);
  const double* s = static_cast<const double*>(p.src);
  const size_t n = p.bytes / sizeof(float);
  for (size_t i = 0; i < n; ++i) d[i] = static_cast<float>(s[i]);
}
void copy_all(const std::vector<HostCopy>& jobs) {
  constexpr size_t kPiece = size_t(1) << 20;
  std::vector<HostCopy> pieces;
  size_t total = 0;
  for (const HostCopy& j : jobs) {
    total += j.f64 ? 2 * j.bytes : j.bytes;
    const size_t scale = j.f64 ? 2 : 1;
    for (size_t o = 0; o < j.bytes; o += kPiece)
      pieces.push_back({static_cast<char*>(j.dst) + o, static_cast<const char*>(j.src) + scale * o,
                        std::min(kPiece, j.bytes - o), j.f64});
  }
  const int np = static_cast<int>(pieces.size());
  if (total < (size_t(4) << 20)) {
    for (const HostCopy& p : pieces) copy_piece(p);
    return;
  }
#pragma omp parallel for schedule(dynamic, 1) num_threads(8)
  for (int k = 0; k < np; ++k) copy_piece(pieces[k]);
}

}  // namespace

void cryo_ctx::io_reserve(size_t bytes) {
  if (bytes <= io_cap) return;
  sync();
  if (io_dev) CK(cudaFree(io_dev));
  if (io_host) CK(cudaFreeHost(io_host));
  io_dev = nullptr;
  io_host = nullptr;
  io_cap = 0;
  const size_t want = bytes + bytes / 8;
  CK(cudaMalloc(&io_dev, want));
  CK(cudaHostAlloc(&io_host, want, cudaHostAllocDefault));
  io_cap = want;
}

extern "C" {

// Solver::set_particles (sph_solver.cu:407-428) + ParticleSystem::upload
// (particle_system.cpp:73-93), from columns of floats or doubles.
int cryo_set_particles_columns(cryo_ctx* c, const cryo_host_columns_t* p, const float* lo, const float* hi) {
  return guard(c, [&] {
    const int n = p->n;
    if (n <= 0) throw std::invalid_argument("Solver::set_particles: no particles");
    if (!p->x || !p->m || !p->rho || !p->T || !p->phase)
      throw std::invalid_argument("Solver::set_particles: x, m, rho, T and phase are required");
    bool vap = false;
    for (int i = 0; i < n; ++i) vap |= p->phase[i] == CRYO_VAPOR;
    uint32_t next_id = (uint32_t)n;
    if (p->id) {
      next_id = 0;
      for (int i = 0; i < n; ++i) next_id = std::max(next_id, p->id[i] + 1);
    }
    c->begin_load(n, vap, lo, hi);
    const IoLayout L = io_layout((size_t)n);
    c->io_reserve(L.bytes);
    char* h = c->io_host;
    const size_t N = (size_t)n;
    int have = 0;
    std::vector<HostCopy> jobs = {{h + L.x, p->x, 12 * N, p->x_f64 != 0},
                                  {h + L.m, p->m, 4 * N, p->m_f64 != 0},
                                  {h + L.rho, p->rho, 4 * N, p->rho_f64 != 0},
                                  {h + L.T, p->T, 4 * N, p->T_f64 != 0},
                                  {h + L.phase, p->phase, N}};
    if (p->v) { jobs.push_back({h + L.v, p->v, 12 * N, p->v_f64 != 0}); have |= IO_V; }
    if (p->nrm) { jobs.push_back({h + L.nrm, p->nrm, 12 * N, p->nrm_f64 != 0}); have |= IO_NRM; }
    if (p->flags) { jobs.push_back({h + L.flags, p->flags, N}); have |= IO_FLAGS; }
    if (p->id) { jobs.push_back({h + L.id, p->id, 4 * N}); have |= IO_ID; }
    copy_all(jobs);
    CK(cudaMemcpyAsync(c->io_dev, h, L.bytes, cudaMemcpyHostToDevice, c->stream));
    const int G = std::max(1, std::min((n + kBlock - 1) / kBlock, c->sm_count * 8));
    k_load_pack<<<G, kBlock, 0, c->stream>>>(n, io_arrays(c->io_dev, L), have, c->view(0));
    LAUNCH_CHECK();
    c->finish_load(n, next_id);  // synchronises: the pinned buffer is free again
  });
}

int cryo_set_particles(cryo_ctx* c, const cryo_host_particles_t* p, const float* lo, const float* hi) {
  const cryo_host_columns_t cols{p->n, p->x, p->v, p->nrm, p->m, p->rho, p->T, 0, 0, 0, 0, 0, 0,
                                 p->phase, p->flags, p->id};
  return cryo_set_particles_columns(c, &cols, lo, hi);
}

// Solver::particles (particle_system.cpp:95-101): the arrays the caller
// passes (null ones are skipped).
int cryo_download(cryo_ctx* c, cryo_host_particles_out_t* o) {
  return guard(c, [&] {
    c->pull();
    const int n = c->has_particles ? c->hdyn->n : 0;
    if (o->n < n) {
      o->n = n;
      throw std::out_of_range("cryo_download: arrays too small");
    }
    o->n = n;
    if (n == 0) return;
    const IoLayout L = io_layout((size_t)n);
    c->io_reserve(L.bytes);
    const int G = std::max(1, std::min((n + kBlock - 1) / kBlock, c->sm_count * 8));
    k_unload<<<G, kBlock, 0, c->stream>>>(n, c->view(c->cur), io_arrays(c->io_dev, L));
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(c->io_host, c->io_dev, L.bytes, cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    const char* h = c->io_host;
    const size_t N = (size_t)n;
    std::vector<HostCopy> jobs;
    if (o->x) jobs.push_back({o->x, h + L.x, 12 * N});
    if (o->v) jobs.push_back({o->v, h + L.v, 12 * N});
    if (o->nrm) jobs.push_back({o->nrm, h + L.nrm, 12 * N});
    if (o->m) jobs.push_back({o->m, h + L.m, 4 * N});
    if (o->rho) jobs.push_back({o->rho, h + L.rho, 4 * N});
    if (o->T) jobs.push_back({o->T, h + L.T, 4 * N});
    if (o->id) jobs.push_back({o->id, h + L.id, 4 * N});
    if (o->phase) jobs.push_back({o->phase, h + L.phase, N});
    if (o->flags) jobs.push_back({o->flags, h + L.flags, N});
    copy_all(jobs);
  });
}

int cryo_frame_vtk(cryo_ctx* c, void* out, size_t cap, int* count) {
  return guard(c, [&] {
    c->pull();
    const int n = c->has_particles ? c->hdyn->n : 0;
    if (count) *count = n;
    const size_t bytes = (size_t)n * CRYO_VTK_WORDS_PER_PARTICLE * 4;
    if (!out) return;  // size query
    if (cap < bytes) throw std::out_of_range("cryo_frame_vtk: buffer too small");
    if (n == 0) return;
    c->io_reserve(bytes);
    const int G = std::max(1, std::min((n + kBlock - 1) / kBlock, c->sm_count * 8));
    k_frame_vtk<<<G, kBlock, 0, c->stream>>>(n, c->view(c->cur), reinterpret_cast<uint32_t*>(c->io_dev));
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(c->io_host, c->io_dev, bytes, cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    std::memcpy(out, c->io_host, bytes);
  });
}

int cryo_frame_viewer(cryo_ctx* c, int include_walls, float* position, float* temperature, float* pressure,
                      float* speed, uint8_t* phase, int cap, int* count) {
  return guard(c, [&] {
    c->pull();
    const int n = c->has_particles ? c->hdyn->n : 0;
    if (!position || !temperature || !pressure || !speed || !phase)
      throw std::invalid_argument("cryo_frame_viewer: every output array is required");
    if (cap < n) {
      if (count) *count = n;
      throw std::out_of_range("cryo_frame_viewer: arrays must hold the particle count");
    }
    if (n == 0) {
      if (count) *count = 0;
      return;
    }
    // device layout: pos 3n, T n, p n, speed n (floats), phase n (bytes), count
    const size_t nf = (size_t)n;
    const size_t bytes = (6 * nf) * 4 + ((nf + 255) & ~size_t(255)) + 256;
    c->io_reserve(bytes);
    float* d = reinterpret_cast<float*>(c->io_dev);
    uint8_t* dph = reinterpret_cast<uint8_t*>(d + 6 * nf);
    int* dcount = reinterpret_cast<int*>(reinterpret_cast<char*>(c->io_dev) + bytes - 256);
    const int G = std::max(1, std::min((n + kChunk - 1) / kChunk, c->sm_count * 8));
    k_frame_count<<<G, kBlock, 0, c->stream>>>(n, c->view(c->cur), c->reduce(), include_walls, dcount);
    LAUNCH_CHECK();
    k_frame_viewer<<<G, kBlock, 0, c->stream>>>(n, c->view(c->cur), c->reduce(), include_walls, d, d + 3 * nf,
                                                d + 4 * nf, d + 5 * nf, dph);
    LAUNCH_CHECK();
    int k = 0;
    CK(cudaMemcpyAsync(c->io_host, c->io_dev, bytes, cudaMemcpyDeviceToHost, c->stream));
    c->sync();
    std::memcpy(&k, c->io_host + (bytes - 256), sizeof(int));
    const float* h = reinterpret_cast<const float*>(c->io_host);
    std::memcpy(position, h, 12 * (size_t)k);
    std::memcpy(temperature, h + 3 * nf, 4 * (size_t)k);
    std::memcpy(pressure, h + 4 * nf, 4 * (size_t)k);
    std::memcpy(speed, h + 5 * nf, 4 * (size_t)k);
    std::memcpy(phase, reinterpret_cast<const uint8_t*>(h + 6 * nf), (size_t)k);
    if (count) *count = k;
  });
}

}  // extern "C"
