// C ABI implementation (include/u1_b200.h): context, lattice, RNG, update,
// measurements, Polyakov correlator and multilevel orchestration.
//
// Host orchestration being replaced:
//   SetupLatticeParameters  reference src/parameters.cu:146-208
//   UpdateLattice           reference src/update.cu:449-456 (+ :301-316, :379-394)
//   Plaquette / Polyakov    reference src/plaquette.cu:169-187,222-228; src/polyakov.cu:124-139,169-174
//   Poly2                   reference src/polyakov.cu:618-654
//   MultiLevel              reference src/multilevel.cu:639-732
// Differences by design: no globals (geometry lives in the lattice handle),
// status codes instead of exit(), explicit streams, no per-op device
// synchronisation except where a host result is returned, and whole sweeps
// replayed as CUDA graphs.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "u1_internal.h"
#include "u1_fused.cuh"
#include "u1_wave.cuh"
#include "u1_multilevel.cuh"

using namespace u1b;

namespace u1i {
static thread_local std::string g_err;
std::atomic<unsigned long long> g_launches{0};
static std::atomic<unsigned long long> g_rng_ids{1};

void set_error(const std::string &msg) { g_err = msg; }
int cuda_fail(cudaError_t e, const char *what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? U1_ERR_NOMEM : U1_ERR_CUDA;
}

// The device allocator (u1_set_device_allocator).  live_allocs counts the
// blocks handed out through dev_alloc and not yet returned, so the allocator
// is never swapped while the library holds memory from the previous one.
struct DevAllocator {
  u1_dev_alloc_fn alloc = nullptr;
  u1_dev_free_fn release = nullptr;
  void *user = nullptr;
};
static std::mutex g_alloc_mu;
static DevAllocator g_alloc;
static std::atomic<long long> g_live_allocs{0};

cudaError_t time_graph_min(cudaGraphExec_t ex, cudaStream_t s, int warm, int reps, double *us) {
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < warm && e == cudaSuccess; ++k) e = cudaGraphLaunch(ex, s);
  std::vector<cudaEvent_t> ev(2 * (size_t)reps, nullptr);
  for (size_t k = 0; k < ev.size() && e == cudaSuccess; ++k) e = cudaEventCreate(&ev[k]);
  for (int r = 0; r < reps && e == cudaSuccess; ++r) {
    e = cudaEventRecord(ev[2 * r], s);
    if (e == cudaSuccess) e = cudaGraphLaunch(ex, s);
    if (e == cudaSuccess) e = cudaEventRecord(ev[2 * r + 1], s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  double best = -1.0;
  for (int r = 0; r < reps && e == cudaSuccess; ++r) {
    float ms = 0.f;
    e = cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]);
    if (e == cudaSuccess && (best < 0.0 || ms < best)) best = ms;
  }
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  *us = 1e3 * best;
  return e;
}

cudaError_t warm_clocks(cudaGraphExec_t ex, cudaStream_t s, double ms) {
  double us = 0.0;
  cudaError_t e = time_graph_min(ex, s, 0, 1, &us);
  const int n = us > 0.0 ? (int)std::min(2000.0, 1e3 * ms / us) : 0;
  for (int k = 0; k < n && e == cudaSuccess; ++k) e = cudaGraphLaunch(ex, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

bool tune_verbose() {
  static const bool v = [] {
    const char *e = std::getenv("U1_TUNE_VERBOSE");
    return e && e[0] == '1';
  }();
  return v;
}

cudaError_t dev_alloc(void **p, size_t bytes) {
  *p = nullptr;
  DevAllocator a;
  {
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    a = g_alloc;
  }
  cudaError_t e;
  if (a.alloc)
    e = (a.alloc(a.user, bytes, p) == 0 && *p) ? cudaSuccess : cudaErrorMemoryAllocation;
  else
    e = cudaMalloc(p, bytes);
  if (e == cudaSuccess)
    g_live_allocs.fetch_add(1, std::memory_order_relaxed);
  else
    *p = nullptr;
  return e;
}

cudaError_t dev_free(void *p) {
  if (!p) return cudaSuccess;
  DevAllocator a;
  {
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    a = g_alloc;
  }
  g_live_allocs.fetch_sub(1, std::memory_order_relaxed);
  if (a.release) {
    // cudaFree waits for the device; a caller's pool gets the same guarantee:
    // no work of this library still uses the block when it is returned
    cudaError_t e = cudaDeviceSynchronize();
    a.release(a.user, p);
    return e;
  }
  return cudaFree(p);
}
static int fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

int ensure_scratch(u1_lattice *lat, size_t partial_doubles, size_t out_doubles) {
  if (partial_doubles > lat->partials_cap) {
    // cached sweep graphs hold the old scratch pointers
    cudaStreamSynchronize(lat->stream);
    for (auto &kv : lat->graphs) cudaGraphExecDestroy(kv.second);
    lat->graphs.clear();
    if (lat->partials) u1i::dev_free(lat->partials);
    lat->partials = nullptr;
    lat->partials_cap = 0;
    U1_CUDA_TRY(u1i::dev_alloc(&lat->partials, partial_doubles * sizeof(double)));
    lat->partials_cap = partial_doubles;
  }
  if (!lat->counter) {
    U1_CUDA_TRY(u1i::dev_alloc(&lat->counter, sizeof(unsigned int)));
    U1_CUDA_TRY(cudaMemset(lat->counter, 0, sizeof(unsigned int)));
  }
  if (out_doubles > lat->d_out_cap) {
    if (lat->d_out) u1i::dev_free(lat->d_out);
    if (lat->h_out) cudaFreeHost(lat->h_out);
    lat->d_out = nullptr;
    lat->h_out = nullptr;
    lat->d_out_cap = lat->h_out_cap = 0;
    U1_CUDA_TRY(u1i::dev_alloc(&lat->d_out, out_doubles * sizeof(double)));
    U1_CUDA_TRY(cudaMallocHost(&lat->h_out, out_doubles * sizeof(double)));
    lat->d_out_cap = lat->h_out_cap = out_doubles;
  }
  return U1_OK;
}

static inline int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

}  // namespace u1i

using u1i::fail;

extern "C" const char *u1_last_error(void) { return u1i::g_err.c_str(); }
extern "C" const char *u1_version(void) { return "latticeu1_b200 0.1 (sm_100a)"; }

extern "C" int u1_kernel_launch_count(uint64_t *out) {
  if (!out) return fail(U1_ERR_INVALID, "u1_kernel_launch_count: null out");
  *out = u1i::g_launches.load();
  return U1_OK;
}

extern "C" int u1_set_device_allocator(u1_dev_alloc_fn alloc, u1_dev_free_fn release, void *user) {
  using namespace u1i;
  if ((alloc == nullptr) != (release == nullptr))
    return fail(U1_ERR_INVALID, "u1_set_device_allocator: give both functions or neither");
  std::lock_guard<std::mutex> lock(g_alloc_mu);
  const long long live = g_live_allocs.load();
  if (live != 0)
    return fail(U1_ERR_STATE, "u1_set_device_allocator: the library still holds " + std::to_string(live) +
                                  " device allocations from the current allocator");
  g_alloc.alloc = alloc;
  g_alloc.release = release;
  g_alloc.user = user;
  return U1_OK;
}

extern "C" int u1_device_allocations(int64_t *live) {
  if (!live) return fail(U1_ERR_INVALID, "u1_device_allocations: null argument");
  *live = u1i::g_live_allocs.load();
  return U1_OK;
}

// ---------------------------------------------------------------- context
extern "C" int u1_ctx_create(int device, u1_ctx **out) {
  if (!out) return fail(U1_ERR_INVALID, "u1_ctx_create: null out");
  *out = nullptr;
  int n = 0;
  U1_CUDA_TRY(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n)
    return fail(U1_ERR_INVALID, "u1_ctx_create: device " + std::to_string(device) + " out of range (" +
                                    std::to_string(n) + " devices)");
  U1_CUDA_TRY(cudaSetDevice(device));
  u1_ctx *ctx = new u1_ctx;
  ctx->device = device;
  cudaError_t e = cudaGetDeviceProperties(&ctx->prop, device);
  if (e != cudaSuccess) {
    delete ctx;
    return u1i::cuda_fail(e, "cudaGetDeviceProperties");
  }
  if (ctx->prop.major != 10) {
    std::string msg = std::string("u1_ctx_create: this library is built for sm_100a (B200); device is ") +
                      ctx->prop.name + " sm_" + std::to_string(ctx->prop.major) + std::to_string(ctx->prop.minor);
    delete ctx;
    return fail(U1_ERR_UNSUPPORTED, msg);
  }
  *out = ctx;
  return U1_OK;
}

extern "C" int u1_ctx_destroy(u1_ctx *ctx) {
  if (!ctx) return U1_OK;
  if (ctx->chk) {
    cudaSetDevice(ctx->device);
    u1i::dev_free(ctx->chk);
  }
  delete ctx;
  return U1_OK;
}

extern "C" int u1_ctx_set_stream(u1_ctx *ctx, void *stream) {
  if (!ctx) return fail(U1_ERR_INVALID, "u1_ctx_set_stream: null ctx");
  ctx->stream = (cudaStream_t)stream;
  return U1_OK;
}

// ---------------------------------------------------------------- lattice
namespace u1i {
int make_geom(const u1_geom *gm, GeomK &g) {
  if (!gm) return fail(U1_ERR_INVALID, "geometry: null");
  const int d = gm->dims;
  if (d < 2 || d > 4) return fail(U1_ERR_INVALID, "geometry: dims must be 2, 3 or 4");
  int Grid[4] = {1, 1, 1, 1};
  const int Nx = gm->N[0], Ny = gm->N[1], Nz = gm->N[2], Nt = gm->N[3];
  Grid[0] = Nx;
  if (d == 2) Grid[1] = Nt;
  else Grid[1] = Ny;
  if (d == 3) Grid[2] = Nt;
  else if (d > 3) Grid[2] = Nz;
  if (d == 4) Grid[3] = Nt;
  long long V = 1;
  for (int k = 0; k < d; ++k) {
    if (Grid[k] < 2 || (Grid[k] % 2) != 0)
      return fail(U1_ERR_INVALID, "geometry: every extent must be even and >= 2 (got " +
                                      std::to_string(Grid[k]) + " in direction " + std::to_string(k) + ")");
    V *= Grid[k];
  }
  if (V * d > (1LL << 31)) return fail(U1_ERR_UNSUPPORTED, "geometry: V*dims exceeds 2^31 links");
  g = GeomK{};
  g.dims = d;
  for (int k = 0; k < 4; ++k) g.N[k] = Grid[k];
  geom_finish(g);
  return U1_OK;
}
}  // namespace u1i

using u1i::make_geom;

extern "C" int u1_geom_validate(const u1_geom *geom, int64_t out[8]) {
  GeomK g{};
  int rc = make_geom(geom, g);
  if (rc) return rc;
  if (!(geom->aniso > 0.0)) return fail(U1_ERR_INVALID, "geometry: aniso must be > 0");
  if (out) {
    out[0] = g.V;
    out[1] = g.Vh;
    out[2] = g.Vs;
    out[3] = g.dims;
    for (int k = 0; k < 4; ++k) out[4 + k] = g.N[k];
  }
  return U1_OK;
}

static void set_coupling(u1_lattice *lat, double beta, double aniso) {
  lat->beta = beta;
  lat->aniso = aniso;
  lat->c.beta = (float)beta;
  lat->c.w_ss = (float)(1.0 / aniso);
  lat->c.w_st = (float)aniso;
}

static void drop_graphs(u1_lattice *lat) {
  for (auto &kv : lat->graphs) cudaGraphExecDestroy(kv.second);
  lat->graphs.clear();
  if (lat->ml_g4) cudaGraphExecDestroy(lat->ml_g4);
  if (lat->ml_g2) cudaGraphExecDestroy(lat->ml_g2);
  lat->ml_g4 = lat->ml_g2 = nullptr;
  lat->ml_key = std::make_tuple(-1, -1, -1, -1, (uint64_t)0, (uint64_t)0);
}

extern "C" int u1_lattice_create(u1_ctx *ctx, const u1_geom *geom, u1_lattice **out) {
  if (!ctx || !out) return fail(U1_ERR_INVALID, "u1_lattice_create: null argument");
  *out = nullptr;
  GeomK g{};
  int rc = make_geom(geom, g);
  if (rc) return rc;
  if (!(geom->aniso > 0.0)) return fail(U1_ERR_INVALID, "u1_lattice_create: aniso must be > 0");
  U1_CUDA_TRY(cudaSetDevice(ctx->device));
  u1_lattice *lat = new u1_lattice;
  lat->ctx = ctx;
  lat->g = g;
  set_coupling(lat, geom->beta, geom->aniso);
  cudaError_t e = cudaStreamCreate(&lat->own_stream);
  if (e != cudaSuccess) {
    delete lat;
    return u1i::cuda_fail(e, "cudaStreamCreate");
  }
  lat->stream = ctx->stream ? ctx->stream : lat->own_stream;
  const size_t nl = (size_t)g.V * g.dims;
  e = u1i::dev_alloc(&lat->links, nl * sizeof(float2));
  if (e != cudaSuccess) {
    u1_lattice_destroy(lat);
    u1i::set_error(std::string("u1_lattice_create: link allocation: ") + cudaGetErrorString(e));
    return U1_ERR_NOMEM;
  }
#ifdef U1_BOUNDS_CHECK
  lat->shadow = u1i::chk_shadow(nl);
  if (!lat->shadow || !u1i::chk_state(ctx)) {
    u1_lattice_destroy(lat);
    return fail(U1_ERR_NOMEM, "u1_lattice_create: no device memory for the access checks");
  }
#endif
  rc = u1_cold_start(lat);
  if (rc) {
    u1_lattice_destroy(lat);
    return rc;
  }
  *out = lat;
  return U1_OK;
}

extern "C" int u1_lattice_destroy(u1_lattice *lat) {
  if (!lat) return U1_OK;
  cudaSetDevice(lat->ctx->device);
  cudaStreamSynchronize(lat->stream);
  drop_graphs(lat);
  if (lat->links) u1i::dev_free(lat->links);
  if (lat->partials) u1i::dev_free(lat->partials);
  if (lat->counter) u1i::dev_free(lat->counter);
  if (lat->d_out) u1i::dev_free(lat->d_out);
  if (lat->h_out) cudaFreeHost(lat->h_out);
  if (lat->pfield) u1i::dev_free(lat->pfield);
  if (lat->stage) u1i::dev_free(lat->stage);
  if (lat->backup) u1i::dev_free(lat->backup);
  if (lat->wave_state) u1i::dev_free(lat->wave_state);
  u1i::dev_free(lat->ml_work);
  u1i::dev_free(lat->ml_P2);
  u1i::dev_free(lat->ml_T2);
  u1i::dev_free(lat->ml_T4);
  u1i::dev_free(lat->shadow);
  if (lat->own_stream) cudaStreamDestroy(lat->own_stream);
  delete lat;
  return U1_OK;
}

extern "C" int u1_lattice_set_stream(u1_lattice *lat, void *stream) {
  if (!lat) return fail(U1_ERR_INVALID, "u1_lattice_set_stream: null lattice");
  lat->stream = stream ? (cudaStream_t)stream : lat->own_stream;
  return U1_OK;
}

extern "C" int u1_lattice_info(const u1_lattice *lat, int64_t out[8]) {
  if (!lat || !out) return fail(U1_ERR_INVALID, "u1_lattice_info: null argument");
  out[0] = lat->g.V;
  out[1] = lat->g.Vh;
  out[2] = lat->g.Vs;
  out[3] = lat->g.dims;
  for (int k = 0; k < 4; ++k) out[4 + k] = lat->g.N[k];
  return U1_OK;
}

extern "C" int u1_lattice_set_coupling(u1_lattice *lat, double beta, double aniso) {
  if (!lat) return fail(U1_ERR_INVALID, "u1_lattice_set_coupling: null lattice");
  if (!(aniso > 0.0)) return fail(U1_ERR_INVALID, "u1_lattice_set_coupling: aniso must be > 0");
  set_coupling(lat, beta, aniso);
  drop_graphs(lat);
  return U1_OK;
}

extern "C" int u1_lattice_set_graphs(u1_lattice *lat, int enable) {
  if (!lat) return fail(U1_ERR_INVALID, "u1_lattice_set_graphs: null lattice");
  lat->use_graphs = enable != 0;
  if (!lat->use_graphs) drop_graphs(lat);
  return U1_OK;
}

extern "C" int u1_lattice_links(u1_lattice *lat, void **dev_ptr) {
  if (!lat || !dev_ptr) return fail(U1_ERR_INVALID, "u1_lattice_links: null argument");
  *dev_ptr = lat->links;
  return U1_OK;
}

extern "C" int u1_lattice_copy(u1_lattice *dst, const u1_lattice *src) {
  if (!dst || !src) return fail(U1_ERR_INVALID, "u1_lattice_copy: null argument");
  if (memcmp(dst->g.N, src->g.N, sizeof(dst->g.N)) != 0 || dst->g.dims != src->g.dims)
    return fail(U1_ERR_INVALID, "u1_lattice_copy: geometry mismatch");
  U1_CUDA_TRY(cudaSetDevice(dst->ctx->device));
  U1_CUDA_TRY(cudaMemcpyAsync(dst->links, src->links, (size_t)src->g.V * src->g.dims * sizeof(float2),
                              cudaMemcpyDeviceToDevice, dst->stream));
  return U1_OK;
}

extern "C" int u1_cold_start(u1_lattice *lat) {
  if (!lat) return fail(U1_ERR_INVALID, "u1_cold_start: null lattice");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  const size_t n = (size_t)lat->g.V * lat->g.dims;
  k_fill_links<<<u1i::blocks_for((long long)n, 256), 256, 0, lat->stream>>>(lat->links, n,
                                                                            make_float2(1.f, 0.f));
  U1_LAUNCH_CHECK("k_fill_links");
  return U1_OK;
}

static int ensure_stage(u1_lattice *lat) {
  if (!lat->stage) U1_CUDA_TRY(u1i::dev_alloc(&lat->stage, (size_t)lat->g.V * lat->g.dims * sizeof(double)));
  return U1_OK;
}

// Import (angles -> float2 links) queued on the lattice's stream; `wait`:
// return only once it has completed.
static int import_angles(u1_lattice *lat, const double *angles, int on_device, bool wait) {
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  const size_t n = (size_t)lat->g.V * lat->g.dims;
  const double *src = angles;
  if (!on_device) {
    int rc = ensure_stage(lat);
    if (rc) return rc;
    U1_CUDA_TRY(cudaMemcpyAsync(lat->stage, angles, n * sizeof(double), cudaMemcpyHostToDevice, lat->stream));
    src = lat->stage;
  }
  k_import_angles<<<u1i::blocks_for((long long)n, 256), 256, 0, lat->stream>>>(lat->links, src, n);
  U1_LAUNCH_CHECK("k_import_angles");
  if (wait) U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
  return U1_OK;
}

extern "C" int u1_lattice_import_angles(u1_lattice *lat, const double *angles, int on_device) {
  if (!lat || !angles) return fail(U1_ERR_INVALID, "u1_lattice_import_angles: null argument");
  return import_angles(lat, angles, on_device, true);
}

extern "C" int u1_lattice_import_angles_async(u1_lattice *lat, const double *angles, int on_device) {
  if (!lat || !angles) return fail(U1_ERR_INVALID, "u1_lattice_import_angles_async: null argument");
  return import_angles(lat, angles, on_device, false);
}

static int wave_check(u1_lattice *lat);

// Export (float2 links -> angles) queued on the lattice's stream; `wait`:
// check the persistent sweep's error word first and return only once the
// export has completed.
static int export_angles(u1_lattice *lat, double *angles, int on_device, bool wait) {
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  if (wait) {
    int rc = wave_check(lat);
    if (rc) return rc;
  }
  const size_t n = (size_t)lat->g.V * lat->g.dims;
  double *dst = angles;
  if (!on_device) {
    int rc = ensure_stage(lat);
    if (rc) return rc;
    dst = lat->stage;
  }
  k_export_angles<<<u1i::blocks_for((long long)n, 256), 256, 0, lat->stream>>>(lat->links, dst, n);
  U1_LAUNCH_CHECK("k_export_angles");
  if (!on_device)
    U1_CUDA_TRY(cudaMemcpyAsync(angles, lat->stage, n * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  if (wait) U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
  return U1_OK;
}

extern "C" int u1_lattice_export_angles(const u1_lattice *clat, double *angles, int on_device) {
  if (!clat || !angles) return fail(U1_ERR_INVALID, "u1_lattice_export_angles: null argument");
  return export_angles(const_cast<u1_lattice *>(clat), angles, on_device, true);  // the staging buffer is a cache
}

extern "C" int u1_lattice_export_angles_async(const u1_lattice *clat, double *angles, int on_device) {
  if (!clat || !angles) return fail(U1_ERR_INVALID, "u1_lattice_export_angles_async: null argument");
  return export_angles(const_cast<u1_lattice *>(clat), angles, on_device, false);
}

extern "C" int u1_lattice_synchronize(u1_lattice *lat) {
  if (!lat) return fail(U1_ERR_INVALID, "u1_lattice_synchronize: null lattice");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
  return wave_check(lat);
}

// ---------------------------------------------------------------- rng
extern "C" int u1_rng_create(u1_ctx *ctx, uint64_t seed, u1_rng **out) {
  if (!ctx || !out) return fail(U1_ERR_INVALID, "u1_rng_create: null argument");
  *out = nullptr;
  U1_CUDA_TRY(cudaSetDevice(ctx->device));
  u1_rng *r = new u1_rng;
  r->ctx = ctx;
  r->seed = seed;
  r->pass = 0;
  r->chain = 0;
  r->id = u1i::g_rng_ids.fetch_add(1);
  cudaError_t e = u1i::dev_alloc(&r->pass_dev, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(r->pass_dev, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    if (r->pass_dev) u1i::dev_free(r->pass_dev);
    delete r;
    return u1i::cuda_fail(e, "u1_rng_create");
  }
  *out = r;
  return U1_OK;
}

extern "C" int u1_rng_destroy(u1_rng *rng) {
  if (!rng) return U1_OK;
  cudaSetDevice(rng->ctx->device);
  cudaDeviceSynchronize();
  if (rng->pass_dev) u1i::dev_free(rng->pass_dev);
  if (rng->replay_dev) u1i::dev_free(rng->replay_dev);
  delete rng;
  return U1_OK;
}

extern "C" int u1_rng_get_state(const u1_rng *rng, uint64_t *seed, uint64_t *pass) {
  if (!rng) return fail(U1_ERR_INVALID, "u1_rng_get_state: null rng");
  if (seed) *seed = rng->seed;
  if (pass) *pass = rng->pass;
  return U1_OK;
}

extern "C" int u1_rng_set_state(u1_rng *rng, uint64_t seed, uint64_t pass) {
  if (!rng) return fail(U1_ERR_INVALID, "u1_rng_set_state: null rng");
  U1_CUDA_TRY(cudaSetDevice(rng->ctx->device));
  U1_CUDA_TRY(cudaDeviceSynchronize());
  unsigned long long v = pass;
  U1_CUDA_TRY(cudaMemcpy(rng->pass_dev, &v, sizeof(v), cudaMemcpyHostToDevice));
  rng->seed = seed;
  rng->pass = pass;
  return U1_OK;
}

extern "C" int u1_rng_set_chain(u1_rng *rng, uint32_t chain) {
  if (!rng) return fail(U1_ERR_INVALID, "u1_rng_set_chain: null rng");
  if (chain > 0xFFFFu) return fail(U1_ERR_INVALID, "u1_rng_set_chain: chain must be < 65536");
  rng->chain = chain;
  return U1_OK;
}

extern "C" int u1_rng_set_replay(u1_rng *rng, const double *pairs, size_t n_pairs) {
  if (!rng) return fail(U1_ERR_INVALID, "u1_rng_set_replay: null rng");
  U1_CUDA_TRY(cudaSetDevice(rng->ctx->device));
  U1_CUDA_TRY(cudaDeviceSynchronize());
  if (rng->replay_dev) u1i::dev_free(rng->replay_dev);
  rng->replay_dev = nullptr;
  rng->replay_pairs = 0;
  if (!pairs || n_pairs == 0) return U1_OK;
  U1_CUDA_TRY(u1i::dev_alloc(&rng->replay_dev, n_pairs * 2 * sizeof(double)));
  U1_CUDA_TRY(cudaMemcpy(rng->replay_dev, pairs, n_pairs * 2 * sizeof(double), cudaMemcpyHostToDevice));
  rng->replay_pairs = n_pairs;
  rng->replay_base = rng->pass;
  return U1_OK;
}

extern "C" int u1_rng_debug_uniforms(u1_lattice *lat, const u1_rng *rng, uint64_t pass, int parity,
                                     int mu, float *out_host) {
  if (!lat || !rng || !out_host) return fail(U1_ERR_INVALID, "u1_rng_debug_uniforms: null argument");
  if (parity < 0 || parity > 1 || mu < 0 || mu >= lat->g.dims)
    return fail(U1_ERR_INVALID, "u1_rng_debug_uniforms: bad parity/mu");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  float *d = nullptr;
  U1_CUDA_TRY(u1i::dev_alloc(&d, (size_t)lat->g.Vh * 2 * sizeof(float)));
  k_rng_debug<<<u1i::blocks_for(lat->g.Vh, 256), 256, 0, lat->stream>>>(
      d, lat->g.Vh, parity, mu, (uint32_t)rng->seed, (uint32_t)(rng->seed >> 32), rng->chain, pass);
  u1i::g_launches++;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out_host, d, (size_t)lat->g.Vh * 2 * sizeof(float), cudaMemcpyDeviceToHost, lat->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lat->stream);
  u1i::dev_free(d);
  if (e != cudaSuccess) return u1i::cuda_fail(e, "k_rng_debug");
  return U1_OK;
}

// ---------------------------------------------------------------- updates
template <int D>
static int launch_hot(u1_lattice *lat, u1_rng *rng) {
  k_hot_start<D><<<u1i::blocks_for(lat->g.Vh, 256), 256, 0, lat->stream>>>(
      lat->links, lat->g, (uint32_t)rng->seed, (uint32_t)(rng->seed >> 32), rng->chain, rng->pass);
  U1_LAUNCH_CHECK("k_hot_start");
  k_pass_add<<<1, 1, 0, lat->stream>>>(rng->pass_dev, 1ull);
  U1_LAUNCH_CHECK("k_pass_add");
  return U1_OK;
}

extern "C" int u1_hot_start(u1_lattice *lat, u1_rng *rng) {
  u1i::NvtxRange nvtx_range("u1_hot_start");
  if (!lat || !rng) return fail(U1_ERR_INVALID, "u1_hot_start: null argument");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  int rc;
  switch (lat->g.dims) {
    case 2: rc = launch_hot<2>(lat, rng); break;
    case 3: rc = launch_hot<3>(lat, rng); break;
    default: rc = launch_hot<4>(lat, rng); break;
  }
  if (rc) return rc;
  rng->pass += 1;
  return U1_OK;
}

// Launch one phase kernel with programmatic stream serialization (PDL): it
// may be scheduled before the previous kernel on the stream finishes and
// waits for it in-kernel (griddepcontrol.wait) before reading links.
template <class K>
static int launch_pdl(K kernel, int blocks, cudaStream_t s, const UpdArgs &a, const char *what,
                      int threads = 256) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, a);
  u1i::g_launches.fetch_add(1, std::memory_order_relaxed);
  if (e != cudaSuccess) return u1i::cuda_fail(e, what);
  return U1_OK;
}

// The phase kernel of the chosen variant; src: the Metropolis proposal
// source (SRC_PHILOX, SRC_REPLAY or SRC_WINDOW; ignored for overrelaxation).
// threads: block size (a multiple of 32 up to 256, the kernels' launch
// bound); the kernels index sites from blockDim, so every block size gives
// the same links.
template <int D, int MU, int SRC>
static int launch_variant(const UpdArgs &a, cudaStream_t s, bool met, int variant, int threads) {
  if (variant == U1V_QUAD) {
    threads = std::min(threads, 128);  // the kernel's launch bound
    const int blocks = u1i::blocks_for(a.g.Vh / 4, threads);
    return met ? launch_pdl(k_update_quad<D, MU, true, SRC>, blocks, s, a, "k_update_quad", threads)
               : launch_pdl(k_update_quad<D, MU, false, SRC_PHILOX>, blocks, s, a, "k_update_quad", threads);
  }
  if (variant == U1V_PAIR32 || variant == U1V_PAIR) {
    const int blocks = u1i::blocks_for(a.g.Vh / 2, threads);
    if (variant == U1V_PAIR32)
      return met ? launch_pdl(k_update_pair<D, MU, true, SRC>, blocks, s, a, "k_update_pair", threads)
                 : launch_pdl(k_update_pair<D, MU, false, SRC_PHILOX>, blocks, s, a, "k_update_pair", threads);
    return met ? launch_pdl(k_update_pair_free<D, MU, true, SRC>, blocks, s, a, "k_update_pair_free", threads)
               : launch_pdl(k_update_pair_free<D, MU, false, SRC_PHILOX>, blocks, s, a, "k_update_pair_free",
                            threads);
  }
  const int blocks = u1i::blocks_for(a.g.Vh, threads);
  return met ? launch_pdl(k_update<D, MU, true, SRC>, blocks, s, a, "k_update", threads)
             : launch_pdl(k_update<D, MU, false, SRC_PHILOX>, blocks, s, a, "k_update", threads);
}

template <int D, int MU>
static int launch_phase_mu(const UpdArgs &a, cudaStream_t s, bool met, int src, int variant, int threads) {
  if (!met || src == SRC_PHILOX) return launch_variant<D, MU, SRC_PHILOX>(a, s, met, variant, threads);
  if (src == SRC_REPLAY) return launch_variant<D, MU, SRC_REPLAY>(a, s, met, variant, threads);
  return launch_variant<D, MU, SRC_WINDOW>(a, s, met, variant, threads);
}

template <int D>
static int launch_phase(const UpdArgs &a, cudaStream_t s, bool met, int src, int variant, int threads) {
  switch (a.mu) {
    case 0: return launch_phase_mu<D, 0>(a, s, met, src, variant, threads);
    case 1: return launch_phase_mu<D, 1>(a, s, met, src, variant, threads);
    case 2:
      if constexpr (D > 2) return launch_phase_mu<D, 2>(a, s, met, src, variant, threads);
      break;
    case 3:
      if constexpr (D > 3) return launch_phase_mu<D, 3>(a, s, met, src, variant, threads);
      break;
  }
  return fail(U1_ERR_INVALID, "k_update: direction out of range");
}

// Whether a four-site phase at the lattice's block size runs as a single
// wave (the SM-local block order then applies); cached per block size.
static void quad_layout(u1_lattice *lat) {
  if (lat->remap_block == lat->block) return;
  const int sms = lat->ctx->prop.multiProcessorCount;
  const int threads = std::min(lat->block, 128);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_update_quad<4, 0, false, SRC_PHILOX>, threads, 0) !=
      cudaSuccess)
    per_sm = 0;
  const long long blocks = ((long long)lat->g.Vh / 4 + threads - 1) / threads;
  lat->remap_sms = (per_sm > 0 && blocks <= (long long)per_sm * sms) ? sms : 0;
  lat->remap_block = lat->block;
}

// Whether consecutive phases alternate their block order (rev_block): for a
// lattice whose links exceed half the L2, each phase then starts on the
// links the previous one left in L2.  U1_ALTERNATE=0 in the environment keeps
// the launch order.
static bool alternate_order(const u1_lattice *lat) {
  static const bool off = [] {
    const char *r = std::getenv("U1_ALTERNATE");
    return r && r[0] == '0';
  }();
  const size_t bytes = (size_t)lat->g.V * lat->g.dims * sizeof(float2);
  return !off && 2 * bytes > (size_t)lat->ctx->prop.l2CacheSize;
}

// SM count for the block-order remap of the four-site phase kernels
// (sm_local_block) when a phase's grid runs as a single wave, else 0 (launch
// order).  Over several waves the remap hands each SM a distant slice of the
// lattice, so a plane and its neighbour planes are loaded many waves apart
// and miss in L2 (measured at 64^4: 1.5x the algorithmic DRAM reads, L2 hit
// rate 22 %).  U1_REMAP=0 in the environment keeps the launch order always.
static int sm_remap(u1_lattice *lat) {
  static const bool off = [] {
    const char *r = std::getenv("U1_REMAP");
    return r && r[0] == '0';
  }();
  quad_layout(lat);
  return off ? 0 : lat->remap_sms;
}

// The proposal settings of `lat` into the kernel arguments.
static void set_proposal(UpdArgs &a, const u1_lattice *lat) {
  a.win = lat->win;
  a.nhits = lat->nhits;
}

// Variant used when the tuner has not chosen one.
static int default_variant(const GeomK &g) { return (g.hN0 & 1) ? U1V_SINGLE : U1V_PAIR32; }

// The persistent sweep needs a fitting geometry, cooperative launch support
// and every tile's block resident at once.
static bool wave_usable(u1_lattice *lat) {
  if (lat->wave_ok >= 0) return lat->wave_ok == 1;
  lat->wave_ok = 0;
  const int threads = wave_threads(lat->g);
  if (!threads) return false;
  int coop = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, lat->ctx->device) != cudaSuccess || !coop)
    return false;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_wave<4>, threads, 0) != cudaSuccess)
    return false;
  if ((long long)per_sm * lat->ctx->prop.multiProcessorCount < wave_tiles(lat->g)) return false;
  const size_t n = (size_t)wave_tiles(lat->g) + 2;  // flags, ticket, error word
  if (u1i::dev_alloc(&lat->wave_state, n * sizeof(unsigned int)) != cudaSuccess) return false;
  if (cudaMemset(lat->wave_state, 0, n * sizeof(unsigned int)) != cudaSuccess) return false;
  lat->wave_ok = 1;
  return true;
}

static bool variant_valid(u1_lattice *lat, int v) {
  const GeomK &g = lat->g;
  if (v == U1V_WAVE) return wave_usable(lat);
  return v == U1V_SINGLE || ((v == U1V_PAIR32 || v == U1V_PAIR) && (g.hN0 & 1) == 0) ||
         (v == U1V_QUAD && (g.hN0 & 3) == 0);
}

// One sweep as a single cooperative launch of k_sweep_wave (see u1_wave.cuh).
static int launch_wave(u1_lattice *lat, float2 *links, u1_rng *rng, int metrop, int ovrn, double *meas) {
  WaveArgs w{};
  w.a.lat = links;
  w.a.g = lat->g;
  w.a.c = lat->c;
  w.a.key0 = (uint32_t)rng->seed;
  w.a.key1 = (uint32_t)(rng->seed >> 32);
  w.a.chain = rng->chain;
  w.a.pass_dev = rng->pass_dev;
  w.metrop = metrop;
  w.ovrn = ovrn;
  w.meas = meas;
  const int tiles = wave_tiles(lat->g);
  w.flags = lat->wave_state;
  w.ticket = lat->wave_state + tiles;
  w.err = lat->wave_state + tiles + 1;
  w.pass_rw = rng->pass_dev;
  w.spin_limit = lat->wave_spin_limit ? lat->wave_spin_limit : kWaveSpinLimit;
  w.stall_tile = lat->wave_stall_tile;
#ifdef U1_BOUNDS_CHECK
  // bounds checks only: the persistent sweep's phases overlap within the
  // launch, so there is no phase end for the race marks
  w.a.chk = lat->ctx->chk;
  w.a.shadow = nullptr;
  w.a.chk_base = links;
#endif
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)tiles);
  cfg.blockDim = dim3((unsigned)wave_threads(lat->g));
  cfg.stream = lat->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_sweep_wave<4>, w);
  u1i::g_launches.fetch_add(1, std::memory_order_relaxed);
  if (e != cudaSuccess) return u1i::cuda_fail(e, "k_sweep_wave");
  return U1_OK;
}

// A wait of the persistent sweep that ran out leaves its phase in the error
// word; synchronous entry points report it (and clear the state).
static int wave_check(u1_lattice *lat) {
  if (lat->wave_ok != 1) return U1_OK;
  const int tiles = wave_tiles(lat->g);
  unsigned int err = 0;
  U1_CUDA_TRY(cudaMemcpyAsync(&err, lat->wave_state + tiles + 1, sizeof(err), cudaMemcpyDeviceToHost, lat->stream));
  U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
  if (!err) return U1_OK;
  cudaMemsetAsync(lat->wave_state, 0, (tiles + 2) * sizeof(unsigned int), lat->stream);
  cudaStreamSynchronize(lat->stream);
  return fail(U1_ERR_CUDA, "persistent sweep: a neighbour wait ran out in phase " + std::to_string(err - 1) +
                               "; the configuration is invalid");
}
static int effective_variant(const u1_lattice *lat) {
  return lat->variant == U1V_AUTO ? default_variant(lat->g) : lat->variant;
}

// Metropolis proposal source of a lattice with this rng: the replay stream
// when one is set, else the windowed multi-hit kernels unless the lattice
// keeps the reference's single whole-circle proposal.
static int metropolis_src(const u1_lattice *lat, const u1_rng *rng) {
  if (rng->replay_dev) return SRC_REPLAY;
  return (lat->win != 0.f || lat->nhits != 1) ? SRC_WINDOW : SRC_PHILOX;
}

// The variant a sweep with proposal source `src` and freeze period ml runs:
// the persistent sweep covers only plain whole-circle sweeps; otherwise a
// lattice set to it runs the default phase kernels (bit-identical).
static int sweep_variant(const u1_lattice *lat, int src, int ml) {
  const int v = effective_variant(lat);
  if (v == U1V_WAVE && (ml != 0 || src != SRC_PHILOX)) return default_variant(lat->g);
  return v;
}

// Phase (1, MU) of the last pass with the measurement terms (u1_fused.cuh),
// writing the per-block partials of slot MU-1 into `partials`.
template <int D, int MU>
static int launch_meas_phase_mu(const UpdArgs &a, cudaStream_t s, bool met, bool win, bool quad,
                                double *partials) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)meas_phase_blocks(a.g));
  cfg.blockDim = dim3(quad ? 128 : 256);  // quad: four sites per thread, the same 512 sites per block
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  double *slot = partials + (size_t)(MU - 1) * meas_phase_blocks(a.g) * 2;
  cudaError_t e;
  if (quad)
    e = !met ? cudaLaunchKernelEx(&cfg, k_update_quad_meas<D, MU, false>, a, slot)
        : win ? cudaLaunchKernelEx(&cfg, k_update_quad_meas<D, MU, true, SRC_WINDOW>, a, slot)
              : cudaLaunchKernelEx(&cfg, k_update_quad_meas<D, MU, true>, a, slot);
  else if ((a.g.hN0 & 1) == 0)
    e = !met ? cudaLaunchKernelEx(&cfg, k_update_pair_meas<D, MU, false>, a, slot)
        : win ? cudaLaunchKernelEx(&cfg, k_update_pair_meas<D, MU, true, SRC_WINDOW>, a, slot)
              : cudaLaunchKernelEx(&cfg, k_update_pair_meas<D, MU, true>, a, slot);
  else
    e = !met ? cudaLaunchKernelEx(&cfg, k_update_meas<D, MU, false>, a, slot)
        : win ? cudaLaunchKernelEx(&cfg, k_update_meas<D, MU, true, SRC_WINDOW>, a, slot)
              : cudaLaunchKernelEx(&cfg, k_update_meas<D, MU, true>, a, slot);
  u1i::g_launches.fetch_add(1, std::memory_order_relaxed);
  if (e != cudaSuccess) return u1i::cuda_fail(e, "k_update_pair_meas");
  return U1_OK;
}

template <int D>
static int launch_meas_phase(const UpdArgs &a, cudaStream_t s, bool met, bool win, bool quad, double *partials) {
  switch (a.mu) {
    case 1: return launch_meas_phase_mu<D, 1>(a, s, met, win, quad, partials);
    case 2:
      if constexpr (D > 2) return launch_meas_phase_mu<D, 2>(a, s, met, win, quad, partials);
      break;
    case 3:
      if constexpr (D > 3) return launch_meas_phase_mu<D, 3>(a, s, met, win, quad, partials);
      break;
  }
  return fail(U1_ERR_INVALID, "measuring phase: direction out of range");
}

// Entries per phase slot of a measured sweep: one per block of the measuring
// phase kernels, or one per tile of the persistent sweep.
static int meas_slot_entries(const u1_lattice *lat, int variant) {
  return variant == U1V_WAVE ? wave_tiles(lat->g) : meas_phase_blocks(lat->g);
}

// Scratch (doubles) of a measured sweep: D-1 phase slots + Polyakov blocks
// (sized for either layout).
static size_t meas_sweep_scratch(const GeomK &g) {
  const size_t slot = (size_t)std::max(meas_phase_blocks(g), wave_tiles(g));
  return (size_t)(g.dims - 1) * slot * 2 + (size_t)measure_layout(g).nb_poly * 2;
}

// The Polyakov loops and the final sum of a measured sweep, into dev_out.
template <int D>
static int launch_poly_finish(u1_lattice *lat, int variant, double *dev_out) {
  const GeomK &g = lat->g;
  MeasK m = measure_layout(g);
  int nSS = 0, nST = 0;
  for (int mu = 0; mu < D - 1; ++mu)
    for (int nu = mu + 1; nu < D; ++nu) (nu == D - 1 ? nST : nSS)++;
  const double normSS = 1.0 / ((double)g.V * nSS), normST = 1.0 / ((double)g.V * nST);
  const double normL = 1.0 / (double)g.Vs;
  const int nbp = meas_slot_entries(lat, variant);
  double *poly = lat->partials + (size_t)(D - 1) * nbp * 2;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)m.nb_poly);
  cfg.blockDim = dim3(kRedThreads);
  cfg.stream = lat->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k_poly_finish<D>, (const float2 *)lat->links, g, m,
                                           (const double *)lat->partials, nbp, poly, lat->counter, dev_out, normSS,
                                           normST, normL);
  u1i::g_launches.fetch_add(1, std::memory_order_relaxed);
  if (e != cudaSuccess) return u1i::cuda_fail(e, "k_poly_finish");
  return U1_OK;
}

// Issue one sweep (metrop Metropolis + ovrn overrelaxation passes) on links
// `links` with freeze period ml.  The device pass counter advances by metrop.
// meas_partials != nullptr: phases (1, mu >= 1) of the sweep's last pass run
// as the measuring kernels, writing their partial plaquette sums there
// (meas_sweep_scratch doubles; k_poly_finish completes the measurement).
static int issue_sweep(u1_lattice *lat, float2 *links, u1_rng *rng, int metrop, int ovrn, int ml,
                       double *meas_partials = nullptr) {
  UpdArgs a{};
  a.lat = links;
  a.g = lat->g;
  a.c = lat->c;
  a.key0 = (uint32_t)rng->seed;
  a.key1 = (uint32_t)(rng->seed >> 32);
  a.chain = rng->chain;
  a.pass_dev = rng->pass_dev;
  a.replay = rng->replay_dev;
  a.replay_base = rng->replay_base;
  a.ml = ml;
  set_proposal(a, lat);
#ifdef U1_BOUNDS_CHECK
  a.chk = lat->ctx->chk;
  a.shadow = lat->shadow;
  a.chk_base = links;
#endif
  // with a freeze period the SM-local order would hand whole frozen slabs to
  // some SMs and none to others (measured 4 % slower multilevel): keep the launch order
  a.sms = ml ? 0 : sm_remap(lat);
  const bool alternate = a.sms == 0 && alternate_order(lat);
  const int src = metropolis_src(lat, rng);
  const int var = sweep_variant(lat, src, ml);
  if (var == U1V_WAVE) return launch_wave(lat, links, rng, metrop, ovrn, meas_partials);
  const int D = lat->g.dims;
  const int total = 2 * D * (metrop + ovrn);
  int phase = 0;
  auto launch = [&](bool met) -> int {
    ++phase;
    a.rev = (alternate && (phase & 1) == 0) ? 1 : 0;  // every second phase runs its blocks backwards
    int rc;
    // the last pass is phases total-2D+1 .. total; its parity-1 half with mu >= 1 measures
    if (meas_partials && phase > total - 2 * D && a.p == 1 && a.mu >= 1)
      rc = D == 2 ? launch_meas_phase<2>(a, lat->stream, met, src == SRC_WINDOW, var == U1V_QUAD, meas_partials)
         : D == 3 ? launch_meas_phase<3>(a, lat->stream, met, src == SRC_WINDOW, var == U1V_QUAD, meas_partials)
                  : launch_meas_phase<4>(a, lat->stream, met, src == SRC_WINDOW, var == U1V_QUAD, meas_partials);
    else
      rc = D == 2 ? launch_phase<2>(a, lat->stream, met, src, var, lat->block)
         : D == 3 ? launch_phase<3>(a, lat->stream, met, src, var, lat->block)
                  : launch_phase<4>(a, lat->stream, met, src, var, lat->block);
#ifdef U1_BOUNDS_CHECK
    if (rc == U1_OK) rc = u1i::chk_phase_end(lat->stream, a.shadow, (size_t)D * lat->g.V, a.chk);
#endif
    return rc;
  };
  for (int m = 0; m < metrop; ++m)
    for (int p = 0; p < 2; ++p)
      for (int mu = 0; mu < D; ++mu) {
        a.p = p;
        a.mu = mu;
        a.hit = m;
        int rc = launch(true);
        if (rc) return rc;
      }
  bool bumped = (metrop == 0);
  for (int o = 0; o < ovrn; ++o)
    for (int p = 0; p < 2; ++p)
      for (int mu = 0; mu < D; ++mu) {
        a.p = p;
        a.mu = mu;
        a.hit = 0;
        a.bump_ptr = bumped ? nullptr : rng->pass_dev;
        a.bump_by = (unsigned)metrop;
        bumped = true;
        int rc = launch(false);
        if (rc) return rc;
      }
  if (!bumped) {
    k_pass_add<<<1, 1, 0, lat->stream>>>(rng->pass_dev, (unsigned long long)metrop);
    U1_LAUNCH_CHECK("k_pass_add");
  }
  return U1_OK;
}

static int check_replay(const u1_lattice *lat, const u1_rng *rng, int metrop) {
  if (!rng->replay_dev) return U1_OK;
  const size_t per_pass = (size_t)lat->g.V * lat->g.dims;
  if (rng->replay_pairs % per_pass != 0)
    return fail(U1_ERR_INVALID, "replay stream length is not a multiple of V*dims pairs");
  const uint64_t avail = rng->replay_pairs / per_pass;
  if (rng->pass < rng->replay_base || rng->pass + (uint64_t)metrop - rng->replay_base > avail)
    return fail(U1_ERR_STATE, "replay stream exhausted");
  return U1_OK;
}

// Capture `fn` (which issues work on lat->stream) into an executable graph.
template <class F>
static int capture_graph(u1_lattice *lat, F fn, cudaGraphExec_t *exec) {
  cudaGraph_t graph = nullptr;
  U1_CUDA_TRY(cudaStreamBeginCapture(lat->stream, cudaStreamCaptureModeThreadLocal));
  const unsigned long long launches0 = u1i::g_launches.load();
  int rc = fn();
  u1i::g_launches.store(launches0);  // captured kernels run (and count) at graph launch
  cudaError_t e = cudaStreamEndCapture(lat->stream, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return u1i::cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return u1i::cuda_fail(e, "cudaGraphInstantiate");
  return U1_OK;
}

// Block sizes the phase kernels accept: whole warps up to their launch bound.
static bool block_valid(int threads) { return threads >= 32 && threads <= 256 && threads % 32 == 0; }

// ---------------------------------------------------------------- tuner
// Replaces the reference's block-size search (src/tune.cpp:306-416,
// include/tune.h:143-260): the candidates are the compiled update-kernel
// variants (two sites per thread with a 32-register cap, two sites
// uncapped, one site), each at 64, 96, 128, 192 and 256 threads per block
// (the four-site kernel up to 128): block counts that fill the SMs evenly
// differ with the lattice size; all give
// bit-identical links, so a trial never changes the Markov chain.  Each
// trial captures its sweep as a CUDA graph, as u1_update runs it, and times
// replays of it from a backed-up state (links and pass counter restored
// afterwards, as the reference's preTune/postTune do), after a clock
// warm-up, in two rounds (the second in reverse order), each candidate scored
// by its shortest single replay; the winner is cached per (device, geometry) in
// memory and, when U1_RESOURCE_PATH names a directory, in
// $U1_RESOURCE_PATH/u1b200_tunecache.tsv (the reference's tunecache.csv
// location rule, src/tune.cpp:160-232).  U1_TUNE=0 disables tuning.
namespace {
struct TuneCache {
  std::mutex mu;
  bool loaded = false;
  std::map<std::string, std::pair<int, int>> best;  // key -> (variant, threads per block)
};
TuneCache &tune_cache() {
  static TuneCache c;
  return c;
}
std::string tune_file() {
  const char *p = std::getenv("U1_RESOURCE_PATH");
  return (p && *p) ? std::string(p) + "/u1b200_tunecache.tsv" : std::string();
}
bool tuning_enabled() {
  const char *e = std::getenv("U1_TUNE");
  return !(e && e[0] == '0');
}
std::string tune_key(const u1_lattice *lat) {
  std::ostringstream k;
  k << lat->ctx->prop.name << "|update|" << lat->g.dims << "|" << lat->g.N[0] << "x" << lat->g.N[1] << "x"
    << lat->g.N[2] << "x" << lat->g.N[3];
  return k.str();
}
void tune_load_locked(TuneCache &c) {
  if (c.loaded) return;
  c.loaded = true;
  const std::string f = tune_file();
  if (f.empty()) return;
  std::ifstream in(f);
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    const size_t t1 = line.find('\t');
    if (t1 == std::string::npos) continue;
    // key <tab> variant <tab> microseconds per sweep [<tab> threads per block]
    std::vector<std::string> col;
    size_t a = 0;
    while (true) {
      const size_t t = line.find('\t', a);
      col.push_back(line.substr(a, t == std::string::npos ? std::string::npos : t - a));
      if (t == std::string::npos) break;
      a = t + 1;
    }
    if (col.size() < 2) continue;
    const int v = std::atoi(col[1].c_str());
    const int threads = col.size() >= 4 ? std::atoi(col[3].c_str()) : 256;
    if (v >= U1V_PAIR32 && v <= U1V_QUAD && block_valid(threads)) c.best[col[0]] = {v, threads};
  }
}
void tune_save(const std::string &key, int v, double us, int threads) {
  const std::string f = tune_file();
  if (f.empty()) return;
  std::ofstream out(f, std::ios::app);
  if (out) out << key << '\t' << v << '\t' << us << '\t' << threads << '\n';
}
}  // namespace

static int tune_update(u1_lattice *lat, u1_rng *rng, bool use_cache) {
  const std::string key = tune_key(lat);
  TuneCache &c = tune_cache();
  if (use_cache) {
    std::lock_guard<std::mutex> lock(c.mu);
    tune_load_locked(c);
    auto it = c.best.find(key);
    if (it != c.best.end() && variant_valid(lat, it->second.first)) {
      lat->variant = it->second.first;
      lat->block = it->second.second;
      drop_graphs(lat);
      return U1_OK;
    }
  }
  std::vector<std::pair<int, int>> cand;  // (variant, threads per block)
  for (int v : {U1V_PAIR32, U1V_QUAD, U1V_PAIR, U1V_SINGLE})  // the persistent sweep is opt-in (u1_wave.cuh)
    if (variant_valid(lat, v))
      for (int t : {256, 192, 128, 96, 64})
        if (v != U1V_QUAD || t <= 128) cand.push_back({v, t});
  std::pair<int, int> best = cand[0];
  double best_us = -1.0;
  if (cand.size() > 1) {
    const size_t n = (size_t)lat->g.V * lat->g.dims;
    if (!lat->backup) U1_CUDA_TRY(u1i::dev_alloc(&lat->backup, n * sizeof(float2)));
    U1_CUDA_TRY(cudaMemcpyAsync(lat->backup, lat->links, n * sizeof(float2), cudaMemcpyDeviceToDevice, lat->stream));
    const unsigned long long pass0 = rng->pass;
    int rc = U1_OK;
    // Two rounds over the candidates, the second in reverse order, keeping
    // each candidate's faster time: a large lattice drives the GPU into its
    // power cap during tuning, and one round would favour whichever
    // candidates ran first (measured at 64^4: the two-site kernel at 96
    // threads picked over the four-site one, 4.8 against 4.0 ms a step).
    // Each trial scores its candidate by the shortest of 5 single replays;
    // the first trial is preceded by about 50 ms of replays to bring the
    // clocks up.
    std::vector<double> cand_us(cand.size(), -1.0);
    std::vector<size_t> order;
    for (size_t k = 0; k < cand.size(); ++k) order.push_back(k);
    for (size_t k = cand.size(); k-- > 0;) order.push_back(k);
    bool warmed = false;
    for (size_t ci : order) {
      const auto &vt = cand[ci];
      lat->variant = vt.first;
      lat->block = vt.second;
      cudaGraphExec_t ex = nullptr;
      rc = capture_graph(lat, [&]() { return issue_sweep(lat, lat->links, rng, 1, 4, 0); }, &ex);
      double us = 0.0;
      if (!rc && !warmed) {
        const cudaError_t er = u1i::warm_clocks(ex, lat->stream, 50.0);
        if (er != cudaSuccess) rc = u1i::cuda_fail(er, "tuning warm-up");
        warmed = true;
      }
      if (!rc) {
        const cudaError_t er = u1i::time_graph_min(ex, lat->stream, 2, 5, &us);
        if (er != cudaSuccess) rc = u1i::cuda_fail(er, "tuning sweep");
      }
      cudaMemcpyAsync(lat->links, lat->backup, n * sizeof(float2), cudaMemcpyDeviceToDevice, lat->stream);
      cudaMemcpyAsync(rng->pass_dev, &pass0, sizeof(pass0), cudaMemcpyHostToDevice, lat->stream);
      cudaStreamSynchronize(lat->stream);
      if (ex) cudaGraphExecDestroy(ex);
      if (rc) break;
      if (u1i::tune_verbose())
        std::fprintf(stderr, "u1_tune %s: variant %d, %d threads: %.1f us per sweep\n", key.c_str(), vt.first,
                     vt.second, us);
      if (cand_us[ci] < 0.0 || us < cand_us[ci]) cand_us[ci] = us;
    }
    for (size_t k = 0; k < cand.size() && !rc; ++k)
      if (best_us < 0.0 || cand_us[k] < best_us) {
        best_us = cand_us[k];
        best = cand[k];
      }
    if (rc) {
      lat->variant = U1V_AUTO;
      lat->block = 256;
      return rc;
    }
  }
  lat->variant = best.first;
  lat->block = best.second;
  drop_graphs(lat);
  std::lock_guard<std::mutex> lock(c.mu);
  tune_load_locked(c);
  c.best[key] = best;
  tune_save(key, best.first, best_us, best.second);
  return U1_OK;
}

extern "C" int u1_tune(u1_lattice *lat, u1_rng *rng, int *variant) {
  u1i::NvtxRange nvtx_range("u1_tune");
  if (!lat || !rng) return fail(U1_ERR_INVALID, "u1_tune: null argument");
  if (rng->replay_dev) return fail(U1_ERR_STATE, "u1_tune: not available while a replay stream is set");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  int rc = tune_update(lat, rng, false);
  if (rc) return rc;
  if (variant) *variant = lat->variant;
  return U1_OK;
}

extern "C" int u1_lattice_set_variant(u1_lattice *lat, int variant) {
  if (!lat) return fail(U1_ERR_INVALID, "u1_lattice_set_variant: null lattice");
  if (variant != U1V_AUTO && !variant_valid(lat, variant))
    return fail(U1_ERR_INVALID, "u1_lattice_set_variant: variant not valid for this geometry (pair variants need Nx/2 even)");
  lat->variant = variant;
  drop_graphs(lat);
  return U1_OK;
}

extern "C" int u1_lattice_set_wave_wait(u1_lattice *lat, unsigned spin_limit, int stall_tile) {
  if (!lat) return fail(U1_ERR_INVALID, "u1_lattice_set_wave_wait: null lattice");
  if (stall_tile >= wave_tiles(lat->g))
    return fail(U1_ERR_INVALID, "u1_lattice_set_wave_wait: stall_tile " + std::to_string(stall_tile) +
                                    " beyond the lattice's " + std::to_string(wave_tiles(lat->g)) + " tiles");
  lat->wave_spin_limit = spin_limit;
  lat->wave_stall_tile = stall_tile < 0 ? -1 : stall_tile;
  return U1_OK;
}

extern "C" int u1_lattice_get_variant(const u1_lattice *lat, int *variant) {
  if (!lat || !variant) return fail(U1_ERR_INVALID, "u1_lattice_get_variant: null argument");
  *variant = lat->variant;
  return U1_OK;
}

extern "C" int u1_lattice_set_block(u1_lattice *lat, int threads) {
  if (!lat) return fail(U1_ERR_INVALID, "u1_lattice_set_block: null lattice");
  if (!block_valid(threads))
    return fail(U1_ERR_INVALID, "u1_lattice_set_block: threads per block must be 32, 64, ..., 256");
  lat->block = threads;
  drop_graphs(lat);
  return U1_OK;
}

extern "C" int u1_lattice_get_block(const u1_lattice *lat, int *threads) {
  if (!lat || !threads) return fail(U1_ERR_INVALID, "u1_lattice_get_block: null argument");
  *threads = lat->block;
  return U1_OK;
}

extern "C" int u1_lattice_set_metropolis(u1_lattice *lat, double delta, int nhits) {
  if (!lat) return fail(U1_ERR_INVALID, "u1_lattice_set_metropolis: null lattice");
  if (!(delta >= 0.0 && delta <= M_PI))
    return fail(U1_ERR_INVALID, "u1_lattice_set_metropolis: delta must lie in [0, pi]");
  if (nhits < 1 || nhits > U1_MAX_HITS)
    return fail(U1_ERR_INVALID, "u1_lattice_set_metropolis: nhits must lie in [1, 127]");
  lat->delta = delta;
  lat->win = (float)(delta / M_PI);
  lat->nhits = nhits;
  drop_graphs(lat);
  return U1_OK;
}

extern "C" int u1_lattice_get_metropolis(const u1_lattice *lat, double *delta, int *nhits) {
  if (!lat || !delta || !nhits) return fail(U1_ERR_INVALID, "u1_lattice_get_metropolis: null argument");
  *delta = lat->delta;
  *nhits = lat->nhits;
  return U1_OK;
}

static int update_impl(u1_lattice *lat, u1_rng *rng, int metrop, int ovrn, double *meas_partials) {
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  int rc = check_replay(lat, rng, metrop);
  if (rc) return rc;
  const bool replay = rng->replay_dev != nullptr;
  if (lat->variant == U1V_AUTO && !replay && tuning_enabled()) {
    rc = tune_update(lat, rng, true);
    if (rc) return rc;
  }
  if (lat->use_graphs && !replay && sweep_variant(lat, metropolis_src(lat, rng), 0) != U1V_WAVE) {
    // graph key: passes, rng object, seed/chain and whether the last pass measures
    auto key = std::make_tuple(metrop * 2 + (meas_partials ? 1 : 0), ovrn, rng->id,
                               rng->seed ^ ((uint64_t)rng->chain << 48));
    auto it = lat->graphs.find(key);
    if (it == lat->graphs.end()) {
      cudaGraphExec_t ex = nullptr;
      rc = capture_graph(lat, [&]() { return issue_sweep(lat, lat->links, rng, metrop, ovrn, 0, meas_partials); },
                         &ex);
      if (rc) return rc;
      it = lat->graphs.emplace(key, ex).first;
    }
    U1_CUDA_TRY(cudaGraphLaunch(it->second, lat->stream));
    u1i::g_launches += (unsigned long long)(2 * lat->g.dims * (metrop + ovrn) + (ovrn == 0 ? 1 : 0));
  } else {
    rc = issue_sweep(lat, lat->links, rng, metrop, ovrn, 0, meas_partials);
    if (rc) return rc;
  }
  rng->pass += (uint64_t)metrop;
  return U1_OK;
}

extern "C" int u1_update(u1_lattice *lat, u1_rng *rng, int metrop, int ovrn) {
  u1i::NvtxRange nvtx_range("u1_update");
  if (!lat || !rng) return fail(U1_ERR_INVALID, "u1_update: null argument");
  if (metrop < 0 || ovrn < 0) return fail(U1_ERR_INVALID, "u1_update: negative pass count");
  if (metrop == 0 && ovrn == 0) return U1_OK;
  return update_impl(lat, rng, metrop, ovrn, nullptr);
}

static int measure_dispatch(u1_lattice *lat, double *dev_out);

extern "C" int u1_update_measure(u1_lattice *lat, u1_rng *rng, int metrop, int ovrn, double *dev_out) {
  u1i::NvtxRange nvtx_range("u1_update_measure");
  if (!lat || !rng || !dev_out) return fail(U1_ERR_INVALID, "u1_update_measure: null argument");
  if (metrop < 0 || ovrn < 0) return fail(U1_ERR_INVALID, "u1_update_measure: negative pass count");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  if ((metrop == 0 && ovrn == 0) || rng->replay_dev != nullptr) {
    // nothing to fuse with (or the test-only replay stream): update, then measure
    int rc = (metrop || ovrn) ? u1_update(lat, rng, metrop, ovrn) : U1_OK;
    if (rc) return rc;
    return measure_dispatch(lat, dev_out);
  }
  int rc = u1i::ensure_scratch(lat, meas_sweep_scratch(lat->g), 8);
  if (rc) return rc;
  rc = update_impl(lat, rng, metrop, ovrn, lat->partials);
  if (rc) return rc;
  const int var = sweep_variant(lat, metropolis_src(lat, rng), 0);
  switch (lat->g.dims) {
    case 2: return launch_poly_finish<2>(lat, var, dev_out);
    case 3: return launch_poly_finish<3>(lat, var, dev_out);
    default: return launch_poly_finish<4>(lat, var, dev_out);
  }
}

extern "C" int u1_update_phase(u1_lattice *lat, u1_rng *rng, int metropolis, int parity, int mu, int hit) {
  if (!lat || !rng) return fail(U1_ERR_INVALID, "u1_update_phase: null argument");
  if (parity < 0 || parity > 1 || mu < 0 || mu >= lat->g.dims || hit < 0)
    return fail(U1_ERR_INVALID, "u1_update_phase: bad parity/mu/hit");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  const bool met = metropolis != 0;
  const bool replay = met && rng->replay_dev != nullptr;
  if (replay) {
    int rc = check_replay(lat, rng, hit + 1);
    if (rc) return rc;
  }
  UpdArgs a{};
  a.lat = lat->links;
  a.g = lat->g;
  a.c = lat->c;
  a.p = parity;
  a.mu = mu;
  a.key0 = (uint32_t)rng->seed;
  a.key1 = (uint32_t)(rng->seed >> 32);
  a.chain = rng->chain;
  a.pass_dev = rng->pass_dev;
  a.hit = hit;
  a.replay = rng->replay_dev;
  a.replay_base = rng->replay_base;
  set_proposal(a, lat);
  a.sms = sm_remap(lat);
#ifdef U1_BOUNDS_CHECK
  a.chk = lat->ctx->chk;
  a.shadow = lat->shadow;
  a.chk_base = lat->links;
#endif
  const int src = metropolis_src(lat, rng);
  const int var = sweep_variant(lat, src, 0);
  int rc;
  switch (lat->g.dims) {
    case 2: rc = launch_phase<2>(a, lat->stream, met, src, var, lat->block); break;
    case 3: rc = launch_phase<3>(a, lat->stream, met, src, var, lat->block); break;
    default: rc = launch_phase<4>(a, lat->stream, met, src, var, lat->block); break;
  }
#ifdef U1_BOUNDS_CHECK
  if (rc == U1_OK) rc = u1i::chk_phase_end(lat->stream, a.shadow, (size_t)lat->g.dims * lat->g.V, a.chk);
#endif
  return rc;
}

// ---------------------------------------------------------------- measurements
template <int D>
static int launch_measure(u1_lattice *lat, double *dev_out) {
  const GeomK &g = lat->g;
  const MeasK m = measure_layout(g);
  const int nb = m.nb_plaq + m.nb_poly;
  int rc = u1i::ensure_scratch(lat, (size_t)nb * 6, 8);
  if (rc) return rc;
  int nSS = 0, nST = 0;
  for (int mu = 0; mu < D - 1; ++mu)
    for (int nu = mu + 1; nu < D; ++nu) (nu == g.tdir ? nST : nSS)++;
  const double normSS = 1.0 / ((double)g.V * nSS);
  const double normST = 1.0 / ((double)g.V * nST);
  const double normL = 1.0 / (double)g.Vs;
  k_measure<D><<<nb, kRedThreads, 0, lat->stream>>>(lat->links, g, m, lat->partials, lat->counter,
                                                   dev_out ? dev_out : lat->d_out, normSS, normST, normL);
  U1_LAUNCH_CHECK("k_measure");
  return U1_OK;
}

static int measure_dispatch(u1_lattice *lat, double *dev_out) {
  switch (lat->g.dims) {
    case 2: return launch_measure<2>(lat, dev_out);
    case 3: return launch_measure<3>(lat, dev_out);
    default: return launch_measure<4>(lat, dev_out);
  }
}

extern "C" int u1_measure_async(u1_lattice *lat, double *dev_out) {
  u1i::NvtxRange nvtx_range("u1_measure_async");
  if (!lat || !dev_out) return fail(U1_ERR_INVALID, "u1_measure_async: null argument");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  return measure_dispatch(lat, dev_out);
}

extern "C" int u1_measure(u1_lattice *lat, double out[6]) {
  u1i::NvtxRange nvtx_range("u1_measure");
  if (!lat || !out) return fail(U1_ERR_INVALID, "u1_measure: null argument");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  int rc = wave_check(lat);
  if (rc) return rc;
  rc = u1i::ensure_scratch(lat, 0, 8);
  if (rc) return rc;
  rc = measure_dispatch(lat, nullptr);
  if (rc) return rc;
  U1_CUDA_TRY(cudaMemcpyAsync(lat->h_out, lat->d_out, 6 * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
  memcpy(out, lat->h_out, 6 * sizeof(double));
  return U1_OK;
}

extern "C" int u1_plaquette(u1_lattice *lat, double out[4]) {
  if (!out) return fail(U1_ERR_INVALID, "u1_plaquette: null out");
  double m[6];
  int rc = u1_measure(lat, m);
  if (rc) return rc;
  memcpy(out, m, 4 * sizeof(double));
  return U1_OK;
}

extern "C" int u1_polyakov(u1_lattice *lat, double out[2]) {
  if (!out) return fail(U1_ERR_INVALID, "u1_polyakov: null out");
  double m[6];
  int rc = u1_measure(lat, m);
  if (rc) return rc;
  out[0] = m[4];
  out[1] = m[5];
  return U1_OK;
}

template <int D>
static int launch_poly_field(u1_lattice *lat, const float2 *links, int multihit) {
  const int nb = u1i::blocks_for(lat->g.Vs, 256);
  if (multihit)
    k_poly_field<D, true><<<nb, 256, 0, lat->stream>>>(links, lat->g, lat->c, lat->pfield);
  else
    k_poly_field<D, false><<<nb, 256, 0, lat->stream>>>(links, lat->g, lat->c, lat->pfield);
  U1_LAUNCH_CHECK("k_poly_field");
  return U1_OK;
}

extern "C" int u1_poly_corr(u1_lattice *lat, int multihit, double *out, int out_len) {
  u1i::NvtxRange nvtx_range("u1_poly_corr");
  if (!lat || !out) return fail(U1_ERR_INVALID, "u1_poly_corr: null argument");
  const int R = lat->g.N[0] / 2;
  if (out_len < 2 * R) return fail(U1_ERR_INVALID, "u1_poly_corr: out_len < 2*R (R = Grid[0]/2)");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  if (!lat->pfield) U1_CUDA_TRY(u1i::dev_alloc(&lat->pfield, (size_t)lat->g.Vs * sizeof(double2)));
  const int nb = u1i::blocks_for(lat->g.Vs, kRedThreads);
  int rc = u1i::ensure_scratch(lat, (size_t)nb * 2 * R, (size_t)2 * R);
  if (rc) return rc;
  switch (lat->g.dims) {
    case 2: rc = launch_poly_field<2>(lat, lat->links, multihit); break;
    case 3: rc = launch_poly_field<3>(lat, lat->links, multihit); break;
    default: rc = launch_poly_field<4>(lat, lat->links, multihit); break;
  }
  if (rc) return rc;
  const double norm = 1.0 / ((double)lat->g.Vs * lat->g.tdir);
  k_poly_corr<<<nb, kRedThreads, 0, lat->stream>>>(lat->pfield, lat->g, R, lat->partials, lat->counter,
                                                   lat->d_out, norm);
  U1_LAUNCH_CHECK("k_poly_corr");
  U1_CUDA_TRY(cudaMemcpyAsync(lat->h_out, lat->d_out, (size_t)2 * R * sizeof(double), cudaMemcpyDeviceToHost,
                              lat->stream));
  U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
  memcpy(out, lat->h_out, (size_t)2 * R * sizeof(double));
  return U1_OK;
}

// ---------------------------------------------------------------- multilevel
extern "C" int u1_multilevel(u1_lattice *lat, u1_rng *rng, int n4, int k4, int n2, int k2, int metrop,
                             int ovrn, double *out, int out_len) {
  u1i::NvtxRange nvtx_range("u1_multilevel");
  if (!lat || !rng || !out) return fail(U1_ERR_INVALID, "u1_multilevel: null argument");
  const GeomK &g = lat->g;
  if (g.dims != 4) return fail(U1_ERR_INVALID, "u1_multilevel: requires a 4D lattice");
  if (g.N[g.tdir] % 4 != 0)
    return fail(U1_ERR_INVALID, "u1_multilevel: Nt is not a multiple of 4 (reference src/multilevel.cu:641)");
  if (n4 < 1 || n2 < 1 || k4 < 0 || k2 < 0 || metrop < 0 || ovrn < 0)
    return fail(U1_ERR_INVALID, "u1_multilevel: bad iteration counts");
  const int R = g.N[0] / 2;
  if (out_len < 2 * R) return fail(U1_ERR_INVALID, "u1_multilevel: out_len < 2*R");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  const size_t size = (size_t)g.Vs * R * g.tdir;
  const int nl2 = g.N[g.tdir] / 2, nl4 = g.N[g.tdir] / 4;
  int rc = U1_OK;
  auto cleanup = [&]() { cudaStreamSynchronize(lat->stream); };
  // The work buffers (the links' working copy, slab products, T2, T4: about
  // 210 MB at 24^3 x 32) are allocated by the first call and kept with the
  // lattice, so later calls neither allocate nor synchronise the device.
  if (!lat->ml_work) {
    float2 *work = nullptr;
    double2 *P2 = nullptr, *T2 = nullptr, *T4 = nullptr;
    cudaError_t e = u1i::dev_alloc(&work, (size_t)g.V * g.dims * sizeof(float2));
    if (e == cudaSuccess) e = u1i::dev_alloc(&P2, (size_t)g.Vs * nl2 * sizeof(double2));
    if (e == cudaSuccess) e = u1i::dev_alloc(&T2, size * nl2 * sizeof(double2));
    if (e == cudaSuccess) e = u1i::dev_alloc(&T4, size * nl4 * sizeof(double2));
    if (e != cudaSuccess) {
      u1i::dev_free(work);
      u1i::dev_free(P2);
      u1i::dev_free(T2);
      u1i::dev_free(T4);
      u1i::set_error(std::string("u1_multilevel: allocation failed: ") + cudaGetErrorString(e));
      return U1_ERR_NOMEM;
    }
    lat->ml_work = work;
    lat->ml_P2 = P2;
    lat->ml_T2 = T2;
    lat->ml_T4 = T4;
  }
  float2 *const work = lat->ml_work;
  double2 *const P2 = lat->ml_P2, *const T2 = lat->ml_T2, *const T4 = lat->ml_T4;
  const int nb_s = u1i::blocks_for(g.Vs, kRedThreads);
  const MlDims md{g.N[0], g.N[1], g.N[2], g.Vs, R, nl2, nl4};
  rc = u1i::ensure_scratch(lat, (size_t)nb_s * 2 * R, (size_t)2 * R);
  if (rc) {
    cleanup();
    return rc;
  }
  // The level-4 update (k4 sweeps, freeze period 4) and one level-2
  // sub-update (k2 sweeps with freeze period 2, the multihit field, the T2
  // accumulation) are each captured once as a CUDA graph and replayed; the
  // Metropolis pass counter lives in device memory, so replays draw fresh
  // numbers exactly as direct launches would.
  auto level4 = [&]() -> int {
    for (int j = 0; j < k4; ++j) {
      int r = issue_sweep(lat, work, rng, metrop, ovrn, 4);
      if (r) return r;
    }
    return U1_OK;
  };
  auto level2 = [&]() -> int {
    for (int l = 0; l < k2; ++l) {
      int r = issue_sweep(lat, work, rng, metrop, ovrn, 2);
      if (r) return r;
    }
    k_ml_slab2<<<u1i::blocks_for((long long)g.Vs * nl2, 256), 256, 0, lat->stream>>>(work, g, lat->c, md, P2);
    U1_LAUNCH_CHECK("k_ml_slab2");
    k_ml_T2<<<u1i::blocks_for((long long)(size / 2) * nl2, 256), 256, 0, lat->stream>>>(P2, md, T2);
    U1_LAUNCH_CHECK("k_ml_T2");
    return U1_OK;
  };
  const unsigned long long per_sweep = 2ull * g.dims * (metrop + ovrn) + (ovrn == 0 ? 1 : 0);
  const bool graphed = lat->use_graphs && !rng->replay_dev;
  // the graphs of the last (k4, k2, metrop, ovrn, rng) are kept with the lattice
  const auto key = std::make_tuple(k4, k2, metrop, ovrn, rng->id, rng->seed ^ ((uint64_t)rng->chain << 48));
  auto body = [&]() -> int {
    U1_CUDA_TRY(cudaMemcpyAsync(work, lat->links, (size_t)g.V * g.dims * sizeof(float2),
                                cudaMemcpyDeviceToDevice, lat->stream));
    U1_CUDA_TRY(cudaMemsetAsync(T4, 0, size * nl4 * sizeof(double2), lat->stream));
    if (graphed && (!lat->ml_g2 || lat->ml_key != key)) {
      if (lat->ml_g4) cudaGraphExecDestroy(lat->ml_g4);
      if (lat->ml_g2) cudaGraphExecDestroy(lat->ml_g2);
      lat->ml_g4 = lat->ml_g2 = nullptr;
      lat->ml_key = std::make_tuple(-1, -1, -1, -1, (uint64_t)0, (uint64_t)0);
      if (k4 > 0) {
        int r = capture_graph(lat, level4, &lat->ml_g4);
        if (r) return r;
      }
      int r = capture_graph(lat, level2, &lat->ml_g2);
      if (r) return r;
      lat->ml_key = key;
    }
    cudaGraphExec_t g4 = lat->ml_g4, g2 = lat->ml_g2;
    for (int i = 0; i < n4; ++i) {
      if (graphed) {
        if (k4 > 0) {
          U1_CUDA_TRY(cudaGraphLaunch(g4, lat->stream));
          u1i::g_launches += per_sweep * (unsigned long long)k4;
        }
      } else {
        int r = level4();
        if (r) return r;
      }
      rng->pass += (uint64_t)metrop * (uint64_t)k4;
      U1_CUDA_TRY(cudaMemsetAsync(T2, 0, size * nl2 * sizeof(double2), lat->stream));
      for (int k = 0; k < n2; ++k) {
        if (graphed) {
          U1_CUDA_TRY(cudaGraphLaunch(g2, lat->stream));
          u1i::g_launches += per_sweep * (unsigned long long)k2 + 2ull;
        } else {
          int r = level2();
          if (r) return r;
        }
        rng->pass += (uint64_t)metrop * (uint64_t)k2;
      }
      k_ml_T4<<<u1i::blocks_for((long long)(size / 2) * nl4, 256), 256, 0, lat->stream>>>(T2, md, 1.0 / (double)n2,
                                                                                        T4);
      U1_LAUNCH_CHECK("k_ml_T4");
    }
    k_ml_final<<<nb_s, kRedThreads, 0, lat->stream>>>(T4, g, R, 1.0 / (double)n4, lat->partials, lat->counter,
                                                      lat->d_out, 1.0 / ((double)g.Vs * g.tdir));
    U1_LAUNCH_CHECK("k_ml_final");
    U1_CUDA_TRY(cudaMemcpyAsync(lat->h_out, lat->d_out, (size_t)2 * R * sizeof(double),
                                cudaMemcpyDeviceToHost, lat->stream));
    U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
    return U1_OK;
  };
  if (rng->replay_dev) {
    uint64_t need = (uint64_t)metrop * ((uint64_t)n4 * k4 + (uint64_t)n4 * n2 * k2);
    rc = check_replay(lat, rng, (int)need);
    if (rc) {
      cleanup();
      return rc;
    }
  }
  rc = body();
  cleanup();
  if (rc) return rc;
  memcpy(out, lat->h_out, (size_t)2 * R * sizeof(double));
  return U1_OK;
}
