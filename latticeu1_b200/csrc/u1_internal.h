// Host-side object layout behind the C ABI (include/u1_b200.h).
#pragma once
#include <nvtx3/nvToolsExt.h>
#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <string>
#include <tuple>

#include "u1_b200.h"
#include "u1_geom.cuh"

namespace u1b {
struct ChkState;
}

struct u1_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaDeviceProp prop{};
  u1b::ChkState *chk = nullptr;     // checked build: access-check counters (device)
};

struct u1_rng {
  u1_ctx *ctx = nullptr;
  uint64_t seed = 0;
  uint64_t pass = 0;                        // host mirror of *pass_dev
  unsigned long long *pass_dev = nullptr;   // device pass counter
  double *replay_dev = nullptr;             // shared-stream pairs (test mode)
  size_t replay_pairs = 0;
  uint64_t replay_base = 0;                 // pass number of the first replay pass
  uint32_t chain = 0;
  uint64_t id = 0;                          // unique per rng object (graph cache key)
};

// Update kernel variants (all bit-identical; the tuner picks the fastest).
enum : int { U1V_AUTO = 0, U1V_PAIR32 = 1, U1V_PAIR = 2, U1V_SINGLE = 3, U1V_WAVE = 4, U1V_QUAD = 5 };

struct u1_lattice {
  u1_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  u1b::GeomK g{};
  u1b::CoupK c{};
  double beta = 0.0, aniso = 1.0;
  float2 *links = nullptr;          // V*dims
  // scratch for reductions: per-block partials + ticket counter
  double *partials = nullptr;
  size_t partials_cap = 0;          // doubles
  unsigned int *counter = nullptr;
  double *d_out = nullptr;          // small device result buffer
  size_t d_out_cap = 0;
  double *h_out = nullptr;          // pinned host result buffer
  size_t h_out_cap = 0;
  double2 *pfield = nullptr;        // Polyakov-loop field (V_s)
  double *stage = nullptr;          // FP64 angle staging buffer for host import/export (V*dims)
  cudaStream_t own_stream = nullptr; // used when no stream is attached
  // cached CUDA graphs of whole sweeps, keyed by (metrop, ovrn, rng id, seed)
  std::map<std::tuple<int, int, uint64_t, uint64_t>, cudaGraphExec_t> graphs;
  bool use_graphs = true;
  int variant = U1V_AUTO;          // update kernel variant (U1V_AUTO: tune on first update)
  int block = 256;                 // threads per block of the phase kernels (tuned with the variant)
  int remap_block = -1;            // block size remap_sms was worked out for
  int remap_sms = 0;               // SM-local block order of the four-site kernels (0: launch order)
  // Metropolis proposal: half-width delta (0: the reference's whole-circle
  // theta' = 2 pi u), win = delta/pi as used by the kernels, hits per link
  double delta = 0.0;
  float win = 0.f;
  int nhits = 1;
  float2 *backup = nullptr;        // link backup used while tuning
  // persistent sweep (U1V_WAVE): per-tile phase flags, then ticket and error word
  unsigned int *wave_state = nullptr;
  int wave_ok = -1;                // -1 unknown, 0 not usable, 1 usable
  // multilevel (u1_multilevel): work copy of the links, level-2 slab products,
  // T2 and T4, kept from the first call until the lattice is destroyed, and
  // the level-4 / level-2 graphs of the last (k4, k2, metrop, ovrn, rng) used
  float2 *ml_work = nullptr;
  double2 *ml_P2 = nullptr, *ml_T2 = nullptr, *ml_T4 = nullptr;
  std::tuple<int, int, int, int, uint64_t, uint64_t> ml_key{-1, -1, -1, -1, 0, 0};
  cudaGraphExec_t ml_g4 = nullptr, ml_g2 = nullptr;
  unsigned wave_spin_limit = 0;    // polls per neighbour wait (0: the kernel's default)
  int wave_stall_tile = -1;        // test hook: this tile never publishes its phases (-1: none)
  unsigned *shadow = nullptr;      // checked build: per-link access marks (V*dims words)
};

namespace u1i {
// NVTX range around a host entry point: named ranges for nsys / ncu
// (--nvtx --nvtx-include); without an attached tool the push and pop return
// at once.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};
void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
extern std::atomic<unsigned long long> g_launches;
int ensure_scratch(u1_lattice *lat, size_t partial_doubles, size_t out_doubles);
// Tuning trials: the shortest of `reps` individually timed replays of graph
// `ex` on stream `s` after `warm` untimed ones, in microseconds.  The
// shortest replay is insensitive to clock ramps and power-cap drift that an
// average over back-to-back replays picks up.
cudaError_t time_graph_min(cudaGraphExec_t ex, cudaStream_t s, int warm, int reps, double *us);
// Replay `ex` for at least `ms` milliseconds of device time (clock warm-up
// before the first trial of a tuning run).
cudaError_t warm_clocks(cudaGraphExec_t ex, cudaStream_t s, double ms);
// U1_TUNE_VERBOSE=1: tuners print every trial to stderr.
bool tune_verbose();
// Every device allocation of the library: cudaMalloc / cudaFree unless the
// caller installed its own pair (u1_set_device_allocator).  A failed
// allocation returns cudaErrorMemoryAllocation and leaves *p null.
cudaError_t dev_alloc(void **p, size_t bytes);
cudaError_t dev_free(void *p);
template <class T>
inline cudaError_t dev_alloc(T **p, size_t bytes) {
  void *v = nullptr;
  cudaError_t e = dev_alloc(&v, bytes);
  *p = static_cast<T *>(v);
  return e;
}
// Checked build (-DU1_BOUNDS_CHECK): counters of the context (allocated on
// first use) and a zeroed shadow of n words; elsewhere both return null.
u1b::ChkState *chk_state(u1_ctx *ctx);
unsigned *chk_shadow(size_t n);
// Checked build: the race check and reset of the shadow after one phase on
// stream s (no-op when shadow is null or in the normal build).
int chk_phase_end(cudaStream_t s, unsigned *shadow, size_t n, u1b::ChkState *st);
// Geometry from the ABI struct (Grid mapping of the reference's
// SetupLatticeParameters); U1_ERR_INVALID on odd extents.
int make_geom(const u1_geom *geom, u1b::GeomK &g);
}  // namespace u1i

#define U1_CUDA_TRY(call)                                            \
  do {                                                               \
    cudaError_t _e = (call);                                         \
    if (_e != cudaSuccess) return u1i::cuda_fail(_e, #call);         \
  } while (0)

#define U1_LAUNCH_CHECK(what)                                        \
  do {                                                               \
    u1i::g_launches.fetch_add(1, std::memory_order_relaxed);         \
    cudaError_t _e = cudaGetLastError();                             \
    if (_e != cudaSuccess) return u1i::cuda_fail(_e, what);          \
  } while (0)
