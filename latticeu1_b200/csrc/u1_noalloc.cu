// u1_measure_noalloc: the fused plaquette + Polyakov measurement for callers
// that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code that must stay inside a fixed
// memory budget handed out by its host framework (every device byte comes
// from that framework's allocator), or latency-critical loops where a
// cudaMalloc/cudaFree could synchronise the device and stall other streams.
// u1_measure_async needs per-lattice scratch (per-block partial sums and a
// ticket counter) that the library allocates; this variant runs the same
// k_measure kernel with that scratch taken from a file-scope __device__
// array, so it allocates nothing.  The caller passes the links (inputs) and
// the 6-double result buffer (output), both device pointers.
//
// Limits and sharing:
//  * The array holds kNoAllocMaxBlocks blocks of partials (~384 KiB, kept by
//    every GPU that loads the library until the process exits), which
//    bounds the lattice at V/2 <= kNoAllocMaxPlaqBlocks * 256 sites
//    (V <= 2,097,152, e.g. 32^4 or 32^3 x 64); larger lattices are rejected
//    with U1_ERR_INVALID before any device work.
//  * Every call shares the one array, and it keeps the last call's contents.
//    The ticket counter is cleared at the start of each call (cudaMemsetAsync
//    on the caller's stream); the partials are fully overwritten before they
//    are read.  Calls whose kernels overlap on the GPU (e.g. on two streams
//    without ordering between them) race on the array.
//  * The first call on a device looks up the array's device address on that
//    device (cudaGetSymbolAddress, with the device current); make that first
//    call before any stream capture.  The address belongs to the device's
//    current CUDA context: when that context changes (cudaDeviceReset, or a
//    host framework that tears its context down and creates a new one) the
//    next call looks the address up again.  The current device must own
//    links, out and stream.
#include <cuda.h>
#include <mutex>
#include <string>

#include "u1_internal.h"
#include "u1_measure.cuh"

using namespace u1b;

namespace {

// Room for the measurement's plaquette blocks (at most V/2 / 256 <= 4096)
// plus its Polyakov blocks (V_s * chunks / 256 <= V/2 / 256, chunks <= Nt/2).
constexpr int kNoAllocMaxPlaqBlocks = 4096;
constexpr int kNoAllocMaxBlocks = 2 * kNoAllocMaxPlaqBlocks;
constexpr int kNoAllocMaxDevices = 64;
// partials (6 doubles per block) followed by one 256-byte slot whose first
// word is the ticket counter.
constexpr size_t kScratchDoubles = (size_t)kNoAllocMaxBlocks * 6 + 32;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_noalloc_mu;
struct ScratchAddr {
  CUcontext ctx = nullptr;  // context the address was looked up in
  double *addr = nullptr;
};
ScratchAddr g_noalloc_addr[kNoAllocMaxDevices];

// The driver's cuCtxGetCurrent, reached through the runtime (no link against
// libcuda); null if the driver does not provide it.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
CtxGetCurrentFn ctx_get_current() {
  static const CtxGetCurrentFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

// Device address of g_noalloc_scratch on the current device, looked up once
// per device and again whenever the device's current context changes.
int noalloc_scratch(double **out) {
  int dev = -1;
  U1_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    u1i::set_error("u1_measure_noalloc: device ordinal out of range");
    return U1_ERR_UNSUPPORTED;
  }
  CUcontext cur = nullptr;
  if (CtxGetCurrentFn f = ctx_get_current()) f(&cur);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  ScratchAddr &c = g_noalloc_addr[dev];
  if (!c.addr || c.ctx != cur) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return u1i::cuda_fail(e, "u1_measure_noalloc: cudaGetSymbolAddress");
    c.addr = (double *)p;
    c.ctx = cur;
  }
  *out = c.addr;
  return U1_OK;
}

template <int D>
int launch_noalloc(const float2 *links, const GeomK &g, double *scratch, double *out, cudaStream_t s) {
  const MeasK m = measure_layout(g);
  const int nb = m.nb_plaq + m.nb_poly;
  // Unreachable after the caller's V/2 check (nb_plaq <= V/2 / 256 and
  // nb_poly <= V/8 / 256); kept so the array can never be overrun.
  if (nb > kNoAllocMaxBlocks) {
    u1i::set_error("u1_measure_noalloc: measurement needs more blocks than the fixed scratch array holds");
    return U1_ERR_INVALID;
  }
  unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + (size_t)kNoAllocMaxBlocks * 6);
  U1_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned int), s));
  int nSS = 0, nST = 0;
  for (int mu = 0; mu < D - 1; ++mu)
    for (int nu = mu + 1; nu < D; ++nu) (nu == g.tdir ? nST : nSS)++;
  const double normSS = 1.0 / ((double)g.V * nSS);
  const double normST = 1.0 / ((double)g.V * nST);
  const double normL = 1.0 / (double)g.Vs;
  k_measure<D><<<nb, kRedThreads, 0, s>>>(links, g, m, scratch, counter, out, normSS, normST, normL);
  U1_LAUNCH_CHECK("k_measure (noalloc)");
  return U1_OK;
}

}  // namespace

extern "C" int u1_measure_noalloc(const void *links_dev, const u1_geom *geom, double *out_dev, void *stream) {
  if (!links_dev || !geom || !out_dev) {
    u1i::set_error("u1_measure_noalloc: null argument");
    return U1_ERR_INVALID;
  }
  GeomK g{};
  int rc = u1i::make_geom(geom, g);
  if (rc) return rc;
  if (g.Vh > kNoAllocMaxPlaqBlocks * kRedThreads) {
    u1i::set_error("u1_measure_noalloc: lattice too large for the fixed scratch array (V/2 = " +
                   std::to_string(g.Vh) + " > maximum " + std::to_string((long long)kNoAllocMaxPlaqBlocks * kRedThreads) +
                   " sites); use u1_measure_async");
    return U1_ERR_INVALID;
  }
  double *scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  const float2 *links = static_cast<const float2 *>(links_dev);
  cudaStream_t s = (cudaStream_t)stream;
  switch (g.dims) {
    case 2: return launch_noalloc<2>(links, g, scratch, out_dev, s);
    case 3: return launch_noalloc<3>(links, g, scratch, out_dev, s);
    default: return launch_noalloc<4>(links, g, scratch, out_dev, s);
  }
}
