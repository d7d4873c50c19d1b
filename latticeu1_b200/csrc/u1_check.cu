// Checked build support: the per-phase race check of the link-access marks
// and the C-ABI entry points that read the counters (include/u1_b200.h,
// u1_check_report, u1_check_selftest).  The checks themselves are chk() in
// u1_update.cuh; they are compiled in only with -DU1_BOUNDS_CHECK
// (libu1b200_check.so, a test build).  In the normal build the entry points
// return U1_ERR_UNSUPPORTED and nothing here is launched.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "u1_internal.h"
#include "u1_update.cuh"

using u1b::ChkState;

namespace {

int fail(int code, const std::string &msg) {
  u1i::set_error(msg);
  return code;
}

#ifdef U1_BOUNDS_CHECK
// After one phase: a link with a write mark (>= 2) that another thread also
// read (bit 0), or with two writes (>= 4), is a race.  Counts the races and
// the marked links, clears the marks and counts the phase.
__global__ void __launch_bounds__(256) k_chk_phase_end(unsigned *shadow, size_t n, ChkState *st) {
  unsigned long long races = 0, marked = 0;
  long long first = -1;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const unsigned w = shadow[k];
    if (w == 0u) continue;
    ++marked;
    if (w >= 4u || (w >= 2u && (w & 1u))) {
      ++races;
      if (first < 0) first = (long long)k;
    }
    shadow[k] = 0u;
  }
  if (marked) atomicAdd(&st->marked, marked);
  if (races && atomicAdd(&st->races, races) == 0ull) st->first_race_link = first;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&st->phases, 1ull);
}

// Self-test of the checker on a 16-link slab that is never dereferenced:
// two accesses the checks must refuse (a four-link access running past the
// half's end, a misaligned two-link access) and marks that make two races
// (link 3 written by one thread and read by another, link 5 written twice)
// and two clean links (7 read by two threads, 9 read and written by its
// owner).  One warp, one lane per access.
__global__ void k_chk_selftest(const float2 *slab, unsigned *shadow, ChkState *st) {
  const u1b::Chk c{st, shadow, slab, 16};
  switch (threadIdx.x) {
    case 0: u1b::chk<4, u1b::CHK_READ>(c, slab, 14); break;  // 14 + 4 > 16
    case 1: u1b::chk<2, u1b::CHK_READ>(c, slab, 1); break;   // 8-byte offset, 16-byte access
    case 2: u1b::chk<1, u1b::CHK_WRITE>(c, slab, 3); break;
    case 3: u1b::chk<1, u1b::CHK_READ>(c, slab, 3); break;
    case 4: u1b::chk<1, u1b::CHK_WRITE>(c, slab, 5); break;
    case 5: u1b::chk<1, u1b::CHK_WRITE>(c, slab, 5); break;
    case 6: u1b::chk<1, u1b::CHK_READ>(c, slab, 7); break;
    case 7: u1b::chk<1, u1b::CHK_READ>(c, slab, 7); break;
    case 8: u1b::chk<1, u1b::CHK_OWN>(c, slab, 9); break;
    case 9: u1b::chk<1, u1b::CHK_WRITE>(c, slab, 9); break;
    default: break;
  }
}

void report(const ChkState &h, int64_t out[8]) {
  out[0] = (int64_t)h.bad;
  out[1] = (int64_t)h.races;
  out[2] = (int64_t)h.phases;
  out[3] = (int64_t)h.marked;
  out[4] = h.first_bad_idx;
  out[5] = h.first_bad_half;
  out[6] = h.first_bad_kind;
  out[7] = h.first_race_link;
}
#endif

}  // namespace

namespace u1i {

ChkState *chk_state(u1_ctx *ctx) {
#ifdef U1_BOUNDS_CHECK
  if (!ctx->chk) {
    ChkState *p = nullptr;
    if (dev_alloc(&p, sizeof(ChkState)) != cudaSuccess) return nullptr;
    ChkState z{};
    z.first_bad_idx = z.first_race_link = -1;
    if (cudaMemcpy(p, &z, sizeof(z), cudaMemcpyHostToDevice) != cudaSuccess) {
      dev_free(p);
      return nullptr;
    }
    ctx->chk = p;
  }
  return ctx->chk;
#else
  (void)ctx;
  return nullptr;
#endif
}

unsigned *chk_shadow(size_t n) {
#ifdef U1_BOUNDS_CHECK
  unsigned *p = nullptr;
  if (dev_alloc(&p, n * sizeof(unsigned)) != cudaSuccess) return nullptr;
  if (cudaMemset(p, 0, n * sizeof(unsigned)) != cudaSuccess) {
    dev_free(p);
    return nullptr;
  }
  return p;
#else
  (void)n;
  return nullptr;
#endif
}

int chk_phase_end(cudaStream_t s, unsigned *shadow, size_t n, ChkState *st) {
#ifdef U1_BOUNDS_CHECK
  if (!shadow || !st) return U1_OK;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
  k_chk_phase_end<<<blocks, 256, 0, s>>>(shadow, n, st);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "k_chk_phase_end");
#else
  (void)s;
  (void)shadow;
  (void)n;
  (void)st;
#endif
  return U1_OK;
}

}  // namespace u1i

extern "C" int u1_check_report(u1_ctx *ctx, int64_t out[8], int reset) {
  if (!ctx || !out) return fail(U1_ERR_INVALID, "u1_check_report: null argument");
#ifdef U1_BOUNDS_CHECK
  U1_CUDA_TRY(cudaSetDevice(ctx->device));
  ChkState *st = u1i::chk_state(ctx);
  if (!st) return fail(U1_ERR_NOMEM, "u1_check_report: no device memory for the counters");
  U1_CUDA_TRY(cudaDeviceSynchronize());
  ChkState h{};
  U1_CUDA_TRY(cudaMemcpy(&h, st, sizeof(h), cudaMemcpyDeviceToHost));
  report(h, out);
  if (reset) {
    ChkState z{};
    z.first_bad_idx = z.first_race_link = -1;
    U1_CUDA_TRY(cudaMemcpy(st, &z, sizeof(z), cudaMemcpyHostToDevice));
  }
  return U1_OK;
#else
  (void)reset;
  std::memset(out, 0, 8 * sizeof(int64_t));
  return fail(U1_ERR_UNSUPPORTED, "u1_check_report: not a checked build (libu1b200_check.so has the checks)");
#endif
}

extern "C" int u1_check_selftest(u1_ctx *ctx, int64_t out[8]) {
  if (!ctx || !out) return fail(U1_ERR_INVALID, "u1_check_selftest: null argument");
#ifdef U1_BOUNDS_CHECK
  U1_CUDA_TRY(cudaSetDevice(ctx->device));
  // one allocation: the counters, 16 shadow words, then the 16-link slab
  // (256-byte aligned from the allocator, so the slab is 16-byte aligned)
  char *buf = nullptr;
  const size_t off_shadow = 256, off_slab = 512, bytes = 512 + 16 * sizeof(float2);
  U1_CUDA_TRY(u1i::dev_alloc(&buf, bytes));
  ChkState z{};
  z.first_bad_idx = z.first_race_link = -1;
  cudaError_t e = cudaMemset(buf, 0, bytes);
  if (e == cudaSuccess) e = cudaMemcpy(buf, &z, sizeof(z), cudaMemcpyHostToDevice);
  ChkState *st = reinterpret_cast<ChkState *>(buf);
  unsigned *shadow = reinterpret_cast<unsigned *>(buf + off_shadow);
  const float2 *slab = reinterpret_cast<const float2 *>(buf + off_slab);
  if (e == cudaSuccess) {
    k_chk_selftest<<<1, 32>>>(slab, shadow, st);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_chk_phase_end<<<1, 256>>>(shadow, 16, st);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  ChkState h{};
  if (e == cudaSuccess) e = cudaMemcpy(&h, st, sizeof(h), cudaMemcpyDeviceToHost);
  u1i::dev_free(buf);
  if (e != cudaSuccess) return u1i::cuda_fail(e, "u1_check_selftest");
  report(h, out);
  return U1_OK;
#else
  std::memset(out, 0, 8 * sizeof(int64_t));
  return fail(U1_ERR_UNSUPPORTED, "u1_check_selftest: not a checked build (libu1b200_check.so has the checks)");
#endif
}
