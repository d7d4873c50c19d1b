// Many independent chains advanced together: one launch per (parity, mu)
// phase covers every chain of the batch.
//
// The reference runs one lattice per process (u1.cpp:99-120); here a batch
// holds chains of any 4D/3D/2D geometry (one dims per batch) and coupling.
// A block->chain table (built on the host) maps each CTA to its chain; the
// chain's geometry, coupling and link pointer sit in a device table that a
// block stages in shared memory.  Each chain draws from the batch's Philox
// key with its own chain number in the counter, so chain c of a batch is
// bit-identical to a single lattice run with the same seed and chain c
// (same update bodies, same counters).  Whole sweeps are captured once into
// a CUDA graph and replayed.  Per-chain plaquette/Polyakov results come from
// per-block partials summed in block order by one CTA per chain.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <array>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "u1_internal.h"
#include "u1_measure.cuh"

using namespace u1b;

namespace {

struct BatchChain {
  float2 *links;
  GeomK g;
  CoupK c;
  uint32_t chain;
  int first_pair;   // first block in the pair (two sites / thread) table
  int first_site;   // first block in the site (one site / thread) table
  int first_quad;   // first block in the quad (four sites / thread) table
  int first_meas;   // first block in the measurement table
  MeasK meas;       // measurement layout (plaquette blocks, then Polyakov blocks)
  int nb_meas;
  double norm[3];   // 1/(V nSS), 1/(V nST), 1/V_s
};

struct BatchPhase {
  int p;
  int hit;
  int block_base;  // first block of the chain group this launch covers
  uint32_t key0, key1;
  const unsigned long long *pass_dev;
  unsigned long long *bump_ptr;
  unsigned int bump_by;
};

__device__ __forceinline__ void stage_chain(const BatchChain *__restrict__ chains, int c, BatchChain &sch) {
  constexpr int words = (int)(sizeof(BatchChain) / 4);
  static_assert(sizeof(BatchChain) % 4 == 0, "BatchChain is copied as 32-bit words");
  const uint32_t *src = reinterpret_cast<const uint32_t *>(chains + c);
  uint32_t *dst = reinterpret_cast<uint32_t *>(&sch);
  for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = __ldg(src + w);
  __syncthreads();
}

// The kernel arguments of block `blk` of a batch phase (the block's chain
// staged in shared memory).
__device__ __forceinline__ UpdArgs batch_args(const BatchChain &sch, const BatchPhase &ph, int mu) {
  UpdArgs a{};
  a.lat = sch.links;
  a.g = sch.g;
  a.c = sch.c;
  a.p = ph.p;
  a.mu = mu;
  a.key0 = ph.key0;
  a.key1 = ph.key1;
  a.chain = sch.chain;
  a.pass_dev = ph.pass_dev;
  a.hit = ph.hit;
  a.bump_ptr = ph.bump_ptr;
  a.bump_by = ph.bump_by;
  return a;
}

// Four sites per thread (every chain of the launch's group has N0/2 a
// multiple of 4), 128 threads and 512 sites per block, as k_update_quad.
template <int D, int MU, bool MET>
__global__ void __launch_bounds__(128, 7)
    k_batch_update_quad(const BatchChain *__restrict__ chains, const int *__restrict__ block_chain, BatchPhase ph) {
  __shared__ BatchChain sch;
  const int blk = (int)blockIdx.x + ph.block_base;
  stage_chain(chains, __ldg(block_chain + blk), sch);
  const UpdArgs a = batch_args(sch, ph, MU);
  update_quad_body<D, MU, MET, SRC_PHILOX>(a, 4 * ((blk - sch.first_quad) * (int)blockDim.x + (int)threadIdx.x));
}

template <int D, int MU, bool MET, bool PAIR>
__global__ void __launch_bounds__(256, 8)
    k_batch_update(const BatchChain *__restrict__ chains, const int *__restrict__ block_chain, BatchPhase ph) {
  __shared__ BatchChain sch;
  const int blk = (int)blockIdx.x + ph.block_base;
  const int cidx = __ldg(block_chain + blk);
  stage_chain(chains, cidx, sch);
  UpdArgs a{};
  a.lat = sch.links;
  a.g = sch.g;
  a.c = sch.c;
  a.p = ph.p;
  a.mu = MU;
  a.key0 = ph.key0;
  a.key1 = ph.key1;
  a.chain = sch.chain;
  a.pass_dev = ph.pass_dev;
  a.hit = ph.hit;
  a.bump_ptr = ph.bump_ptr;
  a.bump_by = ph.bump_by;
  const int local = blk - (PAIR ? sch.first_pair : sch.first_site);
  if (PAIR)
    update_pair_body<D, MU, MET, SRC_PHILOX>(a, 2 * (local * blockDim.x + threadIdx.x));
  else
    update_single_body<D, MU, MET, SRC_PHILOX>(a, local * blockDim.x + threadIdx.x);
}

template <int D>
__global__ void __launch_bounds__(256)
    k_batch_hot_start(const BatchChain *__restrict__ chains, const int *__restrict__ block_chain, uint32_t key0,
                      uint32_t key1, unsigned long long pass) {
  __shared__ BatchChain sch;
  stage_chain(chains, __ldg(block_chain + blockIdx.x), sch);
  const int i = ((int)blockIdx.x - sch.first_site) * blockDim.x + threadIdx.x;
  if (i >= sch.g.Vh) return;
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int mu = 0; mu < D; ++mu) {
      Philox4 r = philox4x32_10((uint32_t)(p * sch.g.Vh + i), u1_rng_word1(mu, U1_TAG_HOTSTART, sch.chain),
                                (uint32_t)pass, (uint32_t)(pass >> 32), key0, key1);
      float sn, cs;
      sincospif(2.0f * u1_uniform_open(r.v[0]), &sn, &cs);
      sch.links[(size_t)mu * sch.g.V + (size_t)p * sch.g.Vh + i] = make_float2(cs, sn);
    }
}

template <int D>
__global__ void __launch_bounds__(kRedThreads)
    k_batch_measure(const BatchChain *__restrict__ chains, const int *__restrict__ block_chain, double *partials) {
  __shared__ BatchChain sch;
  __shared__ double smem[kRedWarps * 6];
  __shared__ float2 lp[kRedThreads];
  stage_chain(chains, __ldg(block_chain + blockIdx.x), sch);
  float vs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const int local = (int)blockIdx.x - sch.first_meas;
  measure_block_values<D>(sch.links, sch.g, local, sch.meas, vs, lp);
  const double tot = measure_block_total(vs, local < sch.meas.nb_plaq, smem);
  if (threadIdx.x < 6) partials[(size_t)blockIdx.x * 6 + threadIdx.x] = tot;
}

// One CTA per chain: sum the chain's measurement blocks in block order.
__global__ void __launch_bounds__(kRedThreads)
    k_batch_measure_finish(const BatchChain *__restrict__ chains, const double *__restrict__ partials, double *out) {
  __shared__ BatchChain sch;
  __shared__ double smem[kRedWarps * 6];
  stage_chain(chains, blockIdx.x, sch);
  double w[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) w[k] = strided_partial_sum(partials + (size_t)sch.first_meas * 6, sch.nb_meas, 6, k);
  block_sum<6>(w, smem);
  if (threadIdx.x < 6) out[(size_t)blockIdx.x * 6 + threadIdx.x] = w[0] * sch.norm[threadIdx.x / 2];
}

}  // namespace

struct u1_batch {
  u1_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  int dims = 0, n = 0;
  bool pair_ok = true;
  uint64_t seed = 0;
  uint64_t pass = 0;                       // host mirror of *pass_dev
  unsigned long long *pass_dev = nullptr;
  std::vector<BatchChain> h_chains;
  BatchChain *d_chains = nullptr;
  float2 *links = nullptr;
  size_t total_links = 0;
  int *d_tab_pair = nullptr, *d_tab_site = nullptr, *d_tab_meas = nullptr, *d_tab_quad = nullptr;
  int nb_pair = 0, nb_site = 0, nb_meas = 0, nb_quad = 0;
  double *partials = nullptr, *d_out = nullptr, *h_out = nullptr;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  // Chain groups swept one after another: consecutive chains whose links
  // together fit comfortably in L2, so that after a group's first phase its
  // links are served from L2.  Each: first pair block, pair blocks, first
  // site block, site blocks, first quad block, quad blocks (0 unless every
  // chain of the group takes four sites per thread).
  std::vector<std::array<int, 6>> groups;
};

using u1i::cuda_fail;

static inline int nblocks(long long n, int threads) { return (int)((n + threads - 1) / threads); }

static int bfail(int code, const std::string &msg) {
  u1i::set_error(msg);
  return code;
}

extern "C" int u1_batch_destroy(u1_batch *b) {
  if (!b) return U1_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->stream);
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  cudaFree(b->links);
  cudaFree(b->d_chains);
  cudaFree(b->d_tab_pair);
  cudaFree(b->d_tab_site);
  cudaFree(b->d_tab_meas);
  cudaFree(b->d_tab_quad);
  cudaFree(b->partials);
  cudaFree(b->d_out);
  cudaFree(b->pass_dev);
  if (b->h_out) cudaFreeHost(b->h_out);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
  return U1_OK;
}

extern "C" int u1_batch_create(u1_ctx *ctx, int nchains, const u1_geom *geoms, uint64_t seed, uint32_t first_chain,
                               u1_batch **out) {
  if (!ctx || !geoms || !out || nchains < 1) return bfail(U1_ERR_INVALID, "u1_batch_create: bad argument");
  if ((uint64_t)first_chain + (uint64_t)nchains > 65536u)
    return bfail(U1_ERR_INVALID, "u1_batch_create: chain numbers must stay below 65536");
  *out = nullptr;
  U1_CUDA_TRY(cudaSetDevice(ctx->device));
  u1_batch *b = new u1_batch;
  b->ctx = ctx;
  b->n = nchains;
  b->seed = seed;
  b->h_chains.resize(nchains);
  std::vector<int> tab_pair, tab_site, tab_meas, tab_quad;
  size_t off = 0;
  std::vector<size_t> offsets(nchains);
  for (int c = 0; c < nchains; ++c) {
    GeomK g{};
    int rc = u1i::make_geom(&geoms[c], g);
    if (rc) {
      delete b;
      return rc;
    }
    if (!(geoms[c].aniso > 0.0)) {
      delete b;
      return bfail(U1_ERR_INVALID, "u1_batch_create: aniso must be > 0");
    }
    if (c == 0) b->dims = g.dims;
    if (g.dims != b->dims) {
      delete b;
      return bfail(U1_ERR_UNSUPPORTED, "u1_batch_create: all chains of a batch must have the same dims");
    }
    if (g.hN0 & 1) b->pair_ok = false;
    BatchChain &ch = b->h_chains[c];
    ch.g = g;
    ch.c.beta = (float)geoms[c].beta;
    ch.c.w_ss = (float)(1.0 / geoms[c].aniso);
    ch.c.w_st = (float)geoms[c].aniso;
    ch.chain = first_chain + (uint32_t)c;
    offsets[c] = off;
    off += (size_t)g.V * g.dims;
    int nSS = 0, nST = 0;
    for (int mu = 0; mu < g.dims - 1; ++mu)
      for (int nu = mu + 1; nu < g.dims; ++nu) (nu == g.dims - 1 ? nST : nSS)++;
    ch.norm[0] = 1.0 / ((double)g.V * nSS);
    ch.norm[1] = 1.0 / ((double)g.V * nST);
    ch.norm[2] = 1.0 / (double)g.Vs;
    const int np = nblocks(g.Vh / 2, 256), ns = nblocks(g.Vh, 256);
    const int nq = (g.hN0 & 3) == 0 ? nblocks(g.Vh / 4, 128) : 0;
    ch.first_pair = (int)tab_pair.size();
    ch.first_site = (int)tab_site.size();
    ch.first_quad = (int)tab_quad.size();
    tab_quad.insert(tab_quad.end(), nq, c);
    ch.first_meas = (int)tab_meas.size();
    ch.meas = measure_layout(g);
    ch.nb_meas = ch.meas.nb_plaq + ch.meas.nb_poly;
    tab_pair.insert(tab_pair.end(), np, c);
    tab_site.insert(tab_site.end(), ns, c);
    tab_meas.insert(tab_meas.end(), ch.nb_meas, c);
  }
  b->total_links = off;
  b->nb_pair = (int)tab_pair.size();
  b->nb_site = (int)tab_site.size();
  b->nb_meas = (int)tab_meas.size();
  b->nb_quad = (int)tab_quad.size();
  {
    // groups of at most U1_BATCH_GROUP_MB (default 64) MiB of links; a
    // single chain may exceed it; 0 puts every chain in one group
    size_t kGroupBytes = 64ull << 20;
    if (const char *env = std::getenv("U1_BATCH_GROUP_MB")) {
      const long long mb = std::atoll(env);
      kGroupBytes = mb > 0 ? (size_t)mb << 20 : SIZE_MAX;
    }
    // U1_BATCH_QUAD=0 keeps every group on the two-site (or one-site) kernel
    const char *qenv = std::getenv("U1_BATCH_QUAD");
    const bool quad_enabled = !(qenv && qenv[0] == '0');
    size_t bytes = 0;
    int c0 = 0;
    auto close_group = [&](int c1) {
      const BatchChain &a = b->h_chains[c0];
      const int pair_end = c1 < nchains ? b->h_chains[c1].first_pair : b->nb_pair;
      const int site_end = c1 < nchains ? b->h_chains[c1].first_site : b->nb_site;
      bool quad = quad_enabled;
      for (int c = c0; c < c1; ++c) quad = quad && (b->h_chains[c].g.hN0 & 3) == 0;
      const int quad_end = c1 < nchains ? b->h_chains[c1].first_quad : b->nb_quad;
      b->groups.push_back({a.first_pair, pair_end - a.first_pair, a.first_site, site_end - a.first_site,
                           a.first_quad, quad ? quad_end - a.first_quad : 0});
    };
    for (int c = 0; c < nchains; ++c) {
      const size_t cb = (size_t)b->h_chains[c].g.V * b->h_chains[c].g.dims * sizeof(float2);
      if (c > c0 && bytes + cb > kGroupBytes) {
        close_group(c);
        c0 = c;
        bytes = 0;
      }
      bytes += cb;
    }
    close_group(nchains);
  }
  cudaError_t e = cudaStreamCreate(&b->own_stream);
  b->stream = ctx->stream ? ctx->stream : b->own_stream;
  if (e == cudaSuccess) e = cudaMalloc(&b->links, b->total_links * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_chains, sizeof(BatchChain) * nchains);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_tab_pair, sizeof(int) * tab_pair.size());
  if (e == cudaSuccess) e = cudaMalloc(&b->d_tab_site, sizeof(int) * tab_site.size());
  if (e == cudaSuccess) e = cudaMalloc(&b->d_tab_meas, sizeof(int) * tab_meas.size());
  if (e == cudaSuccess) e = cudaMalloc(&b->d_tab_quad, sizeof(int) * std::max<size_t>(1, tab_quad.size()));
  if (e == cudaSuccess) e = cudaMalloc(&b->partials, sizeof(double) * 6 * tab_meas.size());
  if (e == cudaSuccess) e = cudaMalloc(&b->d_out, sizeof(double) * 6 * nchains);
  if (e == cudaSuccess) e = cudaMallocHost(&b->h_out, sizeof(double) * 6 * nchains);
  if (e == cudaSuccess) e = cudaMalloc(&b->pass_dev, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(b->pass_dev, 0, sizeof(unsigned long long));
  if (e != cudaSuccess) {
    u1_batch_destroy(b);
    u1i::set_error(std::string("u1_batch_create: ") + cudaGetErrorString(e));
    return U1_ERR_NOMEM;
  }
  for (int c = 0; c < nchains; ++c) b->h_chains[c].links = b->links + offsets[c];
  e = cudaMemcpy(b->d_chains, b->h_chains.data(), sizeof(BatchChain) * nchains, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_tab_pair, tab_pair.data(), sizeof(int) * tab_pair.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_tab_site, tab_site.data(), sizeof(int) * tab_site.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !tab_quad.empty())
    e = cudaMemcpy(b->d_tab_quad, tab_quad.data(), sizeof(int) * tab_quad.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_tab_meas, tab_meas.data(), sizeof(int) * tab_meas.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    u1_batch_destroy(b);
    return cuda_fail(e, "u1_batch_create: upload");
  }
  // cold start
  for (int c = 0; c < nchains; ++c) {
    const size_t nl = (size_t)b->h_chains[c].g.V * b->h_chains[c].g.dims;
    std::vector<float2> one(nl, make_float2(1.f, 0.f));
    e = cudaMemcpy(b->h_chains[c].links, one.data(), nl * sizeof(float2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      u1_batch_destroy(b);
      return cuda_fail(e, "u1_batch_create: cold start");
    }
  }
  *out = b;
  return U1_OK;
}

extern "C" int u1_batch_set_stream(u1_batch *b, void *stream) {
  if (!b) return bfail(U1_ERR_INVALID, "u1_batch_set_stream: null batch");
  b->stream = stream ? (cudaStream_t)stream : b->own_stream;
  return U1_OK;
}

extern "C" int u1_batch_info(const u1_batch *b, int64_t out[4]) {
  if (!b || !out) return bfail(U1_ERR_INVALID, "u1_batch_info: null argument");
  out[0] = b->n;
  out[1] = b->dims;
  out[2] = (int64_t)b->total_links;
  out[3] = b->pair_ok ? 1 : 0;
  return U1_OK;
}

extern "C" int u1_batch_groups(const u1_batch *b, int *groups) {
  if (!b || !groups) return bfail(U1_ERR_INVALID, "u1_batch_groups: null argument");
  *groups = (int)b->groups.size();
  return U1_OK;
}

extern "C" int u1_batch_hot_start(u1_batch *b) {
  if (!b) return bfail(U1_ERR_INVALID, "u1_batch_hot_start: null batch");
  U1_CUDA_TRY(cudaSetDevice(b->ctx->device));
  const uint32_t k0 = (uint32_t)b->seed, k1 = (uint32_t)(b->seed >> 32);
  switch (b->dims) {
    case 2: k_batch_hot_start<2><<<b->nb_site, 256, 0, b->stream>>>(b->d_chains, b->d_tab_site, k0, k1, b->pass); break;
    case 3: k_batch_hot_start<3><<<b->nb_site, 256, 0, b->stream>>>(b->d_chains, b->d_tab_site, k0, k1, b->pass); break;
    default: k_batch_hot_start<4><<<b->nb_site, 256, 0, b->stream>>>(b->d_chains, b->d_tab_site, k0, k1, b->pass);
  }
  U1_LAUNCH_CHECK("k_batch_hot_start");
  k_pass_add<<<1, 1, 0, b->stream>>>(b->pass_dev, 1ull);
  U1_LAUNCH_CHECK("k_pass_add");
  b->pass += 1;
  return U1_OK;
}

template <int D, int MU, bool MET>
static int batch_launch_quad(u1_batch *b, BatchPhase ph, int group) {
  const std::array<int, 6> &gr = b->groups[group];
  ph.block_base = gr[4];
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)gr[5]);
  cfg.blockDim = dim3(128);
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_batch_update_quad<D, MU, MET>, (const BatchChain *)b->d_chains,
                                     (const int *)b->d_tab_quad, ph);
  u1i::g_launches.fetch_add(1, std::memory_order_relaxed);
  if (e != cudaSuccess) return cuda_fail(e, "k_batch_update_quad");
  return U1_OK;
}

template <int D, int MU, bool MET, bool PAIR>
static int batch_launch(u1_batch *b, BatchPhase ph, int group) {
  const std::array<int, 6> &gr = b->groups[group];
  ph.block_base = PAIR ? gr[0] : gr[2];
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(PAIR ? gr[1] : gr[3]));
  cfg.blockDim = dim3(256);
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_batch_update<D, MU, MET, PAIR>, (const BatchChain *)b->d_chains,
                                     (const int *)(PAIR ? b->d_tab_pair : b->d_tab_site), ph);
  u1i::g_launches.fetch_add(1, std::memory_order_relaxed);
  if (e != cudaSuccess) return cuda_fail(e, "k_batch_update");
  return U1_OK;
}

template <int D, int MU>
static int batch_launch_mu(u1_batch *b, const BatchPhase &ph, bool met, int group) {
  if (b->groups[group][5] > 0)
    return met ? batch_launch_quad<D, MU, true>(b, ph, group) : batch_launch_quad<D, MU, false>(b, ph, group);
  if (b->pair_ok)
    return met ? batch_launch<D, MU, true, true>(b, ph, group) : batch_launch<D, MU, false, true>(b, ph, group);
  return met ? batch_launch<D, MU, true, false>(b, ph, group) : batch_launch<D, MU, false, false>(b, ph, group);
}

template <int D>
static int batch_phase(u1_batch *b, const BatchPhase &ph, int mu, bool met, int group) {
  switch (mu) {
    case 0: return batch_launch_mu<D, 0>(b, ph, met, group);
    case 1: return batch_launch_mu<D, 1>(b, ph, met, group);
    case 2:
      if constexpr (D > 2) return batch_launch_mu<D, 2>(b, ph, met, group);
      break;
    case 3:
      if constexpr (D > 3) return batch_launch_mu<D, 3>(b, ph, met, group);
      break;
  }
  return bfail(U1_ERR_INVALID, "batch phase: direction out of range");
}

template <int D>
static int batch_measure_launch(u1_batch *b) {
  k_batch_measure<D><<<b->nb_meas, kRedThreads, 0, b->stream>>>(b->d_chains, b->d_tab_meas, b->partials);
  U1_LAUNCH_CHECK("k_batch_measure");
  k_batch_measure_finish<<<b->n, kRedThreads, 0, b->stream>>>(b->d_chains, b->partials, b->d_out);
  U1_LAUNCH_CHECK("k_batch_measure_finish");
  return U1_OK;
}

static int batch_measure_issue(u1_batch *b) {
  switch (b->dims) {
    case 2: return batch_measure_launch<2>(b);
    case 3: return batch_measure_launch<3>(b);
    default: return batch_measure_launch<4>(b);
  }
}

static int batch_issue_sweep(u1_batch *b, int metrop, int ovrn, bool measure) {
  BatchPhase ph{};
  ph.key0 = (uint32_t)b->seed;
  ph.key1 = (uint32_t)(b->seed >> 32);
  ph.pass_dev = b->pass_dev;
  const int D = b->dims;
  const int ngroups = (int)b->groups.size();
  // Each chain group runs the whole sweep before the next starts.  Every
  // group's Metropolis phases read the same pass counter; the first
  // overrelaxation kernel of the last group (after all of them) bumps it.
  bool bumped = (metrop == 0);
  for (int grp = 0; grp < ngroups; ++grp) {
    auto run = [&](int mu, bool met) {
      return D == 2 ? batch_phase<2>(b, ph, mu, met, grp)
           : D == 3 ? batch_phase<3>(b, ph, mu, met, grp)
                    : batch_phase<4>(b, ph, mu, met, grp);
    };
    for (int m = 0; m < metrop; ++m)
      for (int p = 0; p < 2; ++p)
        for (int mu = 0; mu < D; ++mu) {
          ph.p = p;
          ph.hit = m;
          ph.bump_ptr = nullptr;
          int rc = run(mu, true);
          if (rc) return rc;
        }
    for (int o = 0; o < ovrn; ++o)
      for (int p = 0; p < 2; ++p)
        for (int mu = 0; mu < D; ++mu) {
          ph.p = p;
          ph.hit = 0;
          const bool carry = !bumped && grp == ngroups - 1;
          ph.bump_ptr = carry ? b->pass_dev : nullptr;
          ph.bump_by = (unsigned)metrop;
          if (carry) bumped = true;
          int rc = run(mu, false);
          if (rc) return rc;
        }
  }
  if (!bumped) {  // no overrelaxation kernel carried the pass-counter bump
    k_pass_add<<<1, 1, 0, b->stream>>>(b->pass_dev, (unsigned long long)metrop);
    U1_LAUNCH_CHECK("k_pass_add");
  }
  if (measure) return batch_measure_issue(b);
  return U1_OK;
}

extern "C" int u1_batch_update(u1_batch *b, int metrop, int ovrn, int measure) {
  if (!b) return bfail(U1_ERR_INVALID, "u1_batch_update: null batch");
  if (metrop < 0 || ovrn < 0) return bfail(U1_ERR_INVALID, "u1_batch_update: negative pass count");
  U1_CUDA_TRY(cudaSetDevice(b->ctx->device));
  if (metrop == 0 && ovrn == 0 && !measure) return U1_OK;
  auto key = std::make_pair(metrop * 2 + (measure ? 1 : 0), ovrn);
  auto it = b->graphs.find(key);
  if (it == b->graphs.end()) {
    cudaGraph_t graph = nullptr;
    U1_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const unsigned long long launches0 = u1i::g_launches.load();
    int rc = batch_issue_sweep(b, metrop, ovrn, measure != 0);
    u1i::g_launches.store(launches0);  // captured kernels count at graph launch
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "u1_batch_update: capture");
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "u1_batch_update: instantiate");
    it = b->graphs.emplace(key, ex).first;
  }
  U1_CUDA_TRY(cudaGraphLaunch(it->second, b->stream));
  u1i::g_launches += (unsigned long long)(2 * b->dims * (metrop + ovrn) * b->groups.size() + (measure ? 2 : 0) +
                                          (ovrn == 0 && metrop > 0 ? 1 : 0));
  b->pass += (uint64_t)metrop;
  return U1_OK;
}

extern "C" int u1_batch_measure(u1_batch *b, double *out_host) {
  if (!b || !out_host) return bfail(U1_ERR_INVALID, "u1_batch_measure: null argument");
  U1_CUDA_TRY(cudaSetDevice(b->ctx->device));
  int rc = batch_measure_issue(b);
  if (rc) return rc;
  return u1_batch_results(b, out_host);
}

extern "C" int u1_batch_results(u1_batch *b, double *out_host) {
  if (!b || !out_host) return bfail(U1_ERR_INVALID, "u1_batch_results: null argument");
  U1_CUDA_TRY(cudaMemcpyAsync(b->h_out, b->d_out, sizeof(double) * 6 * b->n, cudaMemcpyDeviceToHost, b->stream));
  U1_CUDA_TRY(cudaStreamSynchronize(b->stream));
  std::memcpy(out_host, b->h_out, sizeof(double) * 6 * b->n);
  return U1_OK;
}

extern "C" int u1_batch_results_device(u1_batch *b, double **dev_ptr) {
  if (!b || !dev_ptr) return bfail(U1_ERR_INVALID, "u1_batch_results_device: null argument");
  *dev_ptr = b->d_out;
  return U1_OK;
}

static int chain_io(u1_batch *b, int chain, double *host, bool import) {
  if (!b || !host || chain < 0 || chain >= b->n) return bfail(U1_ERR_INVALID, "u1_batch angles: bad argument");
  U1_CUDA_TRY(cudaSetDevice(b->ctx->device));
  const BatchChain &ch = b->h_chains[chain];
  const size_t n = (size_t)ch.g.V * ch.g.dims;
  double *tmp = nullptr;
  U1_CUDA_TRY(cudaMalloc(&tmp, n * sizeof(double)));
  cudaError_t e = cudaSuccess;
  if (import) {
    e = cudaMemcpyAsync(tmp, host, n * sizeof(double), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) {
      k_import_angles<<<nblocks((long long)n, 256), 256, 0, b->stream>>>(ch.links, tmp, n);
      e = cudaGetLastError();
    }
  } else {
    k_export_angles<<<nblocks((long long)n, 256), 256, 0, b->stream>>>(ch.links, tmp, n);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
  }
  u1i::g_launches++;
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(e, "u1_batch angles");
  return U1_OK;
}

extern "C" int u1_batch_export_all(u1_batch *b, double *angles_dev) {
  if (!b || !angles_dev) return bfail(U1_ERR_INVALID, "u1_batch_export_all: null argument");
  U1_CUDA_TRY(cudaSetDevice(b->ctx->device));
  // chains are stored back to back, so one elementwise pass converts them all
  k_export_angles<<<nblocks((long long)b->total_links, 256), 256, 0, b->stream>>>(b->links, angles_dev,
                                                                                  b->total_links);
  U1_LAUNCH_CHECK("k_export_angles (batch)");
  return U1_OK;
}

extern "C" int u1_batch_export_angles(u1_batch *b, int chain, double *angles_host) {
  return chain_io(b, chain, angles_host, false);
}
extern "C" int u1_batch_import_angles(u1_batch *b, int chain, const double *angles_host) {
  return chain_io(b, chain, const_cast<double *>(angles_host), true);
}

extern "C" int u1_batch_get_pass(const u1_batch *b, uint64_t *pass) {
  if (!b || !pass) return bfail(U1_ERR_INVALID, "u1_batch_get_pass: null argument");
  *pass = b->pass;
  return U1_OK;
}
