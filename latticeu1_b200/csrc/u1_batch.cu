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
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
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
  int first_upd;    // first block of the chain in the update table (its group's variant and block size)
  int first_site;   // first block in the hot-start table (one site per thread, 256 threads)
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
#ifdef U1_BOUNDS_CHECK
  ChkState *chk;           // checked build: counters, per-link marks of the batch's links
  unsigned *shadow;
  const float2 *chk_base;
#endif
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
#ifdef U1_BOUNDS_CHECK
  a.chk = ph.chk;
  a.shadow = ph.shadow;
  a.chk_base = ph.chk_base;
#endif
  return a;
}

// Four sites per thread (every chain of the launch's group has N0/2 a
// multiple of 4), at most 128 threads per block, as k_update_quad.
template <int D, int MU, bool MET>
__global__ void __launch_bounds__(128, 7)
    k_batch_update_quad(const BatchChain *__restrict__ chains, const int *__restrict__ block_chain, BatchPhase ph) {
  __shared__ BatchChain sch;
  const int blk = (int)blockIdx.x + ph.block_base;
  stage_chain(chains, __ldg(block_chain + blk), sch);
  const UpdArgs a = batch_args(sch, ph, MU);
  update_quad_body<D, MU, MET, SRC_PHILOX>(a, 4 * ((blk - sch.first_upd) * (int)blockDim.x + (int)threadIdx.x));
}

template <int D, int MU, bool MET, bool PAIR>
__global__ void __launch_bounds__(256, 8)
    k_batch_update(const BatchChain *__restrict__ chains, const int *__restrict__ block_chain, BatchPhase ph) {
  __shared__ BatchChain sch;
  const int blk = (int)blockIdx.x + ph.block_base;
  const int cidx = __ldg(block_chain + blk);
  stage_chain(chains, cidx, sch);
  const UpdArgs a = batch_args(sch, ph, MU);
  const int local = blk - sch.first_upd;
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

// A group of consecutive chains [c0, c1) swept together, with the update
// kernel variant (U1V_QUAD, U1V_PAIR32 or U1V_SINGLE: four, two or one site
// per thread) and threads per block its launches use, and its range of the
// update block table.
struct BatchGroup {
  int c0, c1;
  int variant, threads;
  int first_block, nblocks;
};

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
  int *d_tab_upd = nullptr, *d_tab_site = nullptr, *d_tab_meas = nullptr;
  int nb_upd = 0, nb_site = 0, nb_meas = 0;
  size_t tab_upd_cap = 0;                  // ints allocated at d_tab_upd
  double *partials = nullptr, *d_out = nullptr, *h_out = nullptr;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  // Chain groups swept one after another: consecutive chains whose links
  // together fit comfortably in L2, so that after a group's first phase its
  // links are served from L2; each group runs its own kernel variant and
  // block size (u1_batch_tune).
  std::vector<BatchGroup> groups;
  size_t group_bytes = 32ull << 20;       // group size limit the groups were cut with
  // Lanes: with 2, consecutive groups alternate between the batch's stream
  // and a second one inside each sweep, so one group's phase boundaries
  // (drain, launch, refill) overlap another group's phases.  Groups are
  // independent chains: the links are the same with one lane or two.
  int lanes = 2;
  cudaStream_t lane_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool quad_enabled = true;               // four-site kernels allowed (U1_BATCH_QUAD=0: no)
  float2 *backup = nullptr;               // link backup while tuning
  unsigned *shadow = nullptr;              // checked build: per-link access marks (total_links words)
};

using u1i::cuda_fail;

static inline int nblocks(long long n, int threads) { return (int)((n + threads - 1) / threads); }

static int bfail(int code, const std::string &msg) {
  u1i::set_error(msg);
  return code;
}

static int sites_per_thread(int variant) { return variant == U1V_QUAD ? 4 : variant == U1V_PAIR32 ? 2 : 1; }

// Whether every chain of [c0, c1) fits `variant` (four sites per thread:
// N0/2 a multiple of 4; two: N0/2 even) and `threads` suits its kernel.
static bool group_allows(const u1_batch *b, int c0, int c1, int variant, int threads) {
  if (threads < 32 || threads % 32) return false;
  if (variant == U1V_QUAD) {
    if (!b->quad_enabled || threads > 128) return false;
  } else if (variant == U1V_PAIR32 || variant == U1V_SINGLE) {
    if (threads > 256) return false;
  } else {
    return false;
  }
  for (int c = c0; c < c1; ++c) {
    const int h = b->h_chains[c].g.hN0;
    if ((variant == U1V_QUAD && (h & 3)) || (variant == U1V_PAIR32 && (h & 1))) return false;
  }
  return true;
}

// The untuned choice of a group: four sites per thread at 128 threads where
// every chain allows it, else two sites at 256, else one site at 256.
static std::pair<int, int> default_choice(const u1_batch *b, int c0, int c1) {
  if (group_allows(b, c0, c1, U1V_QUAD, 128)) return {U1V_QUAD, 128};
  if (group_allows(b, c0, c1, U1V_PAIR32, 256)) return {U1V_PAIR32, 256};
  return {U1V_SINGLE, 256};
}

// Consecutive chains in groups of at most group_bytes of links (a single
// chain may exceed it).
static std::vector<std::pair<int, int>> split_groups(const u1_batch *b, size_t group_bytes) {
  std::vector<std::pair<int, int>> out;
  size_t bytes = 0;
  int c0 = 0;
  for (int c = 0; c < b->n; ++c) {
    const size_t cb = (size_t)b->h_chains[c].g.V * b->h_chains[c].g.dims * sizeof(float2);
    if (c > c0 && bytes + cb > group_bytes) {
      out.push_back({c0, c});
      c0 = c;
      bytes = 0;
    }
    bytes += cb;
  }
  out.push_back({c0, b->n});
  return out;
}

// Cut the chains into groups of at most group_bytes, give group k the
// (variant, threads) choice[k] (defaults where choice is shorter or a choice
// does not fit the group), lay out the update block table and upload it with
// the chain descriptors.  Cached sweep graphs are dropped.  Every layout
// gives the same links bit for bit: a chain's sites run the same update body
// with the same Philox counters whichever thread takes them.
static int batch_configure(u1_batch *b, size_t group_bytes, const std::vector<std::pair<int, int>> &choice) {
  const std::vector<std::pair<int, int>> cuts = split_groups(b, group_bytes);
  std::vector<BatchGroup> groups;
  std::vector<int> tab;
  for (size_t k = 0; k < cuts.size(); ++k) {
    const int c0 = cuts[k].first, c1 = cuts[k].second;
    std::pair<int, int> vt = k < choice.size() ? choice[k] : default_choice(b, c0, c1);
    if (!group_allows(b, c0, c1, vt.first, vt.second)) vt = default_choice(b, c0, c1);
    BatchGroup gr{c0, c1, vt.first, vt.second, (int)tab.size(), 0};
    const int spt = sites_per_thread(vt.first);
    for (int c = c0; c < c1; ++c) {
      BatchChain &ch = b->h_chains[c];
      ch.first_upd = (int)tab.size();
      tab.insert(tab.end(), nblocks(ch.g.Vh / spt, vt.second), c);
    }
    gr.nblocks = (int)tab.size() - gr.first_block;
    groups.push_back(gr);
  }
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  if (tab.size() > b->tab_upd_cap) {
    u1i::dev_free(b->d_tab_upd);
    b->d_tab_upd = nullptr;
    b->tab_upd_cap = 0;
    U1_CUDA_TRY(u1i::dev_alloc(&b->d_tab_upd, sizeof(int) * tab.size()));
    b->tab_upd_cap = tab.size();
  }
  U1_CUDA_TRY(cudaMemcpy(b->d_tab_upd, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice));
  U1_CUDA_TRY(cudaMemcpy(b->d_chains, b->h_chains.data(), sizeof(BatchChain) * b->n, cudaMemcpyHostToDevice));
  b->groups = groups;
  b->nb_upd = (int)tab.size();
  b->group_bytes = group_bytes;
  return U1_OK;
}

extern "C" int u1_batch_destroy(u1_batch *b) {
  if (!b) return U1_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->stream);
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  u1i::dev_free(b->links);
  u1i::dev_free(b->d_chains);
  u1i::dev_free(b->d_tab_upd);
  u1i::dev_free(b->d_tab_site);
  u1i::dev_free(b->d_tab_meas);
  u1i::dev_free(b->backup);
  u1i::dev_free(b->partials);
  u1i::dev_free(b->d_out);
  u1i::dev_free(b->pass_dev);
  u1i::dev_free(b->shadow);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  if (b->lane_stream) cudaStreamDestroy(b->lane_stream);
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
  std::vector<int> tab_site, tab_meas;
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
    const int ns = nblocks(g.Vh, 256);
    ch.first_upd = 0;  // set by batch_configure
    ch.first_site = (int)tab_site.size();
    ch.first_meas = (int)tab_meas.size();
    ch.meas = measure_layout(g);
    ch.nb_meas = ch.meas.nb_plaq + ch.meas.nb_poly;
    tab_site.insert(tab_site.end(), ns, c);
    tab_meas.insert(tab_meas.end(), ch.nb_meas, c);
  }
  b->total_links = off;
  b->nb_site = (int)tab_site.size();
  b->nb_meas = (int)tab_meas.size();
  // groups of at most U1_BATCH_GROUP_MB (default 32) MiB of links; a single
  // chain may exceed it; 0 puts every chain in one group
  if (const char *env = std::getenv("U1_BATCH_GROUP_MB")) {
    const long long mb = std::atoll(env);
    b->group_bytes = mb > 0 ? (size_t)mb << 20 : SIZE_MAX;
  }
  // U1_BATCH_LANES=1 sweeps the groups one after another on one stream
  if (const char *env = std::getenv("U1_BATCH_LANES")) b->lanes = std::atoi(env) == 1 ? 1 : 2;
  // U1_BATCH_QUAD=0 keeps every group on the two-site (or one-site) kernel
  const char *qenv = std::getenv("U1_BATCH_QUAD");
  b->quad_enabled = !(qenv && qenv[0] == '0');
  cudaError_t e = cudaStreamCreate(&b->own_stream);
  b->stream = ctx->stream ? ctx->stream : b->own_stream;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->lane_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
  if (e == cudaSuccess) e = u1i::dev_alloc(&b->links, b->total_links * sizeof(float2));
  if (e == cudaSuccess) e = u1i::dev_alloc(&b->d_chains, sizeof(BatchChain) * nchains);
  if (e == cudaSuccess) e = u1i::dev_alloc(&b->d_tab_site, sizeof(int) * tab_site.size());
  if (e == cudaSuccess) e = u1i::dev_alloc(&b->d_tab_meas, sizeof(int) * tab_meas.size());
  if (e == cudaSuccess) e = u1i::dev_alloc(&b->partials, sizeof(double) * 6 * tab_meas.size());
  if (e == cudaSuccess) e = u1i::dev_alloc(&b->d_out, sizeof(double) * 6 * nchains);
  if (e == cudaSuccess) e = cudaMallocHost(&b->h_out, sizeof(double) * 6 * nchains);
  if (e == cudaSuccess) e = u1i::dev_alloc(&b->pass_dev, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(b->pass_dev, 0, sizeof(unsigned long long));
  if (e != cudaSuccess) {
    u1_batch_destroy(b);
    u1i::set_error(std::string("u1_batch_create: ") + cudaGetErrorString(e));
    return U1_ERR_NOMEM;
  }
#ifdef U1_BOUNDS_CHECK
  b->shadow = u1i::chk_shadow(b->total_links);
  if (!b->shadow || !u1i::chk_state(ctx)) {
    u1_batch_destroy(b);
    return bfail(U1_ERR_NOMEM, "u1_batch_create: no device memory for the access checks");
  }
#endif
  for (int c = 0; c < nchains; ++c) b->h_chains[c].links = b->links + offsets[c];
  e = cudaMemcpy(b->d_tab_site, tab_site.data(), sizeof(int) * tab_site.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_tab_meas, tab_meas.data(), sizeof(int) * tab_meas.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    u1_batch_destroy(b);
    return cuda_fail(e, "u1_batch_create: upload");
  }
  int rc = batch_configure(b, b->group_bytes, {});  // update table and chain descriptors
  if (rc) {
    u1_batch_destroy(b);
    return rc;
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
static int batch_launch_quad(u1_batch *b, BatchPhase ph, int group, cudaStream_t s) {
  const BatchGroup &gr = b->groups[group];
  ph.block_base = gr.first_block;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)gr.nblocks);
  cfg.blockDim = dim3((unsigned)gr.threads);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_batch_update_quad<D, MU, MET>, (const BatchChain *)b->d_chains,
                                     (const int *)b->d_tab_upd, ph);
  u1i::g_launches.fetch_add(1, std::memory_order_relaxed);
  if (e != cudaSuccess) return cuda_fail(e, "k_batch_update_quad");
  return U1_OK;
}

template <int D, int MU, bool MET, bool PAIR>
static int batch_launch(u1_batch *b, BatchPhase ph, int group, cudaStream_t s) {
  const BatchGroup &gr = b->groups[group];
  ph.block_base = gr.first_block;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)gr.nblocks);
  cfg.blockDim = dim3((unsigned)gr.threads);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_batch_update<D, MU, MET, PAIR>, (const BatchChain *)b->d_chains,
                                     (const int *)b->d_tab_upd, ph);
  u1i::g_launches.fetch_add(1, std::memory_order_relaxed);
  if (e != cudaSuccess) return cuda_fail(e, "k_batch_update");
  return U1_OK;
}

template <int D, int MU>
static int batch_launch_mu(u1_batch *b, const BatchPhase &ph, bool met, int group, cudaStream_t s) {
  const int v = b->groups[group].variant;
  if (v == U1V_QUAD)
    return met ? batch_launch_quad<D, MU, true>(b, ph, group, s) : batch_launch_quad<D, MU, false>(b, ph, group, s);
  if (v == U1V_PAIR32)
    return met ? batch_launch<D, MU, true, true>(b, ph, group, s) : batch_launch<D, MU, false, true>(b, ph, group, s);
  return met ? batch_launch<D, MU, true, false>(b, ph, group, s) : batch_launch<D, MU, false, false>(b, ph, group, s);
}

template <int D>
static int batch_phase(u1_batch *b, const BatchPhase &ph, int mu, bool met, int group, cudaStream_t s) {
  switch (mu) {
    case 0: return batch_launch_mu<D, 0>(b, ph, met, group, s);
    case 1: return batch_launch_mu<D, 1>(b, ph, met, group, s);
    case 2:
      if constexpr (D > 2) return batch_launch_mu<D, 2>(b, ph, met, group, s);
      break;
    case 3:
      if constexpr (D > 3) return batch_launch_mu<D, 3>(b, ph, met, group, s);
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

// Whether a sweep of groups [g0, g1) runs on two lanes.
static bool two_lanes(const u1_batch *b, int g0, int g1) { return b->lanes == 2 && g1 - g0 > 1; }

// The sweep of groups [g0, g1) (all groups by default).
static int batch_issue_sweep(u1_batch *b, int metrop, int ovrn, bool measure, int g0 = 0, int g1 = -1) {
  BatchPhase ph{};
  ph.key0 = (uint32_t)b->seed;
  ph.key1 = (uint32_t)(b->seed >> 32);
  ph.pass_dev = b->pass_dev;
#ifdef U1_BOUNDS_CHECK
  ph.chk = b->ctx->chk;
  ph.shadow = b->shadow;
  ph.chk_base = b->links;
#endif
  const int D = b->dims;
  const int ngroups = g1 < 0 ? (int)b->groups.size() : g1;
  // Each chain group runs the whole sweep before its lane's next group
  // starts.  Every group's Metropolis phases read the same pass counter.  On
  // one lane the first overrelaxation kernel of the last group (after all of
  // them) bumps it; on two lanes (groups alternate between the batch's
  // stream and the second lane, forked from and joined back into the batch's
  // stream) a kernel after the join does.
  const bool lanes2 = two_lanes(b, g0, ngroups);
  bool bumped = (metrop == 0) || lanes2;
  if (lanes2) {
    U1_CUDA_TRY(cudaEventRecord(b->ev_fork, b->stream));
    U1_CUDA_TRY(cudaStreamWaitEvent(b->lane_stream, b->ev_fork, 0));
  }
  for (int grp = g0; grp < ngroups; ++grp) {
    const cudaStream_t s = (lanes2 && ((grp - g0) & 1)) ? b->lane_stream : b->stream;
#ifdef U1_BOUNDS_CHECK
    // the group's own links (its chains are consecutive): the other lane's
    // group marks its links concurrently
    const BatchChain &first = b->h_chains[b->groups[grp].c0], &last = b->h_chains[b->groups[grp].c1 - 1];
    const size_t g_off = (size_t)(first.links - b->links);
    const size_t g_len = (size_t)(last.links - first.links) + (size_t)last.g.V * last.g.dims;
#endif
    auto run = [&](int mu, bool met) {
      int rc = D == 2 ? batch_phase<2>(b, ph, mu, met, grp, s)
             : D == 3 ? batch_phase<3>(b, ph, mu, met, grp, s)
                      : batch_phase<4>(b, ph, mu, met, grp, s);
#ifdef U1_BOUNDS_CHECK
      if (rc == U1_OK) rc = u1i::chk_phase_end(s, ph.shadow + g_off, g_len, ph.chk);
#endif
      return rc;
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
  if (lanes2) {
    U1_CUDA_TRY(cudaEventRecord(b->ev_join, b->lane_stream));
    U1_CUDA_TRY(cudaStreamWaitEvent(b->stream, b->ev_join, 0));
  }
  if (!bumped || (lanes2 && metrop > 0)) {  // no overrelaxation kernel carried the pass-counter bump
    k_pass_add<<<1, 1, 0, b->stream>>>(b->pass_dev, (unsigned long long)metrop);
    U1_LAUNCH_CHECK("k_pass_add");
  }
  if (measure) return batch_measure_issue(b);
  return U1_OK;
}

extern "C" int u1_batch_update(u1_batch *b, int metrop, int ovrn, int measure) {
  u1i::NvtxRange nvtx_range("u1_batch_update");
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
  const bool pass_kernel = metrop > 0 && (ovrn == 0 || two_lanes(b, 0, (int)b->groups.size()));
  u1i::g_launches += (unsigned long long)(2 * b->dims * (metrop + ovrn) * b->groups.size() + (measure ? 2 : 0) +
                                          (pass_kernel ? 1 : 0));
  b->pass += (uint64_t)metrop;
  return U1_OK;
}

extern "C" int u1_batch_measure(u1_batch *b, double *out_host) {
  u1i::NvtxRange nvtx_range("u1_batch_measure");
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
  U1_CUDA_TRY(u1i::dev_alloc(&tmp, n * sizeof(double)));
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
  u1i::dev_free(tmp);
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

// ---------------------------------------------------------------- tuner
// The batch autotuner (no counterpart in the reference, which runs one
// lattice per process; its block-size search is src/tune.cpp:306-416).  It
// chooses the chain-group size (32 ... 96 MiB of links, the groups then
// being swept one after another so each stays in L2) and, per group, the
// update kernel (four, two or one site per thread) and threads per block.
// Every choice gives the same links bit for bit, so trials never change the
// Markov chains; each trial captures its sweep (1 Metropolis + 4 OR) as a
// CUDA graph, as u1_batch_update runs it, and scores it by the shortest of 5
// single replays after 2 warm-up replays (the first trial after about 50 ms
// of clock warm-up), from a backed-up state (links and pass counter restored).
// Stage 1 times whole sweeps for each group size with the default kernels;
// stage 2 times each group's own sweep for each (kernel, threads) it
// allows; the per-group choice is kept only if the whole sweep is faster.
// The result is cached per (device, dims, chain extents) in memory and,
// when U1_RESOURCE_PATH names a directory, in
// $U1_RESOURCE_PATH/u1b200_batch_tunecache.tsv.
namespace {
struct BatchTuneRec {
  size_t group_bytes;
  std::vector<std::pair<int, int>> choice;
  int lanes = 1;
};
std::mutex g_btune_mu;
bool g_btune_loaded = false;
std::map<std::string, BatchTuneRec> g_btune;

std::string batch_tune_file() {
  const char *p = std::getenv("U1_RESOURCE_PATH");
  return (p && *p) ? std::string(p) + "/u1b200_batch_tunecache.tsv" : std::string();
}

// Device, dims, chain count and an FNV-1a hash of every chain's extents.
std::string batch_tune_key(const u1_batch *b) {
  uint64_t h = 1469598103934665603ull;
  for (const BatchChain &ch : b->h_chains)
    for (int k = 0; k < 4; ++k) {
      h ^= (uint64_t)(uint32_t)ch.g.N[k];
      h *= 1099511628211ull;
    }
  std::ostringstream k;
  k << b->ctx->prop.name << "|batch|" << b->dims << "|" << b->n << "|" << std::hex << h;
  return k.str();
}

// key <tab> group MiB <tab> variant:threads,... <tab> microseconds per sweep
// <tab> lanes (absent in older files: one lane)
void batch_tune_load_locked() {
  if (g_btune_loaded) return;
  g_btune_loaded = true;
  const std::string f = batch_tune_file();
  if (f.empty()) return;
  std::ifstream in(f);
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ls(line);
    std::string key, mb, list, us, lanes;
    if (!std::getline(ls, key, '\t') || !std::getline(ls, mb, '\t') || !std::getline(ls, list, '\t')) continue;
    BatchTuneRec rec;
    rec.group_bytes = (size_t)std::atoll(mb.c_str()) << 20;
    if (std::getline(ls, us, '\t') && std::getline(ls, lanes, '\t')) rec.lanes = std::atoi(lanes.c_str()) == 2 ? 2 : 1;
    std::istringstream li(list);
    std::string item;
    while (std::getline(li, item, ',')) {
      const size_t c = item.find(':');
      if (c == std::string::npos) continue;
      rec.choice.push_back({std::atoi(item.substr(0, c).c_str()), std::atoi(item.substr(c + 1).c_str())});
    }
    if (rec.group_bytes > 0 && !rec.choice.empty()) g_btune[key] = rec;
  }
}

void batch_tune_save(const std::string &key, const BatchTuneRec &rec, double us) {
  const std::string f = batch_tune_file();
  if (f.empty()) return;
  std::ofstream out(f, std::ios::app);
  if (!out) return;
  out << key << '\t' << (rec.group_bytes >> 20) << '\t';
  for (size_t k = 0; k < rec.choice.size(); ++k)
    out << (k ? "," : "") << rec.choice[k].first << ':' << rec.choice[k].second;
  out << '\t' << us << '\t' << rec.lanes << '\n';
}

std::vector<std::pair<int, int>> current_choice(const u1_batch *b) {
  std::vector<std::pair<int, int>> c;
  for (const BatchGroup &g : b->groups) c.push_back({g.variant, g.threads});
  return c;
}
}  // namespace

// Microseconds per sweep (1 Metropolis + 4 OR) of groups [g0, g1) in the
// current layout: a captured graph, 2 warm-up replays (after warm_ms of
// clock warm-up), the shortest of 5 single timed replays; the links and the
// pass counter are restored from the backup afterwards.
static int batch_time_sweep(u1_batch *b, int g0, int g1, double *us, double warm_ms = 0.0) {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t ex = nullptr;
  U1_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  const unsigned long long launches0 = u1i::g_launches.load();
  int rc = batch_issue_sweep(b, 1, 4, false, g0, g1);
  u1i::g_launches.store(launches0);
  cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "u1_batch_tune: capture");
  e = cudaGraphInstantiate(&ex, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(e, "u1_batch_tune: instantiate");
  if (warm_ms > 0.0) e = u1i::warm_clocks(ex, b->stream, warm_ms);
  if (e == cudaSuccess) e = u1i::time_graph_min(ex, b->stream, 2, 5, us);
  const unsigned long long pass0 = b->pass;
  cudaError_t r1 = cudaMemcpyAsync(b->links, b->backup, b->total_links * sizeof(float2), cudaMemcpyDeviceToDevice,
                                   b->stream);
  cudaError_t r2 = cudaMemcpyAsync(b->pass_dev, &pass0, sizeof(pass0), cudaMemcpyHostToDevice, b->stream);
  cudaError_t r3 = cudaStreamSynchronize(b->stream);
  cudaGraphExecDestroy(ex);
  if (e == cudaSuccess) e = r1 != cudaSuccess ? r1 : r2 != cudaSuccess ? r2 : r3;
  if (e != cudaSuccess) return cuda_fail(e, "u1_batch_tune: trial");
  if (u1i::tune_verbose())
    std::fprintf(stderr, "u1_batch_tune: groups %d..%d of %d (%zu MiB groups, %d lane%s): %.1f us per sweep\n", g0,
                 g1 - 1, (int)b->groups.size(), b->group_bytes >> 20, two_lanes(b, g0, g1) ? 2 : 1,
                 two_lanes(b, g0, g1) ? "s" : "", *us);
  return U1_OK;
}

static int batch_tune(u1_batch *b) {
  const std::string key = batch_tune_key(b);
  {
    std::lock_guard<std::mutex> lock(g_btune_mu);
    batch_tune_load_locked();
    auto it = g_btune.find(key);
    if (it != g_btune.end()) {
      b->lanes = it->second.lanes;
      return batch_configure(b, it->second.group_bytes, it->second.choice);
    }
  }
  if (!b->backup) U1_CUDA_TRY(u1i::dev_alloc(&b->backup, b->total_links * sizeof(float2)));
  U1_CUDA_TRY(cudaMemcpyAsync(b->backup, b->links, b->total_links * sizeof(float2), cudaMemcpyDeviceToDevice,
                              b->stream));
  U1_CUDA_TRY(cudaStreamSynchronize(b->stream));
  // Each stage times its candidates in two rounds, the second in reverse
  // order, and keeps each candidate's faster time (a large batch drives the
  // GPU into its power cap while tuning; one round would favour whichever
  // candidates ran first).
  auto two_rounds = [](size_t n) {
    std::vector<size_t> order;
    for (size_t k = 0; k < n; ++k) order.push_back(k);
    for (size_t k = n; k-- > 0;) order.push_back(k);
    return order;
  };
  // stage 1: group size and lanes, default kernels
  std::vector<std::pair<int, int>> sizes;  // (MiB, lanes)
  for (int lanes : {1, 2})
    for (int mb : {32, 48, 64, 80, 96}) sizes.push_back({mb, lanes});
  std::vector<double> size_us(sizes.size(), -1.0);
  bool warmed = false;
  for (size_t k : two_rounds(sizes.size())) {
    b->lanes = sizes[k].second;
    int rc = batch_configure(b, (size_t)sizes[k].first << 20, {});
    double us = 0.0;
    if (!rc) rc = batch_time_sweep(b, 0, (int)b->groups.size(), &us, warmed ? 0.0 : 50.0);
    warmed = true;
    if (rc) return rc;
    if (size_us[k] < 0.0 || us < size_us[k]) size_us[k] = us;
  }
  size_t best_bytes = b->group_bytes;
  int best_lanes = b->lanes;
  double best_us = -1.0;
  for (size_t k = 0; k < sizes.size(); ++k)
    if (best_us < 0.0 || size_us[k] < best_us) {
      best_us = size_us[k];
      best_bytes = (size_t)sizes[k].first << 20;
      best_lanes = sizes[k].second;
    }
  b->lanes = best_lanes;
  // stage 2: per group, kernel and threads per block
  int rc = batch_configure(b, best_bytes, {});
  if (rc) return rc;
  std::vector<std::pair<int, int>> choice = current_choice(b);
  for (size_t k = 0; k < choice.size(); ++k) {
    const int c0 = b->groups[k].c0, c1 = b->groups[k].c1;
    std::vector<std::pair<int, int>> cand;
    for (int v : {U1V_QUAD, U1V_PAIR32, U1V_SINGLE})
      for (int t : {64, 96, 128, 192, 256})
        if (group_allows(b, c0, c1, v, t)) cand.push_back({v, t});
    std::vector<double> cand_us(cand.size(), -1.0);
    for (size_t j : two_rounds(cand.size())) {
      std::vector<std::pair<int, int>> trial = choice;
      trial[k] = cand[j];
      double us = 0.0;
      rc = batch_configure(b, best_bytes, trial);
      if (!rc) rc = batch_time_sweep(b, (int)k, (int)k + 1, &us);
      if (rc) return rc;
      if (cand_us[j] < 0.0 || us < cand_us[j]) cand_us[j] = us;
    }
    double best_k_us = -1.0;
    for (size_t j = 0; j < cand.size(); ++j)
      if (best_k_us < 0.0 || cand_us[j] < best_k_us) {
        best_k_us = cand_us[j];
        choice[k] = cand[j];
      }
  }
  rc = batch_configure(b, best_bytes, choice);
  double tuned_us = 0.0;
  if (!rc) rc = batch_time_sweep(b, 0, (int)b->groups.size(), &tuned_us);
  if (rc) return rc;
  if (tuned_us > best_us) {  // the per-group choices did not add up to a faster sweep
    rc = batch_configure(b, best_bytes, {});
    if (rc) return rc;
    tuned_us = best_us;
  }
  u1i::dev_free(b->backup);
  b->backup = nullptr;
  BatchTuneRec rec{b->group_bytes, current_choice(b), b->lanes};
  std::lock_guard<std::mutex> lock(g_btune_mu);
  g_btune[key] = rec;
  batch_tune_save(key, rec, tuned_us);
  return U1_OK;
}

extern "C" int u1_batch_tune(u1_batch *b, int *group_mb) {
  u1i::NvtxRange nvtx_range("u1_batch_tune");
  if (!b) return bfail(U1_ERR_INVALID, "u1_batch_tune: null batch");
  U1_CUDA_TRY(cudaSetDevice(b->ctx->device));
  const int lanes0 = b->lanes;
  int rc = batch_tune(b);
  if (rc) {
    b->lanes = lanes0;
    if (b->backup) {  // a failed trial: put the links and pass counter back
      cudaMemcpyAsync(b->links, b->backup, b->total_links * sizeof(float2), cudaMemcpyDeviceToDevice, b->stream);
      const unsigned long long pass0 = b->pass;
      cudaMemcpyAsync(b->pass_dev, &pass0, sizeof(pass0), cudaMemcpyHostToDevice, b->stream);
      cudaStreamSynchronize(b->stream);
      u1i::dev_free(b->backup);
      b->backup = nullptr;
    }
    return rc;
  }
  if (group_mb) *group_mb = (int)std::min<size_t>(b->group_bytes >> 20, (size_t)INT_MAX);
  return U1_OK;
}

extern "C" int u1_batch_configure(u1_batch *b, int group_mb, int ngroups, const int *variants, const int *threads) {
  if (!b || ngroups < 0 || (ngroups > 0 && (!variants || !threads)))
    return bfail(U1_ERR_INVALID, "u1_batch_configure: bad argument");
  U1_CUDA_TRY(cudaSetDevice(b->ctx->device));
  std::vector<std::pair<int, int>> choice;
  for (int k = 0; k < ngroups; ++k) choice.push_back({variants[k], threads[k]});
  const size_t bytes = group_mb > 0 ? (size_t)group_mb << 20 : b->group_bytes;
  return batch_configure(b, bytes, choice);
}

extern "C" int u1_batch_set_lanes(u1_batch *b, int lanes) {
  if (!b || (lanes != 1 && lanes != 2)) return bfail(U1_ERR_INVALID, "u1_batch_set_lanes: lanes must be 1 or 2");
  U1_CUDA_TRY(cudaSetDevice(b->ctx->device));
  if (lanes == b->lanes) return U1_OK;
  U1_CUDA_TRY(cudaStreamSynchronize(b->stream));
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);  // captured with the other lane count
  b->graphs.clear();
  b->lanes = lanes;
  return U1_OK;
}

extern "C" int u1_batch_get_lanes(const u1_batch *b, int *lanes) {
  if (!b || !lanes) return bfail(U1_ERR_INVALID, "u1_batch_get_lanes: null argument");
  *lanes = b->lanes;
  return U1_OK;
}

extern "C" int u1_batch_group_info(const u1_batch *b, int group, int out[4]) {
  if (!b || !out || group < 0 || group >= (int)b->groups.size())
    return bfail(U1_ERR_INVALID, "u1_batch_group_info: bad argument");
  const BatchGroup &g = b->groups[group];
  out[0] = g.c0;
  out[1] = g.c1;
  out[2] = g.variant;
  out[3] = g.threads;
  return U1_OK;
}
