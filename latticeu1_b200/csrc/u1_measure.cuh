// Measurement kernels: fused plaquette (SS/ST) + Polyakov loop, the
// Polyakov-loop field (plain or analytic multihit) and its correlator.
//
// Reference algorithm being replaced:
//   plaquette        src/plaquette.cu:93-118, norms :156-165
//   Polyakov loop    src/polyakov.cu:60-77, :124-139
//   P(x) field       src/polyakov.cu:415-440 (kernel_polyakov_volume<multihit>)
//   correlator       src/polyakov.cu:514-535, norm :568
//   multihit mean    include/lattice_functions.h:92-105
// Reductions: per-thread values are summed in FP64 with xor-shuffle warp
// reductions, block totals go to a per-block partials array, and the last
// block to finish (ticket counter) sums the partials in block order, so
// every result is deterministic run to run.  The reference instead folds
// shared memory serially in thread 0 and uses FP64 atomicAdd
// (include/reduce_block_1d.h:41-64).
#pragma once
#include "u1_cplx.cuh"
#include "u1_geom.cuh"
#include "u1_update.cuh"

namespace u1b {

constexpr int kRedThreads = 256;
constexpr int kRedWarps = kRedThreads / 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NV values per thread; the totals are valid in threads
// 0..NV-1 (thread k holds value k).  smem must hold kRedWarps*NV doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double w = warp_sum(v[k]);
    if (lane == 0) smem[warp * NV + k] = w;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += smem[w * NV + threadIdx.x];
    v[0] = t;  // caller reads v[0] in thread k as total k
  }
  __syncthreads();
}

// Per-thread sum of partials[b * stride + k] over b = threadIdx.x,
// threadIdx.x + blockDim.x, ... < n, added in that order, with kUnroll loads
// in flight (a plain strided loop would wait for every load in turn).
__device__ __forceinline__ double strided_partial_sum(const double *partials, unsigned n, int stride, int k) {
  constexpr int kUnroll = 8;
  double w = 0.0;
  for (unsigned b0 = threadIdx.x; b0 < n; b0 += kUnroll * blockDim.x) {
    double t[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const unsigned b = b0 + u * blockDim.x;
      t[u] = (b < n) ? __ldcg(partials + (size_t)b * stride + k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) w += t[u];
  }
  return w;
}

// Block totals already reduced (thread k < NV holds total k in tot): store
// them as this block's partials, take a ticket; the last block sums all
// partials in block order and writes out[k] = scale[k] * total_k, then
// resets `counter` to 0.
template <int NV>
__device__ __forceinline__ void finish_block_totals(double tot, double *smem, double *partials,
                                                    unsigned int *counter, double *out,
                                                    const double (&scale)[NV]) {
  __shared__ bool am_last;
  if (threadIdx.x < NV) {
    partials[(size_t)blockIdx.x * NV + threadIdx.x] = tot;
    __threadfence();  // the writers order their partials before the ticket
  }
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  // Thread j sums partials of blocks j, j + blockDim, j + 2 blockDim, ... in
  // that order.  The loads of kUnroll blocks are issued together before they
  // are added, so the pass costs about one L2 round trip per kUnroll * blockDim
  // blocks (a plain strided loop would wait for every load in turn).
  constexpr int kUnroll = 4;
  double w[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) w[k] = 0.0;
  for (unsigned b0 = threadIdx.x; b0 < gridDim.x; b0 += kUnroll * blockDim.x) {
    double t[kUnroll][NV];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const unsigned b = b0 + u * blockDim.x;
#pragma unroll
      for (int k = 0; k < NV; ++k) t[u][k] = (b < gridDim.x) ? __ldcg(partials + (size_t)b * NV + k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int k = 0; k < NV; ++k) w[k] += t[u][k];
  }
  block_sum<NV>(w, smem);
  if (threadIdx.x < NV) out[threadIdx.x] = w[0] * scale[threadIdx.x];
  if (threadIdx.x == 0) *counter = 0u;
}

// Store this block's NV totals, take a ticket; the last block sums all
// partials in block order and writes out[k] = scale[k] * total_k.
template <int NV>
__device__ __forceinline__ void partials_finish(double (&v)[NV], double *smem, double *partials,
                                                unsigned int *counter, double *out,
                                                const double (&scale)[NV]) {
  block_sum<NV>(v, smem);
  finish_block_totals<NV>(v[0], smem, partials, counter, out, scale);
}

// Launch layout of the plaquette + Polyakov measurement.
//  * blocks [0, nb_plaq): plaquettes.  pair != 0 (N0/2 even): thread t
//    takes EO sites i = 2t, 2t+1 of both parities, whose neighbours along
//    x1..x3 sit side by side (128-bit loads); else thread i takes EO site i.
//  * blocks [nb_plaq, nb_plaq + nb_poly): Polyakov loops.  A block holds
//    kRedThreads/chunks spatial sites x `chunks` time chunks; each thread
//    multiplies the Nt/chunks temporal links of its chunk, and the chunk
//    products of a site are combined in shared memory in chunk order.
struct MeasK {
  int nb_plaq;
  int nb_poly;
  int pair;
  int chunks;
};

__host__ inline MeasK measure_layout(const GeomK &g) {
  MeasK m{};
  m.pair = (g.hN0 & 1) == 0;
  const int plaq_threads = m.pair ? g.Vh / 2 : g.Vh;
  m.nb_plaq = (plaq_threads + kRedThreads - 1) / kRedThreads;
  // largest of 8, 4, 2 dividing Nt with at least eight links per chunk (a
  // thread's loads are independent; fewer, fuller blocks cut the per-block
  // reduction cost), else one chunk
  const int Nt = g.N[g.dims - 1];
  m.chunks = 1;
  for (int c = 8; c > 1; c >>= 1)
    if (Nt % c == 0 && Nt / c >= 8) {
      m.chunks = c;
      break;
    }
  m.nb_poly = (g.Vs * m.chunks + kRedThreads - 1) / kRedThreads;
  return m;
}

// Plaquettes (mu < nu) at one site: U_mu(x) U_nu(x+mu) conj(U_mu(x+nu)) conj(U_nu(x)),
// accumulated as (1 - Re P, -Im P) into vs[0..1] (spatial) or vs[2..3] (temporal nu).
__device__ __forceinline__ void plaq_accum(float2 umu, float2 a, float2 b, float2 unu, bool temporal,
                                           float (&vs)[6]) {
  const float2 P = cmulc(cmulc(cmul(umu, a), b), unu);
  const int o = temporal ? 2 : 0;
  vs[o] += 1.f - P.x;
  vs[o + 1] -= P.y;
}

template <int D>
__device__ __forceinline__ void plaq_sites_pair(const float2 *__restrict__ lat, const GeomK &g, int i,
                                                float (&vs)[6]) {
  int x[4], k;
  eo_decode_fast<D>(g, i, 0, x, k);
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    if (p == 1) x[0] = 2 * k + ((x[1] + x[2] + x[3] + 1) & 1);
    int fwd[4], bwd[4];
    eo_steps<D>(g, x, k, fwd, bwd);
    // x0 steps of the second site (x0 + 2): as the first unless it wraps
    const int odd = x[0] & 1;
    const int f0b = odd ? ((k + 1 == g.hN0 - 1) ? g.wrapf[0] : 1) : 0;
    const int q = 1 - p;
    Pair2 U[D];
#pragma unroll
    for (int mu = 0; mu < D; ++mu) U[mu] = ld_vec2(lat + mu * g.V + p * g.Vh, i, no_chk());
#pragma unroll
    for (int mu = 0; mu < D - 1; ++mu) {
#pragma unroll
      for (int nu = mu + 1; nu < D; ++nu) {
        const float2 *Lq_nu = lat + nu * g.V + q * g.Vh;
        const Pair2 a = (mu == 0) ? ld_two(Lq_nu, i + fwd[0], i + 1 + f0b, no_chk()) : ld_vec2(Lq_nu, i + fwd[mu], no_chk());
        const Pair2 b = ld_vec2(lat + mu * g.V + q * g.Vh, i + fwd[nu], no_chk());  // U_mu(x+nu), nu >= 1
        plaq_accum(U[mu].s0, a.s0, b.s0, U[nu].s0, nu == D - 1, vs);
        plaq_accum(U[mu].s1, a.s1, b.s1, U[nu].s1, nu == D - 1, vs);
      }
    }
  }
}

template <int D>
__device__ __forceinline__ void plaq_site(const float2 *__restrict__ lat, const GeomK &g, int i,
                                          float (&vs)[6]) {
  int x[4], k;
  eo_decode_fast<D>(g, i, 0, x, k);
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    if (p == 1) x[0] = 2 * k + ((x[1] + x[2] + x[3] + 1) & 1);
    int fwd[4], bwd[4];
    eo_steps<D>(g, x, k, fwd, bwd);
    const int q = 1 - p;
    float2 U[D];
#pragma unroll
    for (int mu = 0; mu < D; ++mu) U[mu] = __ldg(lat + mu * g.V + p * g.Vh + i);
#pragma unroll
    for (int mu = 0; mu < D - 1; ++mu) {
#pragma unroll
      for (int nu = mu + 1; nu < D; ++nu) {
        const float2 a = __ldg(lat + nu * g.V + q * g.Vh + i + fwd[mu]);  // U_nu(x+mu)
        const float2 b = __ldg(lat + mu * g.V + q * g.Vh + i + fwd[nu]);  // U_mu(x+nu)
        plaq_accum(U[mu], a, b, U[nu], nu == D - 1, vs);
      }
    }
  }
}

// Per-thread terms of measurement block `block` (layout MeasK): vs[0..3] +=
// (1 - Re P, -Im P) of the SS and ST plaquettes, vs[4..5] += the Polyakov
// loop.  lp: kRedThreads float2 of shared memory.  Every thread of the
// block must call it (the Polyakov blocks synchronise).  Shared by the
// single-lattice and batched measurements.
template <int D>
__device__ __forceinline__ void measure_block_values(const float2 *__restrict__ lat, const GeomK &g, int block,
                                                     const MeasK &m, float (&vs)[6], float2 *lp) {
  if (block < m.nb_plaq) {
    const int t = block * blockDim.x + threadIdx.x;
    if (m.pair) {
      if (2 * t < g.Vh) plaq_sites_pair<D>(lat, g, 2 * t, vs);
    } else if (t < g.Vh) {
      plaq_site<D>(lat, g, t, vs);
    }
    return;
  }
  const int per_block = blockDim.x / m.chunks;
  const int sl = threadIdx.x % per_block, c = threadIdx.x / per_block;
  const int j = (block - m.nb_plaq) * per_block + sl;  // spatial site (EO order on the t = 0 slice)
  float2 L = make_float2(1.f, 0.f);
  if (j < g.Vs) {
    const int hs = g.Vs / 2;
    const int p = j >= hs ? 1 : 0;
    const int i = j - p * hs;
    const int Lc = g.N[D - 1] / m.chunks;
    const int est = g.es[D - 1];
    const float2 *base = lat + (D - 1) * g.V + i;
    const int t0 = c * Lc;
    // eight loads in flight, then their products in time order (a padded
    // factor is 1 + 0i, which leaves the product bit for bit unchanged)
    for (int tb = t0; tb < t0 + Lc; tb += 8) {
      float2 u[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int t = tb + k;
        u[k] = (t < t0 + Lc) ? __ldg(base + ((p + t) & 1) * g.Vh + t * est) : make_float2(1.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) L = cmul(L, u[k]);
    }
  }
  lp[threadIdx.x] = L;
  __syncthreads();
  if (c == 0 && j < g.Vs) {
    float2 P = lp[sl];
    for (int cc = 1; cc < m.chunks; ++cc) P = cmul(P, lp[cc * per_block + sl]);
    vs[4] += P.x;
    vs[5] += P.y;
  }
}

// FP64 block totals of the measurement terms: only the values this block
// kind produces (plaquette blocks: 0..3, Polyakov blocks: 4..5) go through
// the warp shuffles.  Thread k < 6 returns total k.
__device__ __forceinline__ double measure_block_total(const float (&vs)[6], bool plaq_block, double *smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int k0 = plaq_block ? 0 : 4, k1 = plaq_block ? 4 : 6;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    if (k < k0 || k >= k1) continue;
    const double w = warp_sum((double)vs[k]);
    if (lane == 0) smem[warp * 6 + k] = w;
  }
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x >= k0 && threadIdx.x < k1)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += smem[w * 6 + threadIdx.x];
  __syncthreads();
  return t;
}

// Fused plaquette + Polyakov loop, one launch of m.nb_plaq + m.nb_poly blocks
// (layout MeasK).  out = {SS re, SS im, ST re, ST im, L re, L im}: mean of
// (1 - e^{i theta_P}) per class and (1/V_s) sum_x prod_t U_t.
template <int D>
static __global__ void __launch_bounds__(kRedThreads)
    k_measure(const float2 *__restrict__ lat, GeomK g, MeasK m, double *partials, unsigned int *counter,
              double *out, double normSS, double normST, double normL) {
  __shared__ double smem[kRedWarps * 6];
  __shared__ float2 lp[kRedThreads];
  float vs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // per-thread partial sums of a few terms
  measure_block_values<D>(lat, g, (int)blockIdx.x, m, vs, lp);
  const double tot = measure_block_total(vs, (int)blockIdx.x < m.nb_plaq, smem);
  const double scale[6] = {normSS, normSS, normST, normST, normL, normL};
  finish_block_totals<6>(tot, smem, partials, counter, out, scale);
}

// I1(x)/I0(x) by backward evaluation of the Gauss continued fraction
// r_k = I_k/I_{k-1} = x / (2k + x r_{k+1}) (from the recurrence
// I_{k-1} - I_{k+1} = (2k/x) I_k), truncated at depth ceil(x)+16 where the
// remaining tail is below float precision.  Replaces CUDA's
// cyl_bessel_i1/cyl_bessel_i0 used by the reference
// (include/lattice_functions.h:101).
__device__ __forceinline__ float bessel_ratio_i1_i0(float x) {
  const int K = (int)x + 16;
  float r = 0.0f;
  for (int k = K; k >= 1; --k) r = __fdividef(x, fmaf(x, r, 2.0f * (float)k));
  return r;
}

// Analytic multihit mean of the temporal link at site x (parity p, EO index
// i): conj(S) * I1(beta|S|) / (|S| I0(beta|S|)).
template <int D>
__device__ __forceinline__ float2 multihit_link(const float2 *__restrict__ lat, const GeomK &g,
                                                const CoupK &c, const int x[4], int i, int p) {
  const float2 S = staple_at<D>(lat, g, c, x, i, p, g.tdir);
  const float alpha = sqrtf(fmaf(S.x, S.x, S.y * S.y));
  if (!(alpha > 0.f)) return make_float2(0.f, 0.f);
  const float t = bessel_ratio_i1_i0(c.beta * alpha) / alpha;
  return make_float2(t * S.x, -t * S.y);
}

// Spatial lexicographic index s -> x[0..tdir-1] (reference indexIdS /
// indexNOSD, include/index.h:19-24,80-84).
__device__ __forceinline__ void spatial_decode(const GeomK &g, int s, int x[4]) {
  x[0] = x[1] = x[2] = x[3] = 0;
  int r = s;
  for (int k = 0; k < g.tdir; ++k) {
    x[k] = r % g.N[k];
    r /= g.N[k];
  }
}

// P(x) = prod_t U_t(x,t) (or of the multihit means) for every spatial site,
// stored in spatial lexicographic order; products in FP64.
template <int D, bool MH>
static __global__ void __launch_bounds__(256)
    k_poly_field(const float2 *__restrict__ lat, GeomK g, CoupK c, double2 *P) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.Vs) return;
  int x[4];
  spatial_decode(g, s, x);
  double2 prod = make_double2(1.0, 0.0);
  const int Nt = g.N[g.tdir];
  for (int t = 0; t < Nt; ++t) {
    int y[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) y[k] = (k == g.tdir) ? t : x[k];
    const int i = eo_index(g, y);
    const int p = (y[0] + y[1] + y[2] + y[3]) & 1;
    float2 u;
    if (MH)
      u = multihit_link<D>(lat, g, c, y, i, p);
    else
      u = __ldg(lat + (size_t)g.tdir * g.V + (size_t)p * g.Vh + i);
    prod = zmul(prod, make_double2((double)u.x, (double)u.y));
  }
  P[s] = prod;
}

// C(r) = norm * sum_x sum_{i<d-1} P(x) conj(P(x + r e_i)), r = 1..R.
// partials: gridDim.x * 2R doubles; out: 2R doubles.
static __global__ void __launch_bounds__(kRedThreads)
    k_poly_corr(const double2 *__restrict__ P, GeomK g, int R, double *partials,
                unsigned int *counter, double *out, double norm) {
  __shared__ double smem[kRedWarps * 2];
  __shared__ bool am_last;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  int x[4];
  double2 P0 = make_double2(0.0, 0.0);
  if (s < g.Vs) {
    spatial_decode(g, s, x);
    P0 = P[s];
  }
  for (int r = 1; r <= R; ++r) {
    double v[2] = {0.0, 0.0};
    if (s < g.Vs) {
      for (int dir = 0; dir < g.tdir; ++dir) {
        int sp = 0, stride = 1;
        for (int k = 0; k < g.tdir; ++k) {
          int xk = x[k];
          if (k == dir) xk = (xk + r) % g.N[k];
          sp += xk * stride;
          stride *= g.N[k];
        }
        double2 q = zmulc(P0, P[sp]);
        v[0] += q.x;
        v[1] += q.y;
      }
    }
    block_sum<2>(v, smem);
    if (threadIdx.x < 2) partials[(size_t)blockIdx.x * 2 * R + 2 * (r - 1) + threadIdx.x] = v[0];
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  for (int k = 0; k < 2 * R; ++k) {
    double w[1] = {strided_partial_sum(partials, gridDim.x, 2 * R, k)};
    block_sum<1>(w, smem);
    if (threadIdx.x == 0) out[k] = w[0] * norm;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

}  // namespace u1b
