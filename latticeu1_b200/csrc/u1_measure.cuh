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

// Store this block's NV totals, take a ticket; the last block sums all
// partials in block order and writes out[k] = scale[k] * total_k.
// Returns nothing; `counter` is reset to 0 by the last block.
template <int NV>
__device__ __forceinline__ void partials_finish(double (&v)[NV], double *smem, double *partials,
                                                unsigned int *counter, double *out,
                                                const double (&scale)[NV]) {
  __shared__ bool am_last;
  block_sum<NV>(v, smem);
  if (threadIdx.x < NV) partials[(size_t)blockIdx.x * NV + threadIdx.x] = v[0];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double w[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
      t += __ldcg(partials + (size_t)b * NV + k);
    w[k] = t;
  }
  block_sum<NV>(w, smem);
  if (threadIdx.x < NV) out[threadIdx.x] = w[0] * scale[threadIdx.x];
  if (threadIdx.x == 0) *counter = 0u;
}

// Per-thread terms of measurement block `block` (layout as k_measure below):
// vs[0..3] += (1 - Re P, -Im P) of the SS and ST plaquettes, vs[4..5] += the
// Polyakov loop.  Shared by the single-lattice and batched measurements.
template <int D>
__device__ __forceinline__ void measure_block_values(const float2 *__restrict__ lat, const GeomK &g, int block,
                                                     int nb_plaq, float (&vs)[6]) {
  if (block < nb_plaq) {
    const int i = block * blockDim.x + threadIdx.x;
    if (i < g.Vh) {
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
            const float2 P = cmulc(cmulc(cmul(U[mu], a), b), U[nu]);
            if (nu == D - 1) {
              vs[2] += 1.f - P.x;
              vs[3] -= P.y;
            } else {
              vs[0] += 1.f - P.x;
              vs[1] -= P.y;
            }
          }
        }
      }
    }
  } else {
    const int j = (block - nb_plaq) * blockDim.x + threadIdx.x;
    if (j < g.Vs) {
      const int hs = g.Vs / 2;
      const int p = j >= hs ? 1 : 0;
      const int i = j - p * hs;
      const int Nt = g.N[D - 1];
      const int est = g.es[D - 1];
      const float2 *base = lat + (D - 1) * g.V + i;
      float2 L0 = make_float2(1.f, 0.f), L1 = L0;  // even / odd t partial products
#pragma unroll 4
      for (int t = 0; t + 1 < Nt; t += 2) {
        L0 = cmul(L0, __ldg(base + ((p + t) & 1) * g.Vh + t * est));
        L1 = cmul(L1, __ldg(base + ((p + t + 1) & 1) * g.Vh + (t + 1) * est));
      }
      const float2 L = cmul(L0, L1);  // Nt is even
      vs[4] += L.x;
      vs[5] += L.y;
    }
  }
}

// Fused plaquette + Polyakov loop, one launch of nb_plaq + nb_poly blocks.
// Blocks [0, nb_plaq): thread i handles the plaquettes mu<nu at EO sites
// (i, parity 0) and (i, parity 1).  Blocks [nb_plaq, ...): thread j handles
// the Polyakov loop of spatial site j (EO order on the t = 0 slice), so the
// Nt-long products are spread over their own blocks.
// out = {SS re, SS im, ST re, ST im, L re, L im}: mean of (1 - e^{i theta_P})
// per class and (1/V_s) sum_x prod_t U_t.
template <int D>
static __global__ void __launch_bounds__(kRedThreads)
    k_measure(const float2 *__restrict__ lat, GeomK g, int nb_plaq, double *partials, unsigned int *counter,
              double *out, double normSS, double normST, double normL) {
  __shared__ double smem[kRedWarps * 6];
  float vs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // per-thread partial sums of a few terms
  measure_block_values<D>(lat, g, (int)blockIdx.x, nb_plaq, vs);
  double v[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = (double)vs[k];
  const double scale[6] = {normSS, normSS, normST, normST, normL, normL};
  partials_finish<6>(v, smem, partials, counter, out, scale);
}

// Blocks of the fused measurement: plaquette blocks then Polyakov blocks.
__host__ inline int measure_plaq_blocks(const GeomK &g) { return (g.Vh + kRedThreads - 1) / kRedThreads; }
__host__ inline int measure_poly_blocks(const GeomK &g) { return (g.Vs + kRedThreads - 1) / kRedThreads; }

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
    double w[1] = {0.0};
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
      w[0] += __ldcg(partials + (size_t)b * 2 * R + k);
    block_sum<1>(w, smem);
    if (threadIdx.x == 0) out[k] = w[0] * norm;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

}  // namespace u1b
