// The last phase of a sweep fused with the plaquette + Polyakov measurement.
//
// The last phase of a pass updates the temporal links of odd sites (parity
// 1, mu = T); every other link is already final.  One thread per
// (pair of spatial sites x0 = 2m, 2m+1; time chunk) walks t through its
// chunk; at each t one of its two sites is odd, and at that site x it:
//   * updates U_T(x) if x is odd, with the same staple and update functions
//     (staple_steps, update_one) as the phase kernels, so the links are
//     bit-identical to an unfused sweep;
//   * adds the spatial-spatial plaquettes at both sites (spatial links are final);
//   * adds the space-time plaquettes that contain the odd link U_T(x):
//     P_jT(x) and P_jT(x - j).  Every space-time plaquette holds exactly one
//     odd-site temporal link, so each is counted once, by that link's owner;
//   * multiplies U_T(x) into the chunk's Polyakov partial product.
// The chunk products of a spatial site are combined in shared memory, and
// all sums go through the deterministic FP64 block/partials reduction.
//
// Reference computations fused here: plaquette src/plaquette.cu:93-118 and
// Polyakov loop src/polyakov.cu:60-77, taken after UpdateLattice
// (reference u1.cpp:120-126 measures right after each update).
#pragma once
#include "u1_measure.cuh"

namespace u1b {

constexpr int kFusedThreads = 256;

template <int D, bool MET>
static __global__ void __launch_bounds__(kFusedThreads)
    k_update_last_measure(const UpdArgs a, int chunks, double *partials, unsigned int *counter, double *out,
                          double normSS, double normST, double normL) {
  __shared__ double smem[kRedWarps * 6];
  __shared__ float2 lp[2][kFusedThreads];
  const GeomK &g = a.g;
  constexpr int T = D - 1;
  // thread <-> (spatial EO row index e on the t = 0 slice, time chunk): the
  // two spatial sites x0 = 2m, 2m+1 share EO index i = e + t*es[T] at every
  // t, one of parity 0 and one of parity 1, so each thread updates exactly
  // one (odd-site) temporal link per time slice: no divergence.
  const int per_block = kFusedThreads / chunks;
  const int sl = threadIdx.x % per_block;
  const int chunk = threadIdx.x / per_block;
  const int e = blockIdx.x * per_block + sl;
  const int Vs2 = g.Vs / 2;
  const bool active = e < Vs2;
  int x[4] = {0, 0, 0, 0};
  int m = 0;
  {
    // e = m + x1*es1 + x2*es2 (spatial part of the EO index)
    int r = active ? e : 0;
    m = r % g.hN0;
    r /= g.hN0;
#pragma unroll
    for (int k = 1; k < T; ++k) {
      x[k] = r % g.N[k];
      r /= g.N[k];
    }
  }
  const int Lc = g.N[T] / chunks;
  pdl_wait_prior_grid();
  if (!MET && a.bump_ptr != nullptr && blockIdx.x == 0 && threadIdx.x == 0) *a.bump_ptr += a.bump_by;
  float vs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // per-thread partial sums (few terms)
  float2 LA = make_float2(1.f, 0.f), LB = LA;    // Polyakov partial products of x0 = 2m and 2m+1
  if (active) {
    const float2 *lat = a.lat;
    for (int tt = 0; tt < Lc; ++tt) {
      x[T] = chunk * Lc + tt;
      const int i = e + x[T] * g.es[T];
      int rest = 0;
#pragma unroll
      for (int k = 1; k < 4; ++k) rest += x[k];
      const int oddbit = (rest + 1) & 1;  // x0 & 1 of the parity-1 site
      // ---- the parity-1 site: update its temporal link
      x[0] = 2 * m + oddbit;
      int fwd[4], bwd[4];
      eo_steps<D>(g, x, m, fwd, bwd);
      float2 *own = a.lat + T * g.V + g.Vh + i;
      const float2 S = staple_steps<D, T>(a.lat, g, a.c, i, 1, fwd, bwd);
      const float2 UT = update_one<D, T, MET, false>(a, i, S, *own);
      *own = UT;
      // space-time plaquettes holding U_T(x): P_jT(x) and P_jT(x - j)
#pragma unroll
      for (int j = 0; j < T; ++j) {
        const float2 uj = __ldg(lat + j * g.V + g.Vh + i);
        const float2 ut_xj = __ldg(lat + T * g.V + i + fwd[j]);
        const float2 uj_xt = __ldg(lat + j * g.V + i + fwd[T]);
        const float2 P1 = cmulc(cmulc(cmul(uj, ut_xj), uj_xt), UT);
        const float2 uj_m = __ldg(lat + j * g.V + i + bwd[j]);
        const float2 uj_mt = __ldg(lat + j * g.V + g.Vh + i + bwd[j] + fwd[T]);
        const float2 ut_m = __ldg(lat + T * g.V + i + bwd[j]);
        const float2 P2 = cmulc(cmulc(cmul(uj_m, UT), uj_mt), ut_m);
        vs[2] += (1.f - P1.x) + (1.f - P2.x);
        vs[3] -= P1.y + P2.y;
      }
      // spatial-spatial plaquettes at both sites (parity 1 then parity 0)
#pragma unroll
      for (int par = 1; par >= 0; --par) {
        int f2[4], b2[4];
        if (par == 0) {
          x[0] = 2 * m + (1 - oddbit);
          eo_steps<D>(g, x, m, f2, b2);
        } else {
#pragma unroll
          for (int k = 0; k < 4; ++k) f2[k] = fwd[k];
        }
        const int q = 1 - par;
#pragma unroll
        for (int mu = 0; mu < T; ++mu) {
#pragma unroll
          for (int nu = mu + 1; nu < T; ++nu) {
            const float2 umu = __ldg(lat + mu * g.V + par * g.Vh + i);
            const float2 unu = __ldg(lat + nu * g.V + par * g.Vh + i);
            const float2 b1 = __ldg(lat + nu * g.V + q * g.Vh + i + f2[mu]);
            const float2 bb = __ldg(lat + mu * g.V + q * g.Vh + i + f2[nu]);
            const float2 P = cmulc(cmulc(cmul(umu, b1), bb), unu);
            vs[0] += 1.f - P.x;
            vs[1] -= P.y;
          }
        }
      }
      // Polyakov partial products: x0 = 2m is the parity-1 site when oddbit == 0
      const float2 UT0 = __ldg(lat + T * g.V + i);
      if (oddbit == 0) {
        LA = cmul(LA, UT);
        LB = cmul(LB, UT0);
      } else {
        LA = cmul(LA, UT0);
        LB = cmul(LB, UT);
      }
    }
  }
  lp[0][threadIdx.x] = LA;
  lp[1][threadIdx.x] = LB;
  __syncthreads();
  double v[6];
#pragma unroll
  for (int k = 0; k < 4; ++k) v[k] = (double)vs[k];
  v[4] = v[5] = 0.0;
  if (active && chunk == 0) {
    float2 PA = lp[0][sl], PB = lp[1][sl];
    for (int c = 1; c < chunks; ++c) {
      PA = cmul(PA, lp[0][c * per_block + sl]);
      PB = cmul(PB, lp[1][c * per_block + sl]);
    }
    v[4] = (double)PA.x + (double)PB.x;
    v[5] = (double)PA.y + (double)PB.y;
  }
  pdl_release_dependents();
  const double scale[6] = {normSS, normSS, normST, normST, normL, normL};
  partials_finish<6>(v, smem, partials, counter, out, scale);
}

// Time chunks per spatial site: the largest of 8, 4, 2, 1 dividing Nt.
__host__ inline int fused_chunks(const GeomK &g) {
  const int Nt = g.N[g.dims - 1];
  for (int c = 8; c > 1; c >>= 1)
    if (Nt % c == 0) return c;
  return 1;
}
__host__ inline int fused_blocks(const GeomK &g) {
  const int per_block = kFusedThreads / fused_chunks(g);
  return (g.Vs / 2 + per_block - 1) / per_block;
}

}  // namespace u1b
