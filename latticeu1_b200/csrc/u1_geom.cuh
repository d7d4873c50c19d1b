// Lattice geometry and even/odd (EO) indexing for the sm_100a kernels.
//
// The EO site index is the reference's (include/index.h:114-153):
//   lexicographic id = x0 + N0*(x1 + N1*(x2 + N2*x3)),  EO index = id >> 1,
//   parity = (x0+x1+x2+x3) & 1,  link (x, mu) at  eo + parity*V/2 + mu*V.
// Because N0 is even, EO index = (x0 >> 1) + hN0*(x1 + N1*(x2 + N2*x3)),
// which is what eo_index() computes; for EO index i of parity p the site is
// x0 = 2*(i mod hN0) + ((x1+x2+x3+p) & 1) (reference include/index.h:114-122).
// Unused directions have extent 1 (reference src/parameters.cu:150-161).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace u1b {

// Division by a runtime constant d as a multiply-high and a shift
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI'94): for 0 <= n < 2^31,
// n / d = (umulhi(n, mul) + n) >> shift with shift = ceil(log2 d) and
// mul = floor(2^32 (2^shift - d) / d) + 1.
struct FastDivK {
  uint32_t mul;
  uint32_t shift;
};

struct GeomK {
  int dims;
  int tdir;
  int N[4];   // Grid[0..3]
  int hN0;    // N[0] / 2
  int es[4];  // EO stride of x1, x2, x3 (es[0] unused = 0)
  int V;      // volume
  int Vh;     // V / 2
  int Vs;     // spatial volume (product of Grid[0..tdir-1])
  FastDivK fd[3];  // division by hN0, N[1], N[2]
  int wrapf[4];    // EO-index step of x -> x + e_nu across the upper boundary
  int wrapb[4];    // EO-index step of x -> x - e_nu across the lower boundary
};

__host__ __device__ inline FastDivK make_fastdiv(uint32_t d) {
  uint32_t sh = 0;
  while ((1ull << sh) < d) ++sh;
  FastDivK f;
  f.shift = sh;
  f.mul = (uint32_t)((((1ull << 32) * ((1ull << sh) - d)) / d) + 1ull);
  return f;
}

__host__ __device__ __forceinline__ uint32_t fast_div(uint32_t n, FastDivK f) {
#if defined(__CUDA_ARCH__)
  return (__umulhi(n, f.mul) + n) >> f.shift;
#else
  return (uint32_t)((((uint64_t)n * f.mul) >> 32) + n) >> f.shift;
#endif
}

// Fill the derived fields (strides, fast divisors, wrap steps) from N[], dims.
__host__ inline void geom_finish(GeomK &g) {
  g.tdir = g.dims - 1;
  g.hN0 = g.N[0] / 2;
  g.es[0] = 0;
  g.es[1] = g.hN0;
  g.es[2] = g.hN0 * g.N[1];
  g.es[3] = g.hN0 * g.N[1] * g.N[2];
  g.V = g.N[0] * g.N[1] * g.N[2] * g.N[3];
  g.Vh = g.V / 2;
  g.Vs = 1;
  for (int k = 0; k < g.tdir; ++k) g.Vs *= g.N[k];
  g.fd[0] = make_fastdiv((uint32_t)g.hN0);
  g.fd[1] = make_fastdiv((uint32_t)g.N[1]);
  g.fd[2] = make_fastdiv((uint32_t)g.N[2]);
  g.wrapf[0] = 1 - g.hN0;
  g.wrapb[0] = g.hN0 - 1;
  for (int k = 1; k < 4; ++k) {
    g.wrapf[k] = -(g.N[k] - 1) * g.es[k];
    g.wrapb[k] = (g.N[k] - 1) * g.es[k];
  }
}

// Staple weights and coupling (reference include/staple.h:79-102).
struct CoupK {
  float beta;
  float w_ss;  // 1/xi  for plaquettes with no temporal link
  float w_st;  // xi    for plaquettes with a temporal link
};

__device__ __forceinline__ void eo_decode(const GeomK &g, int i, int p, int x[4]) {
  int k = i % g.hN0;
  int r = i / g.hN0;
  x[1] = r % g.N[1];
  r /= g.N[1];
  x[2] = r % g.N[2];
  x[3] = r / g.N[2];
  x[0] = 2 * k + ((x[1] + x[2] + x[3] + p) & 1);
}

// Site of EO index i (parity p) via the fast divisors; k = i mod hN0.
template <int D>
__device__ __forceinline__ void eo_decode_fast(const GeomK &g, int i, int p, int x[4], int &k) {
  const uint32_t r = fast_div((uint32_t)i, g.fd[0]);
  k = i - (int)r * g.hN0;
  if (D == 2) {
    x[1] = (int)r;
    x[2] = x[3] = 0;
  } else {
    const uint32_t r1 = fast_div(r, g.fd[1]);
    x[1] = (int)r - (int)r1 * g.N[1];
    if (D == 3) {
      x[2] = (int)r1;
      x[3] = 0;
    } else {
      const uint32_t r2 = fast_div(r1, g.fd[2]);
      x[2] = (int)r1 - (int)r2 * g.N[2];
      x[3] = (int)r2;
    }
  }
  x[0] = 2 * k + ((x[1] + x[2] + x[3] + p) & 1);
}

// EO-index steps from site x (EO index i, row offset k) to its neighbours of
// opposite parity: x + e_nu = i + fwd[nu], x - e_nu = i + bwd[nu].  Along x0
// the step depends on x0's parity (x0 = 2k + odd); along the others it is
// +-es[nu], wrapped at the boundary.  Two steps along different directions
// add: x + e_mu - e_nu = i + fwd[mu] + bwd[nu] (mu != nu).
template <int D>
__device__ __forceinline__ void eo_steps(const GeomK &g, const int x[4], int k, int fwd[4], int bwd[4]) {
  const int odd = x[0] & 1;
  fwd[0] = odd ? ((k == g.hN0 - 1) ? g.wrapf[0] : 1) : 0;
  bwd[0] = odd ? 0 : ((k == 0) ? g.wrapb[0] : -1);
#pragma unroll
  for (int nu = 1; nu < 4; ++nu) {
    if (nu < D) {
      fwd[nu] = (x[nu] == g.N[nu] - 1) ? g.wrapf[nu] : g.es[nu];
      bwd[nu] = (x[nu] == 0) ? g.wrapb[nu] : -g.es[nu];
    } else {
      fwd[nu] = bwd[nu] = 0;
    }
  }
}

__device__ __forceinline__ int eo_index(const GeomK &g, const int x[4]) {
  return (x[0] >> 1) + x[1] * g.es[1] + x[2] * g.es[2] + x[3] * g.es[3];
}

__device__ __forceinline__ int wrap_inc(int v, int n) { return (v + 1 == n) ? 0 : v + 1; }
__device__ __forceinline__ int wrap_dec(int v, int n) { return (v == 0) ? n - 1 : v - 1; }

}  // namespace u1b
