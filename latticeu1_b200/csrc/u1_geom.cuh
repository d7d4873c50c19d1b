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

struct GeomK {
  int dims;
  int tdir;
  int N[4];   // Grid[0..3]
  int hN0;    // N[0] / 2
  int es[4];  // EO stride of x1, x2, x3 (es[0] unused = 0)
  int V;      // volume
  int Vh;     // V / 2
  int Vs;     // spatial volume (product of Grid[0..tdir-1])
};

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

__device__ __forceinline__ int eo_index(const GeomK &g, const int x[4]) {
  return (x[0] >> 1) + x[1] * g.es[1] + x[2] * g.es[2] + x[3] * g.es[3];
}

__device__ __forceinline__ int wrap_inc(int v, int n) { return (v + 1 == n) ? 0 : v + 1; }
__device__ __forceinline__ int wrap_dec(int v, int n) { return (v == 0) ? n - 1 : v - 1; }

}  // namespace u1b
