// Two-level (Luscher-Weisz style) Polyakov-loop correlator kernels.
//
// Reference algorithm being replaced (src/multilevel.cu):
//   multihit field      kernel_l2_multilevel_0<true>   :239-258 (k_ml_slab2)
//   level-2 tensor T2   kernel_l2_multilevel_1         :331-360 (layout :354)
//   level-4 tensor T4   kernel_l2avg_l4_multilevel     :439-456
//   final C(r)          kernel_l4avg_Final_multilevel  :532-553
// Tensor layout (as the reference): element (x, r, i, slab) at
//   x + Vs*(r-1) + Vs*R*i + Vs*R*(d-1)*slab,   x spatial lexicographic.
// Multihit links are formed in FP32 from the float2 links; every slab
// product and the T2/T4 accumulation are FP64 complex.  The multihit links
// of each level-2 slab are multiplied once per (site, slab) (k_ml_slab2),
// so k_ml_T2 is a streaming read-modify-write of T2.
#pragma once
#include "u1_measure.cuh"

namespace u1b {

// Extents of the multilevel tensors (4D lattices: three spatial directions).
struct MlDims {
  int N0, N1, N2;  // spatial extents
  int Vs;          // N0 * N1 * N2
  int R;           // distances r = 1..R
  int nl2, nl4;    // level-2 and level-4 slabs
};

// Level-2 slab products of the multihit temporal links:
//   P2[x + Vs*l] = mh(x, 2l) * mh(x, 2l+1)   (FP64 complex), x spatial lexicographic,
// one thread per (x, l).  Each product is formed once here and read by all
// R*(d-1) partners of x in k_ml_T2 (reference kernel_l2_multilevel_0<true>,
// src/multilevel.cu:239-258, computes the multihit links; its
// kernel_l2_multilevel_1 re-forms both slab products per (x, r, i)).
static __global__ void __launch_bounds__(256)
    k_ml_slab2(const float2 *__restrict__ lat, GeomK g, CoupK c, const MlDims m, double2 *__restrict__ P2) {
  constexpr int D = 4;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= m.Vs * m.nl2) return;
  const int s = id % m.Vs, l = id / m.Vs;
  const int q = s / m.N0;
  int x[4] = {s % m.N0, q % m.N1, q / m.N1, 0};
  double2 p = make_double2(1.0, 0.0);
#pragma unroll
  for (int dt = 0; dt < 2; ++dt) {
    x[3] = 2 * l + dt;
    const int i = eo_index(g, x);
    const int par = (x[0] + x[1] + x[2] + x[3]) & 1;
    const float2 u = multihit_link<D>(lat, g, c, x, i, par);
    p = zmul(p, make_double2((double)u.x, (double)u.y));
  }
  P2[id] = p;
}

// Two consecutive double2 (32 bytes, 32-byte aligned) in one access.  The
// T2 / T4 tensors are streamed once per launch (no reuse): evict-first
// (.cs) keeps the L2-resident slab products and links in L2.
struct Z2 {
  double2 a, b;
};
__device__ __forceinline__ Z2 ld_z2_stream(const double2 *p) {
  Z2 v;
  asm volatile("ld.global.cs.v4.f64 {%0,%1,%2,%3}, [%4];"
               : "=d"(v.a.x), "=d"(v.a.y), "=d"(v.b.x), "=d"(v.b.y)
               : "l"(p));
  return v;
}
__device__ __forceinline__ void st_z2_stream(double2 *p, Z2 v) {
  asm volatile("st.global.cs.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v.a.x), "d"(v.a.y), "d"(v.b.x), "d"(v.b.y)
               : "memory");
}
__device__ __forceinline__ Z2 ld_z2(const double2 *p) {
  Z2 v;
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(v.a.x), "=d"(v.a.y), "=d"(v.b.x), "=d"(v.b.y) : "l"(p));
  return v;
}

// T2[x, r, i, slab] += P2[x, slab] * conj(P2[x + r e_i, slab]) for the
// level-2 slabs of thickness 2 (reference kernel_l2_multilevel_1,
// src/multilevel.cu:331-360; tensor layout :354).  One thread per pair of
// spatial sites (x, x+1) (N0 even: both in one x0-row) and one
// (r, i, slab): a 32-byte read-modify-write of T2 and 32-byte loads of the
// slab products.  Thread order is the tensor's element order, so a warp
// streams 1 KiB of T2.
static __global__ void __launch_bounds__(256)
    k_ml_T2(const double2 *__restrict__ P2, const MlDims m, double2 *__restrict__ T2) {
  const int Vs2 = m.Vs / 2;
  const long long npairs = (long long)Vs2 * m.R * 3 * m.nl2;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= npairs) return;
  const int s = 2 * (int)(id % Vs2);
  const int rest = (int)(id / Vs2);
  const int r = rest % m.R + 1;
  const int dir = (rest / m.R) % 3;
  const int l = rest / (m.R * 3);
  const int x0 = s % m.N0, q = s / m.N0;
  const int x1 = q % m.N1, x2 = q / m.N1;
  const double2 *P2l = P2 + (size_t)l * m.Vs;
  const Z2 pa = ld_z2(P2l + s);
  double2 pb0, pb1;
  if (dir == 0) {  // the shift runs along the row: the partners may wrap apart (r <= N0/2)
    const int row = s - x0;
    int y = x0 + r;
    y -= (y >= m.N0) ? m.N0 : 0;
    pb0 = __ldg(P2l + row + y);
    y += 1;
    y -= (y >= m.N0) ? m.N0 : 0;
    pb1 = __ldg(P2l + row + y);
  } else {  // the partners are consecutive and even (r <= N0/2 may exceed N1, N2)
    const int sp = dir == 1 ? s + ((x1 + r) % m.N1 - x1) * m.N0 : s + ((x2 + r) % m.N2 - x2) * m.N0 * m.N1;
    const Z2 pb = ld_z2(P2l + sp);
    pb0 = pb.a;
    pb1 = pb.b;
  }
  double2 *dst = T2 + 2 * id;  // = s + Vs*(r-1) + Vs*R*dir + Vs*R*3*l
  Z2 t = ld_z2_stream(dst);
  t.a = zadd(t.a, zmulc(pa.a, pb0));
  t.b = zadd(t.b, zmulc(pa.b, pb1));
  st_z2_stream(dst, t);
}

// T4[., slab4] += prod_{two level-2 slabs} (T2 * l2norm) (reference
// kernel_l2avg_l4_multilevel, src/multilevel.cu:439-456).  One thread per
// pair of consecutive tensor elements and level-4 slab: 32-byte accesses.
static __global__ void __launch_bounds__(256)
    k_ml_T4(const double2 *__restrict__ T2, const MlDims m, double l2norm, double2 *__restrict__ T4) {
  const long long half = (long long)m.Vs * m.R * 3 / 2;  // element pairs per slab
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= half * m.nl4) return;
  const long long e2 = id % half;
  const int l4 = (int)(id / half);
  const size_t size = 2 * (size_t)half;
  const Z2 a = ld_z2_stream(T2 + 2 * e2 + size * (2 * l4));
  const Z2 b = ld_z2_stream(T2 + 2 * e2 + size * (2 * l4 + 1));
  double2 *dst = T4 + 2 * e2 + size * l4;
  Z2 t = ld_z2_stream(dst);
  t.a = zadd(t.a, zmul(zscale(a.a, l2norm), zscale(b.a, l2norm)));
  t.b = zadd(t.b, zmul(zscale(a.b, l2norm), zscale(b.b, l2norm)));
  st_z2_stream(dst, t);
}

// C(r) = norm * sum_x sum_i prod_{slab4} (T4 * l4norm), r = 1..R.
static __global__ void __launch_bounds__(kRedThreads)
    k_ml_final(const double2 *__restrict__ T4, GeomK g, int R, double l4norm, double *partials,
               unsigned int *counter, double *out, double norm) {
  __shared__ double smem[kRedWarps * 2];
  __shared__ bool am_last;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t size = (size_t)g.Vs * R * g.tdir;
  const int nl4 = g.N[g.tdir] / 4;
  for (int r = 0; r < R; ++r) {
    double v[2] = {0.0, 0.0};
    if (s < g.Vs) {
      for (int dir = 0; dir < g.tdir; ++dir) {
        double2 pl = make_double2(1.0, 0.0);
        for (int l4 = 0; l4 < nl4; ++l4)
          pl = zmul(pl, zscale(T4[s + (size_t)g.Vs * r + (size_t)g.Vs * R * dir + size * l4], l4norm));
        v[0] += pl.x;
        v[1] += pl.y;
      }
    }
    block_sum<2>(v, smem);
    if (threadIdx.x < 2) partials[(size_t)blockIdx.x * 2 * R + 2 * r + threadIdx.x] = v[0];
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
