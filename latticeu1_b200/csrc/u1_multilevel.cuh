// Two-level (Luscher-Weisz style) Polyakov-loop correlator kernels.
//
// Reference algorithm being replaced (src/multilevel.cu):
//   multihit field      kernel_l2_multilevel_0<true>   :239-258
//   level-2 tensor T2   kernel_l2_multilevel_1         :331-360 (layout :354)
//   level-4 tensor T4   kernel_l2avg_l4_multilevel     :439-456
//   final C(r)          kernel_l4avg_Final_multilevel  :532-553
// Tensor layout (as the reference): element (x, r, i, slab) at
//   x + Vs*(r-1) + Vs*R*i + Vs*R*(d-1)*slab,   x spatial lexicographic.
// Multihit links are formed in FP32 from the float2 links; every slab
// product and the T2/T4 accumulation are FP64 complex.
#pragma once
#include "u1_measure.cuh"

namespace u1b {

// Multihit mean of every temporal link, stored at the 4D lexicographic index.
template <int D>
static __global__ void __launch_bounds__(256)
    k_ml_mhit_field(const float2 *__restrict__ lat, GeomK g, CoupK c, float2 *mh) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.V) return;
  int x[4];
  int r = id;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x[k] = r % g.N[k];
    r /= g.N[k];
  }
  const int i = eo_index(g, x);
  const int p = (x[0] + x[1] + x[2] + x[3]) & 1;
  mh[id] = multihit_link<D>(lat, g, c, x, i, p);
}

__device__ __forceinline__ int spatial_shift(const GeomK &g, const int x[4], int dir, int r) {
  int sp = 0, stride = 1;
  for (int k = 0; k < g.tdir; ++k) {
    int xk = x[k];
    if (k == dir) xk = (xk + r) % g.N[k];
    sp += xk * stride;
    stride *= g.N[k];
  }
  return sp;
}

// T2[x, r, i, slab] += prod_{t in slab} mh(x,t) * prod_{t in slab} conj(mh(x + r e_i, t)),
// slabs of thickness 2.  One thread per (x, r, i).  T2 does not alias mh,
// and the slabs' read-modify-writes touch distinct elements, so four of
// them are unrolled with their loads in flight together.
static __global__ void __launch_bounds__(256)
    k_ml_T2(const float2 *__restrict__ mh, GeomK g, int R, double2 *__restrict__ T2) {
  const size_t size = (size_t)g.Vs * R * g.tdir;
  const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= size) return;
  const int s = (int)(id % g.Vs);
  const int rest = (int)(id / g.Vs);
  const int r = rest % R + 1;
  const int dir = rest / R;
  int x[4];
  spatial_decode(g, s, x);
  const int sp = spatial_shift(g, x, dir, r);
  const int nl2 = g.N[g.tdir] / 2;
#pragma unroll 4
  for (int l = 0; l < nl2; ++l) {
    double2 p0 = make_double2(1.0, 0.0), p1 = make_double2(1.0, 0.0);
#pragma unroll
    for (int dt = 0; dt < 2; ++dt) {
      const int t = 2 * l + dt;
      const float2 a = __ldg(mh + (size_t)t * g.Vs + s);
      const float2 b = __ldg(mh + (size_t)t * g.Vs + sp);
      p0 = zmul(p0, make_double2(a.x, a.y));
      p1 = zmulc(p1, make_double2(b.x, b.y));
    }
    double2 *dst = T2 + id + size * l;
    *dst = zadd(*dst, zmul(p0, p1));
  }
}

// T4[., slab4] += prod_{two level-2 slabs} (T2 * l2norm).  One thread per (x, r, i).
static __global__ void __launch_bounds__(256)
    k_ml_T4(const double2 *__restrict__ T2, GeomK g, int R, double l2norm, double2 *T4) {
  const size_t size = (size_t)g.Vs * R * g.tdir;
  const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= size) return;
  const int nl4 = g.N[g.tdir] / 4;
  for (int l4 = 0; l4 < nl4; ++l4) {
    double2 a = zscale(T2[id + size * (2 * l4)], l2norm);
    double2 b = zscale(T2[id + size * (2 * l4 + 1)], l2norm);
    double2 *dst = T4 + id + size * l4;
    *dst = zadd(*dst, zmul(a, b));
  }
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
