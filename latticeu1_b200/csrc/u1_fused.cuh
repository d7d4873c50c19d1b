// Sweep with the plaquette + Polyakov measurement taken from its last pass.
//
// Phases (parity 1, MU = 1..D-1) of the sweep's last pass run as the
// measuring kernels below: they update their links exactly as the plain
// phase kernels (same body, bit-identical links) and, from the staple terms
// they already hold, add every plaquette (nu, MU), nu < MU, of the final
// configuration once (derivation at update_single_body).  Each writes per-block
// partial sums (re, im) into its slot MU-1.  After the sweep, k_poly_finish
// computes the Polyakov loops (time-chunked, as k_measure) and its last block
// sums all partials in a fixed order into the 6 observables.
//
// Reference computations replaced: plaquette src/plaquette.cu:93-118 and
// Polyakov loop src/polyakov.cu:60-77, taken after UpdateLattice
// (reference u1.cpp:120-126 measures right after each update).
#pragma once
#include "u1_measure.cuh"

namespace u1b {

template <int D, int MU, bool MET, int SRC = SRC_PHILOX>
static __global__ void __launch_bounds__(256, 8) k_update_pair_meas(const UpdArgs a, double *partials) {
  __shared__ double smem[kRedWarps * 2];
  float2 m = make_float2(0.f, 0.f);
  const int b = rev_block(a, (int)blockIdx.x, (int)gridDim.x);
  update_pair_body<D, MU, MET, SRC, true>(a, 2 * (b * (int)blockDim.x + (int)threadIdx.x), &m);
  double v[2] = {(double)m.x, (double)m.y};
  block_sum<2>(v, smem);
  if (threadIdx.x < 2) partials[2 * b + threadIdx.x] = v[0];  // slot of the work item: any block order sums alike
}

template <int D, int MU, bool MET, int SRC = SRC_PHILOX>
static __global__ void __launch_bounds__(256) k_update_meas(const UpdArgs a, double *partials) {
  __shared__ double smem[kRedWarps * 2];
  float2 m = make_float2(0.f, 0.f);
  const int b = rev_block(a, (int)blockIdx.x, (int)gridDim.x);
  update_single_body<D, MU, MET, SRC, true>(a, b * (int)blockDim.x + (int)threadIdx.x, &m);
  double v[2] = {(double)m.x, (double)m.y};
  block_sum<2>(v, smem);
  if (threadIdx.x < 2) partials[2 * b + threadIdx.x] = v[0];  // slot of the work item: any block order sums alike
}

// Four sites per thread, 128 threads (512 sites) per block: the same work
// items and partial slots as k_update_pair_meas.
template <int D, int MU, bool MET, int SRC = SRC_PHILOX>
static __global__ void __launch_bounds__(128, 7) k_update_quad_meas(const UpdArgs a, double *partials) {
  __shared__ double smem[kRedWarps * 2];
  float2 m = make_float2(0.f, 0.f);
  const int b = a.rev ? rev_block(a, (int)blockIdx.x, (int)gridDim.x)
                      : sm_local_block((int)blockIdx.x, (int)gridDim.x, a.sms);
  update_quad_body<D, MU, MET, SRC, true>(a, 4 * (b * (int)blockDim.x + (int)threadIdx.x), &m);
  double v[2] = {(double)m.x, (double)m.y};
  block_sum<2>(v, smem);
  if (threadIdx.x < 2) partials[2 * b + threadIdx.x] = v[0];  // slot of the work item: any block order sums alike
}

// Blocks of one measuring phase (pair kernels when N0/2 is even).
__host__ inline int meas_phase_blocks(const GeomK &g) {
  const int threads = (g.hN0 & 1) ? g.Vh : g.Vh / 2;
  return (threads + 255) / 256;
}

// Polyakov blocks (layout MeasK, poly part) + the final sum.  phase_partials:
// D-1 slots of nb_phase (re, im) pairs; poly_partials: 2 doubles per block.
// out = {SS re, SS im, ST re, ST im, L re, L im} with the norms applied.
template <int D>
static __global__ void __launch_bounds__(kRedThreads)
    k_poly_finish(const float2 *__restrict__ lat, GeomK g, MeasK m, const double *phase_partials, int nb_phase,
                  double *poly_partials, unsigned int *counter, double *out, double normSS, double normST,
                  double normL) {
  __shared__ double smem[kRedWarps * 6];
  __shared__ float2 lp[kRedThreads];
  __shared__ bool am_last;
  float vs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  pdl_wait_prior_grid();  // launched early (programmatic dependent launch): wait for the sweep's last phase
  measure_block_values<D>(lat, g, (int)blockIdx.x + m.nb_plaq, m, vs, lp);  // Polyakov blocks only
  const double tot = measure_block_total(vs, false, smem);                 // threads 4, 5
  if (threadIdx.x >= 4 && threadIdx.x < 6) {
    poly_partials[2 * blockIdx.x + threadIdx.x - 4] = tot;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  // Thread j adds the (re, im) pairs of blocks j, j + blockDim, ... of every
  // slot and of the Polyakov blocks, in that order; the loads of a round (and,
  // unrolled, of four rounds) are independent, so they are in flight together.
  double w[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const int nrounds = (max(nb_phase, (int)gridDim.x) + blockDim.x - 1) / blockDim.x;
#pragma unroll 4
  for (int r = 0; r < nrounds; ++r) {
    const int b = r * blockDim.x + threadIdx.x;
    double2 t[D];  // slots 0..D-2, then the Polyakov pair
#pragma unroll
    for (int s = 0; s < D - 1; ++s)
      t[s] = (b < nb_phase) ? __ldcg(reinterpret_cast<const double2 *>(phase_partials) + (size_t)s * nb_phase + b)
                            : make_double2(0.0, 0.0);
    t[D - 1] = (b < (int)gridDim.x) ? __ldcg(reinterpret_cast<const double2 *>(poly_partials) + b)
                                    : make_double2(0.0, 0.0);
#pragma unroll
    for (int s = 0; s < D - 1; ++s) {
      const int o = (s + 1 == D - 1) ? 2 : 0;  // slot s holds plaquettes (nu, s+1): temporal iff s+1 = D-1
      w[o] += t[s].x;
      w[o + 1] += t[s].y;
    }
    w[4] += t[D - 1].x;
    w[5] += t[D - 1].y;
  }
  block_sum<6>(w, smem);
  const double scale[6] = {normSS, normSS, normST, normST, normL, normL};
  if (threadIdx.x < 6) out[threadIdx.x] = w[0] * scale[threadIdx.x];
  if (threadIdx.x == 0) *counter = 0u;
}

}  // namespace u1b
