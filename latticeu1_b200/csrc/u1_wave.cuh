// One whole sweep in one persistent (cooperative) launch: a wavefront of
// checkerboard phases with neighbour-local synchronisation.
//
// A tile is every site with a given (x2, x3): hN0 * N1 EO sites per parity,
// two per thread (the pair body).  Phase (p, mu) of a tile reads links at
// (x2, x3) displacements of at most one step in each direction (staple
// neighbours x +- e_nu and x + e_mu - e_nu) and writes only its own (p, mu)
// links; within a phase no tile reads what another writes (checkerboard).  So
// a tile may start phase k once its eight (x2, x3) neighbours have finished
// phase k-1: that covers both the reads of links they wrote in phase k-1 and
// their reads of links this tile will overwrite.  Tiles publish completed
// phases in per-tile flags (release after a block barrier and fence; the
// watchers acquire), so the global barrier between phase kernels becomes a
// local one and neighbouring phases overlap across the device.
//
// Every block must be resident at once (the cooperative launch guarantees it
// or fails), so waits cannot deadlock; each wait is still bounded and, if it
// runs out, records the phase in `err` and abandons the sweep.  Links written
// in this launch are read with coherent loads (ld_vec2<true>), never through
// the non-coherent path.
//
// Measured on B200 at 32^4 it is correct (bit-identical to the phase kernels)
// but about 2x slower: the per-phase barrier, fence, flag publication and
// neighbour polling sit on every tile's critical path (2-3 us a phase, with
// no overlap inside a block), more than the ~1.3 us a phase boundary costs
// the phase kernels under programmatic dependent launch.  It is therefore
// opt-in (u1_lattice_set_variant 4) and not a tuner candidate.  The last block to finish bumps the Metropolis pass
// counter and clears the flags for the next launch.
#pragma once
#include "u1_fused.cuh"

namespace u1b {

struct WaveArgs {
  UpdArgs a;                   // links, geometry, coupling, rng key/chain/pass counter
  int metrop, ovrn;
  double *meas;                // measured sweep: D-1 slots of gridDim (re, im) pairs, or nullptr
  unsigned int *flags;         // per tile: phases completed in this sweep (0 at launch)
  unsigned int *ticket;        // blocks finished (0 at launch)
  unsigned int *err;           // 1 + phase of a wait that ran out (0: none)
  unsigned long long *pass_rw; // the pass counter (same address as a.pass_dev)
  unsigned spin_limit;         // polls per neighbour wait (>= 1)
  int stall_tile;              // a tile that never publishes its phases (-1: none; test hook)
};

constexpr unsigned kWaveSpinLimit = 1u << 21;  // default: about a second of polling with the back-off

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <int D, int MU, bool MET, bool MEAS>
__device__ __forceinline__ void wave_phase(const UpdArgs &a, int i, double *slot) {
  if (MEAS) {
    __shared__ double smem[kRedWarps * 2];
    float2 m = make_float2(0.f, 0.f);
    update_pair_body<D, MU, MET, SRC_PHILOX, true, true>(a, i, &m);
    double v[2] = {(double)m.x, (double)m.y};
    block_sum<2>(v, smem);
    if (threadIdx.x < 2) slot[2 * blockIdx.x + threadIdx.x] = v[0];
  } else {
    update_pair_body<D, MU, MET, SRC_PHILOX, false, true>(a, i);
  }
}

template <int D, bool MET>
__device__ __forceinline__ void wave_dispatch(const UpdArgs &a, int mu, bool meas, int i, double *slot) {
  switch (mu) {
    case 0: wave_phase<D, 0, MET, false>(a, i, slot); break;
    case 1:
      if (meas) wave_phase<D, 1, MET, true>(a, i, slot);
      else wave_phase<D, 1, MET, false>(a, i, slot);
      break;
    case 2:
      if constexpr (D > 2) {
        if (meas) wave_phase<D, 2, MET, true>(a, i, slot);
        else wave_phase<D, 2, MET, false>(a, i, slot);
      }
      break;
    default:
      if constexpr (D > 3) {
        if (meas) wave_phase<D, 3, MET, true>(a, i, slot);
        else wave_phase<D, 3, MET, false>(a, i, slot);
      }
      break;
  }
}

template <int D>
static __global__ void __launch_bounds__(256, 8) k_sweep_wave(const WaveArgs w) {
  const GeomK &g = w.a.g;
  const int tile = blockIdx.x;
  const int i = tile * (g.hN0 * g.N[1]) + 2 * threadIdx.x;  // EO index of this thread's first site
  // threads 0..7 each watch one of the eight (x2, x3) neighbour tiles
  int watch = -1;
  if (threadIdx.x < 8) {
    const int N2 = g.N[2], N3 = g.N[3];
    const int x2 = tile % N2, x3 = tile / N2;
    const int d = threadIdx.x < 4 ? threadIdx.x : threadIdx.x + 1;  // 3x3 stencil without its centre
    watch = (x2 + d % 3 - 1 + N2) % N2 + N2 * ((x3 + d / 3 - 1 + N3) % N3);
  }
  __shared__ int failed;
  __shared__ bool last;
  if (threadIdx.x == 0) failed = 0;
  __syncthreads();
  const int nph = 2 * D * (w.metrop + w.ovrn);
  UpdArgs a = w.a;
  for (int ph = 0; ph < nph; ++ph) {
    if (ph > 0) {
      if (watch >= 0) {
        unsigned n = 0;
        // acquire polls (measured faster here than relaxed polls plus one fence)
        while (ld_acquire_gpu(w.flags + watch) < (unsigned)ph) {
          if (n > 16) __nanosleep(32);  // back off after a short spin
          if (++n >= w.spin_limit) {
            atomicMax(w.err, (unsigned)ph + 1u);
            failed = 1;
            break;
          }
        }
      }
      __syncthreads();
      if (failed) break;  // uniform: read after the barrier
    }
    const int pass = ph / (2 * D), within = ph - pass * (2 * D);
    const int mu = within % D;
    a.p = within / D;
    a.mu = mu;
    const bool met = pass < w.metrop;
    a.hit = met ? pass : 0;
    const bool meas = w.meas != nullptr && pass == w.metrop + w.ovrn - 1 && a.p == 1 && mu >= 1;
    double *slot = meas ? w.meas + (size_t)(mu - 1) * gridDim.x * 2 : nullptr;
    if (met)
      wave_dispatch<D, true>(a, mu, meas, i, slot);
    else
      wave_dispatch<D, false>(a, mu, meas, i, slot);
    __syncthreads();
    if (threadIdx.x == 0 && tile != w.stall_tile) {
      __threadfence();
      st_release_gpu(w.flags + tile, (unsigned)ph + 1u);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(w.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {  // every other block has finished its phases
    for (unsigned t = threadIdx.x; t < gridDim.x; t += blockDim.x) w.flags[t] = 0u;
    if (threadIdx.x == 0) {
      *w.pass_rw += (unsigned long long)w.metrop;
      *w.ticket = 0u;
    }
    __threadfence();
  }
}

// Threads per block of the persistent sweep (two sites each), or 0 when the
// geometry does not fit it: 4D, N0/2 even, hN0 * N1 / 2 a multiple of 32 in
// [64, 256].
__host__ inline int wave_threads(const GeomK &g) {
  if (g.dims != 4 || (g.hN0 & 1)) return 0;
  const int t = g.hN0 * g.N[1] / 2;
  return (t % 32 == 0 && t >= 64 && t <= 256) ? t : 0;
}
__host__ inline int wave_tiles(const GeomK &g) { return g.N[2] * g.N[3]; }

}  // namespace u1b
