// Checkerboard link update kernels (one launch per (parity, mu) phase).
//
// Reference algorithm being replaced:
//   staple            include/staple.h:79-102 (anisotropic weights 1/xi, xi)
//   Metropolis        include/lattice_functions.h:68-80, src/update.cu:177-190
//   overrelaxation    include/lattice_functions.h:83-89, src/update.cu:227-231
//   multilevel freeze src/multilevel.cu:41 and :141
// Links are float2 (cos theta, sin theta); the staple is a sum of complex
// products, Metropolis compares exp(beta*Re(S*(U'-U))) with b (the
// reference's exp(beta*|S|*(cos(theta'+argS)-cos(theta+argS))) > b), and the
// overrelaxation reflection theta' = -theta - 2 arg S becomes
// U' = (conj S / |S|)^2 * conj U, with no transcendental call.
#pragma once
#include "u1_cplx.cuh"
#include "u1_geom.cuh"
#include "u1_philox.h"

namespace u1b {

__device__ __forceinline__ float2 ldg2(const float2 *p) { return __ldg(p); }

// Programmatic dependent launch (sm_90+): phase kernels are launched with
// programmatic stream serialization, so the next phase's CTAs are scheduled
// while this phase drains.  Every such kernel waits for the previous grid
// (completion and memory visibility) before touching links or counters, and
// signals its dependents once its stores are issued.  Without the launch
// attribute both instructions are no-ops.
__device__ __forceinline__ void pdl_wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release_dependents() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// Staple S of link (x, mu), x of parity p with EO index i_self, so that the
// local action of the link is beta * Re(S * U_mu(x)).
template <int D>
__device__ __forceinline__ float2 staple_at(const float2 *__restrict__ lat, const GeomK &g,
                                            const CoupK &c, const int x[4], int i_self, int p,
                                            int mu) {
  const int q = 1 - p;
  const size_t offP = (size_t)p * g.Vh, offQ = (size_t)q * g.Vh;
  const size_t Vmu = (size_t)mu * g.V;
  int xm[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) xm[k] = (k == mu) ? wrap_inc(x[k], g.N[k]) : x[k];
  const int i_xm = eo_index(g, xm);  // x + mu, parity q
  float2 ss = make_float2(0.f, 0.f), st = make_float2(0.f, 0.f);
#pragma unroll
  for (int nu = 0; nu < D; ++nu) {
    if (nu == mu) continue;
    const size_t Vnu = (size_t)nu * g.V;
    int xn[4], xd[4], xmd[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      xn[k] = (k == nu) ? wrap_inc(x[k], g.N[k]) : x[k];
      xd[k] = (k == nu) ? wrap_dec(x[k], g.N[k]) : x[k];
      xmd[k] = (k == nu) ? wrap_dec(xm[k], g.N[k]) : xm[k];
    }
    const int i_xn = eo_index(g, xn);    // x + nu       parity q
    const int i_xd = eo_index(g, xd);    // x - nu       parity q
    const int i_xmd = eo_index(g, xmd);  // x + mu - nu  parity p
    // upper: U_nu(x+mu) conj(U_mu(x+nu)) conj(U_nu(x))
    float2 a = ldg2(lat + Vnu + offQ + i_xm);
    float2 b = ldg2(lat + Vmu + offQ + i_xn);
    float2 cc = ldg2(lat + Vnu + offP + i_self);
    float2 up = cmulc(cmulc(a, b), cc);
    // lower: conj(U_nu(x+mu-nu)) conj(U_mu(x-nu)) U_nu(x-nu)
    float2 d = ldg2(lat + Vnu + offP + i_xmd);
    float2 e = ldg2(lat + Vmu + offQ + i_xd);
    float2 f = ldg2(lat + Vnu + offQ + i_xd);
    float2 lo = cmul(cconjmul(d, e), f);
    if (mu == g.tdir || nu == g.tdir)
      st = cadd(st, cadd(up, lo));
    else
      ss = cadd(ss, cadd(up, lo));
  }
  return cweigh(ss, c.w_ss, st, c.w_st);
}

// Overrelaxation of one link: U' = (conj S)^2/|S|^2 * conj U, renormalised.
// |S| == 0 gives U' = conj U (the reference's atan2(0,0) = 0 case).  The
// reciprocal of |S|^2 only scales U' before the renormalisation, so it is the
// approximate one (measured 1.8 % faster per sweep at 32^4 than the IEEE
// division).
__device__ __forceinline__ float2 overrelax_link(float2 S, float2 U) {
  float n2 = fmaf(S.x, S.x, S.y * S.y);
  if (n2 > 0.f) {
    float inv = __fdividef(1.0f, n2);
    float ax = fmaf(S.x, S.x, -(S.y * S.y)) * inv;
    float ay = -2.0f * S.x * S.y * inv;
    float2 Un = make_float2(fmaf(ax, U.x, ay * U.y), fmaf(ay, U.x, -ax * U.y));
    float r = rsqrtf(fmaf(Un.x, Un.x, Un.y * Un.y));
    return make_float2(Un.x * r, Un.y * r);
  }
  return make_float2(U.x, -U.y);
}

struct UpdArgs {
  float2 *lat;
  GeomK g;
  CoupK c;
  int p;
  int mu;
  uint32_t key0, key1;                 // Philox key (seed)
  uint32_t chain;                      // chain number in the counter
  const unsigned long long *pass_dev;  // Metropolis pass counter (device)
  int hit;                             // pass = *pass_dev + hit
  const double *replay;                // shared-stream pairs (test mode)
  unsigned long long replay_base;      // pass number of replay[0]
  unsigned long long *bump_ptr;        // OR kernels: *bump_ptr += bump_by (block 0)
  unsigned int bump_by;
  int ml;                              // multilevel freeze period (0 = none)
  float win;                           // SRC_WINDOW: proposal half-width / pi (0: whole circle)
  int nhits;                           // SRC_WINDOW: Metropolis hits per link and pass
  int sms;                             // k_update_quad: > 0 remaps the block order over this many SMs
  int rev;                             // != 0: blocks take their work in reverse launch order (see rev_block)
#ifdef U1_BOUNDS_CHECK
  struct ChkState *chk;                // checked build: violation counters (see Chk below)
  unsigned *shadow;                    // checked build: per-link marks of this phase (nullptr: no race marks)
  const float2 *chk_base;              // checked build: the link buffer the shadow mirrors
#endif
};

// ---------------------------------------------------------------------------
// Checked build (-DU1_BOUNDS_CHECK, libu1b200_check.so; test infrastructure,
// never the product path).  Every link access of the update bodies passes
// chk(): the index must lie inside the (direction, parity) half it addresses
// (0 <= idx and idx + W <= V/2 for W consecutive links) and a vector access
// must be aligned to its width.  A violation is counted in ChkState (the
// first one recorded) and the access is skipped (a load returns zeros), so
// the kernel never touches memory outside its half of the lattice.  With a
// shadow array (one word per link of the buffer) every access is also marked:
// bit 0 for a read of a link the thread does not own, +2 for a write.
// k_chk_phase_end runs after every phase: a link written and also read by
// another thread, or written twice, within one phase is a checkerboard race;
// it counts them and clears the marks.  In the normal build Chk is empty and
// every check folds to `true`.
struct ChkState {
  unsigned long long bad;        // bounds or alignment violations
  unsigned long long races;      // links written and read (or written twice) within one phase
  unsigned long long phases;     // phases checked by k_chk_phase_end
  unsigned long long marked;     // links accessed, summed over the checked phases
  long long first_bad_idx;       // index, half size and kind of the first violation
  long long first_bad_half;
  long long first_race_link;     // buffer offset of a raced link
  int first_bad_kind;
  int pad;
};

struct Chk {
#ifdef U1_BOUNDS_CHECK
  ChkState *st;
  unsigned *shadow;
  const float2 *base;
  int Vh;
#endif
};

enum : int { CHK_READ = 0, CHK_OWN = 1, CHK_WRITE = 2 };  // another thread's link / the thread's own / a store

__device__ __forceinline__ Chk make_chk(const UpdArgs &a) {
#ifdef U1_BOUNDS_CHECK
  return Chk{a.chk, a.shadow, a.chk_base, a.g.Vh};
#else
  (void)a;
  return Chk{};
#endif
}

// Callers outside the update bodies (the standalone measurement) are not checked.
__device__ __forceinline__ Chk no_chk() { return Chk{}; }

// Whether W consecutive links at slab[idx] may be accessed (always true in
// the normal build); marks them in the checked build.
template <int W, int KIND>
__device__ __forceinline__ bool chk(const Chk &c, const float2 *slab, int idx) {
#ifdef U1_BOUNDS_CHECK
  if (c.st == nullptr) return true;  // an unchecked caller (no_chk)
  const bool ok = idx >= 0 && idx + W <= c.Vh && ((uintptr_t)(slab + idx) & (uintptr_t)(W * 8 - 1)) == 0;
  if (!ok) {
    if (atomicAdd(&c.st->bad, 1ull) == 0ull) {
      c.st->first_bad_idx = idx;
      c.st->first_bad_half = c.Vh;
      c.st->first_bad_kind = KIND;
    }
    return false;
  }
  if (c.shadow != nullptr && KIND != CHK_OWN) {
    unsigned *m = c.shadow + ((slab + idx) - c.base);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      if (KIND == CHK_READ)
        atomicOr(m + k, 1u);
      else
        atomicAdd(m + k, 2u);
    }
  }
  return true;
#else
  (void)c;
  (void)slab;
  (void)idx;
  return true;
#endif
}

// One link through the read-only path, checked.
__device__ __forceinline__ float2 ld1(const float2 *slab, int idx, const Chk &ck) {
  if (!chk<1, CHK_READ>(ck, slab, idx)) return make_float2(0.f, 0.f);
  return __ldg(slab + idx);
}

// Work item of launch-order block b of G when the blocks of a single wave
// are handed to S SMs round-robin: the blocks that share SM s (b = s, s+S,
// s+2S, ...) get consecutive items, so neighbouring x2-planes of the
// lattice meet in the same SM's L1.  A bijection of [0, G) for any G, S.
// Measured on B200 at 32^4: 1.7 % faster for the four-site kernel, 2.5 %
// slower for the two-site kernel, which therefore keeps the launch order.
__device__ __forceinline__ int sm_local_block(int b, int G, int S) {
  if (S <= 0) return b;
  const int q = G / S, rem = G - q * S;
  const int s = b % S, r = b / S;
  return s * q + min(s, rem) + r;
}

// Work item of block b of G in a phase with a.rev set: the last one first.
// A lattice larger than L2 streams every link through it in each phase;
// consecutive phases read 7 of the same 8 (direction, parity) halves, so
// when they alternate direction each phase starts on the links the previous
// one left in L2 instead of on the ones it evicted first.  The links are
// the same in any block order.
__device__ __forceinline__ int rev_block(const UpdArgs &a, int b, int G) { return a.rev ? G - 1 - b : b; }

// Where a Metropolis kernel takes its proposals from.
enum : int {
  SRC_PHILOX = 0,  // theta' = 2 pi u on the whole circle, one hit (the reference's proposal)
  SRC_REPLAY = 1,  // recorded (theta', b) pairs (test mode)
  SRC_WINDOW = 2,  // multi-hit, theta' = theta + pi win (2u - 1) (whole circle when win = 0)
};

// Staple of link (x, MU) from precomputed EO steps (eo_steps): all six
// neighbour indices of each plaquette pair are i plus one or two steps.
// MEAS: also return, over nu < MU, mA = sum (upper + lower) and
// mD = sum (upper - lower) (the plaquette terms of the measurement taken from
// the last pass, see update_pair_body); the staple itself is unchanged.
template <int D, int MU, bool MEAS = false>
__device__ __forceinline__ float2 staple_steps(const float2 *__restrict__ lat, const GeomK &g, const CoupK &c,
                                               int i, int p, const int fwd[4], const int bwd[4], const Chk &ck,
                                               float2 *mA = nullptr, float2 *mD = nullptr) {
  const int q = 1 - p;
  const float2 *Lq_mu = lat + MU * g.V + q * g.Vh;
  const int i_xm = i + fwd[MU];
  float2 ss = make_float2(0.f, 0.f), st = make_float2(0.f, 0.f);
#pragma unroll
  for (int nu = 0; nu < D; ++nu) {
    if (nu == MU) continue;
    const float2 *Lp_nu = lat + nu * g.V + p * g.Vh;
    const float2 *Lq_nu = lat + nu * g.V + q * g.Vh;
    // upper: U_nu(x+mu) conj(U_mu(x+nu)) conj(U_nu(x))
    const float2 a = ld1(Lq_nu, i_xm, ck);
    const float2 b = ld1(Lq_mu, i + fwd[nu], ck);
    const float2 cc = ld1(Lp_nu, i, ck);
    // lower: conj(U_nu(x+mu-nu)) conj(U_mu(x-nu)) U_nu(x-nu)
    const float2 d = ld1(Lp_nu, i_xm + bwd[nu], ck);
    const float2 e = ld1(Lq_mu, i + bwd[nu], ck);
    const float2 f = ld1(Lq_nu, i + bwd[nu], ck);
    const float2 up = cmulc(cmulc(a, b), cc), lo = cmul(cconjmul(d, e), f);
    const float2 sum = cadd(up, lo);
    if (MU == D - 1 || nu == D - 1)
      st = cadd(st, sum);
    else
      ss = cadd(ss, sum);
    if (MEAS && nu < MU) {
      *mA = cadd(*mA, sum);
      *mD = cadd(*mD, csub(up, lo));
    }
  }
  return cweigh(ss, c.w_ss, st, c.w_st);
}

// One link update (Metropolis with Philox or replayed numbers, or
// overrelaxation) given its staple S and current value U.
// blk: the site's Philox block when the caller already drew it (two-site
// bodies draw once for both sites), else nullptr.
// Multi-hit Metropolis of one link (no reference counterpart: the reference
// makes one whole-circle proposal per pass).  The staple S is fixed while
// hit h = 0 .. nhits-1 draws (u, b) from block u1_metropolis_block_hit(h),
// proposes U' = U e^{i pi win (2u - 1)} (a window of half-width pi win
// around the current angle; U' = e^{2 pi i u} when win = 0) and accepts it
// when exp(beta Re(S (U' - U))) > b.  A windowed result is renormalised.
// With win = 0 and one hit this is the SRC_PHILOX update bit for bit.
template <int MU>
__device__ __forceinline__ float2 metropolis_hits(const UpdArgs &a, uint32_t s, unsigned long long pass, float2 S,
                                                  float2 U, const Philox4 *blk0) {
  float2 cur = U;
  for (int h = 0; h < a.nhits; ++h) {
    const Philox4 r = (h == 0 && blk0) ? *blk0 : u1_metropolis_block_hit(s, MU, a.chain, pass, h, a.key0, a.key1);
    float u1, b, sn, cs;
    u1_metropolis_draws(r, s, u1, b);
    float2 Un;
    if (a.win == 0.f) {
      sincospif(2.0f * u1, &sn, &cs);
      Un = make_float2(cs, sn);
    } else {
      sincospif(a.win * (2.0f * u1 - 1.0f), &sn, &cs);
      Un = cmul(cur, make_float2(cs, sn));
    }
    const float dS = a.c.beta * (cre_mul(S, Un) - cre_mul(S, cur));
    if (expf(dS) > b) cur = Un;
  }
  if (a.win != 0.f) {
    const float r = rsqrtf(fmaf(cur.x, cur.x, cur.y * cur.y));
    cur = make_float2(cur.x * r, cur.y * r);
  }
  return cur;
}

template <int D, int MU, bool MET, int SRC>
__device__ __forceinline__ float2 update_one(const UpdArgs &a, int i, float2 S, float2 U,
                                             const Philox4 *blk = nullptr) {
  if (MET) {
    const unsigned long long pass = *a.pass_dev + (unsigned long long)a.hit;
    if (SRC == SRC_WINDOW) return metropolis_hits<MU>(a, (uint32_t)(a.p * a.g.Vh + i), pass, S, U, blk);
    float2 Un;
    float b;
    if (SRC == SRC_REPLAY) {
      const size_t pr = ((((size_t)(pass - a.replay_base) * 2 + a.p) * D + MU) * a.g.Vh + i) * 2;
      double sn, cs;
      sincos(a.replay[pr], &sn, &cs);
      Un = make_float2((float)cs, (float)sn);
      b = (float)a.replay[pr + 1];
    } else {
      const uint32_t s = (uint32_t)(a.p * a.g.Vh + i);
      const Philox4 r = blk ? *blk : u1_metropolis_block(s, MU, a.chain, pass, a.key0, a.key1);
      float u1;
      u1_metropolis_draws(r, s, u1, b);
      float sn, cs;
      sincospif(2.0f * u1, &sn, &cs);
      Un = make_float2(cs, sn);
    }
    const float dS = a.c.beta * (cre_mul(S, Un) - cre_mul(S, U));
    return (expf(dS) > b) ? Un : U;
  }
  return overrelax_link(S, U);
}

// Body of the one-site-per-thread update of EO site i of phase (a.p, MU)
// (i >= V/2: only the kernel entry); shared by the single-lattice and
// batched kernels.
// Entry of every phase kernel: the site decode (pure arithmetic) runs
// before it, overlapping the previous grid's tail under programmatic
// dependent launch.  Waits for the previous grid; an overrelaxation kernel
// that carries the sweep's pass-counter bump then applies it (block 0).
// The bodies signal dependents after their store; threads that leave
// early (out of range, frozen links) count as done when they exit.
template <bool MET>
__device__ __forceinline__ void phase_entry(const UpdArgs &a) {
  pdl_wait_prior_grid();
  if (!MET && a.bump_ptr != nullptr && blockIdx.x == 0 && threadIdx.x == 0) *a.bump_ptr += a.bump_by;
}

// Measurement from the last pass (MEAS): after the final update of the
// links U_MU at parity-1 sites, every plaquette (nu, MU) with nu < MU holds
// exactly one such link (its two U_MU links sit at sites of opposite parity)
// and all its other links are final (directions < MU were updated earlier
// in the pass, U_MU at parity 0 in phase (0, MU)).  With the new link U' the
// staple terms give it directly: upper * U' = conj P_{nu MU}(x),
// lower * U' = P_{nu MU}(x - nu).  So the phase adds, per site,
//   sum (1 - Re P) = 2 MU - Re(mA U'),   -sum Im P = Im(mD U'),
// mA = sum_{nu<MU} (upper + lower), mD = sum_{nu<MU} (upper - lower).
// Phases (1, MU), MU = 1..D-1, of the last pass therefore count every
// plaquette of the final configuration once, from values already loaded.
template <int D, int MU, bool MET, int SRC, bool MEAS = false>
__device__ __forceinline__ void update_single_body(const UpdArgs a, int i, float2 *meas = nullptr) {
  int x[4], k;
  eo_decode_fast<D>(a.g, i, a.p, x, k);
  phase_entry<MET>(a);
  if (i >= a.g.Vh) return;
  // Multilevel freeze rule, reference src/multilevel.cu:41: update unless the
  // site lies on a frozen time slice (x_t multiple of ml, ml = 2 or 4) and
  // the link is spatial (the reference tests the literal direction index 3).
  if (!MEAS && MU != 3 && a.ml > 0 && (x[D - 1] & (a.ml - 1)) == 0) return;
  int fwd[4], bwd[4];
  eo_steps<D>(a.g, x, k, fwd, bwd);
  const Chk ck = make_chk(a);
  float2 *own_slab = a.lat + MU * a.g.V + a.p * a.g.Vh;
  float2 mA = make_float2(0.f, 0.f), mD = mA;
  const float2 S = staple_steps<D, MU, MEAS>(a.lat, a.g, a.c, i, a.p, fwd, bwd, ck, &mA, &mD);
  const float2 U = chk<1, CHK_OWN>(ck, own_slab, i) ? own_slab[i] : make_float2(0.f, 0.f);
  const float2 N = update_one<D, MU, MET, SRC>(a, i, S, U);
  if (chk<1, CHK_WRITE>(ck, own_slab, i)) own_slab[i] = N;
  pdl_release_dependents();
  if (MEAS) *meas = make_float2(2.f * MU - cre_mul(mA, N), cim_mul(mD, N));
}

// ---------------------------------------------------------------------------
// Two sites per thread.  When N0/2 is even, EO sites 2t and 2t+1 of a phase
// lie in the same x0-row: their coordinates x1..x3, their x0 parity and
// every step along x1..x3 are shared, and because those steps are even the
// two neighbour links sit side by side at a 16-byte aligned address: one
// 128-bit load serves both sites.  Steps along x0 are odd or differ at the
// row end, so x0-shifted neighbours are loaded per site.
struct Pair2 {
  float2 s0, s1;
};

// COH = false: read-only (non-coherent) loads, valid because a phase kernel
// never reads what it writes.  COH = true: ordinary coherent (L1-cached) loads,
// for the persistent sweep kernel that reads links other blocks wrote earlier
// in the same launch (ordered by its acquire fences).
template <bool COH = false>
__device__ __forceinline__ Pair2 ld_vec2(const float2 *base, int idx, const Chk &ck) {
  if (!chk<2, CHK_READ>(ck, base, idx)) return Pair2{make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  const float4 *p = reinterpret_cast<const float4 *>(base + idx);
  const float4 t = COH ? __ldca(p) : __ldg(p);
  return Pair2{make_float2(t.x, t.y), make_float2(t.z, t.w)};
}
template <bool COH = false>
__device__ __forceinline__ float2 ld_one(const float2 *base, int idx, const Chk &ck) {
  if (!chk<1, CHK_READ>(ck, base, idx)) return make_float2(0.f, 0.f);
  return COH ? __ldca(base + idx) : __ldg(base + idx);
}
template <bool COH = false>
__device__ __forceinline__ Pair2 ld_two(const float2 *base, int i0, int i1, const Chk &ck) {
  return Pair2{ld_one<COH>(base, i0, ck), ld_one<COH>(base, i1, ck)};
}

// upper + lower staple contributions of one nu for both sites
__device__ __forceinline__ void staple_term2(const Pair2 &a, const Pair2 &b, const Pair2 &c, const Pair2 &d,
                                             const Pair2 &e, const Pair2 &f, float2 &acc0, float2 &acc1) {
  acc0 = cadd(acc0, cadd(cmulc(cmulc(a.s0, b.s0), c.s0), cmul(cconjmul(d.s0, e.s0), f.s0)));
  acc1 = cadd(acc1, cadd(cmulc(cmulc(a.s1, b.s1), c.s1), cmul(cconjmul(d.s1, e.s1), f.s1)));
}

// Body of the two-sites-per-thread update for EO sites i, i+1 (i even) of
// the phase (a.p, MU) (i >= V/2: only the kernel entry); shared by the
// single-lattice and batched kernels.
// Every variant forms the staple and the update with the same operations in
// the same order, so all of them give bit-identical links.
template <int D, int MU, bool MET, int SRC, bool MEAS = false, bool COH = false>
__device__ __forceinline__ void update_pair_body(const UpdArgs a, int i, float2 *meas = nullptr) {
  int x[4], k;
  eo_decode_fast<D>(a.g, i, a.p, x, k);
  phase_entry<MET>(a);
  if (i >= a.g.Vh) return;
  if (!MEAS && MU != 3 && a.ml > 0 && (x[D - 1] & (a.ml - 1)) == 0) return;  // freeze rule, src/multilevel.cu:41
  int fwd[4], bwd[4];
  eo_steps<D>(a.g, x, k, fwd, bwd);  // steps of site i; site i+1 shares those along x1..x3
  // x0 steps of the two sites: x0 = 2k+odd and 2k+2+odd
  const int odd = x[0] & 1;
  const int f0a = fwd[0], b0a = bwd[0];
  const int f0b = odd ? ((k + 1 == a.g.hN0 - 1) ? a.g.wrapf[0] : 1) : 0;
  const int b0b = odd ? 0 : -1;
  const int q = 1 - a.p;
  const int V = a.g.V, Vh = a.g.Vh;
  const float2 *lat = a.lat;
  const float2 *Lq_mu = lat + MU * V + q * Vh;
  const Chk ck = make_chk(a);
  float2 ss0 = make_float2(0.f, 0.f), ss1 = ss0, st0 = ss0, st1 = ss0;
  float2 mA0 = ss0, mA1 = ss0, mD0 = ss0, mD1 = ss0;  // measurement sums (MEAS), see update_single_body
#pragma unroll
  for (int nu = 0; nu < D; ++nu) {
    if (nu == MU) continue;
    const float2 *Lp_nu = lat + nu * V + a.p * Vh;
    const float2 *Lq_nu = lat + nu * V + q * Vh;
    Pair2 A, B, C, Dd, E, F;
    C = ld_vec2<COH>(Lp_nu, i, ck);
    if (MU == 0) {  // nu != 0: steps along nu shared, along x0 per site
      A = ld_two<COH>(Lq_nu, i + f0a, i + 1 + f0b, ck);
      B = ld_vec2<COH>(Lq_mu, i + fwd[nu], ck);
      Dd = ld_two<COH>(Lp_nu, i + f0a + bwd[nu], i + 1 + f0b + bwd[nu], ck);
      E = ld_vec2<COH>(Lq_mu, i + bwd[nu], ck);
      F = ld_vec2<COH>(Lq_nu, i + bwd[nu], ck);
    } else if (nu == 0) {  // MU != 0
      A = ld_vec2<COH>(Lq_nu, i + fwd[MU], ck);
      B = ld_two<COH>(Lq_mu, i + f0a, i + 1 + f0b, ck);
      Dd = ld_two<COH>(Lp_nu, i + fwd[MU] + b0a, i + 1 + fwd[MU] + b0b, ck);
      E = ld_two<COH>(Lq_mu, i + b0a, i + 1 + b0b, ck);
      F = ld_two<COH>(Lq_nu, i + b0a, i + 1 + b0b, ck);
    } else {  // MU != 0, nu != 0: every step even, all loads 128-bit
      A = ld_vec2<COH>(Lq_nu, i + fwd[MU], ck);
      B = ld_vec2<COH>(Lq_mu, i + fwd[nu], ck);
      Dd = ld_vec2<COH>(Lp_nu, i + fwd[MU] + bwd[nu], ck);
      E = ld_vec2<COH>(Lq_mu, i + bwd[nu], ck);
      F = ld_vec2<COH>(Lq_nu, i + bwd[nu], ck);
    }
    if (MEAS && nu < MU) {
      // the same operations as staple_term2, with the upper and lower terms kept
      const float2 up0 = cmulc(cmulc(A.s0, B.s0), C.s0), lo0 = cmul(cconjmul(Dd.s0, E.s0), F.s0);
      const float2 up1 = cmulc(cmulc(A.s1, B.s1), C.s1), lo1 = cmul(cconjmul(Dd.s1, E.s1), F.s1);
      const float2 sum0 = cadd(up0, lo0), sum1 = cadd(up1, lo1);
      if (MU == D - 1) {
        st0 = cadd(st0, sum0);
        st1 = cadd(st1, sum1);
      } else {
        ss0 = cadd(ss0, sum0);
        ss1 = cadd(ss1, sum1);
        mA0 = cadd(mA0, sum0);
        mA1 = cadd(mA1, sum1);
      }
      mD0 = cadd(mD0, csub(up0, lo0));
      mD1 = cadd(mD1, csub(up1, lo1));
    } else if (MU == D - 1 || nu == D - 1) {
      staple_term2(A, B, C, Dd, E, F, st0, st1);
    } else {
      staple_term2(A, B, C, Dd, E, F, ss0, ss1);
    }
  }
  const float2 S0 = cweigh(ss0, a.c.w_ss, st0, a.c.w_st);
  const float2 S1 = cweigh(ss1, a.c.w_ss, st1, a.c.w_st);
  float2 *own_slab = a.lat + MU * V + a.p * Vh;
  float4 *own = reinterpret_cast<float4 *>(own_slab + i);
  const float4 U = chk<2, CHK_OWN>(ck, own_slab, i) ? *own : make_float4(0.f, 0.f, 0.f, 0.f);
  // sites i, i+1 (i even, V/2 even) share one Philox block
  Philox4 blk;
  if (MET && SRC != SRC_REPLAY)
    blk = u1_metropolis_block((uint32_t)(a.p * Vh + i), MU, a.chain, *a.pass_dev + (unsigned long long)a.hit,
                              a.key0, a.key1);
  const float2 N0 = update_one<D, MU, MET, SRC>(a, i, S0, make_float2(U.x, U.y), &blk);
  const float2 N1 = update_one<D, MU, MET, SRC>(a, i + 1, S1, make_float2(U.z, U.w), &blk);
  if (chk<2, CHK_WRITE>(ck, own_slab, i)) *own = make_float4(N0.x, N0.y, N1.x, N1.y);
  pdl_release_dependents();
  if (MEAS) {
    // for MU = D-1 every nu < MU term is in st: mA = st
    const float2 a0 = (MU == D - 1) ? st0 : mA0, a1 = (MU == D - 1) ? st1 : mA1;
    *meas = make_float2(4.f * MU - cre_mul(a0, N0) - cre_mul(a1, N1), cim_mul(mD0, N0) + cim_mul(mD1, N1));
  }
}

// ---------------------------------------------------------------------------
// Four sites per thread.  When N0/2 is a multiple of 4, EO sites 4t..4t+3 of
// a phase lie in one x0-row: they share x1..x3 and every step along them,
// and those steps are multiples of N0/2, so the four neighbour links along
// x1..x3 are consecutive and 32-byte aligned: one 256-bit load serves the
// four sites.  Steps along x0 differ per site (a shift of 0 or 1 within the
// row, wrapping at its end), so x0-shifted neighbours are loaded per site.
// The site decode and the steps are computed once for four sites.
struct Quad2 {
  float2 s[4];
};

// Four consecutive links from a 32-byte aligned address (idx % 4 == 0).
// Non-coherent (read-only path): a phase kernel never reads what it writes.
// volatile + "memory" keep the load after the grid-dependency wait.
__device__ __forceinline__ Quad2 ld_quad(const float2 *base, int idx, const Chk &ck) {
  Quad2 q;
  if (!chk<4, CHK_READ>(ck, base, idx)) {
#pragma unroll
    for (int s = 0; s < 4; ++s) q.s[s] = make_float2(0.f, 0.f);
    return q;
  }
  asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(q.s[0].x), "=f"(q.s[0].y), "=f"(q.s[1].x), "=f"(q.s[1].y), "=f"(q.s[2].x), "=f"(q.s[2].y),
                 "=f"(q.s[3].x), "=f"(q.s[3].y)
               : "l"(base + idx)
               : "memory");
  return q;
}
// The same through the coherent path (the thread's own links, stored later).
__device__ __forceinline__ Quad2 ld_quad_own(const float2 *slab, int idx, const Chk &ck) {
  Quad2 q;
  if (!chk<4, CHK_OWN>(ck, slab, idx)) {
#pragma unroll
    for (int s = 0; s < 4; ++s) q.s[s] = make_float2(0.f, 0.f);
    return q;
  }
  const float2 *p = slab + idx;
  asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(q.s[0].x), "=f"(q.s[0].y), "=f"(q.s[1].x), "=f"(q.s[1].y), "=f"(q.s[2].x), "=f"(q.s[2].y),
                 "=f"(q.s[3].x), "=f"(q.s[3].y)
               : "l"(p)
               : "memory");
  return q;
}
__device__ __forceinline__ void st_quad(float2 *slab, int idx, const float2 n[4], const Chk &ck) {
  if (!chk<4, CHK_WRITE>(ck, slab, idx)) return;
  float2 *p = slab + idx;
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(n[0].x), "f"(n[0].y), "f"(n[1].x),
               "f"(n[1].y), "f"(n[2].x), "f"(n[2].y), "f"(n[3].x), "f"(n[3].y)
               : "memory");
}
// Per-site links at base + i + s + sh[s], s = 0..3.
__device__ __forceinline__ Quad2 ld_shifted(const float2 *base, int i, const int sh[4], const Chk &ck) {
  Quad2 q;
#pragma unroll
  for (int s = 0; s < 4; ++s) q.s[s] = ld1(base, i + s + sh[s], ck);
  return q;
}

// Body of the four-sites-per-thread update for EO sites i..i+3 (i a multiple
// of 4) of the phase (a.p, MU); every site's staple and update use the same
// operations in the same order as the other bodies (bit-identical links).
// MEAS: also add the plaquettes (nu < MU, MU) of the four sites from their
// staple terms into *meas (as update_pair_body).
template <int D, int MU, bool MET, int SRC, bool MEAS = false>
__device__ __forceinline__ void update_quad_body(const UpdArgs a, int i, float2 *meas = nullptr) {
  // site decode and neighbour steps (pure arithmetic) before the wait for
  // the previous phase, overlapping its tail
  int x[4], k;
  eo_decode_fast<D>(a.g, i, a.p, x, k);
  int fwd[4], bwd[4];
  eo_steps<D>(a.g, x, k, fwd, bwd);  // steps of site i; sites i+1..i+3 share those along x1..x3
  const int odd = x[0] & 1;
  int f0[4], b0[4];  // x0 steps of the four sites (k multiple of 4: only site 3 can end the row, site 0 start it)
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    f0[s] = odd ? ((s == 3 && k + 3 == a.g.hN0 - 1) ? a.g.wrapf[0] : 1) : 0;
    b0[s] = odd ? 0 : ((s == 0 && k == 0) ? a.g.wrapb[0] : -1);
  }
  phase_entry<MET>(a);
  if (i >= a.g.Vh) return;
  if (!MEAS && MU != 3 && a.ml > 0 && (x[D - 1] & (a.ml - 1)) == 0) return;  // freeze rule, src/multilevel.cu:41
  const int q = 1 - a.p;
  const int V = a.g.V, Vh = a.g.Vh;
  const float2 *lat = a.lat;
  const float2 *Lq_mu = lat + MU * V + q * Vh;
  const Chk ck = make_chk(a);
  float2 ss[4], st[4], mA[4], mD[4];  // mA, mD: measurement sums (MEAS), see update_single_body
#pragma unroll
  for (int s = 0; s < 4; ++s) ss[s] = st[s] = mA[s] = mD[s] = make_float2(0.f, 0.f);
#pragma unroll
  for (int nu = 0; nu < D; ++nu) {
    if (nu == MU) continue;
    const float2 *Lp_nu = lat + nu * V + a.p * Vh;
    const float2 *Lq_nu = lat + nu * V + q * Vh;
    Quad2 A, B, C, Dd, E, F;
    C = ld_quad(Lp_nu, i, ck);
    if (MU == 0) {  // nu != 0: steps along nu shared, along x0 per site
      A = ld_shifted(Lq_nu, i, f0, ck);
      B = ld_quad(Lq_mu, i + fwd[nu], ck);
      Dd = ld_shifted(Lp_nu, i + bwd[nu], f0, ck);
      E = ld_quad(Lq_mu, i + bwd[nu], ck);
      F = ld_quad(Lq_nu, i + bwd[nu], ck);
    } else if (nu == 0) {  // MU != 0
      A = ld_quad(Lq_nu, i + fwd[MU], ck);
      B = ld_shifted(Lq_mu, i, f0, ck);
      Dd = ld_shifted(Lp_nu, i + fwd[MU], b0, ck);
      E = ld_shifted(Lq_mu, i, b0, ck);
      F = ld_shifted(Lq_nu, i, b0, ck);
    } else {  // MU != 0, nu != 0: every load 256-bit
      A = ld_quad(Lq_nu, i + fwd[MU], ck);
      B = ld_quad(Lq_mu, i + fwd[nu], ck);
      Dd = ld_quad(Lp_nu, i + fwd[MU] + bwd[nu], ck);
      E = ld_quad(Lq_mu, i + bwd[nu], ck);
      F = ld_quad(Lq_nu, i + bwd[nu], ck);
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const float2 up = cmulc(cmulc(A.s[s], B.s[s]), C.s[s]), lo = cmul(cconjmul(Dd.s[s], E.s[s]), F.s[s]);
      const float2 t = cadd(up, lo);
      if (MU == D - 1 || nu == D - 1)
        st[s] = cadd(st[s], t);
      else
        ss[s] = cadd(ss[s], t);
      if (MEAS && nu < MU) {
        if (MU != D - 1) mA[s] = cadd(mA[s], t);  // for MU = D-1 every nu < MU term is in st
        mD[s] = cadd(mD[s], csub(up, lo));
      }
    }
  }
  float2 *own_slab = a.lat + MU * V + a.p * Vh;
  const Quad2 U = ld_quad_own(own_slab, i, ck);
  // sites i, i+1 and i+2, i+3 share one Philox block each
  Philox4 blk0, blk1;
  if (MET && SRC != SRC_REPLAY) {
    const unsigned long long pass = *a.pass_dev + (unsigned long long)a.hit;
    blk0 = u1_metropolis_block((uint32_t)(a.p * Vh + i), MU, a.chain, pass, a.key0, a.key1);
    blk1 = u1_metropolis_block((uint32_t)(a.p * Vh + i + 2), MU, a.chain, pass, a.key0, a.key1);
  }
  float2 N[4];
#pragma unroll
  for (int s = 0; s < 4; ++s)
    N[s] = update_one<D, MU, MET, SRC>(a, i + s, cweigh(ss[s], a.c.w_ss, st[s], a.c.w_st), U.s[s],
                                       s < 2 ? &blk0 : &blk1);
  st_quad(own_slab, i, N, ck);
  pdl_release_dependents();
  if (MEAS) {
    float re = 8.f * MU, im = 0.f;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      re -= cre_mul((MU == D - 1) ? st[s] : mA[s], N[s]);
      im += cim_mul(mD[s], N[s]);
    }
    *meas = make_float2(re, im);
  }
}

// Four sites per thread, at most 128 threads per block and a register budget
// of 72, so 7 CTAs fit an SM (a 32^4 phase, 1024 CTAs, is then a single wave).
template <int D, int MU, bool MET, int SRC>
__global__ void __launch_bounds__(128, 7) k_update_quad(const UpdArgs a) {
  const int b = a.rev ? rev_block(a, (int)blockIdx.x, (int)gridDim.x)
                      : sm_local_block((int)blockIdx.x, (int)gridDim.x, a.sms);
  update_quad_body<D, MU, MET, SRC>(a, 4 * (b * (int)blockDim.x + (int)threadIdx.x));
}

// Two sites per thread, register budget capped at 32 so 8 CTAs of 256
// threads fit an SM (a 32^4 phase is then a single wave).
template <int D, int MU, bool MET, int SRC>
__global__ void __launch_bounds__(256, 8) k_update_pair(const UpdArgs a) {
  const int b = rev_block(a, (int)blockIdx.x, (int)gridDim.x);
  update_pair_body<D, MU, MET, SRC>(a, 2 * (b * (int)blockDim.x + (int)threadIdx.x));
}

// The same with no register cap (fewer CTAs per SM, no spills).
template <int D, int MU, bool MET, int SRC>
__global__ void __launch_bounds__(256) k_update_pair_free(const UpdArgs a) {
  const int b = rev_block(a, (int)blockIdx.x, (int)gridDim.x);
  update_pair_body<D, MU, MET, SRC>(a, 2 * (b * (int)blockDim.x + (int)threadIdx.x));
}

// One site per thread (any geometry, N0/2 odd included).
template <int D, int MU, bool MET, int SRC>
__global__ void __launch_bounds__(256) k_update(const UpdArgs a) {
  const int b = rev_block(a, (int)blockIdx.x, (int)gridDim.x);
  update_single_body<D, MU, MET, SRC>(a, b * (int)blockDim.x + (int)threadIdx.x);
}

// Hot start (reference src/update.cu:30-48): every link gets
// theta = 2 pi u, u from Philox with the hot-start tag.
template <int D>
__global__ void __launch_bounds__(256) k_hot_start(float2 *lat, GeomK g, uint32_t key0,
                                                   uint32_t key1, uint32_t chain,
                                                   unsigned long long pass) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int mu = 0; mu < D; ++mu) {
      Philox4 r = philox4x32_10((uint32_t)(p * g.Vh + i), u1_rng_word1(mu, U1_TAG_HOTSTART, chain),
                                (uint32_t)pass, (uint32_t)(pass >> 32), key0, key1);
      float sn, cs;
      sincospif(2.0f * u1_uniform_open(r.v[0]), &sn, &cs);
      lat[(size_t)mu * g.V + (size_t)p * g.Vh + i] = make_float2(cs, sn);
    }
}

static __global__ void k_import_angles(float2 *lat, const double *ang, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s, c;
  sincos(ang[i], &s, &c);
  lat[i] = make_float2((float)c, (float)s);
}

static __global__ void k_export_angles(const float2 *lat, double *ang, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float2 u = lat[i];
  double t = atan2((double)u.y, (double)u.x);
  if (t < 0.0) t += 2.0 * 3.14159265358979323846;
  ang[i] = t;
}

static __global__ void k_fill_links(float2 *lat, size_t n, float2 v) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) lat[i] = v;
}

static __global__ void k_pass_add(unsigned long long *pass, unsigned long long n) { *pass += n; }

static __global__ void k_rng_debug(float *out, int Vh, int p, int mu, uint32_t key0, uint32_t key1,
                            uint32_t chain, unsigned long long pass) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  const uint32_t s = (uint32_t)(p * Vh + i);
  const Philox4 r = u1_metropolis_block(s, mu, chain, pass, key0, key1);
  u1_metropolis_draws(r, s, out[2 * i], out[2 * i + 1]);
}

}  // namespace u1b
