// Philox4x32-10 counter-based generator, written from the published
// algorithm (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11): ten rounds of
// two 32x32->64 multiplies with the Weyl-sequence key schedule.
//
// It replaces the reference's per-site cuRAND MRG32k3a states
// (reference include/random.h:31-58, src/random.cu:16-36).  A draw is a pure
// function of (key, counter), so a link's random numbers do not depend on
// which thread, tile or launch updates it.
//
// Counter layout used by this library (see u1_rng_counter below):
//   c.x = link-site index within its direction block (id + parity*V/2)
//   c.y = direction mu | stream tag << 8 | chain << 16
//   c.z, c.w = 64-bit pass counter (Metropolis pass / hot start number)
// key = 64-bit user seed.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define U1_HD __host__ __device__ __forceinline__
#else
#define U1_HD inline
#endif

namespace u1b {

struct Philox4 {
  uint32_t v[4];
};

U1_HD void u1_mulhilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
#if defined(__CUDA_ARCH__)
  lo = a * b;
  hi = __umulhi(a, b);
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  lo = (uint32_t)p;
  hi = (uint32_t)(p >> 32);
#endif
}

U1_HD Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                            uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    u1_mulhilo(M0, c0, hi0, lo0);
    u1_mulhilo(M1, c2, hi1, lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += W0;
    k1 += W1;
  }
  Philox4 out;
  out.v[0] = c0;
  out.v[1] = c1;
  out.v[2] = c2;
  out.v[3] = c3;
  return out;
}

// 24-bit uniform strictly inside (0, 1): (u >> 8 + 1/2) * 2^-24.
// Exactly representable in float and double, so host and device agree bit
// for bit.
U1_HD float u1_uniform_open(uint32_t u) {
  return ((float)(u >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

enum : uint32_t {
  U1_TAG_METROPOLIS = 0u,
  U1_TAG_HOTSTART = 1u,
  U1_TAG_FLOW = 2u,
  U1_TAG_HIT = 0x80u,  // multi-hit Metropolis: hit h >= 1 uses tag U1_TAG_HIT | h
};
enum : int { U1_MAX_HITS = 127 };

U1_HD uint32_t u1_rng_word1(int mu, uint32_t tag, uint32_t chain) {
  return (uint32_t)mu | (tag << 8) | (chain << 16);
}

// Metropolis draws of the link (EO site s = parity * V/2 + eo, direction mu)
// in pass `pass`: the proposal u1 (theta' = 2 pi u1) and the accept number b.
// Sites 2k and 2k+1 share one Philox4x32-10 block, counter
// (k, word1(mu, METROPOLIS, chain), pass lo, pass hi), key = seed: the even
// site takes words 0 and 1, the odd site words 2 and 3.
U1_HD Philox4 u1_metropolis_block(uint32_t s, int mu, uint32_t chain, unsigned long long pass, uint32_t key0,
                                  uint32_t key1) {
  return philox4x32_10(s >> 1, u1_rng_word1(mu, U1_TAG_METROPOLIS, chain), (uint32_t)pass, (uint32_t)(pass >> 32),
                       key0, key1);
}
// The block of hit h (0 <= h <= U1_MAX_HITS - 1) of a multi-hit Metropolis
// pass: hit 0 is u1_metropolis_block itself, hit h >= 1 replaces the tag by
// U1_TAG_HIT | h.  Sites 2k and 2k+1 share each block as above.
U1_HD Philox4 u1_metropolis_block_hit(uint32_t s, int mu, uint32_t chain, unsigned long long pass, int h,
                                      uint32_t key0, uint32_t key1) {
  const uint32_t tag = h ? (U1_TAG_HIT | (uint32_t)h) : U1_TAG_METROPOLIS;
  return philox4x32_10(s >> 1, u1_rng_word1(mu, tag, chain), (uint32_t)pass, (uint32_t)(pass >> 32), key0, key1);
}
U1_HD void u1_metropolis_draws(const Philox4 &r, uint32_t s, float &u1, float &b) {
  u1 = u1_uniform_open((s & 1u) ? r.v[2] : r.v[0]);
  b = u1_uniform_open((s & 1u) ? r.v[3] : r.v[1]);
}

}  // namespace u1b
