// u1_oracle.cpp -- FP64 CPU restatement of the reference's U(1) hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the sm_100a
// kernels: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
// / reference legs load it.  The product (latticeu1_b200, libu1b200.so) never
// calls it.
//
// Parity pinning: the functions below are checked against the reference's
// own FP64 CPU functions compiled from the reference sources into
// oracle/_ref/libu1ref.so (metropolis/overrelaxation src/update.cu:51-98,
// plaquette src/plaquette.cu:32-57, polyakov src/polyakov.cu:33-49, the
// host-compiled MultiHit include/lattice_functions.h:92-105) on identical
// inputs, and against the exact 2D plaquette (Bessel-function ratio).
// The reference ships no golden vectors; the fixtures in tests/golden/ were
// produced by oracle/_ref (see tests/golden/make_golden.py).
//
// Layout: angles theta[id + parity*V/2 + mu*V] in [0, 2pi) (reference
// u1.cpp:99, src/update.cu:188).  Geometry as reference
// src/parameters.cu:146-208.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../latticeu1_b200/csrc/u1_geom.cuh"
#include "../latticeu1_b200/csrc/u1_philox.h"

typedef std::complex<double> cd;

extern "C" {

struct OGeom {
  int dims, tdir;
  int N[4];
  int off[4];  // lexicographic offsets (reference PARAMS::Offset)
  long V, Vh, Vs;
  double beta, aniso;
};

// reference src/parameters.cu:146-208 (even-extent check returns -1 here)
int o_setup(OGeom *g, int dims, int Nx, int Ny, int Nz, int Nt, double beta, double aniso) {
  if (dims < 2 || dims > 4) return -1;
  g->dims = dims;
  g->tdir = dims - 1;
  for (int i = 0; i < 4; ++i) {
    g->N[i] = 1;
    g->off[i] = 0;
  }
  g->N[0] = Nx;
  if (dims == 2) g->N[1] = Nt;
  else g->N[1] = Ny;
  if (dims == 3) g->N[2] = Nt;
  else if (dims > 3) g->N[2] = Nz;
  if (dims == 4) g->N[3] = Nt;
  for (int i = 0; i < dims; ++i)
    if (g->N[i] % 2 != 0 || g->N[i] < 2) return -1;
  g->off[0] = 1;
  for (int i = 1; i < dims; ++i) g->off[i] = g->N[i - 1] * g->off[i - 1];
  g->V = 1;
  for (int i = 0; i < 4; ++i) g->V *= g->N[i];
  g->Vh = g->V / 2;
  g->Vs = 1;
  for (int i = 0; i < g->tdir; ++i) g->Vs *= g->N[i];
  g->beta = beta;
  g->aniso = aniso;
  return 0;
}

// reference include/index.h:114-122
void o_index_eo(const OGeom *g, int id, int parity, int x[4]) {
  int za = id / (g->N[0] / 2);
  int zb = za / g->N[1];
  x[1] = za - zb * g->N[1];
  x[3] = zb / g->N[2];
  x[2] = zb - x[3] * g->N[2];
  int xodd = (x[1] + x[2] + x[3] + parity) & 1;
  x[0] = (2 * id + xodd) - za * g->N[0];
}

static inline int lex(const OGeom *g, const int x[4]) {
  int id = x[0];
  for (int i = 1; i < g->dims; ++i) id += x[i] * g->off[i];
  return id;
}
static inline int parity_of(const OGeom *g, const int x[4]) {
  int s = 0;
  for (int i = 0; i < g->dims; ++i) s += x[i];
  return s & 1;
}

// reference include/index.h:134-153: EO index (incl. parity*V/2) of x + lmu e_mu + lnu e_nu
long o_index_eo_neg(const OGeom *g, int id, int parity, int mu, int lmu, int nu, int lnu) {
  int x[4];
  o_index_eo(g, id, parity, x);
  x[mu] = (x[mu] + lmu + g->N[mu]) % g->N[mu];
  if (nu >= 0) x[nu] = (x[nu] + lnu + g->N[nu]) % g->N[nu];
  return (long)(lex(g, x) >> 1) + (long)parity_of(g, x) * g->Vh;
}

static inline double L(const OGeom *g, const double *lat, long eo, int mu) { return lat[eo + mu * g->V]; }

// reference include/staple.h:79-102 (anisotropic complex staple)
void o_staple(const OGeom *g, const double *lat, int id, int parity, int mu, double out[2]) {
  cd ss = 0.0, st = 0.0;
  const long idmu1 = o_index_eo_neg(g, id, parity, mu, 1, -1, 0);
  const long self = id + parity * g->Vh;
  for (int nu = 0; nu < g->dims; ++nu) {
    if (nu == mu) continue;
    double up = L(g, lat, idmu1, nu);
    up -= L(g, lat, o_index_eo_neg(g, id, parity, nu, 1, -1, 0), mu);
    up -= L(g, lat, self, nu);
    double lo = -L(g, lat, o_index_eo_neg(g, id, parity, mu, 1, nu, -1), nu);
    const long xmn = o_index_eo_neg(g, id, parity, nu, -1, -1, 0);
    lo -= L(g, lat, xmn, mu);
    lo += L(g, lat, xmn, nu);
    cd s = std::polar(1.0, up) + std::polar(1.0, lo);
    if (mu == g->tdir || nu == g->tdir) st += s;
    else ss += s;
  }
  cd S = ss / g->aniso + st * g->aniso;
  out[0] = S.real();
  out[1] = S.imag();
}

// Staple of every link in the reference layout: out[2*l], out[2*l+1] for
// l = id + parity*V/2 + mu*V.  Used for conditioning-aware FP32 tolerances.
void o_staple_all(const OGeom *g, const double *lat, double *out) {
  for (int mu = 0; mu < g->dims; ++mu)
    for (int p = 0; p < 2; ++p) {
#pragma omp parallel for schedule(static)
      for (int id = 0; id < (int)g->Vh; ++id) {
        const long l = id + p * g->Vh + mu * g->V;
        o_staple(g, lat, id, p, mu, out + 2 * l);
      }
    }
}

// One Metropolis pass with externally supplied (new_theta, b) pairs in the
// reference CPU draw order parity -> mu -> id (reference src/update.cu:51-79).
// Returns the number of accepted proposals.
long o_metropolis_pairs(const OGeom *g, double *lat, const double *pairs) {
  long acc = 0;
  long k = 0;
  for (int p = 0; p < 2; ++p)
    for (int mu = 0; mu < g->dims; ++mu)
      for (int id = 0; id < g->Vh; ++id, ++k) {
        const long pos = id + p * g->Vh + mu * g->V;
        double S[2];
        o_staple(g, lat, id, p, mu, S);
        const double r = std::sqrt(S[0] * S[0] + S[1] * S[1]);
        const double t2 = std::atan2(S[1], S[0]);
        const double th_new = pairs[2 * k], b = pairs[2 * k + 1];
        const double dS = std::exp(g->beta * r * (std::cos(th_new + t2) - std::cos(lat[pos] + t2)));
        if (dS > b) {
          lat[pos] = th_new;
          ++acc;
        }
      }
  return acc;
}

// Philox draws of link (parity, mu, id) in Metropolis pass `pass`
// (the counter layout of latticeu1_b200/csrc/u1_philox.h: EO sites 2k and
// 2k+1 share one block, words 0,1 and 2,3).
void o_philox_uniforms(const OGeom *g, uint64_t seed, uint32_t chain, uint64_t pass, int p, int mu, int id,
                       float out[2]) {
  const uint32_t s = (uint32_t)(p * g->Vh + id);
  const u1b::Philox4 r = u1b::u1_metropolis_block(s, mu, chain, pass, (uint32_t)seed, (uint32_t)(seed >> 32));
  u1b::u1_metropolis_draws(r, s, out[0], out[1]);
}

void o_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t out[4]) {
  u1b::Philox4 r = u1b::philox4x32_10(c0, c1, c2, c3, k0, k1);
  for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}

// Freeze rule of the multilevel updates (reference src/multilevel.cu:41,141).
static inline bool frozen(const OGeom *g, int id, int p, int mu, int ml) {
  if (ml <= 0 || mu == 3) return false;
  int x[4];
  o_index_eo(g, id, p, x);
  return (x[g->tdir] % ml) == 0;
}

// One Metropolis pass with Philox uniforms (theta' = 2 pi u1, b = u2),
// optional multilevel freeze period ml.  OpenMP-parallel within a phase.
long o_metropolis_philox(const OGeom *g, double *lat, uint64_t seed, uint32_t chain, uint64_t pass, int ml) {
  long acc = 0;
  for (int p = 0; p < 2; ++p)
    for (int mu = 0; mu < g->dims; ++mu) {
#pragma omp parallel for reduction(+ : acc) schedule(static)
      for (int id = 0; id < (int)g->Vh; ++id) {
        if (frozen(g, id, p, mu, ml)) continue;
        const long pos = id + p * g->Vh + mu * g->V;
        double S[2];
        o_staple(g, lat, id, p, mu, S);
        float u[2];
        o_philox_uniforms(g, seed, chain, pass, p, mu, id, u);
        const double th_new = 2.0 * M_PI * (double)u[0];
        // exp(beta Re(S (U' - U))) > b, the same test as reference
        // include/lattice_functions.h:68-80 written with Re(S e^{i theta}).
        const double dS = g->beta * (S[0] * (std::cos(th_new) - std::cos(lat[pos])) -
                                     S[1] * (std::sin(th_new) - std::sin(lat[pos])));
        if (std::exp(dS) > (double)u[1]) {
          lat[pos] = th_new;
          ++acc;
        }
      }
    }
  return acc;
}

// Exactly one (parity p, direction mu) phase of a Metropolis (met != 0) or
// overrelaxation pass.  Metropolis numbers come from `pairs` (V/2 pairs for
// this phase, reference draw order) when non-null, else from Philox
// (seed, chain, pass).  For each site id of the phase it records the staple
// magnitude used (smag[id]) and, for Metropolis, the relative decision
// margin 1 - b/exp(dS) (margin[id]; 0 for overrelaxation), so a test can
// tell an FP32 accept flip at the decision boundary from a wrong result.
void o_phase(const OGeom *g, double *lat, int met, int p, int mu, const double *pairs, uint64_t seed,
             uint32_t chain, uint64_t pass, int ml, double *smag, double *margin) {
#pragma omp parallel for schedule(static)
  for (int id = 0; id < (int)g->Vh; ++id) {
    smag[id] = 0.0;
    margin[id] = 0.0;
    if (frozen(g, id, p, mu, ml)) continue;
    const long pos = id + p * g->Vh + mu * g->V;
    double S[2];
    o_staple(g, lat, id, p, mu, S);
    smag[id] = std::sqrt(S[0] * S[0] + S[1] * S[1]);
    if (met) {
      double th_new, b;
      if (pairs) {
        th_new = pairs[2 * id];
        b = pairs[2 * id + 1];
      } else {
        float u[2];
        o_philox_uniforms(g, seed, chain, pass, p, mu, id, u);
        th_new = 2.0 * M_PI * (double)u[0];
        b = (double)u[1];
      }
      const double dS = g->beta * (S[0] * (std::cos(th_new) - std::cos(lat[pos])) -
                                   S[1] * (std::sin(th_new) - std::sin(lat[pos])));
      const double e = std::exp(dS);
      margin[id] = 1.0 - b / e;
      if (e > b) lat[pos] = th_new;
    } else {
      const double t2 = std::atan2(S[1], S[0]);
      lat[pos] = std::fmod(6. * M_PI - lat[pos] - 2. * t2, 2. * M_PI);
    }
  }
}

// Multi-hit Metropolis with a proposal window, the library's
// u1_lattice_set_metropolis(delta, nhits) (no reference counterpart: the
// reference makes one whole-circle proposal, src/update.cu:181-182).  The
// staple S of the link is fixed; hit h draws (u, b) from the Philox block of
// tag 0 (h = 0) or 0x80 | h (u1_metropolis_block_hit), proposes
// theta' = theta + delta (2u - 1) (theta' = 2 pi u when delta = 0) and
// accepts when exp(beta Re(S (e^{i theta'} - e^{i theta}))) > b, the test of
// include/lattice_functions.h:68-80.  *margin gets the relative decision
// margin 1 - b/exp(dS) of the hit closest to its decision boundary.
static double hits_link(const OGeom *g, double theta, const double S[2], uint64_t seed, uint32_t chain,
                        uint64_t pass, int p, int mu, int id, double delta, int nhits, double *margin) {
  const uint32_t s = (uint32_t)(p * g->Vh + id);
  double best = HUGE_VAL;
  for (int h = 0; h < nhits; ++h) {
    const u1b::Philox4 r =
        u1b::u1_metropolis_block_hit(s, mu, chain, pass, h, (uint32_t)seed, (uint32_t)(seed >> 32));
    float u[2];
    u1b::u1_metropolis_draws(r, s, u[0], u[1]);
    const double th_new = delta == 0.0 ? 2.0 * M_PI * (double)u[0]
                                       : std::fmod(theta + delta * (2.0 * (double)u[0] - 1.0) + 2.0 * M_PI,
                                                   2.0 * M_PI);
    const double dS = g->beta * (S[0] * (std::cos(th_new) - std::cos(theta)) -
                                 S[1] * (std::sin(th_new) - std::sin(theta)));
    const double e = std::exp(dS);
    const double m = 1.0 - (double)u[1] / e;
    if (std::fabs(m) < std::fabs(best)) best = m;
    if (e > (double)u[1]) theta = th_new;
  }
  if (margin) *margin = best;
  return theta;
}

// One multi-hit windowed Metropolis pass (see hits_link), optional multilevel
// freeze period ml.  Returns the number of links whose angle changed.
long o_metropolis_hits(const OGeom *g, double *lat, uint64_t seed, uint32_t chain, uint64_t pass, double delta,
                       int nhits, int ml) {
  long moved = 0;
  for (int p = 0; p < 2; ++p)
    for (int mu = 0; mu < g->dims; ++mu) {
#pragma omp parallel for reduction(+ : moved) schedule(static)
      for (int id = 0; id < (int)g->Vh; ++id) {
        if (frozen(g, id, p, mu, ml)) continue;
        const long pos = id + p * g->Vh + mu * g->V;
        double S[2];
        o_staple(g, lat, id, p, mu, S);
        const double th = hits_link(g, lat[pos], S, seed, chain, pass, p, mu, id, delta, nhits, nullptr);
        moved += th != lat[pos];
        lat[pos] = th;
      }
    }
  return moved;
}

// One (parity, mu) phase of a multi-hit windowed Metropolis pass, recording
// |S| and the decision margin of the closest hit per site (as o_phase).
void o_phase_hits(const OGeom *g, double *lat, int p, int mu, uint64_t seed, uint32_t chain, uint64_t pass,
                  double delta, int nhits, double *smag, double *margin) {
#pragma omp parallel for schedule(static)
  for (int id = 0; id < (int)g->Vh; ++id) {
    const long pos = id + p * g->Vh + mu * g->V;
    double S[2];
    o_staple(g, lat, id, p, mu, S);
    smag[id] = std::sqrt(S[0] * S[0] + S[1] * S[1]);
    lat[pos] = hits_link(g, lat[pos], S, seed, chain, pass, p, mu, id, delta, nhits, &margin[id]);
  }
}

// One overrelaxation pass (reference src/update.cu:84-98,
// include/lattice_functions.h:83-89), optional freeze period ml.
void o_overrelax(const OGeom *g, double *lat, int ml) {
  for (int p = 0; p < 2; ++p)
    for (int mu = 0; mu < g->dims; ++mu) {
#pragma omp parallel for schedule(static)
      for (int id = 0; id < (int)g->Vh; ++id) {
        if (frozen(g, id, p, mu, ml)) continue;
        double S[2];
        o_staple(g, lat, id, p, mu, S);
        const long pos = id + p * g->Vh + mu * g->V;
        const double t2 = std::atan2(S[1], S[0]);
        lat[pos] = std::fmod(6. * M_PI - lat[pos] - 2. * t2, 2. * M_PI);
      }
    }
}

// Hot start with the Philox hot-start stream (theta = 2 pi u).
void o_hot_start_philox(const OGeom *g, double *lat, uint64_t seed, uint32_t chain, uint64_t pass) {
  for (int p = 0; p < 2; ++p)
    for (int mu = 0; mu < g->dims; ++mu)
      for (int id = 0; id < (int)g->Vh; ++id) {
        u1b::Philox4 r = u1b::philox4x32_10((uint32_t)(p * g->Vh + id),
                                            u1b::u1_rng_word1(mu, u1b::U1_TAG_HOTSTART, chain), (uint32_t)pass,
                                            (uint32_t)(pass >> 32), (uint32_t)seed, (uint32_t)(seed >> 32));
        lat[id + p * g->Vh + mu * g->V] = 2.0 * M_PI * (double)u1b::u1_uniform_open(r.v[0]);
      }
}

// reference src/plaquette.cu:93-118 + norms :156-165:
// out = {SS re, SS im, ST re, ST im} of mean(1 - e^{i theta_P}).
void o_plaquette(const OGeom *g, const double *lat, double out[4]) {
  double a[4] = {0, 0, 0, 0};
  int nSS = 0, nST = 0;
  for (int mu = 0; mu < g->dims - 1; ++mu)
    for (int nu = mu + 1; nu < g->dims; ++nu) (mu == g->tdir || nu == g->tdir) ? ++nST : ++nSS;
  for (int p = 0; p < 2; ++p)
    for (int id = 0; id < (int)g->Vh; ++id)
      for (int mu = 0; mu < g->dims - 1; ++mu) {
        const double tmp = lat[id + p * g->Vh + mu * g->V];
        const long idmu1 = o_index_eo_neg(g, id, p, mu, 1, -1, 0);
        for (int nu = mu + 1; nu < g->dims; ++nu) {
          double pl = tmp + L(g, lat, idmu1, nu) - L(g, lat, o_index_eo_neg(g, id, p, nu, 1, -1, 0), mu) -
                      lat[id + p * g->Vh + nu * g->V];
          const int k = (mu == g->tdir || nu == g->tdir) ? 2 : 0;
          a[k] += 1.0 - std::cos(pl);
          a[k + 1] -= std::sin(pl);
        }
      }
  const double nss = 1.0 / ((double)g->V * nSS), nst = 1.0 / ((double)g->V * nST);
  out[0] = a[0] * nss;
  out[1] = a[1] * nss;
  out[2] = a[2] * nst;
  out[3] = a[3] * nst;
}

// reference src/polyakov.cu:33-49
void o_polyakov(const OGeom *g, const double *lat, double out[2]) {
  double re = 0, im = 0;
  for (int p = 0; p < 2; ++p)
    for (int id = 0; id < (int)(g->Vs / 2); ++id) {
      int x[4];
      o_index_eo(g, id, p, x);
      double t = 0;
      for (x[g->tdir] = 0; x[g->tdir] < g->N[g->tdir]; ++x[g->tdir])
        t += lat[(lex(g, x) >> 1) + parity_of(g, x) * g->Vh + g->tdir * g->V];
      re += std::cos(t);
      im += std::sin(t);
    }
  out[0] = re / (double)g->Vs;
  out[1] = im / (double)g->Vs;
}

// The fast division used by the sm_100a kernels' site decode (host build of
// the same header), checked against '/' by tests/test_oracle_pin.py.
uint32_t o_fastdiv(uint32_t n, uint32_t d) { return u1b::fast_div(n, u1b::make_fastdiv(d)); }

double o_bessel_ratio(double x) { return std::cyl_bessel_i(1.0, x) / std::cyl_bessel_i(0.0, x); }

// reference include/lattice_functions.h:92-105
void o_multihit(const OGeom *g, const double *lat, int id, int parity, double out[2]) {
  double S[2];
  o_staple(g, lat, id, parity, g->tdir, S);
  const double alpha = std::sqrt(S[0] * S[0] + S[1] * S[1]);
  const double ba = g->beta * alpha;
  const double t = std::cyl_bessel_i(1.0, ba) / (std::cyl_bessel_i(0.0, ba) * alpha);
  out[0] = t * S[0];
  out[1] = -t * S[1];
}

static void spatial_decode(const OGeom *g, long s, int x[4]) {
  x[0] = x[1] = x[2] = x[3] = 0;
  for (int k = 0; k < g->tdir; ++k) {
    x[k] = (int)(s % g->N[k]);
    s /= g->N[k];
  }
}
static long spatial_index(const OGeom *g, const int x[4]) {
  long s = 0, st = 1;
  for (int k = 0; k < g->tdir; ++k) {
    s += x[k] * st;
    st *= g->N[k];
  }
  return s;
}

// P(x) field: reference src/polyakov.cu:415-440, stored at the spatial lexicographic index.
void o_poly_field(const OGeom *g, const double *lat, int multihit, double *P /* 2*Vs */) {
  for (long s = 0; s < g->Vs; ++s) {
    int x[4];
    spatial_decode(g, s, x);
    cd res = 1.0;
    for (x[g->tdir] = 0; x[g->tdir] < g->N[g->tdir]; ++x[g->tdir]) {
      const int pos = lex(g, x) >> 1, par = parity_of(g, x);
      if (multihit) {
        double m[2];
        o_multihit(g, lat, pos, par, m);
        res *= cd(m[0], m[1]);
      } else {
        res *= std::polar(1.0, lat[pos + par * g->Vh + g->tdir * g->V]);
      }
    }
    P[2 * s] = res.real();
    P[2 * s + 1] = res.imag();
  }
}

// reference src/polyakov.cu:514-535,568,618-631: out[2(r-1)+{0,1}] = C(r), r = 1..R, R = Grid[0]/2.
void o_poly_corr(const OGeom *g, const double *lat, int multihit, double *out) {
  const int R = g->N[0] / 2;
  std::vector<double> P(2 * g->Vs);
  o_poly_field(g, lat, multihit, P.data());
  for (int r = 1; r <= R; ++r) {
    cd acc = 0.0;
    for (long s = 0; s < g->Vs; ++s) {
      int x[4];
      spatial_decode(g, s, x);
      const cd p0(P[2 * s], P[2 * s + 1]);
      for (int dir = 0; dir < g->tdir; ++dir) {
        int y[4] = {x[0], x[1], x[2], x[3]};
        y[dir] = (y[dir] + r) % g->N[dir];
        const long sp = spatial_index(g, y);
        acc += p0 * std::conj(cd(P[2 * sp], P[2 * sp + 1]));
      }
    }
    acc /= (double)g->Vs * (double)(g->dims - 1);
    out[2 * (r - 1)] = acc.real();
    out[2 * (r - 1) + 1] = acc.imag();
  }
}

// Multilevel correlator, reference src/multilevel.cu:639-732 with kernels
// :239-258 (multihit field), :331-360 (T2), :439-456 (T4), :532-553 (final).
// Metropolis draws come from the Philox stream starting at pass *pass
// (advanced on return), so a GPU run with the same (seed, pass) follows the
// same chain up to FP32/FP64 accept-decision flips (none when metrop = 0).
void o_multilevel(const OGeom *g, const double *lat_in, uint64_t seed, uint32_t chain, uint64_t *pass, int n4,
                  int k4, int n2, int k2, int metrop, int ovrn, double *out) {
  const int R = g->N[0] / 2;
  const int nl2 = g->N[g->tdir] / 2, nl4 = g->N[g->tdir] / 4;
  const long size = g->Vs * R * (g->dims - 1);
  std::vector<double> lat(lat_in, lat_in + g->V * g->dims);
  std::vector<cd> mh(g->V), T2(size * nl2), T4(size * nl4, 0.0);
  auto sweep = [&](int ml) {
    for (int m = 0; m < metrop; ++m) o_metropolis_philox(g, lat.data(), seed, chain, (*pass)++, ml);
    for (int o = 0; o < ovrn; ++o) o_overrelax(g, lat.data(), ml);
  };
  for (int i = 0; i < n4; ++i) {
    for (int j = 0; j < k4; ++j) sweep(4);
    std::fill(T2.begin(), T2.end(), cd(0.0));
    for (int k = 0; k < n2; ++k) {
      for (int l = 0; l < k2; ++l) sweep(2);
      for (long id4 = 0; id4 < g->V; ++id4) {
        int x[4];
        long r = id4;
        for (int q = 0; q < 4; ++q) {
          x[q] = (int)(r % g->N[q]);
          r /= g->N[q];
        }
        double m[2];
        o_multihit(g, lat.data(), lex(g, x) >> 1, parity_of(g, x), m);
        mh[id4] = cd(m[0], m[1]);
      }
      for (long s = 0; s < g->Vs; ++s) {
        int x[4];
        spatial_decode(g, s, x);
        for (int dir = 0; dir < g->dims - 1; ++dir)
          for (int rr = 1; rr <= R; ++rr) {
            int y[4] = {x[0], x[1], x[2], x[3]};
            y[dir] = (y[dir] + rr) % g->N[dir];
            const long sp = spatial_index(g, y);
            for (int layer = 0; layer < nl2; ++layer) {
              cd p0 = 1.0, p1 = 1.0;
              for (int t = 2 * layer; t < 2 * layer + 2; ++t) {
                p0 *= mh[s + t * g->Vs];
                p1 *= std::conj(mh[sp + t * g->Vs]);
              }
              T2[s + g->Vs * (rr - 1) + g->Vs * R * dir + size * layer] += p0 * p1;
            }
          }
      }
    }
    const double l2norm = 1.0 / n2;
    for (long id = 0; id < size; ++id)
      for (int l4 = 0; l4 < nl4; ++l4)
        T4[id + size * l4] += (T2[id + size * (2 * l4)] * l2norm) * (T2[id + size * (2 * l4 + 1)] * l2norm);
  }
  const double l4norm = 1.0 / n4;
  for (int r = 0; r < R; ++r) {
    cd acc = 0.0;
    for (long s = 0; s < g->Vs; ++s)
      for (int dir = 0; dir < g->dims - 1; ++dir) {
        cd pl = 1.0;
        for (int l4 = 0; l4 < nl4; ++l4) pl *= T4[s + g->Vs * r + g->Vs * R * dir + size * l4] * l4norm;
        acc += pl;
      }
    acc /= (double)g->Vs * (double)(g->dims - 1);
    out[2 * r] = acc.real();
    out[2 * r + 1] = acc.imag();
  }
}

// Wilson action S = beta * sum_P w_P (1 - cos theta_P), w = 1/xi (SS), xi (ST),
// the action whose local part the reference's staple encodes
// (include/staple.h:75-76).  grad (optional, V*dims) = dS/dtheta.
double o_action(const OGeom *g, const double *lat, double *grad) {
  if (grad) std::memset(grad, 0, sizeof(double) * g->V * g->dims);
  double S = 0.0;
  for (int p = 0; p < 2; ++p)
    for (int id = 0; id < (int)g->Vh; ++id)
      for (int mu = 0; mu < g->dims - 1; ++mu)
        for (int nu = mu + 1; nu < g->dims; ++nu) {
          const long a = id + p * g->Vh + mu * g->V;
          const long b = o_index_eo_neg(g, id, p, mu, 1, -1, 0) + nu * g->V;
          const long c = o_index_eo_neg(g, id, p, nu, 1, -1, 0) + mu * g->V;
          const long d = id + p * g->Vh + nu * g->V;
          const double th = lat[a] + lat[b] - lat[c] - lat[d];
          const double w = (mu == g->tdir || nu == g->tdir) ? g->aniso : 1.0 / g->aniso;
          S += g->beta * w * (1.0 - std::cos(th));
          if (grad) {
            const double s = g->beta * w * std::sin(th);
            grad[a] += s;
            grad[b] += s;
            grad[c] -= s;
            grad[d] -= s;
          }
        }
  return S;
}

// 2D topological charge Q = (1/2pi) sum_x wrap(theta_P(x)), wrap to (-pi, pi].
double o_topological_charge_2d(const OGeom *g, const double *lat) {
  double q = 0.0;
  for (int p = 0; p < 2; ++p)
    for (int id = 0; id < (int)g->Vh; ++id) {
      double th = lat[id + p * g->Vh] + L(g, lat, o_index_eo_neg(g, id, p, 0, 1, -1, 0), 1) -
                  L(g, lat, o_index_eo_neg(g, id, p, 1, 1, -1, 0), 0) - lat[id + p * g->Vh + g->V];
      th = std::remainder(th, 2.0 * M_PI);
      q += th;
    }
  return q / (2.0 * M_PI);
}

}  // extern "C"
