// Circular coupling transform of the 2D U(1) flow: a mixture of
// non-compact projections (NCP) acting on plaquette angles, after the
// gauge-equivariant coupling layers of Kanwar et al., "Equivariant flow-based
// sampling for lattice gauge theory", arXiv:2003.06413 (method only).  The
// reference has no flow; these kernels are the elementwise core of
// latticeu1_b200/flow.py, each with its analytic backward.
//
// For an angle x, centred to xc = remainder(x, 2 pi) in [-pi, pi]:
//   g(xc; alpha) = 2 atan2(alpha sin(xc/2), cos(xc/2))       (monotone, fixes +-pi)
//   g'(xc)       = alpha / (cos^2(xc/2) + alpha^2 sin^2(xc/2))
//   h(xc)        = sum_k w_k g(xc; alpha_k) + shift,  w = softmax(logit),  alpha_k = exp(a_k)
// Per element the parameters are p = (a_0..a_{K-1}, logit_0..logit_{K-1}, shift).
//   forward:  dy = h(xc) - xc (the change the caller adds to the updated link), logd = log h'(xc)
//   inverse:  given y, z = remainder(y - shift, 2 pi); x solves sum_k w_k g(x) = z (bisection);
//             dx = x - z - shift (the change that undoes the forward step), logd = log h'(x)
#include <string>

#include "u1_internal.h"

namespace {

constexpr int kMaxK = 8;
constexpr float kTwoPi = 6.28318530717958647692f;

int flfail(int code, const std::string &msg) {
  u1i::set_error(msg);
  return code;
}

struct Mix {
  float w[kMaxK], al[kMaxK];
  float H;   // sum_k w_k g_k
  float Hp;  // sum_k w_k g'_k  (> 0)
};

// weights, alphas and the mixture values at xc
__device__ __forceinline__ void mix_eval(float xc, const float *__restrict__ p, int K, Mix &m, float (&g)[kMaxK],
                                         float (&gp)[kMaxK], float &s, float &c) {
  float mx = -INFINITY;
  for (int k = 0; k < K; ++k) mx = fmaxf(mx, p[K + k]);
  float z = 0.f;
  for (int k = 0; k < K; ++k) {
    m.w[k] = expf(p[K + k] - mx);
    z += m.w[k];
  }
  const float iz = 1.f / z;
  sincosf(0.5f * xc, &s, &c);
  m.H = 0.f;
  m.Hp = 0.f;
  for (int k = 0; k < K; ++k) {
    m.w[k] *= iz;
    m.al[k] = expf(fminf(fmaxf(p[k], -8.f), 8.f));
    const float a = m.al[k];
    const float den = c * c + a * a * s * s;
    g[k] = 2.f * atan2f(a * s, c);
    gp[k] = a / den;
    m.H += m.w[k] * g[k];
    m.Hp += m.w[k] * gp[k];
  }
}

__global__ void k_ncp_forward(const float *__restrict__ x, const float *__restrict__ prm, long long n, int K,
                              float *__restrict__ dy, float *__restrict__ logd) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float *p = prm + t * (2 * K + 1);
  const float xc = remainderf(x[t], kTwoPi);
  Mix m;
  float g[kMaxK], gp[kMaxK], s, c;
  mix_eval(xc, p, K, m, g, gp, s, c);
  dy[t] = m.H + p[2 * K] - xc;
  logd[t] = logf(m.Hp);
}

// Partials of H, Hp with respect to xc and the parameters, combined with the
// upstream gradients: G_H multiplies dH/d., G_P multiplies dHp/d. (both
// already include every chain factor of the caller).
__device__ __forceinline__ void mix_backward(const Mix &m, const float (&g)[kMaxK], const float (&gp)[kMaxK], float s,
                                             float c, int K, float G_H, float G_P, float &gxc, float *__restrict__ gp_out) {
  float dHp_dx = 0.f;
  for (int k = 0; k < K; ++k) {
    const float a = m.al[k];
    const float den = c * c + a * a * s * s;
    const float iden2 = 1.f / (den * den);
    const float dg_da = 2.f * s * c / den;                       // dg/dalpha
    const float dgp_da = (c * c - a * a * s * s) * iden2;        // dg'/dalpha
    const float dgp_dx = -a * s * c * (a * a - 1.f) * iden2;     // dg'/dx
    dHp_dx += m.w[k] * dgp_dx;
    // a_k: alpha = exp(a) (clamped: zero gradient outside)
    gp_out[k] = (G_H * m.w[k] * dg_da + G_P * m.w[k] * dgp_da) * a;
    // logit_k through the softmax
    gp_out[K + k] = G_H * m.w[k] * (g[k] - m.H) + G_P * m.w[k] * (gp[k] - m.Hp);
  }
  gxc = G_H * m.Hp + G_P * dHp_dx;
}

__global__ void k_ncp_backward(const float *__restrict__ x, const float *__restrict__ prm,
                               const float *__restrict__ gdy, const float *__restrict__ glogd, long long n, int K,
                               float *__restrict__ gx, float *__restrict__ gprm) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float *p = prm + t * (2 * K + 1);
  float *gpo = gprm + t * (2 * K + 1);
  const float xc = remainderf(x[t], kTwoPi);
  Mix m;
  float g[kMaxK], gp[kMaxK], s, c;
  mix_eval(xc, p, K, m, g, gp, s, c);
  const float a = gdy ? gdy[t] : 0.f;   // dL/d(dy): dy = H + shift - xc
  const float b = glogd ? glogd[t] : 0.f;  // dL/d(logd): logd = log Hp
  float gxc;
  mix_backward(m, g, gp, s, c, K, a, b / m.Hp, gxc, gpo);
  for (int k = 0; k < K; ++k)
    if (fabsf(p[k]) > 8.f) gpo[k] = 0.f;
  gpo[2 * K] = a;
  gx[t] = gxc - a;
}

// Bisection on the monotone map xc -> H(xc) over [-pi, pi] (H(-pi) = -pi,
// H(pi) = pi): 40 halvings reach the float resolution of the interval.
__global__ void k_ncp_inverse(const float *__restrict__ y, const float *__restrict__ prm, long long n, int K,
                              float *__restrict__ dx, float *__restrict__ xsol, float *__restrict__ logd) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float *p = prm + t * (2 * K + 1);
  const float shift = p[2 * K];
  const float z = remainderf(y[t] - shift, kTwoPi);
  float lo = -3.14159265358979f, hi = 3.14159265358979f;
  Mix m;
  float g[kMaxK], gp[kMaxK], s, c;
  for (int it = 0; it < 40; ++it) {
    const float mid = 0.5f * (lo + hi);
    mix_eval(mid, p, K, m, g, gp, s, c);
    if (m.H < z)
      lo = mid;
    else
      hi = mid;
  }
  const float xs = 0.5f * (lo + hi);
  mix_eval(xs, p, K, m, g, gp, s, c);
  xsol[t] = xs;
  dx[t] = xs - z - shift;
  logd[t] = logf(m.Hp);
}

// Backward of the inverse by implicit differentiation at the solution xs
// (H(xs) = z = y - shift mod 2 pi):  dxs/dy = 1/Hp, dxs/dq = -(dH/dq)/Hp,
// dxs/dshift = -1/Hp; outputs dx = xs - z - shift and logd = log Hp(xs).
__global__ void k_ncp_inverse_backward(const float *__restrict__ xsol, const float *__restrict__ prm,
                                       const float *__restrict__ gdx, const float *__restrict__ glogd, long long n,
                                       int K, float *__restrict__ gy, float *__restrict__ gprm) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float *p = prm + t * (2 * K + 1);
  float *gpo = gprm + t * (2 * K + 1);
  Mix m;
  float g[kMaxK], gp[kMaxK], s, c;
  mix_eval(xsol[t], p, K, m, g, gp, s, c);
  const float a = gdx ? gdx[t] : 0.f;
  const float b = glogd ? glogd[t] : 0.f;
  // dL/dxs from both outputs: dx = xs - z - shift (explicit xs term 1), logd = log Hp(xs)
  float dHp_dx = 0.f;
  for (int k = 0; k < K; ++k) {
    const float al = m.al[k];
    const float den = c * c + al * al * s * s;
    dHp_dx += m.w[k] * (-al * s * c * (al * al - 1.f)) / (den * den);
  }
  const float Gx = a + b * dHp_dx / m.Hp;  // total dL/dxs
  const float r = Gx / m.Hp;               // dL/dz through xs
  // explicit parameter partials of logd (G_P) and of xs through H (G_H = -r)
  float unused;
  mix_backward(m, g, gp, s, c, K, -r, b / m.Hp, unused, gpo);
  for (int k = 0; k < K; ++k)
    if (fabsf(p[k]) > 8.f) gpo[k] = 0.f;
  // z = y - shift (mod 2 pi); dx = xs - z - shift:  d/dy = r - a,  d/dshift = -r + a - a = -r
  gy[t] = r - a;
  gpo[2 * K] = -r;
}

int check_args(long long n, int K) {
  if (n < 0) return flfail(U1_ERR_INVALID, "ncp: negative element count");
  if (K < 1 || K > kMaxK) return flfail(U1_ERR_INVALID, "ncp: K must be in [1, 8]");
  return U1_OK;
}

int blocks(long long n) { return (int)((n + 255) / 256); }

}  // namespace

extern "C" int u1_ncp_forward(const float *x, const float *params, int64_t n, int K, float *dy, float *logd,
                              void *stream) {
  int rc = check_args(n, K);
  if (rc) return rc;
  if (n == 0) return U1_OK;
  if (!x || !params || !dy || !logd) return flfail(U1_ERR_INVALID, "u1_ncp_forward: null pointer");
  k_ncp_forward<<<blocks(n), 256, 0, (cudaStream_t)stream>>>(x, params, n, K, dy, logd);
  U1_LAUNCH_CHECK("k_ncp_forward");
  return U1_OK;
}

extern "C" int u1_ncp_backward(const float *x, const float *params, const float *gdy, const float *glogd, int64_t n,
                               int K, float *gx, float *gparams, void *stream) {
  int rc = check_args(n, K);
  if (rc) return rc;
  if (n == 0) return U1_OK;
  if (!x || !params || !gx || !gparams) return flfail(U1_ERR_INVALID, "u1_ncp_backward: null pointer");
  k_ncp_backward<<<blocks(n), 256, 0, (cudaStream_t)stream>>>(x, params, gdy, glogd, n, K, gx, gparams);
  U1_LAUNCH_CHECK("k_ncp_backward");
  return U1_OK;
}

extern "C" int u1_ncp_inverse(const float *y, const float *params, int64_t n, int K, float *dx, float *xsol,
                              float *logd, void *stream) {
  int rc = check_args(n, K);
  if (rc) return rc;
  if (n == 0) return U1_OK;
  if (!y || !params || !dx || !xsol || !logd) return flfail(U1_ERR_INVALID, "u1_ncp_inverse: null pointer");
  k_ncp_inverse<<<blocks(n), 256, 0, (cudaStream_t)stream>>>(y, params, n, K, dx, xsol, logd);
  U1_LAUNCH_CHECK("k_ncp_inverse");
  return U1_OK;
}

extern "C" int u1_ncp_inverse_backward(const float *xsol, const float *params, const float *gdx, const float *glogd,
                                       int64_t n, int K, float *gy, float *gparams, void *stream) {
  int rc = check_args(n, K);
  if (rc) return rc;
  if (n == 0) return U1_OK;
  if (!xsol || !params || !gy || !gparams) return flfail(U1_ERR_INVALID, "u1_ncp_inverse_backward: null pointer");
  k_ncp_inverse_backward<<<blocks(n), 256, 0, (cudaStream_t)stream>>>(xsol, params, gdx, glogd, n, K, gy, gparams);
  U1_LAUNCH_CHECK("k_ncp_inverse_backward");
  return U1_OK;
}
