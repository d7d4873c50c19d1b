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
#include <cuda_bf16.h>

#include <string>

#include "u1_internal.h"

namespace {

constexpr int kMaxK = 8;
// Threads per block of the fused layer kernels (one configuration per block):
// their shared memory (up to about 200 KB at L = 32) allows one block per SM,
// so the block itself must bring enough warps to hide shared-memory latency.
constexpr int kFlowThreads = 512;
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

// ---------------------------------------------------------------------------
// One whole coupling layer, forward only (the proposal path of the sampler),
// one block per configuration of an L x L lattice, theta[b][mu][x1][x0]:
//   P(x) = th_0(x) + th_1(x+e0) - th_0(x+e1) - th_1(x);
//   context = (cos P, sin P) on the frozen plaquettes, 0 elsewhere;
//   hidden = LeakyReLU(conv3x3(context; W1, B1)), circular padding;
//   params = conv3x3(hidden; W2, B2) at the active plaquettes;
//   the mixture transform moves each active plaquette, its updated link
//   absorbs the change, and logdet[b] = sum of log H' over the active ones.
// Masks for (mu, off): stripes x_nu = off (mod 4), nu = 1 - mu; the active
// plaquette of link th_mu(x) is P(x) (mu = 0) or P(x - e0) (mu = 1); frozen
// plaquettes have (x_nu - off) mod 4 in {1, 2}.  Weights are rounded to
// bfloat16 on load (the layer's stored precision); activations and sums are
// FP32.  Convolutions are cross-correlations as torch.nn.Conv2d:
//   out[c][y][x] = B[c] + sum_{ci,ky,kx} W[c][ci][ky][kx] in[ci][y+ky-1][x+kx-1].
__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16(v)); }

__device__ __forceinline__ void active_pos(int a, int L, int mu, int off, int &x1, int &x0) {
  if (mu == 0) {
    x1 = 4 * (a / L) + off;
    x0 = a % L;
  } else {
    const int q = L / 4;
    x1 = a / q;
    x0 = 4 * (a % q) + ((off + 3) & 3);
  }
}

// 3x3 circular neighbourhood of pixel (x1, x0): offsets (yy * L + xx), ky-major.
__device__ __forceinline__ void nbr9(int x1, int x0, int L, int (&o)[9]) {
#pragma unroll
  for (int ky = 0; ky < 3; ++ky) {
    int yy = x1 + ky - 1;
    yy = yy < 0 ? yy + L : (yy >= L ? yy - L : yy);
#pragma unroll
    for (int kx = 0; kx < 3; ++kx) {
      int xx = x0 + kx - 1;
      xx = xx < 0 ? xx + L : (xx >= L ? xx - L : xx);
      o[ky * 3 + kx] = yy * L + xx;
    }
  }
}

__device__ __forceinline__ void fma4(float4 &acc, const float4 w, float h) {
  acc.x = fmaf(w.x, h, acc.x);
  acc.y = fmaf(w.y, h, acc.y);
  acc.z = fmaf(w.z, h, acc.z);
  acc.w = fmaf(w.w, h, acc.w);
}

// The mixture transform of one active plaquette: forward, the change dy of
// its updated link and log H'(xc); INV, the inverse transform (bisection on
// the monotone H, as k_ncp_inverse): the change dx that undoes a forward step
// and log H'(xs) at the solution.
template <bool INV>
__device__ __forceinline__ float layer_transform(float P, const float *__restrict__ pp, int K, float &logd) {
  Mix m;
  float g[kMaxK], gp[kMaxK], s, c;
  if (!INV) {
    const float xc = remainderf(P, kTwoPi);
    mix_eval(xc, pp, K, m, g, gp, s, c);
    logd = logf(m.Hp);
    return m.H + pp[2 * K] - xc;
  }
  const float shift = pp[2 * K];
  const float z = remainderf(P - shift, kTwoPi);
  float lo = -3.14159265358979f, hi = 3.14159265358979f;
  for (int it = 0; it < 40; ++it) {
    const float mid = 0.5f * (lo + hi);
    mix_eval(mid, pp, K, m, g, gp, s, c);
    if (m.H < z)
      lo = mid;
    else
      hi = mid;
  }
  const float xs = 0.5f * (lo + hi);
  mix_eval(xs, pp, K, m, g, gp, s, c);
  logd = logf(m.Hp);
  return xs - z - shift;
}

// Shared memory (floats, each part a multiple of 4): th[2 LL], P[LL], ctx[2 LL],
// hid[H LL], w1t[18 H] ([ci*9 + k][c]), b1[H], w2t[9 H CP] ([ci*9 + k][o],
// outputs padded to CP = round4(2K+1) with zeros), b2[CP], prm[LL/4 * CP].
// INV: the inverse layer (the context plaquettes hold no updated link, so the
// same parameters come out; the transform is inverted), as Coupling.inverse.
template <bool INV>
__global__ void __launch_bounds__(kFlowThreads)
    k_flow_layer_forward(const float *__restrict__ th_in, float *__restrict__ th_out, float *__restrict__ logdet,
                         int L, int mu, int off, int K, int H, const float *__restrict__ W1,
                         const float *__restrict__ B1, const float *__restrict__ W2, const float *__restrict__ B2,
                         float slope) {
  extern __shared__ float4 sm4[];
  float *sm = reinterpret_cast<float *>(sm4);
  const int LL = L * L, C2 = 2 * K + 1, CP = (C2 + 3) & ~3, nact = LL / 4;
  float *th = sm;
  float *P = th + 2 * LL;
  float *ctx = P + LL;
  float *hid = ctx + 2 * LL;
  float *w1t = hid + H * LL;
  float *b1 = w1t + 18 * H;
  float *w2t = b1 + H;
  float *b2 = w2t + 9 * H * CP;
  float *prm = b2 + CP;
  __shared__ double red[32];
  const int nt = blockDim.x, tid = threadIdx.x;
  const float *src = th_in + (size_t)blockIdx.x * 2 * LL;
  for (int t = tid; t < 2 * LL; t += nt) th[t] = src[t];
  for (int t = tid; t < 18 * H; t += nt) {  // W1[c][ci][ky][kx] -> w1t[(ci*9 + k) * H + c]
    const int c = t / 18, r = t - c * 18;
    w1t[r * H + c] = bf16_round(W1[t]);
  }
  for (int t = tid; t < H; t += nt) b1[t] = bf16_round(B1[t]);
  for (int t = tid; t < 9 * H * CP; t += nt) {  // W2[o][ci][ky][kx] -> w2t[(ci*9 + k) * CP + o]
    const int r = t / CP, o = t - r * CP;
    w2t[t] = o < C2 ? bf16_round(W2[(size_t)o * H * 9 + r]) : 0.f;
  }
  for (int t = tid; t < CP; t += nt) b2[t] = t < C2 ? bf16_round(B2[t]) : 0.f;
  __syncthreads();
  for (int p = tid; p < LL; p += nt) {
    const int x0 = p % L, x1 = p / L;
    const int x0p = x0 + 1 == L ? 0 : x0 + 1, x1p = x1 + 1 == L ? 0 : x1 + 1;
    const float v = th[p] + th[LL + x1 * L + x0p] - th[x1p * L + x0] - th[LL + p];
    P[p] = v;
    const int xn = mu == 0 ? x1 : x0;
    const int r = (xn - off) & 3;
    const bool frozen = r == 1 || r == 2;
    float sn, cs;
    sincosf(v, &sn, &cs);
    ctx[p] = frozen ? cs : 0.f;
    ctx[LL + p] = frozen ? sn : 0.f;
  }
  __syncthreads();
  // conv1 + LeakyReLU: one pixel per work item, all H channels, four at a time
  const float4 *w1v = reinterpret_cast<const float4 *>(w1t);
  for (int p = tid; p < LL; p += nt) {
    int o9[9];
    nbr9(p / L, p % L, L, o9);
    float in[18];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      in[k] = ctx[o9[k]];
      in[9 + k] = ctx[LL + o9[k]];
    }
    for (int c4 = 0; c4 < H; c4 += 4) {
      float4 acc = make_float4(b1[c4], b1[c4 + 1], b1[c4 + 2], b1[c4 + 3]);
#pragma unroll
      for (int r = 0; r < 18; ++r) fma4(acc, w1v[(r * H + c4) >> 2], in[r]);
      hid[(c4 + 0) * LL + p] = acc.x > 0.f ? acc.x : slope * acc.x;
      hid[(c4 + 1) * LL + p] = acc.y > 0.f ? acc.y : slope * acc.y;
      hid[(c4 + 2) * LL + p] = acc.z > 0.f ? acc.z : slope * acc.z;
      hid[(c4 + 3) * LL + p] = acc.w > 0.f ? acc.w : slope * acc.w;
    }
  }
  __syncthreads();
  // conv2 at the active plaquettes: work item = (active pixel, group of four outputs)
  const float4 *w2v = reinterpret_cast<const float4 *>(w2t);
  const int ng = CP / 4;
  for (int q = tid; q < nact * ng; q += nt) {
    const int a = q / ng, og = q - a * ng;
    int x1, x0;
    active_pos(a, L, mu, off, x1, x0);
    int o9[9];
    nbr9(x1, x0, L, o9);
    float4 acc = make_float4(b2[og * 4], b2[og * 4 + 1], b2[og * 4 + 2], b2[og * 4 + 3]);
    for (int ci = 0; ci < H; ++ci) {
      const float *hc = hid + ci * LL;
#pragma unroll
      for (int k = 0; k < 9; ++k) fma4(acc, w2v[((ci * 9 + k) * CP >> 2) + og], hc[o9[k]]);
    }
    float *dst = prm + a * CP + og * 4;
    dst[0] = acc.x;
    dst[1] = acc.y;
    dst[2] = acc.z;
    dst[3] = acc.w;
  }
  __syncthreads();
  double ld = 0.0;
  for (int a = tid; a < nact; a += nt) {
    int x1, x0;
    active_pos(a, L, mu, off, x1, x0);
    float lg;
    const float dy = layer_transform<INV>(P[x1 * L + x0], prm + a * CP, K, lg);
    ld += (double)lg;
    if (mu == 0)
      th[x1 * L + x0] += dy;
    else
      th[LL + x1 * L + (x0 + 1 == L ? 0 : x0 + 1)] += dy;
  }
  // block sum of the log-derivatives (fixed order)
  for (int o = 16; o > 0; o >>= 1) ld += __shfl_xor_sync(0xffffffffu, ld, o);
  if ((tid & 31) == 0) red[tid >> 5] = ld;
  __syncthreads();
  float *dst = th_out + (size_t)blockIdx.x * 2 * LL;
  for (int t = tid; t < 2 * LL; t += nt) dst[t] = th[t];
  if (tid == 0) {
    double tot = 0.0;
    for (int w = 0; w < (nt + 31) / 32; ++w) tot += red[w];
    logdet[blockIdx.x] = (float)tot;
  }
}

// ---------------------------------------------------------------------------
// Backward of k_flow_layer_forward<INV> for one configuration per block, for
// L up to 32.  The forward is recomputed (plaquettes, context, then the
// parameters, accumulated chunk by chunk over the hidden channels); then,
// given gth_out (dL/dtheta_out) and gld (dL/dlogdet), the adjoint runs
// backwards through the transform, conv2, the LeakyReLU, conv1, the context
// and the plaquette map:
//   gth_in = gth_out + plaquette-adjoint(gP),
//   gP = [active] d/dP of the transform + [frozen] (-sin P, cos P) . g_context.
// Only Cc hidden channels (8, or 4 when H % 8 != 0) are held in shared memory
// at a time: their conv1 pre-activations are recomputed from the context
// (18 multiply-adds per channel and pixel) for the parameter pass and again
// for the adjoint pass, which for each chunk forms dL/dpre, the chunk's
// weight gradients and its share of the context gradient.  This keeps an
// L = 32, H = 32 layer at about 157 KB of shared memory (the whole hidden
// layer and its gradient would take 256 KB).  Convolution adjoints are
// gathers (each output sums over the inputs that read it), so no atomics;
// weight gradients (with respect to the bf16-rounded weights the forward
// used, passed straight to the FP32 master weights) go to per-block partials
// wpart[b][:] = (gW1[c][ci][k], gB1[c], gW2[o][ci][k], gB2[o]), summed over
// blocks in a fixed order by k_flow_wgrad_reduce.
__device__ __forceinline__ float lrelu(float v, float slope) { return v > 0.f ? v : slope * v; }
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <bool INV>
__global__ void __launch_bounds__(kFlowThreads)
    k_flow_layer_backward(const float *__restrict__ th_in, const float *__restrict__ gth_out,
                          const float *__restrict__ gld, float *__restrict__ gth_in, float *__restrict__ wpart, int L,
                          int mu, int off, int K, int H, int Cc, const float *__restrict__ W1,
                          const float *__restrict__ B1, const float *__restrict__ W2, const float *__restrict__ B2,
                          float slope) {
  extern __shared__ float4 sm4[];
  float *sm = reinterpret_cast<float *>(sm4);
  const int LL = L * L, C2 = 2 * K + 1, CP = (C2 + 3) & ~3, nact = LL / 4, ng = CP / 4;
  float *th = sm;                  // 2 LL
  float *P = th + 2 * LL;          // LL
  float *ctx = P + LL;             // 2 LL
  float *w1t = ctx + 2 * LL;       // 18 H   [ci*9 + k][c]
  float *b1 = w1t + 18 * H;        // H
  float *w2t = b1 + H;             // 9 H CP [ci*9 + k][o]
  float *b2 = w2t + 9 * H * CP;    // CP
  float *prm = b2 + CP;            // nact CP
  float *gprmT = prm + nact * CP;  // CP nact  dL/dparams, parameter-major ([o][a]: conflict-free across a)
  float *gctx = gprmT + nact * CP; // 2 LL
  float *gP = gctx + 2 * LL;       // LL
  float *hc = gP + LL;             // Cc LL  pre-activations of the chunk's channels
  float *ghc = hc + Cc * LL;       // Cc LL  dL/dpre of the chunk's channels
  int *amap = reinterpret_cast<int *>(ghc + Cc * LL);  // LL: active index of a plaquette, or -1
  int *apos = amap + LL;                                     // nact: pixel of active plaquette a
  int *nbt = apos + nact;                                    // 9 LL: nbt[k * LL + p] = pixel at offset k of p
  const int nt = blockDim.x, tid = threadIdx.x, b = blockIdx.x;
  const float *src = th_in + (size_t)b * 2 * LL;
  const float *go = gth_out + (size_t)b * 2 * LL;
  for (int t = tid; t < 2 * LL; t += nt) th[t] = src[t];
  for (int t = tid; t < 18 * H; t += nt) {
    const int c = t / 18, r = t - c * 18;
    w1t[r * H + c] = bf16_round(W1[t]);
  }
  for (int t = tid; t < H; t += nt) b1[t] = bf16_round(B1[t]);
  for (int t = tid; t < 9 * H * CP; t += nt) {
    const int r = t / CP, o = t - r * CP;
    w2t[t] = o < C2 ? bf16_round(W2[(size_t)o * H * 9 + r]) : 0.f;
  }
  for (int t = tid; t < CP; t += nt) b2[t] = t < C2 ? bf16_round(B2[t]) : 0.f;
  for (int p = tid; p < LL; p += nt) {
    amap[p] = -1;
    gP[p] = 0.f;
    int o9[9];
    nbr9(p / L, p % L, L, o9);
#pragma unroll
    for (int k = 0; k < 9; ++k) nbt[k * LL + p] = o9[k];
  }
  __syncthreads();
  for (int a = tid; a < nact; a += nt) {
    int x1, x0;
    active_pos(a, L, mu, off, x1, x0);
    amap[x1 * L + x0] = a;
    apos[a] = x1 * L + x0;
  }
  for (int p = tid; p < LL; p += nt) {
    const int x0 = p % L, x1 = p / L;
    const int x0p = x0 + 1 == L ? 0 : x0 + 1, x1p = x1 + 1 == L ? 0 : x1 + 1;
    const float v = th[p] + th[LL + x1 * L + x0p] - th[x1p * L + x0] - th[LL + p];
    P[p] = v;
    const int xn = mu == 0 ? x1 : x0;
    const int r = (xn - off) & 3;
    const bool frozen = r == 1 || r == 2;
    float sn, cs;
    sincosf(v, &sn, &cs);
    ctx[p] = frozen ? cs : 0.f;
    ctx[LL + p] = frozen ? sn : 0.f;
  }
  for (int q = tid; q < nact * CP; q += nt) prm[q] = b2[q % CP];
  for (int t = tid; t < 2 * LL; t += nt) gctx[t] = 0.f;
  __syncthreads();
  const float4 *w1v = reinterpret_cast<const float4 *>(w1t);
  const float4 *w2v = reinterpret_cast<const float4 *>(w2t);
  // conv1 pre-activations of channels c0 .. c0+Cc-1 into hc
  auto conv1_chunk = [&](int c0) {
    for (int p = tid; p < LL; p += nt) {
      float in[18];
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int q = nbt[k * LL + p];
        in[k] = ctx[q];
        in[9 + k] = ctx[LL + q];
      }
      for (int c4 = 0; c4 < Cc; c4 += 4) {
        const int c = c0 + c4;
        float4 acc = make_float4(b1[c], b1[c + 1], b1[c + 2], b1[c + 3]);
#pragma unroll
        for (int r = 0; r < 18; ++r) fma4(acc, w1v[(r * H + c) >> 2], in[r]);
        hc[(c4 + 0) * LL + p] = acc.x;
        hc[(c4 + 1) * LL + p] = acc.y;
        hc[(c4 + 2) * LL + p] = acc.z;
        hc[(c4 + 3) * LL + p] = acc.w;
      }
    }
  };
  // ---- forward recomputation: parameters, summed over the hidden channels in order
  for (int c0 = 0; c0 < H; c0 += Cc) {
    conv1_chunk(c0);
    __syncthreads();
    for (int q = tid; q < nact * ng; q += nt) {
      const int a = q / ng, og = q - a * ng;
      const int pa = apos[a];
      float *dst = prm + a * CP + og * 4;
      float4 acc = make_float4(dst[0], dst[1], dst[2], dst[3]);
      for (int cl = 0; cl < Cc; ++cl) {
        const float *pc = hc + cl * LL;
#pragma unroll
        for (int k = 0; k < 9; ++k)
          fma4(acc, w2v[(((c0 + cl) * 9 + k) * CP >> 2) + og], lrelu(pc[nbt[k * LL + pa]], slope));
      }
      dst[0] = acc.x;
      dst[1] = acc.y;
      dst[2] = acc.z;
      dst[3] = acc.w;
    }
    __syncthreads();
  }
  // ---- transform adjoint: gprm and the active plaquettes' gP
  const float gl = gld ? gld[b] : 0.f;
  for (int a = tid; a < nact; a += nt) {
    const int pa = apos[a];
    const int x1 = pa / L, x0 = pa - x1 * L;
    const float *pp = prm + a * CP;
    float gpo[2 * kMaxK + 1];
    const int link = mu == 0 ? pa : LL + x1 * L + (x0 + 1 == L ? 0 : x0 + 1);
    const float gout = go[link];
    Mix m;
    float g[kMaxK], gp[kMaxK], s, c;
    if (!INV) {  // dy = H(xc) + shift - xc, logd = log H'(xc)
      const float xc = remainderf(P[pa], kTwoPi);
      mix_eval(xc, pp, K, m, g, gp, s, c);
      float gxc;
      mix_backward(m, g, gp, s, c, K, gout, gl / m.Hp, gxc, gpo);
      gpo[2 * K] = gout;
      gP[pa] = gxc - gout;
    } else {  // dx = xs - z - shift with H(xs) = z = P - shift (mod 2 pi), logd = log H'(xs)
      const float shift = pp[2 * K];
      const float z = remainderf(P[pa] - shift, kTwoPi);
      float lo = -3.14159265358979f, hi = 3.14159265358979f;
      for (int it = 0; it < 40; ++it) {
        const float mid = 0.5f * (lo + hi);
        mix_eval(mid, pp, K, m, g, gp, s, c);
        if (m.H < z)
          lo = mid;
        else
          hi = mid;
      }
      mix_eval(0.5f * (lo + hi), pp, K, m, g, gp, s, c);
      // implicit differentiation at the solution, as k_ncp_inverse_backward
      float dHp_dx = 0.f;
      for (int k = 0; k < K; ++k) {
        const float al = m.al[k];
        const float den = c * c + al * al * s * s;
        dHp_dx += m.w[k] * (-al * s * c * (al * al - 1.f)) / (den * den);
      }
      const float r = (gout + gl * dHp_dx / m.Hp) / m.Hp;  // dL/dz through xs
      float unused;
      mix_backward(m, g, gp, s, c, K, -r, gl / m.Hp, unused, gpo);
      gpo[2 * K] = -r;
      gP[pa] = r - gout;
    }
    for (int k = 0; k < K; ++k)
      if (fabsf(pp[k]) > 8.f) gpo[k] = 0.f;
    for (int o = 0; o < C2; ++o) gprmT[o * nact + a] = gpo[o];
  }
  __syncthreads();
  float *wp = wpart + (size_t)b * (H * 18 + H + C2 * H * 9 + C2);
  float *gW1 = wp, *gB1 = wp + H * 18, *gW2 = gB1 + H, *gB2 = gW2 + C2 * H * 9;
  for (int o = tid; o < C2; o += nt) {
    float acc = 0.f;
    for (int a = 0; a < nact; ++a) acc += gprmT[o * nact + a];
    gB2[o] = acc;
  }
  // ---- adjoint, chunk by chunk over the hidden channels
  for (int c0 = 0; c0 < H; c0 += Cc) {
    conv1_chunk(c0);
    __syncthreads();
    // dL/dpre[c][p] = LeakyReLU'(pre) * sum_k sum_o W2[o][c][k] gprm[a][o] over active a whose offset-k neighbour is p
    for (int q = tid; q < Cc * LL; q += nt) {
      const int cl = q / LL, p = q - cl * LL;
      float acc = 0.f;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int a = amap[nbt[(8 - k) * LL + p]];
        if (a >= 0) {
          const float *wr = w2t + ((c0 + cl) * 9 + k) * CP;
          for (int o = 0; o < C2; ++o) acc = fmaf(wr[o], gprmT[o * nact + a], acc);
        }
      }
      ghc[q] = hc[q] > 0.f ? acc : slope * acc;
    }
    __syncthreads();
    // Weight gradients of the chunk as warp reductions: lanes split the sum
    // (active plaquettes or pixels), each lane keeps several independent
    // accumulators, and a fixed xor-shuffle tree adds the lanes (the same
    // order every run).
    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    // gW2[o][c][k] = sum_a gprm[a][o] h[c][nbr(a, k)]: unit = (c, k, eight outputs)
    for (int u = warp; u < Cc * 9 * (CP / 8 + (CP % 8 ? 1 : 0)); u += nwarps) {
      const int n8 = CP / 8 + (CP % 8 ? 1 : 0);
      const int ck = u / n8, o0 = 8 * (u - ck * n8), cl = ck / 9, k = ck - cl * 9;
      const float *pc = hc + cl * LL;
      const int *nk = nbt + k * LL;
      float acc[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] = 0.f;
      for (int a = lane; a < nact; a += 32) {
        const float v = lrelu(pc[nk[apos[a]]], slope);
        const float *gg = gprmT + o0 * nact + a;
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (o0 + j < C2) acc[j] = fmaf(gg[j * nact], v, acc[j]);
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] = warp_sum(acc[j]);
      if (lane < 8 && o0 + lane < C2) {
        float v = acc[0];
#pragma unroll
        for (int j = 1; j < 8; ++j)
          if (lane == j) v = acc[j];
        gW2[(size_t)(o0 + lane) * H * 9 + (c0 + cl) * 9 + k] = v;
      }
    }
    // gW1[c][ci][k] = sum_p dL/dpre[c][p] ctx[ci][nbr(p, k)] and gB1[c] = sum_p dL/dpre[c][p]:
    // unit = (c, ci), nine offsets per lane
    for (int u = warp; u < Cc * 2; u += nwarps) {
      const int cl = u >> 1, ci = u & 1;
      const float *gc = ghc + cl * LL;
      const float *cx = ctx + ci * LL;
      float acc[9], accb = 0.f;
#pragma unroll
      for (int k = 0; k < 9; ++k) acc[k] = 0.f;
      for (int p = lane; p < LL; p += 32) {
        const float gv = gc[p];
        accb += gv;
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[k] = fmaf(gv, cx[nbt[k * LL + p]], acc[k]);
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) acc[k] = warp_sum(acc[k]);
      accb = warp_sum(accb);
      if (lane < 9) {
        float v = acc[0];
#pragma unroll
        for (int k = 1; k < 9; ++k)
          if (lane == k) v = acc[k];
        gW1[(c0 + cl) * 18 + ci * 9 + lane] = v;
      }
      if (ci == 0 && lane == 0) gB1[c0 + cl] = accb;
    }
    // gctx[ci][p] += sum_k sum_{c in chunk} W1[c][ci][k] dL/dpre[c][p - (k offset)]
    for (int q = tid; q < 2 * LL; q += nt) {
      const int ci = q / LL, p = q - ci * LL;
      float acc = gctx[q];
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int pq = nbt[(8 - k) * LL + p];
        const float *wr = w1t + (ci * 9 + k) * H + c0;
        for (int cl = 0; cl < Cc; ++cl) acc = fmaf(wr[cl], ghc[cl * LL + pq], acc);
      }
      gctx[q] = acc;
    }
    __syncthreads();
  }
  // context adjoint into gP (frozen plaquettes): ctx = (cos P, sin P)
  for (int p = tid; p < LL; p += nt) {
    const int xn = mu == 0 ? p / L : p % L;
    const int r = (xn - off) & 3;
    if (r == 1 || r == 2) {
      float sn, cs;
      sincosf(P[p], &sn, &cs);
      gP[p] += -sn * gctx[p] + cs * gctx[LL + p];
    }
  }
  __syncthreads();
  // plaquette adjoint: P(x) = th0(x) + th1(x+e0) - th0(x+e1) - th1(x)
  float *dst = gth_in + (size_t)b * 2 * LL;
  for (int p = tid; p < LL; p += nt) {
    const int x0 = p % L, x1 = p / L;
    const int x0m = x0 == 0 ? L - 1 : x0 - 1, x1m = x1 == 0 ? L - 1 : x1 - 1;
    dst[p] = go[p] + gP[p] - gP[x1m * L + x0];
    dst[LL + p] = go[LL + p] + gP[x1 * L + x0m] - gP[p];
  }
}

// out[j] = sum over blocks b (in order) of wpart[b][j].
__global__ void k_flow_wgrad_reduce(const float *__restrict__ wpart, int nb, int nw, float *__restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nw) return;
  float acc = 0.f;
  for (int b = 0; b < nb; ++b) acc += wpart[(size_t)b * nw + j];
  out[j] = acc;
}

int flow_chunk(int H) { return H % 8 == 0 ? 8 : 4; }

size_t flow_layer_bwd_smem(int L, int K, int H) {
  const size_t LL = (size_t)L * L, CP = (2 * K + 1 + 3) & ~3, nact = LL / 4, Cc = flow_chunk(H);
  return sizeof(float) * (2 * LL + LL + 2 * LL + 18 * H + H + 9 * H * CP + CP + 2 * nact * CP + 2 * LL + LL +
                          2 * Cc * LL) +
         sizeof(int) * (LL + nact + 9 * LL);
}

size_t flow_layer_smem(int L, int K, int H) {
  const size_t LL = (size_t)L * L, CP = (2 * K + 1 + 3) & ~3;
  return sizeof(float) * (2 * LL + LL + 2 * LL + H * LL + 18 * H + H + 9 * H * CP + CP + (LL / 4) * CP);
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

namespace {
template <bool INV>
int flow_layer_fwd(const char *name, const float *theta_in, float *theta_out, float *logdet, int batch, int L, int mu,
                   int off, int K, int hidden, const float *W1, const float *B1, const float *W2, const float *B2,
                   float slope, void *stream) {
  if (!theta_in || !theta_out || !logdet || !W1 || !B1 || !W2 || !B2)
    return flfail(U1_ERR_INVALID, std::string(name) + ": null pointer");
  if (theta_in == theta_out) return flfail(U1_ERR_INVALID, std::string(name) + ": in and out must not alias");
  if (batch < 1 || L < 4 || L > 32 || L % 4 || (mu != 0 && mu != 1) || off < 0 || off > 3 || K < 1 || K > kMaxK ||
      hidden < 4 || hidden > 32 || hidden % 4)
    return flfail(U1_ERR_INVALID, std::string(name) +
                                      ": bad shape (L a multiple of 4 up to 32, K <= 8, hidden a multiple of 4 up to 32)");
  const size_t smem = flow_layer_smem(L, K, hidden);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_flow_layer_forward<INV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return u1i::cuda_fail(e, name);
  }
  k_flow_layer_forward<INV><<<batch, kFlowThreads, smem, (cudaStream_t)stream>>>(theta_in, theta_out, logdet, L, mu, off, K,
                                                                         hidden, W1, B1, W2, B2, slope);
  U1_LAUNCH_CHECK(name);
  return U1_OK;
}

template <bool INV>
int flow_layer_bwd(const char *name, const float *theta_in, const float *grad_theta_out, const float *grad_logdet,
                   float *grad_theta_in, float *wgrad_partials, float *wgrad, int batch, int L, int mu, int off, int K,
                   int hidden, const float *W1, const float *B1, const float *W2, const float *B2, float slope,
                   void *stream) {
  if (!theta_in || !grad_theta_out || !grad_theta_in || !wgrad_partials || !wgrad || !W1 || !B1 || !W2 || !B2)
    return flfail(U1_ERR_INVALID, std::string(name) + ": null pointer");
  if (batch < 1 || L < 4 || L > 32 || L % 4 || (mu != 0 && mu != 1) || off < 0 || off > 3 || K < 1 ||
      K > kMaxK || hidden < 4 || hidden > 32 || hidden % 4)
    return flfail(U1_ERR_INVALID, std::string(name) +
                                      ": bad shape (L a multiple of 4 up to 32, K <= 8, hidden a multiple of 4 up to 32)");
  const size_t smem = flow_layer_bwd_smem(L, K, hidden);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_flow_layer_backward<INV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return u1i::cuda_fail(e, name);
  }
  cudaStream_t s = (cudaStream_t)stream;
  k_flow_layer_backward<INV><<<batch, kFlowThreads, smem, s>>>(theta_in, grad_theta_out, grad_logdet, grad_theta_in,
                                                       wgrad_partials, L, mu, off, K, hidden, flow_chunk(hidden), W1,
                                                       B1, W2, B2, slope);
  U1_LAUNCH_CHECK(name);
  const int nw = hidden * 18 + hidden + (2 * K + 1) * hidden * 9 + (2 * K + 1);
  k_flow_wgrad_reduce<<<(nw + 255) / 256, 256, 0, s>>>(wgrad_partials, batch, nw, wgrad);
  U1_LAUNCH_CHECK("k_flow_wgrad_reduce");
  return U1_OK;
}
}  // namespace

extern "C" int u1_flow_layer_forward(const float *theta_in, float *theta_out, float *logdet, int batch, int L,
                                     int mu, int off, int K, int hidden, const float *W1, const float *B1,
                                     const float *W2, const float *B2, float slope, void *stream) {
  return flow_layer_fwd<false>("u1_flow_layer_forward", theta_in, theta_out, logdet, batch, L, mu, off, K, hidden,
                               W1, B1, W2, B2, slope, stream);
}

extern "C" int u1_flow_layer_inverse(const float *theta_in, float *theta_out, float *logdet, int batch, int L,
                                     int mu, int off, int K, int hidden, const float *W1, const float *B1,
                                     const float *W2, const float *B2, float slope, void *stream) {
  return flow_layer_fwd<true>("u1_flow_layer_inverse", theta_in, theta_out, logdet, batch, L, mu, off, K, hidden, W1,
                              B1, W2, B2, slope, stream);
}

extern "C" int u1_flow_layer_backward(const float *theta_in, const float *grad_theta_out, const float *grad_logdet,
                                      float *grad_theta_in, float *wgrad_partials, float *wgrad, int batch, int L,
                                      int mu, int off, int K, int hidden, const float *W1, const float *B1,
                                      const float *W2, const float *B2, float slope, void *stream) {
  return flow_layer_bwd<false>("u1_flow_layer_backward", theta_in, grad_theta_out, grad_logdet, grad_theta_in,
                               wgrad_partials, wgrad, batch, L, mu, off, K, hidden, W1, B1, W2, B2, slope, stream);
}

extern "C" int u1_flow_layer_inverse_backward(const float *theta_in, const float *grad_theta_out,
                                              const float *grad_logdet, float *grad_theta_in, float *wgrad_partials,
                                              float *wgrad, int batch, int L, int mu, int off, int K, int hidden,
                                              const float *W1, const float *B1, const float *W2, const float *B2,
                                              float slope, void *stream) {
  return flow_layer_bwd<true>("u1_flow_layer_inverse_backward", theta_in, grad_theta_out, grad_logdet, grad_theta_in,
                              wgrad_partials, wgrad, batch, L, mu, off, K, hidden, W1, B1, W2, B2, slope, stream);
}
