// Differentiable Wilson action: S(theta) and its adjoint dS/dtheta, batched,
// in FP32 or FP64, on caller-owned device buffers.
//
//   S = beta * sum_x sum_{mu<nu} w_{mu nu} (1 - cos theta_P(x)),
//   theta_P(x) = theta_mu(x) + theta_nu(x+mu) - theta_mu(x+nu) - theta_nu(x),
//   w = 1/xi for spatial-spatial plaquettes and xi when mu or nu is the time
//   direction (the staple weights of the reference, include/staple.h:75-102).
// Its gradient is the reference's local action turned into a derivative:
//   dS/dtheta_mu(x) = beta sum_{nu != mu} w_{mu nu} [sin theta_{mu nu}(x) - sin theta_{mu nu}(x - nu)]
//                   = beta Im(S_mu(x) U_mu(x))  (S the weighted staple).
// The reference has no action or gradient routine; the per-plaquette angle is
// the one its plaquette kernel sums (src/plaquette.cu:93-118).
//
// Layout: theta[b][mu*V + parity*V/2 + eo] (the reference's angle layout per
// configuration b).  Reductions are deterministic: per-block FP64 partials
// (written to a caller workspace) summed in block order by one CTA per
// configuration.  Nothing here allocates device memory.
#include <string>

#include "u1_internal.h"
#include "u1_measure.cuh"

using namespace u1b;

namespace {

constexpr int kActThreads = 256;

template <typename T>
__device__ __forceinline__ T dcos(T x);
template <>
__device__ __forceinline__ float dcos(float x) {
  return cosf(x);
}
template <>
__device__ __forceinline__ double dcos(double x) {
  return cos(x);
}
template <typename T>
__device__ __forceinline__ T dsin(T x);
template <>
__device__ __forceinline__ float dsin(float x) {
  return sinf(x);
}
template <>
__device__ __forceinline__ double dsin(double x) {
  return sin(x);
}
template <typename T>
__device__ __forceinline__ T dremainder_2pi(T x);
template <>
__device__ __forceinline__ float dremainder_2pi(float x) {
  return remainderf(x, 6.28318530717958647692f);
}
template <>
__device__ __forceinline__ double dremainder_2pi(double x) {
  return remainder(x, 6.28318530717958647692);
}

// Thread per site (t < V: parity t >= V/2).  partials[(b*nb + block)*2 + {0,1}]
// = block sums of w (1 - cos theta_P) and, in 2D, of wrap(theta_P) to (-pi, pi].
template <int D, typename T>
__global__ void __launch_bounds__(kActThreads)
    k_action(const T *__restrict__ theta, GeomK g, T w_ss, T w_st, double *partials) {
  __shared__ double smem[kRedWarps * 2];
  const int b = blockIdx.y;
  const T *th = theta + (size_t)b * g.V * D;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  T acc = 0, qacc = 0;
  if (t < g.V) {
    const int p = t >= g.Vh ? 1 : 0;
    const int i = t - p * g.Vh;
    const int q = 1 - p;
    int x[4], k;
    eo_decode_fast<D>(g, i, p, x, k);
    int fwd[4], bwd[4];
    eo_steps<D>(g, x, k, fwd, bwd);
#pragma unroll
    for (int mu = 0; mu < D - 1; ++mu)
#pragma unroll
      for (int nu = mu + 1; nu < D; ++nu) {
        const T thp = th[mu * g.V + p * g.Vh + i] + th[nu * g.V + q * g.Vh + i + fwd[mu]] -
                      th[mu * g.V + q * g.Vh + i + fwd[nu]] - th[nu * g.V + p * g.Vh + i];
        acc += (nu == D - 1 ? w_st : w_ss) * (T(1) - dcos(thp));
        if (D == 2) qacc += dremainder_2pi(thp);
      }
  }
  double v[2] = {(double)acc, (double)qacc};
  block_sum<2>(v, smem);
  if (threadIdx.x < 2) partials[((size_t)b * gridDim.x + blockIdx.x) * 2 + threadIdx.x] = v[0];
}

// One CTA per configuration: out[b*2] = beta * S_sum, out[b*2+1] = Q.
__global__ void __launch_bounds__(kRedThreads)
    k_action_finish(const double *__restrict__ partials, int nb, double beta, double *out) {
  __shared__ double smem[kRedWarps * 2];
  const int b = blockIdx.x;
  double w[2] = {strided_partial_sum(partials + (size_t)b * nb * 2, nb, 2, 0),
                 strided_partial_sum(partials + (size_t)b * nb * 2, nb, 2, 1)};
  block_sum<2>(w, smem);
  if (threadIdx.x == 0) out[b * 2] = beta * w[0];
  if (threadIdx.x == 1) out[b * 2 + 1] = w[0] * 0.15915494309189533577;  // 1/(2 pi)
}

// Thread per site r = parity*V/2 + eo, computing the gradients of its d
// links (x, mu):
//   grad = scale * beta * sum_{nu != mu} w [sin theta_{mu nu}(x) - sin theta_{mu nu}(x - nu)].
// Each forward plaquette theta_{mu nu}(x), mu < nu, is evaluated once and
// enters link (x, mu) with + and link (x, nu) with - (theta_{nu mu} =
// -theta_{mu nu}); the backward plaquettes theta_{mu nu}(x - nu) are per
// link.  d(d-1)/2 + d(d-1) sines per site instead of 2(d-1) per link.
template <int D, typename T>
__global__ void __launch_bounds__(kActThreads)
    k_action_grad(const T *__restrict__ theta, GeomK g, T beta, T w_ss, T w_st, const double *__restrict__ scale,
                  T *__restrict__ grad) {
  const int b = blockIdx.y;
  const size_t n = (size_t)g.V * D;
  const T *th = theta + (size_t)b * n;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= g.V) return;
  const int p = r >= g.Vh ? 1 : 0;
  const int i = r - p * g.Vh;
  const int q = 1 - p;
  int x[4], k;
  eo_decode_fast<D>(g, i, p, x, k);
  int fwd[4], bwd[4];
  eo_steps<D>(g, x, k, fwd, bwd);
  T own[D], acc[D];
#pragma unroll
  for (int mu = 0; mu < D; ++mu) {
    own[mu] = th[mu * g.V + p * g.Vh + i];
    acc[mu] = 0;
  }
#pragma unroll
  for (int mu = 0; mu < D; ++mu) {
#pragma unroll
    for (int nu = 0; nu < D; ++nu) {
      if (nu == mu) continue;
      const T w = (mu == D - 1 || nu == D - 1) ? w_st : w_ss;
      if (mu < nu) {
        // theta_{mu nu}(x) = theta_mu(x) + theta_nu(x+mu) - theta_mu(x+nu) - theta_nu(x)
        const T a = th[nu * g.V + q * g.Vh + i + fwd[mu]];
        const T bb = th[mu * g.V + q * g.Vh + i + fwd[nu]];
        const T sf = w * dsin(own[mu] + a - bb - own[nu]);
        acc[mu] += sf;
        acc[nu] -= sf;
      }
      // theta_{mu nu}(x-nu) = theta_mu(x-nu) + theta_nu(x-nu+mu) - theta_mu(x) - theta_nu(x-nu)
      const T d = th[mu * g.V + q * g.Vh + i + bwd[nu]];
      const T e = th[nu * g.V + p * g.Vh + i + fwd[mu] + bwd[nu]];
      const T f = th[nu * g.V + q * g.Vh + i + bwd[nu]];
      acc[mu] -= w * dsin(d + e - own[mu] - f);
    }
  }
  const T sc = scale ? (T)scale[b] : T(1);
#pragma unroll
  for (int mu = 0; mu < D; ++mu) grad[(size_t)b * n + mu * g.V + p * g.Vh + i] = sc * beta * acc[mu];
}

int afail(int code, const std::string &msg) {
  u1i::set_error(msg);
  return code;
}

int action_args(const u1_geom *geom, int dtype, int batch, GeomK &g) {
  if (!geom) return afail(U1_ERR_INVALID, "action: null geometry");
  if (dtype != 0 && dtype != 1) return afail(U1_ERR_INVALID, "action: dtype must be 0 (f32) or 1 (f64)");
  if (batch < 1 || batch > 65535) return afail(U1_ERR_INVALID, "action: batch must be in [1, 65535]");
  int rc = u1i::make_geom(geom, g);
  if (rc) return rc;
  if (!(geom->aniso > 0.0)) return afail(U1_ERR_INVALID, "action: aniso must be > 0");
  return U1_OK;
}

int action_blocks(const GeomK &g) { return (g.V + kActThreads - 1) / kActThreads; }

template <int D, typename T>
int launch_action(const GeomK &g, const u1_geom *geom, const void *theta, int batch, double *ws, double *out,
                  cudaStream_t s) {
  const int nb = action_blocks(g);
  const T w_ss = (T)(1.0 / geom->aniso), w_st = (T)geom->aniso;
  k_action<D, T><<<dim3(nb, batch), kActThreads, 0, s>>>(static_cast<const T *>(theta), g, w_ss, w_st, ws);
  U1_LAUNCH_CHECK("k_action");
  k_action_finish<<<batch, kRedThreads, 0, s>>>(ws, nb, geom->beta, out);
  U1_LAUNCH_CHECK("k_action_finish");
  return U1_OK;
}

template <int D, typename T>
int launch_grad(const GeomK &g, const u1_geom *geom, const void *theta, int batch, const double *scale, void *grad,
                cudaStream_t s) {
  const int nb = (int)(((long long)g.V + kActThreads - 1) / kActThreads);  // one thread per site
  k_action_grad<D, T><<<dim3(nb, batch), kActThreads, 0, s>>>(static_cast<const T *>(theta), g, (T)geom->beta,
                                                              (T)(1.0 / geom->aniso), (T)geom->aniso, scale,
                                                              static_cast<T *>(grad));
  U1_LAUNCH_CHECK("k_action_grad");
  return U1_OK;
}

}  // namespace

extern "C" int u1_action_workspace_bytes(const u1_geom *geom, int batch, size_t *bytes) {
  GeomK g{};
  int rc = action_args(geom, 0, batch, g);
  if (rc) return rc;
  if (!bytes) return afail(U1_ERR_INVALID, "u1_action_workspace_bytes: null out");
  *bytes = (size_t)batch * action_blocks(g) * 2 * sizeof(double);
  return U1_OK;
}

extern "C" int u1_wilson_action(const u1_geom *geom, const void *theta_dev, int dtype, int batch, void *workspace,
                                double *out_dev, void *stream) {
  GeomK g{};
  int rc = action_args(geom, dtype, batch, g);
  if (rc) return rc;
  if (!theta_dev || !workspace || !out_dev) return afail(U1_ERR_INVALID, "u1_wilson_action: null pointer");
  double *ws = static_cast<double *>(workspace);
  cudaStream_t s = (cudaStream_t)stream;
  switch (g.dims * 2 + dtype) {
    case 4: return launch_action<2, float>(g, geom, theta_dev, batch, ws, out_dev, s);
    case 5: return launch_action<2, double>(g, geom, theta_dev, batch, ws, out_dev, s);
    case 6: return launch_action<3, float>(g, geom, theta_dev, batch, ws, out_dev, s);
    case 7: return launch_action<3, double>(g, geom, theta_dev, batch, ws, out_dev, s);
    case 8: return launch_action<4, float>(g, geom, theta_dev, batch, ws, out_dev, s);
    default: return launch_action<4, double>(g, geom, theta_dev, batch, ws, out_dev, s);
  }
}

extern "C" int u1_wilson_action_grad(const u1_geom *geom, const void *theta_dev, int dtype, int batch,
                                     const double *scale_dev, void *grad_dev, void *stream) {
  GeomK g{};
  int rc = action_args(geom, dtype, batch, g);
  if (rc) return rc;
  if (!theta_dev || !grad_dev) return afail(U1_ERR_INVALID, "u1_wilson_action_grad: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  switch (g.dims * 2 + dtype) {
    case 4: return launch_grad<2, float>(g, geom, theta_dev, batch, scale_dev, grad_dev, s);
    case 5: return launch_grad<2, double>(g, geom, theta_dev, batch, scale_dev, grad_dev, s);
    case 6: return launch_grad<3, float>(g, geom, theta_dev, batch, scale_dev, grad_dev, s);
    case 7: return launch_grad<3, double>(g, geom, theta_dev, batch, scale_dev, grad_dev, s);
    case 8: return launch_grad<4, float>(g, geom, theta_dev, batch, scale_dev, grad_dev, s);
    default: return launch_grad<4, double>(g, geom, theta_dev, batch, scale_dev, grad_dev, s);
  }
}
