// Data formats around the update path:
//  * u1_convert_order: even/odd <-> natural (lexicographic) order of FP64
//    angle arrays (replaces ConvLattice_EO_NO, reference src/convertOrder.cu:
//    32-63);
//  * u1_plaquette_fields: the six per-site plaquette components 1 - e^{i theta_P}
//    and their means (replaces PlaquetteFields, reference
//    src/plaquette_comps.cu:34-107 and :220-235);
//  * configuration checkpoints (the reference has none): the reference's
//    FP64 angle layout plus the Philox state, and optionally the exact
//    float2 links so that a resumed chain is bit-identical.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "u1_internal.h"
#include "u1_measure.cuh"

using namespace u1b;

namespace {

int ffail(int code, const std::string &msg) {
  u1i::set_error(msg);
  return code;
}

int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

// ------------------------------------------------------------ order converter
// Natural order: theta_no[lex(x) + mu*V], lex(x) = x0 + N0 (x1 + N1 (x2 + N2 x3)).
// Even/odd order: theta_eo[eo(x) + parity(x) V/2 + mu*V], eo(x) = lex(x) >> 1.
template <bool EO_TO_NO>
__global__ void k_convert_order(const double *__restrict__ in, double *__restrict__ out, GeomK g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V) return;
  int x[4], k;
  if (EO_TO_NO) {  // t = eo + parity * V/2
    const int p = t >= g.Vh ? 1 : 0;
    eo_decode_fast<4>(g, t - p * g.Vh, p, x, k);
    const int lex = x[0] + g.N[0] * (x[1] + g.N[1] * (x[2] + g.N[2] * x[3]));
    for (int mu = 0; mu < g.dims; ++mu) out[(size_t)mu * g.V + lex] = in[(size_t)mu * g.V + t];
  } else {  // t = lex
    int r = t;
    x[0] = r % g.N[0];
    r /= g.N[0];
    x[1] = r % g.N[1];
    r /= g.N[1];
    x[2] = r % g.N[2];
    x[3] = r / g.N[2];
    const int p = (x[0] + x[1] + x[2] + x[3]) & 1;
    const int dst = (t >> 1) + p * g.Vh;
    for (int mu = 0; mu < g.dims; ++mu) out[(size_t)mu * g.V + dst] = in[(size_t)mu * g.V + t];
  }
}

// --------------------------------------------------------- plaquette fields
// Components d = 0..5 are (mu, nu) = (0,3), (1,3), (2,3), (1,2), (2,0), (0,1)
// (reference include/lattice_functions.h:38-45); value 1 - e^{i theta_{mu nu}(x)}.
__device__ __forceinline__ float2 plaq_one_minus(const float2 *__restrict__ lat, const GeomK &g, int i, int p,
                                                 int mu, int nu, const int fwd[4]) {
  const int q = 1 - p;
  const float2 umu = __ldg(lat + mu * g.V + p * g.Vh + i);
  const float2 a = __ldg(lat + nu * g.V + q * g.Vh + i + fwd[mu]);  // U_nu(x+mu)
  const float2 b = __ldg(lat + mu * g.V + q * g.Vh + i + fwd[nu]);  // U_mu(x+nu)
  const float2 unu = __ldg(lat + nu * g.V + p * g.Vh + i);
  const float2 P = cmulc(cmulc(cmul(umu, a), b), unu);
  return make_float2(1.f - P.x, -P.y);
}

__device__ __forceinline__ void six_plaquettes(const float2 *__restrict__ lat, const GeomK &g, int i, int p,
                                               float2 (&c)[6]) {
  int x[4], k;
  eo_decode_fast<4>(g, i, p, x, k);
  int fwd[4], bwd[4];
  eo_steps<4>(g, x, k, fwd, bwd);
  const int mus[6] = {0, 1, 2, 1, 2, 0}, nus[6] = {3, 3, 3, 2, 0, 1};
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    const float2 v = plaq_one_minus(lat, g, i, p, mus[d], nus[d], fwd);
    c[d].x += v.x;
    c[d].y += v.y;
  }
}

// spacetime: thread per site (EO t), field[lex(x) + d V] (complex FP64).
// otherwise: thread per spatial site, time average, field[lex_s(x) + d V_s].
// partials[block*12 + 2d + {re, im}] = block sums of the written values.
template <bool SPACETIME>
__global__ void __launch_bounds__(kRedThreads)
    k_plaquette_fields(const float2 *__restrict__ lat, GeomK g, double2 *__restrict__ field, double *partials) {
  __shared__ double smem[kRedWarps * 12];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double v[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) v[k] = 0.0;
  // Thread t owns natural-order site t (spacetime) or spatial site t (time
  // averages), so a warp writes 32 consecutive FP64 complex values of each
  // component (coalesced) and reads the links of both parities in two
  // contiguous runs.
  if (SPACETIME) {
    if (t < g.V) {
      int x[4];
      int r = t;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        x[k] = r % g.N[k];
        r /= g.N[k];
      }
      const int p = (x[0] + x[1] + x[2] + x[3]) & 1;
      float2 c[6];
#pragma unroll
      for (int d = 0; d < 6; ++d) c[d] = make_float2(0.f, 0.f);
      six_plaquettes(lat, g, eo_index(g, x), p, c);
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        field[(size_t)d * g.V + t] = make_double2(c[d].x, c[d].y);
        v[2 * d] = c[d].x;
        v[2 * d + 1] = c[d].y;
      }
    }
  } else if (t < g.Vs) {
    int x[4];
    x[0] = t % g.N[0];
    x[1] = (t / g.N[0]) % g.N[1];
    x[2] = t / (g.N[0] * g.N[1]);
    x[3] = 0;
    const int p0 = (x[0] + x[1] + x[2]) & 1;
    const int i0 = eo_index(g, x);  // the site on the t = 0 slice; (x, tt) is i0 + tt * es[3]
    float2 c[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) c[d] = make_float2(0.f, 0.f);
    for (int tt = 0; tt < g.N[3]; ++tt) six_plaquettes(lat, g, i0 + tt * g.es[3], (p0 + tt) & 1, c);
    const double inv = 1.0 / g.N[3];
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      const double2 m = make_double2(c[d].x * inv, c[d].y * inv);
      field[(size_t)d * g.Vs + t] = m;
      v[2 * d] = m.x;
      v[2 * d + 1] = m.y;
    }
  }
  block_sum<12>(v, smem);
  if (threadIdx.x < 12) partials[(size_t)blockIdx.x * 12 + threadIdx.x] = v[0];
}

__global__ void __launch_bounds__(kRedThreads)
    k_plaquette_fields_finish(const double *__restrict__ partials, int nb, double norm, double *out) {
  __shared__ double smem[kRedWarps * 12];
  double w[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) w[k] = strided_partial_sum(partials, nb, 12, k);
  block_sum<12>(w, smem);
  if (threadIdx.x < 12) out[threadIdx.x] = w[0] * norm;
}

// ---------------------------------------------------------------- checkpoint
// File layout (little endian):
//   [0, 128)  header: magic "U1B200CK", u32 version = 1, u32 header bytes = 128,
//             i32 dims, i32 Grid[4], u32 0, f64 beta, f64 aniso, u64 seed, u64 pass,
//             u32 chain, u32 flags (bit 0: exact float2 section present),
//             u64 nlinks, u32 crc32(angles), u32 crc32(float2 section), zero padding
//   then      nlinks f64 angles in [0, 2pi), theta[eo + parity V/2 + mu V]
//   then      (flag bit 0) nlinks float2 (cos, sin) links, the same order.
struct CkptHeader {
  char magic[8];
  uint32_t version;
  uint32_t header_bytes;
  int32_t dims;
  int32_t grid[4];
  uint32_t reserved;  // 0; keeps the doubles 8-byte aligned
  double beta;
  double aniso;
  uint64_t seed;
  uint64_t pass;
  uint32_t chain;
  uint32_t flags;
  uint64_t nlinks;
  uint32_t crc_angles;
  uint32_t crc_links;
  char pad[32];
};
static_assert(sizeof(CkptHeader) == 128, "checkpoint header is 128 bytes");
constexpr char kMagic[8] = {'U', '1', 'B', '2', '0', '0', 'C', 'K'};

// CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320), table driven.
struct Crc32Table {
  uint32_t t[256];
  Crc32Table() {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1u) ? (0xEDB88320u ^ (c >> 1)) : (c >> 1);
      t[i] = c;
    }
  }
};

uint32_t crc32_update(uint32_t crc, const void *data, size_t n) {
  static const Crc32Table tab;  // thread-safe one-time initialisation
  const uint32_t *table = tab.t;
  const unsigned char *p = static_cast<const unsigned char *>(data);
  crc = ~crc;
  for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
  return ~crc;
}

int read_header(const char *path, CkptHeader &h, FILE **fp_out) {
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return ffail(U1_ERR_INVALID, std::string("checkpoint: cannot open ") + path);
  if (std::fread(&h, sizeof(h), 1, fp) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != 1 ||
      h.header_bytes != sizeof(CkptHeader)) {
    std::fclose(fp);
    return ffail(U1_ERR_INVALID, std::string("checkpoint: not a version-1 checkpoint: ") + path);
  }
  if (fp_out)
    *fp_out = fp;
  else
    std::fclose(fp);
  return U1_OK;
}

}  // namespace

extern "C" int u1_convert_order(const u1_geom *geom, const double *in_dev, double *out_dev, int eo_to_no,
                                void *stream) {
  if (!geom || !in_dev || !out_dev) return ffail(U1_ERR_INVALID, "u1_convert_order: null argument");
  if (in_dev == out_dev) return ffail(U1_ERR_INVALID, "u1_convert_order: in and out must not alias");
  GeomK g{};
  int rc = u1i::make_geom(geom, g);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (eo_to_no)
    k_convert_order<true><<<nblk(g.V, 256), 256, 0, s>>>(in_dev, out_dev, g);
  else
    k_convert_order<false><<<nblk(g.V, 256), 256, 0, s>>>(in_dev, out_dev, g);
  U1_LAUNCH_CHECK("k_convert_order");
  return U1_OK;
}

extern "C" int u1_plaquette_fields(u1_lattice *lat, int spacetime, double *field_dev, double means[12]) {
  if (!lat || !field_dev || !means) return ffail(U1_ERR_INVALID, "u1_plaquette_fields: null argument");
  if (lat->g.dims != 4)
    return ffail(U1_ERR_UNSUPPORTED, "u1_plaquette_fields: only 4D lattices (as the reference)");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  const GeomK &g = lat->g;
  const int n = spacetime ? g.V : g.Vs;
  const int nb = nblk(n, kRedThreads);
  int rc = u1i::ensure_scratch(lat, (size_t)nb * 12, 12);
  if (rc) return rc;
  double2 *field = reinterpret_cast<double2 *>(field_dev);
  if (spacetime)
    k_plaquette_fields<true><<<nb, kRedThreads, 0, lat->stream>>>(lat->links, g, field, lat->partials);
  else
    k_plaquette_fields<false><<<nb, kRedThreads, 0, lat->stream>>>(lat->links, g, field, lat->partials);
  U1_LAUNCH_CHECK("k_plaquette_fields");
  k_plaquette_fields_finish<<<1, kRedThreads, 0, lat->stream>>>(lat->partials, nb, 1.0 / n, lat->d_out);
  U1_LAUNCH_CHECK("k_plaquette_fields_finish");
  U1_CUDA_TRY(cudaMemcpyAsync(lat->h_out, lat->d_out, 12 * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
  std::memcpy(means, lat->h_out, 12 * sizeof(double));
  return U1_OK;
}

extern "C" int u1_checkpoint_save(u1_lattice *lat, const u1_rng *rng, const char *path, int exact) {
  if (!lat || !path) return ffail(U1_ERR_INVALID, "u1_checkpoint_save: null argument");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  const size_t n = (size_t)lat->g.V * lat->g.dims;
  std::vector<double> ang(n);
  int rc = u1_lattice_export_angles(lat, ang.data(), 0);
  if (rc) return rc;
  std::vector<float2> links;
  if (exact) {
    links.resize(n);
    U1_CUDA_TRY(cudaMemcpyAsync(links.data(), lat->links, n * sizeof(float2), cudaMemcpyDeviceToHost, lat->stream));
    U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
  }
  CkptHeader h{};
  std::memcpy(h.magic, kMagic, 8);
  h.version = 1;
  h.header_bytes = sizeof(CkptHeader);
  h.dims = lat->g.dims;
  for (int k = 0; k < 4; ++k) h.grid[k] = lat->g.N[k];
  h.beta = lat->beta;
  h.aniso = lat->aniso;
  h.seed = rng ? rng->seed : 0;
  h.pass = rng ? rng->pass : 0;
  h.chain = rng ? rng->chain : 0;
  h.flags = exact ? 1u : 0u;
  h.nlinks = n;
  h.crc_angles = crc32_update(0, ang.data(), n * sizeof(double));
  h.crc_links = exact ? crc32_update(0, links.data(), n * sizeof(float2)) : 0u;
  const std::string tmp = std::string(path) + ".tmp";
  FILE *fp = std::fopen(tmp.c_str(), "wb");
  if (!fp) return ffail(U1_ERR_INVALID, std::string("u1_checkpoint_save: cannot write ") + tmp);
  bool ok = std::fwrite(&h, sizeof(h), 1, fp) == 1 && std::fwrite(ang.data(), sizeof(double), n, fp) == n;
  if (ok && exact) ok = std::fwrite(links.data(), sizeof(float2), n, fp) == n;
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    return ffail(U1_ERR_INVALID, std::string("u1_checkpoint_save: write failed for ") + path);
  }
  return U1_OK;
}

extern "C" int u1_checkpoint_info(const char *path, u1_geom *geom, uint64_t *seed, uint64_t *pass, uint32_t *chain,
                                  uint32_t *flags) {
  if (!path) return ffail(U1_ERR_INVALID, "u1_checkpoint_info: null path");
  CkptHeader h{};
  int rc = read_header(path, h, nullptr);
  if (rc) return rc;
  if (geom) {
    // back to the ABI's (Nx, Ny, Nz, Nt) convention
    geom->dims = h.dims;
    geom->N[0] = h.grid[0];
    geom->N[1] = h.dims == 2 ? 0 : h.grid[1];
    geom->N[2] = h.dims == 4 ? h.grid[2] : 0;
    geom->N[3] = h.grid[h.dims - 1];
    geom->beta = h.beta;
    geom->aniso = h.aniso;
  }
  if (seed) *seed = h.seed;
  if (pass) *pass = h.pass;
  if (chain) *chain = h.chain;
  if (flags) *flags = h.flags;
  return U1_OK;
}

extern "C" int u1_checkpoint_load(u1_lattice *lat, u1_rng *rng, const char *path) {
  if (!lat || !path) return ffail(U1_ERR_INVALID, "u1_checkpoint_load: null argument");
  CkptHeader h{};
  FILE *fp = nullptr;
  int rc = read_header(path, h, &fp);
  if (rc) return rc;
  bool same = h.dims == lat->g.dims;
  for (int k = 0; k < 4; ++k) same = same && h.grid[k] == lat->g.N[k];
  const size_t n = (size_t)lat->g.V * lat->g.dims;
  if (!same || h.nlinks != n) {
    std::fclose(fp);
    return ffail(U1_ERR_INVALID, "u1_checkpoint_load: geometry differs from the lattice's");
  }
  std::vector<double> ang(n);
  bool ok = std::fread(ang.data(), sizeof(double), n, fp) == n;
  std::vector<float2> links;
  if (ok && (h.flags & 1u)) {
    links.resize(n);
    ok = std::fread(links.data(), sizeof(float2), n, fp) == n;
  }
  std::fclose(fp);
  if (!ok) return ffail(U1_ERR_INVALID, "u1_checkpoint_load: truncated file");
  if (crc32_update(0, ang.data(), n * sizeof(double)) != h.crc_angles ||
      ((h.flags & 1u) && crc32_update(0, links.data(), n * sizeof(float2)) != h.crc_links))
    return ffail(U1_ERR_INVALID, "u1_checkpoint_load: checksum mismatch");
  U1_CUDA_TRY(cudaSetDevice(lat->ctx->device));
  if (h.flags & 1u) {
    U1_CUDA_TRY(cudaMemcpyAsync(lat->links, links.data(), n * sizeof(float2), cudaMemcpyHostToDevice, lat->stream));
    U1_CUDA_TRY(cudaStreamSynchronize(lat->stream));
  } else {
    rc = u1_lattice_import_angles(lat, ang.data(), 0);
    if (rc) return rc;
  }
  if (h.beta != lat->beta || h.aniso != lat->aniso) {
    rc = u1_lattice_set_coupling(lat, h.beta, h.aniso);
    if (rc) return rc;
  }
  if (rng) {
    rc = u1_rng_set_state(rng, h.seed, h.pass);
    if (rc) return rc;
    rc = u1_rng_set_chain(rng, h.chain);
    if (rc) return rc;
  }
  return U1_OK;
}
