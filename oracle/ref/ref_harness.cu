// ref_harness.cu -- extern "C" entry points into the REFERENCE's own code,
// compiled against the reference's headers and linked with the reference's
// sources (built in place by oracle/Makefile into oracle/_ref/libu1ref.so).
//
// TEST INFRASTRUCTURE ONLY: used by tests/ (parity pinning of the oracle and
// of the sm_100a kernels), by tests/golden/make_golden.py, and by bench.py's
// reference / cpu_baseline legs.  Nothing in latticeu1_b200 links it.
//
// CPU side: the reference's FP64 metropolis/overrelaxation
// (src/update.cu:51-98), plaquette (src/plaquette.cu:32-57), polyakov
// (src/polyakov.cu:33-49), staple/MultiHit/indexing (include/staple.h,
// include/lattice_functions.h, include/index.h).  PARAMS::* is filled
// directly, mirroring SetupLatticeParameters (src/parameters.cu:146-208),
// because that function also writes __constant__ memory (needs a GPU).
// GPU side (B200 box only): UpdateLattice, Plaquette, Polyakov, Poly2,
// MultiLevelField, LatticeConvert and PlaquetteFields through the
// reference's public API.
#include <omp.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>

// Same include order as the reference driver (u1.cpp:9-23): complex.h
// defines macros that array.h relies on.
#include "timer.h"
#include "alloc.h"
#include "complex.h"
#include "parameters.h"
#include "random.h"
#include "update.h"
#include "plaquette.h"
#include "polyakov.h"
#include "multilevel.h"
#include "array.h"
#include "cuda_error_check.h"
#include "index.h"
#include "staple.h"
#include "lattice_functions.h"

namespace U1 {
void metropolis(double *lat);       // src/update.cu:51
void overrelaxation(double *lat);   // src/update.cu:84
// src/convertOrder.cu:135-145 (defined there, declared in no header)
Array<double> *LatticeConvert(Array<double> *lat, bool eo_to_no);
}  // namespace U1

using namespace U1;

extern "C" {

int ref_setup_host(int dims, int Nx, int Ny, int Nz, int Nt, double beta, double aniso, int metrop, int ovrn) {
  PARAMS::DIRS = dims;
  PARAMS::TDir = dims - 1;
  for (int i = 0; i < 4; ++i) {
    PARAMS::Grid[i] = 1;
    PARAMS::Offset[i] = 0;
  }
  PARAMS::Grid[0] = Nx;
  if (dims == 2) PARAMS::Grid[1] = Nt;
  else if (dims > 2) PARAMS::Grid[1] = Ny;
  if (dims == 3) PARAMS::Grid[2] = Nt;
  else if (dims > 3) PARAMS::Grid[2] = Nz;
  if (dims == 4) PARAMS::Grid[3] = Nt;
  for (int i = 0; i < dims; ++i)
    if (PARAMS::Grid[i] % 2) return -1;
  PARAMS::Offset[0] = 1;
  for (int i = 1; i < dims; ++i) PARAMS::Offset[i] = PARAMS::Grid[i - 1] * PARAMS::Offset[i - 1];
  PARAMS::volume = 1;
  for (int i = 0; i < 4; ++i) PARAMS::volume *= PARAMS::Grid[i];
  PARAMS::half_volume = PARAMS::volume / 2;
  PARAMS::spatial_volume = 1;
  for (int i = 0; i < PARAMS::TDir; ++i) PARAMS::spatial_volume *= PARAMS::Grid[i];
  PARAMS::Beta = beta;
  PARAMS::Aniso = aniso;
  PARAMS::metrop = metrop;
  PARAMS::ovrn = ovrn;
  return 0;
}

// One std::mt19937 per OpenMP thread for the reference CPU Metropolis
// (the reference's commented-out CPU driver does the same, u1.cpp:190-192).
void ref_seed_cpu(int nthreads, unsigned seed) {
  if (generator) delete[] generator;
  generator = new std::mt19937[nthreads];
  for (int i = 0; i < nthreads; ++i) generator[i].seed(seed * (unsigned)(i + 1));
  omp_set_num_threads(nthreads);
}

void ref_cpu_metropolis(double *lat) { metropolis(lat); }
void ref_cpu_overrelax(double *lat) { overrelaxation(lat); }
void ref_cpu_plaquette(double *lat, double out[2]) { plaquette(lat, out); }
void ref_cpu_polyakov(double *lat, double out[2]) { polyakov(lat, out); }

// The (new_theta, b) pairs the reference's CPU metropolis draws from
// generator[0] (single thread) seeded with `seed`: for each pass, parity,
// mu, id in that order, new_theta = pi*U[0,2) then b = U[0,1)
// (src/update.cu:53-68).
void ref_record_pairs(unsigned seed, int npass, double *out) {
  std::mt19937 g(seed);
  std::uniform_real_distribution<double> rand02(0., 2.);
  std::uniform_real_distribution<double> rand01(0, 1);
  long k = 0;
  for (int ps = 0; ps < npass; ++ps)
    for (int p = 0; p < 2; ++p)
      for (int mu = 0; mu < Dirs(); ++mu)
        for (int id = 0; id < HalfVolume(); ++id) {
          out[k++] = M_PI * rand02(g);
          out[k++] = rand01(g);
        }
}

void ref_index_eo(int id, int parity, int x[4]) { indexEO(id, parity, x); }
int ref_index_eo_neg1(int id, int parity, int mu, int lmu) { return indexEO_neg(id, parity, mu, lmu); }
int ref_index_eo_neg2(int id, int parity, int mu, int lmu, int nu, int lnu) {
  return indexEO_neg(id, parity, mu, lmu, nu, lnu);
}

void ref_host_staple(double *lat, int id, int parity, int mu, double out[2]) {
  complexd s = Staple(lat, id, parity, mu);
  out[0] = s.real();
  out[1] = s.imag();
}

void ref_host_multihit(double *lat, int id, int parity, double out[2]) {
  complexd m = MultiHit(lat, id, parity, TDir());
  out[0] = m.real();
  out[1] = m.imag();
}

// ----------------------------------------------------------------- GPU side
int ref_gpu_start(int dev) {
  Start(dev, SILENT, TUNE_YES);
  return 0;
}

int ref_gpu_setup(int dims, int Nx, int Ny, int Nz, int Nt, double beta, double aniso, int metrop, int ovrn) {
  SetupLatticeParameters(Nx, Ny, Nz, Nt, dims, beta, aniso, metrop, ovrn);
  return 0;
}

static Array<double> *upload(const double *lat_in) {
  const size_t n = (size_t)Volume() * Dirs();
  Array<double> *a = new Array<double>(Device, n);
  cudaMemcpy(a->getPtr(), lat_in, n * sizeof(double), cudaMemcpyHostToDevice);
  return a;
}

// nsweeps of UpdateLattice(metrop, ovrn) on lat_in (rng seeded by CudaRNG),
// after `warmup` untimed sweeps; returns device milliseconds for the timed
// sweeps (CUDA events on the legacy stream) and writes the lattice to lat_out.
double ref_gpu_update(const double *lat_in, double *lat_out, int metrop, int ovrn, int warmup, int nsweeps,
                      int seed) {
  Array<double> *lat = upload(lat_in);
  CudaRNG *rng = new CudaRNG(seed, HalfVolume());
  for (int i = 0; i < warmup; ++i) UpdateLattice(lat, rng, metrop, ovrn);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaDeviceSynchronize();
  cudaEventRecord(a, 0);
  for (int i = 0; i < nsweeps; ++i) UpdateLattice(lat, rng, metrop, ovrn);
  cudaEventRecord(b, 0);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  const size_t n = (size_t)Volume() * Dirs();
  if (lat_out) cudaMemcpy(lat_out, lat->getPtr(), n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  delete rng;
  delete lat;
  return (double)ms;
}

// A Markov chain of the reference's own CUDA code: from lat_in, nsweeps of
// UpdateLattice(metrop, ovrn) with Plaquette and Polyakov after each, as the
// reference driver's loop does; out[6 * sweep + k] = (SS re, im, ST re, im,
// L re, im).
void ref_gpu_chain(const double *lat_in, int metrop, int ovrn, int nsweeps, int seed, double *out) {
  Array<double> *lat = upload(lat_in);
  CudaRNG *rng = new CudaRNG(seed, HalfVolume());
  for (int i = 0; i < nsweeps; ++i) {
    UpdateLattice(lat, rng, metrop, ovrn);
    complexd p[2];
    Plaquette(lat, p, false);
    complexd l = Polyakov(lat, false);
    double *o = out + 6 * (size_t)i;
    o[0] = p[0].real();
    o[1] = p[0].imag();
    o[2] = p[1].real();
    o[3] = p[1].imag();
    o[4] = l.real();
    o[5] = l.imag();
  }
  delete rng;
  delete lat;
}

void ref_gpu_measure(const double *lat_in, double out[6]) {
  Array<double> *lat = upload(lat_in);
  complexd p[2];
  Plaquette(lat, p, false);
  complexd l = Polyakov(lat, false);
  out[0] = p[0].real();
  out[1] = p[0].imag();
  out[2] = p[1].real();
  out[3] = p[1].imag();
  out[4] = l.real();
  out[5] = l.imag();
  delete lat;
}

// Poly2 writes Pot_*.dat into the working directory (src/polyakov.cu:634-650).
void ref_gpu_poly2(const double *lat_in, int multihit, double *out) {
  Array<double> *lat = upload(lat_in);
  Array<complexd> *res = Poly2(lat, multihit != 0);
  for (int r = 0; r < Grid(0) / 2; ++r) {
    out[2 * r] = res->getPtr()[r].real();
    out[2 * r + 1] = res->getPtr()[r].imag();
  }
  delete res;
  delete lat;
}

// MultiLevelField: the same algorithm as MultiLevel but with the ppSpace
// buffer allocated (MultiLevel's L4AvgPP<false> reads an uninitialised
// member, src/multilevel.cu:578,587).  Writes Pot_mlevel_*.dat.
void ref_gpu_multilevel(const double *lat_in, int n4, int k4, int n2, int k2, int metrop, int ovrn, int seed,
                        double *out) {
  Array<double> *lat = upload(lat_in);
  CudaRNG *rng = new CudaRNG(seed, HalfVolume());
  MultiLevelRes *res = MultiLevelField(lat, rng, n4, k4, n2, k2, metrop, ovrn);
  for (int r = 0; r < Grid(0) / 2; ++r) {
    out[2 * r] = res->poly->getPtr()[r].real();
    out[2 * r + 1] = res->poly->getPtr()[r].imag();
  }
  delete res;
  delete rng;
  delete lat;
}

// LatticeConvert (src/convertOrder.cu:135-145): the reference's EO -> natural
// order conversion of a whole lattice (V * dirs FP64 angles in and out).
// Only eo_to_no = 1 runs: the reference's NO -> EO kernel writes
// out[id + parity * V/2 + dir * V] with the natural-order index id < V
// (src/convertOrder.cu:49-58), past the end of its output array.
void ref_gpu_convert(const double *lat_in, int eo_to_no, double *out) {
  if (eo_to_no != 1) return;
  Array<double> *lat = upload(lat_in);
  Array<double> *res = LatticeConvert(lat, eo_to_no != 0);
  const size_t n = (size_t)Volume() * Dirs();
  cudaMemcpy(out, res->getPtr(), n * sizeof(double), cudaMemcpyDeviceToHost);
  delete res;
  delete lat;
}

// PlaquetteFields(lat, arg, spacetime, evenoddOrder = true)
// (src/plaquette_comps.cu:216-227): the six plaquette components per site
// (spacetime) or time-averaged per spatial site, natural site order,
// complexd[6 * size] with component d at [d * size]; means[12] = the six
// component means (re, im).  The lattice is in the library's EO order.
void ref_gpu_plaq_fields(const double *lat_in, int spacetime, double *field, double *means) {
  Array<double> *lat = upload(lat_in);
  PlaqFieldArg arg;
  PlaquetteFields(lat, &arg, spacetime != 0, true);
  cudaMemcpy(field, arg.plaqfield, 6 * arg.size * sizeof(complexd), cudaMemcpyDeviceToHost);
  for (int i = 0; i < 6; ++i) {
    means[2 * i] = arg.plaq[i].real();
    means[2 * i + 1] = arg.plaq[i].imag();
  }
  delete lat;
}

}  // extern "C"
