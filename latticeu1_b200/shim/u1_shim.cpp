// Drop-in implementation of the reference's driver API (namespace U1 as
// used by reference u1.cpp:38-237) on top of the C ABI in
// include/u1_b200.h.  Unmodified driver code that includes the reference's
// header names (timer.h, parameters.h, update.h, plaquette.h, polyakov.h,
// multilevel.h, array.h, random.h, actime.h) compiles against
// latticeu1_b200/shim/include and links with libu1shim.so + libu1b200.so.
//
// Behaviour kept from the reference: the global PARAMS, GetLatticeName(),
// console output and the Pot_*.dat files written by Poly2/MultiLevel
// (reference src/polyakov.cu:634-650, src/multilevel.cu:712-730), and
// process exit on errors (reference src/cuda_error_check.cpp:84-101, where
// the C ABI itself returns status codes).
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "actime.h"
#include "alloc.h"
#include "array.h"
#include "cuda_error_check.h"
#include "multilevel.h"
#include "parameters.h"
#include "plaquette.h"
#include "polyakov.h"
#include "random.h"
#include "u1_b200.h"
#include "update.h"

namespace U1 {

namespace PARAMS {
double Beta = 0.0;
double Aniso = 1.0;
int DIRS = 4;
int TDir = 3;
int volume = 0;
int half_volume = 0;
int spatial_volume = 0;
int Grid[4] = {1, 1, 1, 1};
int Offset[4] = {0, 0, 0, 0};
int iter = 0;
double accept_ratio = 0.0;
int ovrn = 3;
int metrop = 1;
}  // namespace PARAMS

namespace {
u1_ctx *g_ctx = nullptr;
u1_geom g_geom{};
bool g_geom_set = false;
Verbosity g_verb = VERBOSE;
TuneMode g_tune = TUNE_YES;

[[noreturn]] void die(const char *what, int rc) {
  std::fprintf(stderr, "U1 error in %s: [%d] %s\n", what, rc, u1_last_error());
  std::exit(EXIT_FAILURE);
}
void check(int rc, const char *what) {
  if (rc != U1_OK) die(what, rc);
}
u1_ctx *ctx() {
  if (!g_ctx) check(u1_ctx_create(0, &g_ctx), "u1_ctx_create");
  return g_ctx;
}
u1_lattice *lattice_of(Array<double> *a) {
  if (!a || !a->lattice()) {
    std::fprintf(stderr, "U1 error: the gauge field must be an Array<double>(Device, Volume()*Dirs())\n");
    std::exit(EXIT_FAILURE);
  }
  return a->lattice();
}
}  // namespace

Verbosity getVerbosity() { return g_verb; }
TuneMode getTuning() { return g_tune; }
void setVerbosity(Verbosity v) { g_verb = v; }
void setTuning(TuneMode t) { g_tune = t; }

void Start(int gpuid, Verbosity verb, TuneMode tune) {
  g_verb = verb;
  g_tune = tune;
  if (g_ctx) u1_ctx_destroy(g_ctx);
  g_ctx = nullptr;
  check(u1_ctx_create(gpuid, &g_ctx), "Start: u1_ctx_create");
  std::cout << "Using gpu id: " << gpuid << std::endl;
}

void Finalize(int error) {
  if (g_ctx) u1_ctx_destroy(g_ctx);
  g_ctx = nullptr;
  if (error) std::exit(error);
}

void printPeakMemUsage() {}
void assertAllMemFree() {}

void SetupLatticeParameters(int Nx, int Ny, int Nz, int Nt, int dirs, double beta, double aniso, int imetrop,
                            int ovrn) {
  u1_geom g{};
  g.dims = dirs;
  g.N[0] = Nx;
  g.N[1] = Ny;
  g.N[2] = Nz;
  g.N[3] = Nt;
  g.beta = beta;
  g.aniso = aniso;
  int64_t info[8];
  if (u1_geom_validate(&g, info) != U1_OK) {
    std::cout << "Error: Number of points should be an even number..." << std::endl;
    Finalize(1);
  }
  g_geom = g;
  g_geom_set = true;
  PARAMS::DIRS = dirs;
  PARAMS::TDir = dirs - 1;
  for (int i = 0; i < 4; ++i) {
    PARAMS::Grid[i] = (int)info[4 + i];
    PARAMS::Offset[i] = 0;
  }
  PARAMS::Offset[0] = 1;
  for (int i = 1; i < dirs; ++i) PARAMS::Offset[i] = PARAMS::Grid[i - 1] * PARAMS::Offset[i - 1];
  PARAMS::volume = (int)info[0];
  PARAMS::half_volume = (int)info[1];
  PARAMS::spatial_volume = (int)info[2];
  PARAMS::Beta = beta;
  PARAMS::Aniso = aniso;
  PARAMS::metrop = imetrop;
  PARAMS::ovrn = ovrn;
  std::cout << "==========================================" << std::endl;
  std::cout << "Lattice properties:" << std::endl;
  std::cout << "------------------------------------------" << std::endl;
  std::cout << "    Volume: ";
  for (int i = 0; i < dirs; i++) {
    std::cout << Grid(i);
    if (i < dirs - 1) std::cout << "x";
  }
  std::cout << std::endl;
  std::cout << "    Number of directions: " << Dirs() << std::endl;
  std::cout << "    Time indice: " << TDir() << std::endl;
  std::cout << "    Beta: " << Beta() << std::endl;
  std::cout << "    Anisotropy: " << Aniso() << std::endl;
  std::cout << "    Metropolis updates: " << PARAMS::metrop << std::endl;
  std::cout << "    Overrelaxation updates: " << PARAMS::ovrn << std::endl;
  std::cout << "==========================================" << std::endl;
}

std::string GetLatticeName() {
  std::string name;
  for (int i = 0; i < Dirs(); i++) name += ToString(PARAMS::Grid[i]) + "_";
  name += "beta_" + ToString(PARAMS::Beta);
  name += "_xi_" + ToString(PARAMS::Aniso);
  name += "_mtr_" + ToString(PARAMS::metrop);
  name += "_ovr_" + ToString(PARAMS::ovrn);
  return name;
}

std::string GetLatticeNameI() { return GetLatticeName() + "_iter_" + ToString(PARAMS::iter); }

// -- gauge field objects ---------------------------------------------------
u1_lattice *shim_new_lattice() {
  if (!g_geom_set) {
    std::fprintf(stderr, "U1 error: SetupLatticeParameters must be called before creating the gauge field\n");
    std::exit(EXIT_FAILURE);
  }
  u1_lattice *lat = nullptr;
  check(u1_lattice_create(ctx(), &g_geom, &lat), "u1_lattice_create");
  return lat;
}
void shim_free_lattice(u1_lattice *lat) { u1_lattice_destroy(lat); }
void shim_lattice_import(u1_lattice *lat, const double *a) {
  check(u1_lattice_import_angles(lat, a, 0), "u1_lattice_import_angles");
}
void shim_lattice_export(u1_lattice *lat, double *a) {
  check(u1_lattice_export_angles(lat, a, 0), "u1_lattice_export_angles");
}

CudaRNG::CudaRNG() { check(u1_rng_create(ctx(), 1234, &rng_), "u1_rng_create"); }
CudaRNG::CudaRNG(int seed, size_t) { check(u1_rng_create(ctx(), (uint64_t)(uint32_t)seed, &rng_), "u1_rng_create"); }
CudaRNG::~CudaRNG() {
  if (rng_) u1_rng_destroy(rng_);
}
void CudaRNG::Backup() { check(u1_rng_get_state(rng_, &saved_seed_, &saved_pass_), "u1_rng_get_state"); }
void CudaRNG::Restore() { check(u1_rng_set_state(rng_, saved_seed_, saved_pass_), "u1_rng_set_state"); }

// -- hot path ------------------------------------------------------------------
void HotStart(Array<double> *dev_lat, CudaRNG *rng) {
  check(u1_hot_start(lattice_of(dev_lat), rng->getPtr()), "u1_hot_start");
}

void UpdateLattice(Array<double> *dev_lat, CudaRNG *rng, int metrop, int ovrn) {
  check(u1_update(lattice_of(dev_lat), rng->getPtr(), metrop, ovrn), "u1_update");
}

complexd *Plaquette(Array<double> *dev_lat, complexd *plaq, bool print) {
  double out[4];
  check(u1_plaquette(lattice_of(dev_lat), out), "u1_plaquette");
  plaq[0] = complexd(out[0], out[1]);
  plaq[1] = complexd(out[2], out[3]);
  if (print) {
    std::cout << "0plaqSS: " << plaq[0] << "\tplaqST: " << plaq[1] << "\tMean: " << (plaq[0] + plaq[1]) * 0.5
              << std::endl;
    const complexd ss = plaq[0] / Aniso(), st = plaq[1] * Aniso();
    std::cout << "1plaqSS: " << ss << "\tplaqST: " << st << "\tMean: " << (ss + st) * 0.5
              << "\tAction: " << (ss + st) * (0.5 * Beta()) << std::endl;
  }
  return plaq;
}

complexd Polyakov(Array<double> *dev_lat, bool print) {
  double out[2];
  check(u1_polyakov(lattice_of(dev_lat), out), "u1_polyakov");
  const complexd L(out[0], out[1]);
  if (print) std::cout << "L: " << L.real() << '\t' << L.imag() << "\t|L|: " << L.abs() << std::endl;
  return L;
}

namespace {
void write_correlator(const std::string &filename, Array<complexd> *c) {
  std::ofstream f(filename.c_str());
  if (!f.is_open()) {
    std::cout << "Error opening file: " << filename << std::endl;
    std::exit(1);
  }
  f.precision(12);
  for (size_t r = 0; r < c->Size(); ++r) {
    std::cout << r + 1 << '\t' << c->at((int)r).real() << '\t' << c->at((int)r).imag() << std::endl;
    f << r + 1 << '\t' << c->at((int)r).real() << '\t' << c->at((int)r).imag() << std::endl;
  }
}
}  // namespace

Array<complexd> *Poly2(Array<double> *dev_lat, bool multihit) {
  const int R = Grid(0) / 2;
  std::vector<double> out(2 * R);
  check(u1_poly_corr(lattice_of(dev_lat), multihit ? 1 : 0, out.data(), 2 * R), "u1_poly_corr");
  Array<complexd> *res = new Array<complexd>(Host, R);
  for (int r = 0; r < R; ++r) res->at(r) = complexd(out[2 * r], out[2 * r + 1]);
  write_correlator((multihit ? "Pot_mhit_" : "Pot_") + GetLatticeNameI() + ".dat", res);
  return res;
}

Array<complexd> *MultiLevel(Array<double> *dev_lat, CudaRNG *rng, int n4, int k4, int n2, int k2, int metrop,
                            int ovrn) {
  if (Grid(TDir()) % 4 != 0) {
    std::cout << "Error: Cannot Apply MultiLevel Algorithm...\n Nt is not multiple of 4...\n Exiting..." << std::endl;
    std::exit(1);
  }
  const int R = Grid(0) / 2;
  std::vector<double> out(2 * R);
  check(u1_multilevel(lattice_of(dev_lat), rng->getPtr(), n4, k4, n2, k2, metrop, ovrn, out.data(), 2 * R),
        "u1_multilevel");
  Array<complexd> *res = new Array<complexd>(Host, R);
  for (int r = 0; r < R; ++r) res->at(r) = complexd(out[2 * r], out[2 * r + 1]);
  std::string filename = "Pot_mlevel_" + GetLatticeNameI();
  filename += "_" + ToString(n4) + "_" + ToString(k4);
  filename += "_" + ToString(n2) + "_" + ToString(k2);
  filename += "_" + ToString(metrop) + "_" + ToString(ovrn) + ".dat";
  std::ofstream f(filename.c_str());
  if (!f.is_open()) {
    std::cout << "Error opening file: " << filename << std::endl;
    std::exit(1);
  }
  f.precision(12);
  for (int r = 0; r < R; ++r) {
    std::cout << r + 1 << '\t' << res->at(r) << std::endl;
    f << r + 1 << '\t' << res->at(r) << std::endl;
  }
  return res;
}

}  // namespace U1
