// A small driver written against the reference's API (namespace U1, as in
// reference u1.cpp) and linked with the drop-in shim.  Prints the
// plaquette and Polyakov loop after each of a few sweeps, then Poly2 and
// MultiLevel results, one "tag value..." line each, for tests/test_dropin.py.
#include <cstdio>
#include <cstdlib>

#include "array.h"
#include "complex.h"
#include "multilevel.h"
#include "parameters.h"
#include "plaquette.h"
#include "polyakov.h"
#include "random.h"
#include "update.h"

using namespace U1;

int main(int argc, char **argv) {
  const int seed = argc > 1 ? std::atoi(argv[1]) : 1234;
  Start(0, SILENT, TUNE_YES);
  SetupLatticeParameters(8, 6, 6, 8, 4, 1.0, 1.0, 1, 4);
  Array<double> *lattice = new Array<double>(Device, Volume() * Dirs());
  CudaRNG *rng = new CudaRNG(seed, HalfVolume());
  HotStart(lattice, rng);
  complexd plaq[2];
  for (PARAMS::iter = 1; PARAMS::iter <= 3; ++PARAMS::iter) {
    UpdateLattice(lattice, rng, PARAMS::metrop, PARAMS::ovrn);
    Plaquette(lattice, plaq);
    complexd L = Polyakov(lattice);
    std::printf("SWEEP %d %.17g %.17g %.17g %.17g %.17g %.17g\n", PARAMS::iter, plaq[0].real(), plaq[0].imag(),
                plaq[1].real(), plaq[1].imag(), L.real(), L.imag());
  }
  PARAMS::iter = 3;
  Array<complexd> *c = Poly2(lattice, true);
  std::printf("POLY2MH");
  for (size_t r = 0; r < c->Size(); ++r) std::printf(" %.17g %.17g", c->at((int)r).real(), c->at((int)r).imag());
  std::printf("\n");
  delete c;
  Array<complexd> *m = MultiLevel(lattice, rng, 2, 1, 3, 1, 1, 2);
  std::printf("MULTILEVEL");
  for (size_t r = 0; r < m->Size(); ++r) std::printf(" %.17g %.17g", m->at((int)r).real(), m->at((int)r).imag());
  std::printf("\n");
  delete m;
  delete rng;
  delete lattice;
  Finalize(0);
  return 0;
}
