// The reference driver's main workload (reference u1.cpp:42-128: 24^3 x 12,
// beta = 1, 1 Metropolis + 3 overrelaxation per sweep, cold start, 1000
// sweeps, plaquette and Polyakov loop every 100 sweeps, then Poly2 without
// and with multihit), written against the reference's namespace U1 API only,
// so the same source builds against the reference's own objects
// (oracle/Makefile target refdriver-timing) and against the drop-in shim.
// Prints the observables and "TIME <seconds>" of the sweep loop and the
// Poly2 calls (wall clock, including every synchronisation the API does).
#include <chrono>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

#include "timer.h"
#include "alloc.h"
#include "complex.h"

#include "parameters.h"
#include "random.h"
#include "update.h"
#include "plaquette.h"
#include "polyakov.h"

#include "array.h"

using namespace U1;

int main() {
  Start(0, SILENT, TUNE_YES);
  SetupLatticeParameters(24, 24, 24, 12, 4, 1.0, 1.0, 1, 3);
  Array<double> *lattice = new Array<double>(Device, Volume() * Dirs());
  CudaRNG *rng = new CudaRNG(1234, HalfVolume());
  complexd *plaqv = new complexd[2];
  // first calls outside the timed region (kernel tuning on first use)
  UpdateLattice(lattice, rng, PARAMS::metrop, PARAMS::ovrn);
  Plaquette(lattice, plaqv);
  Polyakov(lattice);
  const auto t0 = std::chrono::steady_clock::now();
  for (PARAMS::iter = 1; PARAMS::iter <= 1000; ++PARAMS::iter) {
    UpdateLattice(lattice, rng, PARAMS::metrop, PARAMS::ovrn);
    if (PARAMS::iter % 100 == 0) {
      Plaquette(lattice, plaqv);
      complexd L = Polyakov(lattice);
      std::printf("SWEEP %d %.10f %.10f %.10f\n", PARAMS::iter, plaqv[0].real(), plaqv[1].real(), L.abs());
    }
  }
  Array<complexd> *res = Poly2(lattice, false);
  delete res;
  res = Poly2(lattice, true);
  std::printf("POLY2MH %.10g %.10g\n", res->getPtr()[0].real(), res->getPtr()[1].real());
  delete res;
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf("TIME %.6f\n", s);
  delete[] plaqv;
  delete rng;
  delete lattice;
  Finalize(0);
  return 0;
}
