// Polyakov / Poly2 (reference include/polyakov.h:13-16,
// src/polyakov.cu:169-174,618-654).  Poly2 returns a new host
// Array<complexd> of C(r), r = 1..Grid(0)/2 (caller deletes) and writes
// Pot_[mhit_]<lattice name>_iter_<iter>.dat like the reference.
#ifndef U1_SHIM_POLYAKOV_H
#define U1_SHIM_POLYAKOV_H
#include "array.h"
#include "complex.h"
namespace U1 {
complexd Polyakov(Array<double> *dev_lat, bool print = false);
Array<complexd> *Poly2(Array<double> *dev_lat, bool multihit);
}  // namespace U1
#endif
