// MultiLevel (reference include/multilevel.h:9, src/multilevel.cu:639-732):
// returns a new host Array<complexd> of C(r) (caller deletes) and writes
// Pot_mlevel_<lattice name>_iter_<iter>_<n4>_<k4>_<n2>_<k2>_<metrop>_<ovrn>.dat.
#ifndef U1_SHIM_MULTILEVEL_H
#define U1_SHIM_MULTILEVEL_H
#include "array.h"
#include "random.h"
namespace U1 {
Array<complexd> *MultiLevel(Array<double> *dev_lat, CudaRNG *rng_state, int n4, int k4, int n2, int k2, int metrop,
                            int ovrn);
}  // namespace U1
#endif
