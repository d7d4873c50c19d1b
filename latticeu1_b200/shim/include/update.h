// HotStart / UpdateLattice (reference include/update.h:10-12,
// src/update.cu:43-48,449-456) on the sm_100a kernels.
#ifndef U1_SHIM_UPDATE_H
#define U1_SHIM_UPDATE_H
#include "array.h"
#include "random.h"
namespace U1 {
void HotStart(Array<double> *dev_lat, CudaRNG *rng_state);
void UpdateLattice(Array<double> *dev_lat, CudaRNG *rng_state, int metrop, int ovrn);
}  // namespace U1
#endif
