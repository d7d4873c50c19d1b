// Plaquette (reference include/plaquette.h:12, src/plaquette.cu:222-228):
// plaq[0] = spatial-spatial, plaq[1] = space-time mean of (1 - e^{i theta_P}).
#ifndef U1_SHIM_PLAQUETTE_H
#define U1_SHIM_PLAQUETTE_H
#include "array.h"
#include "complex.h"
namespace U1 {
complexd *Plaquette(Array<double> *dev_lat, complexd *plaq, bool print = false);
}  // namespace U1
#endif
