// Integrated autocorrelation time (reference include/actime.h,
// src/actime.cpp): Wolff's automatic windowing Gamma method
// (U. Wolff, Comput. Phys. Commun. 156 (2004) 143, hep-lat/0306017) and a
// simple summed-autocorrelation window; both print their estimates.
#ifndef U1_SHIM_ACTIME_H
#define U1_SHIM_ACTIME_H
#include <vector>
namespace U1 {
void calculateCorTime(int miniter, int iter, std::vector<double> &gamma, int &nsweep);
void calculateCorTime1(int miniter, int iter, std::vector<double> &gamma, int &nsweep);
}  // namespace U1
#endif
