// Global lattice parameters of the reference's driver surface
// (reference include/parameters.h, src/parameters.cu:90-208).  PARAMS holds
// plain host globals as the reference's driver expects; the lattice
// geometry itself lives in the C ABI lattice objects.
#ifndef U1_SHIM_PARAMETERS_H
#define U1_SHIM_PARAMETERS_H
#include <sstream>
#include <string>

#include "cuda_error_check.h"
#include "enum.h"

namespace U1 {
void SetupLatticeParameters(int Nx, int Ny, int Nz, int Nt, int dirs, double beta, double aniso, int imetrop,
                            int ovrn);
std::string GetLatticeName();
std::string GetLatticeNameI();

namespace PARAMS {
extern double Beta;
extern double Aniso;
extern int DIRS;
extern int TDir;
extern int volume;
extern int half_volume;
extern int spatial_volume;
extern int Grid[4];
extern int Offset[4];
extern int iter;
extern double accept_ratio;
extern int ovrn;
extern int metrop;
}  // namespace PARAMS

inline int Volume() { return PARAMS::volume; }
inline int HalfVolume() { return PARAMS::half_volume; }
inline int SpatialVolume() { return PARAMS::spatial_volume; }
inline int Grid(int dim) { return PARAMS::Grid[dim]; }
inline int Offset(int dim) { return PARAMS::Offset[dim]; }
inline double Beta() { return PARAMS::Beta; }
inline int Dirs() { return PARAMS::DIRS; }
inline int TDir() { return PARAMS::TDir; }
inline double Aniso() { return PARAMS::Aniso; }

template <class T>
inline std::string ToString(const T number) {
  std::stringstream ss;
  ss << number;
  return ss.str();
}
}  // namespace U1
#endif
