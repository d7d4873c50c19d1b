// Force-included (nvcc -include) when compiling the reference sources in
// place.  The reference's MultiHit is __host__ __device__ but calls the
// device-only cyl_bessel_i0/i1 (reference include/lattice_functions.h:101),
// so the reference does not compile as shipped.  These wrappers keep the
// device path on CUDA's functions and give the host path std::cyl_bessel_i,
// which lets the harness call the reference's own MultiHit on the CPU.
// No reference source is modified or copied.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

__host__ __device__ inline double u1ref_bessel_i0(double x) {
#ifdef __CUDA_ARCH__
  return cyl_bessel_i0(x);
#else
  return std::cyl_bessel_i(0.0, x);
#endif
}

__host__ __device__ inline double u1ref_bessel_i1(double x) {
#ifdef __CUDA_ARCH__
  return cyl_bessel_i1(x);
#else
  return std::cyl_bessel_i(1.0, x);
#endif
}

#define cyl_bessel_i0 u1ref_bessel_i0
#define cyl_bessel_i1 u1ref_bessel_i1
