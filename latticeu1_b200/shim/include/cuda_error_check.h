// Start / Finalize of the reference (reference src/cuda_error_check.cpp:24-72).
// Start selects the device through u1_ctx_create; Finalize releases the
// context.  Errors inside the shim print the C ABI message and terminate,
// as the reference's cudaSafeCall does.
#ifndef U1_SHIM_CUDA_ERROR_CHECK_H
#define U1_SHIM_CUDA_ERROR_CHECK_H
#include "enum.h"
namespace U1 {
void Start(int gpuid, Verbosity verb = VERBOSE, TuneMode tune = TUNE_YES);
void Finalize(int error);
Verbosity getVerbosity();
TuneMode getTuning();
void setVerbosity(Verbosity v);
void setTuning(TuneMode t);
}  // namespace U1
#endif
