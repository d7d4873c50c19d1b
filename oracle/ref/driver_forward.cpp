// Lazy forwarders for the four CUDA driver-API calls the reference's
// allocator makes (reference src/alloc.cpp:220,360 and pointer queries).
// Linking libcuda directly would make oracle/_ref/libu1ref.so unloadable on
// a machine without the NVIDIA driver, where the CPU half of the harness
// (the reference's FP64 CPU functions) must still work.  Each forwarder
// resolves the real symbol from libcuda.so.1 on first use and returns
// CUDA_ERROR_NOT_INITIALIZED when no driver is present.
#include <cuda.h>
#include <dlfcn.h>

static void *driver_sym(const char *name) {
  static void *h = dlopen("libcuda.so.1", RTLD_NOW | RTLD_GLOBAL);
  return h ? dlsym(h, name) : nullptr;
}

extern "C" {

CUresult cuMemAlloc_v2(CUdeviceptr *dptr, size_t bytesize) {
  typedef CUresult (*F)(CUdeviceptr *, size_t);
  static F f = (F)driver_sym("cuMemAlloc_v2");
  return f ? f(dptr, bytesize) : CUDA_ERROR_NOT_INITIALIZED;
}

CUresult cuMemFree_v2(CUdeviceptr dptr) {
  typedef CUresult (*F)(CUdeviceptr);
  static F f = (F)driver_sym("cuMemFree_v2");
  return f ? f(dptr) : CUDA_ERROR_NOT_INITIALIZED;
}

CUresult cuGetErrorString(CUresult error, const char **pStr) {
  typedef CUresult (*F)(CUresult, const char **);
  static F f = (F)driver_sym("cuGetErrorString");
  if (f) return f(error, pStr);
  if (pStr) *pStr = "CUDA driver not available";
  return CUDA_ERROR_NOT_INITIALIZED;
}

CUresult cuPointerGetAttributes(unsigned int numAttributes, CUpointer_attribute *attributes, void **data,
                                CUdeviceptr ptr) {
  typedef CUresult (*F)(unsigned int, CUpointer_attribute *, void **, CUdeviceptr);
  static F f = (F)driver_sym("cuPointerGetAttributes");
  return f ? f(numAttributes, attributes, data, ptr) : CUDA_ERROR_NOT_INITIALIZED;
}

}  // extern "C"
