// Memory-tracking entry points of the reference (reference include/alloc.h).
// Device memory is owned by the C ABI objects, so these report nothing.
#ifndef U1_SHIM_ALLOC_H
#define U1_SHIM_ALLOC_H
#include "enum.h"
namespace U1 {
void printPeakMemUsage();
void assertAllMemFree();
}  // namespace U1
#endif
