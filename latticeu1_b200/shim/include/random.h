// CudaRNG of the reference's API (reference include/random.h:31-58): owns a
// counter-based Philox stream of the C ABI (u1_rng).  The reference ignores
// the seed argument (src/random.cu:34); here the seed is used.
#ifndef U1_SHIM_RANDOM_H
#define U1_SHIM_RANDOM_H
#include <cstddef>
#include <cstdint>

struct u1_rng;

namespace U1 {
class CudaRNG {
 public:
  CudaRNG();
  CudaRNG(int seed, size_t size);
  ~CudaRNG();
  CudaRNG(const CudaRNG &) = delete;
  CudaRNG &operator=(const CudaRNG &) = delete;
  u1_rng *getPtr() { return rng_; }
  void Backup();
  void Restore();

 private:
  u1_rng *rng_ = nullptr;
  uint64_t saved_seed_ = 0, saved_pass_ = 0;
};
}  // namespace U1
#endif
