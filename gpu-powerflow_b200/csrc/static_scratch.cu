// static_scratch.cu -- a fixed, statically allocated front-scratch area for
// the allocation-free factorization entry point (cls_factorize_static_scratch).
//
// Levels whose dense fronts do not fit in shared memory next to their staged
// sources keep those fronts in global memory.  The regular path takes that
// memory from the handle's workspace (allocated when the batch grows); the
// static path takes it from this file-scope device array, which exists on
// every device as soon as the library's module is loaded, so the call itself
// allocates nothing.  Its size is fixed: kStaticFrontScratchBytes.
//
// Nothing in the area has to start at zero: the factor kernel zeroes each
// front before assembling into it.  The area is shared by every handle of
// the process on a device, so calls that use it must not overlap in time
// (two at once on one device race on the same memory).
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "static_scratch.hpp"

namespace cupf_b200 {

__device__ __align__(256) unsigned char g_static_front_scratch[kStaticFrontScratchBytes];

void* static_front_scratch() {
  constexpr int kMaxDevices = 64;
  static void* addr[kMaxDevices] = {};
  static std::mutex mu;
  int dev = 0;
  const cudaError_t ge = cudaGetDevice(&dev);
  if (ge != cudaSuccess) throw std::runtime_error(std::string("static front scratch: ") + cudaGetErrorString(ge));
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("static front scratch: device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    // once per device, with that device current
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_front_scratch);
    if (e != cudaSuccess || !p)
      throw std::runtime_error(std::string("static front scratch: cudaGetSymbolAddress failed: ") +
                               cudaGetErrorString(e));
    addr[dev] = p;
  }
  return addr[dev];
}

}  // namespace cupf_b200
