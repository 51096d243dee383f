// static_scratch.hpp -- the statically allocated front-scratch area (see
// static_scratch.cu).
#pragma once

#include <cstddef>

namespace cupf_b200 {

// Size of the static front-scratch area on each device (8 MiB).
constexpr size_t kStaticFrontScratchBytes = size_t(8) << 20;

// Device address of the area on the current device.  The first call on each
// device looks the symbol up (cudaGetSymbolAddress, with that device current),
// which loads the area's module and so reserves its memory, and caches the
// address for the life of the process; later calls only read the cache,
// which a cudaDeviceReset of that device makes stale.  Throws on failure.
// The engine makes the first call when it allocates a workspace.
void* static_front_scratch();

}  // namespace cupf_b200
