// noalloc.hpp -- fixed device scratch of the allocation-free entry point (noalloc.cu).
#pragma once

#include <cstddef>

#include "host.hpp"

namespace ho2d {

// 1 Mi doubles (8 MiB): two face-trace arrays of N_el * 4 * Knod doubles, so the
// allocation-free entry point serves meshes with N_el * Knod <= 131072.
constexpr size_t kNoAllocScratchDoubles = size_t(1) << 20;

// Device address of the fixed scratch on `device`, which must be the current device the
// first time it is asked for; later calls return the cached address.
Error noalloc_scratch(int device, double** ptr);

}  // namespace ho2d
