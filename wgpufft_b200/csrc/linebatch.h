// Batched launches of 1D complex f32 lines of mixed lengths for callers
// that form a new set of lines every time (the serving loop): a registry
// keeps every length's classification, descriptors and tables resident on
// the device, so that a launch over any set of lines only builds and
// uploads its task lists (stream-ordered allocations, nothing synchronous
// on the host once its lengths are known).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/wgpufft_b200.h"

namespace b2f {

struct LineRegistry;

// Registry of one device, direction and normalization.
LineRegistry* line_registry_new(int device, int32_t direction, int32_t normalization);
void line_registry_free(LineRegistry* reg);
// Device bytes the registry holds (descriptors, twiddle arena, tables).
uint64_t line_registry_bytes(const LineRegistry* reg);

// Whether a line of length n can run in a registry launch (one CTA, or the
// two/three-pass long route with factors up to 512); registers it if so.
bool line_registry_accepts(LineRegistry* reg, uint64_t n);

// One launch over n lines on `st`: line i has lengths[i] points at complex
// offset in_off[i] of `in` and out_off[i] of `out` (lines disjoint within
// each buffer; every length accepted by line_registry_accepts).  Task lists,
// counters and long-line scratch come from stream-ordered allocations freed
// on `st` after the kernels; *device_bytes receives their size.
b2f_status line_batch_run(LineRegistry* reg, cudaStream_t st, const uint64_t* lengths,
                          const uint64_t* in_off, const uint64_t* out_off, uint64_t n,
                          const void* in, void* out, uint64_t* device_bytes);

}  // namespace b2f
