// Internal interface of the radix sort (sort.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/dyphur_b200.h"

namespace dyph {

// Workspace for sorting n keys of key_bytes (4 or 8) with uint32 values.
size_t sort_workspace_bytes(size_t n, int key_bytes);

// Pre-set kernel attributes of the sort (call once, outside graph capture).
dyph_status sort_prepare();

// Stable ascending sort of (keys, vals) on the low key_bits bits of keys.
dyph_status sort_u32_u32(uint32_t* keys, uint32_t* vals, size_t n, int key_bits, void* ws, size_t ws_size,
                         cudaStream_t s);
dyph_status sort_u64_u32(uint64_t* keys, uint32_t* vals, size_t n, int key_bits, void* ws, size_t ws_size,
                         cudaStream_t s);

}  // namespace dyph
