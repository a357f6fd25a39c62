// mpm_sort.cuh — stable LSD radix sort of (u32 key, u32 value) pairs.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

namespace mpm {

constexpr uint32_t kSortTile = 4096;  // keys per sort CTA

uint32_t sort_blocks(uint32_t n);
// Words of scratch the `hist` argument needs for n keys.
size_t sort_hist_words(uint32_t n);

// Sorts the pairs (keys_in[i], vals_in[i]) for i < n by the low key_bits
// bits of the key, stably (vals_in == nullptr means the identity 0..n-1).
// keys_in/vals_in are read only; keys_a/keys_b/vals_a/vals_b (n words each)
// are ping-pong scratch and hist needs sort_hist_words(n) words.  On return
// *keys_out / *vals_out point at the scratch buffers holding the result.
// Asynchronous on `stream`; adds the number of kernel launches to *launches.
cudaError_t radix_sort_pairs(cudaStream_t stream, const uint32_t* keys_in, const uint32_t* vals_in,
                             uint32_t* keys_a, uint32_t* keys_b, uint32_t* vals_a, uint32_t* vals_b, uint32_t* hist,
                             uint32_t n, int key_bits, uint32_t** keys_out, uint32_t** vals_out, uint64_t* launches);

// Records the message returned by mpm_last_error on the calling thread.
void set_last_error(const std::string& msg);

}  // namespace mpm
