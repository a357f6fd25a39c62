// mpm_sort.cu — stable LSD radix sort of (u32 key, u32 value) pairs.
//
// Replaces RadixSortKernel / RadixSortDispatch
// (crates/molla-compute-primitives/src/radix_sort.rs:50-110, WGSL
// count_block_bins / scan_global_bins / scatter, radix_sort.wgsl:100-261).
// Same contract: ascending by key, ties keep input order (stable), so the
// output equals a host stable sort of the pairs.  Differences are of
// design, not of result:
//   * only ceil(key_bits / 8) passes run (the upper digits of tile keys are
//     zero, so skipping them leaves the permutation unchanged);
//   * each pass is three kernels: a per-tile digit histogram with
//     warp-aggregated shared-memory counts, a per-digit scan of the tile
//     counts (one CTA per digit), and a scatter that ranks keys stably
//     inside the tile with __match_any_sync and a per-warp prefix;
//   * pass 0 can generate the identity values (0..n-1) itself.
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/molla_mpm.h"
#include "mpm_sort.cuh"

namespace mpm {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRounds = kSortTile / kThreads;  // 16
constexpr int kBins = 256;

__global__ void __launch_bounds__(kThreads) k_sort_hist(const uint32_t* __restrict__ keys, uint32_t n, int shift,
                                                   uint32_t nblocks, uint32_t* __restrict__ hist) {
  __shared__ uint32_t s_h[kBins + 1];
  const int tid = threadIdx.x;
  s_h[tid] = 0;
  if (tid == 0) s_h[kBins] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
  const int lane = tid & 31;
#pragma unroll 4
  for (int r = 0; r < kRounds; ++r) {
    const uint64_t idx = base + (uint64_t)r * kThreads + tid;
    const uint32_t d = idx < n ? (keys[idx] >> shift) & 0xffu : (uint32_t)kBins;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (lane == __ffs(peers) - 1 && d < (uint32_t)kBins) atomicAdd(&s_h[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  hist[(size_t)tid * nblocks + blockIdx.x] = s_h[tid];
}

// One CTA per digit: exclusive scan of hist[d][0..nblocks) in place, total to
// totals[d].
__global__ void __launch_bounds__(1024) k_sort_scan(uint32_t* __restrict__ hist, uint32_t nblocks,
                                                     uint32_t* __restrict__ totals) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  uint32_t* row = hist + (size_t)blockIdx.x * nblocks;
  if (tid == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < nblocks; base += 1024) {
    const uint32_t i = base + tid;
    const uint32_t x = i < nblocks ? row[i] : 0u;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = s_warp[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t carry = s_carry;
    const uint32_t excl = carry + (warp ? s_warp[warp - 1] : 0u) + inc - x;
    if (i < nblocks) row[i] = excl;
    __syncthreads();
    if (tid == 0) s_carry = carry + s_warp[31];
    __syncthreads();
  }
  if (tid == 0) totals[blockIdx.x] = s_carry;
}

__global__ void __launch_bounds__(kThreads) k_sort_scatter(const uint32_t* __restrict__ keys_in,
                                                      const uint32_t* __restrict__ vals_in, int iota,
                                                      uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                      uint32_t n, int shift, uint32_t nblocks,
                                                      const uint32_t* __restrict__ hist,
                                                      const uint32_t* __restrict__ totals) {
  __shared__ uint32_t s_base[kBins];           // global base of each digit for this tile
  __shared__ uint32_t s_cnt[kWarps][kBins];    // per-warp digit counts of the current round
  __shared__ uint32_t s_pre[kWarps][kBins];    // per-warp digit prefix of the current round
  __shared__ uint32_t s_wsum[kWarps];
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;

  // Exclusive scan of the digit totals (256 values) -> digit base.
  {
    const uint32_t x = totals[tid];
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) s_wsum[warp] = inc;
    __syncthreads();
    uint32_t off = 0;
    for (int w = 0; w < warp; ++w) off += s_wsum[w];
    s_base[tid] = off + inc - x + hist[(size_t)tid * nblocks + blockIdx.x];
  }
  for (int w = 0; w < kWarps; ++w) s_cnt[w][tid] = 0;
  __syncthreads();

  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
  const uint32_t lt = (1u << lane) - 1u;
  for (int r = 0; r < kRounds; ++r) {
    const uint64_t idx = base + (uint64_t)r * kThreads + tid;
    const bool valid = idx < n;
    uint32_t key = 0, val = 0, d = kBins;
    if (valid) {
      key = keys_in[idx];
      val = iota ? (uint32_t)idx : vals_in[idx];
      d = (key >> shift) & 0xffu;
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t lrank = __popc(peers & lt);
    if (valid && lrank == 0) s_cnt[warp][d] = __popc(peers);
    __syncthreads();
    {
      // Thread tid owns digit tid: prefix of the per-warp counts in warp
      // order (warp w holds earlier keys than warp w+1 in this round).  The
      // round total is parked in s_cnt[0][tid] until the base is advanced.
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) {
        const uint32_t c = s_cnt[w][tid];
        s_pre[w][tid] = run;
        run += c;
        s_cnt[w][tid] = 0;
      }
      s_cnt[0][tid] = run;
    }
    __syncthreads();
    if (valid) {
      const uint32_t pos = s_base[d] + s_pre[warp][d] + lrank;
      keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads();
    s_base[tid] += s_cnt[0][tid];
    s_cnt[0][tid] = 0;
    __syncthreads();
  }
}

}  // namespace

uint32_t sort_blocks(uint32_t n) { return (n + kSortTile - 1) / kSortTile; }

size_t sort_hist_words(uint32_t n) { return (size_t)kBins * (sort_blocks(n) ? sort_blocks(n) : 1) + kBins; }

cudaError_t radix_sort_pairs(cudaStream_t stream, const uint32_t* keys_in, const uint32_t* vals_in,
                             uint32_t* keys_a, uint32_t* keys_b, uint32_t* vals_a, uint32_t* vals_b, uint32_t* hist,
                             uint32_t n, int key_bits, uint32_t** keys_out, uint32_t** vals_out, uint64_t* launches) {
  if (key_bits < 1) key_bits = 1;
  if (key_bits > 32) key_bits = 32;
  const int passes = (key_bits + 7) / 8;
  const uint32_t nblocks = sort_blocks(n);
  uint32_t* totals = hist + (size_t)kBins * (nblocks ? nblocks : 1);
  if (n == 0) {
    *keys_out = keys_a;
    *vals_out = vals_a;
    return cudaSuccess;
  }
  const uint32_t* kin = keys_in;
  const uint32_t* vin = vals_in;
  int iota = vals_in == nullptr ? 1 : 0;
  uint32_t* kout = keys_a;
  uint32_t* vout = vals_a;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    kout = (p % 2 == 0) ? keys_a : keys_b;
    vout = (p % 2 == 0) ? vals_a : vals_b;
    k_sort_hist<<<nblocks, kThreads, 0, stream>>>(kin, n, shift, nblocks, hist);
    k_sort_scan<<<kBins, 1024, 0, stream>>>(hist, nblocks, totals);
    k_sort_scatter<<<nblocks, kThreads, 0, stream>>>(kin, vin, iota, kout, vout, n, shift, nblocks, hist, totals);
    if (launches) *launches += 3;
    kin = kout;
    vin = vout;
    iota = 0;
  }
  *keys_out = kout;
  *vals_out = vout;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free sort: mpm_radix_sort_pairs_noalloc.
//
// For callers that cannot allocate device memory: code running inside a
// stream-ordered pipeline that must not stall (cudaMalloc and cudaFree can
// synchronise the device), hosts that reserve the whole device budget up
// front and forbid allocations afterwards, and hot paths held to an
// allocation-free guarantee.  The sort's ping-pong buffers and digit
// histograms live in the file-scope array below (8.25 MiB = 8,651,776 bytes,
// sized for kNoAllocMaxPairs pairs); every GPU that loads this library holds
// it until the process exits.

constexpr uint32_t kNoAllocMaxPairs = 1u << 20;  // 1,048,576 (key, value) pairs
constexpr size_t kNoAllocHistWords = (size_t)256 * ((kNoAllocMaxPairs + kSortTile - 1) / kSortTile) + 256;
constexpr size_t kNoAllocWords = 2ull * kNoAllocMaxPairs + kNoAllocHistWords;
static_assert(kNoAllocWords * 4 == 8651776, "the documented size of the allocation-free scratch");

// One key buffer, one value buffer and the histogram/digit totals.  In host
// code this name is only a stand-in for the device array, never a device
// address; the host obtains the address with cudaGetSymbolAddress.
static __device__ __align__(256) uint32_t g_noalloc_sort_scratch[kNoAllocWords];

namespace {
std::mutex g_noalloc_mu;
// Scratch address per CUDA context, keyed by the context's process-unique
// id: a symbol's device address belongs to the context that loaded the
// module, so a non-primary context, or a primary context recreated after
// cudaDeviceReset, gets its own lookup rather than a stale address.
struct NoAllocEntry {
  unsigned long long ctx_id;
  uint32_t* ptr;
};
std::vector<NoAllocEntry> g_noalloc_cache;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the context current on this thread; false if the driver cannot say.
bool current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q2 == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f2);
    resolved = true;
  }
  if (!get_current || !get_id) return false;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
  return get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of the scratch array in the current context: looked up
// with cudaGetSymbolAddress once per context (every call when the driver
// cannot identify the context).
cudaError_t noalloc_scratch(uint32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);  // makes the device's primary context current if none is
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  unsigned long long id = 0;
  const bool known = current_context_id(&id);
  if (known)
    for (const NoAllocEntry& en : g_noalloc_cache)
      if (en.ctx_id == id) {
        *out = en.ptr;
        return cudaSuccess;
      }
  uint32_t* p = nullptr;
  e = cudaGetSymbolAddress((void**)&p, g_noalloc_sort_scratch);
  if (e != cudaSuccess) return e;
  if (known) g_noalloc_cache.push_back({id, p});
  *out = p;
  return cudaSuccess;
}
}  // namespace

}  // namespace mpm

extern "C" int mpm_radix_sort_pairs_noalloc(uint32_t* d_keys, uint32_t* d_values, uint32_t n, uint32_t key_bits,
                                            void* stream) {
  using namespace mpm;
  if (n > kNoAllocMaxPairs) {
    set_last_error("mpm_radix_sort_pairs_noalloc: n=" + std::to_string(n) + " exceeds the allocation-free limit of " +
                   std::to_string(kNoAllocMaxPairs) + " pairs; use mpm_radix_sort_pairs_device");
    return MPM_ERR_INVALID;
  }
  if (key_bits < 1 || key_bits > 32) {
    set_last_error("mpm_radix_sort_pairs_noalloc: key_bits must be in 1..=32");
    return MPM_ERR_INVALID;
  }
  if (n == 0) {
    set_last_error("");
    return MPM_OK;
  }
  if (!d_keys || !d_values) {
    set_last_error("mpm_radix_sort_pairs_noalloc: null device pointer");
    return MPM_ERR_INVALID;
  }
  uint32_t* scratch = nullptr;
  cudaError_t e = noalloc_scratch(&scratch);
  if (e != cudaSuccess) {
    set_last_error(std::string("mpm_radix_sort_pairs_noalloc: scratch set-up failed: ") + cudaGetErrorString(e));
    return MPM_ERR_GPU;
  }
  cudaStream_t st = (cudaStream_t)stream;
  uint32_t* skeys = scratch;
  uint32_t* svals = scratch + kNoAllocMaxPairs;
  uint32_t* hist = scratch + 2ull * kNoAllocMaxPairs;
  const uint32_t nblocks = sort_blocks(n);
  uint32_t* totals = hist + (size_t)256 * nblocks;
  const int passes = ((int)key_bits + 7) / 8;
  // Even passes read the caller's arrays and write the scratch, odd passes
  // the reverse; every word of the histogram and totals is rewritten by each
  // pass, so nothing has to be cleared between calls.
  for (int p = 0; p < passes; ++p) {
    const bool to_scratch = (p % 2) == 0;
    const uint32_t* kin = to_scratch ? d_keys : skeys;
    const uint32_t* vin = to_scratch ? d_values : svals;
    uint32_t* kout = to_scratch ? skeys : d_keys;
    uint32_t* vout = to_scratch ? svals : d_values;
    k_sort_hist<<<nblocks, kThreads, 0, st>>>(kin, n, 8 * p, nblocks, hist);
    k_sort_scan<<<kBins, 1024, 0, st>>>(hist, nblocks, totals);
    k_sort_scatter<<<nblocks, kThreads, 0, st>>>(kin, vin, 0, kout, vout, n, 8 * p, nblocks, hist, totals);
  }
  if (passes % 2 == 1) {
    cudaMemcpyAsync(d_keys, skeys, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d_values, svals, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(std::string("mpm_radix_sort_pairs_noalloc: ") + cudaGetErrorString(e));
    return MPM_ERR_GPU;
  }
  set_last_error("");
  return MPM_OK;
}
