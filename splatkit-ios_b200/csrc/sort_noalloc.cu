// sk_radix_argsort_noalloc: the device argsort of sk_radix_argsort_device with its workspace in
// a fixed array that lives in this module, for callers that may not allocate device memory
// while they run: a render callback with a frame deadline (cudaMalloc and cudaFree
// synchronise the whole device), a host thread that must not take the allocator's locks, or
// code that enqueues work between the two halves of a frame and owns no device allocator.
//
// The scratch holds the key and value ping-pong buffers, the histogram accumulators, the
// look-back status words and the tile counters of the onesweep sort (radix_sort.cu) for up to
// SK_NOALLOC_SORT_MAX_KEYS keys. Its address is looked up once per device, on the first call
// made while that device is current.
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>

#include "../../include/splatkit_b200.h"
#include "sk_kernels.h"

namespace sk {
namespace {

// The workspace size of radix_sort.cu's layout for SK_NOALLOC_SORT_MAX_KEYS keys: three
// 4-byte-per-key buffers, 2 x 4 x 256 histogram words, one 256-word status row of 8-byte words
// per 4096-key tile, and the counters, each part rounded up to 256 bytes. The first call checks
// it against sortWorkspaceBytes() and refuses to run if the layout ever outgrows it.
constexpr size_t roundUp256(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kNoAllocKeys = SK_NOALLOC_SORT_MAX_KEYS;
constexpr size_t kNoAllocScratchBytes = 3 * roundUp256(kNoAllocKeys * 4) + roundUp256(2 * 4 * 256 * 4) +
                                        roundUp256((kNoAllocKeys + 4095) / 4096 * 256 * 8) +
                                        roundUp256(5 * 2 * 4);

// Zero when the module loads. The histogram accumulators and the tile counters must be zero
// when a sort starts: every completed sort leaves them at zero, and each call clears them again
// before it sorts (two small memsets on the caller's stream), so a sort cut short by an error
// cannot poison the next one. The status words need no clearing while the 30-bit epochs are
// new: each call takes four (one per pass). When the epoch counter wraps, after 2^28 calls, the
// call that wraps it zeroes the status words first (a flag of 0 never matches), so a word left
// by a sort 2^28 calls earlier cannot pass for one of the new epochs.
static __device__ __align__(256) unsigned char gSortScratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::atomic<void*> gScratchOnDevice[kMaxDevices];
std::atomic<uint32_t> gEpoch{1};

// The scratch's device address on the current device: looked up on the first call per device.
void* scratchAddress(int device) {
  void* p = gScratchOnDevice[device].load(std::memory_order_acquire);
  if (p) return p;
  if (cudaGetSymbolAddress(&p, gSortScratch) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  gScratchOnDevice[device].store(p, std::memory_order_release);
  return p;
}

}  // namespace
}  // namespace sk

extern "C" sk_status sk_radix_argsort_noalloc(const uint32_t* d_keys, const uint32_t* d_count,
                                              uint32_t capacity, int32_t bits, uint32_t* d_order,
                                              uint32_t* d_error, void* stream) {
  if (!d_keys || !d_count || !d_order || !d_error) return SK_E_INVALID;
  if (bits != 16 && bits != 32) return SK_E_INVALID;
  if (capacity > SK_NOALLOC_SORT_MAX_KEYS) return SK_E_LIMIT;
  if (sk::sortWorkspaceBytes(SK_NOALLOC_SORT_MAX_KEYS) > sk::kNoAllocScratchBytes) return SK_E_LIMIT;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= sk::kMaxDevices) {
    cudaGetLastError();
    return SK_E_DEVICE;
  }
  void* scratch = sk::scratchAddress(device);
  if (!scratch) return SK_E_DEVICE;
  sk::SortArgs a{};
  a.keysIn = d_keys;
  a.valuesIn = nullptr;
  a.keysOut = nullptr;
  a.valuesOut = d_order;
  a.count = d_count;
  a.capacity = capacity;
  a.bits = bits;
  // The layout of the largest sort, whatever the capacity: the status words then always sit
  // at the same place and the region never holds anything but status words.
  sk::sortBindWorkspace(a, scratch, SK_NOALLOC_SORT_MAX_KEYS);
  const uint32_t raw = sk::gEpoch.fetch_add(4);
  a.epoch = raw & 0x3fffffffu;
  a.error = d_error;
  const auto s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaSuccess;
  if (a.epoch == 1 && raw != 1)  // the counter wrapped: the old status words could match again
    e = cudaMemsetAsync(a.status, 0, static_cast<size_t>(a.statusTiles) * 256 * 8, s);
  if (e == cudaSuccess) e = sk::sortResetWorkspace(a, s);
  if (e == cudaSuccess) e = sk::launchSort(a, s);
  return e == cudaSuccess ? SK_OK : SK_E_DEVICE;
}
