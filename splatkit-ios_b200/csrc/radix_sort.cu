// Onesweep LSD radix sort of 32-bit keys with 8-bit digits: stable and ascending, the
// contract of splatkit-ios/.../metal/sort/MetalRadixSort.h:13-19 (an argsort whose first pass
// takes each key's position as its value; the last pass skips the key write unless asked).
//
// The reference runs histogram -> scan -> scatter per pass (SplatRadixSort.metal:17-171). Here:
//   1. one upfront pass reads every key once and builds all digit histograms; the block that
//      finishes last turns them into exclusive digit bases;
//   2. one scatter pass per digit. Each tile (2048, 4096 or 6144 keys, 4096 by default) ranks
//      its keys per warp with ballot matching (8 ballots per row, rows in source order, so
//      ranking is stable), publishes
//      its per-digit counts, and learns how many keys of each digit the tiles before it hold
//      by decoupled look-back (bounded waits), then reorders locally in shared memory and
//      writes each digit run contiguously.
// Tiles are handed out by an atomic counter, so a tile only waits on tiles already running.
#include <cuda_runtime.h>

#include "sk_device.cuh"
#include "sk_kernels.h"
#include "sk_launch.cuh"

namespace sk {
namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kWarps = kThreads / 32;
constexpr uint32_t kPerThread = 16;
constexpr uint32_t kTileKeys = kThreads * kPerThread;  // 4096
constexpr uint32_t kBins = 256;
constexpr uint32_t kMaxPasses = 4;

__device__ __forceinline__ uint32_t clampCount(const uint32_t* count, uint32_t capacity) {
  return min(*count, capacity);
}

// ---- 1. all-digit histogram ------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
    histogramKernel(const uint32_t* __restrict__ keys, const uint32_t* count, uint32_t capacity,
                    uint32_t passes, uint32_t* accum, uint32_t* bases, uint32_t* counters) {
  chainedKernelStart();
  __shared__ uint32_t h[kMaxPasses][kBins];
  for (uint32_t i = threadIdx.x; i < kMaxPasses * kBins; i += kThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  const uint32_t n = clampCount(count, capacity);
  const uint32_t stride = gridDim.x * kThreads * 4;  // keys per grid step of one uint4 per thread
  // four 16-byte loads in flight per thread, then their 16 keys counted
  for (uint32_t base = (blockIdx.x * kThreads + threadIdx.x) * 4; base < n; base += stride * 4) {
    uint4 v[4];
#pragma unroll
    for (uint32_t q = 0; q < 4; ++q) {
      const uint32_t i = base + q * stride;
      if (i + 3 < n) {
        v[q] = __ldg(reinterpret_cast<const uint4*>(keys + i));
      } else {
        v[q].x = i < n ? keys[i] : 0u;
        v[q].y = i + 1 < n ? keys[i + 1] : 0u;
        v[q].z = i + 2 < n ? keys[i + 2] : 0u;
        v[q].w = i + 3 < n ? keys[i + 3] : 0u;
      }
    }
#pragma unroll
    for (uint32_t q = 0; q < 4; ++q) {
      const uint32_t i = base + q * stride;
      const uint32_t k[4] = {v[q].x, v[q].y, v[q].z, v[q].w};
      for (uint32_t j = 0; j < 4; ++j) {
        if (i + j >= n) break;
        for (uint32_t p = 0; p < passes; ++p) atomicAdd(&h[p][(k[j] >> (8 * p)) & 0xffu], 1u);
      }
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < passes * kBins; i += kThreads) {
    const uint32_t v = (&h[0][0])[i];
    if (v) atomicAdd(&accum[i], v);
  }
  if (finishTile(counters)) finishDigitHistograms(accum, bases, passes);
}

// ---- 2. onesweep scatter ----------------------------------------------------------------
// Lanes of this warp whose digit equals this lane's (among valid lanes): 8 ballots.
__device__ __forceinline__ uint32_t matchDigit(uint32_t digit, bool valid) {
  uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
  for (uint32_t b = 0; b < 8; ++b) {
    const bool bit = (digit >> b) & 1u;
    const uint32_t vote = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? vote : ~vote;
  }
  return peers;
}

template <uint32_t kPer>
struct ScatterSmem {
  uint32_t warpCount[kWarps][kBins];
  uint32_t digitTotal[kBins];
  uint32_t localOffset[kBins];
  uint32_t globalBase[kBins];
  uint32_t stage[kThreads * kPer];
  uint32_t warpSums[kWarps];
};

// kPer keys per thread: tiles of 256 * kPer keys (the tile size the autotuner picks from).
template <bool kImplicitValues, bool kWriteKeys, uint32_t kPer>
__global__ void __launch_bounds__(kThreads)
    scatterKernel(const uint32_t* __restrict__ keysIn, const uint32_t* __restrict__ valuesIn,
                  uint32_t* __restrict__ keysOut, uint32_t* __restrict__ valuesOut,
                  const uint32_t* count, uint32_t capacity, uint32_t shift,
                  const uint32_t* __restrict__ digitBase, uint64_t* status, uint32_t* counters,
                  uint32_t epoch, uint32_t* error, uint32_t withheldPlusOne) {
  chainedKernelStart();
  __shared__ ScatterSmem<kPer> s;
  constexpr uint32_t kTile = kThreads * kPer;
  const uint32_t tile = takeTile(counters);
  const uint32_t n = clampCount(count, capacity);
  const uint32_t tiles = (n + kTile - 1) / kTile;
  if (tile < tiles) {
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    for (uint32_t i = threadIdx.x; i < kWarps * kBins; i += kThreads) (&s.warpCount[0][0])[i] = 0;
    uint32_t key[kPer];
    const uint32_t first = tile * kTile + warp * (32 * kPer) + lane;
#pragma unroll
    for (uint32_t r = 0; r < kPer; ++r) {
      const uint32_t e = first + r * 32;
      key[r] = e < n ? keysIn[e] : 0xffffffffu;
    }
    __syncthreads();
    // Rank each key among the equal digits of its warp, row by row (source order).
    uint32_t rank[kPer];
    const uint32_t below = lanemaskLt();
#pragma unroll
    for (uint32_t r = 0; r < kPer; ++r) {
      const bool valid = first + r * 32 < n;
      const uint32_t d = (key[r] >> shift) & 0xffu;
      const uint32_t peers = matchDigit(d, valid);
      const uint32_t base = s.warpCount[warp][d];
      __syncwarp();
      if (valid && (peers & below) == 0u) s.warpCount[warp][d] = base + __popc(peers);
      __syncwarp();
      rank[r] = base + __popc(peers & below);
    }
    __syncthreads();
    // Per digit: exclusive offsets across warps and the tile's total.
    const uint32_t d = threadIdx.x;
    uint32_t total = 0;
#pragma unroll
    for (uint32_t w = 0; w < kWarps; ++w) {
      const uint32_t c = s.warpCount[w][d];
      s.warpCount[w][d] = total;
      total += c;
    }
    s.digitTotal[d] = total;
    // Publish, then look back over earlier tiles for this digit. A tile named by the test hook
    // (withheldPlusOne = tile + 1; 0 names none) publishes nothing, so its successors' bounded
    // waits run out.
    uint64_t* mine = status + static_cast<size_t>(tile) * kBins + d;
    const bool publish = tile + 1u != withheldPlusOne;
    uint32_t exclusive = 0;
    if (tile == 0) {
      if (publish) storeStatus(mine, makeStatus(epoch, kFlagPrefix, total));
    } else {
      if (publish) storeStatus(mine, makeStatus(epoch, kFlagAggregate, total));
      for (int j = static_cast<int>(tile) - 1; j >= 0; --j) {
        const uint64_t w = waitStatus(status + static_cast<size_t>(j) * kBins + d, epoch, error);
        exclusive += static_cast<uint32_t>(w);
        if (((w >> 32) & 3u) == kFlagPrefix) break;
      }
      if (publish) storeStatus(mine, makeStatus(epoch, kFlagPrefix, exclusive + total));
    }
    s.globalBase[d] = digitBase[d] + exclusive;
    // Exclusive scan of the tile's digit totals: where each digit's run starts locally.
    uint32_t inc = total;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= static_cast<uint32_t>(o)) inc += up;
    }
    if (lane == 31) s.warpSums[warp] = inc;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t w = 0; w < warp; ++w) before += s.warpSums[w];
    s.localOffset[d] = before + inc - total;
    __syncthreads();
    // Local positions, keys staged in digit order.
    uint32_t pos[kPer];
#pragma unroll
    for (uint32_t r = 0; r < kPer; ++r) {
      const bool valid = first + r * 32 < n;
      const uint32_t dd = (key[r] >> shift) & 0xffu;
      pos[r] = valid ? s.localOffset[dd] + s.warpCount[warp][dd] + rank[r] : 0xffffffffu;
      if (valid) s.stage[pos[r]] = key[r];
    }
    __syncthreads();
    const uint32_t inTile = min(kTile, n - tile * kTile);
    uint32_t dst[kPer];
#pragma unroll
    for (uint32_t r = 0; r < kPer; ++r) {
      const uint32_t i = threadIdx.x + r * kThreads;
      dst[r] = 0xffffffffu;
      if (i < inTile) {
        const uint32_t k = s.stage[i];
        const uint32_t dd = (k >> shift) & 0xffu;
        const uint32_t at = s.globalBase[dd] + (i - s.localOffset[dd]);
        // Only a look-back that gave up can put `at` past the end; never write there.
        if (at < n) {
          dst[r] = at;
          if (kWriteKeys) keysOut[at] = k;
        } else {
          atomicOr(error, SK_DEVERR_BOUNDS);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (uint32_t r = 0; r < kPer; ++r) {
      const uint32_t e = first + r * 32;
      if (pos[r] != 0xffffffffu) s.stage[pos[r]] = kImplicitValues ? e : valuesIn[e];
    }
    __syncthreads();
#pragma unroll
    for (uint32_t r = 0; r < kPer; ++r) {
      const uint32_t i = threadIdx.x + r * kThreads;
      if (i < inTile && dst[r] != 0xffffffffu) valuesOut[dst[r]] = s.stage[i];
    }
  }
  finishTile(counters);
}

inline size_t alignUp(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace

uint32_t sortTileKeys() { return kTileKeys; }

uint32_t* sortDigitAccumulators(const SortArgs& a) { return a.histogram; }
uint32_t* sortDigitBases(const SortArgs& a) { return a.histogram + kMaxPasses * kBins; }

static uint32_t sortTiles(uint32_t capacity, uint32_t tileKeys = kTileKeys) {
  return max(1u, (capacity + tileKeys - 1) / tileKeys);
}

static uint32_t tileKeysOf(const SortArgs& a) { return a.tileKeys ? a.tileKeys : kTileKeys; }

size_t sortWorkspaceBytesFor(uint32_t capacity, uint32_t minTileKeys) {
  const size_t n = alignUp(static_cast<size_t>(max(capacity, 1u)) * 4, 256);
  return 3 * n                                             // keysA, keysB, valuesTmp
         + alignUp(2 * kMaxPasses * kBins * 4, 256)        // histogram accumulators + bases
         + alignUp(static_cast<size_t>(sortTiles(capacity, minTileKeys)) * kBins * 8, 256)  // status
         + alignUp((kMaxPasses + 1) * 2 * 4, 256);         // counters
}

size_t sortWorkspaceBytes(uint32_t capacity) { return sortWorkspaceBytesFor(capacity, kTileKeys); }

void sortBindWorkspaceFor(SortArgs& a, void* workspace, uint32_t capacity, uint32_t minTileKeys) {
  char* p = static_cast<char*>(workspace);
  const size_t n = alignUp(static_cast<size_t>(max(capacity, 1u)) * 4, 256);
  a.keysA = reinterpret_cast<uint32_t*>(p), p += n;
  a.keysB = reinterpret_cast<uint32_t*>(p), p += n;
  a.valuesTmp = reinterpret_cast<uint32_t*>(p), p += n;
  a.histogram = reinterpret_cast<uint32_t*>(p), p += alignUp(2 * kMaxPasses * kBins * 4, 256);
  a.status = reinterpret_cast<uint64_t*>(p);
  a.statusTiles = sortTiles(capacity, minTileKeys);
  p += alignUp(static_cast<size_t>(a.statusTiles) * kBins * 8, 256);
  a.counters = reinterpret_cast<uint32_t*>(p);
}

void sortBindWorkspace(SortArgs& a, void* workspace, uint32_t capacity) {
  sortBindWorkspaceFor(a, workspace, capacity, kTileKeys);
}

cudaError_t sortResetWorkspace(const SortArgs& a, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(a.histogram, 0, 2 * kMaxPasses * kBins * 4, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(a.counters, 0, (kMaxPasses + 1) * 2 * 4, stream);
  return e;
}

cudaError_t launchSort(const SortArgs& a, cudaStream_t stream) {
  const uint32_t passes = static_cast<uint32_t>(min(max(a.bits, 8), 32) + 7) / 8u;
  const uint32_t tileKeys = tileKeysOf(a);
  if (tileKeys != 2048 && tileKeys != 4096 && tileKeys != 6144) return cudaErrorInvalidValue;
  const uint32_t tiles = sortTiles(a.capacity, tileKeys);
  if (tiles > a.statusTiles) return cudaErrorInvalidValue;  // the workspace was bound for larger tiles
  uint32_t* accum = a.histogram;
  uint32_t* bases = a.histogram + kMaxPasses * kBins;
  cudaError_t e = cudaSuccess;
  if (!a.basesReady) {
    const uint32_t histBlocks = min(sortTiles(a.capacity), 148u * 4u);
    e = launchChained(histogramKernel, histBlocks, kThreads, stream, a.keysIn, a.count, a.capacity,
                      passes, accum, bases, a.counters);
    if (e != cudaSuccess) return e;
  }
  const uint32_t* kin = a.keysIn;
  const uint32_t* vin = a.valuesIn;
  for (uint32_t p = 0; p < passes; ++p) {
    const bool last = p + 1 == passes;
    uint32_t* kout = last ? a.keysOut : (p % 2 == 0 ? a.keysA : a.keysB);
    uint32_t* vout = ((passes - 1 - p) % 2 == 0) ? a.valuesOut : a.valuesTmp;
    uint32_t* counters = a.counters + 2 * (p + 1);
    const uint32_t epoch = (a.epoch + p) & 0x3fffffffu;
    const bool implicit = p == 0 && vin == nullptr;
    const bool writeKeys = kout != nullptr;
#define SK_SCATTER_PER(IMPLICIT, WRITE, PER)                                               \
  e = launchChained(scatterKernel<IMPLICIT, WRITE, PER>, tiles, kThreads, stream, kin, vin,  \
                    kout, vout, a.count, a.capacity, 8 * p, bases + p * kBins, a.status,   \
                    counters, epoch, a.error, p == 0 ? a.withheldTilePlusOne : 0u)
#define SK_SCATTER(IMPLICIT, WRITE)                                                        \
  do {                                                                                     \
    if (tileKeys == 2048) SK_SCATTER_PER(IMPLICIT, WRITE, 8u);                             \
    else if (tileKeys == 6144) SK_SCATTER_PER(IMPLICIT, WRITE, 24u);                       \
    else SK_SCATTER_PER(IMPLICIT, WRITE, 16u);                                             \
  } while (0)
    if (implicit) {
      if (writeKeys) SK_SCATTER(true, true); else SK_SCATTER(true, false);
    } else {
      if (writeKeys) SK_SCATTER(false, true); else SK_SCATTER(false, false);
    }
#undef SK_SCATTER
#undef SK_SCATTER_PER
    if (e != cudaSuccess) return e;
    kin = kout;
    vin = vout;
  }
  return cudaGetLastError();
}

}  // namespace sk
