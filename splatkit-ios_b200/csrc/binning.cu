// Tile binning of the depth-sorted survivors. The reference rasterises instanced quads in four
// indirect batches (splatkit-ios/.../metal/raster/MetalSplatPipeline.mm:188-208,
// .../metal/cull/PrepareIndirect.metalh:4-21); this build composites 16x16 pixel tiles, so each
// survivor is listed once per tile its quad touches.
//
// The visibility pass already decided each survivor's tiles (a span, sk_tiles.cuh). Binning walks
// the depth-sorted list in blocks of 1024 ranks: one pass sums each block's tile count, the next
// adds up the sums of the blocks before its own (no block waits on another) and writes
// (tile id, projected index) pairs at its offsets. Offsets grow with depth rank and the tile sort
// that follows is stable, so every tile's list stays front to back. A count beyond the reserved
// capacity is recorded and nothing past it is written; the host grows the buffers and draws
// again.
#include <cuda_runtime.h>

#include "sk_device.cuh"
#include "sk_kernels.h"
#include "sk_launch.cuh"
#include "sk_tiles.cuh"

namespace sk {
namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kItems = 4;
constexpr uint32_t kTileSplats = kThreads * kItems;

// Pass 1: instances per block of 1024 depth ranks (no waiting on other blocks).
__global__ void __launch_bounds__(kThreads) binCountKernel(const __grid_constant__ BinArgs a) {
  chainedKernelStart();
  __shared__ uint32_t warpSum[kThreads / 32];
  const uint32_t n = min(*a.count, a.capacity);
  const uint32_t block = blockIdx.x;
  if (block * kTileSplats >= n) return;
  uint32_t sum = 0;
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    const uint32_t i = block * kTileSplats + r * kThreads + threadIdx.x;
    if (i < n) sum += spanCount(__ldg(a.spans + __ldg(a.order + i)));
  }
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if (laneId() == 0) warpSum[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t total = 0;
    for (uint32_t w = 0; w < kThreads / 32; ++w) total += warpSum[w];
    a.blockSums[block] = total;
  }
}

// The block's items for the emission loop.
struct ItemStage {
  uint4 span[kTileSplats];
  uint32_t value[kTileSplats];   // projected index
  uint32_t offset[kTileSplats];  // first position in the block's output range
  uint2 grid[kTileSplats];       // batch: (first tile id, tiles per row) of the item's view
  uint32_t total;
};

// The tile ids of one item's box: id(b) for box position b = row * w + col (boxCell).
struct TileGrid {
  uint32_t rowStart, tilesX;
  __device__ __forceinline__ uint32_t id(uint32_t b, uint32_t w) const {
    return boxCell(rowStart, b, w, tilesX);
  }
};

template <bool kBatch>
__device__ __forceinline__ TileGrid gridOf(const BinArgs& a, const ItemStage& stage, uint32_t j,
                                           const uint4 sp) {
  const uint32_t x0 = sp.x & 0xffffu, y0 = sp.x >> 16;
  if constexpr (kBatch) {
    const uint2 g = stage.grid[j];
    return TileGrid{g.x + y0 * g.y + x0, g.y};
  }
  return TileGrid{y0 * a.tilesX + x0, a.tilesX};
}

// Pass 2: each block sums the totals of the blocks before it, then writes its instances.
// kBatch: the survivors are a batch's views back to back in depth-rank order (rank i belongs to
// view v when viewFirst[v] <= i < viewFirst[v + 1]); tile ids are batch-wide.
template <bool kBatch, bool kBalanced>
__global__ void __launch_bounds__(kThreads) binEmitKernel(const __grid_constant__ BinArgs a) {
  chainedKernelStart();
  __shared__ uint32_t warpBase[kThreads / 32];
  __shared__ ItemStage stage;
  __shared__ uint32_t tileBase;
  const uint32_t n = min(*a.count, a.capacity);
  const uint32_t tiles = (n + kTileSplats - 1) / kTileSplats;
  const uint32_t tile = blockIdx.x;
  if (tile == 0 && threadIdx.x == 0 && tiles == 0) {
    *a.instanceCount = 0;
    *a.overflow = 0;
  }
  if (tile < tiles) {
    {
      uint32_t before = 0;
      for (uint32_t b = threadIdx.x; b < tile; b += kThreads) before += __ldcg(a.blockSums + b);
      for (int o = 16; o > 0; o >>= 1) before += __shfl_xor_sync(0xffffffffu, before, o);
      if (laneId() == 0) warpBase[threadIdx.x >> 5] = before;
      __syncthreads();
      if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (uint32_t w = 0; w < kThreads / 32; ++w) s += warpBase[w];
        tileBase = s;
        if (tile == tiles - 1) {
          const uint32_t total = s + __ldcg(a.blockSums + tile);
          *a.instanceCount = total;
          *a.overflow = total > a.instanceCapacity ? 1u : 0u;
        }
      }
      __syncthreads();
    }
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    uint32_t value[kItems], cnt[kItems];
    uint4 span[kItems];
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      const uint32_t i = tile * kTileSplats + warp * (32 * kItems) + r * 32 + lane;
      value[r] = i < n ? __ldg(a.order + i) : 0xffffffffu;
    }
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      span[r] = value[r] != 0xffffffffu ? __ldg(a.spans + value[r]) : make_uint4(0, 0, 0, 0);
      cnt[r] = spanCount(span[r]);
    }
    // Offsets in (warp, row, lane) order = depth order.
    uint32_t rowExclusive[kItems];
    uint32_t warpRun = 0;
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      uint32_t inc = cnt[r];
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= static_cast<uint32_t>(o)) inc += up;
      }
      rowExclusive[r] = warpRun + inc - cnt[r];
      warpRun += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) warpBase[warp] = warpRun;
    __syncthreads();
    if (warp == 0) {
      const uint32_t w = lane < kThreads / 32 ? warpBase[lane] : 0u;
      uint32_t inc = w;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= static_cast<uint32_t>(o)) inc += up;
      }
      if (lane < kThreads / 32) warpBase[lane] = inc - w;
    }
    __syncthreads();
    // Stage the block's items: span, projected index, first position in the block's output
    // range [0, total) (from tileBase on), and for a batch the view's tile grid.
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      const uint32_t at = warp * (32 * kItems) + r * 32 + lane;
      stage.span[at] = span[r];
      stage.value[at] = value[r];
      stage.offset[at] = warpBase[warp] + rowExclusive[r];
      if constexpr (kBatch) {
        const uint32_t i = tile * kTileSplats + at;
        uint32_t lo = 0, hi = a.viewCount;
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) / 2;
          if (__ldg(a.viewFirst + mid) <= i) lo = mid; else hi = mid;
        }
        stage.grid[at] = make_uint2(__ldg(&a.views[lo].binBase), __ldg(&a.views[lo].binsX));
      }
    }
    if (warp == kThreads / 32 - 1 && lane == 31) stage.total = warpBase[warp] + warpRun;
    __syncthreads();
    const uint32_t itemsBegin = warp * (32 * kItems), itemsEnd = itemsBegin + 32 * kItems;
    const uint32_t outBegin = stage.offset[itemsBegin];
    const uint32_t outEnd = warp + 1 < kThreads / 32 ? stage.offset[itemsEnd] : stage.total;
    if constexpr (!kBalanced) {
      // One item at a time, all lanes together: each store covers a contiguous run of the
      // output (the item's tiles in increasing box order). Lane l takes box tiles l and l + 32
      // of a masked span, or every 32nd tile of a span that lists its whole box. Few
      // instructions per instance are spent when most items have few tiles, but the warp walks
      // its items one by one: the better choice when the grid is about one wave.
      const uint32_t below = lanemaskLt();
#pragma unroll
      for (uint32_t r = 0; r < kItems; ++r) {
        uint32_t pending = __ballot_sync(0xffffffffu, cnt[r] != 0);
        while (pending) {
          const uint32_t j = itemsBegin + r * 32 + (__ffs(pending) - 1);
          pending &= pending - 1;
          const uint4 sp = stage.span[j];
          const uint32_t val = stage.value[j], first = tileBase + stage.offset[j];
          const uint32_t w = sp.y & 0xffffu, area = sp.y >> 16;
          const TileGrid g = gridOf<kBatch>(a, stage, j, sp);
          auto emit = [&](uint32_t k, uint32_t slot) {
            if (slot < a.instanceCapacity) {
              a.instanceKeys[slot] = g.id(k, w);
              a.instanceValues[slot] = val;
            }
          };
          if (area > 64) {
            for (uint32_t k = lane; k < area; k += 32) emit(k, first + k);
          } else {
            if ((sp.z >> lane) & 1u) emit(lane, first + __popc(sp.z & below));
            if (sp.w != 0u && ((sp.w >> lane) & 1u))
              emit(lane + 32, first + __popc(sp.z) + __popc(sp.w & below));
          }
        }
      }
    } else {
      // Load-balanced over the warp's output range: lane l writes positions l, l + 32, ..., so
      // every store is 32 consecutive slots whatever the items' sizes. The item holding
      // position p is the last of the warp's items whose offset is <= p (a 7-step search in
      // shared memory) and its k-th tile is decoded from the span: fewer instructions per
      // instance than the item walk, the better choice for grids of many waves.
      for (uint32_t p = outBegin + lane; p < outEnd; p += 32) {
        uint32_t lo = itemsBegin, hi = itemsEnd;
#pragma unroll
        for (int step = 0; step < 7; ++step) {
          const uint32_t mid = (lo + hi) / 2;
          if (stage.offset[mid] <= p) lo = mid; else hi = mid;
        }
        const uint32_t j = lo, k = p - stage.offset[j];
        const uint4 sp = stage.span[j];
        const uint32_t w = sp.y & 0xffffu, area = sp.y >> 16;
        uint32_t bit = k;  // box position of the k-th listed tile
        if (area <= 64) {
          const uint32_t nlo = __popc(sp.z);
          bit = k < nlo ? kthSetBit(sp.z, k) : 32u + kthSetBit(sp.w, k - nlo);
        }
        const uint32_t slot = tileBase + p;
        if (slot < a.instanceCapacity) {
          a.instanceKeys[slot] = gridOf<kBatch>(a, stage, j, sp).id(bit, w);
          a.instanceValues[slot] = stage.value[j];
        }
      }
    }
  }
}

__global__ void rangesKernel(const uint32_t* __restrict__ keys, const uint32_t* count,
                             uint32_t capacity, uint2* ranges, uint32_t tiles) {
  chainedKernelStart();
  const uint32_t n = min(*count, capacity);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    if (k >= tiles) continue;
    if (i == 0 || keys[i - 1] != k) ranges[k].x = i;
    if (i + 1 == n || keys[i + 1] != k) ranges[k].y = i + 1;
  }
}

}  // namespace

uint32_t binBlocks(uint32_t capacity) { return max(1u, (capacity + kTileSplats - 1) / kTileSplats); }

cudaError_t launchBinning(const BinArgs& a, cudaStream_t stream) {
  const uint32_t grid = binBlocks(a.capacity);
  cudaError_t e = launchChained(binCountKernel, grid, kThreads, stream, a);
  if (e != cudaSuccess) return e;
  if (a.viewCount > 0) {
    e = launchChained(a.balanced ? binEmitKernel<true, true> : binEmitKernel<true, false>, grid,
                      kThreads, stream, a);
  } else {
    e = launchChained(a.balanced ? binEmitKernel<false, true> : binEmitKernel<false, false>, grid,
                      kThreads, stream, a);
  }
  return e;
}

cudaError_t clearTileRanges(uint2* ranges, uint32_t tiles, cudaStream_t stream) {
  return cudaMemsetAsync(ranges, 0, static_cast<size_t>(tiles) * sizeof(uint2), stream);
}

cudaError_t launchTileRanges(const uint32_t* sortedKeys, const uint32_t* instanceCount,
                             uint32_t instanceCapacity, uint2* ranges, uint32_t tiles,
                             cudaStream_t stream) {
  const uint32_t grid = max(1u, min(148u * 8u, (instanceCapacity + 255u) / 256u));
  return launchChained(rangesKernel, grid, 256, stream, sortedKeys, instanceCount, instanceCapacity,
                       ranges, tiles);
}

}  // namespace sk
