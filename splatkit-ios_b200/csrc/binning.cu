// Tile binning of the depth-sorted survivors. The reference rasterises instanced quads in four
// indirect batches (splatkit-ios/.../metal/raster/MetalSplatPipeline.mm:188-208,
// .../metal/cull/PrepareIndirect.metalh:4-21); this build composites 16x16 pixel tiles, so each
// survivor is listed once per tile its quad can touch.
//
// One kernel walks the sorted list, counts each splat's tiles from the quad's pixel box
// (radius * (|a1| + |a2|) per axis, the same box the cull's edge test bounds, plus one pixel),
// takes its output offset by decoupled look-back, and writes (tile id, projected index) pairs.
// Offsets grow with depth rank, and the tile sort that follows is stable, so every tile's list
// stays front to back. A count beyond the reserved capacity is recorded and nothing past it
// is written; the host grows the buffers and redraws.
#include <cuda_runtime.h>

#include "sk_device.cuh"
#include "sk_kernels.h"

namespace sk {
namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kItems = 4;
constexpr uint32_t kTileSplats = kThreads * kItems;

struct TileRect {
  uint32_t x0, y0, x1, y1;  // inclusive tile bounds; empty when x0 > x1
};

__device__ __forceinline__ TileRect tileRect(const uint4 lo, const uint4 hi, float width,
                                             float height, uint32_t tilesX, uint32_t tilesY) {
  TileRect t{1, 1, 0, 0};
  const float cx = (asF(lo.x) + 1.0f) * (0.5f * width);
  const float cy = (asF(lo.y) + 1.0f) * (0.5f * height);  // y up
  const float r = asF(hi.z);
  const float ex = r * (fabsf(lowHalf(lo.z)) + fabsf(lowHalf(lo.w))) + 1.0f;
  const float ey = r * (fabsf(highHalf(lo.z)) + fabsf(highHalf(lo.w))) + 1.0f;
  if (!(isfinite(cx) && isfinite(cy) && isfinite(ex) && isfinite(ey))) return t;
  const float xa = floorf(cx - ex), xb = ceilf(cx + ex);
  const float ya = floorf(cy - ey), yb = ceilf(cy + ey);
  if (xb < 0.0f || xa >= width || yb < 0.0f || ya >= height) return t;
  // columns [c0, c1]; rows from the y-up box: row = H - y_up - 0.5
  const uint32_t c0 = static_cast<uint32_t>(fmaxf(xa, 0.0f));
  const uint32_t c1 = static_cast<uint32_t>(fminf(xb, width - 1.0f));
  const uint32_t r0 = static_cast<uint32_t>(fmaxf(height - yb - 1.0f, 0.0f));
  const uint32_t r1 = static_cast<uint32_t>(fminf(fmaxf(height - ya, 0.0f), height - 1.0f));
  t.x0 = c0 / kTileSize;
  t.x1 = min(c1 / kTileSize, tilesX - 1);
  t.y0 = r0 / kTileSize;
  t.y1 = min(r1 / kTileSize, tilesY - 1);
  return t;
}

__global__ void __launch_bounds__(kThreads) binKernel(const __grid_constant__ BinArgs a) {
  __shared__ uint32_t warpBase[kThreads / 32];
  __shared__ uint32_t tileBase;
  const uint32_t tile = takeTile(a.counters);
  const uint32_t n = min(*a.count, a.capacity);
  const uint32_t tiles = (n + kTileSplats - 1) / kTileSplats;
  const float width = static_cast<float>(a.width), height = static_cast<float>(a.height);
  if (tile < tiles) {
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    TileRect rect[kItems];
    uint32_t value[kItems];
    uint32_t cnt[kItems];
    uint32_t mine = 0;
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      const uint32_t i = tile * kTileSplats + warp * (32 * kItems) + r * 32 + lane;
      cnt[r] = 0;
      value[r] = 0;
      if (i < n) {
        value[r] = a.order[i];
        const uint4* p = reinterpret_cast<const uint4*>(a.projected + value[r]);
        rect[r] = tileRect(__ldg(p), __ldg(p + 1), width, height, a.tilesX, a.tilesY);
        if (rect[r].x0 <= rect[r].x1 && rect[r].y0 <= rect[r].y1)
          cnt[r] = (rect[r].x1 - rect[r].x0 + 1) * (rect[r].y1 - rect[r].y0 + 1);
      }
      mine += cnt[r];
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
      const uint32_t aggregate = __shfl_sync(0xffffffffu, inc, 31);
      if (lane < kThreads / 32) warpBase[lane] = inc - w;
      uint32_t exclusive = 0;
      if (tile == 0) {
        if (lane == 0) storeStatus(a.status, makeStatus(a.epoch, kFlagPrefix, aggregate));
      } else {
        if (lane == 0) storeStatus(a.status + tile, makeStatus(a.epoch, kFlagAggregate, aggregate));
        exclusive = warpLookback(a.status, tile, a.epoch, a.error);
        if (lane == 0)
          storeStatus(a.status + tile, makeStatus(a.epoch, kFlagPrefix, exclusive + aggregate));
      }
      if (lane == 0) {
        tileBase = exclusive;
        if (tile == tiles - 1) {
          const uint32_t total = exclusive + aggregate;
          *a.instanceCount = total;
          *a.overflow = total > a.instanceCapacity ? 1u : 0u;
        }
      }
    }
    __syncthreads();
    const uint32_t base = tileBase + warpBase[warp];
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      if (cnt[r] == 0) continue;
      uint32_t at = base + rowExclusive[r];
      for (uint32_t ty = rect[r].y0; ty <= rect[r].y1; ++ty)
        for (uint32_t tx = rect[r].x0; tx <= rect[r].x1; ++tx, ++at) {
          if (at >= a.instanceCapacity) break;
          a.instanceKeys[at] = ty * a.tilesX + tx;
          a.instanceValues[at] = value[r];
        }
    }
  }
  if (tiles == 0 && tile == 0 && threadIdx.x == 0) {
    *a.instanceCount = 0;
    *a.overflow = 0;
  }
  finishTile(a.counters);
}

__global__ void rangesKernel(const uint32_t* __restrict__ keys, const uint32_t* count,
                             uint32_t capacity, uint2* ranges, uint32_t tiles) {
  const uint32_t n = min(*count, capacity);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    if (k >= tiles) continue;
    if (i == 0 || keys[i - 1] != k) ranges[k].x = i;
    if (i + 1 == n || keys[i + 1] != k) ranges[k].y = i + 1;
  }
}

}  // namespace

cudaError_t launchBinning(const BinArgs& a, cudaStream_t stream) {
  const uint32_t grid = max(1u, (a.capacity + kTileSplats - 1) / kTileSplats);
  binKernel<<<grid, kThreads, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launchTileRanges(const uint32_t* sortedKeys, const uint32_t* instanceCount,
                             uint32_t instanceCapacity, uint2* ranges, uint32_t tiles,
                             cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(ranges, 0, static_cast<size_t>(tiles) * sizeof(uint2), stream);
  if (e != cudaSuccess) return e;
  const uint32_t grid = max(1u, min(148u * 8u, (instanceCapacity + 255u) / 256u));
  rangesKernel<<<grid, 256, 0, stream>>>(sortedKeys, instanceCount, instanceCapacity, ranges, tiles);
  return cudaGetLastError();
}

}  // namespace sk
