// Tile binning of the depth-sorted survivors. The reference rasterises instanced quads in four
// indirect batches (splatkit-ios/.../metal/raster/MetalSplatPipeline.mm:188-208,
// .../metal/cull/PrepareIndirect.metalh:4-21); this build composites 16x16 pixel tiles, so each
// survivor is listed once per tile its quad touches.
//
// A splat's quad is the parallelogram c + s a1 + t a2, |s|, |t| <= radius, in pixel units (the
// same half-rounded axes the compositor inverts). Its tiles are those of its pixel box whose
// square it overlaps by the separating-axis test (x, y and the normals of a1 and a2); the tile
// square is the pixel area, half a pixel beyond every pixel centre, so the test can only keep
// too many tiles, never drop one the compositor would cover.
//
// One kernel walks the depth-sorted list, counts each splat's tiles, takes its output offset
// by decoupled look-back, and writes (tile id, projected index) pairs. Offsets grow with depth
// rank and the tile sort that follows is stable, so every tile's list stays front to back. A
// count beyond the reserved capacity is recorded and nothing past it is written; the host
// grows the buffers and draws again.
#include <cuda_runtime.h>

#include "sk_device.cuh"
#include "sk_kernels.h"

namespace sk {
namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kItems = 4;
constexpr uint32_t kTileSplats = kThreads * kItems;

// The quad in y-up pixel coordinates.
struct Quad {
  float cx, cy, a1x, a1y, a2x, a2y, r;
};

__device__ __forceinline__ Quad quadOf(const uint4 lo, const uint4 hi, float halfW, float halfH) {
  Quad q;
  q.cx = (asF(lo.x) + 1.0f) * halfW;
  q.cy = (asF(lo.y) + 1.0f) * halfH;
  q.a1x = lowHalf(lo.z), q.a1y = highHalf(lo.z);
  q.a2x = lowHalf(lo.w), q.a2y = highHalf(lo.w);
  q.r = asF(hi.z);
  return q;
}

struct TileRect {
  uint32_t x0, y0, x1, y1;  // inclusive tile bounds; empty when x0 > x1
};

// Tiles of the quad's pixel box (plus one pixel).
__device__ __forceinline__ TileRect tileRect(const Quad& q, float width, float height,
                                             uint32_t tilesX, uint32_t tilesY) {
  TileRect t{1, 1, 0, 0};
  const float ex = q.r * (fabsf(q.a1x) + fabsf(q.a2x)) + 1.0f;
  const float ey = q.r * (fabsf(q.a1y) + fabsf(q.a2y)) + 1.0f;
  if (!(isfinite(q.cx) && isfinite(q.cy) && isfinite(ex) && isfinite(ey) && q.r >= 0.0f)) return t;
  const float xa = floorf(q.cx - ex), xb = ceilf(q.cx + ex);
  const float ya = floorf(q.cy - ey), yb = ceilf(q.cy + ey);
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

// Separating-axis test of the quad against tile (tx, ty)'s pixel square (y up).
__device__ __forceinline__ bool touches(const Quad& q, uint32_t tx, uint32_t ty, float height) {
  const float half = 0.5f * static_cast<float>(kTileSize);
  const float rx = static_cast<float>(tx * kTileSize) + half;
  const float ry = height - (static_cast<float>(ty * kTileSize) + half);
  const float dx = rx - q.cx, dy = ry - q.cy;
  if (fabsf(dx) > q.r * (fabsf(q.a1x) + fabsf(q.a2x)) + half) return false;
  if (fabsf(dy) > q.r * (fabsf(q.a1y) + fabsf(q.a2y)) + half) return false;
  // normal of a1: the quad's extent along it comes from t a2 only
  const float n1x = -q.a1y, n1y = q.a1x;
  if (fabsf(dx * n1x + dy * n1y) >
      q.r * fabsf(q.a2x * n1x + q.a2y * n1y) + half * (fabsf(n1x) + fabsf(n1y)))
    return false;
  const float n2x = -q.a2y, n2y = q.a2x;
  if (fabsf(dx * n2x + dy * n2y) >
      q.r * fabsf(q.a1x * n2x + q.a1y * n2y) + half * (fabsf(n2x) + fabsf(n2y)))
    return false;
  return true;
}

__global__ void __launch_bounds__(kThreads) binKernel(const __grid_constant__ BinArgs a) {
  __shared__ uint32_t warpBase[kThreads / 32];
  __shared__ uint32_t tileBase;
  const uint32_t tile = takeTile(a.counters);
  const uint32_t n = min(*a.count, a.capacity);
  const uint32_t tiles = (n + kTileSplats - 1) / kTileSplats;
  const float width = static_cast<float>(a.width), height = static_cast<float>(a.height);
  const float halfW = 0.5f * width, halfH = 0.5f * height;
  if (tile < tiles) {
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    uint32_t value[kItems];
    uint4 lo[kItems], hi[kItems];
    // all loads first: the order entries, then the records they name
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      const uint32_t i = tile * kTileSplats + warp * (32 * kItems) + r * 32 + lane;
      value[r] = i < n ? __ldg(a.order + i) : 0xffffffffu;
    }
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      if (value[r] != 0xffffffffu) {
        const uint4* p = reinterpret_cast<const uint4*>(a.projected + value[r]);
        lo[r] = __ldg(p);
        hi[r] = __ldg(p + 1);
      }
    }
    // Each splat's tiles are decided once: a bit per tile of its box (row major), for boxes of
    // up to 64 tiles; a larger box keeps all its tiles. The count and the emission both read
    // this mask, so they cannot disagree.
    uint32_t rx0[kItems], ry0[kItems], rw[kItems], area[kItems], cnt[kItems];
    uint64_t mask[kItems];
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      cnt[r] = 0, mask[r] = 0, area[r] = 0, rx0[r] = 0, ry0[r] = 0, rw[r] = 1;
      if (value[r] == 0xffffffffu) continue;
      const Quad q = quadOf(lo[r], hi[r], halfW, halfH);
      const TileRect t = tileRect(q, width, height, a.tilesX, a.tilesY);
      if (t.x0 > t.x1 || t.y0 > t.y1) continue;
      rx0[r] = t.x0, ry0[r] = t.y0, rw[r] = t.x1 - t.x0 + 1;
      area[r] = rw[r] * (t.y1 - t.y0 + 1);
      if (area[r] > 64) {
        cnt[r] = area[r];
        continue;
      }
      uint64_t m = 0;
      for (uint32_t k = 0; k < area[r]; ++k) {
        const uint32_t tx = t.x0 + k % rw[r], ty = t.y0 + k / rw[r];
        if (touches(q, tx, ty, height)) m |= 1ull << k;
      }
      mask[r] = m;
      cnt[r] = static_cast<uint32_t>(__popcll(m));
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
      const bool all = area[r] > 64;
      uint64_t m = mask[r];
      for (uint32_t k = 0; k < area[r]; ++k) {
        if (!all && !((m >> k) & 1ull)) continue;
        if (at < a.instanceCapacity) {
          a.instanceKeys[at] = (ry0[r] + k / rw[r]) * a.tilesX + rx0[r] + k % rw[r];
          a.instanceValues[at] = value[r];
        }
        ++at;
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
