// LOD cut selection: the level-synchronous walk over interior clusters of
// splatkit-ios/Sources/SplatKitCore/rendering/metal/selection/SplatLOD.metal:26-220 (host order
// MetalLodSelection.mm:109-192), producing the same cut in the same emission order.
//
// Per round the reference dispatches evaluate, scan, budget, compact, scan, commit and scatter.
// Here a round is three kernels:
//   evaluate  drop / split / forced split per frontier cluster; the exclusive prefix of the
//             extra cost by decoupled look-back; the block that finishes last runs the capacity
//             guard (a 256-way search for the largest accepted prefix, SplatLOD.metal:116-132);
//   compact   denies over-budget splits, scans kids / splats / packets (three look-backs) and
//             the block that finishes last commits the round (SplatLOD.metal:165-181);
//   scatter   next frontier, inline leaf indices (<= 32 leaves) and packets (SplatLOD.metal:182-208).
// A round whose frontier is known to fit one tile (round r holds at most fanout^r clusters, the
// tree's fan-out being the most child clusters of any cluster) runs as one single-block kernel:
// the same steps in the same order, block barriers in place of the grid-wide hand-offs.
// A final kernel copies packet leaves (SplatLOD.metal:210-220). Grids are sized by the frontier
// capacity and read the live counts from the state, so no round needs the host; every kernel is
// launched chained (programmatic dependent launch), so a round's kernels follow one another
// without launch gaps.
//
// Built with -fmad=false: lodOutside and lodErrorPixels round every product and sum on their
// own, in the order written, so the split decisions match the host oracle bit for bit.
#include <cuda_runtime.h>

#include <algorithm>

#include "sk_device.cuh"
#include "sk_kernels.h"
#include "sk_launch.cuh"

namespace sk {
namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kItems = 2;  // 512 clusters per tile: 0.229 -> 0.189 ms of walk selection
                                // against 1024
constexpr uint32_t kTileClusters = kThreads * kItems;
constexpr uint32_t kSplit = 0x80000000u;
constexpr uint32_t kDrop = 0x40000000u;
constexpr uint32_t kCost = 0x3fffffffu;

struct RoundSums {
  uint32_t kids, splats, packets;
};

__device__ __forceinline__ void viewPoint(const Camera& cam, const float* c, float* v) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
    v[r] = ((cam.view[r] * c[0] + cam.view[4 + r] * c[1]) + cam.view[8 + r] * c[2]) +
           cam.view[12 + r] * 1.0f;
}

// SplatLOD.metal:26-32
__device__ __forceinline__ bool lodOutside(const Camera& cam, const LodCluster& n) {
  float v[3];
  viewPoint(cam, n.center, v);
  const float z = -v[2], r = n.radius;
  const float tx = cam.tanHalfFov[0], ty = cam.tanHalfFov[1];
  const float guard = (2.0f * fmaxf(z, 0.0f)) / fmaxf(fminf(cam.focal[0], cam.focal[1]), 1.0f);
  if (z + r <= 0.0f) return true;
  const bool outX = fabsf(v[0]) - z * tx > r * sqrtf(1.0f + tx * tx) + guard;
  const bool outY = fabsf(v[1]) - z * ty > r * sqrtf(1.0f + ty * ty) + guard;
  return outX || outY;
}

// SplatLOD.metal:33-43
__device__ __forceinline__ float lodErrorPixels(const Camera& cam, const LodCluster& n,
                                                float colorWeight) {
  float v[3];
  viewPoint(cam, n.center, v);
  const float depth = fmaxf(-v[2] - n.radius, 1e-4f);
  const float perspective = sqrtf(1.0f + (v[0] * v[0] + v[1] * v[1]) / (depth * depth));
  const float appearance = fminf(sqrtf(n.colorVariance), 1.0f);
  const float error = n.error + n.radius * appearance;
  return ((((error * fmaxf(cam.focal[0], cam.focal[1])) / depth) * perspective) *
          fmaxf(n.opacity, 0.1f)) *
         (1.0f + colorWeight * sqrtf(n.colorVariance));
}

__device__ __forceinline__ LodCluster loadCluster(const LodCluster* clusters, uint32_t i) {
  const uint4* p = reinterpret_cast<const uint4*>(clusters + i);
  LodCluster c;
  uint4* d = reinterpret_cast<uint4*>(&c);
  d[0] = __ldg(p), d[1] = __ldg(p + 1), d[2] = __ldg(p + 2), d[3] = __ldg(p + 3);
  return c;
}

// Block-wide exclusive scan of one value per (warp, row, lane) item in source order, plus the
// tile's aggregate, then the tile's global offset by look-back. Returns the per-item exclusive
// global offsets in `out`.
template <int kCount>
__device__ __forceinline__ void tileScan(const uint32_t (&vals)[kCount][kItems], uint32_t tile,
                                         uint64_t* const (&status)[kCount], uint32_t epoch,
                                         uint32_t* error, uint32_t (&out)[kCount][kItems],
                                         uint32_t (&aggregateOut)[kCount],
                                         uint32_t (&exclusiveOut)[kCount]) {
  __shared__ uint32_t warpSums[kCount][kThreads / 32];
  __shared__ uint32_t tileBase[kCount];
  __shared__ uint32_t tileAggregate[kCount];
  const uint32_t warp = threadIdx.x >> 5, lane = laneId();
#pragma unroll
  for (int c = 0; c < kCount; ++c) {
    uint32_t run = 0;
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) {
      uint32_t inc = vals[c][r];
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= static_cast<uint32_t>(o)) inc += up;
      }
      out[c][r] = run + inc - vals[c][r];
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) warpSums[c][warp] = run;
  }
  __syncthreads();
  if (warp < kCount) {
    const int c = warp;
    const uint32_t w = lane < kThreads / 32 ? warpSums[c][lane] : 0u;
    uint32_t inc = w;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= static_cast<uint32_t>(o)) inc += up;
    }
    const uint32_t aggregate = __shfl_sync(0xffffffffu, inc, 31);
    if (lane < kThreads / 32) warpSums[c][lane] = inc - w;
    uint32_t exclusive = 0;
    if (tile == 0) {
      if (lane == 0) storeStatus(status[c], makeStatus(epoch, kFlagPrefix, aggregate));
    } else {
      if (lane == 0) storeStatus(status[c] + tile, makeStatus(epoch, kFlagAggregate, aggregate));
      exclusive = warpLookback(status[c], tile, epoch, error);
      if (lane == 0)
        storeStatus(status[c] + tile, makeStatus(epoch, kFlagPrefix, exclusive + aggregate));
    }
    if (lane == 0) {
      tileBase[c] = exclusive;
      tileAggregate[c] = aggregate;
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < kCount; ++c) {
    const uint32_t base = tileBase[c] + warpSums[c][warp];
#pragma unroll
    for (uint32_t r = 0; r < kItems; ++r) out[c][r] += base;
    aggregateOut[c] = tileAggregate[c];
    exclusiveOut[c] = tileBase[c];
  }
}

__device__ __forceinline__ uint32_t itemIndex(uint32_t tile, uint32_t r) {
  return tile * kTileClusters + (threadIdx.x >> 5) * (32 * kItems) + r * 32 + laneId();
}

__global__ void lodInitKernel(uint32_t* frontier, LodState* state) {
  chainedKernelStart();
  frontier[0] = 0;
  LodState s{};
  s.active = 1;
  *state = s;
}

// Evaluate, tile `tile` (< the round's tiles): drop / split / forced split per frontier cluster,
// the exclusive prefix of the extra cost, and the drops.
__device__ __forceinline__ void evaluateTile(const Camera& cam, const LodArgs& a,
                                             const uint32_t* __restrict__ frontier, uint32_t tile,
                                             uint32_t active, uint32_t tiles, uint32_t epoch) {
  LodState* st = a.state;
  uint32_t extra[1][kItems], word[kItems];
  uint32_t drops = 0;
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    const uint32_t t = itemIndex(tile, r);
    uint32_t e = 0, flags = 0;
    if (t < active) {
      const LodCluster node = loadCluster(a.clusters, frontier[t]);
      if (a.cull && lodOutside(cam, node)) {
        flags = kDrop;
        ++drops;
      } else if (node.childCount + node.leafCount > 1 &&
                 (a.pixelLimit == 0.0f || lodErrorPixels(cam, node, a.colorWeight) > a.pixelLimit)) {
        flags = kSplit;
        e = node.childCount + node.leafCount - 1;
      } else if (node.childCount == 1 && node.leafCount == 0) {
        flags = kSplit;
      }
    }
    extra[0][r] = e;
    word[r] = e | flags;
  }
  uint32_t prefix[1][kItems], aggregate[1], exclusive[1];
  uint64_t* const status[1] = {a.status};
  tileScan<1>(extra, tile, status, epoch, a.error, prefix, aggregate, exclusive);
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    const uint32_t t = itemIndex(tile, r);
    if (t < active) a.costs[t] = make_uint2(word[r], prefix[0][r]);
  }
  for (int o = 16; o > 0; o >>= 1) drops += __shfl_xor_sync(0xffffffffu, drops, o);
  if (laneId() == 0 && drops) atomicAdd(&st->drops, drops);
  if (tile == tiles - 1 && threadIdx.x == 0) st->totalExtra = exclusive[0] + aggregate[0];
}

// The capacity guard (SplatLOD.metal:116-132), in uint32 arithmetic like the reference, once the
// round is evaluated; every thread of one block.
__device__ __forceinline__ void capacityGuard(const LodArgs& a, uint32_t active) {
  LodState* st = a.state;
  __shared__ uint32_t found;
  const uint32_t total = __ldcg(&st->totalExtra);
  const uint32_t available = a.limit - __ldcg(&st->count) - active + __ldcg(&st->drops);
  uint32_t accepted;
  if (total <= available) {
    accepted = total;
  } else {
    // m = how many leading clusters fit: end(t) = prefix(t) + extra(t) <= available for
    // t < m (end grows with t). A 256-way search keeps m in [lo, hi].
    __shared__ uint32_t upper;
    uint32_t lo = 0, hi = active;
    while (lo < hi) {
      if (threadIdx.x == 0) {
        found = lo;
        upper = hi;
      }
      __syncthreads();
      const uint64_t span = hi - lo;
      const uint32_t q =
          lo + static_cast<uint32_t>((span * (threadIdx.x + 1) + kThreads - 1) / kThreads);
      const uint2 c = __ldcg(&a.costs[q - 1]);
      if (c.y + (c.x & kCost) <= available) atomicMax(&found, q);
      __syncthreads();
      const uint32_t f = found;
      if (q > f) atomicMin(&upper, q - 1);
      __syncthreads();
      lo = f;
      hi = upper;
      __syncthreads();
    }
    const uint32_t m = lo;
    if (m == 0) {
      accepted = 0;
    } else {
      const uint2 c = __ldcg(&a.costs[m - 1]);
      accepted = c.y + (c.x & kCost);
    }
  }
  if (threadIdx.x == 0) {
    st->accepted = accepted;
    st->drops = 0;
  }
}

// Compact, tile `tile` (< the round's tiles): denies over-budget splits and scans kids / splats /
// packets into each cluster's offsets.
__device__ __forceinline__ void compactTile(const LodArgs& a, const uint32_t* __restrict__ frontier,
                                            RoundSums* sums, uint32_t tile, uint32_t active,
                                            uint32_t tiles, uint32_t accepted, uint32_t epoch) {
  LodState* st = a.state;
  uint32_t vals[3][kItems], flagsOf[kItems];
  uint32_t denied = 0;
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    const uint32_t t = itemIndex(tile, r);
    uint32_t kids = 0, splats = 0, packets = 0, flags = kDrop;
    if (t < active) {
      const uint2 c = a.costs[t];
      flags = c.x & ~kCost;
      const uint32_t extra = c.x & kCost;
      if ((flags & kSplit) && extra > 0 && c.y + extra > accepted) {
        flags = 0;
        ++denied;
      }
      if (!(flags & kDrop)) {
        const LodCluster node = loadCluster(a.clusters, frontier[t]);
        kids = (flags & kSplit) ? node.childCount : 0;
        splats = (flags & kSplit) ? node.leafCount : 1;
        packets = splats > 32 ? 1 : 0;
      }
    }
    vals[0][r] = kids, vals[1][r] = splats, vals[2][r] = packets;
    flagsOf[r] = flags;
  }
  uint32_t offs[3][kItems], aggregate[3], exclusive[3];
  const size_t stride = (a.frontierCapacity + kTileClusters - 1) / kTileClusters;
  uint64_t* const status[3] = {a.status, a.status + stride, a.status + 2 * stride};
  tileScan<3>(vals, tile, status, epoch, a.error, offs, aggregate, exclusive);
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    const uint32_t t = itemIndex(tile, r);
    if (t < active) a.offsets[t] = make_uint4(offs[0][r], offs[1][r], offs[2][r], flagsOf[r]);
  }
  for (int o = 16; o > 0; o >>= 1) denied += __shfl_xor_sync(0xffffffffu, denied, o);
  if (laneId() == 0 && denied) atomicAdd(&st->limited, denied);
  if (tile == tiles - 1 && threadIdx.x == 0) {
    sums->kids = exclusive[0] + aggregate[0];
    sums->splats = exclusive[1] + aggregate[1];
    sums->packets = exclusive[2] + aggregate[2];
  }
}

// Commits the round (SplatLOD.metal:165-181); one thread, once the round is compacted.
__device__ __forceinline__ void commitRound(const LodArgs& a, const RoundSums* sums, uint32_t active) {
  LodState* st = a.state;
  const volatile RoundSums* v = sums;
  const RoundSums s{v->kids, v->splats, v->packets};
  st->evaluated += active;
  st->scatterActive = active;
  st->scatterCount = st->count;
  st->scatterPackets = st->packets;
  st->count += s.splats;
  st->packets += s.packets;
  st->active = s.kids;
}

// Scatter (SplatLOD.metal:182-208) of clusters first, first + step, ... below `active`: the next
// frontier, inline leaf indices (<= 32 leaves) and packets, from the offsets of the compact.
__device__ __forceinline__ void scatterClusters(const LodArgs& a, const uint32_t* __restrict__ frontier,
                                                uint32_t* __restrict__ next, uint32_t active,
                                                uint32_t countBase, uint32_t packetBase,
                                                uint32_t first, uint32_t step) {
  for (uint32_t t = first; t < active; t += step) {
    const uint4 local = a.offsets[t];
    if (local.w & kDrop) continue;
    const LodCluster node = loadCluster(a.clusters, frontier[t]);
    const bool split = (local.w & kSplit) != 0;
    if (split) {
      if (local.x + node.childCount > a.frontierCapacity) {
        atomicOr(a.error, SK_DEVERR_BOUNDS);
      } else {
        for (uint32_t k = 0; k < node.childCount; ++k) next[local.x + k] = node.childStart + k;
      }
    }
    const uint32_t count = split ? node.leafCount : 1;
    const uint32_t destination = countBase + local.y;
    if (count > 32) {
      if (packetBase + local.z < a.frontierCapacity)
        a.packets[packetBase + local.z] = make_uint4(node.leafStart, count, destination, 1);
      else
        atomicOr(a.error, SK_DEVERR_BOUNDS);
    } else if (destination + count > a.capacity) {
      atomicOr(a.error, SK_DEVERR_BOUNDS);
    } else if (!split) {
      a.indices[destination] = node.node;
    } else {
      for (uint32_t k = 0; k < count; ++k) a.indices[destination + k] = a.leaves[node.leafStart + k];
    }
  }
}

__global__ void __launch_bounds__(kThreads)
    lodEvaluateKernel(const Camera* __restrict__ camera, const __grid_constant__ LodArgs a,
                      const uint32_t* __restrict__ frontier, uint32_t epoch) {
  chainedKernelStart();
  __shared__ Camera cam;
  loadCamera(camera, &cam);
  LodState* st = a.state;
  const uint32_t tile = takeTile(a.counters);  // its barrier also publishes the camera
  // The guard keeps the frontier within the capacity; clamp anyway so no index leaves the
  // buffers (and say so).
  const uint32_t active = min(st->active, a.frontierCapacity);
  if (tile == 0 && threadIdx.x == 0 && st->active > a.frontierCapacity) atomicOr(a.error, SK_DEVERR_BOUNDS);
  const uint32_t tiles = (active + kTileClusters - 1) / kTileClusters;
  if (tile < tiles) evaluateTile(cam, a, frontier, tile, active, tiles, epoch);
  if (tiles == 0 && tile == 0 && threadIdx.x == 0) st->totalExtra = 0;
  if (finishTile(a.counters)) capacityGuard(a, active);
}

__global__ void __launch_bounds__(kThreads)
    lodCompactKernel(const __grid_constant__ LodArgs a, const uint32_t* __restrict__ frontier,
                     RoundSums* sums, uint32_t epoch) {
  chainedKernelStart();
  LodState* st = a.state;
  const uint32_t tile = takeTile(a.counters);
  const uint32_t active = min(st->active, a.frontierCapacity);
  const uint32_t accepted = st->accepted;
  const uint32_t tiles = (active + kTileClusters - 1) / kTileClusters;
  if (tile < tiles) compactTile(a, frontier, sums, tile, active, tiles, accepted, epoch);
  if (tiles == 0 && tile == 0 && threadIdx.x == 0) *sums = RoundSums{0, 0, 0};
  if (finishTile(a.counters) && threadIdx.x == 0) commitRound(a, sums, active);
}

__global__ void __launch_bounds__(kThreads)
    lodScatterKernel(const __grid_constant__ LodArgs a, const uint32_t* __restrict__ frontier,
                     uint32_t* __restrict__ next) {
  chainedKernelStart();
  const LodState* st = a.state;
  scatterClusters(a, frontier, next, min(st->scatterActive, a.frontierCapacity), st->scatterCount,
                  st->scatterPackets, blockIdx.x * kThreads + threadIdx.x, gridDim.x * kThreads);
}

// A round whose frontier fits one tile (the host knows it from the tree's fan-out): evaluate,
// guard, compact, commit and scatter in one block, block barriers in place of the grid-wide
// hand-offs of the three kernels, the same arithmetic and order.
__global__ void __launch_bounds__(kThreads)
    lodSmallRoundKernel(const Camera* __restrict__ camera, const __grid_constant__ LodArgs a,
                        const uint32_t* __restrict__ frontier, uint32_t* __restrict__ next,
                        RoundSums* sums, uint32_t epoch) {
  chainedKernelStart();
  __shared__ Camera cam;
  loadCamera(camera, &cam);
  __syncthreads();
  LodState* st = a.state;
  const uint32_t held = st->active;
  if (held > kTileClusters || held > a.frontierCapacity) {  // the host's bound did not hold
    if (threadIdx.x == 0) atomicOr(a.error, SK_DEVERR_BOUNDS);
    return;
  }
  const uint32_t active = held, tiles = active > 0 ? 1u : 0u;
  if (tiles) evaluateTile(cam, a, frontier, 0, active, tiles, epoch);
  if (!tiles && threadIdx.x == 0) st->totalExtra = 0;
  __syncthreads();
  capacityGuard(a, active);
  __syncthreads();
  const uint32_t accepted = __ldcg(&st->accepted);
  const uint32_t countBase = __ldcg(&st->count), packetBase = __ldcg(&st->packets);
  if (tiles) compactTile(a, frontier, sums, 0, active, tiles, accepted, (epoch + 1) & 0x3fffffffu);
  if (!tiles && threadIdx.x == 0) *sums = RoundSums{0, 0, 0};
  __syncthreads();
  if (threadIdx.x == 0) commitRound(a, sums, active);
  scatterClusters(a, frontier, next, active, countBase, packetBase, threadIdx.x, kThreads);
}

__global__ void __launch_bounds__(kThreads) lodEmitKernel(const __grid_constant__ LodArgs a) {
  chainedKernelStart();
  const uint32_t packets = min(a.state->packets, a.frontierCapacity);
  for (uint32_t p = blockIdx.x; p < packets; p += gridDim.x) {
    const uint4 packet = a.packets[p];
    if (packet.z + packet.y > a.capacity) {
      if (threadIdx.x == 0) atomicOr(a.error, SK_DEVERR_BOUNDS);
      continue;
    }
    for (uint32_t k = threadIdx.x; k < packet.y; k += kThreads)
      a.indices[packet.z + k] = packet.w ? a.leaves[packet.x + k] : packet.x;
  }
}

__global__ void lodReportKernel(const LodState* state, uint32_t* report) {
  chainedKernelStart();
  if (threadIdx.x < 6) report[threadIdx.x] = reinterpret_cast<const uint32_t*>(state)[threadIdx.x];
}

}  // namespace

uint32_t lodTileClusters() { return kTileClusters; }

cudaError_t launchLodSelect(const Camera* cam, const LodArgs& a, cudaStream_t stream) {
  const uint32_t grid = max(1u, (a.frontierCapacity + kTileClusters - 1) / kTileClusters);
  RoundSums* sums = reinterpret_cast<RoundSums*>(reinterpret_cast<char*>(a.state) + sizeof(LodState));
  cudaError_t e = launchChained(lodInitKernel, 1, 1, stream, a.frontier[0], a.state);
  uint64_t most = 1;  // clusters the round's frontier can hold: the root, then fanout times more
  for (uint32_t level = 0; e == cudaSuccess && level < a.rounds; ++level) {
    const uint32_t* cur = a.frontier[level & 1u];
    uint32_t* nxt = a.frontier[(level + 1) & 1u];
    const uint32_t epoch = (a.epoch + 2 * level) & 0x3fffffffu;
    if (a.fanout != 0 && most <= kTileClusters) {
      e = launchChained(lodSmallRoundKernel, 1, kThreads, stream, cam, a, cur, nxt, sums, epoch);
    } else {
      e = launchChained(lodEvaluateKernel, grid, kThreads, stream, cam, a, cur, epoch);
      if (e == cudaSuccess)
        e = launchChained(lodCompactKernel, grid, kThreads, stream, a, cur, sums,
                          (epoch + 1) & 0x3fffffffu);
      if (e == cudaSuccess)
        e = launchChained(lodScatterKernel, min(grid * kItems, 148u * 8u), kThreads, stream, a, cur, nxt);
    }
    most = std::min<uint64_t>(most * std::max(a.fanout, 1u), uint64_t{1} << 40);
  }
  const uint32_t packetGrid = max(1u, min(a.frontierCapacity, 148u * 8u));
  if (e == cudaSuccess) e = launchChained(lodEmitKernel, packetGrid, kThreads, stream, a);
  if (e == cudaSuccess) e = launchChained(lodReportKernel, 1, 32, stream, a.state, a.report);
  return e;
}

}  // namespace sk
