// The LOD tree build on the GPU: the octree of the reference's builder
// (splat-core/src/lod/LodTree.cpp:17-344), built breadth first, one set of kernels (classify,
// scan, expand) per tree level.
//
//   1. per leaf: semi-axes and merge area (ellipsoid surface), node size, Morton key (3 bits per
//      octree level, at most 63);
//   2. the leaves sorted by (key, index): two stable 32-bit radix argsorts (low word, then high);
//   3. level by level from the root: every element of the level is a sorted range. A range of one
//      splat is that leaf; a range of at most clusterLeaves splats, at the depth limit, or of one
//      key merges its leaves; any other range skips the levels where all its keys share the
//      octant and splits into the runs of the first octant digit that differs. Each element's
//      children are the next level's elements in order, so the levels laid out one after the
//      other are the reference's breadth-first layout (LodTree.cpp:209-243);
//   4. deepest level first, each node merges its children's weighted moments (LodTree.cpp:47-102)
//      in the reference's order of float operations.
// The structure (child ranges) is the reference builder's exactly. The attributes match to a few
// ulp: the eigen-solve's acos and cos are CUDA's double functions, and the surface formula's
// and the opacity reach's float pow and log are taken in double and rounded once (the correctly
// rounded value, which the host library's powf and logf give for all but a small share of
// inputs), so they are not always the host library's.
//
// Built with -fmad=false: every product and sum rounds on its own, as in the reference build.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

#include "sk_device.cuh"
#include "sk_kernels.h"

namespace sk {
namespace {

constexpr uint32_t kThreads = 256;

// SymmetricEigen.cpp:8-41 (the trigonometric solution of the characteristic cubic, in the
// reference's double operations): eigenvalues of the symmetric 3x3 (upper triangle),
// descending, as floats.
__device__ void eigenvaluesDesc(const float* u, float* out) {
  const double xx = u[0], xy = u[1], xz = u[2], yy = u[3], yz = u[4], zz = u[5];
  const double p1 = xy * xy + xz * xz + yz * yz;
  double e0, e1, e2;
  if (p1 < 1e-30) {
    e0 = xx, e1 = yy, e2 = zz;
  } else {
    const double q = (xx + yy + zz) / 3;
    const double p2 = (xx - q) * (xx - q) + (yy - q) * (yy - q) + (zz - q) * (zz - q) + 2 * p1;
    const double p = sqrt(p2 / 6);
    const double bxx = (xx - q) / p, byy = (yy - q) / p, bzz = (zz - q) / p;
    const double bxy = xy / p, bxz = xz / p, byz = yz / p;
    const double det = bxx * (byy * bzz - byz * byz) - bxy * (bxy * bzz - byz * bxz) +
                       bxz * (bxy * byz - byy * bxz);
    const double r = fmin(fmax(det / 2, -1.0), 1.0);
    const double phi = acos(r) / 3;
    const double a = q + 2 * p * cos(phi);
    const double c = q + 2 * p * cos(phi + 2 * 3.141592653589793 / 3);
    e0 = a, e1 = 3 * q - a - c, e2 = c;
  }
  // descending
  if (e0 < e1) { const double t = e0; e0 = e1; e1 = t; }
  if (e1 < e2) { const double t = e1; e1 = e2; e2 = t; }
  if (e0 < e1) { const double t = e0; e0 = e1; e1 = t; }
  out[0] = static_cast<float>(e0), out[1] = static_cast<float>(e1), out[2] = static_cast<float>(e2);
}

__device__ void semiAxes(const float* cov, float* s) {
  float e[3];
  eigenvaluesDesc(cov, e);
  for (int i = 0; i < 3; ++i) s[i] = sqrtf(fmaxf(e[i], 0.0f));
}

// x^y of floats as the nearest float to the exact power: the double power has far more bits
// than the float result needs, so rounding it once gives the correctly rounded float except on
// inputs within a double ulp of a rounding boundary.
__device__ __forceinline__ float powRounded(float x, float y) {
  return static_cast<float>(pow(static_cast<double>(x), static_cast<double>(y)));
}
__device__ __forceinline__ float logRounded(float x) {
  return static_cast<float>(log(static_cast<double>(x)));
}

// LodTree.cpp:17-22 (Knud Thomsen's ellipsoid surface approximation)
__device__ float ellipsoidArea(const float* s) {
  constexpr float kP = 1.6075f;
  const float sum = powRounded(s[0] * s[1], kP) + powRounded(s[0] * s[2], kP) +
                    powRounded(s[1] * s[2], kP);
  return 4.0f * 3.14159274f * powRounded(sum / 3.0f, 1.0f / kP);
}

// LodTree.cpp:27-29
__device__ float lodOpacityReach(float alpha) {
  return alpha > 1.0f ? sqrtf(1.0f + 2.71828175f * logRounded(alpha)) : 1.0f;
}

__device__ __forceinline__ uint64_t spreadBits3(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

// 1. per leaf: size, merge area, Morton key (LodTree.cpp:133-142)
__global__ void leafPrepKernel(uint32_t n, const float* __restrict__ positions,
                               const float* __restrict__ covariances, float3 boundsMin,
                               float extent, uint32_t depth, float* size, float* area,
                               uint32_t* keyLo, uint32_t* keyHi) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float axes[3];
  semiAxes(covariances + size_t{i} * 6, axes);
  size[i] = 2.0f * axes[0];
  area[i] = ellipsoidArea(axes);
  const uint32_t resolution = 1u << depth;
  const float lo[3] = {boundsMin.x, boundsMin.y, boundsMin.z};
  uint64_t key = 0;
  for (uint32_t c = 0; c < 3; ++c) {
    const float unit = fminf(fmaxf((positions[size_t{i} * 3 + c] - lo[c]) / extent, 0.0f), 1.0f);
    const uint32_t grid =
        min(static_cast<uint32_t>(unit * static_cast<float>(resolution)), resolution - 1);
    key |= spreadBits3(grid) << c;
  }
  keyLo[i] = static_cast<uint32_t>(key);
  keyHi[i] = static_cast<uint32_t>(key >> 32);
}

__global__ void gatherKernel(uint32_t n, const uint32_t* __restrict__ src,
                             const uint32_t* __restrict__ index, uint32_t* dst) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[index[i]];
}

// A range of the sorted leaves at a level of the build. kind: 0 leaf, 1 merged leaves,
// 2 interior (level = the level whose octant digit splits it).
struct Element {
  uint32_t begin, end, level, kind;
};

__device__ __forceinline__ uint64_t sortedKey(const uint32_t* lo, const uint32_t* hi, uint32_t i) {
  return (static_cast<uint64_t>(hi[i]) << 32) | lo[i];
}

// First position in [b, e) whose key >> shift is >= target (keys ascending).
__device__ uint32_t lowerBound(const uint32_t* lo, const uint32_t* hi, uint32_t b, uint32_t e,
                               uint32_t shift, uint64_t target) {
  while (b < e) {
    const uint32_t mid = b + (e - b) / 2;
    if ((sortedKey(lo, hi, mid) >> shift) < target) b = mid + 1; else e = mid;
  }
  return b;
}

// Calls run(start, stop) for each non-empty run of one octant digit at the element's level, in
// key order (at most 8: the element's keys share every digit above it).
template <typename Run>
__device__ __forceinline__ void forOctantRuns(const Element& el, const uint32_t* keyLo,
                                              const uint32_t* keyHi, uint32_t depth, Run run) {
  const uint32_t shift = 3 * (depth - el.level - 1);
  const uint64_t prefix = sortedKey(keyLo, keyHi, el.begin) >> shift;
  const uint64_t last = sortedKey(keyLo, keyHi, el.end - 1) >> shift;
  uint32_t start = el.begin;
  for (uint64_t d = prefix; d <= last; ++d) {
    const uint32_t stop = lowerBound(keyLo, keyHi, start, el.end, shift, d + 1);
    if (stop > start) run(start, stop);
    start = stop;
  }
}

// 3a. the kind of every element of the level and its number of children (LodTree.cpp:182-196)
__global__ void classifyKernel(uint32_t m, Element* elements, const uint32_t* keyLo,
                               const uint32_t* keyHi, uint32_t clusterLeaves, uint32_t depth,
                               uint32_t* counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  Element el = elements[i];
  const uint32_t size = el.end - el.begin;
  uint32_t count = 0;
  if (size == 1) {
    el.kind = 0;
  } else if (size <= clusterLeaves || el.level >= depth) {
    el.kind = 1;
    count = size;
  } else {
    const uint64_t x = sortedKey(keyLo, keyHi, el.begin) ^ sortedKey(keyLo, keyHi, el.end - 1);
    if (x == 0) {  // one key: the levels run out and the leaves merge at the depth limit
      el.kind = 1;
      count = size;
    } else {
      const uint32_t hb = 63 - __clzll(static_cast<long long>(x));
      el.level = max(el.level, depth - 1 - hb / 3);
      el.kind = 2;
      forOctantRuns(el, keyLo, keyHi, depth, [&](uint32_t, uint32_t) { ++count; });
    }
  }
  elements[i] = el;
  counts[i] = count;
}

// 3b. the level's children, in order, and every element's child range in the layout
__global__ void expandKernel(uint32_t m, const Element* elements, const uint32_t* offsets,
                             const uint32_t* keyLo, const uint32_t* keyHi, uint32_t depth,
                             uint32_t levelBase, uint32_t nextBase, Element* next,
                             uint32_t* childStart, uint32_t* childCount, uint32_t* leafOf,
                             const uint32_t* sortedIndex) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const Element el = elements[i];
  const uint32_t node = levelBase + i, out = offsets[i];
  childStart[node] = nextBase + out;  // a leaf's too: where its children would start
  leafOf[node] = el.kind == 0 ? sortedIndex[el.begin] : 0xffffffffu;
  uint32_t written = 0;
  if (el.kind == 1) {
    for (uint32_t j = el.begin; j < el.end; ++j)
      next[out + written++] = Element{j, j + 1, el.level + 1, 0};
  } else if (el.kind == 2) {
    forOctantRuns(el, keyLo, keyHi, depth, [&](uint32_t start, uint32_t stop) {
      next[out + written++] = Element{start, stop, el.level + 1, 0};
    });
  }
  childCount[node] = written;
}

// Exclusive scan of counts: per-block scans, then the block totals, then the offsets added.
__global__ void blockScanKernel(uint32_t m, const uint32_t* counts, uint32_t* offsets,
                                uint32_t* blockTotals) {
  __shared__ uint32_t warpSums[32];
  const uint32_t i = blockIdx.x * 1024 + threadIdx.x, lane = laneId(), warp = threadIdx.x >> 5;
  const uint32_t v = i < m ? counts[i] : 0u;
  uint32_t inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= static_cast<uint32_t>(o)) inc += up;
  }
  if (lane == 31) warpSums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const uint32_t s = warpSums[lane];
    uint32_t si = s;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t up = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= static_cast<uint32_t>(o)) si += up;
    }
    warpSums[lane] = si - s;
    if (lane == 31) blockTotals[blockIdx.x] = si;
  }
  __syncthreads();
  if (i < m) offsets[i] = warpSums[warp] + inc - v;
}

__global__ void totalsScanKernel(uint32_t blocks, uint32_t* blockTotals, uint32_t* grand) {
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < blocks; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < blocks ? blockTotals[i] : 0u;
    __shared__ uint32_t warpSums[32];
    const uint32_t lane = laneId(), warp = threadIdx.x >> 5;
    uint32_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= static_cast<uint32_t>(o)) inc += up;
    }
    if (lane == 31) warpSums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      const uint32_t s = warpSums[lane];
      uint32_t si = s;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t up = __shfl_up_sync(0xffffffffu, si, o);
        if (lane >= static_cast<uint32_t>(o)) si += up;
      }
      warpSums[lane] = si - s;
    }
    __syncthreads();
    const uint32_t before = carry;
    if (i < blocks) blockTotals[i] = before + warpSums[warp] + inc - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry = before + warpSums[warp] + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0) *grand = carry;
}

__global__ void addOffsetsKernel(uint32_t m, uint32_t* offsets, const uint32_t* blockTotals) {
  const uint32_t i = blockIdx.x * 1024 + threadIdx.x;
  if (i < m) offsets[i] += blockTotals[blockIdx.x];
}

// Node attributes in layout order.
struct NodeArrays {
  float* positions;    // 3 per node
  float* covariances;  // 6
  float* colors;       // 3
  float* alphas;
  float* sh;           // shStride
  float* area;         // merge weight per unit opacity
  LodNode* layout;     // position, size, child range
};

// 4. one level, deepest first: leaves copy their splat, the others merge their children
// (LodTree.cpp:47-102, the host restatement's order of float operations).
__global__ void mergeKernel(uint32_t m, uint32_t levelBase, const uint32_t* childStart,
                            const uint32_t* childCount, const uint32_t* leafOf,
                            const float* __restrict__ inPositions,
                            const float* __restrict__ inCovariances,
                            const float* __restrict__ inColors, const float* __restrict__ inAlphas,
                            const float* __restrict__ inSh, const float* __restrict__ leafSize,
                            const float* __restrict__ leafArea, uint32_t shStride, NodeArrays out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t node = levelBase + i;
  const uint32_t cnt = childCount[node];
  if (cnt == 0) {
    const uint32_t s = leafOf[node];
    for (int c = 0; c < 3; ++c) out.positions[size_t{node} * 3 + c] = inPositions[size_t{s} * 3 + c];
    for (int c = 0; c < 6; ++c) out.covariances[size_t{node} * 6 + c] = inCovariances[size_t{s} * 6 + c];
    for (int c = 0; c < 3; ++c) out.colors[size_t{node} * 3 + c] = inColors[size_t{s} * 3 + c];
    out.alphas[node] = inAlphas[s];
    for (uint32_t c = 0; c < shStride; ++c) out.sh[size_t{node} * shStride + c] = inSh[size_t{s} * shStride + c];
    out.area[node] = leafArea[s];
    out.layout[node] = LodNode{{inPositions[size_t{s} * 3], inPositions[size_t{s} * 3 + 1],
                                inPositions[size_t{s} * 3 + 2]},
                               leafSize[s], childStart[node], 0u};
    return;
  }
  const uint32_t first = childStart[node];
  float total = 0.0f;
  for (uint32_t k = 0; k < cnt; ++k) total += out.area[first + k] * out.alphas[first + k];
  auto weight = [&](uint32_t k) {
    const float w = out.area[first + k] * out.alphas[first + k];
    return total > 1e-30f ? w / total : 1.0f / static_cast<float>(cnt);
  };
  float center[3] = {0, 0, 0}, rgb[3] = {0, 0, 0};
  for (uint32_t k = 0; k < cnt; ++k) {
    const float w = weight(k);
    const size_t c3 = size_t{first + k} * 3;
    for (int c = 0; c < 3; ++c) {
      center[c] += w * out.positions[c3 + c];
      rgb[c] += w * out.colors[c3 + c];
    }
  }
  for (uint32_t c = 0; c < shStride; ++c) {
    float acc = 0.0f;
    for (uint32_t k = 0; k < cnt; ++k) acc += weight(k) * out.sh[size_t{first + k} * shStride + c];
    out.sh[size_t{node} * shStride + c] = acc;
  }
  for (float& channel : rgb) channel = fminf(fmaxf(channel, 0.0f), 1.0f);
  float cov[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t k = 0; k < cnt; ++k) {
    const uint32_t j = first + k;
    const float dx = out.positions[size_t{j} * 3] - center[0];
    const float dy = out.positions[size_t{j} * 3 + 1] - center[1];
    const float dz = out.positions[size_t{j} * 3 + 2] - center[2];
    const float* c = out.covariances + size_t{j} * 6;
    const float w = weight(k);
    cov[0] += w * (dx * dx + c[0]);
    cov[1] += w * (dx * dy + c[1]);
    cov[2] += w * (dx * dz + c[2]);
    cov[3] += w * (dy * dy + c[3]);
    cov[4] += w * (dy * dz + c[4]);
    cov[5] += w * (dz * dz + c[5]);
  }
  float axes[3];
  semiAxes(cov, axes);
  const float a = ellipsoidArea(axes);
  const float alpha = fminf(fmaxf(total / fmaxf(a, 1e-30f), 0.0f), 1000.0f);
  for (int c = 0; c < 3; ++c) out.positions[size_t{node} * 3 + c] = center[c];
  for (int c = 0; c < 6; ++c) out.covariances[size_t{node} * 6 + c] = cov[c];
  for (int c = 0; c < 3; ++c) out.colors[size_t{node} * 3 + c] = rgb[c];
  out.alphas[node] = alpha;
  out.area[node] = a;
  out.layout[node] = LodNode{{center[0], center[1], center[2]},
                             2.0f * axes[0] * lodOpacityReach(alpha), first, cnt};
}

uint32_t blocksOf(uint32_t n, uint32_t per) { return std::max(1u, (n + per - 1) / per); }

// Touches every 4 KB page of a fresh host array on several threads, so the page faults of the
// download that follows are taken in parallel instead of inside the driver's one copy thread.
void touchPages(void* data, size_t bytes) {
  constexpr size_t kPage = 4096;
  auto* bytesOf = static_cast<volatile unsigned char*>(data);
  const size_t pages = (bytes + kPage - 1) / kPage;
  const unsigned workers = static_cast<unsigned>(
      std::min<size_t>(std::min(32u, std::max(1u, std::thread::hardware_concurrency())),
                       std::max<size_t>(pages / 4096, 1)));
  auto touch = [=](size_t first, size_t last) {
    for (size_t pg = first; pg < last; ++pg) bytesOf[pg * kPage] = 0;
  };
  if (workers <= 1) return touch(0, pages);
  std::vector<std::thread> pool;
  for (unsigned w = 0; w < workers; ++w) pool.emplace_back(touch, pages * w / workers, pages * (w + 1) / workers);
  for (auto& t : pool) t.join();
}

// Carves one device allocation into the build's arrays (256-byte aligned); a first pass with no
// base only sums the sizes.
struct Arena {
  uint8_t* base = nullptr;
  size_t bytes = 0;
  template <typename T>
  T* get(size_t count) {
    const size_t at = (bytes + 255) & ~size_t{255};
    bytes = at + std::max<size_t>(count, 1) * sizeof(T);
    return base ? reinterpret_cast<T*>(base + at) : nullptr;
  }
};

}  // namespace

cudaError_t buildLodTreeGpu(const LodBuildInput& in, LodBuildOutput& out) {
  const uint32_t n = in.count;
  const size_t shStride = in.shStride;
  if (n == 0 || n > kMaxLodBuildLeaves) return cudaErrorInvalidValue;  // 2n - 1 nodes fit 32 bits
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return e;
  uint8_t* memory = nullptr;
  {
    Arena b;
    float *positions, *covariances, *colors, *alphas, *sh, *leafSize, *leafArea;
    uint32_t *keyLo, *keyHi, *orderLo, *hiByLo, *sortedIndex, *sortedLo, *sortedHi, *sortCount,
        *sortError, *counts, *offsets, *blockTotals, *grand, *childStart, *childCount, *leafOf;
    void* sortWork;
    Element *levelA, *levelB;
    NodeArrays nodes;
    const uint32_t maxNodes = 2 * n;  // every interior node has two children or more
    auto carve = [&] {
      positions = b.get<float>(size_t{n} * 3);
      covariances = b.get<float>(size_t{n} * 6);
      colors = b.get<float>(size_t{n} * 3);
      alphas = b.get<float>(n);
      sh = b.get<float>(size_t{n} * shStride);
      leafSize = b.get<float>(n);
      leafArea = b.get<float>(n);
      keyLo = b.get<uint32_t>(n);
      keyHi = b.get<uint32_t>(n);
      orderLo = b.get<uint32_t>(n);
      hiByLo = b.get<uint32_t>(n);
      sortedIndex = b.get<uint32_t>(n);
      sortedLo = b.get<uint32_t>(n);
      sortedHi = b.get<uint32_t>(n);
      sortCount = b.get<uint32_t>(1);
      sortError = b.get<uint32_t>(1);
      sortWork = b.get<uint8_t>(sortWorkspaceBytes(n));
      levelA = b.get<Element>(n);
      levelB = b.get<Element>(n);
      counts = b.get<uint32_t>(n);
      offsets = b.get<uint32_t>(n);
      blockTotals = b.get<uint32_t>(blocksOf(n, 1024));
      grand = b.get<uint32_t>(1);
      childStart = b.get<uint32_t>(maxNodes);
      childCount = b.get<uint32_t>(maxNodes);
      leafOf = b.get<uint32_t>(maxNodes);
      nodes = NodeArrays{b.get<float>(size_t{maxNodes} * 3), b.get<float>(size_t{maxNodes} * 6),
                         b.get<float>(size_t{maxNodes} * 3), b.get<float>(maxNodes),
                         b.get<float>(size_t{maxNodes} * shStride), b.get<float>(maxNodes),
                         b.get<LodNode>(maxNodes)};
    };
    carve();
    if ((e = cudaMalloc(&memory, b.bytes)) != cudaSuccess) {
      cudaStreamDestroy(s);
      return e;
    }
    b = Arena{memory, 0};
    carve();
    auto up = [&](void* dst, const void* src, size_t bytes) {
      if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    };
    up(positions, in.positions, size_t{n} * 12);
    up(covariances, in.covariances, size_t{n} * 24);
    up(colors, in.colors, size_t{n} * 12);
    up(alphas, in.alphas, size_t{n} * 4);
    if (shStride) up(sh, in.sh, size_t{n} * shStride * 4);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sortCount, &n, 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(sortWork, 0, sortWorkspaceBytes(n), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(sortError, 0, 4, s);
    if (e == cudaSuccess) {
      leafPrepKernel<<<blocksOf(n, kThreads), kThreads, 0, s>>>(
          n, positions, covariances, make_float3(in.boundsMin[0], in.boundsMin[1], in.boundsMin[2]),
          in.extent, in.depth, leafSize, leafArea, keyLo, keyHi);
      e = cudaGetLastError();
    }
    // (key, index) order: stable by the low word, then stably by the high word
    const uint32_t keyBits = 3 * in.depth;
    if (e == cudaSuccess) {
      SortArgs a{};
      a.keysIn = keyLo;
      a.valuesOut = orderLo;
      a.count = sortCount;
      a.capacity = n;
      a.bits = static_cast<int>(std::min(32u, (std::min(32u, keyBits) + 7) / 8 * 8));
      sortBindWorkspace(a, sortWork, n);
      a.epoch = 1;
      a.error = sortError;
      e = launchSort(a, s);
    }
    if (e == cudaSuccess && keyBits > 32) {
      gatherKernel<<<blocksOf(n, kThreads), kThreads, 0, s>>>(n, keyHi, orderLo, hiByLo);
      SortArgs a{};
      a.keysIn = hiByLo;
      a.valuesIn = orderLo;
      a.valuesOut = sortedIndex;
      a.count = sortCount;
      a.capacity = n;
      a.bits = static_cast<int>((keyBits - 32 + 7) / 8 * 8);
      sortBindWorkspace(a, sortWork, n);
      a.epoch = 9;
      a.error = sortError;
      e = launchSort(a, s);
    } else if (e == cudaSuccess) {
      e = cudaMemcpyAsync(sortedIndex, orderLo, size_t{n} * 4, cudaMemcpyDeviceToDevice, s);
    }
    if (e == cudaSuccess) {
      gatherKernel<<<blocksOf(n, kThreads), kThreads, 0, s>>>(n, keyLo, sortedIndex, sortedLo);
      gatherKernel<<<blocksOf(n, kThreads), kThreads, 0, s>>>(n, keyHi, sortedIndex, sortedHi);
      e = cudaGetLastError();
    }
    uint32_t sortStatus = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&sortStatus, sortError, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && sortStatus != 0) e = cudaErrorLaunchFailure;  // a look-back gave up
    // 3. levels from the root
    std::vector<uint32_t> levelBase{0}, levelSize{1};
    const Element root{0, n, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(levelA, &root, sizeof(Element), cudaMemcpyHostToDevice, s);
    Element* cur = levelA;
    Element* next = levelB;
    uint32_t total = 1;
    while (e == cudaSuccess) {
      const uint32_t m = levelSize.back(), base = levelBase.back();
      classifyKernel<<<blocksOf(m, kThreads), kThreads, 0, s>>>(m, cur, sortedLo, sortedHi,
                                                              in.clusterLeaves, in.depth, counts);
      const uint32_t blocks = blocksOf(m, 1024);
      blockScanKernel<<<blocks, 1024, 0, s>>>(m, counts, offsets, blockTotals);
      totalsScanKernel<<<1, 1024, 0, s>>>(blocks, blockTotals, grand);
      addOffsetsKernel<<<blocks, 1024, 0, s>>>(m, offsets, blockTotals);
      expandKernel<<<blocksOf(m, kThreads), kThreads, 0, s>>>(
          m, cur, offsets, sortedLo, sortedHi, in.depth, base, base + m, next, childStart,
          childCount, leafOf, sortedIndex);
      uint32_t children = 0;
      if ((e = cudaGetLastError()) != cudaSuccess) break;
      if ((e = cudaMemcpyAsync(&children, grand, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) break;
      if ((e = cudaStreamSynchronize(s)) != cudaSuccess) break;
      if (children == 0) break;
      if (uint64_t{total} + children > maxNodes) {
        e = cudaErrorInvalidValue;
        break;
      }
      levelBase.push_back(base + m);
      levelSize.push_back(children);
      total += children;
      std::swap(cur, next);
    }
    // 4. deepest level first
    for (size_t l = levelSize.size(); e == cudaSuccess && l-- > 0;) {
      mergeKernel<<<blocksOf(levelSize[l], kThreads), kThreads, 0, s>>>(
          levelSize[l], levelBase[l], childStart, childCount, leafOf, positions, covariances,
          colors, alphas, sh, leafSize, leafArea, static_cast<uint32_t>(shStride), nodes);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      out.count = total;
      out.positions.resize(size_t{total} * 3);
      out.covariances.resize(size_t{total} * 6);
      out.colors.resize(size_t{total} * 3);
      out.alphas.resize(total);
      out.sh.resize(size_t{total} * shStride);
      out.layout.resize(total);
      auto down = [&](void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes) {
          touchPages(dst, bytes);
          e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
        }
      };
      down(out.positions.data(), nodes.positions, size_t{total} * 12);
      down(out.covariances.data(), nodes.covariances, size_t{total} * 24);
      down(out.colors.data(), nodes.colors, size_t{total} * 12);
      down(out.alphas.data(), nodes.alphas, size_t{total} * 4);
      if (shStride) down(out.sh.data(), nodes.sh, size_t{total} * shStride * 4);
      down(out.layout.data(), nodes.layout, size_t{total} * sizeof(LodNode));
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e != cudaSuccess) cudaStreamSynchronize(s);
  }
  cudaFree(memory);
  cudaStreamDestroy(s);
  return e;
}

}  // namespace sk
