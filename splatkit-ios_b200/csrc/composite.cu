// Front-to-back compositing of 16x16 pixel tiles.
//
// The equations are the reference's raster stage (splatkit-ios/.../metal/raster/
// SplatRaster.metal:27-44, .../metal/layout/SplatProjection.metalh:155-175, blend state
// .../metal/raster/MetalSplatPipeline.mm:116-140): a pixel offset d = s a1 + t a2 inside the quad
// |s|, |t| <= radius gets alpha = min(1, peak * exp(-(s^2 + t^2) / 2)), dropped below 1/255;
// colour and coverage blend "under": C += (1 - A) alpha c, A += (1 - A) alpha; the background
// goes under what is left. The reference's fp16 target, unorm10 vertex colour and saturation
// mask between four draw batches are replaced by FP32 accumulation and per-pixel early
// termination when the remaining transmittance drops below `cutoff`.
//
// A block of 128 threads owns a 16x16 tile; each thread owns two horizontally adjacent pixels and
// each warp an 8x8-pixel quadrant. The tile reads the list of the 32x32 binning cell it lies in
// (the splats touching the cell, front to back) in batches of 128 records: thread i
// fetches record i (two 128-bit loads), turns it into the coverage form (pixel centre, inverse
// axes, radius, log cutoff, colour) in shared memory and marks which of the four quadrants its
// quad overlaps (separating-axis test). Each warp compacts, by ballot, the batch entries that
// reach it and sweeps only those, both of its pixels per entry. The coverage decision (quad bound and 1/255 cutoff)
// is a fixed sequence of correctly rounded operations, bit-identical to the host oracle's FP32
// formula.
#include <cuda_runtime.h>

#include "sk_device.cuh"
#include "sk_kernels.h"
#include "sk_launch.cuh"

namespace sk {
namespace {

constexpr uint32_t kThreads = kTileSize * kTileSize / 2;  // 128: two pixels per thread
constexpr uint32_t kWarps = kThreads / 32;
constexpr uint32_t kEntries = kThreads;  // list entries staged per batch (one per thread)
constexpr uint32_t kQuadrant = kTileSize / 2;  // each warp owns an 8x8 quadrant

struct alignas(16) Splat2D {
  float cx, cy, m00, m01;
  float m10, m11, radius, lcut;
  float lpeak, r, g, b;  // lpeak = log2 of the peak alpha
};
static_assert(sizeof(Splat2D) == 48, "Splat2D is three 16-byte words");

struct CompositeSmem {
  Splat2D splat[kEntries];
  uint8_t list[kWarps][kEntries];  // per warp: batch entries whose quad reaches its quadrant
  uint8_t reach[kEntries];         // per entry: bit w set when it reaches quadrant w
};

// Fills the coverage form; returns the bitmask of the warp quadrants its quad overlaps.
__device__ __forceinline__ uint32_t coverageForm(const uint4 lo, const uint4 hi, float halfW,
                                                 float halfH, float tileX, float tileTop,
                                                 Splat2D& s) {
  s.cx = __fmul_rn(__fadd_rn(asF(lo.x), 1.0f), halfW);
  s.cy = __fmul_rn(__fadd_rn(asF(lo.y), 1.0f), halfH);
  const float a1x = lowHalf(lo.z), a1y = highHalf(lo.z);
  const float a2x = lowHalf(lo.w), a2y = highHalf(lo.w);
  const float det = __fsub_rn(__fmul_rn(a1x, a2y), __fmul_rn(a2x, a1y));
  const float inv = __fdiv_rn(1.0f, det);
  s.m00 = __fmul_rn(a2y, inv);
  s.m01 = -__fmul_rn(a2x, inv);
  s.m10 = -__fmul_rn(a1y, inv);
  s.m11 = __fmul_rn(a1x, inv);
  const float peak = highHalf(hi.y);
  s.lcut = __fmul_rn(2.0f, lnF32(__fmul_rn(255.0f, peak)));  // 2 ln(255 peak), exact doubling
  s.lpeak = __log2f(peak);
  s.radius = asF(hi.z);
  s.r = lowHalf(hi.x);
  s.g = highHalf(hi.x);
  s.b = lowHalf(hi.y);
  const bool any = det != 0.0f && isfinite(inv) && isfinite(s.cx) && isfinite(s.cy);
  if (!any) {
    s.radius = -1.0f;
    return 0u;
  }
  // Separating axes of the quad c + s a1 + t a2 (|s|, |t| <= radius) against each quadrant's
  // square, taken half a pixel beyond its pixel centres (4 px from the quadrant centre): the
  // screen x and y axes and the normals of a1 and a2. The slack keeps the test conservative
  // against the rounding of the inverse used by the coverage decision.
  constexpr float kHalf = 0.5f * kQuadrant;
  const float ex = s.radius * (fabsf(a1x) + fabsf(a2x)) + kHalf;
  const float ey = s.radius * (fabsf(a1y) + fabsf(a2y)) + kHalf;
  const float n1x = -a1y, n1y = a1x, n2x = -a2y, n2y = a2x;
  const float e1 = s.radius * fabsf(a2x * n1x + a2y * n1y) + kHalf * (fabsf(n1x) + fabsf(n1y));
  const float e2 = s.radius * fabsf(a1x * n2x + a1y * n2y) + kHalf * (fabsf(n2x) + fabsf(n2y));
  uint32_t reach = 0;
#pragma unroll
  for (uint32_t w = 0; w < kWarps; ++w) {
    // quadrant w's centre, y up
    const float qx = tileX + static_cast<float>((w & 1u) * kQuadrant) + kHalf;
    const float qy = tileTop - static_cast<float>((w >> 1) * kQuadrant) - kHalf;
    const float dx = qx - s.cx, dy = qy - s.cy;
    const bool hit = fabsf(dx) <= ex && fabsf(dy) <= ey && fabsf(dx * n1x + dy * n1y) <= e1 &&
                     fabsf(dx * n2x + dy * n2y) <= e2;
    reach |= hit ? (1u << w) : 0u;
  }
  return reach;
}

// A thread's two pixels, packed so that Blackwell's paired FP32 instructions (FADD2, FMUL2,
// FFMA2: two independent IEEE operations, each rounded like its scalar form) work on both at once.
// A pixel is finished once its transmittance T is below the cutoff (T never grows); a pixel
// outside the target starts at T = -1.
struct PixelPair {
  float2 T = make_float2(1.0f, 1.0f), r = make_float2(0.0f, 0.0f), g = make_float2(0.0f, 0.0f),
         b = make_float2(0.0f, 0.0f);
};

__device__ __forceinline__ float2 pair(float v) { return make_float2(v, v); }

// 2^x by the hardware approximation (relative error about 2^-22).
__device__ __forceinline__ float exp2Approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Both pixels against one splat. px = the two pixel centres' x; m01dy, m11dy = m01 dy and
// m11 dy, shared by the row. The coverage terms u, v, q are the oracle's FP32 sequence per pixel
// (px - cx is px + (-cx) exactly); an uncovered or finished pixel takes alpha 0, which leaves
// its colour and transmittance bit for bit as they were, so a warp none of whose pixels the splat
// covers runs the blend all the same (no vote: the unrolled sweep keeps no branch between
// entries). alpha = min(1, 2^(log2 peak - q log2(e) / 2)) and T -= T alpha.
template <bool kCount>
__device__ __forceinline__ void blendPair(PixelPair& p, const float4 w0, const float4 w1,
                                          const float4 c, float2 px, float m01dy, float m11dy,
                                          float cutoff, uint32_t& blended) {
  const float2 dx = __fadd2_rn(px, pair(-w0.x));
  const float2 u = __ffma2_rn(pair(w0.z), dx, pair(m01dy));
  const float2 v = __ffma2_rn(pair(w1.x), dx, pair(m11dy));
  // q = u^2 + v^2 against 2 ln(255 peak): the oracle's (u^2 + v^2) / 2 <= ln(255 peak) with both
  // sides doubled, which is exact, so every decision is the same
  const float2 q = __ffma2_rn(u, u, __fmul2_rn(v, v));
  // |u|, |v| <= radius as one bound on the larger (a NaN u or v makes q NaN, so the q test
  // still fails as the separate bounds would)
  const bool c0 = p.T.x >= cutoff && fmaxf(fabsf(u.x), fabsf(v.x)) <= w1.z && q.x <= w1.w;
  const bool c1 = p.T.y >= cutoff && fmaxf(fabsf(u.y), fabsf(v.y)) <= w1.z && q.y <= w1.w;
  const float2 e = __ffma2_rn(q, pair(-0.7213475204444817f), pair(c.x));  // -q log2(e) / 2
  const float a0 = c0 ? fminf(exp2Approx(e.x), 1.0f) : 0.0f;
  const float a1 = c1 ? fminf(exp2Approx(e.y), 1.0f) : 0.0f;
  const float2 alpha = make_float2(a0, a1);
  const float2 weight = __fmul2_rn(p.T, alpha);
  p.r = __ffma2_rn(weight, pair(c.y), p.r);
  p.g = __ffma2_rn(weight, pair(c.z), p.g);
  p.b = __ffma2_rn(weight, pair(c.w), p.b);
  p.T = __ffma2_rn(pair(-1.0f), weight, p.T);
  if constexpr (kCount) blended += static_cast<uint32_t>(c0) + static_cast<uint32_t>(c1);
}

// The target one tile block draws into: the context's image, or its view's part of a batch image.
struct Target {
  uint32_t width, height, tilesX, tile, binsX, binBase;
  void* image;
};

template <int kFormat>
__device__ __forceinline__ void writePixel(const CompositeArgs& a, const Target& t, float T,
                                           float r, float g, float b, uint32_t col, uint32_t row) {
  if (col >= t.width || row >= t.height) return;
  float outR, outG, outB, outA;
  if (a.opaque) {
    outR = r + T * a.background[0];
    outG = g + T * a.background[1];
    outB = b + T * a.background[2];
    outA = 1.0f;
  } else {
    outR = r, outG = g, outB = b, outA = 1.0f - T;
  }
  outR = fminf(fmaxf(outR, 0.0f), 1.0f);
  outG = fminf(fmaxf(outG, 0.0f), 1.0f);
  outB = fminf(fmaxf(outB, 0.0f), 1.0f);
  outA = fminf(fmaxf(outA, 0.0f), 1.0f);
  const size_t at = static_cast<size_t>(row) * t.width + col;
  if constexpr (kFormat == kRgba32f) {
    reinterpret_cast<float4*>(t.image)[at] = make_float4(outR, outG, outB, outA);
  } else {
    const uint32_t r8 = __float2uint_rn(outR * 255.0f), g8 = __float2uint_rn(outG * 255.0f);
    const uint32_t b8 = __float2uint_rn(outB * 255.0f), a8 = __float2uint_rn(outA * 255.0f);
    reinterpret_cast<uint32_t*>(t.image)[at] = r8 | (g8 << 8) | (b8 << 16) | (a8 << 24);
  }
}

// kBatch: block b is batch-wide tile b; its view is the last one whose first tile is <= b.
// kCount: count blended fragments (a statistic; without it the loop saves an add per splat).
template <int kFormat, bool kBatch, bool kCount>
__global__ void __launch_bounds__(kThreads) compositeKernel(const __grid_constant__ CompositeArgs a) {
  chainedKernelStart();
  __shared__ CompositeSmem sm;
  Target t{a.width, a.height, a.tilesX, blockIdx.x, a.binsX, 0u, a.image};
  if constexpr (kBatch) {
    uint32_t lo = 0, hi = a.viewCount;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) / 2;
      if (__ldg(&a.views[mid].tileBase) <= blockIdx.x) lo = mid; else hi = mid;
    }
    const BatchView* v = a.views + lo;
    t.width = __ldg(&v->width);
    t.height = __ldg(&v->height);
    t.tilesX = __ldg(&v->tilesX);
    t.tile = blockIdx.x - __ldg(&v->tileBase);
    t.binsX = __ldg(&v->binsX);
    t.binBase = __ldg(&v->binBase);
    t.image = static_cast<char*>(a.image) +
              __ldg(reinterpret_cast<const unsigned long long*>(&v->pixelOffset)) *
                  (kFormat == kRgba32f ? 16u : 4u);
  }
  const uint32_t tx = t.tile % t.tilesX, ty = t.tile / t.tilesX;
  // the binning cell holding this tile (cells are 2x2 tiles)
  const uint32_t bin = t.binBase + (ty / 2) * t.binsX + tx / 2;
  const uint32_t warp = threadIdx.x >> 5, lane = laneId();
  const uint32_t col = tx * kTileSize + (warp & 1u) * kQuadrant + (lane % 4u) * 2u;  // and col + 1
  const uint32_t row = ty * kTileSize + (warp >> 1) * kQuadrant + lane / 4u;
  const float height = static_cast<float>(t.height);
  const float px0 = static_cast<float>(col) + 0.5f, px1 = px0 + 1.0f;
  const float py = static_cast<float>(t.height - row) - 0.5f;  // y up, as NDC
  const float tileX = static_cast<float>(tx * kTileSize);
  const float tileTop = height - static_cast<float>(ty * kTileSize);
  const float halfW = 0.5f * static_cast<float>(t.width);
  const float halfH = 0.5f * height;
  const uint2 range = a.ranges[bin];
  const uint32_t below = lanemaskLt();
  const float2 px = make_float2(px0, px1);
  PixelPair p;
  if (!(col < t.width && row < t.height)) p.T.x = -1.0f;
  if (!(col + 1 < t.width && row < t.height)) p.T.y = -1.0f;
  const float cutoff = a.cutoff;
  auto finished = [&] { return p.T.x < cutoff && p.T.y < cutoff; };
  uint32_t blended = 0, loaded = 0;
  for (uint32_t start = range.x; start < range.y; start += kEntries) {
    const uint32_t inBatch = min(kEntries, range.y - start);
    loaded += inBatch;
#pragma unroll
    for (uint32_t e = threadIdx.x; e < kEntries; e += kThreads) {
      if (e < inBatch) {
        const uint32_t v = a.values[start + e];
        const uint4* p = reinterpret_cast<const uint4*>(a.projected + v);
        Splat2D s;
        sm.reach[e] =
            static_cast<uint8_t>(coverageForm(__ldg(p), __ldg(p + 1), halfW, halfH, tileX, tileTop, s));
        sm.splat[e] = s;
      }
    }
    __syncthreads();
    if (!__all_sync(0xffffffffu, finished())) {
      // this warp's entries, in batch (= depth) order
      uint32_t count = 0;
      for (uint32_t c = 0; c < inBatch; c += 32) {
        const uint32_t j = c + lane;
        const bool mine = j < inBatch && ((sm.reach[j] >> warp) & 1u);
        const uint32_t m = __ballot_sync(0xffffffffu, mine);
        if (mine) sm.list[warp][count + __popc(m & below)] = static_cast<uint8_t>(j);
        count += __popc(m);
      }
      __syncwarp();
      for (uint32_t k0 = 0; k0 < count; k0 += 16) {
        if (__all_sync(0xffffffffu, finished())) break;
        const uint32_t k1 = min(count, k0 + 16);
#pragma unroll 4
        for (uint32_t k = k0; k < k1; ++k) {
          const Splat2D& s = sm.splat[sm.list[warp][k]];
          const float4 w0 = reinterpret_cast<const float4*>(&s)[0];
          const float4 w1 = reinterpret_cast<const float4*>(&s)[1];
          const float4 c = reinterpret_cast<const float4*>(&s)[2];
          const float dy = __fsub_rn(py, w0.y);
          const float m01dy = __fmul_rn(w0.w, dy), m11dy = __fmul_rn(w1.y, dy);
          blendPair<kCount>(p, w0, w1, c, px, m01dy, m11dy, cutoff, blended);
        }
      }
    }
    if (__syncthreads_count(finished() ? 0 : 1) == 0) break;
  }
  // blended fragments: one 64-bit add per block
  __shared__ unsigned long long blockFragments;
  if (threadIdx.x == 0) blockFragments = 0;
  __syncthreads();
  uint32_t warpSum = blended;
  for (int o = 16; o > 0; o >>= 1) warpSum += __shfl_xor_sync(0xffffffffu, warpSum, o);
  if (lane == 0 && warpSum) atomicAdd(&blockFragments, static_cast<unsigned long long>(warpSum));
  __syncthreads();
  if (kCount && threadIdx.x == 0 && blockFragments)
    atomicAdd(reinterpret_cast<unsigned long long*>(a.fragments), blockFragments);
  if (threadIdx.x == 0 && loaded) atomicAdd(a.loaded, loaded);
  writePixel<kFormat>(a, t, p.T.x, p.r.x, p.g.x, p.b.x, col, row);
  writePixel<kFormat>(a, t, p.T.y, p.r.y, p.g.y, p.b.y, col + 1, row);
}

}  // namespace

cudaError_t launchComposite(const CompositeArgs& a, cudaStream_t stream) {
  const uint32_t tiles = a.viewCount > 0 ? a.batchTiles : a.tilesX * a.tilesY;
  if (tiles == 0) return cudaSuccess;
  const bool f32 = a.format == kRgba32f, count = a.countFragments != 0;
  void (*kernel)(CompositeArgs);
  if (a.viewCount > 0) {
    kernel = f32 ? (count ? compositeKernel<kRgba32f, true, true> : compositeKernel<kRgba32f, true, false>)
                 : (count ? compositeKernel<kRgba8, true, true> : compositeKernel<kRgba8, true, false>);
  } else {
    kernel = f32 ? (count ? compositeKernel<kRgba32f, false, true> : compositeKernel<kRgba32f, false, false>)
                 : (count ? compositeKernel<kRgba8, false, true> : compositeKernel<kRgba8, false, false>);
  }
  return launchChained(kernel, tiles, kThreads, stream, a);
}

}  // namespace sk
