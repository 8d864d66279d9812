// Front-to-back compositing of 16x16 pixel tiles, one thread per pixel.
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
// Each block walks its tile's list in batches of 256 records. Thread i fetches record i of the
// batch (two 128-bit loads), turns it into the coverage form (pixel centre, inverse axes,
// radius, log cutoff, colour, pixel box) in shared memory, then every warp sweeps the batch
// over its 8x4 pixels, skipping at once the splats whose box misses them. The coverage decision
// uses explicit round-to-nearest intrinsics in a fixed order, so it is bit-identical to the
// host oracle's FP32 formula.
#include <cuda_runtime.h>

#include "sk_device.cuh"
#include "sk_kernels.h"

namespace sk {
namespace {

constexpr uint32_t kThreads = kTileSize * kTileSize;  // 256
constexpr uint32_t kWarpCols = 8, kWarpRows = 4;      // a warp's pixels

struct alignas(16) Splat2D {
  float cx, cy, m00, m01;
  float m10, m11, radius, lcut;
  float alpha, r, g, b;
  float x0, x1, y0, y1;  // box (y up) outside which no pixel centre is covered
};
static_assert(sizeof(Splat2D) == 64, "Splat2D is four 16-byte words");

__device__ __forceinline__ Splat2D coverageForm(const uint4 lo, const uint4 hi, float halfW,
                                                float halfH) {
  Splat2D s;
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
  s.alpha = highHalf(hi.y);
  s.lcut = lnF32(__fmul_rn(255.0f, s.alpha));
  s.radius = asF(hi.z);
  const bool any = det != 0.0f && isfinite(inv) && isfinite(s.cx) && isfinite(s.cy);
  if (!any) s.radius = -1.0f;
  s.r = lowHalf(hi.x);
  s.g = highHalf(hi.x);
  s.b = lowHalf(hi.y);
  // |s|,|t| <= radius bounds the offset by radius * (|a1| + |a2|) per axis; half a pixel of
  // slack keeps the box conservative against the rounding of the inverse.
  const float ex = s.radius * (fabsf(a1x) + fabsf(a2x)) + 0.5f;
  const float ey = s.radius * (fabsf(a1y) + fabsf(a2y)) + 0.5f;
  s.x0 = s.cx - ex, s.x1 = s.cx + ex, s.y0 = s.cy - ey, s.y1 = s.cy + ey;
  if (!any) s.x0 = 1.0f, s.x1 = -1.0f;
  return s;
}

template <int kFormat>
__global__ void __launch_bounds__(kThreads) compositeKernel(const __grid_constant__ CompositeArgs a) {
  __shared__ Splat2D batch[kThreads];
  const uint32_t tile = blockIdx.x;
  const uint32_t tx = tile % a.tilesX, ty = tile / a.tilesX;
  const uint32_t warp = threadIdx.x >> 5, lane = laneId();
  const uint32_t wx = warp & 1u, wy = warp >> 1;
  const uint32_t col0 = tx * kTileSize + wx * kWarpCols;
  const uint32_t row0 = ty * kTileSize + wy * kWarpRows;
  const uint32_t col = col0 + (lane % kWarpCols);
  const uint32_t row = row0 + (lane / kWarpCols);
  const bool inside = col < a.width && row < a.height;
  const float height = static_cast<float>(a.height);
  const float px = static_cast<float>(col) + 0.5f;
  const float py = static_cast<float>(a.height - row) - 0.5f;  // y up, as NDC
  // the warp's pixel centres, y up
  const float wx0 = static_cast<float>(col0) + 0.5f, wx1 = wx0 + (kWarpCols - 1);
  const float wy1 = height - (static_cast<float>(row0) + 0.5f), wy0 = wy1 - (kWarpRows - 1);
  const float halfW = 0.5f * static_cast<float>(a.width);
  const float halfH = 0.5f * height;
  const uint2 range = a.ranges[tile];
  float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
  bool done = !inside;
  uint32_t blended = 0, loaded = 0;
  for (uint32_t start = range.x; start < range.y; start += kThreads) {
    const uint32_t inBatch = min(kThreads, range.y - start);
    loaded += inBatch;
    if (threadIdx.x < inBatch) {
      const uint32_t v = a.values[start + threadIdx.x];
      const uint4* p = reinterpret_cast<const uint4*>(a.projected + v);
      batch[threadIdx.x] = coverageForm(__ldg(p), __ldg(p + 1), halfW, halfH);
    }
    __syncthreads();
    if (!__all_sync(0xffffffffu, done)) {
      for (uint32_t j = 0; j < inBatch; ++j) {
        const float4 box = reinterpret_cast<const float4*>(&batch[j])[3];
        // warp-uniform: the splat's box misses all 32 pixel centres of this warp
        if (box.y < wx0 || box.x > wx1 || box.w < wy0 || box.z > wy1) continue;
        if (done) continue;
        const float4 w0 = reinterpret_cast<const float4*>(&batch[j])[0];
        const float4 w1 = reinterpret_cast<const float4*>(&batch[j])[1];
        const float dx = __fsub_rn(px, w0.x), dy = __fsub_rn(py, w0.y);
        const float u = __fadd_rn(__fmul_rn(w0.z, dx), __fmul_rn(w0.w, dy));
        const float v = __fadd_rn(__fmul_rn(w1.x, dx), __fmul_rn(w1.y, dy));
        if (!(fabsf(u) <= w1.z && fabsf(v) <= w1.z)) continue;
        const float q = __fmul_rn(0.5f, __fadd_rn(__fmul_rn(u, u), __fmul_rn(v, v)));
        if (!(q <= w1.w)) continue;
        const float4 c = reinterpret_cast<const float4*>(&batch[j])[2];
        const float alpha = fminf(c.x * __expf(-q), 1.0f);
        const float weight = T * alpha;
        cr += weight * c.y;
        cg += weight * c.z;
        cb += weight * c.w;
        T *= 1.0f - alpha;
        ++blended;
        if (T < a.cutoff) done = true;
      }
    }
    if (__syncthreads_count(done ? 0 : 1) == 0) break;
  }
  // blended fragments: one 64-bit add per block
  __shared__ unsigned long long blockFragments;
  if (threadIdx.x == 0) blockFragments = 0;
  __syncthreads();
  uint32_t warpSum = blended;
  for (int o = 16; o > 0; o >>= 1) warpSum += __shfl_xor_sync(0xffffffffu, warpSum, o);
  if (lane == 0 && warpSum) atomicAdd(&blockFragments, static_cast<unsigned long long>(warpSum));
  __syncthreads();
  if (threadIdx.x == 0 && blockFragments)
    atomicAdd(reinterpret_cast<unsigned long long*>(a.fragments), blockFragments);
  if (threadIdx.x == 0 && loaded) atomicAdd(a.loaded, loaded);
  if (!inside) return;
  float outR, outG, outB, outA;
  if (a.opaque) {
    outR = cr + T * a.background[0];
    outG = cg + T * a.background[1];
    outB = cb + T * a.background[2];
    outA = 1.0f;
  } else {
    outR = cr, outG = cg, outB = cb, outA = 1.0f - T;
  }
  outR = fminf(fmaxf(outR, 0.0f), 1.0f);
  outG = fminf(fmaxf(outG, 0.0f), 1.0f);
  outB = fminf(fmaxf(outB, 0.0f), 1.0f);
  outA = fminf(fmaxf(outA, 0.0f), 1.0f);
  const size_t at = static_cast<size_t>(row) * a.width + col;
  if constexpr (kFormat == kRgba32f) {
    reinterpret_cast<float4*>(a.image)[at] = make_float4(outR, outG, outB, outA);
  } else {
    const uint32_t r8 = __float2uint_rn(outR * 255.0f), g8 = __float2uint_rn(outG * 255.0f);
    const uint32_t b8 = __float2uint_rn(outB * 255.0f), a8 = __float2uint_rn(outA * 255.0f);
    reinterpret_cast<uint32_t*>(a.image)[at] = r8 | (g8 << 8) | (b8 << 16) | (a8 << 24);
  }
}

}  // namespace

cudaError_t launchComposite(const CompositeArgs& a, cudaStream_t stream) {
  const uint32_t tiles = a.tilesX * a.tilesY;
  if (tiles == 0) return cudaSuccess;
  if (a.format == kRgba32f) compositeKernel<kRgba32f><<<tiles, kThreads, 0, stream>>>(a);
  else compositeKernel<kRgba8><<<tiles, kThreads, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace sk
