// The visibility pass: per splat, reveal clip, opacity cut, view transform, near/far test,
// 2D covariance, ellipse axes, quad radius, edge margin, sub-pixel cut, SH colour and depth
// key; survivors compacted in SOURCE order.
//
// Follows splatkit-ios/Sources/SplatKitCore/rendering/metal/layout/SplatProjection.metalh:6-141
// and .../metal/cull/SplatVisibility.metal:16-106. The reference compacts with one atomic per
// SIMD group, so its survivor order depends on scheduling; here each 1024-splat tile counts
// its survivors, takes its offset by decoupled look-back and writes them in source order, so
// the sorted order downstream is deterministic and equal to a stable sort of (key, source
// position).
//
// Built with -fmad=false: every product and sum rounds on its own, in the order written.
#include <cuda_runtime.h>

#include "sk_device.cuh"
#include "sk_kernels.h"
#include "sk_launch.cuh"
#include "sk_tiles.cuh"

namespace sk {
namespace {

constexpr float kQuadMinAlpha = 2.0f / 255.0f;
constexpr float kBoundsRadius = 2.5f;
constexpr float kLodBoundsRadius = 5.0f;
constexpr float kMaxPixelRadius = 512.0f;
constexpr float kLowPassVariance = 0.3f;
constexpr float kProjectionFovClamp = 1.3f;
constexpr uint32_t kDepthKeyShift = 11;
constexpr uint32_t kDepthKeyMax = 65535;

constexpr uint32_t kThreads = 256;
constexpr uint32_t kItems = 4;
constexpr uint32_t kTileSplats = kThreads * kItems;

// Per block: i / 255 for the 8-bit colour and opacity channels (the same IEEE quotients the
// division gives, computed once per block instead of four times per splat) and the camera's
// near distance proj[14] / proj[10].
__shared__ float blockUnorm8[256];
__shared__ float blockZNear;

// Fills the block constants; the camera must be in shared memory. Ends with a barrier.
__device__ __forceinline__ void loadBlockConstants(const Camera& cam) {
  blockUnorm8[threadIdx.x] = static_cast<float>(threadIdx.x) / 255.0f;
  if (threadIdx.x == 0) blockZNear = cam.proj[14] / cam.proj[10];
  __syncthreads();
}

__device__ __forceinline__ void mulPoint(const float* m, float x, float y, float z, float w,
                                         float* o) {
#pragma unroll
  for (int r = 0; r < 4; ++r) o[r] = ((m[r] * x + m[4 + r] * y) + m[8 + r] * z) + m[12 + r] * w;
}

template <int D>
struct ShWords {
  static constexpr uint32_t kWords = shDeviceStride(D);
  uint32_t w[kWords > 0 ? kWords : 1];
  __device__ __forceinline__ void load(const uint32_t* sh, uint32_t index, uint32_t stride) {
    if constexpr (kWords > 0) {
      const uint4* p = reinterpret_cast<const uint4*>(sh + static_cast<size_t>(index) * stride);
#pragma unroll
      for (uint32_t i = 0; i < kWords / 4; ++i) {
        const uint4 v = __ldg(p + i);
        w[i * 4 + 0] = v.x, w[i * 4 + 1] = v.y, w[i * 4 + 2] = v.z, w[i * 4 + 3] = v.w;
      }
    }
  }
  __device__ __forceinline__ float at(uint32_t k, uint32_t ch) const {
    const uint32_t h = k * 3u + ch;
    return (h & 1u) ? highHalf(w[h >> 1]) : lowHalf(w[h >> 1]);
  }
};

// SplatProjection.metalh:50-76, summed in the order the oracle writes.
template <int D>
__device__ __forceinline__ void shColor(const ShWords<D>& s, float x, float y, float z,
                                        float* rgb) {
  const float C1 = 0.4886025119f;
  const float b0 = (-C1) * y, b1 = C1 * z, b2 = C1 * x;
  float q3 = 0, q4 = 0, q5 = 0, q6 = 0, q7 = 0;
  float q8 = 0, q9 = 0, q10 = 0, q11 = 0, q12 = 0, q13 = 0, q14 = 0;
  if constexpr (D >= 2) {
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    q3 = 1.0925484306f * xy;
    q4 = -1.0925484306f * yz;
    q5 = 0.3153915653f * (((2.0f * zz) - xx) - yy);
    q6 = -1.0925484306f * xz;
    q7 = 0.5462742153f * (xx - yy);
    if constexpr (D >= 3) {
      q8 = (-0.5900435899f * y) * ((3.0f * xx) - yy);
      q9 = (2.8906114426f * xy) * z;
      q10 = (-0.4570457995f * y) * (((4.0f * zz) - xx) - yy);
      q11 = (0.3731763326f * z) * (((2.0f * zz) - (3.0f * xx)) - (3.0f * yy));
      q12 = (-0.4570457995f * x) * (((4.0f * zz) - xx) - yy);
      q13 = (1.4453057213f * z) * (xx - yy);
      q14 = (-0.5900435899f * x) * (xx - (3.0f * yy));
    }
  }
#pragma unroll
  for (uint32_t ch = 0; ch < 3; ++ch) {
    float c = (b0 * s.at(0, ch) + b1 * s.at(1, ch)) - b2 * s.at(2, ch);
    if constexpr (D >= 2) {
      const float s2 =
          (((q3 * s.at(3, ch) + q4 * s.at(4, ch)) + q5 * s.at(5, ch)) + q6 * s.at(6, ch)) +
          q7 * s.at(7, ch);
      c = c + s2;
      if constexpr (D >= 3) {
        const float s3 = (((((q8 * s.at(8, ch) + q9 * s.at(9, ch)) + q10 * s.at(10, ch)) +
                            q11 * s.at(11, ch)) +
                           q12 * s.at(12, ch)) +
                          q13 * s.at(13, ch)) +
                         q14 * s.at(14, ch);
        c = c + s3;
      }
    }
    rgb[ch] = c;
  }
}

// SplatProjection.metalh:78-141 and SplatVisibility.metal:86-92. Writes the 8 words of a
// Projected record and the depth key; returns whether the splat survives.
template <int D, bool kKey16>
__device__ __forceinline__ bool projectSplat(const Camera& cam, const uint4 lo, const uint4 hi,
                                             uint32_t index, const uint32_t* sh, uint32_t shStride,
                                             uint32_t& key, uint32_t* out) {
  const float px = asF(lo.x), py = asF(lo.y), pz = asF(lo.z);
  const uint32_t rgba8 = lo.w;
  const uint32_t cov0 = hi.x, cov1 = hi.y, cov2 = hi.z, lodAlpha = hi.w;
  if (!(cam.reveal[0] - py >= 0.0f)) return false;
  const float ca = blockUnorm8[rgba8 >> 24];
  const float alpha = lodAlpha != 0u ? asF(lodAlpha) : ca;
  if (alpha < kQuadMinAlpha) return false;

  float v[4];
  mulPoint(cam.view, px, py, pz, 1.0f, v);
  if (v[2] >= 0.0f) return false;
  float clip[4];
  mulPoint(cam.proj, v[0], v[1], v[2], v[3], clip);
  if (clip[2] < 0.0f || clip[2] > clip[3]) return false;
  if (clip[3] <= blockZNear) return false;

  // projectCovariance (SplatProjection.metalh:6-24)
  const float vz = v[2];
  const float invZ = 1.0f / vz;
  const float invZ2 = invZ * invZ;
  const float limX = kProjectionFovClamp * cam.tanHalfFov[0];
  const float limY = kProjectionFovClamp * cam.tanHalfFov[1];
  const float vx = fminf(fmaxf(v[0] * invZ, -limX), limX) * vz;
  const float vy = fminf(fmaxf(v[1] * invZ, -limY), limY) * vz;
  const float fx = cam.focal[0], fy = cam.focal[1];
  const float j00 = fx * invZ;
  const float j11 = fy * invZ;
  const float j02 = ((-fx) * vx) * invZ2;
  const float j12 = ((-fy) * vy) * invZ2;
  float t0[3], t1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    t0[c] = j00 * cam.view[c * 4 + 0] + j02 * cam.view[c * 4 + 2];
    t1[c] = j11 * cam.view[c * 4 + 1] + j12 * cam.view[c * 4 + 2];
  }
  const float xx = lowHalf(cov0), xy = highHalf(cov0), xz = lowHalf(cov1);
  const float yy = highHalf(cov1), yz = lowHalf(cov2), zz = highHalf(cov2);
  const float V[3][3] = {{xx, xy, xz}, {xy, yy, yz}, {xz, yz, zz}};
  float m0[3], m1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    m0[c] = (t0[0] * V[0][c] + t0[1] * V[1][c]) + t0[2] * V[2][c];
    m1[c] = (t1[0] * V[0][c] + t1[1] * V[1][c]) + t1[2] * V[2][c];
  }
  const float ca2 = ((m0[0] * t0[0] + m0[1] * t0[1]) + m0[2] * t0[2]) + kLowPassVariance;
  const float cb2 = (m1[0] * t0[0] + m1[1] * t0[1]) + m1[2] * t0[2];
  const float cd2 = ((m1[0] * t1[0] + m1[1] * t1[1]) + m1[2] * t1[2]) + kLowPassVariance;

  // ellipseAxes (SplatProjection.metalh:26-37)
  const float det = ca2 * cd2 - cb2 * cb2;
  const float mean = 0.5f * (ca2 + cd2);
  const float dist = fmaxf(0.1f, sqrtf(fmaxf(mean * mean - det, 0.0f)));
  const float lambda1 = mean + dist;
  const float lambda2 = mean - dist;
  float e1x, e1y;
  if (cb2 == 0.0f) {
    e1x = (ca2 > cd2) ? 1.0f : 0.0f;
    e1y = (ca2 > cd2) ? 0.0f : 1.0f;
  } else {
    const float nx = cb2, ny = cd2 - lambda2;
    const float len = sqrtf(nx * nx + ny * ny);
    e1x = nx / len;
    e1y = ny / len;
  }
  const float s1 = sqrtf(lambda1);
  const float s2 = sqrtf(fmaxf(lambda2, 0.0f));
  const float a1x = e1x * s1, a1y = e1y * s1;
  const float a2x = e1y * s2, a2y = (-e1x) * s2;

  float radius = fminf(lodAlpha != 0u ? kLodBoundsRadius : kBoundsRadius,
                       sqrtf(2.0f * lnF32(fmaxf(alpha / kQuadMinAlpha, 1.0f))));
  const float sigmaPixels = sqrtf(fmaxf(a1x * a1x + a1y * a1y, a2x * a2x + a2y * a2y));
  radius = fminf(radius, kMaxPixelRadius / fmaxf(sigmaPixels, 1e-6f));

  const uint32_t axis1 = packHalf2(a1x, a1y);
  const uint32_t axis2 = packHalf2(a2x, a2y);
  const float extX = radius * (fabsf(lowHalf(axis1)) + fabsf(lowHalf(axis2)));
  const float extY = radius * (fabsf(highHalf(axis1)) + fabsf(highHalf(axis2)));
  const float marginX = (((extX + 0.5f) * 2.0f) * clip[3]) / cam.screenSize[0];
  const float marginY = (((extY + 0.5f) * 2.0f) * clip[3]) / cam.screenSize[1];
  if (fabsf(clip[0]) > clip[3] + marginX || fabsf(clip[1]) > clip[3] + marginY) return false;

  const float halfDifference = 0.5f * (ca2 - cd2);
  const float sourceVariance =
      (0.5f * (ca2 + cd2) + sqrtf(fmaxf(halfDifference * halfDifference + cb2 * cb2, 0.0f))) -
      kLowPassVariance;
  if (!(sqrtf(fmaxf(sourceVariance, 0.0f)) * radius >= cam.minPixelRadius)) return false;

  const float depth = -v[2];
  if (!isfinite(depth)) return false;

  float rgb[3] = {blockUnorm8[rgba8 & 0xffu], blockUnorm8[(rgba8 >> 8) & 0xffu],
                  blockUnorm8[(rgba8 >> 16) & 0xffu]};
  if constexpr (D >= 1) {
    ShWords<D> words;
    words.load(sh, index, shStride);
    const float dx = px - cam.cameraPosition[0];
    const float dy = py - cam.cameraPosition[1];
    const float dz = pz - cam.cameraPosition[2];
    const float len = sqrtf((dx * dx + dy * dy) + dz * dz);
    float c[3];
    shColor<D>(words, dx / len, dy / len, dz / len, c);
#pragma unroll
    for (int j = 0; j < 3; ++j) rgb[j] = fmaxf(rgb[j] + c[j], 0.0f);
  }

  if constexpr (kKey16) {
    const float zNear = blockZNear;
    const uint32_t steps = asU(fmaxf(depth, zNear)) - asU(zNear);
    key = min(steps >> kDepthKeyShift, kDepthKeyMax);
  } else {
    key = asU(depth);
  }
  out[0] = asU(clip[0] / clip[3]);
  out[1] = asU(clip[1] / clip[3]);
  out[2] = axis1;
  out[3] = axis2;
  out[4] = packHalf2(rgb[0], rgb[1]);
  out[5] = packHalf2(rgb[2], alpha);
  out[6] = asU(radius);
  out[7] = index;
  return true;
}

// SplatVisibility.metal:69-84: a labelled part's tint, brightness and opacity applied to the
// packed colours, in the same rounded steps as the host; false when the opacity drops the splat.
// A label without a state, or a state without a palette entry, draws unstyled.
__device__ __forceinline__ bool styleRecord(const PartLabels& parts, uint32_t index, uint32_t* rec) {
  const uint32_t label = parts.labels[index];
  if (label >= parts.stateCount) return true;
  const uint32_t state = __ldg(parts.states + label);
  if (state >= kPartStyles) return true;
  const PartStyle st = parts.palette[state];
  if (!(st.tintAmount != 0.0f || st.brightness != 1.0f || st.opacity != 1.0f)) return true;
  const float r = lowHalf(rec[4]), g = highHalf(rec[4]), b = lowHalf(rec[5]), a = highHalf(rec[5]);
  const float r2 = (r + (st.tint[0] - r) * st.tintAmount) * st.brightness;
  const float g2 = (g + (st.tint[1] - g) * st.tintAmount) * st.brightness;
  const float b2 = (b + (st.tint[2] - b) * st.tintAmount) * st.brightness;
  const float alpha = a * st.opacity;
  rec[4] = packHalf2(r2, g2);
  rec[5] = packHalf2(b2, alpha);
  return alpha >= kQuadMinAlpha;
}

// SplatProjection.metalh:177-189 for an encoded-space target: splats below the reveal level
// within `band` of it glow toward the reveal tint and brighten.
__device__ __forceinline__ void revealGlow(const Camera& cam, float height, uint32_t* rec) {
  if (!(cam.reveal[1] > 0.0f)) return;
  float glow = fminf(fmaxf(1.0f - (cam.reveal[0] - height) / cam.reveal[1], 0.0f), 1.0f);
  glow = glow * glow;
  if (!(glow > 0.0f)) return;
  const float r = lowHalf(rec[4]), g = highHalf(rec[4]), b = lowHalf(rec[5]), a = highHalf(rec[5]);
  const float t = cam.reveal[2] * glow, boost = 1.0f + cam.reveal[3] * glow;
  const float r2 = (r + (cam.revealTint[0] - r) * t) * boost;
  const float g2 = (g + (cam.revealTint[1] - g) * t) * boost;
  const float b2 = (b + (cam.revealTint[2] - b) * t) * boost;
  rec[4] = packHalf2(r2, g2);
  rec[5] = packHalf2(b2, a);
}

__device__ __forceinline__ uint32_t sourceIndex(const VisibilityArgs& a, uint32_t t) {
  if (a.rangeCount == 1) return a.single.offset + t;
  // SplatVisibility.metal:30-37: the range whose start is the last one <= t.
  uint32_t lo = 0, hi = a.rangeCount;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (a.rangeStarts[mid] <= t) lo = mid; else hi = mid;
  }
  return a.ranges[lo].offset + (t - a.rangeStarts[lo]);
}

// Shared memory of one tile: survivors staged at their source slot, then compacted.
struct VisibilitySmem {
  uint4 rec[kTileSplats * 2];     // projected records by source slot
  uint32_t key[kTileSplats];      // depth keys by source slot
  uint16_t slotOf[kTileSplats];   // survivor k of the tile -> its source slot
  uint32_t rowMask[kThreads / 32][kItems];
  uint32_t warpBase[kThreads / 32];
  uint32_t tileBase, tileCount;
};

// Projects one 1024-record tile into shared memory: survivors' keys and records at their
// source slot, and per warp row the mask of survivors. Part styles (when labels are given) and
// the reveal glow are applied to each survivor's record after its projection. indexOf(t) gives the record index of
// tile position t, or 0xffffffff past the end. keyHigh is or-ed into every key (the view id of a
// batch, above a 16-bit key). One record per row of the warp, not unrolled (the projection is
// large); the next row's record is fetched while this one is projected.
template <int D, bool kKey16, typename IndexOf>
__device__ __forceinline__ void projectTile(VisibilitySmem& s, const Camera& cam,
                                            const GpuSplat* __restrict__ splats,
                                            const uint32_t* __restrict__ sh, uint32_t shStride,
                                            const PartLabels& parts, uint32_t first,
                                            uint32_t keyHigh, IndexOf indexOf) {
  const uint32_t warp = threadIdx.x >> 5, lane = laneId();
  uint32_t index = indexOf(first);
  uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
  if (index != 0xffffffffu) {
    const uint4* p = reinterpret_cast<const uint4*>(splats + index);
    lo = __ldg(p), hi = __ldg(p + 1);
  }
#pragma unroll 1
  for (uint32_t r = 0; r < kItems; ++r) {
    uint32_t nextIndex = 0xffffffffu;
    uint4 nextLo = make_uint4(0, 0, 0, 0), nextHi = nextLo;
    if (r + 1 < kItems) {
      nextIndex = indexOf(first + (r + 1) * 32);
      if (nextIndex != 0xffffffffu) {
        const uint4* p = reinterpret_cast<const uint4*>(splats + nextIndex);
        nextLo = __ldg(p), nextHi = __ldg(p + 1);
      }
    }
    bool visible = false;
    const uint32_t slot = warp * (32 * kItems) + r * 32 + lane;
    if (index != 0xffffffffu) {
      uint32_t key, rec[8];
      visible = projectSplat<D, kKey16>(cam, lo, hi, index, sh, shStride, key, rec);
      if (visible && parts.labels) visible = styleRecord(parts, index, rec);
      if (visible) revealGlow(cam, asF(lo.y), rec);
      if (visible) {
        s.key[slot] = key | keyHigh;
        s.rec[2 * slot] = make_uint4(rec[0], rec[1], rec[2], rec[3]);
        s.rec[2 * slot + 1] = make_uint4(rec[4], rec[5], rec[6], rec[7]);
      }
    }
    const uint32_t mask = __ballot_sync(0xffffffffu, visible);
    if (lane == 0) s.rowMask[warp][r] = mask;
    index = nextIndex, lo = nextLo, hi = nextHi;
  }
  __syncwarp();
}

// Order-preserving compaction of the tile's survivors: warp totals, the tile's offset by
// decoupled look-back over status[0 .. tile], then survivor k of the tile -> its source slot.
// Leaves the offset and count in s.tileBase / s.tileCount.
__device__ __forceinline__ void compactTile(VisibilitySmem& s, uint64_t* status, uint32_t tile,
                                            uint32_t epoch, uint32_t* error) {
  const uint32_t warp = threadIdx.x >> 5, lane = laneId();
  uint32_t warpTotal = 0;
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) warpTotal += __popc(s.rowMask[warp][r]);
  if (lane == 0) s.warpBase[warp] = warpTotal;
  __syncthreads();
  if (warp == 0) {
    const uint32_t mine = lane < kThreads / 32 ? s.warpBase[lane] : 0u;
    uint32_t inclusive = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t up = __shfl_up_sync(0xffffffffu, inclusive, o);
      if (lane >= static_cast<uint32_t>(o)) inclusive += up;
    }
    const uint32_t aggregate = __shfl_sync(0xffffffffu, inclusive, 31);
    if (lane < kThreads / 32) s.warpBase[lane] = inclusive - mine;
    uint32_t exclusive = 0;
    if (tile == 0) {
      if (lane == 0) storeStatus(status, makeStatus(epoch, kFlagPrefix, aggregate));
    } else {
      if (lane == 0) storeStatus(status + tile, makeStatus(epoch, kFlagAggregate, aggregate));
      exclusive = warpLookback(status, tile, epoch, error);
      if (lane == 0) storeStatus(status + tile, makeStatus(epoch, kFlagPrefix, exclusive + aggregate));
    }
    if (lane == 0) {
      s.tileBase = exclusive;
      s.tileCount = aggregate;
    }
  }
  __syncthreads();
  uint32_t pos = s.warpBase[warp];
  const uint32_t below = lanemaskLt();
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    const uint32_t mask = s.rowMask[warp][r];
    if (mask & (1u << lane)) s.slotOf[pos + __popc(mask & below)] = warp * (32 * kItems) + r * 32 + lane;
    pos += __popc(mask);
  }
  __syncthreads();
}

// Coalesced copy-out: consecutive threads write consecutive survivors, with the tiles each
// survivor's quad touches on a width x height target.
// With digitPasses > 0 each key's 8-bit digits are counted into digits[pass][digit].
__device__ __forceinline__ void copyOutTile(const VisibilitySmem& s, uint32_t* keys,
                                            Projected* projected, uint4* spans, float width,
                                            float height, uint32_t tilesX, uint32_t tilesY,
                                            uint32_t (*digits)[256] = nullptr,
                                            uint32_t digitPasses = 0) {
  const uint32_t count = s.tileCount, base = s.tileBase;
  for (uint32_t k = threadIdx.x; k < count; k += kThreads) {
    const uint32_t slot = s.slotOf[k];
    const uint32_t key = s.key[slot];
    keys[base + k] = key;
    for (uint32_t p = 0; p < digitPasses; ++p) atomicAdd(&digits[p][(key >> (8 * p)) & 0xffu], 1u);
    const uint4 lo = s.rec[2 * slot], hi = s.rec[2 * slot + 1];
    uint4* o = reinterpret_cast<uint4*>(projected + base + k);
    o[0] = lo;
    o[1] = hi;
    spans[base + k] = tileSpan(lo, hi, width, height, tilesX, tilesY);
  }
}

template <int D, bool kKey16, bool kIndexed>
__global__ void __launch_bounds__(kThreads, 4)
    visibilityKernel(const Camera* __restrict__ camera, const __grid_constant__ VisibilityArgs a) {
  chainedKernelStart();
  __shared__ VisibilitySmem s;
  __shared__ Camera cam;
  __shared__ uint32_t digits[4][256];
  loadCamera(camera, &cam);
  for (uint32_t p = 0; p < a.sortPasses; ++p) digits[p][threadIdx.x] = 0;
  const uint32_t tile = takeTile(a.counters);  // its barrier also publishes the camera
  loadBlockConstants(cam);
  const uint32_t total = kIndexed ? min(*a.indexCount, a.total) : a.total;
  const uint32_t tiles = (total + kTileSplats - 1) / kTileSplats;
  if (tile < tiles) {
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    const uint32_t first = tile * kTileSplats + warp * (32 * kItems) + lane;
    auto indexOf = [&](uint32_t t) -> uint32_t {
      if (t >= total) return 0xffffffffu;
      const uint32_t index = kIndexed ? a.indices[t] : sourceIndex(a, t);
      if (index >= a.worldCount) {
        atomicOr(a.error, SK_DEVERR_BOUNDS);
        return 0xffffffffu;
      }
      return index;
    };
    projectTile<D, kKey16>(s, cam, a.splats, a.sh, a.shStride, a.parts, first, 0u, indexOf);
    compactTile(s, a.status, tile, a.epoch, a.error);
    if (tile == tiles - 1 && threadIdx.x == 0) *a.visibleCount = s.tileBase + s.tileCount;
    copyOutTile(s, a.keys, a.projected, a.spans, cam.screenSize[0], cam.screenSize[1], a.tilesX,
                a.tilesY, digits, a.sortPasses);
  }
  if (tiles == 0 && tile == 0 && threadIdx.x == 0) *a.visibleCount = 0;
  if (a.sortPasses) {
    __syncthreads();
    for (uint32_t p = 0; p < a.sortPasses; ++p) {
      const uint32_t v = digits[p][threadIdx.x];
      if (v) atomicAdd(&a.sortAccum[p * 256 + threadIdx.x], v);
    }
    if (finishTile(a.counters)) finishDigitHistograms(a.sortAccum, a.sortBases, a.sortPasses);
    return;
  }
  finishTile(a.counters);
}

// A batch of views in one launch. Work item i is a 1024-record chunk of one view's range (or of
// a LOD view's cut, in emission order: the chunks past the cut's length hold nothing); items
// are numbered view by view, so one look-back chain over all items places every view's
// survivors contiguously, in (view, source) order, and the first item of each view records
// where that view starts. Keys carry the view id above the 16-bit depth key, so one stable
// sort orders all views at once.
template <int D>
__global__ void __launch_bounds__(kThreads, 4)
    visibilityBatchKernel(const __grid_constant__ BatchVisibilityArgs a) {
  chainedKernelStart();
  __shared__ VisibilitySmem s;
  __shared__ Camera cam;
  __shared__ uint32_t viewOf;
  __shared__ BatchView view;
  const uint32_t item = takeTile(a.counters);
  if (item < a.items) {
    if (threadIdx.x == 0) {
      // the last view whose first item is <= item
      uint32_t lo = 0, hi = a.viewCount;
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (__ldg(&a.views[mid].itemStart) <= item) lo = mid; else hi = mid;
      }
      viewOf = lo;
    }
    __syncthreads();
    const uint32_t v = viewOf;
    loadCamera(a.cameras + v, &cam);
    if (threadIdx.x < sizeof(BatchView) / 4)
      reinterpret_cast<uint32_t*>(&view)[threadIdx.x] =
          __ldg(reinterpret_cast<const uint32_t*>(a.views + v) + threadIdx.x);
    __syncthreads();
    loadBlockConstants(cam);
    const uint32_t chunk = item - view.itemStart;
    const uint32_t warp = threadIdx.x >> 5, lane = laneId();
    const uint32_t first = chunk * kTileSplats + warp * (32 * kItems) + lane;
    // a LOD view draws its cut (written by this stream's selection before this kernel)
    const uint32_t drawn = view.indices ? min(view.count, *view.indexCount) : view.count;
    auto indexOf = [&](uint32_t t) -> uint32_t {
      if (t >= drawn) return 0xffffffffu;
      if (!view.indices) return view.offset + t;
      const uint32_t index = view.indices[t];
      if (index >= view.worldCount) {
        atomicOr(a.error, SK_DEVERR_BOUNDS);
        return 0xffffffffu;
      }
      return index;
    };
    projectTile<D, true>(s, cam, view.splats, view.sh, view.shStride, PartLabels{}, first, v << 16,
                         indexOf);
    compactTile(s, a.status, item, a.epoch, a.error);
    if (threadIdx.x == 0) {
      if (chunk == 0) a.viewFirst[v] = s.tileBase;
      if (item == a.items - 1) {
        a.viewFirst[a.viewCount] = s.tileBase + s.tileCount;
        *a.visibleCount = s.tileBase + s.tileCount;
      }
    }
    copyOutTile(s, a.keys, a.projected, a.spans, static_cast<float>(view.width),
                static_cast<float>(view.height), view.binsX, view.binsY);
  }
  finishTile(a.counters);
}


template <int D, bool kKey16, bool kIndexed>
void launchOne(const Camera* cam, const VisibilityArgs& a, uint32_t grid, cudaStream_t stream) {
  launchChained(visibilityKernel<D, kKey16, kIndexed>, grid, kThreads, stream, cam, a);
}

template <int D>
void launchDegree(const Camera* cam, const VisibilityArgs& a, bool key16, bool indexed,
                  uint32_t grid, cudaStream_t stream) {
  if (key16) {
    if (indexed) launchOne<D, true, true>(cam, a, grid, stream);
    else launchOne<D, true, false>(cam, a, grid, stream);
  } else {
    if (indexed) launchOne<D, false, true>(cam, a, grid, stream);
    else launchOne<D, false, false>(cam, a, grid, stream);
  }
}

}  // namespace

uint32_t visibilityTileSplats() { return kTileSplats; }

cudaError_t launchVisibilityBatch(const BatchVisibilityArgs& args, int shDegree,
                                  cudaStream_t stream) {
  if (args.items == 0 || args.viewCount == 0) return cudaSuccess;
  switch (shDegree) {
    case 0: launchChained(visibilityBatchKernel<0>, args.items, kThreads, stream, args); break;
    case 1: launchChained(visibilityBatchKernel<1>, args.items, kThreads, stream, args); break;
    case 2: launchChained(visibilityBatchKernel<2>, args.items, kThreads, stream, args); break;
    default: launchChained(visibilityBatchKernel<3>, args.items, kThreads, stream, args); break;
  }
  return cudaGetLastError();
}

cudaError_t launchVisibility(const Camera* cam, const VisibilityArgs& args, int shDegree,
                             bool key16, bool indexed, cudaStream_t stream) {
  const uint32_t grid = max(1u, (args.total + kTileSplats - 1) / kTileSplats);
  switch (shDegree) {
    case 0: launchDegree<0>(cam, args, key16, indexed, grid, stream); break;
    case 1: launchDegree<1>(cam, args, key16, indexed, grid, stream); break;
    case 2: launchDegree<2>(cam, args, key16, indexed, grid, stream); break;
    default: launchDegree<3>(cam, args, key16, indexed, grid, stream); break;
  }
  return cudaGetLastError();
}

}  // namespace sk
