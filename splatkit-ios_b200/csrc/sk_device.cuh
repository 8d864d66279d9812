// Device-side building blocks shared by the splat kernels: records, the per-view camera,
// IEEE helpers, the project's own binary16 conversion and natural log, and the decoupled
// look-back used by every order-preserving scan (visibility compaction, radix scatter,
// tile binning, LOD rounds).
//
// Bit-exactness contract: the cull/projection and LOD kernels are compiled with -fmad=false
// and IEEE divide/sqrt, and every expression keeps the operand order written here, so each
// product and sum rounds on its own. The composite kernel does its coverage decision with
// explicit __fmul_rn/__fadd_rn intrinsics for the same reason.
#pragma once
#include <cuda_fp16.h>

#include <cstdint>

#include "sk_layout.h"

namespace sk {

// ---- bit casts -------------------------------------------------------------------------
__device__ __forceinline__ uint32_t asU(float f) { return __float_as_uint(f); }
__device__ __forceinline__ float asF(uint32_t u) { return __uint_as_float(u); }

__device__ __forceinline__ uint32_t laneId() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemaskLt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---- binary16, round to nearest even, saturating to 65504, NaN kept -----------------
// The reference's float -> half packing rule (splat-core/include/splat/math/Half.h:12-38),
// written from the IEEE encodings.
// The hardware conversion rounds to nearest even (subnormals included); clamping to the largest
// finite half first turns its overflow to infinity into the saturation Half.h specifies, and
// a NaN keeps its sign with the quiet-NaN payload 0x7e00.
__device__ __forceinline__ uint32_t floatToHalf(float v) {
  if (v != v) return ((asU(v) >> 16) & 0x8000u) | 0x7e00u;
  const float c = fminf(fmaxf(v, -65504.0f), 65504.0f);
  return static_cast<uint32_t>(__half_as_ushort(__float2half_rn(c)));
}

// binary16 -> binary32 is exact, so the hardware conversion gives the same bits as any correct
// conversion (the host side decodes the IEEE fields by hand).
__device__ __forceinline__ float halfToFloat(uint32_t h) {
  return __half2float(__ushort_as_half(static_cast<unsigned short>(h & 0xffffu)));
}

__device__ __forceinline__ float lowHalf(uint32_t w) { return halfToFloat(w & 0xffffu); }
__device__ __forceinline__ float highHalf(uint32_t w) { return halfToFloat(w >> 16); }
__device__ __forceinline__ uint32_t packHalf2(float lo, float hi) {
  return floatToHalf(lo) | (floatToHalf(hi) << 16);
}
__device__ __forceinline__ float halfRound(float v) { return halfToFloat(floatToHalf(v)); }

// ---- natural log ----------------------------------------------------------------------
// Exponent/mantissa reduction to m in (sqrt(1/2), sqrt(2)], ln m = 2 atanh((m-1)/(m+1))
// (Abramowitz & Stegun 4.1.27) summed as f - s (f - R), and ln 2 split in a 16-bit head and
// a tail (Cody & Waite). Only rounded multiplies, adds and one IEEE divide: identical on the
// host and here. Within 1 ulp of the true log over the range the cull uses.
__device__ __forceinline__ float lnF32(float x) {
  if (x != x) return x;
  if (x < 0.0f) return __int_as_float(0x7fc00000);
  if (x == 0.0f) return -__int_as_float(0x7f800000);
  if (x == __int_as_float(0x7f800000)) return x;
  uint32_t bits = asU(x);
  int e = 0;
  if (bits < 0x00800000u) {
    x = __fmul_rn(x, 8388608.0f);
    bits = asU(x);
    e = -23;
  }
  e += static_cast<int>(bits >> 23) - 127;
  uint32_t mb = (bits & 0x007fffffu) | 0x3f800000u;
  if (mb > 0x3fb504f3u) {
    mb -= 0x00800000u;
    e += 1;
  }
  const float m = asF(mb);
  const float f = __fsub_rn(m, 1.0f);
  const float s = __fdiv_rn(f, __fadd_rn(2.0f, f));
  const float z = __fmul_rn(s, s);
  float r = 0.15384615384615385f;
  r = __fadd_rn(__fmul_rn(r, z), 0.18181818181818182f);
  r = __fadd_rn(__fmul_rn(r, z), 0.22222222222222222f);
  r = __fadd_rn(__fmul_rn(r, z), 0.2857142857142857f);
  r = __fadd_rn(__fmul_rn(r, z), 0.4f);
  r = __fadd_rn(__fmul_rn(r, z), 0.6666666666666666f);
  r = __fmul_rn(r, z);
  const float lnm = __fsub_rn(f, __fmul_rn(s, __fsub_rn(f, r)));
  const float fe = static_cast<float>(e);
  return __fadd_rn(__fmul_rn(fe, 0.693145751953125f),
                   __fadd_rn(lnm, __fmul_rn(fe, 1.428606820309417e-06f)));
}

// ---- programmatic dependent launch --------------------------------------------------------
// The frame's kernels are launched with programmatic stream serialization (launchChained): a
// kernel's blocks may be dispatched while its predecessor's last blocks still run, which hides
// the launch gap between dependent kernels. Every such kernel first waits for the predecessor
// to finish and flush (griddepcontrol.wait; a no-op when launched without the attribute), then
// lets its own successor be dispatched once all of its blocks are running.
__device__ __forceinline__ void chainedKernelStart() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Copies the 208-byte camera from device memory into shared memory (the caller syncs).
__device__ __forceinline__ void loadCamera(const Camera* __restrict__ src, Camera* dst) {
  constexpr uint32_t kWords = sizeof(Camera) / 4;
  if (threadIdx.x < kWords)
    reinterpret_cast<uint32_t*>(dst)[threadIdx.x] = __ldg(reinterpret_cast<const uint32_t*>(src) + threadIdx.x);
}

// ---- decoupled look-back ----------------------------------------------------------------
// A status word is [epoch:30 | flag:2 | value:32]. flag 1: the tile's own aggregate; flag 2:
// its inclusive prefix. Each launch uses a fresh epoch, so words left by earlier launches read
// as "not ready" and the status array never needs clearing. Every wait is bounded: after
// kSpinLimit polls the kernel records SK_DEVERR_LOOKBACK in the error word and carries on,
// so a lost predecessor costs a wrong frame and an error status, never a hung GPU.
constexpr uint32_t kFlagAggregate = 1u;
constexpr uint32_t kFlagPrefix = 2u;
constexpr uint32_t kSpinLimit = 1u << 21;

__device__ __forceinline__ uint64_t makeStatus(uint32_t epoch, uint32_t flag, uint32_t value) {
  return (static_cast<uint64_t>(epoch) << 34) | (static_cast<uint64_t>(flag) << 32) | value;
}
__device__ __forceinline__ void storeStatus(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t loadStatus(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Waits (bounded) until `p` holds a word of this epoch; returns it, or an aggregate of 0 with
// the error recorded when the wait gives up.
__device__ __forceinline__ uint64_t waitStatus(const uint64_t* p, uint32_t epoch,
                                               uint32_t* error) {
  for (uint32_t spin = 0; spin < kSpinLimit; ++spin) {
    const uint64_t w = loadStatus(p);
    if (static_cast<uint32_t>(w >> 34) == (epoch & 0x3fffffffu) && ((w >> 32) & 3u) != 0u) return w;
    if (spin > 64) __nanosleep(64);
  }
  atomicOr(error, SK_DEVERR_LOOKBACK);
  return makeStatus(epoch, kFlagPrefix, 0u);
}

// Look-back for one running sum, done by one warp: returns the exclusive prefix of `tile`.
// Lane i inspects predecessor (start - i); the window moves back 32 tiles at a time until a
// predecessor's inclusive prefix is found. All lanes return the same value.
__device__ __forceinline__ uint32_t warpLookback(const uint64_t* status, uint32_t tile,
                                                 uint32_t epoch, uint32_t* error) {
  uint32_t exclusive = 0;
  int start = static_cast<int>(tile) - 1;
  const uint32_t lane = laneId();
  while (start >= 0) {
    const int j = start - static_cast<int>(lane);
    uint64_t w = 0;
    if (j >= 0) w = waitStatus(status + j, epoch, error);
    const uint32_t flag = j >= 0 ? static_cast<uint32_t>((w >> 32) & 3u) : kFlagPrefix;
    const uint32_t value = j >= 0 ? static_cast<uint32_t>(w) : 0u;
    const uint32_t prefixMask = __ballot_sync(0xffffffffu, flag == kFlagPrefix);
    // the nearest predecessor holding a prefix closes the window
    const uint32_t stop = prefixMask ? (__ffs(prefixMask) - 1) : 32u;
    uint32_t mine = lane <= stop ? value : 0u;
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    exclusive += mine;
    if (prefixMask) break;
    start -= 32;
  }
  return exclusive;
}

// The dynamic tile index: tiles are handed out in the order blocks start, which is what makes
// waiting on a lower tile safe. The last block to finish resets both counters for the next
// launch on this stream (no spin: a plain arrival count).
__device__ __forceinline__ uint32_t takeTile(uint32_t* counters) {
  __shared__ uint32_t tile;
  if (threadIdx.x == 0) tile = atomicAdd(&counters[0], 1u);
  __syncthreads();
  return tile;
}
// Returns true in the block that arrived last (after every other block finished its writes).
__device__ __forceinline__ bool finishTile(uint32_t* counters) {
  __shared__ uint32_t last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t arrived = atomicAdd(&counters[1], 1u);
    last = arrived == gridDim.x - 1 ? 1u : 0u;
    if (last) {
      counters[0] = 0;
      counters[1] = 0;
      __threadfence();
    }
  }
  __syncthreads();
  return last != 0u;
}

// The end of a radix sort's digit histogram, run by the last block of the kernel that summed it
// (256 threads): accum[p][d] (the counts of digit d of pass p over all keys) become the exclusive
// digit bases bases[p][d], and the accumulators are cleared for the next sort.
__device__ __forceinline__ void finishDigitHistograms(uint32_t* accum, uint32_t* bases,
                                                      uint32_t passes) {
  __shared__ uint32_t warpSums[8];
  const uint32_t d = threadIdx.x, lane = laneId();
  for (uint32_t p = 0; p < passes; ++p) {
    const uint32_t v = __ldcg(&accum[p * 256 + d]);
    uint32_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= static_cast<uint32_t>(o)) inc += up;
    }
    if (lane == 31) warpSums[d >> 5] = inc;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t w = 0; w < (d >> 5); ++w) before += warpSums[w];
    bases[p * 256 + d] = before + inc - v;
    accum[p * 256 + d] = 0;
    __syncthreads();
  }
}

}  // namespace sk
