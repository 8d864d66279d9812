// Which binning cells (kBinSize pixels square) a projected splat's quad touches.
//
// The quad is the parallelogram c + s a1 + t a2, |s|, |t| <= radius, in pixel units (y up), with
// the half-rounded axes the compositor inverts. Its tiles are those of its pixel box whose
// square it overlaps by the separating-axis test (x, y and the normals of a1 and a2). The cell
// square is the pixel area, half a pixel beyond every pixel centre, so the test can only keep
// too many cells, never drop one the compositor would cover. ("Tile" below means a cell.)
//
// A span packs the result in 16 bytes: (x0 | y0 << 16, width | area << 16, mask lo, mask hi),
// bit k of the mask standing for box tile (x0 + k % width, y0 + k / width). A box of more than
// 64 tiles keeps all of them (its mask is unused); area 0 means no tile.
#pragma once
#include "sk_device.cuh"

namespace sk {

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

// The span of one projected record (two uint4 words) on a width x height target.
__device__ __forceinline__ uint4 tileSpan(const uint4 lo, const uint4 hi, float width, float height,
                                          uint32_t tilesX, uint32_t tilesY) {
  const Quad q = quadOf(lo, hi, 0.5f * width, 0.5f * height);
  const float ex = q.r * (fabsf(q.a1x) + fabsf(q.a2x)) + 1.0f;
  const float ey = q.r * (fabsf(q.a1y) + fabsf(q.a2y)) + 1.0f;
  if (!(isfinite(q.cx) && isfinite(q.cy) && isfinite(ex) && isfinite(ey) && q.r >= 0.0f))
    return make_uint4(0, 0, 0, 0);
  const float xa = floorf(q.cx - ex), xb = ceilf(q.cx + ex);
  const float ya = floorf(q.cy - ey), yb = ceilf(q.cy + ey);
  if (xb < 0.0f || xa >= width || yb < 0.0f || ya >= height) return make_uint4(0, 0, 0, 0);
  // columns [c0, c1]; rows from the y-up box: row = H - y_up - 0.5
  const uint32_t c0 = static_cast<uint32_t>(fmaxf(xa, 0.0f));
  const uint32_t c1 = static_cast<uint32_t>(fminf(xb, width - 1.0f));
  const uint32_t r0 = static_cast<uint32_t>(fmaxf(height - yb - 1.0f, 0.0f));
  const uint32_t r1 = static_cast<uint32_t>(fminf(fmaxf(height - ya, 0.0f), height - 1.0f));
  const uint32_t x0 = c0 / kBinSize, x1 = min(c1 / kBinSize, tilesX - 1);
  const uint32_t y0 = r0 / kBinSize, y1 = min(r1 / kBinSize, tilesY - 1);
  if (x0 > x1 || y0 > y1) return make_uint4(0, 0, 0, 0);
  const uint32_t w = x1 - x0 + 1, area = w * (y1 - y0 + 1);
  uint64_t mask = 0;
  if (area <= 64) {
    // Separating-axis test of the quad against each cell's pixel square (y up), the box's cells
    // row by row (bit k = cell (x0 + k % w, y0 + k / w)); the quad's extents along x, y and the
    // normals of a1 and a2 (along a normal of a1 the extent comes from t a2 only) are taken once.
    const float half = 0.5f * static_cast<float>(kBinSize);
    const float exq = q.r * (fabsf(q.a1x) + fabsf(q.a2x)) + half;
    const float eyq = q.r * (fabsf(q.a1y) + fabsf(q.a2y)) + half;
    const float n1x = -q.a1y, n1y = q.a1x, n2x = -q.a2y, n2y = q.a2x;
    const float e1 = q.r * fabsf(q.a2x * n1x + q.a2y * n1y) + half * (fabsf(n1x) + fabsf(n1y));
    const float e2 = q.r * fabsf(q.a1x * n2x + q.a1y * n2y) + half * (fabsf(n2x) + fabsf(n2y));
    uint32_t k = 0;
    for (uint32_t ty = y0; ty <= y1; ++ty) {
      const float ry = height - (static_cast<float>(ty * kBinSize) + half);
      const float dy = ry - q.cy;
      const bool rowIn = !(fabsf(dy) > eyq);
      for (uint32_t tx = x0; tx <= x1; ++tx, ++k) {
        const float rx = static_cast<float>(tx * kBinSize) + half;
        const float dx = rx - q.cx;
        const bool hit = rowIn && !(fabsf(dx) > exq) && !(fabsf(dx * n1x + dy * n1y) > e1) &&
                         !(fabsf(dx * n2x + dy * n2y) > e2);
        if (hit) mask |= 1ull << k;
      }
    }
    if (mask == 0) return make_uint4(0, 0, 0, 0);
  }
  return make_uint4(x0 | (y0 << 16), w | (area << 16), static_cast<uint32_t>(mask),
                    static_cast<uint32_t>(mask >> 32));
}

// Tiles a span lists.
__device__ __forceinline__ uint32_t spanCount(const uint4 s) {
  const uint32_t area = s.y >> 16;
  if (area > 64) return area;
  return static_cast<uint32_t>(__popc(s.z) + __popc(s.w));
}

// Position of the k-th (from 0) set bit of x; x holds more than k set bits. Bisection on halves.
__device__ __forceinline__ uint32_t kthSetBit(uint32_t x, uint32_t k) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t width = 16; width > 0; width >>= 1) {
    const uint32_t low = __popc(x & ((1u << width) - 1u));
    if (k >= low) {
      k -= low;
      x >>= width;
      pos += width;
    }
  }
  return pos;
}

// Cell of box position b of a box w cells wide whose first cell is `first`, on a grid tilesX
// cells wide. b / w in float: (b + 1/2) / w lies at least 1/(2w) from an integer, and the fast
// divide errs by at most 2 ulp of the quotient, less than that for b < 2^19 (a box holds at most
// 512 x 512 cells), so truncation gives the quotient.
__device__ __forceinline__ uint32_t boxCell(uint32_t first, uint32_t b, uint32_t w,
                                            uint32_t tilesX) {
  const uint32_t q = static_cast<uint32_t>(
      __fdividef(static_cast<float>(b) + 0.5f, static_cast<float>(w)));
  return first + q * tilesX + (b - q * w);
}

// First cell of a span's box on a grid tilesX cells wide.
__device__ __forceinline__ uint32_t spanFirstCell(const uint4 s, uint32_t tilesX) {
  return (s.x >> 16) * tilesX + (s.x & 0xffffu);
}

// The k-th (from 0) cell a span lists, k < spanCount(s).
__device__ __forceinline__ uint32_t spanCell(const uint4 s, uint32_t k, uint32_t tilesX) {
  const uint32_t w = s.y & 0xffffu, area = s.y >> 16;
  uint32_t bit = k;
  if (area <= 64) {
    const uint32_t nlo = __popc(s.z);
    bit = k < nlo ? kthSetBit(s.z, k) : 32u + kthSetBit(s.w, k - nlo);
  }
  return boxCell(spanFirstCell(s, tilesX), bit, w, tilesX);
}

// visit(cell) for every cell a span lists. A masked span is walked by its own lane; a box of
// more than 64 cells by the whole warp. Every lane of the warp calls this.
template <typename Visit>
__device__ __forceinline__ void visitCells(const uint4 s, uint32_t tilesX, Visit visit) {
  const uint32_t w = s.y & 0xffffu, area = s.y >> 16;
  const uint32_t first = spanFirstCell(s, tilesX);
  if (area <= 64) {
    for (uint32_t m = s.z; m != 0u; m &= m - 1) visit(boxCell(first, __ffs(m) - 1, w, tilesX));
    for (uint32_t m = s.w; m != 0u; m &= m - 1) visit(boxCell(first, 31 + __ffs(m), w, tilesX));
  }
  uint32_t big = __ballot_sync(0xffffffffu, area > 64);
  while (big != 0u) {
    const uint32_t src = __ffs(big) - 1;
    big &= big - 1;
    const uint32_t bw = __shfl_sync(0xffffffffu, w, src);
    const uint32_t barea = __shfl_sync(0xffffffffu, area, src);
    const uint32_t bfirst = __shfl_sync(0xffffffffu, first, src);
    for (uint32_t k = threadIdx.x & 31u; k < barea; k += 32) visit(boxCell(bfirst, k, bw, tilesX));
  }
}

}  // namespace sk
