#include "world_prep.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>

namespace sk::host {
namespace {

uint32_t asUint(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

template <typename F>
void parallelFor(size_t n, int threads, F&& body) {
  threads = std::max(1, std::min<int>(threads, static_cast<int>((n + 65535) / 65536)));
  if (threads <= 1) {
    body(size_t{0}, n);
    return;
  }
  const size_t per = (n + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    const size_t b = std::min(n, per * t), e = std::min(n, b + per);
    pool.emplace_back([&, b, e] { body(b, e); });
  }
  for (auto& th : pool) th.join();
}

uint32_t packRgba8(float r, float g, float b, float a) {
  auto q = [](float v) {
    return static_cast<uint32_t>(std::lround(std::clamp(v, 0.0f, 1.0f) * 255.0f));
  };
  return q(r) | (q(g) << 8) | (q(b) << 16) | (q(a) << 24);
}

uint32_t packHalf2(float lo, float hi) {
  return static_cast<uint32_t>(floatToHalf(lo)) | (static_cast<uint32_t>(floatToHalf(hi)) << 16);
}

}  // namespace

uint16_t floatToHalf(float v) {
  const uint32_t x = asUint(v);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const uint32_t ax = x & 0x7fffffffu;
  const uint32_t e = ax >> 23;
  const uint32_t mant = ax & 0x7fffffu;
  if (e == 0xffu) return static_cast<uint16_t>(sign | (mant ? 0x7e00u : 0x7bffu));
  if (e < 113u) {
    const uint32_t shift = 126u - e;
    if (shift > 24u) return static_cast<uint16_t>(sign);
    const uint32_t full = mant | 0x800000u;
    const uint32_t h = full >> shift;
    const uint32_t rem = full & ((1u << shift) - 1u);
    const uint32_t mid = 1u << (shift - 1u);
    const uint32_t up = (rem > mid || (rem == mid && (h & 1u))) ? 1u : 0u;
    return static_cast<uint16_t>(sign | (h + up));
  }
  uint32_t h = ((e - 112u) << 10) | (mant >> 13);
  const uint32_t rem = mant & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;
  if (h >= 0x7c00u) h = 0x7bffu;
  return static_cast<uint16_t>(sign | h);
}

float halfToFloat(uint16_t h) {
  const uint32_t sign = (static_cast<uint32_t>(h) & 0x8000u) << 16;
  const uint32_t e = (h >> 10) & 0x1fu;
  const uint32_t m = h & 0x3ffu;
  uint32_t bits;
  if (e == 0) {
    float mag = static_cast<float>(m) * 5.9604644775390625e-08f;
    std::memcpy(&bits, &mag, 4);
    bits |= sign;
  } else if (e == 31) {
    bits = sign | 0x7f800000u | (m << 13);
  } else {
    bits = sign | ((e + 112u) << 23) | (m << 13);
  }
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

void packSplats(const CloudRef& c, size_t offset, size_t count, GpuSplat* out, int threads) {
  parallelFor(count, threads, [&](size_t b, size_t e) {
    for (size_t k = b; k < e; ++k) {
      const size_t i = offset + k;
      GpuSplat& g = out[k];
      std::memcpy(g.position, &c.positions[i * 3], sizeof(g.position));
      const float alpha = c.alphas[i];
      g.rgba8 = packRgba8(c.colors[i * 3], c.colors[i * 3 + 1], c.colors[i * 3 + 2], alpha);
      g.lodAlpha = alpha > 1.0f ? asUint(alpha) : 0u;
      const float* v = &c.covariances[i * 6];
      g.cov[0] = packHalf2(v[0], v[1]);
      g.cov[1] = packHalf2(v[2], v[3]);
      g.cov[2] = packHalf2(v[4], v[5]);
    }
  });
}

void packSh(const CloudRef& c, int degree, size_t offset, size_t count, uint32_t* out,
            uint32_t stride, int threads) {
  if (degree <= 0 || count == 0) return;
  const size_t source = size_t{3} * shCoefficients(c.shDegree);
  const size_t halves = size_t{3} * shCoefficients(degree);
  parallelFor(count, threads, [&](size_t b, size_t e) {
    for (size_t k = b; k < e; ++k) {
      const float* src = &c.sh[(offset + k) * source];
      for (size_t w = 0; w < stride; ++w) {
        const size_t h = w * 2;
        const uint32_t lo = h < halves ? floatToHalf(src[h]) : 0u;
        const uint32_t hi = h + 1 < halves ? floatToHalf(src[h + 1]) : 0u;
        out[k * stride + w] = lo | (hi << 16);
      }
    }
  });
}

int64_t lodDepth(const LodNode* layout, uint32_t nodeCount, uint32_t leafCount,
                 std::string* error) {
  constexpr uint32_t kMaxDepth = 255;
  auto fail = [&](const char* why) {
    if (error) *error = why;
    return int64_t{-1};
  };
  if (nodeCount == 0) return fail("LOD tree has no nodes");
  std::vector<uint32_t> depth(nodeCount, 0);
  size_t next = 1, leaves = 0;
  uint32_t deepest = 0;
  for (size_t i = 0; i < nodeCount; ++i) {
    if (i >= next) return fail("LOD has unreachable nodes");
    const LodNode& node = layout[i];
    if (node.childCount == 0) {
      ++leaves;
      continue;
    }
    if (node.childStart != next || node.childCount > nodeCount - next || depth[i] >= kMaxDepth)
      return fail("LOD child ranges are not a bounded BFS tree");
    for (size_t k = next; k < next + node.childCount; ++k) depth[k] = depth[i] + 1;
    deepest = std::max(deepest, depth[i] + 1);
    next += node.childCount;
  }
  if (next != nodeCount || leaves != leafCount) return fail("LOD topology or leaf count invalid");
  return deepest;
}

float LodThreshold::update(uint32_t selected, uint32_t limited, uint32_t limit) {
  constexpr float kRaise = 1.1f;
  constexpr float kRelax = 1.03f;
  if (limited > 0) {
    pixels_ = std::min(pixels_ * kRaise, std::max(kCeilingPixels, policy_));
  } else if (selected < limit / 10 * 9) {
    pixels_ = std::max(pixels_ / kRelax, policy_);
  }
  return pixels_;
}

uint64_t worldBytes(uint64_t records, int shDegree, uint64_t drawCapacity, uint64_t clusters,
                    uint64_t leafRefs) {
  const uint64_t drawBytesPerSplat = sizeof(Projected) + 2 * 2 * 4 + 4;
  const uint64_t walkBytesPerCluster = 16 + 8 + 16 + 2 * 4;
  const uint64_t packedSh = shDegree <= 0 ? 0 : (uint64_t{shCoefficients(shDegree)} * 3 + 1) / 2;
  const uint64_t record = sizeof(GpuSplat) + packedSh * 4;
  return records * record + drawCapacity * drawBytesPerSplat +
         clusters * (sizeof(LodCluster) + walkBytesPerCluster) + leafRefs * 4;
}

}  // namespace sk::host
