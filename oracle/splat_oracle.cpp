// Test infrastructure only — see splat_oracle.h for what this restates and the arithmetic
// contract it shares with the CUDA kernels. Every function cites the reference lines it
// follows (paths inside packages/splatkit-ios/Sources/SplatKitCore/rendering/metal/ unless
// given in full).
#include "splat_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>
#include <thread>
#include <vector>

namespace {

// ---- bit casts and IEEE helpers -------------------------------------------------------

inline uint32_t asUint(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline float asFloat(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
// Metal's min/max/clamp return the non-NaN operand, like C's fmin/fmax and CUDA's fminf.
inline float fmn(float a, float b) { return std::fmin(a, b); }
inline float fmx(float a, float b) { return std::fmax(a, b); }
inline float clampf(float x, float lo, float hi) { return fmn(fmx(x, lo), hi); }

template <typename F>
void parallelFor(size_t n, int threads, F&& body) {
  threads = std::max(1, threads);
  if (threads == 1 || n < 2) {
    body(0, n, 0);
    return;
  }
  const size_t per = (n + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    const size_t begin = std::min(n, per * t), end = std::min(n, begin + per);
    pool.emplace_back([&, begin, end, t] { body(begin, end, t); });
  }
  for (auto& th : pool) th.join();
}

// ---- project-owned numerics ----------------------------------------------------------

// Natural log for binary32: exponent/mantissa reduction to m in (sqrt(1/2), sqrt(2)], then
// ln m = 2 atanh(s) with s = (m - 1) / (m + 1) (Abramowitz & Stegun 4.1.27), summed as
// f - s (f - R) with R the atanh series beyond its first term, and ln 2 split in a
// 16-bit head and a tail (Cody & Waite) so e * ln2_hi is exact.
float lnF32(float x) {
  if (x != x) return x;
  if (x < 0.0f) return std::numeric_limits<float>::quiet_NaN();
  if (x == 0.0f) return -std::numeric_limits<float>::infinity();
  if (x == std::numeric_limits<float>::infinity()) return x;
  uint32_t bits = asUint(x);
  int e = 0;
  if (bits < 0x00800000u) {  // subnormal: scale into the normal range
    x = x * 8388608.0f;
    bits = asUint(x);
    e = -23;
  }
  e += static_cast<int>(bits >> 23) - 127;
  uint32_t mb = (bits & 0x007fffffu) | 0x3f800000u;
  if (mb > 0x3fb504f3u) {
    mb -= 0x00800000u;
    e += 1;
  }
  const float m = asFloat(mb);
  const float f = m - 1.0f;
  const float s = f / (2.0f + f);
  const float z = s * s;
  float r = 0.15384615384615385f;  // 2/13
  r = r * z + 0.18181818181818182f;  // 2/11
  r = r * z + 0.22222222222222222f;  // 2/9
  r = r * z + 0.2857142857142857f;   // 2/7
  r = r * z + 0.4f;                  // 2/5
  r = r * z + 0.6666666666666666f;   // 2/3
  r = r * z;
  const float lnm = f - s * (f - r);
  const float fe = static_cast<float>(e);
  const float kLn2Hi = 0.693145751953125f;
  const float kLn2Lo = 1.428606820309417e-06f;
  return fe * kLn2Hi + (lnm + fe * kLn2Lo);
}

// float -> binary16, round to nearest even, saturating at 65504, NaN kept (the reference's
// core/include/splat/math/Half.h:12-38 semantics, written from the IEEE encoding).
uint16_t floatToHalf(float v) {
  const uint32_t x = asUint(v);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const uint32_t ax = x & 0x7fffffffu;
  const uint32_t e = ax >> 23;
  const uint32_t mant = ax & 0x7fffffu;
  if (e == 0xffu) return static_cast<uint16_t>(sign | (mant ? 0x7e00u : 0x7bffu));
  if (e < 113u) {  // below 2^-14: a subnormal half or zero
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
  if (e == 0) {
    // m * 2^-24, exact in binary32.
    const float mag = static_cast<float>(m) * 5.9604644775390625e-08f;
    return asFloat(asUint(mag) | sign);
  }
  if (e == 31) return asFloat(sign | 0x7f800000u | (m << 13));
  return asFloat(sign | ((e + 112u) << 23) | (m << 13));
}

inline float halfRound(float v) { return halfToFloat(floatToHalf(v)); }
inline float lowHalf(uint32_t packed) { return halfToFloat(static_cast<uint16_t>(packed & 0xffffu)); }
inline float highHalf(uint32_t packed) { return halfToFloat(static_cast<uint16_t>(packed >> 16)); }
inline uint32_t packHalf2(float lo, float hi) {
  return static_cast<uint32_t>(floatToHalf(lo)) | (static_cast<uint32_t>(floatToHalf(hi)) << 16);
}

// ---- constants (metal/layout/SplatTypes.metalh:81-118, MetalShaderTypes.h:35) --------
constexpr float kQuadMinAlpha = 2.0f / 255.0f;
constexpr float kBoundsRadius = 2.5f;
constexpr float kLodBoundsRadius = 5.0f;
constexpr float kMaxPixelRadius = 512.0f;
constexpr float kLowPassVariance = 0.3f;
constexpr float kProjectionFovClamp = 1.3f;
constexpr uint32_t kDepthKeyShift = 11;   // metal/cull/SplatVisibility.metal:21
constexpr uint32_t kDepthKeyMax = 65535;  // metal/cull/SplatVisibility.metal:22

// Column-major 4x4 times (x, y, z, w): ((m0 x + m1 y) + m2 z) + m3 w, per row.
inline void mulPoint(const float* m, float x, float y, float z, float w, float* out4) {
  for (int r = 0; r < 4; ++r) {
    const float a = m[r] * x;
    const float b = m[4 + r] * y;
    const float c = m[8 + r] * z;
    const float d = m[12 + r] * w;
    out4[r] = ((a + b) + c) + d;
  }
}

// metal/layout/SplatProjection.metalh:6-24. Returns (a, b, d) of the 2D covariance + low pass.
void projectCovariance(const sko_camera& cam, const float* viewPos, float xx, float xy, float xz,
                       float yy, float yz, float zz, float* cov3) {
  const float vz = viewPos[2];
  const float invZ = 1.0f / vz;
  const float invZ2 = invZ * invZ;
  const float limX = kProjectionFovClamp * cam.tanHalfFov[0];
  const float limY = kProjectionFovClamp * cam.tanHalfFov[1];
  const float vx = clampf(viewPos[0] * invZ, -limX, limX) * vz;
  const float vy = clampf(viewPos[1] * invZ, -limY, limY) * vz;
  const float fx = cam.focal[0], fy = cam.focal[1];
  // J rows: (j00, 0, j02), (0, j11, j12); the third row is zero.
  const float j00 = fx * invZ;
  const float j11 = fy * invZ;
  const float j02 = ((-fx) * vx) * invZ2;
  const float j12 = ((-fy) * vy) * invZ2;
  // W[k][c] = view column c, row k (the upper 3x3).
  const float* v = cam.view;
  float t0[3], t1[3];
  for (int c = 0; c < 3; ++c) {
    const float w0 = v[c * 4 + 0], w1 = v[c * 4 + 1], w2 = v[c * 4 + 2];
    t0[c] = j00 * w0 + j02 * w2;
    t1[c] = j11 * w1 + j12 * w2;
  }
  const float V[3][3] = {{xx, xy, xz}, {xy, yy, yz}, {xz, yz, zz}};
  float m0[3], m1[3];  // rows of T * V
  for (int c = 0; c < 3; ++c) {
    m0[c] = (t0[0] * V[0][c] + t0[1] * V[1][c]) + t0[2] * V[2][c];
    m1[c] = (t1[0] * V[0][c] + t1[1] * V[1][c]) + t1[2] * V[2][c];
  }
  const float a = (m0[0] * t0[0] + m0[1] * t0[1]) + m0[2] * t0[2];
  const float b = (m1[0] * t0[0] + m1[1] * t0[1]) + m1[2] * t0[2];
  const float d = (m1[0] * t1[0] + m1[1] * t1[1]) + m1[2] * t1[2];
  cov3[0] = a + kLowPassVariance;
  cov3[1] = b;
  cov3[2] = d + kLowPassVariance;
}

// metal/layout/SplatProjection.metalh:26-37.
void ellipseAxes(const float* cov3, float* axis1, float* axis2) {
  const float a = cov3[0], b = cov3[1], d = cov3[2];
  const float det = a * d - b * b;
  const float mean = 0.5f * (a + d);
  const float dist = fmx(0.1f, std::sqrt(fmx(mean * mean - det, 0.0f)));
  const float lambda1 = mean + dist;
  const float lambda2 = mean - dist;
  float e1x, e1y;
  if (b == 0.0f) {
    e1x = (a > d) ? 1.0f : 0.0f;
    e1y = (a > d) ? 0.0f : 1.0f;
  } else {
    const float nx = b, ny = d - lambda2;
    const float len = std::sqrt(nx * nx + ny * ny);
    e1x = nx / len;
    e1y = ny / len;
  }
  const float s1 = std::sqrt(lambda1);
  const float s2 = std::sqrt(fmx(lambda2, 0.0f));
  axis1[0] = e1x * s1;
  axis1[1] = e1y * s1;
  axis2[0] = e1y * s2;
  axis2[1] = (-e1x) * s2;
}

// metal/layout/SplatProjection.metalh:39-76. Coefficient k, channel ch of splat `index`.
inline float shValue(const uint32_t* sh, uint32_t base, uint32_t k, uint32_t ch) {
  const uint32_t h = k * 3u + ch;
  const uint32_t word = sh[base + h / 2u];
  return (h & 1u) == 0u ? lowHalf(word) : highHalf(word);
}

void shColor(const uint32_t* sh, uint32_t base, int degree, float x, float y, float z,
             float* rgb) {
  const float C1 = 0.4886025119f;
  const float C2_0 = 1.0925484306f, C2_1 = -1.0925484306f, C2_2 = 0.3153915653f,
              C2_3 = -1.0925484306f, C2_4 = 0.5462742153f;
  const float C3_0 = -0.5900435899f, C3_1 = 2.8906114426f, C3_2 = -0.4570457995f,
              C3_3 = 0.3731763326f, C3_4 = -0.4570457995f, C3_5 = 1.4453057213f,
              C3_6 = -0.5900435899f;
  const float b0 = (-C1) * y, b1 = C1 * z, b2 = C1 * x;
  float xx = 0, yy = 0, zz = 0, xy = 0, yz = 0, xz = 0;
  float q3 = 0, q4 = 0, q5 = 0, q6 = 0, q7 = 0;
  float q8 = 0, q9 = 0, q10 = 0, q11 = 0, q12 = 0, q13 = 0, q14 = 0;
  if (degree >= 2) {
    xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    q3 = C2_0 * xy;
    q4 = C2_1 * yz;
    q5 = C2_2 * (((2.0f * zz) - xx) - yy);
    q6 = C2_3 * xz;
    q7 = C2_4 * (xx - yy);
    if (degree >= 3) {
      q8 = (C3_0 * y) * ((3.0f * xx) - yy);
      q9 = (C3_1 * xy) * z;
      q10 = (C3_2 * y) * (((4.0f * zz) - xx) - yy);
      q11 = (C3_3 * z) * (((2.0f * zz) - (3.0f * xx)) - (3.0f * yy));
      q12 = (C3_4 * x) * (((4.0f * zz) - xx) - yy);
      q13 = (C3_5 * z) * (xx - yy);
      q14 = (C3_6 * x) * (xx - (3.0f * yy));
    }
  }
  for (uint32_t ch = 0; ch < 3; ++ch) {
    float c = (b0 * shValue(sh, base, 0, ch) + b1 * shValue(sh, base, 1, ch)) -
              b2 * shValue(sh, base, 2, ch);
    if (degree >= 2) {
      const float s2 = (((q3 * shValue(sh, base, 3, ch) + q4 * shValue(sh, base, 4, ch)) +
                         q5 * shValue(sh, base, 5, ch)) +
                        q6 * shValue(sh, base, 6, ch)) +
                       q7 * shValue(sh, base, 7, ch);
      c = c + s2;
      if (degree >= 3) {
        const float s3 =
            (((((q8 * shValue(sh, base, 8, ch) + q9 * shValue(sh, base, 9, ch)) +
                q10 * shValue(sh, base, 10, ch)) +
               q11 * shValue(sh, base, 11, ch)) +
              q12 * shValue(sh, base, 12, ch)) +
             q13 * shValue(sh, base, 13, ch)) +
            q14 * shValue(sh, base, 14, ch);
        c = c + s3;
      }
    }
    rgb[ch] = c;
  }
}

// metal/layout/SplatProjection.metalh:78-141 plus the key of metal/cull/SplatVisibility.metal:86-92.
bool projectOne(const sko_camera& cam, const sko_splat& s, uint32_t index, const uint32_t* sh,
                uint32_t shStride, int shDegree, int keyBits, uint32_t* keyOut,
                sko_projected* out) {
  if (!(cam.reveal[0] - s.position[1] >= 0.0f)) return false;
  const float ca = static_cast<float>(s.rgba8 >> 24) / 255.0f;
  const float alpha = s.lodAlpha != 0u ? asFloat(s.lodAlpha) : ca;
  if (alpha < kQuadMinAlpha) return false;

  float view4[4];
  mulPoint(cam.view, s.position[0], s.position[1], s.position[2], 1.0f, view4);
  if (view4[2] >= 0.0f) return false;
  float clip[4];
  mulPoint(cam.proj, view4[0], view4[1], view4[2], view4[3], clip);
  if (clip[2] < 0.0f || clip[2] > clip[3]) return false;
  if (clip[3] <= cam.proj[14] / cam.proj[10]) return false;

  float cov2[3];
  projectCovariance(cam, view4, lowHalf(s.cov[0]), highHalf(s.cov[0]), lowHalf(s.cov[1]),
                    highHalf(s.cov[1]), lowHalf(s.cov[2]), highHalf(s.cov[2]), cov2);
  float axis1[2], axis2[2];
  ellipseAxes(cov2, axis1, axis2);

  float radius = fmn(s.lodAlpha != 0u ? kLodBoundsRadius : kBoundsRadius,
                     std::sqrt(2.0f * lnF32(fmx(alpha / kQuadMinAlpha, 1.0f))));
  const float sigmaPixels = std::sqrt(
      fmx(axis1[0] * axis1[0] + axis1[1] * axis1[1], axis2[0] * axis2[0] + axis2[1] * axis2[1]));
  radius = fmn(radius, kMaxPixelRadius / fmx(sigmaPixels, 1e-6f));

  const float p1x = halfRound(axis1[0]), p1y = halfRound(axis1[1]);
  const float p2x = halfRound(axis2[0]), p2y = halfRound(axis2[1]);
  const float extX = radius * (std::fabs(p1x) + std::fabs(p2x));
  const float extY = radius * (std::fabs(p1y) + std::fabs(p2y));
  const float marginX = (((extX + 0.5f) * 2.0f) * clip[3]) / cam.screenSize[0];
  const float marginY = (((extY + 0.5f) * 2.0f) * clip[3]) / cam.screenSize[1];
  if (std::fabs(clip[0]) > clip[3] + marginX || std::fabs(clip[1]) > clip[3] + marginY)
    return false;

  const float halfDifference = 0.5f * (cov2[0] - cov2[2]);
  const float sourceVariance =
      (0.5f * (cov2[0] + cov2[2]) +
       std::sqrt(fmx(halfDifference * halfDifference + cov2[1] * cov2[1], 0.0f))) -
      kLowPassVariance;
  if (!(std::sqrt(fmx(sourceVariance, 0.0f)) * radius >= cam.minPixelRadius)) return false;

  float rgb[3] = {static_cast<float>(s.rgba8 & 0xffu) / 255.0f,
                  static_cast<float>((s.rgba8 >> 8) & 0xffu) / 255.0f,
                  static_cast<float>((s.rgba8 >> 16) & 0xffu) / 255.0f};
  if (shDegree >= 1) {
    const float dx = s.position[0] - cam.cameraPosition[0];
    const float dy = s.position[1] - cam.cameraPosition[1];
    const float dz = s.position[2] - cam.cameraPosition[2];
    const float len = std::sqrt((dx * dx + dy * dy) + dz * dz);
    float c[3];
    shColor(sh, index * shStride, shDegree, dx / len, dy / len, dz / len, c);
    for (int j = 0; j < 3; ++j) rgb[j] = fmx(rgb[j] + c[j], 0.0f);
  }

  // metal/cull/SplatVisibility.metal:90-92: both key widths order by view depth; the splat is
  // visible only when that depth is finite.
  const float depth = -view4[2];
  if (!std::isfinite(depth)) return false;
  uint32_t key;
  if (keyBits == 16) {
    const float zNear = cam.proj[14] / cam.proj[10];
    const uint32_t steps = asUint(fmx(depth, zNear)) - asUint(zNear);
    key = std::min(steps >> kDepthKeyShift, kDepthKeyMax);
  } else {
    key = asUint(depth);
  }

  out->center[0] = clip[0] / clip[3];
  out->center[1] = clip[1] / clip[3];
  out->axis1 = packHalf2(axis1[0], axis1[1]);
  out->axis2 = packHalf2(axis2[0], axis2[1]);
  out->color0 = packHalf2(rgb[0], rgb[1]);
  out->color1 = packHalf2(rgb[2], alpha);
  out->radius = radius;
  out->index = index;
  *keyOut = key;
  return true;
}

// ---- LOD (metal/selection/SplatLOD.metal:26-43) --------------------------------------

bool lodOutside(const sko_camera& cam, const sko_cluster& node) {
  float v[4];
  mulPoint(cam.view, node.center[0], node.center[1], node.center[2], 1.0f, v);
  const float z = -v[2], r = node.radius;
  const float tx = cam.tanHalfFov[0], ty = cam.tanHalfFov[1];
  const float guard = (2.0f * fmx(z, 0.0f)) / fmx(fmn(cam.focal[0], cam.focal[1]), 1.0f);
  if (z + r <= 0.0f) return true;
  const bool outX = std::fabs(v[0]) - z * tx > r * std::sqrt(1.0f + tx * tx) + guard;
  const bool outY = std::fabs(v[1]) - z * ty > r * std::sqrt(1.0f + ty * ty) + guard;
  return outX || outY;
}

float lodErrorPixels(const sko_camera& cam, const sko_cluster& node, float colorWeight) {
  float v[4];
  mulPoint(cam.view, node.center[0], node.center[1], node.center[2], 1.0f, v);
  const float depth = fmx(-v[2] - node.radius, 1e-4f);
  const float perspective = std::sqrt(1.0f + (v[0] * v[0] + v[1] * v[1]) / (depth * depth));
  const float appearance = fmn(std::sqrt(node.colorVariance), 1.0f);
  const float error = node.error + node.radius * appearance;
  return ((((error * fmx(cam.focal[0], cam.focal[1])) / depth) * perspective) *
          fmx(node.opacity, 0.1f)) *
         (1.0f + colorWeight * std::sqrt(node.colorVariance));
}

constexpr uint32_t kLodSplit = 0x80000000u;
constexpr uint32_t kLodDrop = 0x40000000u;

// ---- composite ------------------------------------------------------------------------

// Per-splat values the coverage decision reads, computed in FP32 exactly as the kernel does.
struct Support {
  float cx, cy, m00, m01, m10, m11, radius, lcut;
  float a1x, a1y, a2x, a2y, alpha, rgb[3];
  bool any;
};

Support supportOf(const sko_projected& p, float width, float height) {
  Support s{};
  const float halfW = 0.5f * width, halfH = 0.5f * height;
  s.cx = (p.center[0] + 1.0f) * halfW;
  s.cy = (p.center[1] + 1.0f) * halfH;
  s.a1x = lowHalf(p.axis1), s.a1y = highHalf(p.axis1);
  s.a2x = lowHalf(p.axis2), s.a2y = highHalf(p.axis2);
  const float det = s.a1x * s.a2y - s.a2x * s.a1y;
  const float inv = 1.0f / det;
  s.m00 = s.a2y * inv;
  s.m01 = -(s.a2x * inv);
  s.m10 = -(s.a1y * inv);
  s.m11 = s.a1x * inv;
  s.radius = p.radius;
  s.alpha = highHalf(p.color1);
  s.lcut = lnF32(255.0f * s.alpha);
  s.rgb[0] = lowHalf(p.color0), s.rgb[1] = highHalf(p.color0), s.rgb[2] = lowHalf(p.color1);
  s.any = det != 0.0f && std::isfinite(inv) && std::isfinite(s.cx) && std::isfinite(s.cy);
  return s;
}

// The kernel's coverage test for pixel centre (px, py), y up. Writes q = (s^2 + t^2) / 2.
// Each fma rounds once; every other product and sum rounds on its own.
inline bool covers(const Support& s, float px, float py, float* q) {
  const float dx = px - s.cx, dy = py - s.cy;
  const float u = std::fma(s.m00, dx, s.m01 * dy);
  const float v = std::fma(s.m10, dx, s.m11 * dy);
  if (!(std::fabs(u) <= s.radius && std::fabs(v) <= s.radius)) return false;
  const float qq = 0.5f * std::fma(u, u, v * v);
  if (!(qq <= s.lcut)) return false;
  *q = qq;
  return true;
}

constexpr uint32_t kTile = 16;

// Splat lists per 16x16 tile, front to back, by a conservative pixel box.
std::vector<std::vector<uint32_t>> binTiles(const std::vector<Support>& sup, uint32_t width,
                                            uint32_t height) {
  const uint32_t tx = (width + kTile - 1) / kTile, ty = (height + kTile - 1) / kTile;
  std::vector<std::vector<uint32_t>> tiles(size_t{tx} * ty);
  for (uint32_t i = 0; i < sup.size(); ++i) {
    const Support& s = sup[i];
    if (!s.any) continue;
    const float ex = s.radius * (std::fabs(s.a1x) + std::fabs(s.a2x)) + 1.0f;
    const float ey = s.radius * (std::fabs(s.a1y) + std::fabs(s.a2y)) + 1.0f;
    // pixel columns whose centres lie in [cx - ex, cx + ex]; rows from y-up bounds.
    const double x0 = std::floor(double(s.cx) - ex), x1 = std::ceil(double(s.cx) + ex);
    const double yu0 = std::floor(double(s.cy) - ey), yu1 = std::ceil(double(s.cy) + ey);
    if (x1 < 0 || x0 >= width || yu1 < 0 || yu0 >= height) continue;
    const uint32_t c0 = static_cast<uint32_t>(std::max(0.0, x0));
    const uint32_t c1 = static_cast<uint32_t>(std::min(double(width - 1), x1));
    // y_up = H - row - 0.5 -> row = H - y_up - 0.5
    const double r0d = double(height) - yu1 - 1.0, r1d = double(height) - yu0;
    const uint32_t r0 = static_cast<uint32_t>(std::max(0.0, r0d));
    const uint32_t r1 = static_cast<uint32_t>(std::min(double(height - 1), std::max(0.0, r1d)));
    for (uint32_t ty0 = r0 / kTile; ty0 <= r1 / kTile; ++ty0)
      for (uint32_t tx0 = c0 / kTile; tx0 <= c1 / kTile; ++tx0) tiles[size_t{ty0} * tx + tx0].push_back(i);
  }
  return tiles;
}

}  // namespace

extern "C" {

float sko_ln(float x) { return lnF32(x); }
uint16_t sko_float_to_half(float x) { return floatToHalf(x); }
float sko_half_to_float(uint16_t h) { return halfToFloat(h); }

void sko_camera_make(const float* view16, const float* proj16, const float* cameraPosition3,
                     uint32_t width, uint32_t height, float minPixelRadius, sko_camera* out) {
  std::memset(out, 0, sizeof(*out));
  std::memcpy(out->view, view16, 64);
  std::memcpy(out->proj, proj16, 64);
  out->screenSize[0] = static_cast<float>(width);
  out->screenSize[1] = static_cast<float>(height);
  out->focal[0] = (out->screenSize[0] * proj16[0]) / 2.0f;
  out->focal[1] = (out->screenSize[1] * proj16[5]) / 2.0f;
  out->tanHalfFov[0] = 1.0f / proj16[0];
  out->tanHalfFov[1] = 1.0f / proj16[5];
  out->minPixelRadius = minPixelRadius;
  out->cameraPosition[0] = cameraPosition3[0];
  out->cameraPosition[1] = cameraPosition3[1];
  out->cameraPosition[2] = cameraPosition3[2];
  out->cameraPosition[3] = 1.0f;
  out->reveal[0] = std::numeric_limits<float>::infinity();
}

namespace {

float lowOf(uint32_t w) { return halfToFloat(static_cast<uint16_t>(w & 0xffffu)); }
float highOf(uint32_t w) { return halfToFloat(static_cast<uint16_t>(w >> 16)); }

// metal/cull/SplatVisibility.metal:69-84: a labelled part's tint, brightness and opacity on the
// packed colours; false when the opacity drops the splat. A label without a state, or a state
// without a palette entry, draws unstyled.
bool stylePart(const sko_parts& parts, uint32_t index, sko_projected& p) {
  const uint32_t label = parts.labels[index];
  if (label >= parts.stateCount) return true;
  const uint32_t state = parts.states[label];
  if (state >= 10) return true;
  const float* st = parts.palette + state * 8;  // tint[3], tintAmount, brightness, opacity
  if (!(st[3] != 0.0f || st[4] != 1.0f || st[5] != 1.0f)) return true;
  const float r = lowOf(p.color0), g = highOf(p.color0), b = lowOf(p.color1), a = highOf(p.color1);
  const float r2 = (r + (st[0] - r) * st[3]) * st[4];
  const float g2 = (g + (st[1] - g) * st[3]) * st[4];
  const float b2 = (b + (st[2] - b) * st[3]) * st[4];
  const float alpha = a * st[5];
  p.color0 = packHalf2(r2, g2);
  p.color1 = packHalf2(b2, alpha);
  return alpha >= kQuadMinAlpha;
}

// metal/layout/SplatProjection.metalh:177-189 for an encoded-space target (outputLinear 0).
void revealGlow(const sko_camera& cam, float height, sko_projected& p) {
  if (!(cam.reveal[1] > 0.0f)) return;
  float glow = std::fmin(std::fmax(1.0f - (cam.reveal[0] - height) / cam.reveal[1], 0.0f), 1.0f);
  glow = glow * glow;
  if (!(glow > 0.0f)) return;
  const float r = lowOf(p.color0), g = highOf(p.color0), b = lowOf(p.color1), a = highOf(p.color1);
  const float t = cam.reveal[2] * glow, boost = 1.0f + cam.reveal[3] * glow;
  const float r2 = (r + (cam.revealTint[0] - r) * t) * boost;
  const float g2 = (g + (cam.revealTint[1] - g) * t) * boost;
  const float b2 = (b + (cam.revealTint[2] - b) * t) * boost;
  p.color0 = packHalf2(r2, g2);
  p.color1 = packHalf2(b2, a);
}

}  // namespace

int sko_project_one(const sko_camera* cam, const sko_splat* splat, uint32_t index,
                    const uint32_t* sh, uint32_t shStride, int shDegree, int keyBits,
                    uint32_t* keyOut, sko_projected* out) {
  return projectOne(*cam, *splat, index, sh, shStride, shDegree, keyBits, keyOut, out) ? 1 : 0;
}

// metal/cull/SplatVisibility.metal:39-106 with the survivors kept in source order.
uint32_t sko_visibility(const sko_camera* cam, const sko_splat* splats, const uint32_t* sh,
                        uint32_t shStride, int shDegree, int keyBits, const sko_range* ranges,
                        uint32_t rangeCount, const uint32_t* indices, uint32_t indexCount,
                        uint32_t* keysOut, sko_projected* projectedOut, int threads,
                        const sko_parts* parts) {
  std::vector<uint32_t> sources;
  if (indices != nullptr) {
    sources.assign(indices, indices + indexCount);
  } else {
    for (uint32_t r = 0; r < rangeCount; ++r)
      for (uint32_t k = 0; k < ranges[r].count; ++k) sources.push_back(ranges[r].offset + k);
  }
  const size_t n = sources.size();
  threads = std::max(1, threads);
  std::vector<std::vector<uint32_t>> keys(threads);
  std::vector<std::vector<sko_projected>> proj(threads);
  parallelFor(n, threads, [&](size_t begin, size_t end, int t) {
    for (size_t i = begin; i < end; ++i) {
      uint32_t key;
      sko_projected p;
      const uint32_t index = sources[i];
      if (projectOne(*cam, splats[index], index, sh, shStride, shDegree, keyBits, &key, &p)) {
        if (parts && parts->labels && !stylePart(*parts, index, p)) continue;
        revealGlow(*cam, splats[index].position[1], p);
        keys[t].push_back(key);
        proj[t].push_back(p);
      }
    }
  });
  uint32_t count = 0;
  for (int t = 0; t < threads; ++t) {
    std::copy(keys[t].begin(), keys[t].end(), keysOut + count);
    std::copy(proj[t].begin(), proj[t].end(), projectedOut + count);
    count += static_cast<uint32_t>(keys[t].size());
  }
  return count;
}

void sko_stable_argsort(const uint32_t* keys, uint32_t n, uint32_t* orderOut) {
  for (uint32_t i = 0; i < n; ++i) orderOut[i] = i;
  std::stable_sort(orderOut, orderOut + n,
                   [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
}

void sko_radix_argsort(const uint32_t* keys, uint32_t n, int bits, uint32_t* orderOut,
                       int threads) {
  threads = std::max(1, threads);
  std::vector<uint32_t> k0(keys, keys + n), k1(n), v0(n), v1(n);
  for (uint32_t i = 0; i < n; ++i) v0[i] = i;
  const int passes = bits == 16 ? 2 : 4;
  std::vector<uint32_t> hist(static_cast<size_t>(threads) * 256);
  const size_t per = (n + threads - 1) / std::max(1, threads);
  for (int pass = 0; pass < passes; ++pass) {
    const uint32_t shift = pass * 8;
    std::fill(hist.begin(), hist.end(), 0u);
    parallelFor(n, threads, [&](size_t b, size_t e, int t) {
      uint32_t* h = &hist[static_cast<size_t>(t) * 256];
      for (size_t i = b; i < e; ++i) ++h[(k0[i] >> shift) & 0xffu];
    });
    // exclusive offsets, digit-major then thread: stable across chunks
    uint32_t run = 0;
    for (int d = 0; d < 256; ++d)
      for (int t = 0; t < threads; ++t) {
        const uint32_t c = hist[static_cast<size_t>(t) * 256 + d];
        hist[static_cast<size_t>(t) * 256 + d] = run;
        run += c;
      }
    parallelFor(n, threads, [&](size_t b, size_t e, int t) {
      (void)per;
      uint32_t* h = &hist[static_cast<size_t>(t) * 256];
      for (size_t i = b; i < e; ++i) {
        const uint32_t dst = h[(k0[i] >> shift) & 0xffu]++;
        k1[dst] = k0[i];
        v1[dst] = v0[i];
      }
    });
    k0.swap(k1);
    v0.swap(v1);
  }
  std::copy(v0.begin(), v0.end(), orderOut);
}

// metal/selection/SplatLOD.metal:44-220 and MetalLodSelection.mm:109-192, one round at a time.
uint32_t sko_lod_select(const sko_camera* cam, const sko_cluster* clusters, uint32_t clusterCount,
                        const uint32_t* leaves, uint32_t rounds, uint32_t capacity,
                        float pixelLimit, float colorWeight, uint32_t cull, uint32_t* indicesOut,
                        uint32_t* stats6) {
  (void)clusterCount;
  uint32_t count = 0, active = 1, packets = 0, accepted = 0, limited = 0, evaluated = 0;
  std::vector<uint32_t> frontier{0}, next;
  struct Packet {
    uint32_t leafStart, count, destination;
  };
  std::vector<Packet> packetList;
  std::vector<uint32_t> cost, flagsOf;
  std::vector<uint32_t> out(capacity, 0u);
  for (uint32_t level = 0; level < rounds; ++level) {
    // evaluate
    cost.assign(active, 0u);
    flagsOf.assign(active, 0u);
    uint32_t totalExtra = 0, drops = 0;
    for (uint32_t t = 0; t < active; ++t) {
      const sko_cluster& node = clusters[frontier[t]];
      uint32_t extra = 0, flags = 0;
      if (cull && lodOutside(*cam, node)) {
        flags = kLodDrop;
        ++drops;
      } else if (node.childCount + node.leafCount > 1 &&
                 (pixelLimit == 0.0f || lodErrorPixels(*cam, node, colorWeight) > pixelLimit)) {
        flags = kLodSplit;
        extra = node.childCount + node.leafCount - 1;
      } else if (node.childCount == 1 && node.leafCount == 0) {
        flags = kLodSplit;
      }
      cost[t] = extra;
      flagsOf[t] = flags;
      totalExtra += extra;
    }
    // budget (uint32 arithmetic as on the GPU)
    const uint32_t available = capacity - count - active + drops;
    if (totalExtra <= available) {
      accepted = totalExtra;
    } else {
      uint32_t run = 0, best = 0;
      for (uint32_t t = 0; t < active; ++t) {
        run += cost[t];
        if (run <= available) best = run; else break;
      }
      accepted = best;
    }
    // compact
    std::vector<uint32_t> kids(active), splats(active), pk(active), fl(active);
    uint32_t prefix = 0, denied = 0, sumKids = 0, sumSplats = 0, sumPackets = 0;
    for (uint32_t t = 0; t < active; ++t) {
      uint32_t flags = flagsOf[t];
      const uint32_t extra = cost[t];
      if ((flags & kLodSplit) && extra > 0 && prefix + extra > accepted) {
        flags = 0;
        ++denied;
      }
      prefix += extra;
      uint32_t k = 0, s = 0, p = 0;
      if (!(flags & kLodDrop)) {
        const sko_cluster& node = clusters[frontier[t]];
        k = (flags & kLodSplit) ? node.childCount : 0;
        s = (flags & kLodSplit) ? node.leafCount : 1;
        p = s > 32 ? 1 : 0;
      }
      kids[t] = sumKids, splats[t] = sumSplats, pk[t] = sumPackets, fl[t] = flags;
      sumKids += k, sumSplats += s, sumPackets += p;
    }
    // commit
    limited += denied;
    evaluated += active;
    const uint32_t scatterCount = count, scatterPackets = packets;
    count += sumSplats;
    packets += sumPackets;
    // scatter
    next.assign(sumKids, 0u);
    packetList.resize(packets);
    for (uint32_t t = 0; t < active; ++t) {
      if (fl[t] & kLodDrop) continue;
      const sko_cluster& node = clusters[frontier[t]];
      const bool split = (fl[t] & kLodSplit) != 0;
      if (split)
        for (uint32_t k = 0; k < node.childCount; ++k) next[kids[t] + k] = node.childStart + k;
      const uint32_t c = split ? node.leafCount : 1;
      const uint32_t destination = scatterCount + splats[t];
      if (c > 32) {
        packetList[scatterPackets + pk[t]] = {node.leafStart, c, destination};
      } else if (!split) {
        if (destination < capacity) out[destination] = node.node;
      } else {
        for (uint32_t k = 0; k < c; ++k)
          if (destination + k < capacity) out[destination + k] = leaves[node.leafStart + k];
      }
    }
    active = sumKids;
    frontier.swap(next);
  }
  for (const Packet& p : packetList)
    for (uint32_t k = 0; k < p.count; ++k)
      if (p.destination + k < capacity) out[p.destination + k] = leaves[p.leafStart + k];
  const uint32_t written = std::min(count, capacity);
  std::copy(out.begin(), out.begin() + written, indicesOut);
  if (stats6) {
    stats6[0] = count, stats6[1] = active, stats6[2] = packets;
    stats6[3] = accepted, stats6[4] = limited, stats6[5] = evaluated;
  }
  return written;
}

void sko_composite(const sko_projected* projected, const uint32_t* order, uint32_t count,
                   uint32_t width, uint32_t height, const float* background3, int opaque,
                   float transmittanceCutoff, int precision, float* rgbaOut, int threads) {
  std::vector<Support> sup(count);
  for (uint32_t i = 0; i < count; ++i)
    sup[i] = supportOf(projected[order[i]], static_cast<float>(width), static_cast<float>(height));
  const auto tiles = binTiles(sup, width, height);
  const uint32_t tilesX = (width + kTile - 1) / kTile;
  parallelFor(tiles.size(), threads, [&](size_t begin, size_t end, int) {
    for (size_t tileIndex = begin; tileIndex < end; ++tileIndex) {
      const auto& list = tiles[tileIndex];
      const uint32_t x0 = static_cast<uint32_t>(tileIndex % tilesX) * kTile;
      const uint32_t y0 = static_cast<uint32_t>(tileIndex / tilesX) * kTile;
      for (uint32_t row = y0; row < std::min(height, y0 + kTile); ++row)
        for (uint32_t col = x0; col < std::min(width, x0 + kTile); ++col) {
          const float px = static_cast<float>(col) + 0.5f;
          const float py = static_cast<float>(height - row) - 0.5f;
          double C[3] = {0, 0, 0}, T = 1.0;
          float Cf[3] = {0, 0, 0}, Tf = 1.0f;
          for (uint32_t i : list) {
            const Support& s = sup[i];
            float q;
            if (!covers(s, px, py, &q)) continue;
            if (precision == 64) {
              // FP64 evaluation of the same Gaussian from the same record values.
              const double dx = double(px) - (double(projected[order[i]].center[0]) + 1.0) * 0.5 * width;
              const double dy = double(py) - (double(projected[order[i]].center[1]) + 1.0) * 0.5 * height;
              const double det = double(s.a1x) * s.a2y - double(s.a2x) * s.a1y;
              const double u = (dx * s.a2y - double(s.a2x) * dy) / det;
              const double v = (double(s.a1x) * dy - dx * s.a1y) / det;
              const double g = double(s.alpha) * std::exp(-0.5 * (u * u + v * v));
              const double a = std::min(g, 1.0);
              for (int c = 0; c < 3; ++c) C[c] += T * a * s.rgb[c];
              T *= 1.0 - a;
              if (T < transmittanceCutoff) break;
            } else {
              const float g = s.alpha * std::exp(-q);
              const float a = fmn(g, 1.0f);
              for (int c = 0; c < 3; ++c) Cf[c] += Tf * a * s.rgb[c];
              Tf *= 1.0f - a;
              if (Tf < transmittanceCutoff) break;
            }
          }
          if (precision != 64) {
            for (int c = 0; c < 3; ++c) C[c] = Cf[c];
            T = Tf;
          }
          float* o = &rgbaOut[(size_t{row} * width + col) * 4];
          for (int c = 0; c < 3; ++c) {
            const double v = opaque ? C[c] + T * background3[c] : C[c];
            o[c] = static_cast<float>(std::min(1.0, std::max(0.0, v)));
          }
          o[3] = opaque ? 1.0f : static_cast<float>(std::min(1.0, std::max(0.0, 1.0 - T)));
        }
    }
  });
}

uint64_t sko_composite_fragments(const sko_projected* projected, const uint32_t* order,
                                 uint32_t count, uint32_t width, uint32_t height,
                                 float transmittanceCutoff, int threads) {
  std::vector<Support> sup(count);
  for (uint32_t i = 0; i < count; ++i)
    sup[i] = supportOf(projected[order[i]], static_cast<float>(width), static_cast<float>(height));
  const auto tiles = binTiles(sup, width, height);
  const uint32_t tilesX = (width + kTile - 1) / kTile;
  std::vector<uint64_t> perThread(std::max(1, threads), 0);
  parallelFor(tiles.size(), threads, [&](size_t begin, size_t end, int th) {
    uint64_t n = 0;
    for (size_t tileIndex = begin; tileIndex < end; ++tileIndex) {
      const uint32_t x0 = static_cast<uint32_t>(tileIndex % tilesX) * kTile;
      const uint32_t y0 = static_cast<uint32_t>(tileIndex / tilesX) * kTile;
      for (uint32_t row = y0; row < std::min(height, y0 + kTile); ++row)
        for (uint32_t col = x0; col < std::min(width, x0 + kTile); ++col) {
          const float px = static_cast<float>(col) + 0.5f;
          const float py = static_cast<float>(height - row) - 0.5f;
          float T = 1.0f;
          for (uint32_t i : tiles[tileIndex]) {
            float q;
            if (!covers(sup[i], px, py, &q)) continue;
            ++n;
            const float a = fmn(sup[i].alpha * std::exp(-q), 1.0f);
            T *= 1.0f - a;
            if (T < transmittanceCutoff) break;
          }
        }
    }
    perThread[th] += n;
  });
  uint64_t total = 0;
  for (uint64_t v : perThread) total += v;
  return total;
}

void sko_mt19937(uint32_t seed, uint32_t n, uint32_t* out) {
  std::mt19937 rng(seed);
  for (uint32_t i = 0; i < n; ++i) out[i] = static_cast<uint32_t>(rng());
}

}  // extern "C"
