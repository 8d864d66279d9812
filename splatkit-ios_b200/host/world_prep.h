// Host-side world preparation: the GPU record packing and the LOD selection metadata the
// kernels read. Restated from the reference's engine/core C++ so a world packs to the same
// bytes:
//   packSplatRange / packShRange   splatkit-engine/src/rendering/GpuLayout.cpp:92-137
//   toHalf                         splat-core/include/splat/math/Half.h:12-38
//   buildLodSelectionData          splat-core/src/lod/LodSelection.cpp:47-133 (selection.cpp)
//   LOD depth (validateLodTree)    splat-core/src/lod/LodFile.cpp:103-141,336-344
//   LodThreshold                   splatkit-engine/include/splatkit/rendering/LodThreshold.h:12-43
//   gpuWorldBytes                  splatkit-engine/src/rendering/GpuLayout.cpp:14-20,72-77
#pragma once
#include <cstddef>
#include <cstdint>
#include <thread>
#include <string>
#include <vector>

#include "../csrc/sk_layout.h"

namespace sk::host {

struct CloudRef {
  const float* positions = nullptr;
  const float* covariances = nullptr;
  const float* colors = nullptr;
  const float* alphas = nullptr;
  const float* sh = nullptr;  // 3 * ((shDegree + 1)^2 - 1) floats per splat
  uint32_t count = 0;
  int shDegree = 0;
};

uint16_t floatToHalf(float v);
float halfToFloat(uint16_t h);

// Harmonics coefficients per channel, bands 1..degree.
// Runs fn(w, begin, end) over `workers` contiguous slices of [0, n) on host threads.
template <typename Fn>
void forSlices(size_t n, int workers, Fn fn) {
  if (workers <= 1) return fn(0, size_t{0}, n);
  std::vector<std::thread> pool;
  for (int w = 0; w < workers; ++w) pool.emplace_back(fn, w, n * w / workers, n * (w + 1) / workers);
  for (auto& t : pool) t.join();
}

inline uint32_t shCoefficients(int degree) {
  return degree <= 0 ? 0u : static_cast<uint32_t>((degree + 1) * (degree + 1) - 1);
}

// Splats [offset, offset + count) of `cloud` as 32-byte records.
void packSplats(const CloudRef& cloud, size_t offset, size_t count, GpuSplat* out, int threads);
// Harmonics bands 1..degree as halves, channel fastest, `stride` words per splat (the device
// stride; the words past the reference's packed stride are zero).
void packSh(const CloudRef& cloud, int degree, size_t offset, size_t count, uint32_t* out,
            uint32_t stride, int threads);

// The interior-cluster records and leaf references of a BFS-laid-out tree (selection.cpp). False,
// with both left empty, when the layout is not breadth first.
bool buildSelection(const CloudRef& nodes, const LodNode* layout, uint32_t nodeCount,
                    std::vector<LodCluster>& clusters, std::vector<uint32_t>& leaves);

// Checks the BFS topology and the leaf count; returns the deepest node depth (the number of
// refinement rounds is that plus one), or -1 with `error` set.
int64_t lodDepth(const LodNode* layout, uint32_t nodeCount, uint32_t leafCount, std::string* error);

// Adaptive screen-space error threshold (LodThreshold.h:12-43).
class LodThreshold {
 public:
  static constexpr float kMinPolicyPixels = 0.1f;
  static constexpr float kMaxPolicyPixels = 16.0f;
  static constexpr float kCeilingPixels = 64.0f;
  explicit LodThreshold(float policyPixels = 1.0f) { reset(policyPixels); }
  void reset(float policyPixels) {
    policy_ = policyPixels;
    pixels_ = policyPixels;
  }
  float update(uint32_t selected, uint32_t limited, uint32_t limit);
  float pixels() const { return pixels_; }
  float policyPixels() const { return policy_; }
  void restore(float pixels) { pixels_ = pixels; }

 private:
  float policy_ = 1.0f;
  float pixels_ = 1.0f;
};

// Device bytes a world of this shape takes, priced like gpuWorldBytes: records, per-draw
// scratch (projection, double-buffered sort key/value, selection index), selection data.
uint64_t worldBytes(uint64_t records, int shDegree, uint64_t drawCapacity, uint64_t clusters,
                    uint64_t leafRefs);

}  // namespace sk::host
