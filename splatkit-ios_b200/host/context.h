// The renderer context behind the C ABI: device buffers of the resident world and of one
// frame's scratch, the policy, the adaptive LOD threshold and the frame statistics.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "../../include/splatkit_b200.h"
#include "../csrc/sk_kernels.h"
#include "world_prep.h"

namespace sk {

inline constexpr uint32_t kMaxLodBudgetPublic = 4000000;  // MetalLodSelection.h:18
inline int hostThreadsPublic() {
  return static_cast<int>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
}

// Owning device allocation; allocate() only grows, and keeps the old memory when it fails.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      bytes = o.bytes;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DeviceBuffer() { release(); }
  cudaError_t allocate(size_t n);
  void release();
};

// A resident world: packed records, harmonics at the device stride, and for a hierarchy its
// selection data.
struct World {
  DeviceBuffer splats, sh;
  uint32_t count = 0;
  int shDegree = 0;
  bool lod = false;
  DeviceBuffer clusters, leaves;
  uint32_t clusterCount = 0, leafRefCount = 0, rounds = 0, lodCapacity = 0;
};

// Everything one frame writes. One per stream that renders concurrently.
struct FrameScratch {
  uint32_t sources = 0, instanceCapacity = 0, tilesX = 0, tilesY = 0;
  DeviceBuffer keys, projected, order, sortWorkspace, visStatus, binStatus;
  DeviceBuffer instKeys, instValues, instKeysSorted, instValuesSorted, tileSortWorkspace;
  DeviceBuffer ranges, image, rangeBuffer, rangeStarts, counters, frameCounters;
  DeviceBuffer lodIndices, lodFrontier[2], lodCosts, lodOffsets, lodPackets, lodState, lodStatus,
      lodCounters;
  uint32_t lodFrontierCapacity = 0;
  FrameCounters* hostCounters = nullptr;  // pinned
  cudaEvent_t events[6] = {};
  cudaEvent_t done = nullptr;
  FrameScratch() = default;
  FrameScratch(const FrameScratch&) = delete;
  FrameScratch& operator=(const FrameScratch&) = delete;
  ~FrameScratch() {
    if (hostCounters) cudaFreeHost(hostCounters);
    for (auto& e : events)
      if (e) cudaEventDestroy(e);
    if (done) cudaEventDestroy(done);
  }
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t width = 0, height = 0;
  int imageFormat = SK_FORMAT_RGBA8;
  bool timeStages = true;
  sk_policy policy{};
  uint32_t lodLimit = 0;
  host::LodThreshold threshold;
  World world;
  FrameScratch frame;
  bool frameInFlight = false;
  sk_frame lastFrame{};
  std::vector<sk_range> lastRanges;
  uint32_t lastTotal = 0;
  FrameCounters lastCounters{};
  sk_stats stats{};
  uint64_t submitted = 0, completed = 0;
  uint32_t epoch = 1;
  std::atomic<bool> failed{false};
  std::string error;

  ~Context() {
    if (stream) cudaStreamDestroy(stream);
  }

  sk_status fail(sk_status code, const std::string& message);
  sk_status check(cudaError_t e, const char* what);
  uint32_t nextEpoch(uint32_t n);
  sk_status reserveFrame(FrameScratch& f, uint32_t sources, uint32_t instances);
  sk_status reserveLod(FrameScratch& f, const World& w);
  Camera cameraFor(const sk_frame& frame) const;
  sk_status validateRanges(const sk_frame& frame, uint32_t* total) const;
  sk_status enqueueFrame(FrameScratch& f, const sk_frame& frame, uint32_t total, cudaStream_t s,
                         bool timed);
  sk_status finishFrame(bool wait);
  sk_status uploadCloud(const sk_cloud_view& cloud, int maxSh, World& w);
};

}  // namespace sk
