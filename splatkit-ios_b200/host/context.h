// The renderer context behind the C ABI: device buffers of the resident world, the reusable
// scratch of one frame pipeline, the per-view outputs, the policy, the adaptive LOD threshold
// and the frame statistics.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <deque>
#include <string>
#include <thread>
#include <vector>

#include "../../include/splatkit_b200.h"
#include "../csrc/sk_kernels.h"
#include "world_prep.h"

namespace sk {

inline constexpr uint32_t kMaxLodBudgetPublic = 4000000;  // MetalLodSelection.h:18
inline constexpr uint32_t kMaxRanges = 65536;             // MetalVisibilityPass.h:72
inline constexpr float kTransmittanceCutoff = 1e-4f;
// Scatter tile size of the plain frame's tile sort (measured: 4096 beats 2048 at 4.5M pairs).
inline constexpr uint32_t kTileSortTileKeys = 4096;
inline int hostThreadsPublic() {
  return static_cast<int>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
}

// Test hook (sk_testing_fail_device_allocations): how many of the next device allocations fail.
extern std::atomic<uint32_t> gTestFailedAllocations;

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
  // Stream-ordered growth on stream s (the only stream that uses the buffer): the new memory
  // comes from the device's memory pool and the old goes back to it after s's earlier work,
  // so growing neither waits for the device nor, once the pool holds the memory, for the driver.
  cudaError_t allocateOn(size_t n, cudaStream_t s);
  void release();
};

// Owning pinned host allocation.
struct PinnedBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  PinnedBuffer() = default;
  PinnedBuffer(const PinnedBuffer&) = delete;
  PinnedBuffer& operator=(const PinnedBuffer&) = delete;
  ~PinnedBuffer() { release(); }
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
  uint32_t lodFanout = 0;  // most child clusters of any cluster
};

// Everything one pipeline run writes besides its outputs; reused frame after frame on one
// stream. One per stream that renders concurrently.
struct FrameScratch {
  uint32_t sources = 0, instanceCapacity = 0, maxTiles = 0;
  DeviceBuffer keys, projected, spans, order, sortWorkspace, visStatus, binSums;
  DeviceBuffer instKeys, instValues, instKeysSorted, instValuesSorted, tileSortWorkspace;
  DeviceBuffer ranges, rangeBuffer, rangeStarts, counters;
  DeviceBuffer cellLists;  // direct cell-major lists: block x cell counts and starts
  DeviceBuffer lodIndices, lodFrontier[2], lodCosts, lodOffsets, lodPackets, lodState, lodStatus,
      lodCounters;
  uint32_t lodFrontierCapacity = 0;
  FrameScratch() = default;
  FrameScratch(const FrameScratch&) = delete;
  FrameScratch& operator=(const FrameScratch&) = delete;
};

// Where one view's results go.
struct ViewTarget {
  uint32_t width = 0, height = 0;
  void* image = nullptr;                   // device, the context's pixel format
  FrameCounters* counters = nullptr;       // device
  FrameCounters* hostCounters = nullptr;   // pinned; null: no readback
  const Camera* camera = nullptr;          // device, written before the pipeline runs
  uint32_t tilesX() const { return (width + kTileSize - 1) / kTileSize; }
  uint32_t tilesY() const { return (height + kTileSize - 1) / kTileSize; }
  uint32_t binsX() const { return (width + kBinSize - 1) / kBinSize; }
  uint32_t binsY() const { return (height + kBinSize - 1) / kBinSize; }
};

// The per-view camera block of a frame on a width x height target.
Camera cameraOf(const sk_frame& frame, uint32_t width, uint32_t height, float minPixelRadius);

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t width = 0, height = 0;
  int imageFormat = SK_FORMAT_RGBA8;
  uint32_t timeStages = 1;  // 0 none, 1 per stage, 2 frame only
  uint32_t binningMode = SK_BINNING_AUTO;
  sk_policy policy{};
  uint32_t lodLimit = 0;
  host::LodThreshold threshold;
  World world;
  // part labels of the flat world (cleared with it) and the styles they are drawn with
  DeviceBuffer labels, stylePalette, styleStateTable;
  uint32_t styleStateCount = 0;
  FrameScratch scratch;
  // the plain renderer's own view: image, counters, camera
  DeviceBuffer image, frameCounters, camera;
  // Frame slots: like the reference's frame loop (MetalFrameSlots.h:8) a flat world keeps two
  // frames in flight, so the host enqueues the next frame while the GPU draws the last; a
  // slot holds what finishing (or drawing again) its frame needs. LOD worlds keep one, so the
  // adaptive threshold sees every frame's cut before the next selection. Slot 1 draws on its
  // own stream with its own scratch, counters, camera and image (set up the first time two
  // frames are in flight), so the two frames' kernels run side by side on the device.
  static constexpr uint32_t kFrameSlots = 2;
  cudaStream_t stream2 = nullptr;
  FrameScratch scratch2;
  DeviceBuffer frameCounters2, camera2;
  uint32_t lastSlot = 0;  // slot of the last finished frame (whose scratch the read-backs copy)
  FrameScratch& scratchOf(uint32_t slot) { return slot ? scratch2 : scratch; }
  cudaStream_t streamOf(uint32_t slot) const { return slot ? stream2 : stream; }
  // Slot 1's stream, scratch (as large as slot 0's) and view buffers, and a second image.
  sk_status prepareSecondSlot();
  // Waits for everything enqueued on the frame streams.
  cudaError_t syncStreams();
  struct Slot {
    PinnedBuffer hostCounters, hostCamera;
    cudaEvent_t done = nullptr;
    cudaEvent_t events[6] = {};
    sk_frame frame{};
    std::vector<sk_range> ranges;
    uint32_t total = 0, image = 0;
    uint64_t number = 0;  // the submitted-frame count it was drawn as
  };
  Slot slots[kFrameSlots];
  std::deque<uint32_t> inFlight;  // slots of the frames in flight, oldest first
  // Frame captures (captureNextFrame): once one is requested the frames alternate between two
  // images, so the copy of one frame's image to the host (on copyStream) overlaps the drawing of
  // the next; a frame waits for the copy that still reads its image before it draws.
  struct Capture {
    uint64_t ticket = 0, frame = 0;  // the frame: the submitted-frame count it was drawn as
    void* host = nullptr;
    size_t bytes = 0;
    cudaEvent_t copied = nullptr;
    bool issued = false, tooSmall = false;  // tooSmall: the target grew past the buffer
  };
  DeviceBuffer image2;
  bool twoImages = false;
  uint32_t imageSlot = 0;  // image of the frame in flight or last drawn
  cudaStream_t copyStream = nullptr;
  cudaEvent_t imageFree[2] = {};
  bool imageCopied[2] = {};
  std::deque<Capture> captures;  // requested, in flight or landed but not waited for
  uint64_t nextCapture = 1;
  void* imageOf(uint32_t slot) { return slot ? image2.ptr : image.ptr; }
  size_t imageBytes() const;
  sk_status issueCapture(Capture& c, const Slot& slot);
  FrameCounters lastCounters{};
  sk_stats stats{};
  uint64_t submitted = 0, completed = 0;
  uint32_t epoch = 1;
  std::atomic<bool> failed{false};
  std::string error;
  // test hooks (include/splatkit_b200_testing.h), each used once: the depth-sort tile of the next
  // frame that withholds its status words (tile + 1; 0: none), and the CUDA status the next
  // check() reads instead of its own
  uint32_t testWithheldTile = 0;
  cudaError_t testInjectedError = cudaSuccess;

  ~Context();

  sk_status fail(sk_status code, const std::string& message);
  sk_status check(cudaError_t e, const char* what);
  uint32_t nextEpoch(uint32_t n);
  // Scratch for `sources` splats, `instances` tile instances and targets up to maxTiles tiles.
  sk_status reserveScratch(FrameScratch& f, uint32_t sources, uint32_t instances, uint32_t maxTiles,
                           cudaStream_t s);
  sk_status reserveLod(FrameScratch& f, const World& w, cudaStream_t s);
  sk_status reserveView(uint32_t width, uint32_t height);
  Camera cameraFor(const sk_frame& frame, uint32_t width, uint32_t height) const;
  sk_status validateRanges(const sk_frame& frame, uint32_t* total) const;
  // The whole frame pipeline for one view on stream s; nothing waits on the host.
  sk_status enqueuePipeline(FrameScratch& f, const ViewTarget& v, const sk_frame& frame,
                            uint32_t total, cudaStream_t s, uint32_t timing, cudaEvent_t* events);
  ViewTarget plainView(const Slot& slot);
  sk_status enqueueSlot(uint32_t slot);
  // Finishes the oldest frame in flight (waiting for it); grows the list buffers and draws
  // every frame in flight again when one overflowed.
  sk_status finishOldest();
  // Finishes every frame in flight (with wait false, only those already complete); reports the
  // first error but always drains what it waits for.
  sk_status finishFrame(bool wait);
  // Finishes the frames in flight up to frame `number`.
  sk_status finishThrough(uint64_t number);
  sk_status uploadCloud(const sk_cloud_view& cloud, int maxSh, World& w);
  uint32_t instanceGuess(uint32_t sources) const;
};

}  // namespace sk
