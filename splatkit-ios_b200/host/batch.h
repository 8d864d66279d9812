// Batched multi-view rendering: many views, of one or several resident worlds and of different
// target sizes, drawn by one pass of each stage over the whole batch (one launch per stage).
//
// Each lane is a CUDA stream with its own scratch; a submission goes to the next lane and runs
// while the host prepares the next one, so several batches overlap on the device. Results
// (images, survivor counts, counters) are copied back into the lane's pinned memory by the
// same stream, so they are on the host once the submission completes. A lane can capture its
// stage sequence as a CUDA graph and replay it while its views keep their worlds and sizes.
//
// A view of a LOD world first has its cut selected on the lane's stream (the selection kernels
// of csrc/lod.cu with the view's camera and its context's adaptive threshold, one view after
// another in the lane's own LOD scratch); the batch's visibility pass then draws each such view
// from its cut. The selection reports (cut length, limited) come back with the other results,
// for the caller to feed its threshold.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/splatkit_b200.h"
#include "../csrc/sk_kernels.h"
#include "context.h"

namespace sk {

inline constexpr uint32_t kMinSortTileKeys = 2048;  // lane sort workspaces fit every tile size

// Tunable launch parameters of a batch (the autotuner picks among them).
struct BatchTuning {
  uint32_t lanes = 2;           // lanes created
  uint32_t activeLanes = 2;     // lanes submissions rotate over (<= lanes)
  uint32_t maxViews = 64;       // views one submission may hold
  bool graphs = false;          // replay captured stage sequences
  bool balancedEmit = true;     // binning emission strategy (BinArgs::balanced)
  uint32_t sortTileKeys = 4096; // keys per radix scatter tile: 2048, 4096 or 6144
  bool sortedLists = false;     // cell lists by the batch-wide sort even where in place fits
};

// The selection one LOD view of a submission runs (LodArgs less the lane's scratch).
struct LodPlan {
  uint32_t view = 0;            // index in the submission
  const LodCluster* clusters = nullptr;
  const uint32_t* leaves = nullptr;
  uint32_t clusterCount = 0, capacity = 0, limit = 0, rounds = 0, fanout = 0;
  float pixelLimit = 1.0f;
  uint32_t indexOffset = 0;     // where its cut starts in the lane's index buffer
};

struct BatchLane {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr, start = nullptr, end = nullptr;
  // capacities
  uint32_t sources = 0, instances = 0, items = 0, tiles = 0, views = 0;
  uint64_t pixels = 0;
  // device
  DeviceBuffer keys, projected, spans, order, sortWorkspace, visStatus, binSums;
  DeviceBuffer instKeys, instValues, instKeysSorted, instValuesSorted, tileSortWorkspace;
  DeviceBuffer ranges, viewFirst, counters, frameCounters, viewTable, cameras, image;
  // direct cell lists (every view at most kDirectMaxCells cells), all views in one launch per
  // pass: every view's block rows, the look-back words of the batch's cell groups, the view
  // table (host copy in hostCellViews) and its totals
  DeviceBuffer cellLists, cellStatus, cellViews;
  bool directLists = false;
  CellListBatch cellBatch{};
  // LOD views: every view's cut, each view's six report words (LodState's first six), and the
  // selection scratch the views share in turn (sized for the largest)
  DeviceBuffer lodIndices, lodReports, lodFrontier[2], lodCosts, lodOffsets, lodPackets, lodState,
      lodStatus, lodCounters;
  uint32_t lodIndexCapacity = 0, lodFrontierCapacity = 0, lodReportViews = 0;
  std::vector<LodPlan> lodPlans;
  // pinned host
  PinnedBuffer hostViews, hostCameras, hostCounters, hostViewFirst, hostImage, hostLodReports,
      hostCellViews;
  // the submission it holds
  uint64_t ticket = 0;
  bool busy = false, harvested = true;
  sk_status status = SK_OK;
  std::vector<BatchView> table;          // host copy of the view table
  std::vector<Camera> cams;
  std::vector<const void*> worlds;       // per view: the world it draws (graph signature)
  std::vector<void*> destinations;       // per view: pinned host image to copy into (else hostImage)
  uint32_t viewCount = 0, totalItems = 0, totalTiles = 0, totalBins = 0, shDegree = 0;
  uint64_t totalPixels = 0;
  float gpuMs = 0;
  FrameCounters result{};
  // captured stage sequence and the shape it was captured for
  cudaGraphExec_t graph = nullptr;
  std::vector<uint64_t> graphShape;
  ~BatchLane();
};

// Lane buffers grow stream-ordered from the device's default memory pool, which from the first
// batch or server on keeps the memory lanes give back: later growth, in this or a later batch or
// server, reuses it instead of asking the driver (driver allocations took up to ~100 ms each
// on a B200 while other lanes ran, and each free waited for the whole device).
void holdPooledMemory(int device);

struct Batch {
  int device = 0;
  BatchTuning tuning;
  sk_policy policy{};
  std::vector<BatchLane> lanes;
  uint32_t nextLane = 0;
  uint64_t submitted = 0;
  uint32_t epoch = 1;
  std::string error;
  bool failed = false;

  sk_status fail(sk_status code, const std::string& message);
  sk_status check(cudaError_t e, const char* what);
  uint32_t nextEpoch(uint32_t n);
  sk_status reserve(BatchLane& lane, uint32_t sources, uint32_t instances, uint32_t items,
                    uint32_t tiles, uint32_t views, uint64_t pixels);
  // The LOD views' cuts (indices in total), reports and selection scratch (frontier entries).
  sk_status reserveLod(BatchLane& lane, uint32_t indices, uint32_t frontier, uint32_t views);
  // Fills the lane's view table and cameras from the request; no device work.
  sk_status prepare(BatchLane& lane, const sk_batch_view* views, uint32_t count);
  // Enqueues the lane's whole batch on its stream (uploads, stages, readbacks, done event).
  sk_status enqueue(BatchLane& lane);
  sk_status enqueueStages(BatchLane& lane, bool clearStatus);
  // Waits for (or polls) the lane's submission; grows and redraws on instance overflow.
  sk_status finish(BatchLane& lane, bool wait);
  BatchLane* laneOf(uint64_t ticket);
};

}  // namespace sk
