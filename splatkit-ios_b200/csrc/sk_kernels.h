// Kernel launch interfaces (host side). Each launcher enqueues on `stream` and returns the
// launch status; none synchronises. Sizes that only the GPU knows (survivor count, instance
// count, LOD cut size) are passed as device pointers and every grid is sized by a host-known
// capacity, so a whole frame enqueues without a host round trip.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

#include "sk_layout.h"

namespace sk {

// ---- visibility (visibility.cu) --------------------------------------------------------
struct VisibilityArgs {
  const GpuSplat* splats;
  const uint32_t* sh;  // shStride words per splat
  uint32_t shStride;   // shDeviceStride(world degree); the frame may use fewer bands
  uint32_t worldCount;
  const Range* ranges;  // ranges mode (device), used when rangeCount > 1
  const uint32_t* rangeStarts;
  uint32_t rangeCount;
  Range single;  // the range itself when rangeCount == 1 (no device copy needed)
  const uint32_t* indices;     // indexed (LOD) mode
  const uint32_t* indexCount;  // indexed mode: entries in indices (device)
  uint32_t total;              // ranges mode: sum of counts; indexed mode: capacity bound
  uint32_t* keys;
  Projected* projected;
  uint4* spans;  // per survivor: the binning cells its quad touches (sk_tiles.cuh)
  uint32_t tilesX, tilesY;  // binning cells (kBinSize pixels) per row and column
  uint32_t* visibleCount;
  uint64_t* status;    // one word per 1024-splat tile
  uint32_t* counters;  // two words
  uint32_t epoch;
  uint32_t* error;
  PartLabels parts;  // labels.labels null: no part styling
  // the depth sort's digit histogram, summed over the survivors' keys as they are written (the
  // last block turns it into digit bases); sortPasses 0: not summed
  uint32_t* sortAccum;
  uint32_t* sortBases;
  uint32_t sortPasses;
};
uint32_t visibilityTileSplats();
// `cam` is a device pointer: the kernels stage it in shared memory, so a captured graph can be
// replayed with new cameras written into the same buffer.
cudaError_t launchVisibility(const Camera* cam, const VisibilityArgs& args, int shDegree,
                             bool key16, bool indexed, cudaStream_t stream);

// A batch of views (visibility.cu): one launch over every view's records, 16-bit depth keys with
// the view id above them, survivors of all views contiguous in (view, source) order.
struct BatchVisibilityArgs {
  const BatchView* views;   // viewCount entries
  const Camera* cameras;    // one per view (device)
  uint32_t viewCount;
  uint32_t items;           // work items: sum over views of max(1, ceil(count / 1024))
  uint32_t* keys;
  Projected* projected;
  uint4* spans;
  uint32_t* viewFirst;      // viewCount + 1 words: each view's first survivor, then the total
  uint32_t* visibleCount;
  uint64_t* status;         // one word per item
  uint32_t* counters;       // two words
  uint32_t epoch;
  uint32_t* error;
};
cudaError_t launchVisibilityBatch(const BatchVisibilityArgs& args, int shDegree,
                                  cudaStream_t stream);

// ---- radix sort (radix_sort.cu) --------------------------------------------------------
// Stable ascending sort of `count` (key, value) pairs with 8-bit digits: one histogram pass,
// then one onesweep scatter pass per digit. valuesIn null: values are the key positions.
// keysIn is left untouched; keysOut (optional) receives the sorted keys.
struct SortArgs {
  const uint32_t* keysIn;
  const uint32_t* valuesIn;
  uint32_t* keysOut;
  uint32_t* valuesOut;
  const uint32_t* count;  // device
  uint32_t capacity;      // count is clamped to this
  int bits;               // key bits: 8, 16, 24 or 32 (one 8-bit digit pass each)
  // workspace (sortWorkspaceBytes)
  uint32_t* keysA;
  uint32_t* keysB;
  uint32_t* valuesTmp;
  uint32_t* histogram;  // 2 * 4 * 256 words
  uint64_t* status;     // sortTiles(capacity) * 256 words
  uint32_t* counters;   // 2 * 5 words
  uint32_t epoch;       // uses epoch .. epoch + 3
  uint32_t* error;
  uint32_t tileKeys;    // keys per scatter tile: 2048, 4096 (0: the default) or 6144
  uint32_t statusTiles; // tiles the bound status region holds (set by the bind)
  // 1: the kernel that wrote the keys already summed their digits and left the bases in the
  // workspace (VisibilityArgs.sortPasses); the histogram pass is skipped
  uint32_t basesReady;
  // test hook (sk_testing_withhold_sort_status): tile + 1 of the first pass whose look-back
  // status words are not published; 0: none
  uint32_t withheldTilePlusOne;
};
// Where a bound workspace keeps the digit accumulators (zero between sorts) and the bases.
uint32_t* sortDigitAccumulators(const SortArgs& args);
uint32_t* sortDigitBases(const SortArgs& args);
uint32_t sortTileKeys();
size_t sortWorkspaceBytes(uint32_t capacity);
// Carves the workspace into the SortArgs fields.
void sortBindWorkspace(SortArgs& args, void* workspace, uint32_t capacity);
// The same for sorts that may use tiles as small as minTileKeys keys.
size_t sortWorkspaceBytesFor(uint32_t capacity, uint32_t minTileKeys);
void sortBindWorkspaceFor(SortArgs& args, void* workspace, uint32_t capacity, uint32_t minTileKeys);
cudaError_t launchSort(const SortArgs& args, cudaStream_t stream);
// Clears the counters and histogram accumulators of a bound workspace.
cudaError_t sortResetWorkspace(const SortArgs& args, cudaStream_t stream);

// ---- tile binning (binning.cu) ---------------------------------------------------------
struct BinArgs {
  const uint4* spans;     // per survivor tile spans, indexed like the projected records
  const uint32_t* order;  // depth order (indices into projected)
  const uint32_t* count;  // survivors (device)
  uint32_t capacity;      // bound on count
  uint32_t width, height, tilesX, tilesY;  // tilesX/Y: binning cells per row and column
  uint32_t* instanceKeys;    // binning cell per instance
  uint32_t* instanceValues;  // projected index per instance
  uint32_t instanceCapacity;
  uint32_t* instanceCount;  // FrameCounters.instances
  uint32_t* overflow;       // FrameCounters.overflow
  uint32_t* blockSums;      // binBlocks(capacity) words of scratch
  // a batch (viewCount > 0): tile ids are batch-wide, each view's from its table entry
  const BatchView* views;
  const uint32_t* viewFirst;  // viewCount + 1 words (BatchVisibilityArgs)
  uint32_t viewCount;
  // emission: 0 walks each warp's items one by one (best near one wave of blocks), 1 balances
  // each warp's output over its lanes (fewer instructions per instance; best for large grids)
  uint32_t balanced;
};
uint32_t binBlocks(uint32_t capacity);
cudaError_t launchBinning(const BinArgs& args, cudaStream_t stream);

// Per binning cell, the [start, end) range of its entries in the cell-sorted instance keys.
// ranges: one uint2 per cell, cleared beforehand by clearTileRanges (cells with no entry keep
// (0, 0)); the clear is issued early so the chained kernels of a frame run back to back.
cudaError_t clearTileRanges(uint2* ranges, uint32_t tiles, cudaStream_t stream);
cudaError_t launchTileRanges(const uint32_t* sortedKeys, const uint32_t* instanceCount,
                             uint32_t instanceCapacity, uint2* ranges, uint32_t tiles,
                             cudaStream_t stream);

// Direct cell-major lists (cell_lists.cu): the per-cell lists that binning + stable tile sort +
// ranges produce, written in place on targets of at most kDirectMaxCells binning cells. A count
// pass histograms every block of 512 depth ranks (1024 in a batch) by cell, a scan pass turns the histograms
// into each block's first position in every cell's list (and the lists' ranges, by look-back
// across groups of cells), and the emission pass writes each instance there in depth order.
// args.instanceValues receives the lists; instanceKeys and blockSums are unused.
constexpr uint32_t kDirectMaxCells = 4096;
struct CellLists {
  uint32_t cells;       // binning cells of the target (args.tilesX * args.tilesY)
  void* workspace;      // cellListBytes(capacity, cells), no clearing needed
  uint2* ranges;        // per cell [start, end), clamped to the instance capacity
  uint32_t* counters;   // two words, zero before the first launch (each launch restores them)
  uint32_t epoch;       // look-back epoch, fresh per launch
  uint32_t* error;      // SK_DEVERR_* bits
};
// Whether a target of `cells` cells takes the direct path.
bool cellListsFit(uint32_t capacity, uint32_t cells);
size_t cellListBytes(uint32_t capacity, uint32_t cells);
cudaError_t launchCellLists(const BinArgs& args, const CellLists& lists, cudaStream_t stream);

// Every view of a batch in one launch per pass. View v's ranks are [viewFirst[v], viewFirst[v+1])
// of args.order (at most `capacity` of them), its cells binBase .. binBase + cells of the batch's
// ranges; its count/emit blocks are blockBase .. blockBase + blocks (cellListBlocks(capacity)),
// its cell groups groupBase .. groupBase + (cells + 31) / 32, and its block rows the
// cellListRowBytes(capacity, cells) bytes at workspace + work. The look-back runs over the groups
// of all views in view order, so view v's entries follow those of views 0..v-1; args.instanceCount
// receives the total and args.overflow whether it exceeds args.instanceCapacity.
struct CellListView {
  uint32_t blockBase, groupBase, cells, tilesX;
  uint32_t binBase, capacity, blocks, pad;
  uint64_t work;
};
struct CellListBatch {
  const CellListView* views;  // device table, views in order
  uint32_t viewCount;
  const uint32_t* viewFirst;  // viewCount + 1 rank offsets (device)
  void* workspace;            // the views' block rows, no clearing needed
  uint64_t* status;           // one look-back word per cell group of the batch, zero beforehand
  uint2* ranges;              // the batch's cells
  uint32_t* counters;         // two words, zero before the first launch (each launch restores them)
  uint32_t epoch;
  uint32_t* error;
  uint32_t blocks, groups, mostCells;  // totals over the views; the largest view's cells
};
uint32_t cellListBlocks(uint32_t capacity);
size_t cellListRowBytes(uint32_t capacity, uint32_t cells);
cudaError_t launchCellListsBatch(const BinArgs& args, const CellListBatch& lists, cudaStream_t stream);
// Sets the emission kernel's shared-memory limit (once; before any stream capture).
cudaError_t cellListsConfigure();

// ---- composite (composite.cu) ----------------------------------------------------------
enum PixelFormat : int { kRgba8 = 0, kRgba32f = 1 };
struct CompositeArgs {
  const Projected* projected;
  const uint32_t* values;  // tile-sorted projected indices
  const uint2* ranges;  // per binning cell
  uint32_t width, height, tilesX, tilesY;  // composite tiles (kTileSize pixels)
  uint32_t binsX;                          // binning cells per row
  float background[3];
  int opaque;
  float cutoff;  // transmittance below which a pixel stops
  void* image;   // row 0 on top
  int format;
  uint32_t* fragments;  // FrameCounters.fragments_lo/hi (64-bit add), when countFragments
  uint32_t countFragments;
  uint32_t* loaded;     // FrameCounters.loaded
  // a batch (viewCount > 0): one block per batch-wide tile, image = the batch image
  const BatchView* views;
  uint32_t viewCount;
  uint32_t batchTiles;
};
cudaError_t launchComposite(const CompositeArgs& args, cudaStream_t stream);

// ---- LOD selection (lod.cu) ------------------------------------------------------------
struct LodArgs {
  const LodCluster* clusters;
  const uint32_t* leaves;
  uint32_t clusterCount;
  uint32_t capacity;  // indices buffer size and the guard's bound
  uint32_t limit;     // splats one selection may emit (<= capacity)
  float pixelLimit;
  float colorWeight;
  uint32_t cull;
  uint32_t rounds;
  uint32_t fanout;    // most child clusters of any cluster: round r's frontier holds at most
                      // fanout^r clusters (0: unknown)
  uint32_t frontierCapacity;
  uint32_t* frontier[2];
  uint2* costs;     // (extra | flags, exclusive prefix of extra)
  uint4* offsets;   // (kids, splats, packets exclusive, flags)
  uint4* packets;   // (leafStart, count, destination, 1)
  uint32_t* indices;
  LodState* state;
  uint64_t* status;  // 3 arrays of lodTiles(frontierCapacity) words
  uint32_t* counters;
  uint32_t epoch;  // uses epoch .. epoch + 2 * rounds
  uint32_t* error;
  uint32_t* report;  // six words copied from the state at the end (FrameCounters.lod)
};
uint32_t lodTileClusters();
cudaError_t launchLodSelect(const Camera* cam, const LodArgs& args, cudaStream_t stream);

// ---- LOD tree build (tree_build.cu) -----------------------------------------------------
// The octree of sk_build_lod_tree built on the device from host arrays; the nodes come back in
// the breadth-first layout (node 0 the root), childStart/childCount per node (0/0 for a leaf).
struct LodBuildInput {
  const float* positions;    // host, 3 per splat
  const float* covariances;  // 6
  const float* colors;       // 3
  const float* alphas;
  const float* sh;           // shStride per splat (nullptr when shStride is 0)
  uint32_t count;
  uint32_t shStride;
  float boundsMin[3];
  float extent;  // the largest side of the bounds (at least 1e-6)
  uint32_t depth;          // 1 .. 21
  uint32_t clusterLeaves;  // >= 2
};
// Host arrays that a resize leaves uninitialised (a default-initialising allocator): the arrays
// of a built tree are filled by a bulk copy or a parallel loop right after they are sized, so
// zeroing hundreds of MB on one thread first would only add time.
template <typename T>
struct UninitAllocator : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = UninitAllocator<U>;
  };
  UninitAllocator() = default;
  template <typename U>
  UninitAllocator(const UninitAllocator<U>&) noexcept {}
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U* p, Args&&... args) {
    ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
  }
};
template <typename T>
using HostArray = std::vector<T, UninitAllocator<T>>;

struct LodBuildOutput {
  uint32_t count = 0;
  HostArray<float> positions, covariances, colors, alphas, sh;
  HostArray<LodNode> layout;
};
constexpr uint32_t kMaxLodBuildLeaves = 0x7fffffffu;
cudaError_t buildLodTreeGpu(const LodBuildInput& in, LodBuildOutput& out);

}  // namespace sk
