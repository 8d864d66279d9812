// Batched multi-view rendering behind the sk_batch_* calls of include/splatkit_b200.h.
//
// One submission = a view table (world range, target size, where its items, tiles and pixels
// start in the batch-wide arrays) plus one camera per view. The stages are the frame
// pipeline's, each launched once over the whole batch:
//   visibility (all views, one look-back chain: survivors contiguous in (view, source) order,
//   key = view << 16 | 16-bit depth key) -> one stable radix sort of those keys (every view's
//   depth order, views back to back) -> binning with batch-wide tile ids -> stable tile sort ->
//   tile ranges -> composite of every tile of every view -> images, survivor counts and
//   counters copied to pinned memory.
// A view of a LOD world selects its cut first (on the lane's stream, with its context's current
// threshold) and its visibility items draw the cut instead of a range.
// The arithmetic per view is the plain frame's, so the images and counts equal sk_draw's.
#include "batch.h"

#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstring>
#include <mutex>
#include <memory>

namespace sk {

BatchLane::~BatchLane() {
  if (graph) cudaGraphExecDestroy(graph);
  if (done) cudaEventDestroy(done);
  if (start) cudaEventDestroy(start);
  if (end) cudaEventDestroy(end);
  if (stream) cudaStreamDestroy(stream);
}

void holdPooledMemory(int device) {
  static std::mutex m;
  static std::vector<bool> held;
  std::lock_guard<std::mutex> g(m);
  if (held.size() <= static_cast<size_t>(device)) held.resize(device + 1, false);
  if (held[device]) return;
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess)
      held[device] = true;
  }
  cudaGetLastError();
}

sk_status Batch::fail(sk_status code, const std::string& message) {
  error = message;
  return code;
}

sk_status Batch::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SK_OK;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return fail(SK_E_OOM, std::string(what) + ": out of device memory");
  }
  failed = true;
  return fail(SK_E_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}

uint32_t Batch::nextEpoch(uint32_t n) {
  const uint32_t e = epoch;
  epoch += n;
  if (epoch >= 0x3fff0000u) epoch = 1;
  return e;
}

namespace {
uint32_t bitsFor(uint64_t values) {  // key bits, a multiple of 8, for keys < values
  uint32_t b = 8;
  while (b < 32 && (uint64_t{1} << b) < values) b += 8;
  return b;
}
}  // namespace

sk_status Batch::reserve(BatchLane& l, uint32_t sources, uint32_t instances, uint32_t items,
                         uint32_t tiles, uint32_t views, uint64_t pixels) {
  // A buffer that must grow grows by at least half again: freeing the old one waits for the
  // whole device, so a lane should reach its working size in a few steps, not one per batch.
  auto grown32 = [](uint32_t need, uint32_t have) -> uint32_t {
    return need > have ? static_cast<uint32_t>(std::min<uint64_t>(
                             std::max<uint64_t>(need, uint64_t{have} + have / 2), 0x7fffffffu))
                       : need;
  };
  sources = grown32(std::max(sources, 1u), l.sources);
  instances = grown32(std::max(instances, 1u), l.instances);
  items = grown32(items, l.items);
  tiles = grown32(tiles, l.tiles);
  views = grown32(views, l.views);
  if (pixels > l.pixels) pixels = std::max(pixels, l.pixels + l.pixels / 2);
  cudaError_t e = cudaSuccess;
  auto grab = [&](DeviceBuffer& b, size_t n) {
    if (e == cudaSuccess) e = b.allocateOn(n, l.stream);
  };
  auto pin = [&](PinnedBuffer& b, size_t n) {
    if (e == cudaSuccess) e = b.allocate(n);
  };
  const bool grewSources = sources > l.sources, grewInstances = instances > l.instances;
  const bool grewItems = items > l.items;
  grab(l.keys, size_t{sources} * 4);
  grab(l.projected, size_t{sources} * sizeof(Projected));
  grab(l.spans, size_t{sources} * 16);
  grab(l.order, size_t{sources} * 4);
  grab(l.sortWorkspace, sortWorkspaceBytesFor(sources, kMinSortTileKeys));
  grab(l.binSums, size_t{binBlocks(sources)} * 4);
  grab(l.visStatus, size_t{std::max(items, 1u)} * 8);
  grab(l.instKeys, size_t{instances} * 4);
  grab(l.instValues, size_t{instances} * 4);
  grab(l.instKeysSorted, size_t{instances} * 4);
  grab(l.instValuesSorted, size_t{instances} * 4);
  grab(l.tileSortWorkspace, sortWorkspaceBytesFor(instances, kMinSortTileKeys));
  grab(l.ranges, size_t{std::max(tiles, 1u)} * sizeof(uint2));
  grab(l.viewFirst, size_t{views + 1} * 4);
  grab(l.viewTable, size_t{views} * sizeof(BatchView));
  grab(l.cameras, size_t{views} * sizeof(Camera));
  grab(l.image, pixels * 4);
  const bool freshCounters = l.counters.ptr == nullptr;
  grab(l.counters, 64 * 4);
  grab(l.frameCounters, sizeof(FrameCounters));
  pin(l.hostViews, size_t{views} * sizeof(BatchView));
  pin(l.hostCameras, size_t{views} * sizeof(Camera));
  pin(l.hostCounters, sizeof(FrameCounters));
  pin(l.hostViewFirst, size_t{views + 1} * 4);
  if (l.destinations.empty()) pin(l.hostImage, pixels * 4);  // else views go to the caller's buffers
  if (e == cudaSuccess && freshCounters) e = cudaMemsetAsync(l.counters.ptr, 0, 64 * 4, l.stream);
  // fresh sort workspaces: counters and histogram accumulators start at zero
  if (e == cudaSuccess && grewSources)
    e = cudaMemsetAsync(l.sortWorkspace.ptr, 0, l.sortWorkspace.bytes, l.stream);
  if (e == cudaSuccess && grewInstances)
    e = cudaMemsetAsync(l.tileSortWorkspace.ptr, 0, l.tileSortWorkspace.bytes, l.stream);
  // look-back status words of a fresh buffer must read "not ready"
  if (e == cudaSuccess && grewItems) e = cudaMemsetAsync(l.visStatus.ptr, 0, l.visStatus.bytes, l.stream);
  if (e != cudaSuccess) return check(e, "batch buffers");
  if (grewSources || grewInstances || items > l.items || tiles > l.tiles || views > l.views ||
      pixels > l.pixels) {
    // buffers moved: a captured graph points at the old ones
    if (l.graph) cudaGraphExecDestroy(l.graph);
    l.graph = nullptr;
    l.graphShape.clear();
  }
  l.sources = std::max(l.sources, sources);
  l.instances = std::max(l.instances, instances);
  l.items = std::max(l.items, items);
  l.tiles = std::max(l.tiles, tiles);
  l.views = std::max(l.views, views);
  l.pixels = std::max(l.pixels, pixels);
  return SK_OK;
}

sk_status Batch::reserveLod(BatchLane& l, uint32_t indices, uint32_t frontier, uint32_t views) {
  cudaError_t e = cudaSuccess;
  auto grab = [&](DeviceBuffer& b, size_t n) {
    if (e == cudaSuccess) e = b.allocateOn(n, l.stream);
  };
  frontier = std::max({frontier, l.lodFrontierCapacity, 1u});
  const uint32_t tiles = (frontier + lodTileClusters() - 1) / lodTileClusters();
  const void* before[3] = {l.lodStatus.ptr, l.lodCounters.ptr, l.lodState.ptr};
  grab(l.lodIndices, size_t{std::max(indices, 1u)} * 4);
  grab(l.lodReports, size_t{std::max(views, 1u)} * 8 * 4);
  grab(l.lodFrontier[0], size_t{frontier} * 4);
  grab(l.lodFrontier[1], size_t{frontier} * 4);
  grab(l.lodCosts, size_t{frontier} * 8);
  grab(l.lodOffsets, size_t{frontier} * 16);
  grab(l.lodPackets, size_t{frontier} * 16);
  grab(l.lodState, 256);
  grab(l.lodStatus, size_t{tiles} * 3 * 8);
  grab(l.lodCounters, 2 * 4);
  if (e == cudaSuccess) e = l.hostLodReports.allocate(size_t{std::max(views, 1u)} * 8 * 4);
  // fresh selection scratch: status words read "not ready", counters and state start at zero
  if (e == cudaSuccess && (before[0] != l.lodStatus.ptr || before[1] != l.lodCounters.ptr ||
                           before[2] != l.lodState.ptr)) {
    e = cudaMemsetAsync(l.lodStatus.ptr, 0, l.lodStatus.bytes, l.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(l.lodCounters.ptr, 0, l.lodCounters.bytes, l.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(l.lodState.ptr, 0, l.lodState.bytes, l.stream);
  }
  if (e != cudaSuccess) return check(e, "batch LOD buffers");
  l.lodFrontierCapacity = frontier;
  l.lodIndexCapacity = std::max(l.lodIndexCapacity, indices);
  l.lodReportViews = std::max(l.lodReportViews, views);
  return SK_OK;
}

sk_status Batch::prepare(BatchLane& l, const sk_batch_view* views, uint32_t count) {
  l.table.resize(count);
  l.cams.resize(count);
  l.worlds.resize(count);
  l.lodPlans.clear();
  uint32_t items = 0, tiles = 0, bins = 0, degree = 0, lodIndices = 0, lodFrontier = 0;
  uint64_t pixels = 0, sources = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const sk_batch_view& v = views[i];
    auto* ctx = reinterpret_cast<Context*>(v.world);
    if (!ctx || ctx->device != device) return fail(SK_E_INVALID, "a view has no context on this device");
    const World& w = ctx->world;
    if (!w.splats.ptr) return fail(SK_E_INVALID, "a view's context holds no world");
    if (v.width == 0 || v.height == 0 || v.width > 16384 || v.height > 16384)
      return fail(SK_E_INVALID, "view size out of range");
    uint32_t offset = 0, n = w.count;
    if (v.frame.range_count > 1) return fail(SK_E_INVALID, "a batch view draws at most one range");
    if (w.lod) {
      // the view draws the cut its selection writes: at most the world's cut capacity
      if (v.frame.range_count != 0) return fail(SK_E_INVALID, "a LOD view draws its cut, not a range");
      n = w.lodCapacity;
      LodPlan plan;
      plan.view = i;
      plan.clusters = static_cast<const LodCluster*>(w.clusters.ptr);
      plan.leaves = static_cast<const uint32_t*>(w.leaves.ptr);
      plan.clusterCount = w.clusterCount;
      plan.capacity = w.lodCapacity;
      plan.limit = ctx->lodLimit == 0 ? w.lodCapacity : std::min(ctx->lodLimit, w.lodCapacity);
      plan.rounds = w.rounds;
      plan.fanout = w.lodFanout;
      plan.pixelLimit = ctx->threshold.pixels();
      plan.indexOffset = lodIndices;
      if (uint64_t{lodIndices} + n > 0x7fffffffu) return fail(SK_E_INVALID, "batch too large");
      lodIndices += n;
      lodFrontier = std::max(lodFrontier, std::max(1u, std::min(w.lodCapacity, w.clusterCount)));
      l.lodPlans.push_back(plan);
    } else if (v.frame.range_count == 1) {
      if (!v.frame.ranges) return fail(SK_E_INVALID, "range missing");
      offset = v.frame.ranges[0].offset;
      n = v.frame.ranges[0].count;
      if (offset > w.count || n > w.count - offset) return fail(SK_E_INVALID, "invalid range");
    }
    const uint32_t d = static_cast<uint32_t>(std::max(0, std::min(v.frame.sh_degree, w.shDegree)));
    if (i == 0) degree = d;
    if (d != degree) return fail(SK_E_INVALID, "views of one batch draw one harmonics degree");
    BatchView& t = l.table[i];
    t = BatchView{};
    t.splats = static_cast<const GpuSplat*>(w.splats.ptr);
    t.sh = static_cast<const uint32_t*>(w.sh.ptr);
    t.shStride = shDeviceStride(w.shDegree);
    t.offset = offset;
    t.count = n;
    t.itemStart = items;
    t.tileBase = tiles;
    t.binBase = bins;
    t.width = v.width;
    t.height = v.height;
    t.tilesX = (v.width + kTileSize - 1) / kTileSize;
    const uint32_t tilesY = (v.height + kTileSize - 1) / kTileSize;
    t.binsX = (v.width + kBinSize - 1) / kBinSize;
    t.binsY = (v.height + kBinSize - 1) / kBinSize;
    t.pixelOffset = pixels;
    t.worldCount = w.count;
    const uint64_t chunks = std::max<uint64_t>(1, (uint64_t{n} + visibilityTileSplats() - 1) /
                                                      visibilityTileSplats());
    if (uint64_t{items} + chunks > 0x7fffffffu || uint64_t{tiles} + t.tilesX * tilesY > 0x7fffffffu ||
        sources + n > 0x7fffffffu)
      return fail(SK_E_INVALID, "batch too large");
    items += static_cast<uint32_t>(chunks);
    tiles += t.tilesX * tilesY;
    bins += t.binsX * t.binsY;
    pixels += uint64_t{v.width} * v.height;
    sources += n;
    l.cams[i] = cameraOf(v.frame, v.width, v.height, policy.subpixel_threshold);
    l.worlds[i] = w.splats.ptr;
  }
  l.viewCount = count;
  l.totalItems = items;
  l.totalTiles = tiles;
  l.totalBins = bins;
  l.totalPixels = pixels;
  l.shDegree = degree;
  const uint32_t guess = static_cast<uint32_t>(std::min<uint64_t>(
      std::max<uint64_t>(l.instances, sources * 4), 0x7fffffffu));
  sk_status st = reserve(l, static_cast<uint32_t>(sources), guess, items, tiles, count, pixels);
  if (st != SK_OK) return st;
  if (!l.lodPlans.empty()) {
    st = reserveLod(l, lodIndices, lodFrontier, static_cast<uint32_t>(l.lodPlans.size()));
    if (st != SK_OK) return st;
    for (size_t k = 0; k < l.lodPlans.size(); ++k) {
      BatchView& t = l.table[l.lodPlans[k].view];
      t.indices = static_cast<const uint32_t*>(l.lodIndices.ptr) + l.lodPlans[k].indexOffset;
      t.indexCount = static_cast<const uint32_t*>(l.lodReports.ptr) + k * 8;  // report word 0
    }
  }
  // Every view's lists written in place when each has at most kDirectMaxCells cells.
  uint32_t mostCells = 1;
  for (const BatchView& t : l.table) mostCells = std::max(mostCells, t.binsX * t.binsY);
  l.directLists = !tuning.sortedLists && mostCells <= kDirectMaxCells &&
                  cellListsConfigure() == cudaSuccess;
  if (l.directLists) {
    // view v's count/emit blocks, cell groups and block rows follow those of views 0..v-1
    CellListBatch& cb = l.cellBatch;
    cb = CellListBatch{};
    cb.viewCount = count;
    cb.mostCells = mostCells;
    std::vector<CellListView> cellViews(count);
    uint64_t rowBytes = 0;
    for (uint32_t v = 0; v < count; ++v) {
      const BatchView& t = l.table[v];
      CellListView& c = cellViews[v];
      c.capacity = std::max(t.count, 1u);
      c.cells = t.binsX * t.binsY;
      c.tilesX = t.binsX;
      c.binBase = t.binBase;
      c.blocks = cellListBlocks(c.capacity);
      c.blockBase = cb.blocks;
      c.groupBase = cb.groups;
      c.work = rowBytes;
      cb.blocks += c.blocks;
      cb.groups += (c.cells + 31) / 32;
      rowBytes += cellListRowBytes(c.capacity, c.cells);
    }
    void* before[3] = {l.cellLists.ptr, l.cellStatus.ptr, l.cellViews.ptr};
    cudaError_t e = l.cellLists.allocateOn(
        rowBytes > l.cellLists.bytes ? std::max<uint64_t>(rowBytes, l.cellLists.bytes + l.cellLists.bytes / 2)
                                     : rowBytes, l.stream);
    if (e == cudaSuccess) e = l.cellStatus.allocateOn(size_t{cb.groups} * 8, l.stream);
    if (e == cudaSuccess) e = l.cellViews.allocateOn(size_t{count} * sizeof(CellListView), l.stream);
    if (e == cudaSuccess) e = l.hostCellViews.allocate(size_t{count} * sizeof(CellListView));
    if (e != cudaSuccess) return check(e, "batch cell lists");
    std::memcpy(l.hostCellViews.ptr, cellViews.data(), size_t{count} * sizeof(CellListView));
    if (before[0] != l.cellLists.ptr || before[1] != l.cellStatus.ptr || before[2] != l.cellViews.ptr) {
      if (l.graph) cudaGraphExecDestroy(l.graph);  // a captured graph points at the old buffers
      l.graph = nullptr;
      l.graphShape.clear();
    }
  }
  std::memcpy(l.hostViews.ptr, l.table.data(), size_t{count} * sizeof(BatchView));
  std::memcpy(l.hostCameras.ptr, l.cams.data(), size_t{count} * sizeof(Camera));
  return SK_OK;
}

// The stages of one submission on the lane's stream. clearStatus: zero the look-back status
// words first (a replayed graph reuses the epochs it was captured with).
sk_status Batch::enqueueStages(BatchLane& l, bool clearStatus) {
  const cudaStream_t s = l.stream;
  FrameCounters* fc = static_cast<FrameCounters*>(l.frameCounters.ptr);
  uint32_t* error = &fc->error;
  uint32_t* counters = static_cast<uint32_t*>(l.counters.ptr);
  const auto* views = static_cast<const BatchView*>(l.viewTable.ptr);
  const auto* viewFirst = static_cast<const uint32_t*>(l.viewFirst.ptr);
  cudaError_t e = cudaMemsetAsync(fc, 0, sizeof(FrameCounters), s);
  if (e == cudaSuccess && !l.directLists)
    e = clearTileRanges(static_cast<uint2*>(l.ranges.ptr), l.totalBins, s);
  if (e == cudaSuccess && l.directLists) {
    // the look-back words of the batch's cell groups must read "not ready" (a replayed graph
    // reuses its epochs); the view table goes up with the other tables
    e = cudaMemsetAsync(l.cellStatus.ptr, 0, size_t{l.cellBatch.groups} * 8, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(l.cellViews.ptr, l.hostCellViews.ptr,
                          size_t{l.viewCount} * sizeof(CellListView), cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess && clearStatus) {
    e = cudaMemsetAsync(l.visStatus.ptr, 0, size_t{l.totalItems} * 8, s);
    SortArgs probe{};
    sortBindWorkspaceFor(probe, l.sortWorkspace.ptr, l.sources, kMinSortTileKeys);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(probe.status, 0, sortWorkspaceBytesFor(l.sources, kMinSortTileKeys) -
                          (reinterpret_cast<char*>(probe.status) - static_cast<char*>(l.sortWorkspace.ptr)), s);
    sortBindWorkspaceFor(probe, l.tileSortWorkspace.ptr, l.instances, kMinSortTileKeys);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(probe.status, 0, sortWorkspaceBytesFor(l.instances, kMinSortTileKeys) -
                          (reinterpret_cast<char*>(probe.status) - static_cast<char*>(l.tileSortWorkspace.ptr)), s);
  }
  // every LOD view's cut, one view after another in the lane's selection scratch
  for (size_t k = 0; e == cudaSuccess && k < l.lodPlans.size(); ++k) {
    const LodPlan& p = l.lodPlans[k];
    LodArgs a{};
    a.clusters = p.clusters;
    a.leaves = p.leaves;
    a.clusterCount = p.clusterCount;
    a.capacity = p.capacity;
    a.limit = p.limit;
    a.pixelLimit = p.pixelLimit;
    a.colorWeight = 4.0f;
    a.cull = policy.enable_frustum_culling ? 1u : 0u;
    a.rounds = p.rounds;
    a.fanout = p.fanout;
    a.frontierCapacity = l.lodFrontierCapacity;
    a.frontier[0] = static_cast<uint32_t*>(l.lodFrontier[0].ptr);
    a.frontier[1] = static_cast<uint32_t*>(l.lodFrontier[1].ptr);
    a.costs = static_cast<uint2*>(l.lodCosts.ptr);
    a.offsets = static_cast<uint4*>(l.lodOffsets.ptr);
    a.packets = static_cast<uint4*>(l.lodPackets.ptr);
    a.indices = static_cast<uint32_t*>(l.lodIndices.ptr) + p.indexOffset;
    a.state = static_cast<LodState*>(l.lodState.ptr);
    a.status = static_cast<uint64_t*>(l.lodStatus.ptr);
    a.counters = static_cast<uint32_t*>(l.lodCounters.ptr);
    a.epoch = nextEpoch(2 * p.rounds + 2);
    a.error = error;
    a.report = static_cast<uint32_t*>(l.lodReports.ptr) + k * 8;
    e = launchLodSelect(static_cast<const Camera*>(l.cameras.ptr) + p.view, a, s);
  }
  if (e == cudaSuccess) {
    BatchVisibilityArgs v{};
    v.views = views;
    v.cameras = static_cast<const Camera*>(l.cameras.ptr);
    v.viewCount = l.viewCount;
    v.items = l.totalItems;
    v.keys = static_cast<uint32_t*>(l.keys.ptr);
    v.projected = static_cast<Projected*>(l.projected.ptr);
    v.spans = static_cast<uint4*>(l.spans.ptr);
    v.viewFirst = static_cast<uint32_t*>(l.viewFirst.ptr);
    v.visibleCount = &fc->visible;
    v.status = static_cast<uint64_t*>(l.visStatus.ptr);
    v.counters = counters + 0;
    v.epoch = nextEpoch(1);
    v.error = error;
    e = launchVisibilityBatch(v, static_cast<int>(l.shDegree), s);
  }
  if (e == cudaSuccess) {
    // depth order of every view at once: the view id sits above the 16-bit key
    SortArgs a{};
    a.keysIn = static_cast<const uint32_t*>(l.keys.ptr);
    a.valuesOut = static_cast<uint32_t*>(l.order.ptr);
    a.count = &fc->visible;
    a.capacity = l.sources;
    a.bits = static_cast<int>(bitsFor(uint64_t{l.viewCount} << 16));
    sortBindWorkspaceFor(a, l.sortWorkspace.ptr, l.sources, kMinSortTileKeys);
    a.tileKeys = tuning.sortTileKeys;
    a.epoch = nextEpoch(4);
    a.error = error;
    e = launchSort(a, s);
  }
  if (e == cudaSuccess && l.directLists) {
    // every view's lists in one launch per pass: view v's ranks are order[viewFirst[v] ..
    // viewFirst[v + 1]) (views in order by the key's high bits), its cells binBase .. binBase +
    // binsX * binsY of the batch
    BinArgs b{};
    b.spans = static_cast<const uint4*>(l.spans.ptr);
    b.order = static_cast<const uint32_t*>(l.order.ptr);
    b.count = &fc->visible;
    b.capacity = l.sources;
    b.instanceValues = static_cast<uint32_t*>(l.instValuesSorted.ptr);
    b.instanceCapacity = l.instances;
    b.instanceCount = &fc->instances;
    b.overflow = &fc->overflow;
    CellListBatch cl = l.cellBatch;
    cl.views = static_cast<const CellListView*>(l.cellViews.ptr);
    cl.viewFirst = viewFirst;
    cl.workspace = l.cellLists.ptr;
    cl.status = static_cast<uint64_t*>(l.cellStatus.ptr);
    cl.ranges = static_cast<uint2*>(l.ranges.ptr);
    cl.counters = counters + 8;
    cl.epoch = nextEpoch(1);
    cl.error = error;
    e = launchCellListsBatch(b, cl, s);
  }
  if (e == cudaSuccess && !l.directLists) {
    BinArgs b{};
    b.spans = static_cast<const uint4*>(l.spans.ptr);
    b.order = static_cast<const uint32_t*>(l.order.ptr);
    b.count = &fc->visible;
    b.capacity = l.sources;
    b.instanceKeys = static_cast<uint32_t*>(l.instKeys.ptr);
    b.instanceValues = static_cast<uint32_t*>(l.instValues.ptr);
    b.instanceCapacity = l.instances;
    b.instanceCount = &fc->instances;
    b.overflow = &fc->overflow;
    b.blockSums = static_cast<uint32_t*>(l.binSums.ptr);
    b.views = views;
    b.viewFirst = viewFirst;
    b.viewCount = l.viewCount;
    b.balanced = tuning.balancedEmit ? 1u : 0u;
    e = launchBinning(b, s);
  }
  if (e == cudaSuccess && !l.directLists) {
    SortArgs a{};
    a.keysIn = static_cast<const uint32_t*>(l.instKeys.ptr);
    a.valuesIn = static_cast<const uint32_t*>(l.instValues.ptr);
    a.keysOut = static_cast<uint32_t*>(l.instKeysSorted.ptr);
    a.valuesOut = static_cast<uint32_t*>(l.instValuesSorted.ptr);
    a.count = &fc->instances;
    a.capacity = l.instances;
    a.bits = static_cast<int>(bitsFor(l.totalBins));
    sortBindWorkspaceFor(a, l.tileSortWorkspace.ptr, l.instances, kMinSortTileKeys);
    a.tileKeys = tuning.sortTileKeys;
    a.epoch = nextEpoch(4);
    a.error = error;
    e = launchSort(a, s);
  }
  if (e == cudaSuccess && !l.directLists)
    e = launchTileRanges(static_cast<const uint32_t*>(l.instKeysSorted.ptr), &fc->instances,
                         l.instances, static_cast<uint2*>(l.ranges.ptr), l.totalBins, s);
  if (e == cudaSuccess) {
    CompositeArgs c{};
    c.projected = static_cast<const Projected*>(l.projected.ptr);
    c.values = static_cast<const uint32_t*>(l.instValuesSorted.ptr);
    c.ranges = static_cast<const uint2*>(l.ranges.ptr);
    for (int j = 0; j < 3; ++j) c.background[j] = static_cast<float>(policy.background[j]);
    c.opaque = 1;
    c.cutoff = policy.enable_early_termination ? kTransmittanceCutoff : 0.0f;
    c.image = l.image.ptr;
    c.format = kRgba8;
    c.fragments = &fc->fragments_lo;
    c.countFragments = 1;
    c.loaded = &fc->loaded;
    c.views = views;
    c.viewCount = l.viewCount;
    c.batchTiles = l.totalTiles;
    e = launchComposite(c, s);
  }
  return check(e, "batch stages");
}

sk_status Batch::enqueue(BatchLane& l) {
  const cudaStream_t s = l.stream;
  // the shape a captured graph is valid for: every view's world, range and size
  std::vector<uint64_t> shape;
  // a LOD view's selection bakes its context's threshold into the launch: no graph replay
  const bool useGraph = tuning.graphs && l.lodPlans.empty();
  if (useGraph) {
    shape.reserve(size_t{l.viewCount} * 4 + 2);
    shape.push_back(l.viewCount);
    shape.push_back(l.shDegree);
    // the launch shapes it was captured with
    shape.push_back((uint64_t{tuning.sortTileKeys} << 2) | (tuning.balancedEmit ? 2u : 0u) |
                    (l.directLists ? 1u : 0u));
    for (uint32_t i = 0; i < l.viewCount; ++i) {
      const BatchView& t = l.table[i];
      shape.push_back(reinterpret_cast<uint64_t>(t.splats));
      shape.push_back((uint64_t{t.offset} << 32) | t.count);
      shape.push_back((uint64_t{t.width} << 32) | t.height);
      shape.push_back(t.shStride);
    }
  }
  cudaError_t e = cudaEventRecord(l.start, s);
  auto body = [&](bool clearStatus) -> sk_status {
    cudaError_t r = cudaMemcpyAsync(l.viewTable.ptr, l.hostViews.ptr,
                                    size_t{l.viewCount} * sizeof(BatchView), cudaMemcpyHostToDevice, s);
    if (r == cudaSuccess)
      r = cudaMemcpyAsync(l.cameras.ptr, l.hostCameras.ptr, size_t{l.viewCount} * sizeof(Camera),
                          cudaMemcpyHostToDevice, s);
    if (r != cudaSuccess) return check(r, "batch upload");
    sk_status st = enqueueStages(l, clearStatus);
    if (st != SK_OK) return st;
    r = cudaMemcpyAsync(l.hostCounters.ptr, l.frameCounters.ptr, sizeof(FrameCounters),
                        cudaMemcpyDeviceToHost, s);
    if (r == cudaSuccess)
      r = cudaMemcpyAsync(l.hostViewFirst.ptr, l.viewFirst.ptr, size_t{l.viewCount + 1} * 4,
                          cudaMemcpyDeviceToHost, s);
    if (r == cudaSuccess && !l.lodPlans.empty())
      r = cudaMemcpyAsync(l.hostLodReports.ptr, l.lodReports.ptr, l.lodPlans.size() * 8 * 4,
                          cudaMemcpyDeviceToHost, s);
    if (l.destinations.empty()) {
      if (r == cudaSuccess)
        r = cudaMemcpyAsync(l.hostImage.ptr, l.image.ptr, l.totalPixels * 4, cudaMemcpyDeviceToHost, s);
    } else {
      for (uint32_t i = 0; i < l.viewCount && r == cudaSuccess; ++i) {
        const BatchView& t = l.table[i];
        if (l.destinations[i])
          r = cudaMemcpyAsync(l.destinations[i], static_cast<const uint8_t*>(l.image.ptr) + t.pixelOffset * 4,
                              size_t{t.width} * t.height * 4, cudaMemcpyDeviceToHost, s);
      }
    }
    return check(r, "batch readback");
  };
  sk_status st = SK_OK;
  if (e != cudaSuccess) return check(e, "batch");
  if (useGraph) {
    if (!l.graph || l.graphShape != shape) {
      if (l.graph) cudaGraphExecDestroy(l.graph);
      l.graph = nullptr;
      cudaGraph_t g = nullptr;
      e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return check(e, "graph capture");
      st = body(true);
      const cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (st != SK_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
      }
      if (ce != cudaSuccess) return check(ce, "graph capture");
      e = cudaGraphInstantiate(&l.graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        l.graph = nullptr;
        return check(e, "graph instantiate");
      }
      l.graphShape = shape;
    }
    e = cudaGraphLaunch(l.graph, s);
    if (e != cudaSuccess) return check(e, "graph launch");
  } else {
    st = body(false);
    if (st != SK_OK) return st;
  }
  e = cudaEventRecord(l.end, s);
  if (e == cudaSuccess) e = cudaEventRecord(l.done, s);
  return check(e, "batch");
}

sk_status Batch::finish(BatchLane& l, bool wait) {
  if (!l.busy || l.harvested) return l.status;
  if (wait) {
    const cudaError_t e = cudaEventSynchronize(l.done);
    if (e != cudaSuccess) return l.status = check(e, "batch wait");
  } else if (cudaEventQuery(l.done) != cudaSuccess) {
    cudaGetLastError();  // cudaErrorNotReady is not an error
    return SK_OK;
  }
  FrameCounters c = *static_cast<const FrameCounters*>(l.hostCounters.ptr);
  if (c.overflow) {
    // Grow the instance buffers to what the batch needed and draw it again.
    const uint32_t need = static_cast<uint32_t>(std::min<uint64_t>(
        uint64_t{c.instances} + c.instances / 4 + 1024, 0x7fffffffu));
    sk_status st = reserve(l, l.sources, need, l.items, l.tiles, l.views, l.pixels);
    if (st == SK_OK) st = enqueue(l);
    if (st != SK_OK) {
      l.harvested = true;
      return l.status = st;
    }
    return finish(l, true);
  }
  l.result = c;
  l.harvested = true;
  cudaEventElapsedTime(&l.gpuMs, l.start, l.end);
  l.status = c.error ? fail(SK_E_TIMEOUT, "a bounded device wait or bounds check failed in the batch")
                     : SK_OK;
  return l.status;
}

BatchLane* Batch::laneOf(uint64_t ticket) {
  for (auto& l : lanes)
    if (l.busy && l.ticket == ticket) return &l;
  return nullptr;
}

}  // namespace sk

using sk::Batch;
using sk::BatchLane;

extern "C" {

sk_status sk_batch_create(const sk_batch_config* config, sk_batch** out) {
  if (!config || !out) return SK_E_INVALID;
  *out = nullptr;
  if (config->lanes == 0 || config->lanes > 16 || config->max_views == 0 || config->max_views > 65536)
    return SK_E_INVALID;
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || config->device < 0 || config->device >= devices) {
    cudaGetLastError();
    return SK_E_DEVICE;
  }
  if (cudaSetDevice(config->device) != cudaSuccess) return SK_E_DEVICE;
  auto b = std::make_unique<Batch>();
  b->device = config->device;
  b->tuning.lanes = config->lanes;
  b->tuning.maxViews = config->max_views;
  b->tuning.graphs = config->use_graphs != 0;
  b->tuning.activeLanes = config->lanes;
  sk_default_policy(&b->policy);
  b->lanes = std::vector<BatchLane>(config->lanes);
  for (auto& l : b->lanes) {
    if (cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&l.start) != cudaSuccess || cudaEventCreate(&l.end) != cudaSuccess)
      return SK_E_DEVICE;
  }
  sk::holdPooledMemory(config->device);
  *out = reinterpret_cast<sk_batch*>(b.release());
  return SK_OK;
}

void sk_batch_destroy(sk_batch* handle) {
  auto* b = reinterpret_cast<Batch*>(handle);
  if (!b) return;
  cudaSetDevice(b->device);
  for (auto& l : b->lanes)
    if (l.stream) cudaStreamSynchronize(l.stream);
  delete b;
}

const char* sk_batch_last_error(const sk_batch* handle) {
  const auto* b = reinterpret_cast<const Batch*>(handle);
  return b ? b->error.c_str() : "no batch";
}

#define SK_BATCH(handle)                              \
  auto* b = reinterpret_cast<Batch*>(handle);         \
  if (!b) return SK_E_INVALID;                        \
  if (b->failed) return SK_E_DEVICE;                  \
  cudaSetDevice(b->device)

sk_status sk_batch_apply_render_policy(sk_batch* handle, const sk_policy* p) {
  SK_BATCH(handle);
  if (!p) return SK_E_INVALID;
  const bool ok = std::isfinite(p->subpixel_threshold) && p->subpixel_threshold >= 0.0f &&
                  p->sort_depth_bits == 16 &&
                  std::all_of(p->background, p->background + 3,
                              [](double c) { return std::isfinite(c) && c >= 0 && c <= 1; });
  if (!ok) return b->fail(SK_E_INVALID, "batch policy out of range (16-bit depth keys only)");
  b->policy = *p;
  return SK_OK;
}

sk_status sk_batch_submit(sk_batch* handle, const sk_batch_view* views, uint32_t count,
                          uint64_t* ticket) {
  SK_BATCH(handle);
  if (!views || count == 0 || count > b->tuning.maxViews)
    return b->fail(SK_E_INVALID, "a submission holds 1 to max_views views");
  const uint32_t active = std::max(1u, std::min(b->tuning.activeLanes, static_cast<uint32_t>(b->lanes.size())));
  if (b->nextLane >= active) b->nextLane = 0;
  BatchLane& l = b->lanes[b->nextLane];
  b->nextLane = (b->nextLane + 1) % active;
  if (l.busy) {
    const sk_status st = b->finish(l, true);
    if (st == SK_E_DEVICE) return st;
  }
  l.busy = false;
  sk_status st = b->prepare(l, views, count);
  if (st != SK_OK) return st;
  st = b->enqueue(l);
  if (st != SK_OK) return st;
  l.busy = true;
  l.harvested = false;
  l.status = SK_OK;
  l.ticket = ++b->submitted;
  if (ticket) *ticket = l.ticket;
  return SK_OK;
}

sk_status sk_batch_poll(sk_batch* handle, uint64_t ticket, int32_t* done) {
  SK_BATCH(handle);
  BatchLane* l = b->laneOf(ticket);
  if (!l) return b->fail(SK_E_INVALID, "unknown ticket or its lane was reused");
  const sk_status st = b->finish(*l, false);
  if (done) *done = l->harvested ? 1 : 0;
  return st;
}

sk_status sk_batch_wait(sk_batch* handle, uint64_t ticket) {
  SK_BATCH(handle);
  BatchLane* l = b->laneOf(ticket);
  if (!l) return b->fail(SK_E_INVALID, "unknown ticket or its lane was reused");
  return b->finish(*l, true);
}

sk_status sk_batch_read_image(sk_batch* handle, uint64_t ticket, uint32_t view, void* host,
                              size_t bytes) {
  SK_BATCH(handle);
  BatchLane* l = b->laneOf(ticket);
  if (!l || !host) return b->fail(SK_E_INVALID, "unknown ticket or no buffer");
  const sk_status st = b->finish(*l, true);
  if (st != SK_OK) return st;
  if (view >= l->viewCount) return b->fail(SK_E_INVALID, "view out of range");
  const sk::BatchView& t = l->table[view];
  const size_t need = size_t{t.width} * t.height * 4;
  if (bytes < need) return b->fail(SK_E_INVALID, "image buffer too small");
  std::memcpy(host, static_cast<const uint8_t*>(l->hostImage.ptr) + t.pixelOffset * 4, need);
  return SK_OK;
}

sk_status sk_batch_view_visible(sk_batch* handle, uint64_t ticket, uint32_t view,
                                uint32_t* visible) {
  SK_BATCH(handle);
  BatchLane* l = b->laneOf(ticket);
  if (!l || !visible) return b->fail(SK_E_INVALID, "unknown ticket");
  const sk_status st = b->finish(*l, true);
  if (st != SK_OK) return st;
  if (view >= l->viewCount) return b->fail(SK_E_INVALID, "view out of range");
  const auto* first = static_cast<const uint32_t*>(l->hostViewFirst.ptr);
  *visible = first[view + 1] - first[view];
  return SK_OK;
}

sk_status sk_batch_get_stats(sk_batch* handle, uint64_t ticket, sk_batch_stats* out) {
  SK_BATCH(handle);
  BatchLane* l = b->laneOf(ticket);
  if (!l || !out) return b->fail(SK_E_INVALID, "unknown ticket");
  const sk_status st = b->finish(*l, true);
  if (st != SK_OK && st != SK_E_TIMEOUT) return st;
  out->views = l->viewCount;
  out->visible = l->result.visible;
  out->instances = l->result.instances;
  out->device_error = l->result.error;
  out->gpu_ms = l->gpuMs;
  out->fragments = uint64_t{l->result.fragments_lo} | (uint64_t{l->result.fragments_hi} << 32);
  return st;
}

}  // extern "C"

// ---- autotuner ---------------------------------------------------------------------------------
namespace {

// Draws the views once on lane l and waits; the lane is left idle.
sk_status runOnce(Batch& b, BatchLane& l, const sk_batch_view* views, uint32_t count) {
  if (l.busy) b.finish(l, true);
  l.busy = false;
  sk_status st = b.prepare(l, views, count);
  if (st == SK_OK) st = b.enqueue(l);
  if (st != SK_OK) return st;
  l.busy = true;
  l.harvested = false;
  l.ticket = 0;
  st = b.finish(l, true);
  l.busy = false;
  return st;
}

}  // namespace

extern "C" {

sk_status sk_batch_autotune(sk_batch* handle, const sk_batch_view* views, uint32_t count,
                            sk_batch_tuning* out) {
  SK_BATCH(handle);
  if (!views || count == 0 || count > b->tuning.maxViews || !out)
    return b->fail(SK_E_INVALID, "autotune needs 1 to max_views views");
  for (auto& l : b->lanes)
    if (l.busy) b->finish(l, true);
  for (auto& l : b->lanes) l.busy = false;
  const bool graphs = b->tuning.graphs;
  b->tuning.graphs = false;
  // 1. per cell-list construction, its kernel shapes timed on the device: emission strategy
  // (which only the sorted lists use) x radix tile size
  sk::BatchLane& lane = b->lanes[0];
  sk::BatchTuning shapes[2] = {b->tuning, b->tuning};
  double deviceMs[2] = {1e30, 1e30};
  for (int sorted = 0; sorted < 2; ++sorted) {
    for (const bool balanced : {false, true}) {
      if (!sorted && !balanced) continue;  // in-place lists emit no (cell, splat) pairs
      for (const uint32_t tileKeys : {2048u, 4096u, 6144u}) {
        b->tuning.sortedLists = sorted != 0;
        b->tuning.balancedEmit = balanced;
        b->tuning.sortTileKeys = tileKeys;
        double ms = 0;
        for (int rep = 0; rep < 3; ++rep) {  // the first run allocates and warms up
          const sk_status st = runOnce(*b, lane, views, count);
          if (st != SK_OK) {
            b->tuning.graphs = graphs;
            return st;
          }
          if (rep > 0) ms += lane.gpuMs;
        }
        if (ms < deviceMs[sorted]) {
          deviceMs[sorted] = ms;
          shapes[sorted] = b->tuning;
        }
      }
    }
  }
  // 2. per construction, 1..lanes submissions in flight, timed on the host with every image
  // copied back (the constructions load the device differently when lanes overlap)
  double bestRate = 0;
  uint32_t bestLanes = 1;
  sk::BatchTuning chosen = shapes[0];
  double best = deviceMs[0];
  for (int sorted = 0; sorted < 2; ++sorted) {
    b->tuning.sortedLists = shapes[sorted].sortedLists;
    b->tuning.balancedEmit = shapes[sorted].balancedEmit;
    b->tuning.sortTileKeys = shapes[sorted].sortTileKeys;
    for (uint32_t n = 1; n <= b->lanes.size(); ++n) {
      b->tuning.activeLanes = n;
      b->nextLane = 0;
      for (uint32_t k = 0; k < n; ++k) {  // every lane allocates and warms up untimed
        const sk_status st = runOnce(*b, b->lanes[k], views, count);
        if (st != SK_OK) {
          b->tuning.graphs = graphs;
          return st;
        }
      }
      const uint32_t rounds = 3 * n + 3;
      std::vector<uint64_t> tickets;
      const auto t0 = std::chrono::steady_clock::now();
      for (uint32_t k = 0; k < rounds; ++k) {
        uint64_t t = 0;
        const sk_status st = sk_batch_submit(handle, views, count, &t);
        if (st != SK_OK) {
          b->tuning.graphs = graphs;
          return st;
        }
        tickets.push_back(t);
      }
      for (uint32_t k = rounds - std::min(rounds, n); k < rounds; ++k) sk_batch_wait(handle, tickets[k]);
      const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      const double rate = rounds * count / s;
      if (rate > bestRate * 1.03) {  // more lanes, or the other construction, only when clearly faster
        bestRate = rate;
        bestLanes = n;
        chosen = shapes[sorted];
        best = deviceMs[sorted];
      }
    }
  }
  b->tuning.sortedLists = chosen.sortedLists;
  b->tuning.balancedEmit = chosen.balancedEmit;
  b->tuning.sortTileKeys = chosen.sortTileKeys;
  b->tuning.activeLanes = bestLanes;
  b->tuning.graphs = graphs;
  b->nextLane = 0;
  out->emission_balanced = chosen.balancedEmit ? 1u : 0u;
  out->sort_tile_keys = chosen.sortTileKeys;
  out->lanes = bestLanes;
  out->sorted_lists = chosen.sortedLists ? 1u : 0u;
  out->gpu_ms = best / 2.0;
  out->views_per_s = bestRate;
  return SK_OK;
}

sk_status sk_batch_set_tuning(sk_batch* handle, const sk_batch_tuning* t) {
  SK_BATCH(handle);
  if (!t || (t->sort_tile_keys != 2048 && t->sort_tile_keys != 4096 && t->sort_tile_keys != 6144) ||
      t->lanes == 0 || t->lanes > b->lanes.size())
    return b->fail(SK_E_INVALID, "tuning out of range");
  b->tuning.balancedEmit = t->emission_balanced != 0;
  b->tuning.sortTileKeys = t->sort_tile_keys;
  b->tuning.activeLanes = t->lanes;
  b->tuning.sortedLists = t->sorted_lists != 0;
  b->nextLane = 0;
  return SK_OK;
}

}  // extern "C"
