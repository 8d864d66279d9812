// The C ABI of include/splatkit_b200.h: a headless renderer context that mirrors
// splatkit::SplatRenderer (packages/splatkit-engine/include/splatkit/rendering/SplatRenderer.h)
// and the Metal renderer's frame (splatkit-ios/.../metal/MetalSplatRenderer.mm:166-308).
//
// A frame is enqueued on the context's stream without a host round trip:
//   [LOD cut] -> visibility (cull, project, SH, depth key, tile span, source-order compaction)
//   -> depth sort (onesweep radix, 16- or 32-bit keys) -> tile binning -> stable tile sort
//   -> tile ranges -> composite, then a 64-byte counter block is copied back asynchronously.
// Every grid is sized by a host-known capacity; live counts stay on the device.
#include "context.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "world_prep.h"

namespace sk {

// ---- buffers ------------------------------------------------------------------------------

std::atomic<uint32_t> gTestFailedAllocations{0};

cudaError_t DeviceBuffer::allocate(size_t n) {
  n = std::max<size_t>(n, 256);
  if (n <= bytes && ptr) return cudaSuccess;
  // test hook (sk_testing_fail_device_allocations): this allocation fails as if out of memory
  for (uint32_t left = gTestFailedAllocations.load(); left > 0;)
    if (gTestFailedAllocations.compare_exchange_weak(left, left - 1)) return cudaErrorMemoryAllocation;
  void* fresh = nullptr;
  const cudaError_t e = cudaMalloc(&fresh, n);
  if (e != cudaSuccess) {
    cudaGetLastError();  // an allocation failure is not a sticky error
    return e;
  }
  release();
  ptr = fresh;
  bytes = n;
  return cudaSuccess;
}

cudaError_t DeviceBuffer::allocateOn(size_t n, cudaStream_t s) {
  n = std::max<size_t>(n, 256);
  if (n <= bytes && ptr) return cudaSuccess;
  for (uint32_t left = gTestFailedAllocations.load(); left > 0;)
    if (gTestFailedAllocations.compare_exchange_weak(left, left - 1)) return cudaErrorMemoryAllocation;
  void* fresh = nullptr;
  const cudaError_t e = cudaMallocAsync(&fresh, n, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e;
  }
  if (ptr) cudaFreeAsync(ptr, s);
  ptr = fresh;
  bytes = n;
  return cudaSuccess;
}

void DeviceBuffer::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

cudaError_t PinnedBuffer::allocate(size_t n) {
  n = std::max<size_t>(n, 64);
  if (n <= bytes && ptr) return cudaSuccess;
  void* fresh = nullptr;
  const cudaError_t e = cudaMallocHost(&fresh, n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e;
  }
  release();
  ptr = fresh;
  bytes = n;
  std::memset(ptr, 0, n);
  return cudaSuccess;
}

void PinnedBuffer::release() {
  if (ptr) cudaFreeHost(ptr);
  ptr = nullptr;
  bytes = 0;
}

// ---- context ------------------------------------------------------------------------------

Context::~Context() {
  if (copyStream) cudaStreamSynchronize(copyStream);
  for (auto& c : captures)
    if (c.copied) cudaEventDestroy(c.copied);
  for (auto& e : imageFree)
    if (e) cudaEventDestroy(e);
  if (copyStream) cudaStreamDestroy(copyStream);
  for (auto& sl : slots) {
    if (sl.done) cudaEventDestroy(sl.done);
    for (auto& ev : sl.events)
      if (ev) cudaEventDestroy(ev);
  }
  if (stream) cudaStreamDestroy(stream);
  if (stream2) cudaStreamDestroy(stream2);
}

sk_status Context::fail(sk_status code, const std::string& message) {
  error = message;
  return code;
}

sk_status Context::check(cudaError_t e, const char* what) {
  if (testInjectedError != cudaSuccess) {  // test hook: a stand-in for a failing call
    e = testInjectedError;
    testInjectedError = cudaSuccess;
  }
  if (e == cudaSuccess) return SK_OK;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return fail(SK_E_OOM, std::string(what) + ": out of device memory");
  }
  failed.store(true);
  return fail(SK_E_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}

uint32_t Context::nextEpoch(uint32_t n) {
  const uint32_t e = epoch;
  epoch += n;
  if (epoch >= 0x3fff0000u) epoch = 1;  // status words of old epochs never match a new one
  return e;
}

uint32_t Context::instanceGuess(uint32_t sources) const {
  return static_cast<uint32_t>(std::min<uint64_t>(uint64_t{std::max(sources, 1u)} * 8, 0x7fffffffu));
}

sk_status Context::reserveScratch(FrameScratch& f, uint32_t sources, uint32_t instances,
                                  uint32_t maxTiles, cudaStream_t s) {
  sources = std::max(sources, 1u);
  instances = std::max(instances, 1u);
  maxTiles = std::max(maxTiles, 1u);
  cudaError_t e = cudaSuccess;
  auto grab = [&](DeviceBuffer& b, size_t n) {
    if (e == cudaSuccess) e = b.allocate(n);
  };
  const uint32_t visTiles = (sources + visibilityTileSplats() - 1) / visibilityTileSplats();
  grab(f.keys, size_t{sources} * 4);
  grab(f.projected, size_t{sources} * sizeof(Projected));
  grab(f.spans, size_t{sources} * 16);
  grab(f.order, size_t{sources} * 4);
  grab(f.sortWorkspace, sortWorkspaceBytes(sources));
  grab(f.visStatus, size_t{visTiles} * 8);
  grab(f.binSums, size_t{binBlocks(sources)} * 4);
  grab(f.instKeys, size_t{instances} * 4);
  grab(f.instValues, size_t{instances} * 4);
  grab(f.instKeysSorted, size_t{instances} * 4);
  grab(f.instValuesSorted, size_t{instances} * 4);
  grab(f.tileSortWorkspace, sortWorkspaceBytesFor(instances, kTileSortTileKeys));
  grab(f.ranges, size_t{maxTiles} * sizeof(uint2));
  grab(f.cellLists, cellListBytes(sources, std::min(std::max(maxTiles, f.maxTiles), kDirectMaxCells)));
  grab(f.rangeBuffer, size_t{kMaxRanges} * sizeof(Range));
  grab(f.rangeStarts, size_t{kMaxRanges + 1} * 4);
  const bool fresh = f.counters.ptr == nullptr;
  grab(f.counters, 64 * 4);
  if (e == cudaSuccess && fresh) e = cudaMemsetAsync(f.counters.ptr, 0, 64 * 4, s);
  // Sort workspaces hold counters that must start at zero; status words carry epochs.
  if (e == cudaSuccess) e = cudaMemsetAsync(f.sortWorkspace.ptr, 0, f.sortWorkspace.bytes, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(f.tileSortWorkspace.ptr, 0, f.tileSortWorkspace.bytes, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(f.visStatus.ptr, 0, f.visStatus.bytes, s);
  if (e != cudaSuccess) return check(e, "frame buffers");
  f.sources = sources;
  f.instanceCapacity = instances;
  f.maxTiles = std::max(f.maxTiles, maxTiles);
  return SK_OK;
}

sk_status Context::reserveLod(FrameScratch& f, const World& w, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  auto grab = [&](DeviceBuffer& b, size_t n) {
    if (e == cudaSuccess) e = b.allocate(n);
  };
  const uint32_t frontier = std::max(1u, std::min(w.lodCapacity, w.clusterCount));
  const uint32_t tiles = (frontier + lodTileClusters() - 1) / lodTileClusters();
  grab(f.lodIndices, size_t{w.lodCapacity} * 4);
  grab(f.lodFrontier[0], size_t{frontier} * 4);
  grab(f.lodFrontier[1], size_t{frontier} * 4);
  grab(f.lodCosts, size_t{frontier} * 8);
  grab(f.lodOffsets, size_t{frontier} * 16);
  grab(f.lodPackets, size_t{frontier} * 16);
  grab(f.lodState, 256);
  grab(f.lodStatus, size_t{tiles} * 3 * 8);
  grab(f.lodCounters, 2 * 4);
  if (e == cudaSuccess) e = cudaMemsetAsync(f.lodStatus.ptr, 0, f.lodStatus.bytes, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(f.lodCounters.ptr, 0, f.lodCounters.bytes, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(f.lodState.ptr, 0, f.lodState.bytes, s);
  if (e != cudaSuccess) return check(e, "LOD buffers");
  f.lodFrontierCapacity = frontier;
  return SK_OK;
}

sk_status Context::reserveView(uint32_t w, uint32_t h) {
  const size_t pixelBytes = imageFormat == SK_FORMAT_RGBA32F ? 16 : 4;
  if (copyStream) cudaStreamSynchronize(copyStream);  // no capture copy reads an image freed here
  cudaError_t e = image.allocate(size_t{w} * h * pixelBytes);
  if (e == cudaSuccess && twoImages) e = image2.allocate(size_t{w} * h * pixelBytes);
  if (e == cudaSuccess) e = frameCounters.allocate(sizeof(FrameCounters));
  if (e == cudaSuccess) e = camera.allocate(sizeof(Camera));
  for (auto& sl : slots) {
    if (e == cudaSuccess) e = sl.hostCounters.allocate(sizeof(FrameCounters));
    if (e == cudaSuccess) e = sl.hostCamera.allocate(sizeof(Camera));
  }
  return check(e, "view buffers");
}

Camera cameraOf(const sk_frame& frame, uint32_t w, uint32_t h, float minPixelRadius) {
  Camera c{};
  std::memcpy(c.view, frame.view, 64);
  std::memcpy(c.proj, frame.proj, 64);
  c.screenSize[0] = static_cast<float>(w);
  c.screenSize[1] = static_cast<float>(h);
  // MetalFrameCompute.mm:148-151
  c.focal[0] = (c.screenSize[0] * frame.proj[0]) / 2.0f;
  c.focal[1] = (c.screenSize[1] * frame.proj[5]) / 2.0f;
  c.tanHalfFov[0] = 1.0f / frame.proj[0];
  c.tanHalfFov[1] = 1.0f / frame.proj[5];
  c.outputLinear = 0;
  c.minPixelRadius = minPixelRadius;
  c.cameraPosition[0] = frame.camera_position[0];
  c.cameraPosition[1] = frame.camera_position[1];
  c.cameraPosition[2] = frame.camera_position[2];
  c.cameraPosition[3] = 1.0f;
  c.reveal[0] = frame.reveal_level;
  c.reveal[1] = frame.reveal_band;
  c.reveal[2] = frame.reveal_tint_amount;
  c.reveal[3] = frame.reveal_brightness_boost;
  for (int j = 0; j < 3; ++j) c.revealTint[j] = frame.reveal_tint[j];
  return c;
}

Camera Context::cameraFor(const sk_frame& frame, uint32_t w, uint32_t h) const {
  return cameraOf(frame, w, h, policy.subpixel_threshold);
}

// Validates ranges before anything is written (MetalVisibilityPass.mm:150-162).
sk_status Context::validateRanges(const sk_frame& frame, uint32_t* total) const {
  if (frame.range_count > kMaxRanges || (frame.range_count > 0 && frame.ranges == nullptr))
    return SK_E_INVALID;
  uint32_t sum = 0;
  const uint32_t capacity = world.count;
  for (uint32_t i = 0; i < frame.range_count; ++i) {
    const sk_range& r = frame.ranges[i];
    if (r.offset > world.count || r.count > world.count - r.offset || r.count > capacity - sum)
      return SK_E_INVALID;
    sum += r.count;
  }
  *total = sum;
  return SK_OK;
}

sk_status Context::enqueuePipeline(FrameScratch& f, const ViewTarget& view, const sk_frame& frame,
                                   uint32_t total, cudaStream_t s, uint32_t timing,
                                   cudaEvent_t* events) {
  // Events between stages separate the chained launches, so frame-only timing records just
  // the outer pair.
  const bool timed = timing == 1;
  const int degree = std::max(0, std::min(frame.sh_degree, world.shDegree));
  const bool key16 = policy.sort_depth_bits == 16;
  const uint32_t tilesX = view.tilesX(), tilesY = view.tilesY();
  const uint32_t binsX = view.binsX(), binsY = view.binsY();
  uint32_t* counters = static_cast<uint32_t*>(f.counters.ptr);
  FrameCounters* fc = view.counters;
  uint32_t* error = &fc->error;
  // Direct cell lists write every range; the sorted path only those of non-empty cells.
  const uint32_t cells = binsX * binsY;
  const bool direct = binningMode == SK_BINNING_AUTO && cellListsFit(f.sources, cells) &&
                      f.cellLists.bytes >= cellListBytes(f.sources, cells);
  cudaError_t e = cudaMemsetAsync(fc, 0, sizeof(FrameCounters), s);
  if (e == cudaSuccess && !direct) e = clearTileRanges(static_cast<uint2*>(f.ranges.ptr), cells, s);
  if (timing != 0) cudaEventRecord(events[0], s);

  const bool lod = world.lod;
  if (lod && e == cudaSuccess) {
    LodArgs a{};
    a.clusters = static_cast<const LodCluster*>(world.clusters.ptr);
    a.leaves = static_cast<const uint32_t*>(world.leaves.ptr);
    a.clusterCount = world.clusterCount;
    a.capacity = world.lodCapacity;
    a.limit = lodLimit == 0 ? world.lodCapacity : std::min(lodLimit, world.lodCapacity);
    a.pixelLimit = threshold.pixels();
    a.colorWeight = 4.0f;
    a.cull = policy.enable_frustum_culling ? 1u : 0u;
    a.rounds = world.rounds;
    a.fanout = world.lodFanout;
    a.frontierCapacity = f.lodFrontierCapacity;
    a.frontier[0] = static_cast<uint32_t*>(f.lodFrontier[0].ptr);
    a.frontier[1] = static_cast<uint32_t*>(f.lodFrontier[1].ptr);
    a.costs = static_cast<uint2*>(f.lodCosts.ptr);
    a.offsets = static_cast<uint4*>(f.lodOffsets.ptr);
    a.packets = static_cast<uint4*>(f.lodPackets.ptr);
    a.indices = static_cast<uint32_t*>(f.lodIndices.ptr);
    a.state = static_cast<LodState*>(f.lodState.ptr);
    a.status = static_cast<uint64_t*>(f.lodStatus.ptr);
    a.counters = static_cast<uint32_t*>(f.lodCounters.ptr);
    a.epoch = nextEpoch(2 * world.rounds + 2);
    a.error = error;
    a.report = fc->lod;
    e = launchLodSelect(view.camera, a, s);
  }
  if (timed) cudaEventRecord(events[1], s);

  if (e == cudaSuccess && !lod && frame.range_count > 1) {
    // Ranges and their starts (SplatVisibility.metal:30-37); pageable copies are staged at once.
    // A single range travels in the kernel parameters instead.
    std::vector<uint32_t> starts(frame.range_count + 1, 0);
    for (uint32_t i = 0; i < frame.range_count; ++i) starts[i + 1] = starts[i] + frame.ranges[i].count;
    e = cudaMemcpyAsync(f.rangeBuffer.ptr, frame.ranges, size_t{frame.range_count} * sizeof(Range),
                        cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(f.rangeStarts.ptr, starts.data(), starts.size() * 4,
                          cudaMemcpyHostToDevice, s);
  }
  // The depth sort's workspace: the cull sums the digits of the keys it writes into it.
  SortArgs depthSort{};
  sortBindWorkspace(depthSort, f.sortWorkspace.ptr, f.sources);
  if (e == cudaSuccess) {
    VisibilityArgs v{};
    v.splats = static_cast<const GpuSplat*>(world.splats.ptr);
    v.sh = static_cast<const uint32_t*>(world.sh.ptr);
    v.shStride = shDeviceStride(world.shDegree);
    v.worldCount = world.count;
    v.ranges = static_cast<const Range*>(f.rangeBuffer.ptr);
    v.rangeStarts = static_cast<const uint32_t*>(f.rangeStarts.ptr);
    v.rangeCount = lod ? 0 : frame.range_count;
    if (!lod && frame.range_count == 1) v.single = Range{frame.ranges[0].offset, frame.ranges[0].count};
    v.indices = lod ? static_cast<const uint32_t*>(f.lodIndices.ptr) : nullptr;
    v.indexCount = lod ? &fc->lod[0] : nullptr;
    v.total = lod ? world.lodCapacity : total;
    v.keys = static_cast<uint32_t*>(f.keys.ptr);
    v.projected = static_cast<Projected*>(f.projected.ptr);
    v.spans = static_cast<uint4*>(f.spans.ptr);
    v.tilesX = binsX;
    v.tilesY = binsY;
    v.visibleCount = &fc->visible;
    v.status = static_cast<uint64_t*>(f.visStatus.ptr);
    v.counters = counters + 0;
    v.epoch = nextEpoch(1);
    v.error = error;
    if (!lod && labels.ptr && styleStateCount > 0)
      v.parts = PartLabels{static_cast<const uint16_t*>(labels.ptr),
                           static_cast<const PartStyle*>(stylePalette.ptr),
                           static_cast<const uint32_t*>(styleStateTable.ptr), styleStateCount};
    v.sortAccum = sortDigitAccumulators(depthSort);
    v.sortBases = sortDigitBases(depthSort);
    v.sortPasses = key16 ? 2u : 4u;
    e = launchVisibility(view.camera, v, degree, key16, lod, s);
  }
  if (timed) cudaEventRecord(events[2], s);
  if (e == cudaSuccess) {
    SortArgs a = depthSort;
    a.keysIn = static_cast<const uint32_t*>(f.keys.ptr);
    a.valuesIn = nullptr;
    a.keysOut = nullptr;
    a.valuesOut = static_cast<uint32_t*>(f.order.ptr);
    a.count = &fc->visible;
    a.capacity = f.sources;
    a.bits = key16 ? 16 : 32;
    a.basesReady = 1;
    a.epoch = nextEpoch(4);
    a.error = error;
    a.withheldTilePlusOne = testWithheldTile;
    testWithheldTile = 0;
    e = launchSort(a, s);
  }
  if (timed) cudaEventRecord(events[3], s);
  if (e == cudaSuccess && direct) {
    // each cell's list written in place, front to back, with its range
    BinArgs b{};
    b.spans = static_cast<const uint4*>(f.spans.ptr);
    b.order = static_cast<const uint32_t*>(f.order.ptr);
    b.count = &fc->visible;
    b.capacity = f.sources;
    b.width = view.width, b.height = view.height, b.tilesX = binsX, b.tilesY = binsY;
    b.instanceValues = static_cast<uint32_t*>(f.instValuesSorted.ptr);
    b.instanceCapacity = f.instanceCapacity;
    b.instanceCount = &fc->instances;
    b.overflow = &fc->overflow;
    CellLists cl{};
    cl.cells = cells;
    cl.workspace = f.cellLists.ptr;
    cl.ranges = static_cast<uint2*>(f.ranges.ptr);
    cl.counters = counters + 8;
    cl.epoch = nextEpoch(1);
    cl.error = error;
    e = launchCellLists(b, cl, s);
  }
  if (e == cudaSuccess && !direct) {
    BinArgs b{};
    b.spans = static_cast<const uint4*>(f.spans.ptr);
    b.order = static_cast<const uint32_t*>(f.order.ptr);
    b.count = &fc->visible;
    b.capacity = f.sources;
    b.width = view.width, b.height = view.height, b.tilesX = binsX, b.tilesY = binsY;
    b.instanceKeys = static_cast<uint32_t*>(f.instKeys.ptr);
    b.instanceValues = static_cast<uint32_t*>(f.instValues.ptr);
    b.instanceCapacity = f.instanceCapacity;
    b.instanceCount = &fc->instances;
    b.overflow = &fc->overflow;
    b.blockSums = static_cast<uint32_t*>(f.binSums.ptr);
    b.balanced = 1;
    e = launchBinning(b, s);
  }
  if (e == cudaSuccess && !direct) {
    SortArgs a{};
    a.keysIn = static_cast<const uint32_t*>(f.instKeys.ptr);
    a.valuesIn = static_cast<const uint32_t*>(f.instValues.ptr);
    a.keysOut = static_cast<uint32_t*>(f.instKeysSorted.ptr);
    a.valuesOut = static_cast<uint32_t*>(f.instValuesSorted.ptr);
    a.count = &fc->instances;
    a.capacity = f.instanceCapacity;
    a.bits = 16;
    sortBindWorkspaceFor(a, f.tileSortWorkspace.ptr, f.instanceCapacity, kTileSortTileKeys);
    a.tileKeys = kTileSortTileKeys;
    a.epoch = nextEpoch(4);
    a.error = error;
    e = launchSort(a, s);
  }
  if (e == cudaSuccess && !direct)
    e = launchTileRanges(static_cast<const uint32_t*>(f.instKeysSorted.ptr), &fc->instances,
                         f.instanceCapacity, static_cast<uint2*>(f.ranges.ptr), binsX * binsY, s);
  if (timed) cudaEventRecord(events[4], s);
  if (e == cudaSuccess) {
    CompositeArgs c{};
    c.projected = static_cast<const Projected*>(f.projected.ptr);
    c.values = static_cast<const uint32_t*>(f.instValuesSorted.ptr);
    c.ranges = static_cast<const uint2*>(f.ranges.ptr);
    c.width = view.width, c.height = view.height, c.tilesX = tilesX, c.tilesY = tilesY;
    c.binsX = binsX;
    for (int j = 0; j < 3; ++j) c.background[j] = static_cast<float>(policy.background[j]);
    c.opaque = 1;
    c.cutoff = policy.enable_early_termination ? kTransmittanceCutoff : 0.0f;
    c.image = view.image;
    c.format = imageFormat == SK_FORMAT_RGBA32F ? kRgba32f : kRgba8;
    c.fragments = &fc->fragments_lo;
    c.countFragments = timing == 1 ? 1u : 0u;
    c.loaded = &fc->loaded;
    e = launchComposite(c, s);
  }
  if (timing != 0) cudaEventRecord(events[5], s);
  if (e == cudaSuccess && view.hostCounters)
    e = cudaMemcpyAsync(view.hostCounters, fc, sizeof(FrameCounters), cudaMemcpyDeviceToHost, s);
  return check(e, "frame");
}

ViewTarget Context::plainView(const Slot& slot) {
  const bool second = &slot == &slots[1];
  ViewTarget v;
  v.width = width;
  v.height = height;
  v.image = imageOf(slot.image);
  v.counters = static_cast<FrameCounters*>(second ? frameCounters2.ptr : frameCounters.ptr);
  v.hostCounters = static_cast<FrameCounters*>(slot.hostCounters.ptr);
  v.camera = static_cast<const Camera*>(second ? camera2.ptr : camera.ptr);
  return v;
}

sk_status Context::prepareSecondSlot() {
  cudaError_t e = cudaSuccess;
  if (!stream2) e = cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = frameCounters2.allocate(sizeof(FrameCounters));
  if (e == cudaSuccess) e = camera2.allocate(sizeof(Camera));
  if (e != cudaSuccess) return check(e, "second frame slot");
  if (!twoImages) {  // the slots' frames must not draw into one image
    twoImages = true;
    const sk_status st = reserveView(width, height);
    if (st != SK_OK) {
      twoImages = false;
      return st;
    }
  }
  if (scratch2.sources < scratch.sources || scratch2.instanceCapacity < scratch.instanceCapacity ||
      scratch2.maxTiles < scratch.maxTiles)
    return reserveScratch(scratch2, std::max(scratch.sources, scratch2.sources),
                          std::max(scratch.instanceCapacity, scratch2.instanceCapacity),
                          scratch.maxTiles, stream2);
  return SK_OK;
}

cudaError_t Context::syncStreams() {
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess && stream2) e = cudaStreamSynchronize(stream2);
  return e;
}

// Enqueues the slot's frame on the slot's stream. Its pinned camera is free: the frame that used
// the slot before has finished. The slot's device camera is rewritten after that frame's
// kernels, in stream order.
sk_status Context::enqueueSlot(uint32_t index) {
  Slot& slot = slots[index];
  const cudaStream_t s = streamOf(index);
  *static_cast<Camera*>(slot.hostCamera.ptr) = cameraFor(slot.frame, width, height);
  const ViewTarget view = plainView(slot);
  cudaError_t e = cudaMemcpyAsync(const_cast<Camera*>(view.camera), slot.hostCamera.ptr,
                                  sizeof(Camera), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return check(e, "camera upload");
  // the image this frame draws into may still be on its way to a capture's host buffer
  if (imageCopied[slot.image]) {
    e = cudaStreamWaitEvent(s, imageFree[slot.image], 0);
    if (e != cudaSuccess) return check(e, "capture wait");
  }
  sk_status st = enqueuePipeline(scratchOf(index), view, slot.frame, slot.total, s, timeStages,
                                 slot.events);
  if (st != SK_OK) return st;
  st = check(cudaEventRecord(slot.done, s), "frame");
  if (st != SK_OK) return st;
  // captures of this frame copy its image once it is drawn (again after a redraw)
  for (auto& c : captures)
    if (c.frame == slot.number && (st = issueCapture(c, slot)) != SK_OK) return st;
  return SK_OK;
}

size_t Context::imageBytes() const {
  return size_t{width} * height * (imageFormat == SK_FORMAT_RGBA32F ? 16 : 4);
}

sk_status Context::issueCapture(Capture& c, const Slot& slot) {
  if (c.bytes < imageBytes()) {
    c.tooSmall = true;
    return SK_OK;
  }
  cudaError_t e = cudaStreamWaitEvent(copyStream, slot.done, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c.host, imageOf(slot.image), imageBytes(), cudaMemcpyDeviceToHost, copyStream);
  if (e == cudaSuccess) e = cudaEventRecord(c.copied, copyStream);
  if (e == cudaSuccess) e = cudaEventRecord(imageFree[slot.image], copyStream);
  if (e != cudaSuccess) return check(e, "capture copy");
  imageCopied[slot.image] = true;
  c.issued = true;
  return SK_OK;
}

sk_status Context::finishOldest() {
  if (inFlight.empty()) return SK_OK;
  Slot& slot = slots[inFlight.front()];
  cudaError_t e = cudaEventSynchronize(slot.done);
  if (e != cudaSuccess) return check(e, "frame wait");
  const FrameCounters c = *static_cast<const FrameCounters*>(slot.hostCounters.ptr);
  if (c.overflow) {
    // Every frame in flight drew with these list buffers (or after one that did, into the same
    // image): wait for all of them, grow the buffers and draw them all again, in order.
    e = syncStreams();
    if (e != cudaSuccess) return check(e, "frame wait");
    uint32_t most = c.instances;
    for (const uint32_t k : inFlight) {
      const auto* fc = static_cast<const FrameCounters*>(slots[k].hostCounters.ptr);
      most = std::max(most, fc->instances);
    }
    const uint32_t need = static_cast<uint32_t>(
        std::min<uint64_t>(uint64_t{most} + most / 4 + 1024, 0x7fffffffu));
    sk_status st = reserveScratch(scratch, scratch.sources, need, scratch.maxTiles, stream);
    if (st == SK_OK && stream2) st = prepareSecondSlot();
    for (size_t k = 0; st == SK_OK && k < inFlight.size(); ++k) st = enqueueSlot(inFlight[k]);
    if (st != SK_OK) {
      inFlight.clear();  // nothing of theirs is left running
      return st;
    }
    return finishOldest();
  }
  lastSlot = inFlight.front();
  inFlight.pop_front();
  ++completed;
  lastCounters = c;
  if (timeStages != 0) {
    float ms[5] = {0, 0, 0, 0, 0};
    if (timeStages == 1)
      for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&ms[i], slot.events[i], slot.events[i + 1]);
    float all = 0;
    cudaEventElapsedTime(&all, slot.events[0], slot.events[5]);
    stats.select_ms = ms[0], stats.cull_ms = ms[1], stats.sort_ms = ms[2];
    stats.bin_ms = ms[3], stats.composite_ms = ms[4], stats.gpu_ms = all;
  }
  if (world.lod) {
    threshold.update(c.lod[0], c.lod[4],
                     lodLimit == 0 ? world.lodCapacity : std::min(lodLimit, world.lodCapacity));
  }
  if (c.error) return fail(SK_E_TIMEOUT, "a bounded device wait or bounds check failed in the last frame");
  return SK_OK;
}

sk_status Context::finishFrame(bool wait) {
  sk_status first = SK_OK;
  while (!inFlight.empty()) {
    if (!wait && cudaEventQuery(slots[inFlight.front()].done) != cudaSuccess) break;
    const sk_status st = finishOldest();
    if (st == SK_E_DEVICE) return st;
    if (first == SK_OK) first = st;
  }
  return first;
}

sk_status Context::finishThrough(uint64_t number) {
  sk_status first = SK_OK;
  while (!inFlight.empty() && slots[inFlight.front()].number <= number) {
    const sk_status st = finishOldest();
    if (st == SK_E_DEVICE) return st;
    if (first == SK_OK) first = st;
  }
  return first;
}

sk_status Context::uploadCloud(const sk_cloud_view& cloud, int maxSh, World& w) {
  if (cloud.count > 0 && (!cloud.positions || !cloud.covariances || !cloud.colors || !cloud.alphas))
    return fail(SK_E_INVALID, "cloud arrays missing");
  host::CloudRef ref{cloud.positions, cloud.covariances, cloud.colors, cloud.alphas, cloud.sh,
                     cloud.count, cloud.sh ? std::max(0, std::min(cloud.sh_degree, 3)) : 0};
  const int degree = std::max(0, std::min({maxSh, ref.shDegree, 3}));
  const uint32_t stride = shDeviceStride(degree);
  std::vector<GpuSplat> packed(cloud.count);
  host::packSplats(ref, 0, cloud.count, packed.data(), hostThreadsPublic());
  std::vector<uint32_t> sh(size_t{cloud.count} * stride);
  host::packSh(ref, degree, 0, cloud.count, sh.data(), stride, hostThreadsPublic());
  cudaError_t e = w.splats.allocate(packed.size() * sizeof(GpuSplat));
  if (e == cudaSuccess) e = w.sh.allocate(sh.size() * 4);
  if (e != cudaSuccess) return check(e, "world upload");
  if (cloud.count) {
    e = cudaMemcpy(w.splats.ptr, packed.data(), packed.size() * sizeof(GpuSplat), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !sh.empty())
      e = cudaMemcpy(w.sh.ptr, sh.data(), sh.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return check(e, "world upload");
  }
  w.count = cloud.count;
  w.shDegree = degree;
  return SK_OK;
}

}  // namespace sk

using sk::Context;

extern "C" {

void sk_default_policy(sk_policy* out) {
  if (!out) return;
  // RenderPolicy{} (RenderPolicy.h:17-40)
  out->lod_error_pixels = 1.0f;
  out->lod_splat_limit = 0;
  out->alpha_threshold = 1.0f / 255.0f;
  out->subpixel_threshold = 1.0f;
  out->enable_frustum_culling = 1;
  out->enable_early_termination = 1;
  out->sort_depth_bits = 16;
  out->background[0] = 0.05, out->background[1] = 0.05, out->background[2] = 0.08;
}

sk_status sk_create(const sk_config* config, sk_context** out) {
  if (!config || !out) return SK_E_INVALID;
  *out = nullptr;
  if (config->image_format != SK_FORMAT_RGBA8 && config->image_format != SK_FORMAT_RGBA32F)
    return SK_E_INVALID;
  if (config->width == 0 || config->height == 0 || config->width > 16384 || config->height > 16384)
    return SK_E_INVALID;
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || config->device < 0 || config->device >= devices) {
    cudaGetLastError();
    return SK_E_DEVICE;
  }
  auto ctx = std::make_unique<Context>();
  ctx->device = config->device;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return SK_E_DEVICE;
  ctx->width = config->width;
  ctx->height = config->height;
  ctx->imageFormat = config->image_format;
  ctx->timeStages = std::min<uint32_t>(config->time_stages, 2);
  sk_default_policy(&ctx->policy);
  ctx->threshold.reset(ctx->policy.lod_error_pixels);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return SK_E_DEVICE;
  for (auto& sl : ctx->slots) {
    if (cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess) return SK_E_DEVICE;
    for (auto& ev : sl.events)
      if (cudaEventCreate(&ev) != cudaSuccess) return SK_E_DEVICE;
  }
  if (ctx->reserveView(ctx->width, ctx->height) != SK_OK) return SK_E_DEVICE;
  const uint32_t tiles = ((ctx->width + 15) / 16) * ((ctx->height + 15) / 16);
  if (ctx->reserveScratch(ctx->scratch, 1, 1024, tiles, ctx->stream) != SK_OK) return SK_E_DEVICE;
  *out = reinterpret_cast<sk_context*>(ctx.release());
  return SK_OK;
}

void sk_destroy(sk_context* handle) {
  auto* ctx = reinterpret_cast<Context*>(handle);
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) ctx->syncStreams();
  delete ctx;
}

const char* sk_last_error(const sk_context* handle) {
  const auto* ctx = reinterpret_cast<const Context*>(handle);
  return ctx ? ctx->error.c_str() : "no context";
}

#define SK_CTX(handle)                                          \
  auto* ctx = reinterpret_cast<Context*>(handle);               \
  if (!ctx) return SK_E_INVALID;                                \
  if (ctx->failed.load()) return SK_E_DEVICE;                   \
  cudaSetDevice(ctx->device)

sk_status sk_resize(sk_context* handle, uint32_t width, uint32_t height) {
  SK_CTX(handle);
  if (width == 0 || height == 0 || width > 16384 || height > 16384) return SK_E_INVALID;
  sk_status st = ctx->finishFrame(true);
  if (st != SK_OK && st != SK_E_TIMEOUT) return st;
  st = ctx->reserveView(width, height);
  if (st != SK_OK) return st;
  const uint32_t tiles = ((width + 15) / 16) * ((height + 15) / 16);
  st = ctx->reserveScratch(ctx->scratch, ctx->scratch.sources, ctx->scratch.instanceCapacity, tiles,
                           ctx->stream);
  if (st != SK_OK) return st;
  ctx->width = width;
  ctx->height = height;
  return SK_OK;
}

sk_status sk_device_capabilities(sk_context* handle, sk_capabilities* out) {
  SK_CTX(handle);
  if (!out) return SK_E_INVALID;
  std::memset(out, 0, sizeof(*out));
  out->max_lod_capacity_splats = sk::kMaxLodBudgetPublic;
  out->min_residency_capacity_splats = 1;
  out->max_residency_capacity_splats = 0x7fffffffu;
  out->supports_subgroups = 1;
  out->max_texture_dimension = 16384;
  out->sorts_on_gpu = 1;
  out->selects_lod_on_gpu = 1;
  size_t freeBytes = 0, total = 0;
  if (cudaMemGetInfo(&freeBytes, &total) == cudaSuccess) out->total_memory = total;
  return SK_OK;
}

sk_status sk_apply_render_policy(sk_context* handle, const sk_policy* p) {
  SK_CTX(handle);
  if (!p) return SK_E_INVALID;
  // validRenderPolicy (splatkit-engine/src/rendering/RenderPolicy.cpp:29-52)
  const bool ok = std::isfinite(p->lod_error_pixels) && p->lod_error_pixels > 0.0f &&
                  std::isfinite(p->alpha_threshold) && p->alpha_threshold >= 0.0f &&
                  p->alpha_threshold <= 1.0f && std::isfinite(p->subpixel_threshold) &&
                  p->subpixel_threshold >= 0.0f &&
                  (p->sort_depth_bits == 16 || p->sort_depth_bits == 32) &&
                  std::all_of(p->background, p->background + 3,
                              [](double c) { return std::isfinite(c) && c >= 0 && c <= 1; });
  if (!ok) return ctx->fail(SK_E_INVALID, "render policy out of range");
  const bool lodChanged = p->lod_error_pixels != ctx->threshold.policyPixels() ||
                          p->lod_splat_limit != ctx->lodLimit;
  ctx->policy = *p;
  if (lodChanged) {
    ctx->threshold.reset(p->lod_error_pixels);
    ctx->lodLimit = p->lod_splat_limit;
  }
  return SK_OK;
}

sk_status sk_available_memory(sk_context* handle, uint64_t* bytes) {
  SK_CTX(handle);
  if (!bytes) return SK_E_INVALID;
  size_t freeBytes = 0, total = 0;
  if (cudaMemGetInfo(&freeBytes, &total) != cudaSuccess) return ctx->check(cudaGetLastError(), "memory");
  *bytes = freeBytes;
  return SK_OK;
}

int32_t sk_gpu_failed(sk_context* handle) {
  auto* ctx = reinterpret_cast<Context*>(handle);
  return ctx && ctx->failed.load() ? 1 : 0;
}

sk_status sk_upload_world(sk_context* handle, const sk_cloud_view* cloud, int32_t maxSh) {
  SK_CTX(handle);
  if (!cloud) return SK_E_INVALID;
  sk_status st = ctx->finishFrame(true);
  if (st == SK_E_DEVICE) return st;
  ctx->syncStreams();
  // Build the new world aside; the old one stays until everything succeeded.
  sk::World fresh;
  st = ctx->uploadCloud(*cloud, maxSh, fresh);
  if (st != SK_OK) return st;
  st = ctx->reserveScratch(ctx->scratch, cloud->count,
                           std::max(ctx->scratch.instanceCapacity, ctx->instanceGuess(cloud->count)),
                           ctx->scratch.maxTiles, ctx->stream);
  if (st != SK_OK) return st;
  ctx->world = std::move(fresh);
  ctx->labels.release();  // labels belong to the world they were uploaded for
  return SK_OK;
}

sk_status sk_create_slab(sk_context* handle, uint32_t capacity, int32_t shDegree) {
  SK_CTX(handle);
  if (shDegree < 0 || shDegree > 3) return SK_E_INVALID;
  sk_status st = ctx->finishFrame(true);
  if (st == SK_E_DEVICE) return st;
  ctx->syncStreams();
  sk::World fresh;
  cudaError_t e = fresh.splats.allocate(size_t{capacity} * sizeof(sk::GpuSplat));
  if (e == cudaSuccess) e = fresh.sh.allocate(size_t{capacity} * sk::shDeviceStride(shDegree) * 4);
  if (e == cudaSuccess) e = cudaMemset(fresh.splats.ptr, 0, fresh.splats.bytes);
  if (e == cudaSuccess) e = cudaMemset(fresh.sh.ptr, 0, fresh.sh.bytes);
  if (e != cudaSuccess) return ctx->check(e, "slab");
  st = ctx->reserveScratch(ctx->scratch, capacity,
                           std::max(ctx->scratch.instanceCapacity, ctx->instanceGuess(capacity)),
                           ctx->scratch.maxTiles, ctx->stream);
  if (st != SK_OK) return st;
  fresh.count = capacity;
  fresh.shDegree = shDegree;
  ctx->world = std::move(fresh);
  ctx->labels.release();  // labels belong to the world they were uploaded for
  return SK_OK;
}

sk_status sk_upload_tile(sk_context* handle, uint32_t offset, const sk_cloud_view* cloud) {
  SK_CTX(handle);
  if (!cloud || ctx->world.lod) return SK_E_INVALID;
  if (offset > ctx->world.count || cloud->count > ctx->world.count - offset) return SK_E_INVALID;
  if (cloud->count == 0) return SK_OK;
  sk::host::CloudRef ref{cloud->positions, cloud->covariances, cloud->colors, cloud->alphas,
                         cloud->sh, cloud->count,
                         cloud->sh ? std::max(0, std::min(cloud->sh_degree, 3)) : 0};
  if (!ref.positions || !ref.covariances || !ref.colors || !ref.alphas) return SK_E_INVALID;
  const int degree = std::min(ctx->world.shDegree, ref.shDegree);
  const uint32_t stride = sk::shDeviceStride(ctx->world.shDegree);
  std::vector<sk::GpuSplat> packed(cloud->count);
  sk::host::packSplats(ref, 0, cloud->count, packed.data(), sk::hostThreadsPublic());
  std::vector<uint32_t> sh(size_t{cloud->count} * stride, 0u);
  if (degree > 0) sk::host::packSh(ref, degree, 0, cloud->count, sh.data(), stride, sk::hostThreadsPublic());
  sk_status st = ctx->finishFrame(true);
  if (st == SK_E_DEVICE) return st;
  cudaError_t e = cudaMemcpy(static_cast<sk::GpuSplat*>(ctx->world.splats.ptr) + offset, packed.data(),
                             packed.size() * sizeof(sk::GpuSplat), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && stride > 0)
    e = cudaMemcpy(static_cast<uint32_t*>(ctx->world.sh.ptr) + size_t{offset} * stride, sh.data(),
                   sh.size() * 4, cudaMemcpyHostToDevice);
  return ctx->check(e, "tile upload");
}

sk_status sk_upload_lod_world(sk_context* handle, const sk_lod_view* tree, int32_t maxSh,
                              uint32_t budget) {
  SK_CTX(handle);
  if (!tree || !tree->layout || tree->node_count == 0 || tree->nodes.count != tree->node_count)
    return ctx->fail(SK_E_INVALID, "invalid LOD tree view");
  std::string why;
  const int64_t depth = sk::host::lodDepth(reinterpret_cast<const sk::LodNode*>(tree->layout),
                                           tree->node_count, tree->leaf_count, &why);
  if (depth < 0) return ctx->fail(SK_E_INVALID, "invalid LOD hierarchy: " + why);
  if (budget == 0) return ctx->fail(SK_E_INVALID, "LOD budget is zero");
  sk_status st = ctx->finishFrame(true);
  if (st == SK_E_DEVICE) return st;
  ctx->syncStreams();
  // Selection data: the tree's own, else built once here (MetalLodSelection.mm:68-74).
  std::vector<sk::LodCluster> clusters;
  std::vector<uint32_t> leaves;
  if (tree->cluster_count > 0 && tree->clusters && tree->leaves) {
    clusters.resize(tree->cluster_count);
    std::memcpy(clusters.data(), tree->clusters, clusters.size() * sizeof(sk::LodCluster));
    leaves.assign(tree->leaves, tree->leaves + tree->leaf_ref_count);
  } else {
    sk::host::CloudRef ref{tree->nodes.positions, tree->nodes.covariances, tree->nodes.colors,
                           tree->nodes.alphas, tree->nodes.sh, tree->nodes.count,
                           tree->nodes.sh ? std::max(0, std::min(tree->nodes.sh_degree, 3)) : 0};
    if (!sk::host::buildSelection(ref, reinterpret_cast<const sk::LodNode*>(tree->layout),
                                  tree->node_count, clusters, leaves))
      return ctx->fail(SK_E_INVALID, "invalid LOD hierarchy: the layout is not breadth first");
  }
  sk::World fresh;
  st = ctx->uploadCloud(tree->nodes, maxSh, fresh);
  if (st != SK_OK) return st;
  const uint32_t capacity = std::min({budget, sk::kMaxLodBudgetPublic, std::max(tree->leaf_count, 1u)});
  cudaError_t e = fresh.clusters.allocate(clusters.size() * sizeof(sk::LodCluster));
  if (e == cudaSuccess) e = fresh.leaves.allocate(leaves.size() * 4);
  if (e == cudaSuccess)
    e = cudaMemcpy(fresh.clusters.ptr, clusters.data(), clusters.size() * sizeof(sk::LodCluster),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !leaves.empty())
    e = cudaMemcpy(fresh.leaves.ptr, leaves.data(), leaves.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return ctx->check(e, "LOD upload");
  fresh.lod = true;
  fresh.clusterCount = static_cast<uint32_t>(clusters.size());
  fresh.leafRefCount = static_cast<uint32_t>(leaves.size());
  fresh.rounds = static_cast<uint32_t>(depth) + 1;
  for (const sk::LodCluster& c : clusters) fresh.lodFanout = std::max(fresh.lodFanout, c.childCount);
  fresh.lodCapacity = capacity;
  st = ctx->reserveLod(ctx->scratch, fresh, ctx->stream);
  if (st != SK_OK) return st;
  // Projections and sort scratch scale with the cut, not with all resident nodes.
  st = ctx->reserveScratch(ctx->scratch, capacity,
                           std::max(ctx->scratch.instanceCapacity, ctx->instanceGuess(capacity)),
                           ctx->scratch.maxTiles, ctx->stream);
  if (st != SK_OK) return st;
  ctx->world = std::move(fresh);
  ctx->labels.release();  // labels belong to the world they were uploaded for
  ctx->threshold.reset(ctx->threshold.policyPixels());
  return SK_OK;
}

sk_status sk_world_info(sk_context* handle, uint32_t* count, int32_t* shDegree) {
  SK_CTX(handle);
  if (!ctx->world.splats.ptr) return SK_E_NO_WORLD;
  if (count) *count = ctx->world.count;
  if (shDegree) *shDegree = ctx->world.shDegree;
  return SK_OK;
}

sk_status sk_draw(sk_context* handle, const sk_frame* frame) {
  SK_CTX(handle);
  if (!frame) return SK_E_INVALID;
  uint32_t total = 0;
  if (!ctx->world.lod && ctx->world.splats.ptr) {
    if (ctx->validateRanges(*frame, &total) != SK_OK)
      return ctx->fail(SK_E_INVALID, "invalid visibility ranges");
  }
  // Two frames in flight (one on a LOD world): the oldest finishes first when all slots are busy.
  const size_t depth = ctx->world.lod ? 1 : sk::Context::kFrameSlots;
  while (ctx->inFlight.size() >= depth) {
    const sk_status st = ctx->finishOldest();
    if (st == SK_E_DEVICE) return st;
  }
  if (!ctx->world.splats.ptr) total = 0;
  uint32_t index = 0;
  while (std::find(ctx->inFlight.begin(), ctx->inFlight.end(), index) != ctx->inFlight.end()) ++index;
  if (index == 1) {
    const sk_status st = ctx->prepareSecondSlot();
    if (st != SK_OK) return st;
  }
  sk::Context::Slot& slot = ctx->slots[index];
  if (ctx->twoImages) ctx->imageSlot ^= 1u;
  slot.frame = *frame;
  slot.total = total;
  slot.ranges.assign(frame->ranges, frame->ranges + (frame->ranges ? frame->range_count : 0));
  slot.frame.ranges = slot.ranges.data();
  slot.image = ctx->imageSlot;
  slot.number = ++ctx->submitted;  // pending captures are bound to this number
  for (auto& c : ctx->captures)
    if (c.frame == 0) c.frame = slot.number;
  const sk_status st = ctx->enqueueSlot(index);
  if (st != SK_OK) {
    for (auto& c : ctx->captures)
      if (c.frame == slot.number) c.frame = 0;
    --ctx->submitted;
    return st;
  }
  ctx->inFlight.push_back(index);
  return SK_OK;
}

sk_status sk_wait_idle(sk_context* handle) {
  SK_CTX(handle);
  const sk_status st = ctx->finishFrame(true);
  if (st != SK_OK) return st;
  return ctx->check(ctx->syncStreams(), "wait");
}

sk_status sk_read_image(sk_context* handle, void* host, size_t bytes, int32_t format) {
  SK_CTX(handle);
  if (!host) return SK_E_INVALID;
  sk_status st = ctx->finishFrame(true);
  if (st != SK_OK) return st;
  const size_t pixels = size_t{ctx->width} * ctx->height;
  const bool deviceFloat = ctx->imageFormat == SK_FORMAT_RGBA32F;
  const size_t need = pixels * (format == SK_FORMAT_RGBA32F ? 16 : 4);
  if (bytes < need) return ctx->fail(SK_E_INVALID, "image buffer too small");
  if (format == SK_FORMAT_RGBA32F && !deviceFloat)
    return ctx->fail(SK_E_INVALID, "the context renders 8-bit images");
  if ((format == SK_FORMAT_RGBA8 && !deviceFloat) || (format == SK_FORMAT_RGBA32F && deviceFloat))
    return ctx->check(cudaMemcpy(host, ctx->imageOf(ctx->imageSlot), need, cudaMemcpyDeviceToHost),
                      "readback");
  // Conversions on the host.
  std::vector<uint8_t> staging(pixels * (deviceFloat ? 16 : 4));
  cudaError_t e = cudaMemcpy(staging.data(), ctx->imageOf(ctx->imageSlot), staging.size(),
                             cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return ctx->check(e, "readback");
  uint8_t* out = static_cast<uint8_t*>(host);
  for (size_t i = 0; i < pixels; ++i) {
    uint8_t rgba[4];
    if (deviceFloat) {
      const float* f = reinterpret_cast<const float*>(staging.data()) + i * 4;
      for (int c = 0; c < 4; ++c)
        rgba[c] = static_cast<uint8_t>(std::lround(std::min(1.0f, std::max(0.0f, f[c])) * 255.0f));
    } else {
      std::memcpy(rgba, staging.data() + i * 4, 4);
    }
    if (format == SK_FORMAT_BGRA8) std::swap(rgba[0], rgba[2]);
    std::memcpy(out + i * 4, rgba, 4);
  }
  return SK_OK;
}

sk_status sk_capture_next_frame(sk_context* handle, void* host, size_t bytes, int32_t format,
                                uint64_t* ticket) {
  SK_CTX(handle);
  if (!host || !ticket) return SK_E_INVALID;
  const int32_t native = ctx->imageFormat == SK_FORMAT_RGBA32F ? SK_FORMAT_RGBA32F : SK_FORMAT_RGBA8;
  if (format != native) return ctx->fail(SK_E_INVALID, "a capture copies the context's own pixel format");
  if (bytes < ctx->imageBytes()) return ctx->fail(SK_E_INVALID, "capture buffer too small");
  for (const auto& c : ctx->captures)
    if (c.frame == 0) return ctx->fail(SK_E_INVALID, "a capture is already waiting for the next frame");
  if (!ctx->copyStream) {
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->copyStream, cudaStreamNonBlocking);
    for (auto& ev : ctx->imageFree)
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return ctx->check(e, "capture set-up");
  }
  if (!ctx->twoImages) {
    const sk_status st = ctx->finishFrame(true);
    if (st != SK_OK) return st;
    ctx->twoImages = true;
    const sk_status vs = ctx->reserveView(ctx->width, ctx->height);
    if (vs != SK_OK) {
      ctx->twoImages = false;
      return vs;
    }
  }
  Context::Capture c;
  c.ticket = ctx->nextCapture++;
  c.host = host;
  c.bytes = bytes;
  const cudaError_t e = cudaEventCreateWithFlags(&c.copied, cudaEventDisableTiming);
  if (e != cudaSuccess) return ctx->check(e, "capture event");
  ctx->captures.push_back(c);
  *ticket = c.ticket;
  return SK_OK;
}

sk_status sk_wait_capture(sk_context* handle, uint64_t ticket) {
  SK_CTX(handle);
  auto it = std::find_if(ctx->captures.begin(), ctx->captures.end(),
                         [&](const Context::Capture& c) { return c.ticket == ticket; });
  if (it == ctx->captures.end() || it->frame == 0)
    return ctx->fail(SK_E_INVALID, "no such capture, or its frame is not drawn yet");
  sk_status st = SK_OK;
  st = ctx->finishThrough(it->frame);  // may draw it again
  it = std::find_if(ctx->captures.begin(), ctx->captures.end(),
                    [&](const Context::Capture& c) { return c.ticket == ticket; });
  const cudaError_t e = cudaEventSynchronize(it->copied);
  const bool tooSmall = it->tooSmall;
  cudaEventDestroy(it->copied);
  ctx->captures.erase(it);
  if (e != cudaSuccess) return ctx->check(e, "capture wait");
  if (tooSmall) return ctx->fail(SK_E_INVALID, "the target was resized past the capture buffer");
  return st;
}

sk_status sk_set_binning(sk_context* handle, uint32_t mode) {
  SK_CTX(handle);
  if (mode != SK_BINNING_AUTO && mode != SK_BINNING_SORTED) return SK_E_INVALID;
  const sk_status st = ctx->finishFrame(true);
  if (st != SK_OK) return st;
  ctx->binningMode = mode;
  return SK_OK;
}

sk_status sk_set_timing(sk_context* handle, uint32_t time_stages) {
  SK_CTX(handle);
  if (time_stages > 2) return SK_E_INVALID;
  const sk_status st = ctx->finishFrame(true);
  if (st != SK_OK) return st;
  ctx->timeStages = time_stages;
  return SK_OK;
}

sk_status sk_get_stats(sk_context* handle, sk_stats* out) {
  SK_CTX(handle);
  if (!out) return SK_E_INVALID;
  ctx->finishFrame(false);
  sk_stats s = ctx->stats;
  s.submitted_frames = ctx->submitted;
  s.completed_frames = ctx->completed;
  const sk::FrameCounters& c = ctx->lastCounters;
  s.draw_count = c.visible;
  s.selected_count = ctx->world.lod ? std::min(c.lod[0], ctx->world.lodCapacity) : 0;
  s.lod_limited = c.lod[4];
  s.lod_evaluated = c.lod[5];
  s.instances = c.instances;
  s.device_error = c.error;
  s.fragments = uint64_t{c.fragments_lo} | (uint64_t{c.fragments_hi} << 32);
  s.lod_pixels = ctx->threshold.pixels();
  s.instances_read = c.loaded;
  *out = s;
  return SK_OK;
}

sk_status sk_read_visible(sk_context* handle, uint32_t* keys, void* projected, uint32_t capacity,
                          uint32_t* count) {
  SK_CTX(handle);
  sk_status st = ctx->finishFrame(true);
  if (st != SK_OK) return st;
  const uint32_t n = ctx->lastCounters.visible;
  if (count) *count = n;
  const uint32_t copy = std::min(n, capacity);
  cudaError_t e = cudaSuccess;
  if (keys && copy) e = cudaMemcpy(keys, ctx->scratchOf(ctx->lastSlot).keys.ptr, size_t{copy} * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && projected && copy)
    e = cudaMemcpy(projected, ctx->scratchOf(ctx->lastSlot).projected.ptr, size_t{copy} * 32, cudaMemcpyDeviceToHost);
  return ctx->check(e, "readback");
}

sk_status sk_read_order(sk_context* handle, uint32_t* order, uint32_t capacity, uint32_t* count) {
  SK_CTX(handle);
  sk_status st = ctx->finishFrame(true);
  if (st != SK_OK) return st;
  const uint32_t n = ctx->lastCounters.visible;
  if (count) *count = n;
  const uint32_t copy = std::min(n, capacity);
  if (!order || !copy) return SK_OK;
  return ctx->check(cudaMemcpy(order, ctx->scratchOf(ctx->lastSlot).order.ptr, size_t{copy} * 4, cudaMemcpyDeviceToHost),
                    "readback");
}

sk_status sk_read_cut(sk_context* handle, uint32_t* indices, uint32_t capacity, uint32_t* count,
                      uint32_t* lod6) {
  SK_CTX(handle);
  sk_status st = ctx->finishFrame(true);
  if (st != SK_OK) return st;
  if (!ctx->world.lod) return ctx->fail(SK_E_INVALID, "not a LOD world");
  const uint32_t n = std::min(ctx->lastCounters.lod[0], ctx->world.lodCapacity);
  if (count) *count = n;
  if (lod6) std::memcpy(lod6, ctx->lastCounters.lod, 24);
  const uint32_t copy = std::min(n, capacity);
  if (!indices || !copy) return SK_OK;
  return ctx->check(cudaMemcpy(indices, ctx->scratchOf(ctx->lastSlot).lodIndices.ptr, size_t{copy} * 4, cudaMemcpyDeviceToHost),
                    "readback");
}

sk_status sk_read_tile_lists(sk_context* handle, uint32_t* ranges, uint32_t* values,
                             uint32_t capacity, uint32_t* count) {
  SK_CTX(handle);
  sk_status st = ctx->finishFrame(true);
  if (st != SK_OK) return st;
  const uint32_t n = std::min(ctx->lastCounters.instances, ctx->scratchOf(ctx->lastSlot).instanceCapacity);
  if (count) *count = n;
  cudaError_t e = cudaSuccess;
  const size_t bins = size_t{(ctx->width + sk::kBinSize - 1) / sk::kBinSize} *
                      ((ctx->height + sk::kBinSize - 1) / sk::kBinSize);
  if (ranges) e = cudaMemcpy(ranges, ctx->scratchOf(ctx->lastSlot).ranges.ptr, bins * 8, cudaMemcpyDeviceToHost);
  const uint32_t copy = std::min(n, capacity);
  if (e == cudaSuccess && values && copy)
    e = cudaMemcpy(values, ctx->scratchOf(ctx->lastSlot).instValuesSorted.ptr, size_t{copy} * 4, cudaMemcpyDeviceToHost);
  return ctx->check(e, "readback");
}

size_t sk_sort_workspace_bytes(uint32_t capacity) { return sk::sortWorkspaceBytes(capacity); }

sk_status sk_radix_argsort_device(const uint32_t* d_keys, const uint32_t* d_count,
                                  uint32_t capacity, int32_t bits, uint32_t* d_order,
                                  void* d_workspace, size_t workspaceBytes, uint32_t* d_error,
                                  void* stream) {
  if (!d_keys || !d_count || !d_order || !d_workspace || !d_error) return SK_E_INVALID;
  if (bits != 16 && bits != 32) return SK_E_INVALID;
  if (workspaceBytes < sk::sortWorkspaceBytes(capacity)) return SK_E_INVALID;
  static std::atomic<uint32_t> epochs{1};
  sk::SortArgs a{};
  a.keysIn = d_keys;
  a.valuesIn = nullptr;
  a.keysOut = nullptr;
  a.valuesOut = d_order;
  a.count = d_count;
  a.capacity = capacity;
  a.bits = bits;
  sk::sortBindWorkspace(a, d_workspace, capacity);
  a.epoch = epochs.fetch_add(4) & 0x3fffffffu;
  a.error = d_error;
  const auto s = static_cast<cudaStream_t>(stream);
  // Counters and histogram accumulators start at zero; status words carry the epoch.
  cudaError_t e = sk::sortResetWorkspace(a, s);
  if (e == cudaSuccess) e = sk::launchSort(a, s);
  return e == cudaSuccess ? SK_OK : SK_E_DEVICE;
}

}  // extern "C"

extern "C" {

sk_status sk_upload_labels(sk_context* handle, uint32_t offset, const uint16_t* labels, uint32_t count) {
  SK_CTX(handle);
  if (!labels || !ctx->world.splats.ptr || ctx->world.lod || offset > ctx->world.count ||
      count > ctx->world.count - offset)
    return ctx->fail(SK_E_INVALID, "labels need a flat world and a range inside it");
  sk_status st = ctx->finishFrame(true);
  if (st == SK_E_DEVICE) return st;
  const bool fresh = ctx->labels.ptr == nullptr;
  cudaError_t e = ctx->labels.allocate(size_t{ctx->world.count} * 2);
  if (e == cudaSuccess && fresh) e = cudaMemset(ctx->labels.ptr, 0, ctx->labels.bytes);
  if (e == cudaSuccess && count)
    e = cudaMemcpy(static_cast<uint16_t*>(ctx->labels.ptr) + offset, labels, size_t{count} * 2,
                   cudaMemcpyHostToDevice);
  return ctx->check(e, "labels");
}

sk_status sk_set_part_styles(sk_context* handle, const sk_part_style* palette, const uint32_t* states,
                             uint32_t state_count) {
  SK_CTX(handle);
  if (state_count > 65536 || (state_count && (!palette || !states)))
    return ctx->fail(SK_E_INVALID, "part styles: palette and states required");
  for (uint32_t i = 0; i < state_count; ++i)
    if (states[i] >= sk::kPartStyles) return ctx->fail(SK_E_INVALID, "a state names no palette entry");
  sk_status st = ctx->finishFrame(true);
  if (st == SK_E_DEVICE) return st;
  if (state_count == 0) {
    ctx->styleStateCount = 0;
    return SK_OK;
  }
  static_assert(sizeof(sk_part_style) == sizeof(sk::PartStyle), "PartStyle layout");
  cudaError_t e = ctx->stylePalette.allocate(sk::kPartStyles * sizeof(sk::PartStyle));
  if (e == cudaSuccess) e = ctx->styleStateTable.allocate(size_t{state_count} * 4);
  if (e == cudaSuccess)
    e = cudaMemcpy(ctx->stylePalette.ptr, palette, sk::kPartStyles * sizeof(sk::PartStyle),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(ctx->styleStateTable.ptr, states, size_t{state_count} * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return ctx->check(e, "part styles");
  ctx->styleStateCount = state_count;
  return SK_OK;
}

}  // extern "C"
