// Direct cell-major lists: each binning cell's front-to-back list of survivors, written in place.
//
// Binning + a stable sort of (cell, projected index) pairs by cell + a ranges pass build the
// same lists (binning.cu, radix_sort.cu). On a target of at most kDirectMaxCells cells this file
// builds them without the sort:
//   1. count: every block of 512 depth ranks (1024 in a batch) histograms its instances by cell;
//   2. scan: per cell, the running sum of the block histograms (32 cells per block of this pass,
//      the rows held in registers) gives each block's first slot in the cell's list; the lists'
//      starts come from a decoupled look-back across the groups of 32 cells, in cell order; the
//      ranges and the instance count follow;
//   3. emit: every block histograms its 8 warps' ranks (128 each) by cell again, so that warp w
//      starts each cell after warps 0..w-1, then each warp walks its output 32 entries at a time
//      in depth order and writes each entry at its cell's next slot (lanes of one round that
//      share a cell take consecutive slots).
// A batch of views runs each pass once for all of them (launchCellListsBatch): every block finds
// its view in a table (its first count/emit block and first cell group), works on that view's
// ranks, cells and workspace rows, and the look-back of pass 2 runs over the groups of all views
// in order, so each view's entries start where the previous view's end.
// Entries of a cell therefore appear in depth order, which is exactly what the stable sort
// gives.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "sk_device.cuh"
#include "sk_kernels.h"
#include "sk_launch.cuh"
#include "sk_tiles.cuh"

namespace sk {
namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kWarps = kThreads / 32;
// Ranks per lane: a frame's blocks take 512 depth ranks (100.8 -> 81.8 us for the three passes
// against 1024-rank blocks), a batch's 1024 (it holds every view's block rows at once, and twice
// the rows cost the 64-view batch more than the smaller blocks save).
constexpr uint32_t kFrameItems = 2;
constexpr uint32_t kBatchItems = 4;
constexpr uint32_t kScanThreads = 1024;
constexpr uint32_t kScanWarps = kScanThreads / 32;
constexpr uint32_t kRowsInRegisters = 32;         // block rows one scan warp keeps

struct Work {
  uint32_t* blockRows;  // blocks x cells: each block's count per cell, then (after pass 2) its
                        // first slot in each cell's list
  uint64_t* status;     // one look-back word per group of 32 cells
  // a whole batch in one launch (views non-null): the view table, each view's ranks
  // [viewFirst[v], viewFirst[v + 1]) of args.order, and the workspace its rows are in
  const CellListView* views;
  uint32_t viewCount;
  const uint32_t* viewFirst;
  uint8_t* base;
};

// What one block of a pass works on: its block (or cell group) within its view, the view's ranks
// [first, first + n) of the depth order, cells, workspace rows and cell ranges.
struct Job {
  uint32_t block, first, n, cells, tilesX;
  uint32_t* blockRows;
  uint2* ranges;
};

__host__ __device__ inline uint32_t cellWords(uint32_t cells) { return (cells + 1) / 2; }
__host__ __device__ inline size_t align16(size_t n) { return (n + 15) & ~size_t{15}; }
__host__ __device__ inline uint32_t cellGroups(uint32_t cells) { return (cells + 31) / 32; }
template <uint32_t kItems>
__host__ __device__ inline uint32_t blocksFor(uint32_t capacity) {
  constexpr uint32_t kBlockRanks = kThreads * kItems;
  return (capacity + kBlockRanks - 1) / kBlockRanks;
}

// The job of block (or cell group, byGroup) `index` of a pass.
__device__ __forceinline__ Job jobOf(const BinArgs& a, const Work& w, uint32_t cells,
                                     uint32_t index, bool byGroup, uint2* ranges) {
  Job j;
  if (!w.views) {  // a frame: the ranks [0, count) of the depth order
    j.block = index;
    j.first = 0;
    j.n = min(*a.count, a.capacity);
    j.cells = cells;
    j.tilesX = a.tilesX;
    j.blockRows = w.blockRows;
    j.ranges = ranges;
    return j;
  }
  uint32_t lo = 0, hi = w.viewCount;  // the last view whose first block (group) is <= index
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    const uint32_t start = byGroup ? w.views[mid].groupBase : w.views[mid].blockBase;
    if (start <= index) lo = mid; else hi = mid;
  }
  const CellListView v = w.views[lo];
  j.block = index - (byGroup ? v.groupBase : v.blockBase);
  j.first = w.viewFirst[lo];
  j.n = min(w.viewFirst[lo + 1] - j.first, v.capacity);
  j.cells = v.cells;
  j.tilesX = v.tilesX;
  j.blockRows = reinterpret_cast<uint32_t*>(w.base + v.work);
  j.ranges = ranges + v.binBase;
  return j;
}

__host__ __device__ inline Work workOf(void* workspace, uint32_t blocks, uint32_t cells) {
  uint8_t* p = static_cast<uint8_t*>(workspace);
  Work w{};
  w.blockRows = reinterpret_cast<uint32_t*>(p);
  p += align16(size_t{blocks} * cells * 4);
  w.status = reinterpret_cast<uint64_t*>(p);
  return w;
}

size_t workBytes(uint32_t blocks, uint32_t cells) {
  return align16(size_t{blocks} * cells * 4) + size_t{cellGroups(cells)} * 8;
}

// Pass 1: each block's instances per cell.
template <uint32_t kItems>
__global__ void __launch_bounds__(kThreads)
    cellCountKernel(const __grid_constant__ BinArgs a, Work work, uint32_t cells) {
  constexpr uint32_t kBlockRanks = kThreads * kItems;
  chainedKernelStart();
  __shared__ uint32_t hist[kDirectMaxCells];
  const Job job = jobOf(a, work, cells, blockIdx.x, false, nullptr);
  const uint32_t n = job.n;
  cells = job.cells;
  const uint32_t* order = a.order + job.first;
  const uint32_t begin = job.block * kBlockRanks;
  if (begin >= n) return;  // rows of idle blocks are never read
  for (uint32_t c = threadIdx.x; c < cells; c += kThreads) hist[c] = 0;
  __syncthreads();
  uint32_t value[kItems];
  uint4 span[kItems];
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    const uint32_t i = begin + r * kThreads + threadIdx.x;
    value[r] = i < n ? order[i] : 0xffffffffu;
  }
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r)
    span[r] = value[r] != 0xffffffffu ? __ldg(a.spans + value[r]) : make_uint4(0, 0, 0, 0);
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r)
    visitCells(span[r], job.tilesX, [](uint32_t c) { atomicAdd(&hist[c], 1u); });
  __syncthreads();
  uint32_t* row = job.blockRows + size_t{job.block} * cells;
  for (uint32_t c = threadIdx.x; c < cells; c += kThreads) row[c] = hist[c];
}

// Pass 2: one block per group of 32 cells (groups handed out in start order, so a group only
// waits on groups already running). Lane = cell of the group; warp w scans a contiguous share
// of the block rows, the first 32 of them kept in registers between the two sweeps.
template <uint32_t kItems>
__global__ void __launch_bounds__(kScanThreads, 1)
    cellScanKernel(const __grid_constant__ BinArgs a, Work work, uint32_t cells, uint2* ranges,
                   uint32_t* counters, uint32_t epoch, uint32_t* error) {
  chainedKernelStart();
  __shared__ uint32_t part[kScanWarps][33];
  __shared__ uint32_t cellStart[32];
  const uint32_t group = takeTile(counters);  // over all views of a batch
  const Job job = jobOf(a, work, cells, group, true, ranges);
  cells = job.cells;
  const uint32_t active = blocksFor<kItems>(job.n);
  const uint32_t warp = threadIdx.x >> 5, lane = laneId();
  const uint32_t cell = job.block * 32 + lane;
  const bool valid = cell < cells;
  const uint32_t share = (active + kScanWarps - 1) / kScanWarps;
  const uint32_t r0 = min(warp * share, active), r1 = min(r0 + share, active);
  uint32_t* rows = job.blockRows + cell;
  uint32_t v[kRowsInRegisters];
  uint32_t sum = 0;
#pragma unroll
  for (uint32_t k = 0; k < kRowsInRegisters; ++k) {
    const uint32_t row = r0 + k;
    v[k] = valid && row < r1 ? __ldcg(rows + size_t{row} * cells) : 0u;
    sum += v[k];
  }
  if (valid)
    for (uint32_t row = r0 + kRowsInRegisters; row < r1; ++row)
      sum += __ldcg(rows + size_t{row} * cells);
  part[warp][lane] = sum;
  __syncthreads();
  uint32_t run = 0;
  for (uint32_t w = 0; w < warp; ++w) run += part[w][lane];
  if (warp == 0) {
    uint32_t total = 0;
    for (uint32_t w = 0; w < kScanWarps; ++w) total += part[w][lane];
    uint32_t inc = total;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= static_cast<uint32_t>(o)) inc += up;
    }
    const uint32_t aggregate = __shfl_sync(0xffffffffu, inc, 31);
    uint32_t before = 0;
    if (group == 0) {
      if (lane == 0) storeStatus(work.status, makeStatus(epoch, kFlagPrefix, aggregate));
    } else {
      if (lane == 0) storeStatus(work.status + group, makeStatus(epoch, kFlagAggregate, aggregate));
      before = warpLookback(work.status, group, epoch, error);
      if (lane == 0)
        storeStatus(work.status + group, makeStatus(epoch, kFlagPrefix, before + aggregate));
    }
    const uint32_t start = before + inc - total;
    cellStart[lane] = start;
    if (valid)
      job.ranges[cell] = make_uint2(min(start, a.instanceCapacity),
                                    min(start + total, a.instanceCapacity));
    if (group == gridDim.x - 1 && lane == 31) {
      const uint32_t entries = before + aggregate;
      *a.instanceCount = entries;
      *a.overflow = entries > a.instanceCapacity ? 1u : 0u;
    }
  }
  __syncthreads();
  if (valid) {  // each count becomes the block's first slot in the cell, in place
    run += cellStart[lane];
#pragma unroll
    for (uint32_t k = 0; k < kRowsInRegisters; ++k) {
      const uint32_t row = r0 + k;
      if (row < r1) rows[size_t{row} * cells] = run;
      run += v[k];
    }
    for (uint32_t row = r0 + kRowsInRegisters; row < r1; ++row) {
      const uint32_t count = __ldcg(rows + size_t{row} * cells);
      rows[size_t{row} * cells] = run;
      run += count;
    }
  }
  finishTile(counters);
}

// visit(cell, position, item) for every cell of the warp's items whose position offset + k lies
// in [lo, hi); k numbers a span's cells as spanCell does (mask bits upward, or box order), item
// is itemBase + the owning lane. A masked span is walked by its own lane, a box of more than 64
// cells by the whole warp. Every lane calls this.
template <typename Visit>
__device__ __forceinline__ void visitPositions(const uint4 s, uint32_t tilesX, uint32_t offset,
                                               uint32_t lo, uint32_t hi, uint32_t itemBase,
                                               Visit visit) {
  const uint32_t w = s.y & 0xffffu, area = s.y >> 16;
  const uint32_t first = spanFirstCell(s, tilesX);
  const uint32_t lane = laneId();
  if (area <= 64 && offset < hi && offset + __popc(s.z) + __popc(s.w) > lo) {
    uint32_t pos = offset;
    for (uint32_t m = s.z; m != 0u; m &= m - 1, ++pos)
      if (pos >= lo && pos < hi) visit(boxCell(first, __ffs(m) - 1, w, tilesX), pos, itemBase + lane);
    for (uint32_t m = s.w; m != 0u; m &= m - 1, ++pos)
      if (pos >= lo && pos < hi) visit(boxCell(first, 31 + __ffs(m), w, tilesX), pos, itemBase + lane);
  }
  uint32_t big = __ballot_sync(0xffffffffu, area > 64 && offset < hi && offset + area > lo);
  while (big != 0u) {
    const uint32_t src = __ffs(big) - 1;
    big &= big - 1;
    const uint32_t bw = __shfl_sync(0xffffffffu, w, src);
    const uint32_t barea = __shfl_sync(0xffffffffu, area, src);
    const uint32_t bfirst = __shfl_sync(0xffffffffu, first, src);
    const uint32_t boff = __shfl_sync(0xffffffffu, offset, src);
    const uint32_t k0 = lo > boff ? lo - boff : 0u, k1 = min(barea, hi - boff);
    for (uint32_t k = k0 + lane; k < k1; k += 32) visit(boxCell(bfirst, k, bw, tilesX), boff + k, itemBase + src);
  }
}

// Pass 3. Dynamic shared memory: kWarps x words per-warp slot counters (16-bit halves: a warp's
// slots count from the block's first slot in the cell, at most 1024 on), then each cell's first
// slot for the block. A warp's entries, in depth order, are staged as (cell, item) pairs kWindow
// positions at a time: the counting walk stages the first window, and a warp with more entries
// walks its items again for each further one.
constexpr uint32_t kWindow = 1024;

template <uint32_t kItems>
__global__ void __launch_bounds__(kThreads)
    cellEmitKernel(const __grid_constant__ BinArgs a, Work work, uint32_t cells) {
  constexpr uint32_t kChunk = 32 * kItems;  // ranks per warp
  constexpr uint32_t kBlockRanks = kThreads * kItems;
  chainedKernelStart();
  extern __shared__ uint32_t cellSmem[];
  __shared__ uint32_t stageValue[kWarps][kChunk];
  __shared__ uint16_t stageCell[kWarps][kWindow];
  __shared__ uint8_t stageItem[kWarps][kWindow];
  const Job job = jobOf(a, work, cells, blockIdx.x, false, nullptr);
  const uint32_t n = job.n, tilesX = job.tilesX;
  cells = job.cells;
  const uint32_t* order = a.order + job.first;
  const uint32_t begin = job.block * kBlockRanks;
  if (begin >= n) return;
  const uint32_t words = cellWords(cells);
  uint32_t* slots = cellSmem;
  uint32_t* where = cellSmem + kWarps * words;
  for (uint32_t i = threadIdx.x; i < kWarps * words; i += kThreads) slots[i] = 0;
  const uint32_t* starts = job.blockRows + size_t{job.block} * cells;
  for (uint32_t c = threadIdx.x; c < cells; c += kThreads) where[c] = __ldcg(starts + c);
  __syncthreads();

  const uint32_t warp = threadIdx.x >> 5, lane = laneId();
  uint32_t* mine = slots + warp * words;
  uint32_t* sValue = stageValue[warp];
  uint16_t* sCell = stageCell[warp];
  uint8_t* sItem = stageItem[warp];
  uint32_t value[kItems];
  uint4 span[kItems];
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    const uint32_t i = begin + warp * kChunk + r * 32 + lane;
    value[r] = i < n ? order[i] : 0xffffffffu;
  }
  // the warp's items in (row, lane) order = depth order, with their first output position
  uint32_t offset[kItems];
  uint32_t total = 0;
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    span[r] = value[r] != 0xffffffffu ? __ldg(a.spans + value[r]) : make_uint4(0, 0, 0, 0);
    sValue[r * 32 + lane] = value[r];
    const uint32_t cnt = spanCount(span[r]);
    uint32_t inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t up = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= static_cast<uint32_t>(o)) inc += up;
    }
    offset[r] = total + inc - cnt;
    total += __shfl_sync(0xffffffffu, inc, 31);
  }
  // count every entry by cell; stage the first window
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r)
    visitPositions(span[r], tilesX, offset[r], 0u, 0xffffffffu, r * 32,
                   [mine, sCell, sItem](uint32_t c, uint32_t pos, uint32_t item) {
                     atomicAdd(mine + (c >> 1), 1u << ((c & 1u) * 16));
                     if (pos < kWindow) {
                       sCell[pos] = static_cast<uint16_t>(c);
                       sItem[pos] = static_cast<uint8_t>(item);
                     }
                   });
  __syncthreads();
  // warp w's first slot per cell: the counts of warps 0..w-1 (both halves of a word at once)
  for (uint32_t q = threadIdx.x; q < words; q += kThreads) {
    uint32_t run = 0;
#pragma unroll
    for (uint32_t w = 0; w < kWarps; ++w) {
      const uint32_t v = slots[w * words + q];
      slots[w * words + q] = run;
      run += v;
    }
  }
  __syncthreads();

  const uint32_t below = lanemaskLt();
  for (uint32_t w0 = 0; w0 < total; w0 += kWindow) {
    const uint32_t w1 = min(total, w0 + kWindow);
    if (w0 > 0) {  // stage the next window (its spans re-read from L2)
      __syncwarp();
#pragma unroll
      for (uint32_t r = 0; r < kItems; ++r) {
        const uint4 sp = value[r] != 0xffffffffu ? __ldg(a.spans + value[r]) : make_uint4(0, 0, 0, 0);
        visitPositions(sp, tilesX, offset[r], w0, w1, r * 32,
                       [sCell, sItem, w0](uint32_t c, uint32_t pos, uint32_t item) {
                         sCell[pos - w0] = static_cast<uint16_t>(c);
                         sItem[pos - w0] = static_cast<uint8_t>(item);
                       });
      }
    }
    __syncwarp();
    for (uint32_t p0 = w0; p0 < w1; p0 += 32) {
      const uint32_t p = p0 + lane;
      const bool valid = p < w1;
      uint32_t cell = 0xffffffffu, val = 0;
      if (valid) {
        cell = sCell[p - w0];
        val = sValue[sItem[p - w0]];
      }
      // lanes of this round with the same cell: 13 ballots (cells are below 4096; an idle lane's
      // 0xffffffff differs from every cell in bit 12)
      uint32_t peers = 0xffffffffu;
#pragma unroll
      for (uint32_t b = 0; b < 13; ++b) {
        const bool bit = (cell >> b) & 1u;
        const uint32_t vote = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? vote : ~vote;
      }
      const uint32_t half = (cell & 1u) * 16;
      uint32_t slot = 0;
      if (valid) slot = where[cell] + ((mine[cell >> 1] >> half) & 0xffffu) + __popc(peers & below);
      __syncwarp();
      if (valid && lane == 31 - __clz(peers)) atomicAdd(mine + (cell >> 1), __popc(peers) << half);
      __syncwarp();
      if (valid && slot < a.instanceCapacity) a.instanceValues[slot] = val;
    }
  }
}

size_t emitDynamicBytes(uint32_t cells) {
  return (size_t{kWarps} * cellWords(cells) + cells) * sizeof(uint32_t);
}

}  // namespace

bool cellListsFit(uint32_t capacity, uint32_t cells) {
  return cells > 0 && cells <= kDirectMaxCells && capacity > 0;
}

size_t cellListBytes(uint32_t capacity, uint32_t cells) {
  return workBytes(blocksFor<kFrameItems>(std::max(capacity, 1u)), std::max(cells, 1u));
}

cudaError_t cellListsConfigure() {
  static bool configured = false;
  if (configured) return cudaSuccess;
  cudaError_t e =
      cudaFuncSetAttribute(cellEmitKernel<kFrameItems>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(emitDynamicBytes(kDirectMaxCells)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(cellEmitKernel<kBatchItems>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(emitDynamicBytes(kDirectMaxCells)));
  if (e == cudaSuccess) configured = true;
  return e;
}

cudaError_t launchCellLists(const BinArgs& a, const CellLists& lists, cudaStream_t stream) {
  const uint32_t cells = lists.cells;
  if (!cellListsFit(a.capacity, cells) || cells != a.tilesX * a.tilesY)
    return cudaErrorInvalidValue;
  cudaError_t e = cellListsConfigure();
  if (e != cudaSuccess) return e;
  const uint32_t blocks = blocksFor<kFrameItems>(a.capacity);
  const Work work = workOf(lists.workspace, blocks, cells);
  e = launchChained(cellCountKernel<kFrameItems>, blocks, kThreads, stream, a, work, cells);
  if (e != cudaSuccess) return e;
  e = launchChained(cellScanKernel<kFrameItems>, cellGroups(cells), kScanThreads, stream, a, work, cells,
                    lists.ranges, lists.counters, lists.epoch, lists.error);
  if (e != cudaSuccess) return e;
  return launchChainedShared(cellEmitKernel<kFrameItems>, blocks, kThreads, emitDynamicBytes(cells), stream, a,
                             work, cells);
}

uint32_t cellListBlocks(uint32_t capacity) { return blocksFor<kBatchItems>(std::max(capacity, 1u)); }

size_t cellListRowBytes(uint32_t capacity, uint32_t cells) {
  return align16(size_t{cellListBlocks(capacity)} * cells * 4);
}

cudaError_t launchCellListsBatch(const BinArgs& a, const CellListBatch& lists, cudaStream_t stream) {
  if (lists.viewCount == 0 || lists.blocks == 0 || lists.groups == 0 || lists.mostCells == 0 ||
      lists.mostCells > kDirectMaxCells)
    return cudaErrorInvalidValue;
  cudaError_t e = cellListsConfigure();
  if (e != cudaSuccess) return e;
  Work work{};
  work.status = lists.status;
  work.views = lists.views;
  work.viewCount = lists.viewCount;
  work.viewFirst = lists.viewFirst;
  work.base = static_cast<uint8_t*>(lists.workspace);
  const uint32_t cells = lists.mostCells;  // each block reads its own view's from the table
  e = launchChained(cellCountKernel<kBatchItems>, lists.blocks, kThreads, stream, a, work, cells);
  if (e != cudaSuccess) return e;
  e = launchChained(cellScanKernel<kBatchItems>, lists.groups, kScanThreads, stream, a, work, cells,
                    lists.ranges, lists.counters, lists.epoch, lists.error);
  if (e != cudaSuccess) return e;
  return launchChainedShared(cellEmitKernel<kBatchItems>, lists.blocks, kThreads, emitDynamicBytes(cells),
                             stream, a, work, cells);
}

}  // namespace sk
