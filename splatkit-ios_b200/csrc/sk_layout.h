// Record layouts shared by the host layer and the kernels. Sizes and field orders follow the
// reference's GPU records so that a packed world or a projected buffer means the same bytes:
//   GpuSplat, ProjectedSplat   engine/include/splatkit/rendering/GpuLayout.h:50-70
//   Camera uniform             splatkit-ios/.../metal/layout/SplatTypes.metalh:7-22,
//                              splatkit-ios/.../metal/layout/MetalShaderTypes.h:14-30
//   LodCluster                 splat-core/include/splat/lod/LodTree.h:28-35
//   LodNode                    splat-core/include/splat/lod/LodTree.h:13-23
#pragma once
#include <cstddef>
#include <cstdint>

namespace sk {

struct alignas(16) GpuSplat {
  float position[3];
  uint32_t rgba8;     // r | g << 8 | b << 16 | a << 24
  uint32_t cov[3];    // halves (xx, xy), (xz, yy), (yz, zz), low half first
  uint32_t lodAlpha;  // float bits of an opacity above 1, else 0
};
static_assert(sizeof(GpuSplat) == 32, "GpuSplat is 32 bytes");

struct alignas(16) Projected {
  float center[2];  // NDC
  uint32_t axis1;   // halves: major axis, sigma in pixels
  uint32_t axis2;   // halves: minor axis
  uint32_t color0;  // halves: r, g
  uint32_t color1;  // halves: b, peak opacity
  float radius;     // quad half width in sigma
  uint32_t index;   // source splat
};
static_assert(sizeof(Projected) == 32, "Projected is 32 bytes");
static_assert(offsetof(Projected, index) == 28, "Projected index offset");

struct alignas(16) Camera {
  float view[16];  // column major, m[col * 4 + row]
  float proj[16];
  float focal[2];       // W * P00 / 2, H * P11 / 2
  float tanHalfFov[2];  // 1 / P00, 1 / P11
  float screenSize[2];
  uint32_t outputLinear;  // always 0 here: blending happens in the encoded space
  float minPixelRadius;
  float cameraPosition[4];
  float reveal[4];  // x: reveal level; +inf when idle
  float revealTint[4];
};
static_assert(sizeof(Camera) == 208, "Camera is 208 bytes");
static_assert(offsetof(Camera, focal) == 128, "Camera focal offset");
static_assert(offsetof(Camera, minPixelRadius) == 156, "Camera cutoff offset");
static_assert(offsetof(Camera, reveal) == 176, "Camera reveal offset");

struct Range {
  uint32_t offset;
  uint32_t count;
};

// PartStyle (splatkit-ios/.../metal/cull/SplatVisibility.metal:5-11): how a labelled part is
// drawn. A world label picks a state, a state picks one of kPartStyles palette entries.
struct PartStyle {
  float tint[3];
  float tintAmount;
  float brightness;
  float opacity;
  float reserved[2];
};
static_assert(sizeof(PartStyle) == 32, "PartStyle is 32 bytes");
constexpr uint32_t kPartStyles = 10;

// Part labels of a flat world and the styles they are drawn with (all device pointers).
struct PartLabels {
  const uint16_t* labels;   // one per world record; null: no styling
  const PartStyle* palette; // kPartStyles entries
  const uint32_t* states;   // stateCount entries, each < kPartStyles
  uint32_t stateCount;
};

struct LodNode {
  float position[3];
  float size;
  uint32_t childStart;
  uint32_t childCount;
};
static_assert(sizeof(LodNode) == 24, "LodNode is 24 bytes");

struct alignas(16) LodCluster {
  float center[3], radius;
  float extent[3], error;
  float colorVariance, opacity;
  uint32_t node, childStart, childCount, leafStart, leafCount, subtreeLeaves;
};
static_assert(sizeof(LodCluster) == 64, "LodCluster is 64 bytes");

// The LOD walk's counters; the first six words are what a frame reports (count, active,
// packets, accepted, limited, evaluated), like LodState's leading fields
// (splatkit-ios/.../metal/selection/SplatLOD.metal:12-20).
struct LodState {
  uint32_t count, active, packets, accepted;
  uint32_t limited, evaluated, totalExtra, drops;
  uint32_t scatterActive, scatterCount, scatterPackets, pad;
};

// Per-frame device counters the host reads back after a frame completes.
struct FrameCounters {
  uint32_t visible;       // survivors of the cull
  uint32_t instances;     // tile instances the binning needed
  uint32_t overflow;      // 1 when instances exceeded the reserved capacity
  uint32_t error;         // SK_DEVERR_* bits
  uint32_t lod[6];        // LOD counters of this frame
  uint32_t fragments_lo;  // blended fragments (pixel x splat), when counted
  uint32_t fragments_hi;
  uint32_t loaded;  // tile-list records the composite read before its tiles terminated
  uint32_t pad[3];
};
static_assert(sizeof(FrameCounters) == 64, "FrameCounters is 64 bytes");

// Device error bits.
constexpr uint32_t SK_DEVERR_LOOKBACK = 1u;  // a look-back wait ran out of polls
constexpr uint32_t SK_DEVERR_BOUNDS = 2u;    // an index fell outside its buffer and was skipped
constexpr uint32_t SK_DEVERR_BARRIER = 4u;   // an mbarrier wait ran out of polls

// Harmonics words per splat in the device layout: the reference's packed stride
// (splatkit-engine/src/rendering/GpuLayout.cpp:66-70) rounded up to a multiple of four so each
// splat starts on a 16-byte boundary and loads as whole uint4s.
inline constexpr uint32_t shPackedStride(int degree) {
  return degree <= 0 ? 0u : static_cast<uint32_t>((((degree + 1) * (degree + 1) - 1) * 3 + 1) / 2);
}
inline constexpr uint32_t shDeviceStride(int degree) {
  return (shPackedStride(degree) + 3u) & ~3u;
}

constexpr uint32_t kTileSize = 16;  // composite tile edge in pixels
// Binning cell edge: a 2x2 block of composite tiles. Splats are listed once per cell they touch
// (about 2.6x fewer list entries than per tile at 1080p); each composite tile reads its cell's
// list and keeps, per warp quadrant, only the splats that reach it.
constexpr uint32_t kBinSize = 2 * kTileSize;

// One view of a batch (device table, 96 bytes): the world range it draws (or, for a LOD world,
// the cut its selection wrote), where its work items, tiles and pixels start in the batch-wide
// arrays, and its target size. Views are listed in submission order; itemStart, tileBase and
// pixelOffset grow with the view index.
struct alignas(16) BatchView {
  const GpuSplat* splats;
  const uint32_t* sh;
  uint32_t shStride;     // harmonics words per record of this world
  uint32_t offset;       // first record drawn
  uint32_t count;        // records drawn
  uint32_t itemStart;    // first visibility work item (1024-record chunk) of this view
  uint32_t tileBase;     // first batch-wide composite tile of this view
  uint32_t binBase;      // first batch-wide binning cell of this view
  uint32_t tilesX;       // composite tiles per row
  uint32_t binsX, binsY; // binning cells per row and column
  uint32_t width, height;
  uint64_t pixelOffset;  // first pixel of this view in the batch image
  const uint32_t* indices;     // a LOD view: its cut, the record indices to draw in emission
                               // order (null: the range offset .. offset + count)
  const uint32_t* indexCount;  // a LOD view: the cut's length (device word); count bounds it
  uint32_t worldCount;         // records of the world (every cut index is below it)
  uint32_t pad;
};
static_assert(sizeof(BatchView) == 96, "BatchView is 96 bytes");

}  // namespace sk
