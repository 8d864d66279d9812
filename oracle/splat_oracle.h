// Test infrastructure only — the CPU oracle for the splat frame path.
//
// This is a restatement, in plain C++, of the reference's per-frame shader math. The
// reference runs it only as Metal shaders; the restatement follows them line by line:
//   cull + projection + SH      splatkit-ios/.../metal/layout/SplatProjection.metalh:6-141
//   depth keys + compaction     splatkit-ios/.../metal/cull/SplatVisibility.metal:16-106
//   constants                   splatkit-ios/.../metal/layout/SplatTypes.metalh:81-118,
//                               splatkit-ios/.../metal/layout/MetalShaderTypes.h:35
//   radix sort (the contract)   splatkit-ios/.../metal/sort/MetalRadixSort.h:13-19 and its
//                               test oracle, std::stable_sort (MetalRadixSortTest.mm:58-62)
//   LOD cut rounds              splatkit-ios/.../metal/selection/SplatLOD.metal:26-220,
//                               host MetalLodSelection.mm:109-192
//   composite equations         splatkit-ios/.../metal/raster/SplatRaster.metal:27-44,
//                               SplatProjection.metalh:143-175, MetalSplatPipeline.mm:46-71,153-161
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg may load it. The product
// never links or calls it.
//
// Arithmetic contract shared with the CUDA kernels (so that cull, keys, sort and LOD cut are
// bit-exact): IEEE binary32, every product and sum rounded on its own (no FMA), IEEE divide
// and sqrt, fmin/fmax NaN semantics, sums in the order written in splat_oracle.cpp, a
// project-owned natural log (ln_f32) and a project-owned float->half conversion with the
// reference's Half.h semantics (round to nearest even, saturate to 65504, NaN stays NaN).
#pragma once
#include <cstddef>
#include <cstdint>

extern "C" {

// 32-byte world record (engine/include/splatkit/rendering/GpuLayout.h:50-56).
typedef struct {
  float position[3];
  uint32_t rgba8;
  uint32_t cov[3];  // halves (xx, xy), (xz, yy), (yz, zz), low half first
  uint32_t lodAlpha;
} sko_splat;

// 32-byte projected record (engine/include/splatkit/rendering/GpuLayout.h:60-70).
typedef struct {
  float center[2];
  uint32_t axis1, axis2, color0, color1;
  float radius;
  uint32_t index;
} sko_projected;

// The per-view uniform (metal/layout/SplatTypes.metalh:7-22), 208 bytes.
typedef struct {
  float view[16];  // column major: m[col * 4 + row]
  float proj[16];
  float focal[2];
  float tanHalfFov[2];
  float screenSize[2];
  uint32_t outputLinear;
  float minPixelRadius;
  float cameraPosition[4];
  float reveal[4];  // x: reveal level (+inf when idle)
  float revealTint[4];
} sko_camera;

// Interior LOD cluster (core/include/splat/lod/LodTree.h:28-35), 64 bytes.
typedef struct {
  float center[3], radius;
  float extent[3], error;
  float colorVariance, opacity;
  uint32_t node, childStart, childCount, leafStart, leafCount, subtreeLeaves;
} sko_cluster;

typedef struct {
  uint32_t offset, count;
} sko_range;

// Fills the uniform the way MetalFrameCompute::updateCamera does (MetalFrameCompute.mm:141-164).
void sko_camera_make(const float* view16, const float* proj16, const float* cameraPosition3,
                     uint32_t width, uint32_t height, float minPixelRadius, sko_camera* out);

// Project-owned numerics, exported so tests can pin them.
float sko_ln(float x);
uint16_t sko_float_to_half(float x);
float sko_half_to_float(uint16_t h);

// Cull + project + SH + depth key of one splat. Returns 1 when it survives.
int sko_project_one(const sko_camera* cam, const sko_splat* splat, uint32_t index,
                    const uint32_t* sh, uint32_t shStride, int shDegree, int keyBits,
                    uint32_t* keyOut, sko_projected* out);

// The visibility pass over ranges (or, when `indices` is not null, over indices[0..indexCount)),
// survivors compacted in source order. Returns the survivor count. `threads` > 1 splits the
// source range over std::threads; the output is identical.
// Part labels and styles (metal/cull/SplatVisibility.metal:4-12,69-84): palette of 10 entries of
// 8 floats (tint rgb, tint amount, brightness, opacity, 2 reserved), states[label] < 10.
typedef struct {
  const uint16_t* labels;
  const float* palette;
  const uint32_t* states;
  uint32_t stateCount;
} sko_parts;

// parts null: no part styling. The reveal glow follows the camera's reveal fields.
uint32_t sko_visibility(const sko_camera* cam, const sko_splat* splats, const uint32_t* sh,
                        uint32_t shStride, int shDegree, int keyBits, const sko_range* ranges,
                        uint32_t rangeCount, const uint32_t* indices, uint32_t indexCount,
                        uint32_t* keysOut, sko_projected* projectedOut, int threads,
                        const sko_parts* parts);

// Stable ascending argsort: std::stable_sort of (key, position) pairs.
void sko_stable_argsort(const uint32_t* keys, uint32_t n, uint32_t* orderOut);
// The same order by an LSD counting sort with 8-bit digits over `bits` (16 or 32) key bits,
// in the style of core/src/sorting/SpatialOrder.cpp:57-82; multi-threaded histograms and
// scatter when threads > 1.
void sko_radix_argsort(const uint32_t* keys, uint32_t n, int bits, uint32_t* orderOut, int threads);

// The LOD cut (SplatLOD.metal rounds, simulated in order). stats: count, active, packets,
// accepted, limited, evaluated. Returns the number of indices written (min(count, capacity)).
uint32_t sko_lod_select(const sko_camera* cam, const sko_cluster* clusters, uint32_t clusterCount,
                        const uint32_t* leaves, uint32_t rounds, uint32_t capacity,
                        float pixelLimit, float colorWeight, uint32_t cull, uint32_t* indicesOut,
                        uint32_t* stats6);

// Front-to-back composite of `count` projected records in `order`, W x H, RGBA, row 0 on
// top. precision 64: the FP64 evaluation the kernels are checked against; 32: the same in
// FP32 (the CPU baseline). Coverage decisions (quad bound, 1/255 cutoff) use the FP32
// formula the kernel uses, so both sides agree on each splat's support.
// `opaque`: 1 puts the background under the remainder (alpha 1); 0 leaves coverage in alpha.
void sko_composite(const sko_projected* projected, const uint32_t* order, uint32_t count,
                   uint32_t width, uint32_t height, const float* background3, int opaque,
                   float transmittanceCutoff, int precision, float* rgbaOut, int threads);

// Counts composited fragments the way the kernel does (pixel x splat pairs evaluated
// before each pixel terminates).
uint64_t sko_composite_fragments(const sko_projected* projected, const uint32_t* order,
                                 uint32_t count, uint32_t width, uint32_t height,
                                 float transmittanceCutoff, int threads);

// std::mt19937 output (used to rebuild the reference tests' random keys).
void sko_mt19937(uint32_t seed, uint32_t n, uint32_t* out);
}
