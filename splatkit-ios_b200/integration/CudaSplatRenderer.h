// CudaSplatRenderer: the reference engine's renderer interface
// (packages/splatkit-engine/include/splatkit/rendering/SplatRenderer.h:36-160) implemented over
// this project's C ABI (include/splatkit_b200.h), for a maintainer who adds a CUDA backend to the
// engine beside its Metal (iOS) and Vulkan (Android) ones. Header-only; it compiles against the
// engine's own headers and links against libsplatkit_b200.so.
//
// The target is headless: the surface verbs (render scale, vsync, linear blending, present
// times) keep their state but have no display behind them; readImage() takes the place of the
// Metal renderer's captureNextFrame (splatkit-ios/.../metal/MetalSplatRenderer.mm:310-316).
#pragma once

#include <cmath>
#include <cstdint>
#include <optional>
#include <string>
#include <vector>

#include "splat/formats/SplatCloud.h"
#include "splat/lod/LodTree.h"
#include "splatkit/rendering/RenderPolicy.h"
#include "splatkit/rendering/SplatRenderer.h"
#include "splatkit_b200.h"

namespace splatkit {

class CudaSplatRenderer final : public SplatRenderer {
 public:
  CudaSplatRenderer(int device, uint32_t width, uint32_t height) : surface_{width, height} {
    sk_config config{device, width, height, SK_FORMAT_RGBA8, 1u};
    if (sk_create(&config, &ctx_) != SK_OK) ctx_ = nullptr;
  }
  ~CudaSplatRenderer() override { sk_destroy(ctx_); }
  CudaSplatRenderer(const CudaSplatRenderer&) = delete;
  CudaSplatRenderer& operator=(const CudaSplatRenderer&) = delete;

  // ---- surface (headless) ----
  void setRenderScale(float scale) override {
    scale_ = std::fmin(2.0f, std::fmax(0.1f, scale));
    const Extent e = drawExtent();
    if (ctx_ && sk_resize(ctx_, e.width, e.height) == SK_OK) ++generation_;
  }
  float renderScale() const override { return scale_; }
  void setLinearBlending(bool) override {}  // blends in the encoded space only
  bool linearBlending() const override { return false; }
  void setVsync(bool vsync) override { vsync_ = vsync; }
  bool ready() const override { return ctx_ != nullptr; }
  Extent drawExtent() const override {
    return {static_cast<uint32_t>(std::lround(surface_.width * scale_)),
            static_cast<uint32_t>(std::lround(surface_.height * scale_))};
  }
  uint32_t generation() const override { return generation_; }

  // ---- capabilities and policy ----
  DeviceCapabilities deviceCapabilities() const override {
    DeviceCapabilities caps;
    sk_capabilities c{};
    if (!ctx_ || sk_device_capabilities(ctx_, &c) != SK_OK) return caps;
    caps.limits.maxLodCapacitySplats = c.max_lod_capacity_splats;
    caps.limits.minResidencyCapacitySplats = c.min_residency_capacity_splats;
    caps.limits.maxResidencyCapacitySplats = c.max_residency_capacity_splats;
    caps.supportsSubgroups = c.supports_subgroups != 0;
    caps.maxTextureDimension = c.max_texture_dimension;
    caps.policy.lodErrorPixels = caps.policy.lodSplatLimit = true;
    caps.policy.subpixelThreshold = caps.policy.enableFrustumCulling = true;
    caps.policy.enableEarlyTermination = caps.policy.sortDepth = true;
    caps.policy.backgroundColor = true;
    return caps;
  }
  bool applyRenderPolicy(const RenderPolicy& p, std::string* reason) override {
    sk_policy q{};
    q.lod_error_pixels = p.lodErrorPixels;
    q.lod_splat_limit = p.lodSplatLimit;
    q.alpha_threshold = p.alphaThreshold;
    q.subpixel_threshold = p.subpixelThreshold;
    q.enable_frustum_culling = p.enableFrustumCulling ? 1u : 0u;
    q.enable_early_termination = p.enableEarlyTermination ? 1u : 0u;
    q.sort_depth_bits = static_cast<uint32_t>(p.sortDepth);
    for (int i = 0; i < 3; ++i) q.background[i] = p.backgroundColor[i];
    const bool ok = ctx_ && sk_apply_render_policy(ctx_, &q) == SK_OK;
    if (reason) *reason = ok ? std::string() : std::string(sk_last_error(ctx_));
    return ok;
  }
  std::optional<std::uint64_t> availableMemory() const override {
    uint64_t bytes = 0;
    if (!ctx_ || sk_available_memory(ctx_, &bytes) != SK_OK) return std::nullopt;
    return bytes;
  }
  bool gpuFailed() override { return !ctx_ || sk_gpu_failed(ctx_) != 0; }
  bool hasCompletedWorldFrame() override { return world().has_value() && completedFrames() > 0; }

  // ---- worlds ----
  bool uploadWorld(const splat::SplatCloud& cloud, int maxShDegree) override {
    const sk_cloud_view v = view(cloud);
    return ctx_ && sk_upload_world(ctx_, &v, maxShDegree) == SK_OK;
  }
  bool selectsLodOnGpu() const override { return true; }
  bool uploadLodWorld(const splat::LodTree& tree, int maxShDegree, uint32_t budget) override {
    static_assert(sizeof(splat::LodNode) == sizeof(sk_lod_node), "LodNode layout");
    static_assert(sizeof(splat::LodCluster) == sizeof(sk_lod_cluster), "LodCluster layout");
    sk_lod_view t{};
    t.nodes = view(tree.nodes);
    t.layout = reinterpret_cast<const sk_lod_node*>(tree.layout.data());
    t.node_count = static_cast<uint32_t>(tree.layout.size());
    t.leaf_count = static_cast<uint32_t>(tree.leafCount);
    t.clusters = reinterpret_cast<const sk_lod_cluster*>(tree.selection.clusters.data());
    t.cluster_count = static_cast<uint32_t>(tree.selection.clusters.size());
    t.leaves = tree.selection.leaves.data();
    t.leaf_ref_count = static_cast<uint32_t>(tree.selection.leaves.size());
    return ctx_ && sk_upload_lod_world(ctx_, &t, maxShDegree, budget) == SK_OK;
  }
  bool createSlab(uint32_t capacity, int shDegree) override {
    return ctx_ && sk_create_slab(ctx_, capacity, shDegree) == SK_OK;
  }
  bool uploadTile(uint32_t offset, const splat::SplatCloud& cloud) override {
    const sk_cloud_view v = view(cloud);
    return ctx_ && sk_upload_tile(ctx_, offset, &v) == SK_OK;
  }
  std::optional<GpuWorldInfo> world() const override {
    uint32_t count = 0;
    int32_t degree = 0;
    if (!ctx_ || sk_world_info(ctx_, &count, &degree) != SK_OK) return std::nullopt;
    return GpuWorldInfo{count, degree};
  }

  // ---- frames ----
  bool sortsOnGpu() const override { return true; }
  bool draw(const Frame& frame) override {
    if (!ctx_ || frame.orderSource != OrderSource::gpu) return false;
    static_assert(sizeof(Range) == sizeof(sk_range), "Range layout");
    sk_frame f{};
    for (int i = 0; i < 16; ++i) f.view[i] = frame.view.m[i], f.proj[i] = frame.proj.m[i];
    f.camera_position[0] = frame.cameraPosition.x;
    f.camera_position[1] = frame.cameraPosition.y;
    f.camera_position[2] = frame.cameraPosition.z;
    f.reveal_level = frame.reveal.level;
    f.reveal_band = frame.reveal.band;
    f.reveal_tint_amount = frame.reveal.tintAmount;
    f.reveal_brightness_boost = frame.reveal.brightnessBoost;
    for (int j = 0; j < 3; ++j) f.reveal_tint[j] = frame.reveal.tint[j];
    f.ranges = reinterpret_cast<const sk_range*>(frame.ranges);
    f.range_count = frame.rangeCount;
    f.sh_degree = frame.shDegree;
    return sk_draw(ctx_, &f) == SK_OK;
  }
  uint64_t submittedFrames() const override { return stats().submitted_frames; }
  uint64_t completedFrames() override { return stats().completed_frames; }
  double lastGpuMillis() const override { return stats().gpu_ms; }
  double lastSortMillis() const override { return stats().sort_ms; }
  double lastCullMillis() const override { return stats().cull_ms; }
  uint32_t lastDrawCount() const override { return stats().draw_count; }
  uint32_t lastSelectedCount() const override { return stats().selected_count; }
  double lastSelectMillis() const override { return stats().select_ms; }
  const std::string& deviceDescription() const override { return description_; }

  // The last frame as RGBA8 rows, top row first (waits for it).
  bool readImage(std::vector<uint8_t>& rgba) {
    const Extent e = drawExtent();
    rgba.resize(size_t{e.width} * e.height * 4);
    return ctx_ && sk_read_image(ctx_, rgba.data(), rgba.size(), SK_FORMAT_RGBA8) == SK_OK;
  }

 private:
  static sk_cloud_view view(const splat::SplatCloud& c) {
    sk_cloud_view v{};
    v.positions = c.positions.data();
    v.covariances = c.covariances.data();
    v.colors = c.colors.data();
    v.alphas = c.alphas.data();
    v.sh = c.sh.empty() ? nullptr : c.sh.data();
    v.count = static_cast<uint32_t>(c.count());
    v.sh_degree = c.shDegree;
    return v;
  }
  sk_stats stats() const {
    sk_stats s{};
    if (ctx_) sk_get_stats(ctx_, &s);
    return s;
  }

  sk_context* ctx_ = nullptr;
  Extent surface_;
  float scale_ = 1.0f;
  bool vsync_ = true;
  uint32_t generation_ = 0;
  std::string description_ = "CUDA sm_100a (splatkit_b200)";
};

}  // namespace splatkit
