// Test infrastructure only: a C ABI over the reference's own C++ (splat-core and
// splatkit-engine sources, compiled unmodified from the reference checkout by
// oracle/Makefile into oracle/_ref/libsk_ref.so). Only tests/, the smoke check and the
// CPU-baseline leg of bench.py load it; the product never does.
//
// What it exposes, by reference file:
//   packages/splat-core/include/splat/math/Half.h:12-65          toHalf / fromHalf
//   packages/splat-core/include/splat/math/Mat4.h:75-86          Mat4::perspective
//   packages/splat-core/src/math/Covariance.cpp:7-17             covarianceFromQuaternionScale
//   packages/splatkit-engine/src/camera/WalkCamera.cpp:218-227,535-537  setLookAt + viewMatrix
//   packages/splatkit-engine/src/rendering/GpuLayout.cpp:66-137  shStride, gpuWorldBytes,
//                                                                packSplatRange, packShRange
//   packages/splat-core/src/lod/LodTree.cpp:323-342              buildLodTree
//   packages/splat-core/src/lod/LodSelection.cpp:47-133          buildLodSelectionData
//   packages/splat-core/src/lod/LodFile.cpp:336-459              validateLodTree, LODSPLAT I/O
//   packages/splatkit-engine/include/splatkit/rendering/LodThreshold.h:27-36
//   packages/splatkit-engine/src/rendering/RenderPolicy.cpp:29-52  validRenderPolicy
//   packages/splat-core/src/sorting/SpatialOrder.cpp:48-92       reorderSpatially
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "splat/formats/SplatCloud.h"
#include "splat/lod/LodFile.h"
#include "splat/lod/LodTree.h"
#include "splat/math/Covariance.h"
#include "splat/math/Half.h"
#include "splat/math/Mat4.h"
#include "splat/sorting/SpatialOrder.h"
#include "splatkit/camera/WalkCamera.h"
#include "splatkit/rendering/GpuLayout.h"
#include "splatkit/rendering/LodThreshold.h"
#include "splatkit/rendering/RenderPolicy.h"

namespace {

splat::SplatCloud cloudFrom(const float* positions, const float* covariances, const float* colors,
                            const float* alphas, const float* sh, size_t n, int shDegree,
                            const float* boundsMin, const float* boundsMax) {
  splat::SplatCloud c;
  c.positions.assign(positions, positions + n * 3);
  c.covariances.assign(covariances, covariances + n * 6);
  c.colors.assign(colors, colors + n * 3);
  c.alphas.assign(alphas, alphas + n);
  c.shDegree = shDegree;
  const size_t coefficients = static_cast<size_t>((shDegree + 1) * (shDegree + 1) - 1) * 3;
  if (sh != nullptr && coefficients > 0) c.sh.assign(sh, sh + n * coefficients);
  if (boundsMin != nullptr && boundsMax != nullptr) {
    for (int j = 0; j < 3; ++j) {
      c.bounds.min[j] = boundsMin[j];
      c.bounds.max[j] = boundsMax[j];
    }
  }
  return c;
}

}  // namespace

extern "C" {

uint16_t skref_to_half(float value) { return splat::toHalf(value); }
float skref_from_half(uint16_t half) { return splat::fromHalf(half); }

void skref_perspective(float fovy, float aspect, float nearPlane, float farPlane, float* out16) {
  const auto m = splat::Mat4::perspective(fovy, aspect, nearPlane, farPlane);
  std::memcpy(out16, m.m.data(), 64);
}

void skref_look_at_view(const float* position, const float* target, const float* up,
                        float* out16) {
  splatkit::WalkCamera camera;
  camera.setLookAt({position[0], position[1], position[2]}, {target[0], target[1], target[2]},
                   {up[0], up[1], up[2]});
  const auto m = camera.viewMatrix();
  std::memcpy(out16, m.m.data(), 64);
}

void skref_covariance(const float* quaternion, const float* scale, float* out6) {
  const auto c = splat::covarianceFromQuaternionScale(quaternion, scale);
  std::memcpy(out6, c.data(), 24);
}

size_t skref_sh_stride(int degree) { return splatkit::shStride(degree); }

uint64_t skref_gpu_world_bytes(uint64_t records, int shDegree, uint64_t drawCapacity,
                               uint64_t clusters, uint64_t leafRefs) {
  splat::LoadCost cost;
  cost.records = records;
  cost.shDegree = shDegree;
  cost.drawCapacity = drawCapacity;
  cost.clusters = clusters;
  cost.leafRefs = leafRefs;
  return splatkit::gpuWorldBytes(cost);
}

// out: n GpuSplat records of 32 bytes.
void skref_pack_splats(const float* positions, const float* covariances, const float* colors,
                       const float* alphas, size_t n, void* out) {
  const auto cloud =
      cloudFrom(positions, covariances, colors, alphas, nullptr, n, 0, nullptr, nullptr);
  splatkit::packSplatRange(cloud, 0, n, static_cast<splatkit::GpuSplat*>(out));
}

// sh: n * 3 * ((cloudDegree+1)^2 - 1) floats; out: n * shStride(degree) words.
void skref_pack_sh(const float* sh, size_t n, int cloudDegree, int degree, uint32_t* out) {
  std::vector<float> zeros(n * 3, 0.0f);
  std::vector<float> covs(n * 6, 0.0f);
  std::vector<float> ones(n, 1.0f);
  const auto cloud = cloudFrom(zeros.data(), covs.data(), zeros.data(), ones.data(), sh, n,
                               cloudDegree, nullptr, nullptr);
  splatkit::packShRange(cloud, degree, 0, n, out);
}

// ---- LOD trees -------------------------------------------------------------------------

void* skref_build_lod_tree(const float* positions, const float* covariances, const float* colors,
                           const float* alphas, const float* sh, size_t n, int shDegree,
                           const float* boundsMin, const float* boundsMax, uint32_t octreeDepth,
                           uint32_t clusterLeaves) {
  auto cloud = cloudFrom(positions, covariances, colors, alphas, sh, n, shDegree, boundsMin,
                         boundsMax);
  splat::LodBuildOptions options;
  if (octreeDepth != 0) options.octreeDepth = octreeDepth;
  if (clusterLeaves != 0) options.clusterLeaves = clusterLeaves;
  return new splat::LodTree(splat::buildLodTree(std::move(cloud), options));
}

// A tree given explicitly: nodes as a cloud plus the BFS layout (24-byte LodNode records).
void* skref_make_tree(const float* positions, const float* covariances, const float* colors,
                      const float* alphas, const float* sh, size_t nodes, int shDegree,
                      const void* layout, size_t leafCount) {
  auto* tree = new splat::LodTree();
  tree->nodes =
      cloudFrom(positions, covariances, colors, alphas, sh, nodes, shDegree, nullptr, nullptr);
  tree->layout.resize(nodes);
  std::memcpy(tree->layout.data(), layout, nodes * sizeof(splat::LodNode));
  tree->leafCount = leafCount;
  return tree;
}

void skref_tree_build_selection(void* handle) {
  auto* tree = static_cast<splat::LodTree*>(handle);
  tree->selection = splat::buildLodSelectionData(*tree);
}

int64_t skref_validate_lod_tree(void* handle) {
  const auto valid = splat::validateLodTree(*static_cast<splat::LodTree*>(handle));
  return valid ? static_cast<int64_t>(valid.value()) : -1;
}

size_t skref_tree_node_count(void* handle) {
  return static_cast<splat::LodTree*>(handle)->nodeCount();
}
size_t skref_tree_leaf_count(void* handle) {
  return static_cast<splat::LodTree*>(handle)->leafCount;
}
int skref_tree_sh_degree(void* handle) {
  return static_cast<splat::LodTree*>(handle)->nodes.shDegree;
}
size_t skref_tree_cluster_count(void* handle) {
  return static_cast<splat::LodTree*>(handle)->selection.clusters.size();
}
size_t skref_tree_leaf_ref_count(void* handle) {
  return static_cast<splat::LodTree*>(handle)->selection.leaves.size();
}
size_t skref_tree_sh_floats(void* handle) {
  return static_cast<splat::LodTree*>(handle)->nodes.sh.size();
}

void skref_tree_copy_nodes(void* handle, float* positions, float* covariances, float* colors,
                           float* alphas, float* sh) {
  const auto& c = static_cast<splat::LodTree*>(handle)->nodes;
  std::memcpy(positions, c.positions.data(), c.positions.size() * 4);
  std::memcpy(covariances, c.covariances.data(), c.covariances.size() * 4);
  std::memcpy(colors, c.colors.data(), c.colors.size() * 4);
  std::memcpy(alphas, c.alphas.data(), c.alphas.size() * 4);
  if (sh != nullptr && !c.sh.empty()) std::memcpy(sh, c.sh.data(), c.sh.size() * 4);
}

void skref_tree_copy_layout(void* handle, void* out) {
  const auto& l = static_cast<splat::LodTree*>(handle)->layout;
  std::memcpy(out, l.data(), l.size() * sizeof(splat::LodNode));
}

void skref_tree_copy_clusters(void* handle, void* out) {
  const auto& c = static_cast<splat::LodTree*>(handle)->selection.clusters;
  std::memcpy(out, c.data(), c.size() * sizeof(splat::LodCluster));
}

void skref_tree_copy_leaves(void* handle, uint32_t* out) {
  const auto& l = static_cast<splat::LodTree*>(handle)->selection.leaves;
  std::memcpy(out, l.data(), l.size() * 4);
}

void skref_free_tree(void* handle) { delete static_cast<splat::LodTree*>(handle); }

// Writes a .lodsplat (version 2 when the tree has selection data). 0 on success.
int skref_write_lodsplat(void* handle, const char* path) {
  return splat::writeLodSplat(*static_cast<splat::LodTree*>(handle), path) ? 0 : -1;
}

// Decodes a .lodsplat held in memory into a new tree handle, or null.
void* skref_decode_lodsplat(const uint8_t* data, size_t size, int maxShDegree) {
  auto tree = splat::decodeLodSplat(data, size, maxShDegree);
  if (!tree) return nullptr;
  return new splat::LodTree(std::move(tree.value()));
}

// ---- policy ----------------------------------------------------------------------------

void* skref_lod_threshold_new(float policyPixels) {
  return new splatkit::LodThreshold(policyPixels);
}
float skref_lod_threshold_update(void* handle, uint32_t selected, uint32_t limited,
                                 uint32_t limit) {
  return static_cast<splatkit::LodThreshold*>(handle)->update(selected, limited, limit);
}
void skref_lod_threshold_free(void* handle) { delete static_cast<splatkit::LodThreshold*>(handle); }

int skref_valid_render_policy(float lodErrorPixels, uint32_t lodSplatLimit, float alphaThreshold,
                              float subpixelThreshold, uint32_t sortDepth, const double* background) {
  splatkit::RenderPolicy p;
  p.lodErrorPixels = lodErrorPixels;
  p.lodSplatLimit = lodSplatLimit;
  p.alphaThreshold = alphaThreshold;
  p.subpixelThreshold = subpixelThreshold;
  p.sortDepth = static_cast<splatkit::SortKeyBits>(sortDepth);
  for (int j = 0; j < 3; ++j) p.backgroundColor[j] = background[j];
  std::string error;
  return splatkit::validRenderPolicy(p, &error) ? 1 : 0;
}

// Reorders a cloud in place into the reference's Morton order (SoA arrays, shDegree bands).
void skref_reorder_spatially(float* positions, float* covariances, float* colors, float* alphas,
                             float* sh, size_t n, int shDegree, const float* boundsMin,
                             const float* boundsMax) {
  auto cloud = cloudFrom(positions, covariances, colors, alphas, sh, n, shDegree, boundsMin,
                         boundsMax);
  splat::reorderSpatially(cloud);
  std::memcpy(positions, cloud.positions.data(), n * 12);
  std::memcpy(covariances, cloud.covariances.data(), n * 24);
  std::memcpy(colors, cloud.colors.data(), n * 12);
  std::memcpy(alphas, cloud.alphas.data(), n * 4);
  if (sh != nullptr && !cloud.sh.empty()) std::memcpy(sh, cloud.sh.data(), cloud.sh.size() * 4);
}

}  // extern "C"
