// LOD trees built by this library: sk_build_lod_tree_device drives the GPU build
// (csrc/tree_build.cu: Morton keys, radix sort, the octree level by level, merges deepest level
// first) and, when asked, attaches the selection data (selection.cpp); the tree is then read in
// place through sk_lod_tree_view until sk_lod_tree_free.
//
// The tree is the reference's buildLodTree (splat-core/src/lod/LodTree.cpp:308-330) over the same
// cloud and bounds: the layout is the same exactly, node attributes to a few ulp (the eigen-solve's
// acos/cos and the surface formula's powf are the device's, not the host library's).
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/splatkit_b200.h"
#include "context.h"
#include "world_prep.h"

namespace sk {

namespace {
constexpr uint32_t kMaxOctreeDepth = 21;  // three key bits per level in a 63-bit Morton key
}  // namespace

// A built tree: the nodes as a cloud in layout order, the layout, and optionally the selection
// data, owned until sk_lod_tree_free.
struct BuiltTree {
  HostArray<float> positions, covariances, colors, alphas, sh;
  HostArray<LodNode> layout;
  std::vector<LodCluster> clusters;
  std::vector<uint32_t> leaves;
  uint32_t leafCount = 0;
  int shDegree = 0;
  float boundsMin[3] = {0, 0, 0}, boundsMax[3] = {0, 0, 0};
};

namespace {

// The build's bounds: the caller's (a loader's cloud bounds), else the positions' own box.
void treeBounds(const sk_cloud_view* cloud, const float* bounds_min, const float* bounds_max,
                BuiltTree& tree) {
  const size_t n = cloud->count;
  for (int c = 0; c < 3; ++c) {
    if (bounds_min && bounds_max) {
      tree.boundsMin[c] = bounds_min[c];
      tree.boundsMax[c] = bounds_max[c];
      continue;
    }
    float lo = cloud->positions[c], hi = lo;
    for (size_t i = 1; i < n; ++i) {
      lo = std::min(lo, cloud->positions[i * 3 + c]);
      hi = std::max(hi, cloud->positions[i * 3 + c]);
    }
    tree.boundsMin[c] = lo;
    tree.boundsMax[c] = hi;
  }
}

bool attachSelection(BuiltTree& tree) {
  const size_t shStride = static_cast<size_t>((tree.shDegree + 1) * (tree.shDegree + 1) - 1) * 3;
  const auto total = static_cast<uint32_t>(tree.layout.size());
  host::CloudRef ref{tree.positions.data(), tree.covariances.data(), tree.colors.data(),
                     tree.alphas.data(), shStride ? tree.sh.data() : nullptr, total, tree.shDegree};
  return host::buildSelection(ref, tree.layout.data(), total, tree.clusters, tree.leaves);
}

}  // namespace
}  // namespace sk

extern "C" {

sk_status sk_build_lod_tree_device(const sk_cloud_view* cloud, const float* bounds_min,
                                   const float* bounds_max, uint32_t octree_depth,
                                   uint32_t cluster_leaves, int32_t build_selection,
                                   sk_lod_tree** out) {
  if (!cloud || !out || cloud->count == 0 || !cloud->positions || !cloud->covariances ||
      !cloud->colors || !cloud->alphas)
    return SK_E_INVALID;
  *out = nullptr;
  if (cloud->count > sk::kMaxLodBuildLeaves) return SK_E_LIMIT;
  const int degree = cloud->sh ? std::max(0, std::min(cloud->sh_degree, 3)) : 0;
  const auto shStride = static_cast<uint32_t>(((degree + 1) * (degree + 1) - 1) * 3);
  auto tree = std::make_unique<sk::BuiltTree>();
  sk::treeBounds(cloud, bounds_min, bounds_max, *tree);
  sk::LodBuildInput in{};
  in.positions = cloud->positions;
  in.covariances = cloud->covariances;
  in.colors = cloud->colors;
  in.alphas = cloud->alphas;
  in.sh = shStride ? cloud->sh : nullptr;
  in.count = cloud->count;
  in.shStride = shStride;
  in.extent = 1e-6f;
  for (int c = 0; c < 3; ++c) {
    in.boundsMin[c] = tree->boundsMin[c];
    in.extent = std::max(in.extent, tree->boundsMax[c] - tree->boundsMin[c]);
  }
  in.depth = std::clamp(octree_depth == 0 ? sk::kMaxOctreeDepth : octree_depth, 1u, sk::kMaxOctreeDepth);
  in.clusterLeaves = std::max(cluster_leaves == 0 ? 32u : cluster_leaves, 2u);
  sk::LodBuildOutput built;
  if (sk::buildLodTreeGpu(in, built) != cudaSuccess) return SK_E_DEVICE;
  tree->positions = std::move(built.positions);
  tree->covariances = std::move(built.covariances);
  tree->colors = std::move(built.colors);
  tree->alphas = std::move(built.alphas);
  tree->sh = std::move(built.sh);
  tree->layout = std::move(built.layout);
  tree->leafCount = cloud->count;
  tree->shDegree = degree;
  if (build_selection && !sk::attachSelection(*tree)) return SK_E_DEVICE;  // not breadth first
  *out = reinterpret_cast<sk_lod_tree*>(tree.release());
  return SK_OK;
}

sk_status sk_lod_tree_view(const sk_lod_tree* handle, sk_lod_view* out, float* bounds_min,
                           float* bounds_max) {
  const auto* t = reinterpret_cast<const sk::BuiltTree*>(handle);
  if (!t || !out) return SK_E_INVALID;
  std::memset(out, 0, sizeof(*out));
  out->nodes.positions = t->positions.data();
  out->nodes.covariances = t->covariances.data();
  out->nodes.colors = t->colors.data();
  out->nodes.alphas = t->alphas.data();
  out->nodes.sh = t->sh.empty() ? nullptr : t->sh.data();
  out->nodes.count = static_cast<uint32_t>(t->alphas.size());
  out->nodes.sh_degree = t->shDegree;
  out->layout = reinterpret_cast<const sk_lod_node*>(t->layout.data());
  out->node_count = static_cast<uint32_t>(t->layout.size());
  out->leaf_count = t->leafCount;
  out->clusters = t->clusters.empty() ? nullptr : reinterpret_cast<const sk_lod_cluster*>(t->clusters.data());
  out->cluster_count = static_cast<uint32_t>(t->clusters.size());
  out->leaves = t->leaves.empty() ? nullptr : t->leaves.data();
  out->leaf_ref_count = static_cast<uint32_t>(t->leaves.size());
  for (int c = 0; c < 3; ++c) {
    if (bounds_min) bounds_min[c] = t->boundsMin[c];
    if (bounds_max) bounds_max[c] = t->boundsMax[c];
  }
  return SK_OK;
}

void sk_lod_tree_free(sk_lod_tree* handle) { delete reinterpret_cast<sk::BuiltTree*>(handle); }

}  // extern "C"
