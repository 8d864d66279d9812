// The LOD tree builder: a cloud's splats become the leaves of an octree whose interior nodes
// each stand in for their children, laid out root first, level by level (what .lodsplat files
// hold and what sk_upload_lod_world takes).
//
// Restated from the reference's builder (splat-core/src/lod/LodTree.cpp:17-344, eigenvalues
// from splat-core/src/math/SymmetricEigen.cpp:8-41), step for step in the same order with the
// same float and double arithmetic, so on the same inputs it writes the same tree bit for bit:
// leaves sorted by Morton key (ties by index), cells of at most clusterLeaves leaves (or at the
// depth limit) merged into one node, single-octant cells skipped, every merge matching the
// members' weighted moments (weight = ellipsoid area x opacity), node size = twice the largest
// semi-axis (times the opacity reach of a merged node). Part labels are not carried (this build
// has none in its worlds).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/splatkit_b200.h"
#include "context.h"
#include "world_prep.h"

namespace sk {
namespace {

constexpr uint32_t kMaxOctreeDepth = 21;

// SymmetricEigen.cpp:8-41: eigenvalues of the symmetric 3x3 (upper triangle), descending.
std::array<float, 3> symmetricEigenvalues(const float* u) {
  const double xx = u[0], xy = u[1], xz = u[2], yy = u[3], yz = u[4], zz = u[5];
  const double p1 = xy * xy + xz * xz + yz * yz;
  std::array<double, 3> e;
  if (p1 < 1e-30) {
    e = {xx, yy, zz};
  } else {
    const double q = (xx + yy + zz) / 3;
    const double p2 = (xx - q) * (xx - q) + (yy - q) * (yy - q) + (zz - q) * (zz - q) + 2 * p1;
    const double p = std::sqrt(p2 / 6);
    const double bxx = (xx - q) / p, byy = (yy - q) / p, bzz = (zz - q) / p;
    const double bxy = xy / p, bxz = xz / p, byz = yz / p;
    const double det = bxx * (byy * bzz - byz * byz) - bxy * (bxy * bzz - byz * bxz) +
                       bxz * (bxy * byz - byy * bxz);
    const double r = std::clamp(det / 2, -1.0, 1.0);
    const double phi = std::acos(r) / 3;
    const double e0 = q + 2 * p * std::cos(phi);
    const double e2 = q + 2 * p * std::cos(phi + 2 * M_PI / 3);
    e = {e0, 3 * q - e0 - e2, e2};
  }
  std::sort(e.begin(), e.end(), [](double a, double b) { return a > b; });
  return {static_cast<float>(e[0]), static_cast<float>(e[1]), static_cast<float>(e[2])};
}

// LodTree.cpp:17-22 (Knud Thomsen's ellipsoid surface approximation)
float ellipsoidArea(const std::array<float, 3>& s) {
  constexpr float kP = 1.6075f;
  const float sum = std::pow(s[0] * s[1], kP) + std::pow(s[0] * s[2], kP) + std::pow(s[1] * s[2], kP);
  return 4.0f * static_cast<float>(M_PI) * std::pow(sum / 3.0f, 1.0f / kP);
}

// LodTree.cpp:27-29
float lodOpacityReach(float alpha) {
  return alpha > 1.0f ? std::sqrt(1.0f + static_cast<float>(M_E) * std::log(alpha)) : 1.0f;
}

std::array<float, 3> semiAxes(const float* cov) {
  const auto e = symmetricEigenvalues(cov);
  return {std::sqrt(std::max(e[0], 0.0f)), std::sqrt(std::max(e[1], 0.0f)), std::sqrt(std::max(e[2], 0.0f))};
}

struct Nodes {
  std::vector<float> positions, covariances, colors, alphas, sh, size;
  std::vector<std::vector<uint32_t>> children;
  size_t shStride = 0;

  size_t count() const { return alphas.size(); }

  // LodTree.cpp:47-102: one splat matching the members' weighted spatial moments.
  uint32_t merge(const std::vector<uint32_t>& members) {
    std::vector<float> weights(members.size());
    float total = 0.0f;
    for (size_t k = 0; k < members.size(); ++k) {
      const uint32_t i = members[k];
      weights[k] = ellipsoidArea(semiAxes(&covariances[i * 6])) * alphas[i];
      total += weights[k];
    }
    for (float& w : weights) w = total > 1e-30f ? w / total : 1.0f / members.size();
    float center[3] = {0, 0, 0}, rgb[3] = {0, 0, 0};
    std::vector<float> shSum(shStride, 0.0f);
    for (size_t k = 0; k < members.size(); ++k) {
      const uint32_t i = members[k];
      for (int c = 0; c < 3; ++c) {
        center[c] += weights[k] * positions[i * 3 + c];
        rgb[c] += weights[k] * colors[i * 3 + c];
      }
      for (size_t c = 0; c < shStride; ++c) shSum[c] += weights[k] * sh[i * shStride + c];
    }
    for (float& channel : rgb) channel = std::clamp(channel, 0.0f, 1.0f);
    float cov[6] = {0, 0, 0, 0, 0, 0};
    for (size_t k = 0; k < members.size(); ++k) {
      const uint32_t i = members[k];
      const float dx = positions[i * 3] - center[0];
      const float dy = positions[i * 3 + 1] - center[1];
      const float dz = positions[i * 3 + 2] - center[2];
      const float* c = &covariances[i * 6];
      const float w = weights[k];
      cov[0] += w * (dx * dx + c[0]);
      cov[1] += w * (dx * dy + c[1]);
      cov[2] += w * (dx * dz + c[2]);
      cov[3] += w * (dy * dy + c[3]);
      cov[4] += w * (dy * dz + c[4]);
      cov[5] += w * (dz * dz + c[5]);
    }
    const auto axes = semiAxes(cov);
    const float alpha = std::clamp(total / std::max(ellipsoidArea(axes), 1e-30f), 0.0f, 1000.0f);
    const auto index = static_cast<uint32_t>(count());
    positions.insert(positions.end(), center, center + 3);
    covariances.insert(covariances.end(), cov, cov + 6);
    colors.insert(colors.end(), rgb, rgb + 3);
    alphas.push_back(alpha);
    sh.insert(sh.end(), shSum.begin(), shSum.end());
    size.push_back(2.0f * axes[0] * lodOpacityReach(alpha));
    children.push_back(members);
    return index;
  }
};

struct Cell {
  uint64_t key;
  uint32_t node;
};

// LodTree.cpp:133-142
uint64_t mortonKey(const float* position, const float* boundsMin, float extent, uint32_t depth) {
  const uint32_t resolution = 1u << depth;
  uint64_t key = 0;
  for (uint32_t c = 0; c < 3; ++c) {
    const float unit = std::clamp((position[c] - boundsMin[c]) / extent, 0.0f, 1.0f);
    const uint32_t grid = std::min(static_cast<uint32_t>(unit * resolution), resolution - 1);
    for (uint32_t bit = 0; bit < depth; ++bit) key |= uint64_t{(grid >> bit) & 1u} << (3 * bit + c);
  }
  return key;
}

// LodTree.cpp:162-196
struct OctreeBuilder {
  Nodes& nodes;
  const std::vector<Cell>& sorted;
  size_t clusterLeaves;
  uint32_t depth;

  uint32_t mergeLeaves(size_t begin, size_t end) {
    std::vector<uint32_t> members;
    for (size_t j = begin; j < end; ++j) members.push_back(sorted[j].node);
    return nodes.merge(members);
  }
  std::vector<uint32_t> buildChildren(size_t begin, size_t end, uint32_t level, uint32_t shift) {
    std::vector<uint32_t> members;
    for (size_t first = begin; first < end;) {
      size_t last = first + 1;
      while (last < end && (sorted[last].key >> shift) == (sorted[first].key >> shift)) ++last;
      members.push_back(build(first, last, level + 1));
      first = last;
    }
    return members;
  }
  uint32_t build(size_t begin, size_t end, uint32_t level) {
    if (end - begin == 1) return sorted[begin].node;
    if (end - begin <= clusterLeaves || level == depth) return mergeLeaves(begin, end);
    const uint32_t shift = 3 * (depth - level - 1);
    if ((sorted[begin].key >> shift) == (sorted[end - 1].key >> shift)) return build(begin, end, level + 1);
    return nodes.merge(buildChildren(begin, end, level, shift));
  }
};

}  // namespace

// The tree of a build: the nodes as a cloud in layout order plus the layout (and optionally
// the selection data), owned until sk_lod_tree_free.
struct BuiltTree {
  std::vector<float> positions, covariances, colors, alphas, sh;
  std::vector<LodNode> layout;
  std::vector<LodCluster> clusters;
  std::vector<uint32_t> leaves;
  uint32_t leafCount = 0;
  int shDegree = 0;
  float boundsMin[3] = {0, 0, 0}, boundsMax[3] = {0, 0, 0};
};

}  // namespace sk

extern "C" {

sk_status sk_build_lod_tree(const sk_cloud_view* cloud, const float* bounds_min,
                            const float* bounds_max, uint32_t octree_depth, uint32_t cluster_leaves,
                            int32_t build_selection, sk_lod_tree** out) {
  if (!cloud || !out || cloud->count == 0 || !cloud->positions || !cloud->covariances ||
      !cloud->colors || !cloud->alphas)
    return SK_E_INVALID;
  *out = nullptr;
  const size_t n = cloud->count;
  const int degree = cloud->sh ? std::max(0, std::min(cloud->sh_degree, 3)) : 0;
  const size_t shStride = static_cast<size_t>((degree + 1) * (degree + 1) - 1) * 3;
  auto tree = std::make_unique<sk::BuiltTree>();
  // bounds: the caller's (a loader's cloud bounds), else the positions' own box
  for (int c = 0; c < 3; ++c) {
    if (bounds_min && bounds_max) {
      tree->boundsMin[c] = bounds_min[c];
      tree->boundsMax[c] = bounds_max[c];
    } else {
      float lo = cloud->positions[c], hi = lo;
      for (size_t i = 1; i < n; ++i) {
        lo = std::min(lo, cloud->positions[i * 3 + c]);
        hi = std::max(hi, cloud->positions[i * 3 + c]);
      }
      tree->boundsMin[c] = lo;
      tree->boundsMax[c] = hi;
    }
  }
  sk::Nodes nodes;
  nodes.positions.assign(cloud->positions, cloud->positions + n * 3);
  nodes.covariances.assign(cloud->covariances, cloud->covariances + n * 6);
  nodes.colors.assign(cloud->colors, cloud->colors + n * 3);
  nodes.alphas.assign(cloud->alphas, cloud->alphas + n);
  if (shStride) nodes.sh.assign(cloud->sh, cloud->sh + n * shStride);
  nodes.shStride = shStride;
  nodes.size.resize(n);
  nodes.children.resize(n);
  for (size_t i = 0; i < n; ++i) nodes.size[i] = 2.0f * sk::semiAxes(&nodes.covariances[i * 6])[0];
  // LodTree.cpp:145-156, 198-204: Morton order and the octree
  const uint32_t depth = std::clamp(octree_depth == 0 ? sk::kMaxOctreeDepth : octree_depth, 1u,
                                    sk::kMaxOctreeDepth);
  float extent = 1e-6f;
  for (int c = 0; c < 3; ++c) extent = std::max(extent, tree->boundsMax[c] - tree->boundsMin[c]);
  std::vector<sk::Cell> sorted(n);
  for (uint32_t i = 0; i < n; ++i)
    sorted[i] = {sk::mortonKey(&nodes.positions[i * 3], tree->boundsMin, extent, depth), i};
  std::sort(sorted.begin(), sorted.end(), [](const sk::Cell& a, const sk::Cell& b) {
    return a.key == b.key ? a.node < b.node : a.key < b.key;
  });
  sk::OctreeBuilder builder{nodes, sorted, std::max<size_t>(cluster_leaves == 0 ? 32 : cluster_leaves, 2), depth};
  const uint32_t root = builder.build(0, sorted.size(), 0);
  // LodTree.cpp:209-243: breadth-first layout, attributes copied in layout order
  const size_t total = nodes.count();
  std::vector<uint32_t> order;
  order.reserve(total);
  tree->layout.assign(total, sk::LodNode{});
  order.push_back(root);
  for (size_t head = 0; head < order.size(); ++head) {
    const auto& kids = nodes.children[order[head]];
    tree->layout[head].childStart = static_cast<uint32_t>(order.size());
    tree->layout[head].childCount = static_cast<uint32_t>(kids.size());
    for (const uint32_t kid : kids) order.push_back(kid);
  }
  tree->positions.resize(total * 3);
  tree->covariances.resize(total * 6);
  tree->colors.resize(total * 3);
  tree->alphas.resize(total);
  tree->sh.resize(total * shStride);
  for (size_t i = 0; i < total; ++i) {
    const uint32_t old = order[i];
    std::copy_n(&nodes.positions[old * 3], 3, &tree->positions[i * 3]);
    std::copy_n(&nodes.positions[old * 3], 3, tree->layout[i].position);
    tree->layout[i].size = nodes.size[old];
    std::copy_n(&nodes.covariances[old * 6], 6, &tree->covariances[i * 6]);
    std::copy_n(&nodes.colors[old * 3], 3, &tree->colors[i * 3]);
    tree->alphas[i] = nodes.alphas[old];
    if (shStride) std::copy_n(&nodes.sh[old * shStride], shStride, &tree->sh[i * shStride]);
  }
  tree->leafCount = static_cast<uint32_t>(n);
  tree->shDegree = degree;
  if (build_selection) {
    sk::host::CloudRef ref{tree->positions.data(), tree->covariances.data(), tree->colors.data(),
                           tree->alphas.data(), shStride ? tree->sh.data() : nullptr,
                           static_cast<uint32_t>(total), degree};
    sk::host::buildSelection(ref, tree->layout.data(), static_cast<uint32_t>(total), tree->clusters,
                             tree->leaves);
  }
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
