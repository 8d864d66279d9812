// LOD selection data: what the cut rounds (csrc/lod.cu) read about a breadth-first laid-out tree.
// One 64-byte record per interior node (a "cluster": its bounding box and sphere, how far its
// merged splat strays from what it stands for, the colour variance beneath it, its opacity and
// leaf count, and where its interior and leaf children are), plus the list of every cluster's
// leaf children.
//
// The values are those of the reference's buildLodSelectionData
// (splat-core/src/lod/LodSelection.cpp:47-133): the cut is compared with the reference's bit for
// bit, so each quantity is formed from the same float operations in the same order (the fourth
// root of the off-diagonal-weighted covariance distance, the per-band harmonics bound with
// (2l+1)/4pi, the 255-alpha reach of a leaf, the children-then-leaves order of the running sums
// and of the transmittance product). How they are computed is this file's own:
//   1. the topology comes from prefix sums over the layout, not from a walk: in a breadth-first
//      layout the interior nodes in layout order are the clusters in order;
//   2. the clusters are finished a tree level at a time, deepest first, the clusters of a level
//      on all host threads. Each cluster gathers its members (interior children, then leaf
//      children) into a table of what each contributes (its box, the error and variance it
//      carries, its leaf weight, its discrepancy from the cluster's own splat); every output is
//      then one fold over that table.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "world_prep.h"

namespace sk::host {
namespace {

constexpr float kFourPi = 4.0f * static_cast<float>(M_PI);
// covariance entries (xx, xy, xz, yy, yz, zz): the off-diagonal ones stand for two matrix entries
constexpr float kEntryWeight[6] = {1.0f, 2.0f, 2.0f, 1.0f, 2.0f, 1.0f};

// |a - b| for 3-vectors, squares summed x, y, z.
float distance3(const float* a, const float* b) {
  float sum = 0.0f;
  for (int axis = 0; axis < 3; ++axis) {
    const float d = a[axis] - b[axis];
    sum += d * d;
  }
  return std::sqrt(sum);
}

// How far apart two covariances are, in world length: the fourth root of the squared Frobenius
// distance (each off-diagonal entry counted for both of its matrix places).
float shapeDiscrepancy(const float* a, const float* b) {
  float sum = 0.0f;
  for (int k = 0; k < 6; ++k) {
    const float d = a[k] - b[k];
    sum += d * d * kEntryWeight[k];
  }
  return std::sqrt(std::sqrt(sum));
}

// The largest, over the three channels, of the base colour difference plus a bound on the
// directional difference of each harmonics band: sqrt(|dc_l|^2 (2l + 1) / 4 pi) per band l.
float appearanceGap(const CloudRef& c, uint32_t a, uint32_t b) {
  const size_t stride = size_t{3} * shCoefficients(c.shDegree);
  const float* shA = c.shDegree > 0 ? c.sh + a * stride : nullptr;
  const float* shB = c.shDegree > 0 ? c.sh + b * stride : nullptr;
  float widest = 0.0f;
  for (int channel = 0; channel < 3; ++channel) {
    float gap = std::abs(c.colors[a * 3 + channel] - c.colors[b * 3 + channel]);
    uint32_t first = 0;  // first coefficient of the band
    for (int band = 1; band <= c.shDegree; ++band) {
      const uint32_t width = 2u * band + 1u;
      float energy = 0.0f;
      for (uint32_t k = first; k < first + width; ++k) {
        const float d = shA[k * 3 + channel] - shB[k * 3 + channel];
        energy += d * d;
      }
      gap += std::sqrt(energy * static_cast<float>(width) / kFourPi);
      first += width;
    }
    widest = std::max(widest, gap);
  }
  return widest;
}

// What one member (an interior child's cluster, or a leaf splat) contributes to its cluster.
struct Member {
  uint32_t node;
  float lo[3], hi[3];  // the box it covers
  float carriedError;  // the child cluster's own error (0 for a leaf)
  float variance;      // the child cluster's colour variance (0 for a leaf)
  uint32_t leaves;     // leaves it stands for
};

Member childMember(const LodCluster& child) {
  Member m;
  m.node = child.node;
  for (int a = 0; a < 3; ++a) {
    m.lo[a] = child.center[a] - child.extent[a];
    m.hi[a] = child.center[a] + child.extent[a];
  }
  m.carriedError = child.error;
  m.variance = child.colorVariance;
  m.leaves = child.subtreeLeaves;
  return m;
}

// A leaf's box: its centre out to the renderer's alpha-dependent cutoff along each axis, the
// cutoff reach sqrt(2 ln(255 alpha)) standard deviations (none below alpha = 1/255).
Member leafMember(const CloudRef& c, uint32_t node) {
  Member m;
  m.node = node;
  const float reach = std::sqrt(2 * std::log(std::max(255.0f * c.alphas[node], 1.0f)));
  const float* p = &c.positions[node * 3];
  const float* v = &c.covariances[node * 6];
  const float sigma[3] = {std::sqrt(std::max(v[0], 0.0f)), std::sqrt(std::max(v[3], 0.0f)),
                          std::sqrt(std::max(v[5], 0.0f))};
  for (int a = 0; a < 3; ++a) {
    const float extent = reach * sigma[a];
    m.lo[a] = p[a] - extent;
    m.hi[a] = p[a] + extent;
  }
  m.carriedError = 0.0f;
  m.variance = 0.0f;
  m.leaves = 1;
  return m;
}

// Fills a cluster's attributes from its member table (members in the order interior children,
// then leaf children, which the running sums below depend on).
void foldMembers(const CloudRef& c, const std::vector<Member>& members, LodCluster& out) {
  const uint32_t self = out.node;
  const float* selfPos = &c.positions[self * 3];
  const float* selfCov = &c.covariances[self * 6];
  // the box
  float lo[3], hi[3];
  std::fill(lo, lo + 3, std::numeric_limits<float>::max());
  std::fill(hi, hi + 3, std::numeric_limits<float>::lowest());
  for (const Member& m : members)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], m.lo[a]);
      hi[a] = std::max(hi[a], m.hi[a]);
    }
  // the largest error a member brings: its own, plus how far it lies and differs in shape from
  // the cluster's splat
  float error = 0.0f;
  for (const Member& m : members) {
    const float stray = distance3(&c.positions[m.node * 3], selfPos);
    const float reshape = shapeDiscrepancy(&c.covariances[m.node * 6], selfCov);
    error = std::max(error, m.carriedError + stray + reshape);
  }
  // colour variance: the members' variance plus their squared colour gap, weighted by opacity
  // times leaves
  float weighted = 0.0f, weights = 0.0f;
  for (const Member& m : members) {
    const float gap = appearanceGap(c, self, m.node);
    const float w = std::max(c.alphas[m.node], 0.0f) * m.leaves;
    weighted += w * (m.variance + gap * gap);
    weights += w;
  }
  // opacity, leaves, and the light the members let through where they coincide
  float opacity = std::clamp(c.alphas[self], 0.0f, 1.0f);
  float through = 1.0f;
  uint32_t leaves = 0;
  for (const Member& m : members) {
    leaves += m.leaves;
    through *= 1.0f - std::clamp(c.alphas[m.node], 0.0f, 1.0f);
    opacity = std::max(opacity, std::min(c.alphas[m.node], 1.0f));
  }
  for (int a = 0; a < 3; ++a) {
    out.center[a] = (lo[a] + hi[a]) * 0.5f;
    out.extent[a] = (hi[a] - lo[a]) * 0.5f;
  }
  out.radius = distance3(hi, out.center);
  // the cluster's splat against the members' combined peak opacity
  const float peakGap = std::abs(std::min(c.alphas[self], 1.0f) - (1.0f - through));
  out.error = std::max(error, out.radius * peakGap);
  out.colorVariance = weights > 0 ? weighted / weights : 0;
  out.opacity = opacity;
  out.subtreeLeaves = leaves;
}

// Cluster topology of a breadth-first layout by prefix sums (see the file comment). False when
// the child ranges are not consecutive from node 1 on or a node comes before its parent.
bool clusterTopology(const LodNode* layout, uint32_t nodeCount, int threads,
                     std::vector<LodCluster>& clusters, std::vector<uint32_t>& leaves) {
  const int workers = std::max(1, std::min<int>(threads, static_cast<int>(nodeCount / 65536)));
  // per slice: interiors and children, then each node's exclusive counts
  std::vector<uint64_t> sliceInteriors(workers + 1, 0), sliceChildren(workers + 1, 0);
  forSlices(nodeCount, workers, [&](int w, size_t b, size_t e) {
    uint64_t interiors = 0, children = 0;
    for (size_t i = b; i < e; ++i) {
      interiors += layout[i].childCount != 0;
      children += layout[i].childCount;
    }
    sliceInteriors[w + 1] = interiors;
    sliceChildren[w + 1] = children;
  });
  for (int w = 0; w < workers; ++w) {
    sliceInteriors[w + 1] += sliceInteriors[w];
    sliceChildren[w + 1] += sliceChildren[w];
  }
  if (sliceChildren[workers] + 1 != nodeCount) return false;
  // each node's interior rank, and the interior nodes in order
  const auto count = static_cast<uint32_t>(sliceInteriors[workers]);
  std::vector<uint32_t> rank(size_t{nodeCount} + 1), nodeOf(count);
  std::vector<char> bad(workers, 0);
  forSlices(nodeCount, workers, [&](int w, size_t b, size_t e) {
    uint64_t interiors = sliceInteriors[w], next = 1 + sliceChildren[w];
    for (size_t i = b; i < e; ++i) {
      rank[i] = static_cast<uint32_t>(interiors);
      if (i >= next) bad[w] = 1;  // every node after the one whose range holds it
      if (layout[i].childCount) {
        if (layout[i].childStart != next) bad[w] = 1;
        nodeOf[interiors++] = static_cast<uint32_t>(i);
        next += layout[i].childCount;
      }
    }
  });
  rank[nodeCount] = count;
  for (char b : bad)
    if (b) return false;
  // each cluster's children and leaves
  clusters.assign(count, LodCluster{});
  const int clusterWorkers = std::max(1, std::min<int>(threads, static_cast<int>(count / 16384)));
  std::vector<uint64_t> sliceLeaves(clusterWorkers + 1, 0);
  forSlices(count, clusterWorkers, [&](int w, size_t b, size_t e) {
    uint64_t leafTotal = 0;
    for (size_t k = b; k < e; ++k) {
      const LodNode& node = layout[nodeOf[k]];
      LodCluster& c = clusters[k];
      c.node = nodeOf[k];
      c.childStart = rank[node.childStart];
      c.childCount = rank[node.childStart + node.childCount] - c.childStart;
      c.leafCount = node.childCount - c.childCount;
      leafTotal += c.leafCount;
    }
    sliceLeaves[w + 1] = leafTotal;
  });
  for (int w = 0; w < clusterWorkers; ++w) sliceLeaves[w + 1] += sliceLeaves[w];
  leaves.resize(sliceLeaves[clusterWorkers]);
  forSlices(count, clusterWorkers, [&](int w, size_t b, size_t e) {
    auto at = static_cast<uint32_t>(sliceLeaves[w]);
    for (size_t k = b; k < e; ++k) {
      LodCluster& c = clusters[k];
      c.leafStart = at;
      const LodNode& node = layout[c.node];
      for (uint32_t j = 0; j < node.childCount; ++j)
        if (layout[node.childStart + j].childCount == 0) leaves[at++] = node.childStart + j;
    }
  });
  return true;
}

}  // namespace

bool buildSelection(const CloudRef& cloud, const LodNode* layout, uint32_t nodeCount,
                    std::vector<LodCluster>& clusters, std::vector<uint32_t>& leaves) {
  clusters.clear();
  leaves.clear();
  if (nodeCount == 0) return true;
  const int threads = std::max(1, static_cast<int>(std::thread::hardware_concurrency()));
  if (layout[0].childCount == 0) {
    // a tree of one splat: one cluster whose only leaf is the root itself
    if (nodeCount != 1) return false;
    clusters.assign(1, LodCluster{});
    clusters[0].childStart = 1;  // where its interior children would start: after itself
    clusters[0].leafCount = 1;
    leaves.assign(1, 0u);
  } else if (!clusterTopology(layout, nodeCount, threads, clusters, leaves)) {
    return false;
  }
  // The levels, deepest last: clusters are in breadth-first order, so the level after [a, b)
  // runs from b to the end of cluster b - 1's interior children.
  std::vector<size_t> levelStart{0};
  for (size_t a = 0, b = clusters.empty() ? 0 : 1; a < b;) {
    levelStart.push_back(b);
    const size_t next = size_t{clusters[b - 1].childStart} + clusters[b - 1].childCount;
    a = b;
    b = std::max(next, b);
  }
  for (size_t level = levelStart.size() - 1; level-- > 0;) {
    const size_t first = levelStart[level], count = levelStart[level + 1] - first;
    const int workers = std::max(1, std::min<int>(threads, static_cast<int>(count / 2048)));
    forSlices(count, workers, [&](int, size_t b, size_t e) {
      std::vector<Member> members;
      for (size_t k = first + b; k < first + e; ++k) {
        LodCluster& cluster = clusters[k];
        members.clear();
        for (uint32_t j = 0; j < cluster.childCount; ++j)
          members.push_back(childMember(clusters[cluster.childStart + j]));
        for (uint32_t j = 0; j < cluster.leafCount; ++j)
          members.push_back(leafMember(cloud, leaves[cluster.leafStart + j]));
        foldMembers(cloud, members, cluster);
      }
    });
  }
  return true;
}

}  // namespace sk::host
