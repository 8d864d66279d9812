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
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <thread>
#include <utility>
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

// Node attributes, structure of arrays. `area` caches ellipsoidArea(semiAxes(covariance)), the
// merge weight per unit opacity, so each node's eigenvalues are taken once. Node k's children
// are kids[kidStart[k] .. kidStart[k] + kidCount[k]).
struct Store {
  HostArray<float> positions, covariances, colors, alphas, sh, size, area;
  HostArray<uint32_t> kidStart, kidCount, kids;
  size_t count() const { return alphas.size(); }
};

// Where a node id lives: ids below `split` in `low`, the others at id - base in `high` (the
// nodes this builder adds). A worker reads the shared leaves and writes its own store; the last,
// sequential pass holds everything in one store.
struct Nodes {
  const Store* low;
  Store* high;
  uint32_t split, base;
  size_t shStride;

  const Store& at(uint32_t id, size_t& i) const {
    if (id < split) {
      i = id;
      return *low;
    }
    i = id - base;
    return *high;
  }

  // LodTree.cpp:47-102: one splat matching the members' weighted spatial moments.
  uint32_t merge(const std::vector<uint32_t>& members) {
    const size_t m = members.size();
    std::vector<float> weights(m);
    std::vector<std::pair<const Store*, size_t>> ref(m);
    float total = 0.0f;
    for (size_t k = 0; k < m; ++k) {
      size_t i;
      const Store& st = at(members[k], i);
      ref[k] = {&st, i};
      weights[k] = st.area[i] * st.alphas[i];
      total += weights[k];
    }
    for (float& w : weights) w = total > 1e-30f ? w / total : 1.0f / m;
    float center[3] = {0, 0, 0}, rgb[3] = {0, 0, 0};
    std::vector<float> shSum(shStride, 0.0f);
    for (size_t k = 0; k < m; ++k) {
      const Store& st = *ref[k].first;
      const size_t i = ref[k].second;
      for (int c = 0; c < 3; ++c) {
        center[c] += weights[k] * st.positions[i * 3 + c];
        rgb[c] += weights[k] * st.colors[i * 3 + c];
      }
      for (size_t c = 0; c < shStride; ++c) shSum[c] += weights[k] * st.sh[i * shStride + c];
    }
    for (float& channel : rgb) channel = std::clamp(channel, 0.0f, 1.0f);
    float cov[6] = {0, 0, 0, 0, 0, 0};
    for (size_t k = 0; k < m; ++k) {
      const Store& st = *ref[k].first;
      const size_t i = ref[k].second;
      const float dx = st.positions[i * 3] - center[0];
      const float dy = st.positions[i * 3 + 1] - center[1];
      const float dz = st.positions[i * 3 + 2] - center[2];
      const float* c = &st.covariances[i * 6];
      const float w = weights[k];
      cov[0] += w * (dx * dx + c[0]);
      cov[1] += w * (dx * dy + c[1]);
      cov[2] += w * (dx * dz + c[2]);
      cov[3] += w * (dy * dy + c[3]);
      cov[4] += w * (dy * dz + c[4]);
      cov[5] += w * (dz * dz + c[5]);
    }
    const auto axes = semiAxes(cov);
    const float area = ellipsoidArea(axes);
    const float alpha = std::clamp(total / std::max(area, 1e-30f), 0.0f, 1000.0f);
    Store& out = *high;
    const auto id = static_cast<uint32_t>(base + out.count());
    out.positions.insert(out.positions.end(), center, center + 3);
    out.covariances.insert(out.covariances.end(), cov, cov + 6);
    out.colors.insert(out.colors.end(), rgb, rgb + 3);
    out.alphas.push_back(alpha);
    out.sh.insert(out.sh.end(), shSum.begin(), shSum.end());
    out.size.push_back(2.0f * axes[0] * lodOpacityReach(alpha));
    out.area.push_back(area);
    out.kidStart.push_back(static_cast<uint32_t>(out.kids.size()));
    out.kidCount.push_back(static_cast<uint32_t>(m));
    out.kids.insert(out.kids.end(), members.begin(), members.end());
    return id;
  }
};

struct Cell {
  uint64_t key;
  uint32_t node;
};

// LodTree.cpp:133-142
// Bit k of a 21-bit value to bit 3k.
uint64_t spreadBits3(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

uint64_t mortonKey(const float* position, const float* boundsMin, float extent, uint32_t depth) {
  const uint32_t resolution = 1u << depth;
  uint64_t key = 0;
  for (uint32_t c = 0; c < 3; ++c) {
    const float unit = std::clamp((position[c] - boundsMin[c]) / extent, 0.0f, 1.0f);
    const uint32_t grid = std::min(static_cast<uint32_t>(unit * resolution), resolution - 1);
    key |= spreadBits3(grid) << c;  // grid < 2^depth: bit k of axis c lands at 3k + c
  }
  return key;
}

// A subtree built on its own: the sorted range, the level its build starts at, and its root.
struct Task {
  size_t begin, end;
  uint32_t level;
  uint32_t root = 0;
  uint32_t worker = 0;
};

// LodTree.cpp:162-196. With `tasks` set, a call on a task's range returns the task's root
// instead of building it (the subtrees were built beforehand, in parallel).
struct OctreeBuilder {
  Nodes& nodes;
  const HostArray<Cell>& sorted;
  size_t clusterLeaves;
  uint32_t depth;
  const std::vector<Task>* tasks = nullptr;

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
    if (tasks) {
      auto it = std::lower_bound(tasks->begin(), tasks->end(), begin,
                                 [](const Task& t, size_t b) { return t.begin < b; });
      if (it != tasks->end() && it->begin == begin && it->end == end && it->level == level)
        return it->root;
    }
    if (end - begin == 1) return sorted[begin].node;
    if (end - begin <= clusterLeaves || level == depth) return mergeLeaves(begin, end);
    const uint32_t shift = 3 * (depth - level - 1);
    if ((sorted[begin].key >> shift) == (sorted[end - 1].key >> shift)) return build(begin, end, level + 1);
    return nodes.merge(buildChildren(begin, end, level, shift));
  }

  // The same descent without merging: every range of at most `limit` leaves the build reaches
  // becomes a task.
  void plan(size_t begin, size_t end, uint32_t level, size_t limit, std::vector<Task>& out) const {
    if (end - begin <= limit || end - begin <= clusterLeaves || level == depth) {
      out.push_back(Task{begin, end, level});
      return;
    }
    const uint32_t shift = 3 * (depth - level - 1);
    if ((sorted[begin].key >> shift) == (sorted[end - 1].key >> shift)) return plan(begin, end, level + 1, limit, out);
    for (size_t first = begin; first < end;) {
      size_t last = first + 1;
      while (last < end && (sorted[last].key >> shift) == (sorted[first].key >> shift)) ++last;
      plan(first, last, level + 1, limit, out);
      first = last;
    }
  }
};

unsigned workerCount() { return std::max(1u, std::min(64u, std::thread::hardware_concurrency())); }

// Runs fn(i) for i in [0, n) on the worker threads, in contiguous slices.
template <typename Fn>
void parallelFor(size_t n, Fn fn) {
  const unsigned workers = static_cast<unsigned>(std::min<size_t>(workerCount(), std::max<size_t>(n / 4096, 1)));
  if (workers <= 1) {
    for (size_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> pool;
  for (unsigned w = 0; w < workers; ++w)
    pool.emplace_back([&, w] {
      for (size_t i = n * w / workers, e = n * (w + 1) / workers; i < e; ++i) fn(i);
    });
  for (auto& t : pool) t.join();
}

// Sorts by (key, node): slices sorted in parallel, then merged pairwise. The order is total, so
// the result is the one sequential sort gives.
void sliceMergeSort(HostArray<Cell>& cells) {
  auto less = [](const Cell& a, const Cell& b) { return a.key == b.key ? a.node < b.node : a.key < b.key; };
  const size_t n = cells.size();
  const unsigned slices = static_cast<unsigned>(std::min<size_t>(workerCount(), std::max<size_t>(n / 65536, 1)));
  std::vector<size_t> bounds(slices + 1);
  for (unsigned s = 0; s <= slices; ++s) bounds[s] = n * s / slices;
  {
    std::vector<std::thread> pool;
    for (unsigned s = 0; s < slices; ++s)
      pool.emplace_back([&, s] { std::sort(cells.begin() + bounds[s], cells.begin() + bounds[s + 1], less); });
    for (auto& t : pool) t.join();
  }
  for (size_t width = 1; width < slices; width *= 2) {
    std::vector<std::thread> pool;
    for (size_t s = 0; s + width < slices; s += 2 * width) {
      const size_t lo = bounds[s], mid = bounds[s + width], hi = bounds[std::min<size_t>(s + 2 * width, slices)];
      pool.emplace_back([&, lo, mid, hi] {
        std::inplace_merge(cells.begin() + lo, cells.begin() + mid, cells.begin() + hi, less);
      });
    }
    for (auto& t : pool) t.join();
  }
}

// Sorts by (key, node), keys below 2^keyBits: the cells are scattered by their top 12 key bits
// into buckets in key order (counts per thread, then a parallel scatter), and the buckets are
// sorted on all threads. The order is total, so the result is the one sequential sort gives. A
// bucket holding more than half the cells (a tiny or degenerate cloud) falls back to
// sliceMergeSort.
void parallelSort(HostArray<Cell>& cells, uint32_t keyBits) {
  constexpr uint32_t kBucketBits = 12, kBuckets = 1u << kBucketBits;
  const size_t n = cells.size();
  const unsigned workers = static_cast<unsigned>(std::min<size_t>(workerCount(), std::max<size_t>(n / 65536, 1)));
  if (workers <= 1) return sliceMergeSort(cells);
  const uint32_t shift = keyBits > kBucketBits ? keyBits - kBucketBits : 0;
  auto bucketOf = [shift](const Cell& c) { return static_cast<uint32_t>(std::min<uint64_t>(c.key >> shift, kBuckets - 1)); };
  std::vector<uint32_t> counts(size_t{workers} * kBuckets, 0);
  host::forSlices(n, static_cast<int>(workers), [&](int w, size_t b, size_t e) {
    uint32_t* mine = &counts[size_t(w) * kBuckets];
    for (size_t i = b; i < e; ++i) ++mine[bucketOf(cells[i])];
  });
  // bucket starts, then each slice's first position in every bucket (bucket-major order)
  std::vector<size_t> bucketStart(kBuckets + 1, 0), at(size_t{workers} * kBuckets);
  size_t largest = 0;
  for (uint32_t k = 0; k < kBuckets; ++k) {
    size_t run = bucketStart[k];
    for (unsigned w = 0; w < workers; ++w) {
      at[size_t(w) * kBuckets + k] = run;
      run += counts[size_t(w) * kBuckets + k];
    }
    bucketStart[k + 1] = run;
    largest = std::max(largest, run - bucketStart[k]);
  }
  if (largest > n / 2) return sliceMergeSort(cells);
  HostArray<Cell> out(n);  // every element is written by the scatter
  host::forSlices(n, static_cast<int>(workers), [&](int w, size_t b, size_t e) {
    size_t* mine = &at[size_t(w) * kBuckets];
    for (size_t i = b; i < e; ++i) out[mine[bucketOf(cells[i])]++] = cells[i];
  });
  auto less = [](const Cell& a, const Cell& b) { return a.key == b.key ? a.node < b.node : a.key < b.key; };
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> pool;
  for (unsigned w = 0; w < workers; ++w)
    pool.emplace_back([&] {
      for (uint32_t k; (k = next.fetch_add(1)) < kBuckets;)
        std::sort(out.begin() + bucketStart[k], out.begin() + bucketStart[k + 1], less);
    });
  for (auto& t : pool) t.join();
  cells.swap(out);
}

}  // namespace

// The tree of a build: the nodes as a cloud in layout order plus the layout (and optionally
// the selection data), owned until sk_lod_tree_free.
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
    } else {
      float lo = cloud->positions[c], hi = lo;
      for (size_t i = 1; i < n; ++i) {
        lo = std::min(lo, cloud->positions[i * 3 + c]);
        hi = std::max(hi, cloud->positions[i * 3 + c]);
      }
      tree.boundsMin[c] = lo;
      tree.boundsMax[c] = hi;
    }
  }
}

// The selection data of a laid-out tree (buildLodSelectionData).
void attachSelection(BuiltTree& tree) {
  const size_t shStride = static_cast<size_t>((tree.shDegree + 1) * (tree.shDegree + 1) - 1) * 3;
  const auto total = static_cast<uint32_t>(tree.layout.size());
  host::CloudRef ref{tree.positions.data(), tree.covariances.data(), tree.colors.data(),
                     tree.alphas.data(), shStride ? tree.sh.data() : nullptr, total, tree.shDegree};
  host::buildSelection(ref, tree.layout.data(), total, tree.clusters, tree.leaves);
}

}  // namespace
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
  sk::treeBounds(cloud, bounds_min, bounds_max, *tree);
  // The leaves, with their size and merge area (eigenvalues per leaf), copied and solved on all
  // host threads. The arrays are reserved for every node of the tree (at most 2n - 1), so the
  // interior nodes appended later never move the leaves; untouched capacity costs no memory.
  sk::Store store;
  const size_t nodeBound = 2 * n;
  auto sized = [&](auto& array, size_t perNode) {
    array.reserve(nodeBound * perNode);
    array.resize(n * perNode);
  };
  sized(store.positions, 3);
  sized(store.covariances, 6);
  sized(store.colors, 3);
  sized(store.alphas, 1);
  sized(store.sh, shStride);
  sized(store.size, 1);
  sized(store.area, 1);
  sized(store.kidStart, 1);
  sized(store.kidCount, 1);
  sk::parallelFor(n, [&](size_t i) {
    std::copy_n(cloud->positions + i * 3, 3, &store.positions[i * 3]);
    std::copy_n(cloud->covariances + i * 6, 6, &store.covariances[i * 6]);
    std::copy_n(cloud->colors + i * 3, 3, &store.colors[i * 3]);
    store.alphas[i] = cloud->alphas[i];
    if (shStride) std::copy_n(cloud->sh + i * shStride, shStride, &store.sh[i * shStride]);
    store.kidStart[i] = 0;
    store.kidCount[i] = 0;
    const auto axes = sk::semiAxes(&store.covariances[i * 6]);
    store.size[i] = 2.0f * axes[0];
    store.area[i] = sk::ellipsoidArea(axes);
  });
  // LodTree.cpp:145-156, 198-204: Morton order and the octree
  const uint32_t depth = std::clamp(octree_depth == 0 ? sk::kMaxOctreeDepth : octree_depth, 1u,
                                    sk::kMaxOctreeDepth);
  float extent = 1e-6f;
  for (int c = 0; c < 3; ++c) extent = std::max(extent, tree->boundsMax[c] - tree->boundsMin[c]);
  sk::HostArray<sk::Cell> sorted(n);  // every element is written below
  sk::parallelFor(n, [&](size_t i) {
    sorted[i] = {sk::mortonKey(&store.positions[i * 3], tree->boundsMin, extent, depth),
                 static_cast<uint32_t>(i)};
  });
  sk::parallelSort(sorted, 3 * depth);
  const size_t clusterLeaves = std::max<size_t>(cluster_leaves == 0 ? 32 : cluster_leaves, 2);
  // Subtrees of at most `limit` leaves are built in parallel, each worker into a store of its
  // own (node ids from n on); the nodes above them are built last. Node creation order differs
  // from a sequential build, but the breadth-first layout below depends only on the tree, so the
  // file is the same.
  const unsigned workers = sk::workerCount();
  const auto leafCount = static_cast<uint32_t>(n);
  sk::Nodes shared{&store, &store, 0, 0, shStride};
  sk::OctreeBuilder planner{shared, sorted, clusterLeaves, depth};
  std::vector<sk::Task> tasks;
  planner.plan(0, n, 0, std::max<size_t>(n / (16 * workers), 256), tasks);
  std::vector<sk::Store> own(workers);
  {
    std::vector<size_t> bySize(tasks.size());
    for (size_t t = 0; t < tasks.size(); ++t) bySize[t] = t;
    std::sort(bySize.begin(), bySize.end(), [&](size_t a, size_t b) {
      return tasks[a].end - tasks[a].begin > tasks[b].end - tasks[b].begin;
    });
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < workers; ++w)
      pool.emplace_back([&, w] {
        sk::Nodes mine{&store, &own[w], leafCount, leafCount, shStride};
        sk::OctreeBuilder builder{mine, sorted, clusterLeaves, depth};
        for (size_t k; (k = next.fetch_add(1)) < bySize.size();) {
          sk::Task& t = tasks[bySize[k]];
          t.root = builder.build(t.begin, t.end, t.level);
          t.worker = w;
        }
      });
    for (auto& t : pool) t.join();
  }
  // Workers' nodes after the leaves, in worker order; their ids (n + local) shifted to match.
  std::vector<uint32_t> offset(workers, 0);
  for (unsigned w = 1; w < workers; ++w) offset[w] = offset[w - 1] + static_cast<uint32_t>(own[w - 1].count());
  {
    // room for every worker's nodes and the few built last, so appending never moves the leaves
    size_t interior = 0, kids = 0;
    for (const auto& o : own) interior += o.count(), kids += o.kids.size();
    const size_t nodesTotal = n + interior + tasks.size() + 64;
    store.positions.reserve(nodesTotal * 3);
    store.covariances.reserve(nodesTotal * 6);
    store.colors.reserve(nodesTotal * 3);
    store.alphas.reserve(nodesTotal);
    if (shStride) store.sh.reserve(nodesTotal * shStride);
    store.size.reserve(nodesTotal);
    store.area.reserve(nodesTotal);
    store.kidStart.reserve(nodesTotal);
    store.kidCount.reserve(nodesTotal);
    store.kids.reserve(kids + n + 64 * clusterLeaves);
  }
  // Each worker's block has a known place (nodes from n + offset[w], child ids from
  // kidOffset[w]), so the blocks are copied in parallel, one thread per worker store.
  std::vector<size_t> kidOffset(workers + 1, store.kids.size());
  for (unsigned w = 0; w < workers; ++w) kidOffset[w + 1] = kidOffset[w] + own[w].kids.size();
  const size_t merged = n + offset[workers - 1] + own[workers - 1].count();
  store.positions.resize(merged * 3);
  store.covariances.resize(merged * 6);
  store.colors.resize(merged * 3);
  store.alphas.resize(merged);
  store.sh.resize(merged * shStride);
  store.size.resize(merged);
  store.area.resize(merged);
  store.kidStart.resize(merged);
  store.kidCount.resize(merged);
  store.kids.resize(kidOffset[workers]);
  sk::host::forSlices(workers, static_cast<int>(workers), [&](int w, size_t, size_t) {
    sk::Store& o = own[w];
    const size_t base = n + offset[w], m = o.count();
    const uint32_t shift = offset[w];
    const auto kidBase = static_cast<uint32_t>(kidOffset[w]);
    for (size_t j = 0; j < o.kids.size(); ++j) {
      const uint32_t id = o.kids[j];
      store.kids[kidOffset[w] + j] = id >= leafCount ? id + shift : id;
    }
    for (size_t j = 0; j < m; ++j) {
      store.kidStart[base + j] = o.kidStart[j] + kidBase;
      store.kidCount[base + j] = o.kidCount[j];
    }
    std::copy_n(o.positions.data(), m * 3, store.positions.data() + base * 3);
    std::copy_n(o.covariances.data(), m * 6, store.covariances.data() + base * 6);
    std::copy_n(o.colors.data(), m * 3, store.colors.data() + base * 3);
    std::copy_n(o.alphas.data(), m, store.alphas.data() + base);
    if (shStride) std::copy_n(o.sh.data(), m * shStride, store.sh.data() + base * shStride);
    std::copy_n(o.size.data(), m, store.size.data() + base);
    std::copy_n(o.area.data(), m, store.area.data() + base);
    o = sk::Store{};
  });
  for (auto& t : tasks)
    if (t.root >= leafCount) t.root += offset[t.worker];
  std::sort(tasks.begin(), tasks.end(), [](const sk::Task& a, const sk::Task& b) { return a.begin < b.begin; });
  sk::Nodes top{&store, &store, 0, 0, shStride};
  sk::OctreeBuilder builder{top, sorted, clusterLeaves, depth, &tasks};
  const uint32_t root = builder.build(0, sorted.size(), 0);
  auto& nodes = store;
  // LodTree.cpp:209-243: breadth-first layout, attributes copied in layout order
  // The queue of the breadth-first walk, one level at a time on all host threads: a level's
  // nodes count their children, the counts are summed per slice, and each node writes its
  // children at the queue's tail plus the children of the nodes before it in the level (the
  // position a sequential walk gives them).
  const size_t total = nodes.count();
  sk::HostArray<uint32_t> order(total);  // node ids in layout order; every node appears once
  tree->layout.resize(total);            // every field is written below
  order[0] = root;
  size_t levelEnd = 1;
  for (size_t levelBegin = 0; levelBegin < levelEnd;) {
    const size_t width = levelEnd - levelBegin;
    const int slices = static_cast<int>(std::min<size_t>(workers, std::max<size_t>(width / 16384, 1)));
    std::vector<uint64_t> sliceKids(slices + 1, 0);
    sk::host::forSlices(width, slices, [&](int w, size_t b, size_t e) {
      uint64_t kids = 0;
      for (size_t k = levelBegin + b; k < levelBegin + e; ++k) kids += nodes.kidCount[order[k]];
      sliceKids[w + 1] = kids;
    });
    for (int w = 0; w < slices; ++w) sliceKids[w + 1] += sliceKids[w];
    if (sliceKids[slices] > total - levelEnd) return SK_E_INVALID;  // a node reached twice: not a tree
    sk::host::forSlices(width, slices, [&](int w, size_t b, size_t e) {
      size_t tail = levelEnd + sliceKids[w];
      for (size_t head = levelBegin + b; head < levelBegin + e; ++head) {
        const uint32_t id = order[head];
        const uint32_t first = nodes.kidStart[id], count = nodes.kidCount[id];
        tree->layout[head].childStart = static_cast<uint32_t>(tail);
        tree->layout[head].childCount = count;
        std::copy_n(nodes.kids.data() + first, count, order.data() + tail);
        tail += count;
      }
    });
    levelBegin = levelEnd;
    levelEnd += sliceKids[slices];
  }
  if (levelEnd != total) return SK_E_INVALID;  // a node the walk never reached
  tree->positions.resize(total * 3);
  tree->covariances.resize(total * 6);
  tree->colors.resize(total * 3);
  tree->alphas.resize(total);
  tree->sh.resize(total * shStride);
  sk::parallelFor(total, [&](size_t i) {
    const uint32_t old = order[i];
    std::copy_n(&nodes.positions[old * 3], 3, &tree->positions[i * 3]);
    std::copy_n(&nodes.positions[old * 3], 3, tree->layout[i].position);
    tree->layout[i].size = nodes.size[old];
    std::copy_n(&nodes.covariances[old * 6], 6, &tree->covariances[i * 6]);
    std::copy_n(&nodes.colors[old * 3], 3, &tree->colors[i * 3]);
    tree->alphas[i] = nodes.alphas[old];
    if (shStride) std::copy_n(&nodes.sh[old * shStride], shStride, &tree->sh[i * shStride]);
  });
  tree->leafCount = static_cast<uint32_t>(n);
  tree->shDegree = degree;
  if (build_selection) sk::attachSelection(*tree);
  *out = reinterpret_cast<sk_lod_tree*>(tree.release());
  return SK_OK;
}

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
  if (build_selection) sk::attachSelection(*tree);
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
