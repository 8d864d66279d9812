#include "world_prep.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>

namespace sk::host {
namespace {

uint32_t asUint(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

template <typename F>
void parallelFor(size_t n, int threads, F&& body) {
  threads = std::max(1, std::min<int>(threads, static_cast<int>((n + 65535) / 65536)));
  if (threads <= 1) {
    body(size_t{0}, n);
    return;
  }
  const size_t per = (n + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    const size_t b = std::min(n, per * t), e = std::min(n, b + per);
    pool.emplace_back([&, b, e] { body(b, e); });
  }
  for (auto& th : pool) th.join();
}

uint32_t packRgba8(float r, float g, float b, float a) {
  auto q = [](float v) {
    return static_cast<uint32_t>(std::lround(std::clamp(v, 0.0f, 1.0f) * 255.0f));
  };
  return q(r) | (q(g) << 8) | (q(b) << 16) | (q(a) << 24);
}

uint32_t packHalf2(float lo, float hi) {
  return static_cast<uint32_t>(floatToHalf(lo)) | (static_cast<uint32_t>(floatToHalf(hi)) << 16);
}

float length3(const float* a, const float* b) {
  float s = 0;
  for (int j = 0; j < 3; ++j) s += (a[j] - b[j]) * (a[j] - b[j]);
  return std::sqrt(s);
}

// Frobenius distance of two covariances, off-diagonal terms counted twice, fourth root.
float covarianceError(const float* a, const float* b) {
  float s = 0;
  for (int j = 0; j < 6; ++j) {
    const float d = a[j] - b[j];
    s += d * d * ((j == 1 || j == 2 || j == 4) ? 2 : 1);
  }
  return std::sqrt(std::sqrt(s));
}

// Largest per-channel colour difference plus the per-band SH amplitude bound.
float appearanceDifference(const CloudRef& c, uint32_t a, uint32_t b) {
  float difference = 0;
  const size_t stride = size_t{3} * shCoefficients(c.shDegree);
  for (int ch = 0; ch < 3; ++ch) {
    float d = std::abs(c.colors[a * 3 + ch] - c.colors[b * 3 + ch]);
    for (int band = 1, start = 0; band <= c.shDegree; ++band) {
      float norm = 0;
      for (int k = 0; k < 2 * band + 1; ++k) {
        const float v = c.sh[a * stride + (start + k) * 3 + ch] - c.sh[b * stride + (start + k) * 3 + ch];
        norm += v * v;
      }
      d += std::sqrt(norm * (2 * band + 1) / (4.0f * static_cast<float>(M_PI)));
      start += 2 * band + 1;
    }
    difference = std::max(difference, d);
  }
  return difference;
}

}  // namespace

uint16_t floatToHalf(float v) {
  const uint32_t x = asUint(v);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const uint32_t ax = x & 0x7fffffffu;
  const uint32_t e = ax >> 23;
  const uint32_t mant = ax & 0x7fffffu;
  if (e == 0xffu) return static_cast<uint16_t>(sign | (mant ? 0x7e00u : 0x7bffu));
  if (e < 113u) {
    const uint32_t shift = 126u - e;
    if (shift > 24u) return static_cast<uint16_t>(sign);
    const uint32_t full = mant | 0x800000u;
    const uint32_t h = full >> shift;
    const uint32_t rem = full & ((1u << shift) - 1u);
    const uint32_t mid = 1u << (shift - 1u);
    const uint32_t up = (rem > mid || (rem == mid && (h & 1u))) ? 1u : 0u;
    return static_cast<uint16_t>(sign | (h + up));
  }
  uint32_t h = ((e - 112u) << 10) | (mant >> 13);
  const uint32_t rem = mant & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;
  if (h >= 0x7c00u) h = 0x7bffu;
  return static_cast<uint16_t>(sign | h);
}

float halfToFloat(uint16_t h) {
  const uint32_t sign = (static_cast<uint32_t>(h) & 0x8000u) << 16;
  const uint32_t e = (h >> 10) & 0x1fu;
  const uint32_t m = h & 0x3ffu;
  uint32_t bits;
  if (e == 0) {
    float mag = static_cast<float>(m) * 5.9604644775390625e-08f;
    std::memcpy(&bits, &mag, 4);
    bits |= sign;
  } else if (e == 31) {
    bits = sign | 0x7f800000u | (m << 13);
  } else {
    bits = sign | ((e + 112u) << 23) | (m << 13);
  }
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

void packSplats(const CloudRef& c, size_t offset, size_t count, GpuSplat* out, int threads) {
  parallelFor(count, threads, [&](size_t b, size_t e) {
    for (size_t k = b; k < e; ++k) {
      const size_t i = offset + k;
      GpuSplat& g = out[k];
      std::memcpy(g.position, &c.positions[i * 3], sizeof(g.position));
      const float alpha = c.alphas[i];
      g.rgba8 = packRgba8(c.colors[i * 3], c.colors[i * 3 + 1], c.colors[i * 3 + 2], alpha);
      g.lodAlpha = alpha > 1.0f ? asUint(alpha) : 0u;
      const float* v = &c.covariances[i * 6];
      g.cov[0] = packHalf2(v[0], v[1]);
      g.cov[1] = packHalf2(v[2], v[3]);
      g.cov[2] = packHalf2(v[4], v[5]);
    }
  });
}

void packSh(const CloudRef& c, int degree, size_t offset, size_t count, uint32_t* out,
            uint32_t stride, int threads) {
  if (degree <= 0 || count == 0) return;
  const size_t source = size_t{3} * shCoefficients(c.shDegree);
  const size_t halves = size_t{3} * shCoefficients(degree);
  parallelFor(count, threads, [&](size_t b, size_t e) {
    for (size_t k = b; k < e; ++k) {
      const float* src = &c.sh[(offset + k) * source];
      for (size_t w = 0; w < stride; ++w) {
        const size_t h = w * 2;
        const uint32_t lo = h < halves ? floatToHalf(src[h]) : 0u;
        const uint32_t hi = h + 1 < halves ? floatToHalf(src[h + 1]) : 0u;
        out[k * stride + w] = lo | (hi << 16);
      }
    }
  });
}

namespace {

// The clusters and leaf references of a breadth-first layout without walking it: the
// breadth-first order of the interior nodes alone is their layout order, so cluster k is the
// k-th interior node, its interior children are the clusters ranked from the interior count
// before its first child, and its leaf children follow the leaf children of clusters 0..k-1.
// The same arrays the walk below gives. Returns false, leaving both empty, when the child ranges
// are not consecutive from node 1 on or a node comes before its parent (not a breadth-first
// layout).
bool selectionFromBreadthFirst(const LodNode* layout, uint32_t nodeCount, int threads,
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

void buildSelection(const CloudRef& cloud, const LodNode* layout, uint32_t nodeCount,
                    std::vector<LodCluster>& clusters, std::vector<uint32_t>& leaves) {
  clusters.clear();
  leaves.clear();
  if (nodeCount == 0) return;
  const int threads = std::max(1, static_cast<int>(std::thread::hardware_concurrency()));
  const bool laidOut = layout[0].childCount != 0 &&
                       selectionFromBreadthFirst(layout, nodeCount, threads, clusters, leaves);
  // Otherwise interiors in BFS order by a walk; each cluster's interior children are
  // consecutive clusters.
  std::vector<uint32_t> order{0};
  if (!laidOut) clusters.resize(1);
  for (size_t head = 0; !laidOut && head < order.size(); ++head) {
    const uint32_t index = order[head];
    const LodNode& node = layout[index];
    LodCluster cluster{};
    cluster.node = index;
    cluster.childStart = static_cast<uint32_t>(order.size());
    cluster.leafStart = static_cast<uint32_t>(leaves.size());
    if (node.childCount == 0) leaves.push_back(index);  // a single-splat root
    for (uint32_t j = 0; j < node.childCount; ++j) {
      const uint32_t child = node.childStart + j;
      if (layout[child].childCount) order.push_back(child);
      else leaves.push_back(child);
    }
    cluster.childCount = static_cast<uint32_t>(order.size()) - cluster.childStart;
    cluster.leafCount = static_cast<uint32_t>(leaves.size()) - cluster.leafStart;
    clusters.resize(order.size());
    clusters[head] = cluster;
  }
  // Bottom up: bounds, merge error, colour variance, opacity, leaf count. A cluster reads only
  // its own node and its children, which sit in the next BFS level, so the levels are done
  // deepest first and the clusters of one level on all host threads. Clusters are in BFS order,
  // so the level after [a, b) is [b, the end of cluster b-1's children).
  std::vector<size_t> levelStart{0};
  for (size_t a = 0, b = clusters.empty() ? 0 : 1; a < b;) {
    levelStart.push_back(b);
    const size_t next = size_t{clusters[b - 1].childStart} + clusters[b - 1].childCount;
    a = b;
    b = std::max(next, b);
  }
  auto finish = [&](size_t k) {
    LodCluster& cluster = clusters[k];
    const float* parent = &cloud.positions[cluster.node * 3];
    const float* parentCov = &cloud.covariances[cluster.node * 6];
    float lo[3], hi[3];
    for (int j = 0; j < 3; ++j) {
      lo[j] = std::numeric_limits<float>::max();
      hi[j] = std::numeric_limits<float>::lowest();
    }
    float weightedVariance = 0, weightSum = 0, coincidentTransmittance = 1;
    cluster.opacity = std::clamp(cloud.alphas[cluster.node], 0.0f, 1.0f);
    auto include = [&](uint32_t index, const float* center, const float* extent, float error,
                       float variance, uint32_t leafCount) {
      for (int j = 0; j < 3; ++j) {
        lo[j] = std::min(lo[j], center[j] - extent[j]);
        hi[j] = std::max(hi[j], center[j] + extent[j]);
      }
      const float displacement = length3(&cloud.positions[index * 3], parent);
      const float shape = covarianceError(&cloud.covariances[index * 6], parentCov);
      cluster.error = std::max(cluster.error, error + displacement + shape);
      const float difference = appearanceDifference(cloud, cluster.node, index);
      const float weight = std::max(cloud.alphas[index], 0.0f) * leafCount;
      weightedVariance += weight * (variance + difference * difference);
      weightSum += weight;
      cluster.subtreeLeaves += leafCount;
      coincidentTransmittance *= 1.0f - std::clamp(cloud.alphas[index], 0.0f, 1.0f);
      cluster.opacity = std::max(cluster.opacity, std::min(cloud.alphas[index], 1.0f));
    };
    for (uint32_t j = 0; j < cluster.childCount; ++j) {
      const LodCluster& child = clusters[cluster.childStart + j];
      include(child.node, child.center, child.extent, child.error, child.colorVariance,
              child.subtreeLeaves);
    }
    for (uint32_t j = 0; j < cluster.leafCount; ++j) {
      const uint32_t index = leaves[cluster.leafStart + j];
      const float* cov = &cloud.covariances[index * 6];
      const float reach = std::sqrt(2 * std::log(std::max(255.0f * cloud.alphas[index], 1.0f)));
      const float extent[3] = {reach * std::sqrt(std::max(cov[0], 0.0f)),
                               reach * std::sqrt(std::max(cov[3], 0.0f)),
                               reach * std::sqrt(std::max(cov[5], 0.0f))};
      include(index, &cloud.positions[index * 3], extent, 0, 0, 1);
    }
    for (int j = 0; j < 3; ++j) {
      cluster.center[j] = (lo[j] + hi[j]) * 0.5f;
      cluster.extent[j] = (hi[j] - lo[j]) * 0.5f;
    }
    cluster.radius = length3(hi, cluster.center);
    const float peakDifference =
        std::abs(std::min(cloud.alphas[cluster.node], 1.0f) - (1.0f - coincidentTransmittance));
    cluster.error = std::max(cluster.error, cluster.radius * peakDifference);
    cluster.colorVariance = weightSum > 0 ? weightedVariance / weightSum : 0;
  };
  for (size_t l = levelStart.size() - 1; l-- > 0;) {
    const size_t first = levelStart[l], count = levelStart[l + 1] - first;
    const int workers = std::max(1, std::min<int>(threads, static_cast<int>(count / 2048)));
    if (workers == 1) {
      for (size_t k = 0; k < count; ++k) finish(first + k);
      continue;
    }
    std::vector<std::thread> pool;
    for (int w = 0; w < workers; ++w)
      pool.emplace_back([&, w] {
        for (size_t k = count * w / workers, e = count * (w + 1) / workers; k < e; ++k) finish(first + k);
      });
    for (auto& t : pool) t.join();
  }
}

int64_t lodDepth(const LodNode* layout, uint32_t nodeCount, uint32_t leafCount,
                 std::string* error) {
  constexpr uint32_t kMaxDepth = 255;
  auto fail = [&](const char* why) {
    if (error) *error = why;
    return int64_t{-1};
  };
  if (nodeCount == 0) return fail("LOD tree has no nodes");
  std::vector<uint32_t> depth(nodeCount, 0);
  size_t next = 1, leaves = 0;
  uint32_t deepest = 0;
  for (size_t i = 0; i < nodeCount; ++i) {
    if (i >= next) return fail("LOD has unreachable nodes");
    const LodNode& node = layout[i];
    if (node.childCount == 0) {
      ++leaves;
      continue;
    }
    if (node.childStart != next || node.childCount > nodeCount - next || depth[i] >= kMaxDepth)
      return fail("LOD child ranges are not a bounded BFS tree");
    for (size_t k = next; k < next + node.childCount; ++k) depth[k] = depth[i] + 1;
    deepest = std::max(deepest, depth[i] + 1);
    next += node.childCount;
  }
  if (next != nodeCount || leaves != leafCount) return fail("LOD topology or leaf count invalid");
  return deepest;
}

float LodThreshold::update(uint32_t selected, uint32_t limited, uint32_t limit) {
  constexpr float kRaise = 1.1f;
  constexpr float kRelax = 1.03f;
  if (limited > 0) {
    pixels_ = std::min(pixels_ * kRaise, std::max(kCeilingPixels, policy_));
  } else if (selected < limit / 10 * 9) {
    pixels_ = std::max(pixels_ / kRelax, policy_);
  }
  return pixels_;
}

uint64_t worldBytes(uint64_t records, int shDegree, uint64_t drawCapacity, uint64_t clusters,
                    uint64_t leafRefs) {
  const uint64_t drawBytesPerSplat = sizeof(Projected) + 2 * 2 * 4 + 4;
  const uint64_t walkBytesPerCluster = 16 + 8 + 16 + 2 * 4;
  const uint64_t packedSh = shDegree <= 0 ? 0 : (uint64_t{shCoefficients(shDegree)} * 3 + 1) / 2;
  const uint64_t record = sizeof(GpuSplat) + packedSh * 4;
  return records * record + drawCapacity * drawBytesPerSplat +
         clusters * (sizeof(LodCluster) + walkBytesPerCluster) + leafRefs * 4;
}

}  // namespace sk::host
