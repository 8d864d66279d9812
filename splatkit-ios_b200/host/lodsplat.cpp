// The .lodsplat reader: a LOD tree file straight into a context's device memory.
//
// Format (splat-core/include/splat/lod/LodFile.h:12-16, .../src/lod/LodFile.cpp:14-28,335-423):
// little-endian; a 64-byte header (magic "LODSPLAT", version, node count, leaf count, SH degree,
// depth, cluster count, bounds min/max, leaf-reference count, cluster record size), then one
// record per node (LodNode: position, size, child start, child count; covariance[6]; RGB; alpha;
// then the SH coefficients), and for version 2 the LodCluster records (16 words each) and the
// leaf references. The reader checks what the reference's decoder checks on the header and the
// length, the topology (BFS order, contiguous children, depth equal to the header's) and the
// attribute ranges, then hands the arrays to the LOD upload; a version-1 file gets its selection
// data built there. Not checked here: covariance positive-semidefiniteness and the clusters'
// bounds and member bookkeeping, which the upload trusts as it trusts an in-memory tree.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/splatkit_b200.h"
#include "context.h"
#include "world_prep.h"

namespace sk {
namespace {

constexpr char kMagic[8] = {'L', 'O', 'D', 'S', 'P', 'L', 'A', 'T'};
constexpr size_t kHeader = 64;
constexpr size_t kNodeFixedBytes = 64;
constexpr size_t kClusterBytes = 64;
constexpr size_t kMaxNodes = 20000000;
constexpr uint32_t kMaxDepth = 64;

uint32_t u32(const uint8_t* p) {
  return uint32_t{p[0]} | (uint32_t{p[1]} << 8) | (uint32_t{p[2]} << 16) | (uint32_t{p[3]} << 24);
}
float f32(const uint8_t* p) {
  const uint32_t bits = u32(p);
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}
size_t shFloats(int degree) { return static_cast<size_t>((degree + 1) * (degree + 1) - 1) * 3; }

// The header, checked against the file's length; an empty string means valid.
std::string readHeader(const uint8_t* data, size_t size, sk_lodsplat_header& h) {
  if (!data || size < sizeof(kMagic) || std::memcmp(data, kMagic, sizeof(kMagic)) != 0)
    return "not a LODSPLAT file";
  if (size < kHeader) return "truncated LODSPLAT header";
  h = sk_lodsplat_header{};
  h.version = u32(data + 8);
  if (h.version != 1 && h.version != 2) return "unsupported LODSPLAT version";
  h.node_count = u32(data + 12);
  h.leaf_count = u32(data + 16);
  const uint32_t degree = u32(data + 20);
  h.depth = u32(data + 24);
  h.cluster_count = u32(data + 28);
  h.leaf_ref_count = u32(data + 56);
  for (int j = 0; j < 3; ++j) {
    h.bounds_min[j] = f32(data + 32 + j * 4);
    h.bounds_max[j] = f32(data + 44 + j * 4);
  }
  const size_t n = h.node_count, clusters = h.cluster_count, refs = h.leaf_ref_count;
  const uint32_t clusterBytes = u32(data + 60);
  if (n == 0 || n > kMaxNodes || degree > 3 || h.depth > kMaxDepth || clusters > n || refs > n ||
      h.leaf_count > n || (h.version == 1 && (clusters || refs || clusterBytes)) ||
      (h.version == 2 && (!clusters || refs != h.leaf_count || clusterBytes != kClusterBytes)))
    return "invalid LODSPLAT header";
  h.sh_degree = static_cast<int32_t>(degree);
  const size_t stride = kNodeFixedBytes + shFloats(h.sh_degree) * 4;
  if (size != kHeader + n * stride + clusters * kClusterBytes + refs * 4)
    return "LODSPLAT length does not match node records";
  return {};
}

struct Decoded {
  sk_lodsplat_header header{};
  int degree = 0;  // kept harmonics degree
  std::vector<float> positions, covariances, colors, alphas, sh;
  std::vector<LodNode> layout;
  std::vector<LodCluster> clusters;
  std::vector<uint32_t> leaves;
};

bool finite(float v) { return std::isfinite(v); }

// Decodes and checks; an empty string means valid.
std::string decode(const uint8_t* data, size_t size, int maxSh, Decoded& d) {
  std::string why = readHeader(data, size, d.header);
  if (!why.empty()) return why;
  const sk_lodsplat_header& h = d.header;
  const size_t n = h.node_count;
  const size_t fileSh = shFloats(h.sh_degree);
  const size_t stride = kNodeFixedBytes + fileSh * 4;
  d.degree = std::min(h.sh_degree, std::clamp(maxSh, 0, 3));
  const size_t sh = shFloats(d.degree);
  d.positions.resize(n * 3);
  d.covariances.resize(n * 6);
  d.colors.resize(n * 3);
  d.alphas.resize(n);
  d.sh.resize(n * sh);
  d.layout.resize(n);
  for (size_t i = 0; i < n; ++i) {
    const uint8_t* p = data + kHeader + i * stride;
    LodNode& node = d.layout[i];
    for (int j = 0; j < 3; ++j) node.position[j] = d.positions[i * 3 + j] = f32(p + j * 4);
    node.size = f32(p + 12);
    node.childStart = u32(p + 16);
    node.childCount = u32(p + 20);
    for (int j = 0; j < 6; ++j) d.covariances[i * 6 + j] = f32(p + 24 + j * 4);
    for (int j = 0; j < 3; ++j) d.colors[i * 3 + j] = f32(p + 48 + j * 4);
    d.alphas[i] = f32(p + 60);
    for (size_t j = 0; j < fileSh; ++j)
      if (!finite(f32(p + kNodeFixedBytes + j * 4))) return "LOD SH is non-finite";
    for (size_t j = 0; j < sh; ++j) d.sh[i * sh + j] = f32(p + kNodeFixedBytes + j * 4);
    // LodFile.cpp:74-86 (size, opacity, position and colour ranges)
    if (!finite(node.size) || node.size < 0 || !finite(d.alphas[i]) || d.alphas[i] < 0 ||
        d.alphas[i] > 1000)
      return "LOD size or opacity invalid";
    for (int j = 0; j < 3; ++j) {
      const float c = d.colors[i * 3 + j];
      if (!finite(node.position[j]) || !finite(c) || c < 0 || c > 1) return "LOD position or colour invalid";
    }
    for (int j = 0; j < 6; ++j)
      if (!finite(d.covariances[i * 6 + j])) return "LOD covariance is non-finite";
  }
  for (int j = 0; j < 3; ++j)
    if (!finite(h.bounds_min[j]) || !finite(h.bounds_max[j]) || h.bounds_min[j] > h.bounds_max[j])
      return "LOD bounds invalid";
  std::string topology;
  const int64_t depth = host::lodDepth(d.layout.data(), static_cast<uint32_t>(n), h.leaf_count, &topology);
  if (depth < 0) return "invalid LOD hierarchy: " + topology;
  if (static_cast<uint64_t>(depth) != h.depth) return "LODSPLAT declared depth differs from topology";
  if (h.version == 2) {
    const uint8_t* p = data + kHeader + n * stride;
    d.clusters.resize(h.cluster_count);
    for (size_t k = 0; k < h.cluster_count; ++k)
      for (size_t j = 0; j < kClusterBytes / 4; ++j) {
        const uint32_t word = u32(p + k * kClusterBytes + j * 4);
        std::memcpy(reinterpret_cast<uint8_t*>(&d.clusters[k]) + j * 4, &word, 4);
      }
    p += h.cluster_count * kClusterBytes;
    d.leaves.resize(h.leaf_ref_count);
    for (size_t k = 0; k < h.leaf_ref_count; ++k) {
      d.leaves[k] = u32(p + k * 4);
      if (d.leaves[k] >= n) return "LOD selection leaf reference out of range";
    }
    // LodFile.cpp:247-251 (dimensions of the selection data)
    if (d.clusters.size() != std::max<size_t>(1, n - h.leaf_count) || d.clusters[0].node != 0)
      return "LOD selection dimensions invalid";
    for (const LodCluster& c : d.clusters)
      if (c.node >= n || uint64_t{c.childStart} + c.childCount > d.clusters.size() ||
          uint64_t{c.leafStart} + c.leafCount > d.leaves.size())
        return "LOD selection ranges invalid";
  }
  return {};
}

sk_status uploadDecoded(sk_context* handle, const Decoded& d, int32_t maxSh, uint32_t budget) {
  sk_lod_view t{};
  t.nodes.positions = d.positions.data();
  t.nodes.covariances = d.covariances.data();
  t.nodes.colors = d.colors.data();
  t.nodes.alphas = d.alphas.data();
  t.nodes.sh = d.degree > 0 ? d.sh.data() : nullptr;
  t.nodes.count = d.header.node_count;
  t.nodes.sh_degree = d.degree;
  t.layout = reinterpret_cast<const sk_lod_node*>(d.layout.data());
  t.node_count = d.header.node_count;
  t.leaf_count = d.header.leaf_count;
  t.clusters = d.clusters.empty() ? nullptr : reinterpret_cast<const sk_lod_cluster*>(d.clusters.data());
  t.cluster_count = static_cast<uint32_t>(d.clusters.size());
  t.leaves = d.leaves.empty() ? nullptr : d.leaves.data();
  t.leaf_ref_count = static_cast<uint32_t>(d.leaves.size());
  return sk_upload_lod_world(handle, &t, maxSh, budget);
}

}  // namespace
}  // namespace sk

extern "C" {

sk_status sk_lodsplat_read_header(const void* data, size_t size, sk_lodsplat_header* out) {
  if (!out) return SK_E_INVALID;
  return sk::readHeader(static_cast<const uint8_t*>(data), size, *out).empty() ? SK_OK : SK_E_INVALID;
}

sk_status sk_lodsplat_decode(const void* data, size_t size, int32_t max_sh_degree, float* positions,
                             float* covariances, float* colors, float* alphas, float* sh,
                             sk_lod_node* layout, sk_lod_cluster* clusters, uint32_t* leaves) {
  sk::Decoded d;
  if (!sk::decode(static_cast<const uint8_t*>(data), size, max_sh_degree, d).empty()) return SK_E_INVALID;
  auto copy = [](void* dst, const void* src, size_t bytes) {
    if (dst && bytes) std::memcpy(dst, src, bytes);
  };
  copy(positions, d.positions.data(), d.positions.size() * 4);
  copy(covariances, d.covariances.data(), d.covariances.size() * 4);
  copy(colors, d.colors.data(), d.colors.size() * 4);
  copy(alphas, d.alphas.data(), d.alphas.size() * 4);
  copy(sh, d.sh.data(), d.sh.size() * 4);
  copy(layout, d.layout.data(), d.layout.size() * sizeof(sk::LodNode));
  copy(clusters, d.clusters.data(), d.clusters.size() * sizeof(sk::LodCluster));
  copy(leaves, d.leaves.data(), d.leaves.size() * 4);
  return SK_OK;
}

sk_status sk_upload_lodsplat(sk_context* ctx, const void* data, size_t size, int32_t max_sh_degree,
                             uint32_t budget) {
  if (!ctx) return SK_E_INVALID;
  sk::Decoded d;
  const std::string why = sk::decode(static_cast<const uint8_t*>(data), size, max_sh_degree, d);
  if (!why.empty()) return reinterpret_cast<sk::Context*>(ctx)->fail(SK_E_INVALID, why);
  return sk::uploadDecoded(ctx, d, max_sh_degree, budget);
}

sk_status sk_upload_lodsplat_file(sk_context* ctx, const char* path, int32_t max_sh_degree,
                                  uint32_t budget) {
  if (!ctx || !path) return SK_E_INVALID;
  auto* c = reinterpret_cast<sk::Context*>(ctx);
  const int fd = open(path, O_RDONLY | O_CLOEXEC);
  if (fd < 0) return c->fail(SK_E_INVALID, std::string("cannot open ") + path);
  struct stat st {};
  if (fstat(fd, &st) != 0 || st.st_size <= 0) {
    close(fd);
    return c->fail(SK_E_INVALID, "not a LODSPLAT file");
  }
  const size_t size = static_cast<size_t>(st.st_size);
  void* map = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
  close(fd);
  if (map == MAP_FAILED) return c->fail(SK_E_INVALID, "cannot map the file");
  madvise(map, size, MADV_SEQUENTIAL);
  const sk_status result = sk_upload_lodsplat(ctx, map, size, max_sh_degree, budget);
  munmap(map, size);
  return result;
}

}  // extern "C"

// writeLodSplat (LodFile.cpp:425-458): the header, the node records, and for a tree with
// selection data the clusters and leaf references (version 2). Refuses an existing path.
extern "C" sk_status sk_write_lodsplat(const sk_lod_view* tree, const float* bounds_min,
                                       const float* bounds_max, const char* path) {
  if (!tree || !tree->layout || !path || !bounds_min || !bounds_max || tree->node_count == 0 ||
      tree->nodes.count != tree->node_count)
    return SK_E_INVALID;
  const int degree = tree->nodes.sh ? std::max(0, std::min(tree->nodes.sh_degree, 3)) : 0;
  const int64_t depth = sk::host::lodDepth(reinterpret_cast<const sk::LodNode*>(tree->layout),
                                           tree->node_count, tree->leaf_count, nullptr);
  if (depth < 0) return SK_E_INVALID;
  const bool selection = tree->cluster_count > 0 && tree->clusters && tree->leaves;
  const size_t n = tree->node_count, sh = sk::shFloats(degree);
  const size_t stride = sk::kNodeFixedBytes + sh * 4;
  std::vector<uint8_t> out(sk::kHeader + n * stride +
                           (selection ? tree->cluster_count * sk::kClusterBytes + tree->leaf_ref_count * 4 : 0));
  auto put = [&](size_t at, uint32_t v) {
    for (int j = 0; j < 4; ++j) out[at + j] = static_cast<uint8_t>(v >> (8 * j));
  };
  auto putF = [&](size_t at, float f) {
    uint32_t bits;
    std::memcpy(&bits, &f, 4);
    put(at, bits);
  };
  std::memcpy(out.data(), sk::kMagic, 8);
  put(8, selection ? 2u : 1u);
  put(12, tree->node_count);
  put(16, tree->leaf_count);
  put(20, static_cast<uint32_t>(degree));
  put(24, static_cast<uint32_t>(depth));
  put(28, selection ? tree->cluster_count : 0u);
  for (int j = 0; j < 3; ++j) {
    putF(32 + j * 4, bounds_min[j]);
    putF(44 + j * 4, bounds_max[j]);
  }
  put(56, selection ? tree->leaf_ref_count : 0u);
  put(60, selection ? static_cast<uint32_t>(sk::kClusterBytes) : 0u);
  for (size_t i = 0; i < n; ++i) {
    const size_t p = sk::kHeader + i * stride;
    const sk_lod_node& node = tree->layout[i];
    for (int j = 0; j < 3; ++j) putF(p + j * 4, node.position[j]);
    putF(p + 12, node.size);
    put(p + 16, node.child_start);
    put(p + 20, node.child_count);
    for (int j = 0; j < 6; ++j) putF(p + 24 + j * 4, tree->nodes.covariances[i * 6 + j]);
    for (int j = 0; j < 3; ++j) putF(p + 48 + j * 4, tree->nodes.colors[i * 3 + j]);
    putF(p + 60, tree->nodes.alphas[i]);
    for (size_t j = 0; j < sh; ++j) putF(p + sk::kNodeFixedBytes + j * 4, tree->nodes.sh[i * sh + j]);
  }
  if (selection) {
    size_t p = sk::kHeader + n * stride;
    for (uint32_t k = 0; k < tree->cluster_count; ++k)
      for (size_t j = 0; j < sk::kClusterBytes / 4; ++j) {
        uint32_t word;
        std::memcpy(&word, reinterpret_cast<const uint8_t*>(tree->clusters + k) + j * 4, 4);
        put(p + k * sk::kClusterBytes + j * 4, word);
      }
    p += size_t{tree->cluster_count} * sk::kClusterBytes;
    for (uint32_t k = 0; k < tree->leaf_ref_count; ++k) put(p + k * 4, tree->leaves[k]);
  }
  FILE* f = std::fopen(path, "wbx");
  if (!f) return SK_E_INVALID;
  const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
  return (std::fclose(f) == 0 && ok) ? SK_OK : SK_E_INVALID;
}
