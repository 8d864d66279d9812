// Host-side world preparation behind the C ABI: the packing, selection-building, depth
// validation, residency pricing and LOD threshold steps a caller runs before (or beside)
// uploading a world. No device work happens here.
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/splatkit_b200.h"
#include "context.h"
#include "world_prep.h"

namespace {
sk::host::CloudRef cloudRef(const sk_cloud_view& c) {
  return sk::host::CloudRef{c.positions, c.covariances, c.colors, c.alphas, c.sh, c.count,
                            c.sh ? std::max(0, std::min(c.sh_degree, 3)) : 0};
}
}  // namespace

extern "C" {

uint32_t sk_sh_device_stride(int32_t degree) { return sk::shDeviceStride(degree); }

sk_status sk_pack_splats(const sk_cloud_view* cloud, uint32_t offset, uint32_t count, void* out) {
  if (!cloud || !out || offset > cloud->count || count > cloud->count - offset) return SK_E_INVALID;
  const auto ref = cloudRef(*cloud);
  if (count && (!ref.positions || !ref.covariances || !ref.colors || !ref.alphas)) return SK_E_INVALID;
  sk::host::packSplats(ref, offset, count, static_cast<sk::GpuSplat*>(out), sk::hostThreadsPublic());
  return SK_OK;
}

sk_status sk_pack_sh(const sk_cloud_view* cloud, int32_t degree, uint32_t offset, uint32_t count,
                     uint32_t* out, uint32_t stride) {
  if (!cloud || !out || offset > cloud->count || count > cloud->count - offset) return SK_E_INVALID;
  const auto ref = cloudRef(*cloud);
  if (degree < 0 || degree > ref.shDegree || stride < sk::shPackedStride(degree)) return SK_E_INVALID;
  sk::host::packSh(ref, degree, offset, count, out, stride, sk::hostThreadsPublic());
  return SK_OK;
}

sk_status sk_build_lod_selection(const sk_lod_view* tree, sk_lod_cluster* clusters,
                                 uint32_t clusterCapacity, uint32_t* clusterCount,
                                 uint32_t* leaves, uint32_t leafCapacity, uint32_t* leafCount) {
  if (!tree || !tree->layout || tree->nodes.count != tree->node_count) return SK_E_INVALID;
  std::vector<sk::LodCluster> c;
  std::vector<uint32_t> l;
  if (!sk::host::buildSelection(cloudRef(tree->nodes),
                                reinterpret_cast<const sk::LodNode*>(tree->layout), tree->node_count,
                                c, l))
    return SK_E_INVALID;  // not a breadth-first layout
  if (clusterCount) *clusterCount = static_cast<uint32_t>(c.size());
  if (leafCount) *leafCount = static_cast<uint32_t>(l.size());
  if (clusters) std::memcpy(clusters, c.data(), std::min<size_t>(c.size(), clusterCapacity) * 64);
  if (leaves) std::memcpy(leaves, l.data(), std::min<size_t>(l.size(), leafCapacity) * 4);
  return SK_OK;
}

int64_t sk_lod_depth(const sk_lod_node* layout, uint32_t nodeCount, uint32_t leafCount) {
  if (!layout) return -1;
  return sk::host::lodDepth(reinterpret_cast<const sk::LodNode*>(layout), nodeCount, leafCount, nullptr);
}

uint64_t sk_world_bytes(uint64_t records, int32_t shDegree, uint64_t drawCapacity,
                        uint64_t clusters, uint64_t leafRefs) {
  return sk::host::worldBytes(records, shDegree, drawCapacity, clusters, leafRefs);
}

float sk_lod_threshold_update(float* state, uint32_t selected, uint32_t limited, uint32_t limit) {
  if (!state) return 0.0f;
  sk::host::LodThreshold t(state[0]);
  t.restore(state[1]);
  state[1] = t.update(selected, limited, limit);
  return state[1];
}

}  // extern "C"
