// Draws one frame through the reference engine's renderer interface (splatkit::SplatRenderer,
// packages/splatkit-engine/include/splatkit/rendering/SplatRenderer.h:36-160) as implemented over
// this library by splatkit-ios_b200/integration/CudaSplatRenderer.h, the way the engine would:
// applyRenderPolicy(RenderPolicy{}), uploadWorld (or createSlab + uploadTile per tile), draw(Frame)
// with the GPU order source, then the image read back. Test support for tests/test_gpu_adapter.py,
// which compares the image with the one the C ABI draws for the same cloud and camera.
//
//   draw_through_renderer <input> <output>
//
// input (little endian): u32 count, i32 sh_degree, u32 width, u32 height, u32 tiles (0: one
// uploadWorld; k: a slab of `count` records filled by k uploadTile calls of equal parts, drawn
// through k ranges), f32 view[16], proj[16], eye[3], then positions[3n], covariances[6n],
// colors[3n], alphas[n], sh[3 ((d+1)^2 - 1) n]. output: the RGBA8 image, rows top first.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "CudaSplatRenderer.h"

namespace {

template <typename T>
bool take(std::ifstream& in, T* out, size_t n) {
  return static_cast<bool>(in.read(reinterpret_cast<char*>(out), static_cast<std::streamsize>(n * sizeof(T))));
}

splat::SplatCloud slice(const splat::SplatCloud& c, size_t begin, size_t end) {
  splat::SplatCloud part;
  part.shDegree = c.shDegree;
  const size_t shPer = c.count() ? c.sh.size() / c.count() : 0;
  part.positions.assign(c.positions.begin() + begin * 3, c.positions.begin() + end * 3);
  part.covariances.assign(c.covariances.begin() + begin * 6, c.covariances.begin() + end * 6);
  part.colors.assign(c.colors.begin() + begin * 3, c.colors.begin() + end * 3);
  part.alphas.assign(c.alphas.begin() + begin, c.alphas.begin() + end);
  part.sh.assign(c.sh.begin() + begin * shPer, c.sh.begin() + end * shPer);
  return part;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
    return 2;
  }
  std::ifstream in(argv[1], std::ios::binary);
  uint32_t count = 0, width = 0, height = 0, tiles = 0;
  int32_t degree = 0;
  float view[16], proj[16], eye[3];
  if (!take(in, &count, 1) || !take(in, &degree, 1) || !take(in, &width, 1) || !take(in, &height, 1) ||
      !take(in, &tiles, 1) || !take(in, view, 16) || !take(in, proj, 16) || !take(in, eye, 3))
    return 3;
  splat::SplatCloud cloud;
  cloud.shDegree = degree;
  cloud.positions.resize(size_t{count} * 3);
  cloud.covariances.resize(size_t{count} * 6);
  cloud.colors.resize(size_t{count} * 3);
  cloud.alphas.resize(count);
  cloud.sh.resize(size_t{count} * 3 * ((degree + 1) * (degree + 1) - 1));
  if (!take(in, cloud.positions.data(), cloud.positions.size()) ||
      !take(in, cloud.covariances.data(), cloud.covariances.size()) ||
      !take(in, cloud.colors.data(), cloud.colors.size()) || !take(in, cloud.alphas.data(), count) ||
      !take(in, cloud.sh.data(), cloud.sh.size()))
    return 3;

  splatkit::CudaSplatRenderer renderer(0, width, height);
  splatkit::SplatRenderer& engine = renderer;  // everything below goes through the interface
  if (!engine.ready()) return 4;
  std::string why;
  if (!engine.applyRenderPolicy(splatkit::RenderPolicy{}, &why)) return 5;
  std::vector<splatkit::SplatRenderer::Range> ranges;
  if (tiles == 0) {
    if (!engine.uploadWorld(cloud, degree)) return 6;
    ranges.push_back({0, count});
  } else {
    if (!engine.createSlab(count, degree)) return 6;
    for (uint32_t k = 0; k < tiles; ++k) {
      const uint32_t begin = static_cast<uint32_t>(uint64_t{count} * k / tiles);
      const uint32_t end = static_cast<uint32_t>(uint64_t{count} * (k + 1) / tiles);
      if (!engine.uploadTile(begin, slice(cloud, begin, end))) return 6;
      ranges.push_back({begin, end - begin});
    }
  }
  const auto world = engine.world();
  if (!world || world->count != count) return 7;
  splatkit::SplatRenderer::Frame frame;
  frame.orderSource = splatkit::SplatRenderer::OrderSource::gpu;
  frame.ranges = ranges.data();
  frame.rangeCount = static_cast<uint32_t>(ranges.size());
  frame.shDegree = degree;
  for (int i = 0; i < 16; ++i) frame.view.m[i] = view[i], frame.proj.m[i] = proj[i];
  frame.cameraPosition = {eye[0], eye[1], eye[2]};
  if (!engine.draw(frame)) return 8;
  std::vector<uint8_t> rgba;
  if (!renderer.readImage(rgba)) return 9;
  if (engine.gpuFailed() || engine.completedFrames() < 1 || engine.submittedFrames() < 1) return 10;
  std::ofstream out(argv[2], std::ios::binary);
  out.write(reinterpret_cast<const char*>(rgba.data()), static_cast<std::streamsize>(rgba.size()));
  std::printf("drawn=%u submitted=%llu completed=%llu\n", engine.lastDrawCount(),
              static_cast<unsigned long long>(engine.submittedFrames()),
              static_cast<unsigned long long>(engine.completedFrames()));
  return out ? 0 : 11;
}
