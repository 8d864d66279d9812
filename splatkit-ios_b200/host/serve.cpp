// Continuous-batching render server behind the sk_server_* calls of include/splatkit_b200.h.
//
// A scheduler thread owns a Batch (host/batch.h). Requests land in a queue with their arrival
// time; whenever a lane is free the scheduler takes queued requests in arrival order into one
// batch (same harmonics degree, within the view, record and memory limits) and enqueues it,
// so requests that arrive while other batches are on the GPU join the next one and their work
// overlaps with what is in flight. Completed lanes are harvested by polling their events; each
// request's image has already been copied into its caller's buffer by the lane's stream.
//
// A scene is a context with a flat world or a LOD world. What stays on the device between
// requests for a scene: its records, harmonics and (LOD) selection data, and each lane's scratch,
// cuts and selection buffers; what carries from one request to the next on the host is a LOD
// scene's adaptive threshold (LodThreshold), fed by every completed request's selection report
// the way a context feeds it from its own frames, so a scene's cuts track its load.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "batch.h"
#include "world_prep.h"

namespace sk {
namespace {

using Clock = std::chrono::steady_clock;

inline constexpr uint64_t kDrawBytesPerSplat = 52;  // GpuLayout.cpp:16-17

struct Pending {
  uint64_t id = 0;
  sk_request request{};
  sk_range range{};
  uint32_t degree = 0;
  uint64_t splats = 0, priced = 0;
  Clock::time_point arrival;
};

struct Scene {
  Context* ctx = nullptr;
  uint64_t worldBytes = 0;
  uint64_t requests = 0;  // completed requests (a LOD scene's threshold has seen each)
};

struct LaneWork {
  std::vector<Pending> requests;
  Clock::time_point start;
  uint64_t priced = 0;
};

}  // namespace

struct Server {
  sk_server_config config{};
  Batch batch;
  std::vector<Scene> scenes;
  std::vector<LaneWork> work;  // per lane
  std::mutex mutex;
  std::condition_variable arrived, finished;
  std::deque<Pending> queue;        // arrived, not yet batched
  std::deque<sk_completion> done;   // completed, not yet taken
  uint64_t nextId = 0, submitted = 0, completed = 0;
  uint64_t inFlightBytes = 0, residentBytes = 0;
  bool stop = false;
  std::string error;
  std::thread scheduler;

  sk_status fail(sk_status code, const std::string& message) {
    std::lock_guard<std::mutex> g(mutex);
    error = message;
    return code;
  }
  void complete(const Pending& p, sk_status st, uint32_t visible, uint32_t views,
                Clock::time_point start, Clock::time_point end);
  void harvest(uint32_t laneIndex);
  bool launch(uint32_t laneIndex);
  void run();
};

void Server::complete(const Pending& p, sk_status st, uint32_t visible, uint32_t views,
                      Clock::time_point start, Clock::time_point end) {
  sk_completion c{};
  c.id = p.id;
  c.status = st;
  c.visible = visible;
  c.batch_views = views;
  c.queue_ms = std::chrono::duration<double, std::milli>(start - p.arrival).count();
  c.latency_ms = std::chrono::duration<double, std::milli>(end - p.arrival).count();
  std::lock_guard<std::mutex> g(mutex);
  done.push_back(c);
  ++completed;
  finished.notify_all();
}

// Collects a finished lane's requests (called with the lane's done event complete).
void Server::harvest(uint32_t i) {
  BatchLane& l = batch.lanes[i];
  const sk_status st = batch.finish(l, true);
  const auto end = Clock::now();
  LaneWork& w = work[i];
  const auto* first = static_cast<const uint32_t*>(l.hostViewFirst.ptr);
  // LOD scenes: each request's cut feeds its scene's threshold (LodThreshold::update with the
  // selected and limited counts, as a context does after each of its frames)
  const auto* reports = static_cast<const uint32_t*>(l.hostLodReports.ptr);
  for (size_t k = 0; st == SK_OK && k < l.lodPlans.size(); ++k) {
    const uint32_t* r = reports + k * 8;
    Scene& scene = scenes[w.requests[l.lodPlans[k].view].request.scene];
    scene.ctx->threshold.update(r[0], r[4], l.lodPlans[k].limit);
  }
  for (const Pending& p : w.requests) ++scenes[p.request.scene].requests;
  for (size_t k = 0; k < w.requests.size(); ++k) {
    const uint32_t visible = st == SK_OK ? first[k + 1] - first[k] : 0u;
    complete(w.requests[k], st == SK_OK ? SK_OK : st, visible,
             static_cast<uint32_t>(w.requests.size()), w.start, end);
  }
  {
    std::lock_guard<std::mutex> g(mutex);
    inFlightBytes -= w.priced;
  }
  w.requests.clear();
  w.priced = 0;
  l.busy = false;
}

// Forms a batch from the head of the queue and enqueues it on lane i; false when nothing to do.
bool Server::launch(uint32_t i) {
  BatchLane& l = batch.lanes[i];
  LaneWork& w = work[i];
  const auto now = Clock::now();
  std::vector<Pending> shed;
  {
    std::lock_guard<std::mutex> g(mutex);
    const uint64_t room = config.memory_budget > residentBytes ? config.memory_budget - residentBytes : 0;
    // shed what waited too long, and what can never fit
    while (!queue.empty()) {
      const Pending& p = queue.front();
      const double waited = std::chrono::duration<double, std::milli>(now - p.arrival).count();
      if ((config.max_queue_ms > 0 && waited > config.max_queue_ms) || p.priced > room ||
          p.splats > config.max_batch_splats) {
        shed.push_back(p);
        queue.pop_front();
      } else {
        break;
      }
    }
    if (!queue.empty()) {
      const uint32_t degree = queue.front().degree;
      uint64_t splats = 0;
      while (!queue.empty() && w.requests.size() < config.max_batch_views) {
        const Pending& p = queue.front();
        if (p.degree != degree || splats + p.splats > config.max_batch_splats ||
            inFlightBytes + w.priced + p.priced > room)
          break;
        splats += p.splats;
        w.priced += p.priced;
        w.requests.push_back(p);
        queue.pop_front();
      }
      inFlightBytes += w.priced;
    }
  }
  for (const Pending& p : shed) complete(p, SK_E_ADMISSION, 0, 0, now, now);
  if (w.requests.empty()) return !shed.empty();
  std::vector<sk_batch_view> views(w.requests.size());
  l.destinations.assign(w.requests.size(), nullptr);
  for (size_t k = 0; k < w.requests.size(); ++k) {
    const Pending& p = w.requests[k];
    views[k].world = reinterpret_cast<sk_context*>(scenes[p.request.scene].ctx);
    views[k].frame = p.request.frame;
    const bool lod = scenes[p.request.scene].ctx->world.lod;
    views[k].frame.ranges = lod ? nullptr : &p.range;
    views[k].frame.range_count = lod ? 0 : 1;
    views[k].width = p.request.width;
    views[k].height = p.request.height;
    l.destinations[k] = p.request.image;
  }
  w.start = Clock::now();
  sk_status st = batch.prepare(l, views.data(), static_cast<uint32_t>(views.size()));
  if (st == SK_OK) st = batch.enqueue(l);
  if (st != SK_OK) {
    const auto end = Clock::now();
    for (const Pending& p : w.requests) complete(p, st, 0, 0, w.start, end);
    std::lock_guard<std::mutex> g(mutex);
    inFlightBytes -= w.priced;
    w.requests.clear();
    w.priced = 0;
    return true;
  }
  l.busy = true;
  l.harvested = false;
  l.status = SK_OK;
  return true;
}

void Server::run() {
  cudaSetDevice(config.device);
  const uint32_t lanes = static_cast<uint32_t>(batch.lanes.size());
  uint32_t next = 0;
  for (;;) {
    bool progressed = false;
    // harvest finished lanes
    for (uint32_t i = 0; i < lanes; ++i) {
      BatchLane& l = batch.lanes[i];
      if (l.busy && cudaEventQuery(l.done) == cudaSuccess) {
        harvest(i);
        progressed = true;
      } else {
        cudaGetLastError();  // cudaErrorNotReady
      }
    }
    // fill free lanes, oldest requests first, lanes in turn
    for (uint32_t n = 0; n < lanes; ++n) {
      const uint32_t i = (next + n) % lanes;
      if (batch.lanes[i].busy) continue;
      if (launch(i)) {
        progressed = true;
        next = (i + 1) % lanes;
      }
    }
    std::unique_lock<std::mutex> g(mutex);
    if (stop && queue.empty()) {
      bool idle = true;
      for (auto& l : batch.lanes) idle = idle && !l.busy;
      if (idle) break;
    }
    if (!progressed) arrived.wait_for(g, std::chrono::microseconds(20));
  }
}

}  // namespace sk

using sk::Server;

extern "C" {

sk_status sk_server_create(const sk_server_config* config, sk_server** out) {
  if (!config || !out) return SK_E_INVALID;
  *out = nullptr;
  if (config->lanes == 0 || config->lanes > 16 || config->max_batch_views == 0 ||
      config->max_batch_views > 65536 || config->max_batch_splats == 0)
    return SK_E_INVALID;
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || config->device < 0 || config->device >= devices) {
    cudaGetLastError();
    return SK_E_DEVICE;
  }
  if (cudaSetDevice(config->device) != cudaSuccess) return SK_E_DEVICE;
  auto s = std::make_unique<Server>();
  s->config = *config;
  s->batch.device = config->device;
  s->batch.tuning.lanes = config->lanes;
  s->batch.tuning.maxViews = config->max_batch_views;
  s->batch.tuning.graphs = false;
  sk_default_policy(&s->batch.policy);
  s->batch.lanes = std::vector<sk::BatchLane>(config->lanes);
  for (auto& l : s->batch.lanes) {
    if (cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&l.start) != cudaSuccess || cudaEventCreate(&l.end) != cudaSuccess)
      return SK_E_DEVICE;
  }
  s->work = std::vector<sk::LaneWork>(config->lanes);
  sk::holdPooledMemory(config->device);
  // The lanes grow from the device's memory pool; give the pool their working size now (one
  // driver allocation here, not while requests wait): about 192 bytes per drawn record of
  // max_batch_splats per lane, within a quarter of the memory budget.
  {
    const uint64_t want = std::min<uint64_t>(uint64_t{config->lanes} * config->max_batch_splats * 192,
                                             config->memory_budget / 4);
    cudaStream_t first = s->batch.lanes[0].stream;
    void* block = nullptr;
    if (want > 0 && cudaMallocAsync(&block, want, first) == cudaSuccess) cudaFreeAsync(block, first);
    cudaGetLastError();  // the pool simply starts empty when that fails
    cudaStreamSynchronize(first);
  }
  Server* raw = s.get();
  s->scheduler = std::thread([raw] { raw->run(); });
  *out = reinterpret_cast<sk_server*>(s.release());
  return SK_OK;
}

void sk_server_destroy(sk_server* handle) {
  auto* s = reinterpret_cast<Server*>(handle);
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mutex);
    s->stop = true;
    s->arrived.notify_all();
  }
  if (s->scheduler.joinable()) s->scheduler.join();
  for (auto& l : s->batch.lanes)
    if (l.stream) cudaStreamSynchronize(l.stream);
  delete s;
}

const char* sk_server_last_error(const sk_server* handle) {
  const auto* s = reinterpret_cast<const Server*>(handle);
  return s ? s->error.c_str() : "no server";
}

sk_status sk_server_add_scene(sk_server* handle, sk_context* world, uint32_t* scene) {
  auto* s = reinterpret_cast<Server*>(handle);
  auto* ctx = reinterpret_cast<sk::Context*>(world);
  if (!s || !ctx) return SK_E_INVALID;
  if (ctx->device != s->config.device || !ctx->world.splats.ptr)
    return s->fail(SK_E_INVALID, "a scene is a context with a world on the server's device");
  const sk::World& w = ctx->world;
  const uint64_t bytes = sk::host::worldBytes(w.count, w.shDegree, 0, w.lod ? w.clusterCount : 0,
                                              w.lod ? w.leafRefCount : 0);
  std::lock_guard<std::mutex> g(s->mutex);
  if (s->residentBytes + bytes > s->config.memory_budget) {
    s->error = "the scene does not fit the memory budget";
    return SK_E_ADMISSION;
  }
  s->residentBytes += bytes;
  s->scenes.push_back({ctx, bytes});
  if (scene) *scene = static_cast<uint32_t>(s->scenes.size() - 1);
  return SK_OK;
}

sk_status sk_server_submit(sk_server* handle, const sk_request* r, uint64_t* id) {
  auto* s = reinterpret_cast<Server*>(handle);
  if (!s || !r) return SK_E_INVALID;
  std::lock_guard<std::mutex> g(s->mutex);
  if (r->scene >= s->scenes.size() || r->width == 0 || r->height == 0 || r->width > 16384 ||
      r->height > 16384 || r->frame.range_count > 1 || (r->frame.range_count == 1 && !r->frame.ranges)) {
    s->error = "invalid request";
    return SK_E_INVALID;
  }
  const sk::Context* ctx = s->scenes[r->scene].ctx;
  const bool lod = ctx->world.lod;
  if (lod && r->frame.range_count != 0) {
    s->error = "a request for a LOD scene draws its cut, not a range";
    return SK_E_INVALID;
  }
  sk::Pending p;
  p.id = ++s->nextId;
  p.request = *r;
  p.range = r->frame.range_count == 1 ? r->frame.ranges[0] : sk_range{0, ctx->world.count};
  if (p.range.offset > ctx->world.count || p.range.count > ctx->world.count - p.range.offset) {
    s->error = "invalid range";
    return SK_E_INVALID;
  }
  p.request.frame.ranges = nullptr;
  p.degree = static_cast<uint32_t>(std::max(0, std::min(r->frame.sh_degree, ctx->world.shDegree)));
  p.splats = lod ? ctx->world.lodCapacity : p.range.count;  // a cut draws at most its capacity
  p.priced = sk::kDrawBytesPerSplat * p.splats + uint64_t{r->width} * r->height * 4;
  p.arrival = sk::Clock::now();
  s->queue.push_back(p);
  ++s->submitted;
  s->arrived.notify_all();
  if (id) *id = p.id;
  return SK_OK;
}

sk_status sk_server_take_completions(sk_server* handle, sk_completion* out, uint32_t capacity,
                                     uint32_t* count) {
  auto* s = reinterpret_cast<Server*>(handle);
  if (!s || (!out && capacity)) return SK_E_INVALID;
  std::lock_guard<std::mutex> g(s->mutex);
  uint32_t n = 0;
  while (n < capacity && !s->done.empty()) {
    out[n++] = s->done.front();
    s->done.pop_front();
  }
  if (count) *count = n;
  return SK_OK;
}

sk_status sk_server_drain(sk_server* handle) {
  auto* s = reinterpret_cast<Server*>(handle);
  if (!s) return SK_E_INVALID;
  std::unique_lock<std::mutex> g(s->mutex);
  s->finished.wait(g, [s] { return s->completed == s->submitted; });
  return SK_OK;
}

sk_status sk_server_replay(sk_server* handle, const sk_request* requests, const double* arrival_us,
                           uint32_t count, sk_completion* out) {
  auto* s = reinterpret_cast<Server*>(handle);
  if (!s || (count && (!requests || !arrival_us || !out))) return SK_E_INVALID;
  std::vector<uint64_t> ids(count);
  const auto t0 = sk::Clock::now();
  for (uint32_t i = 0; i < count; ++i) {
    std::this_thread::sleep_until(t0 + std::chrono::nanoseconds(static_cast<int64_t>(arrival_us[i] * 1e3)));
    const sk_status st = sk_server_submit(handle, requests + i, &ids[i]);
    if (st != SK_OK) return st;
  }
  sk_server_drain(handle);
  std::vector<sk_completion> all;
  std::vector<sk_completion> chunk(256);
  uint32_t n = 0;
  do {
    sk_server_take_completions(handle, chunk.data(), 256, &n);
    all.insert(all.end(), chunk.begin(), chunk.begin() + n);
  } while (n > 0);
  std::sort(all.begin(), all.end(), [](const sk_completion& a, const sk_completion& b) { return a.id < b.id; });
  for (uint32_t i = 0; i < count; ++i) {
    const auto it = std::lower_bound(all.begin(), all.end(), ids[i],
                                     [](const sk_completion& c, uint64_t id) { return c.id < id; });
    out[i] = (it != all.end() && it->id == ids[i]) ? *it : sk_completion{ids[i], SK_E_INVALID, 0, 0, 0, 0};
  }
  return SK_OK;
}

void* sk_server_alloc_host(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, std::max<size_t>(bytes, 64)) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void sk_server_free_host(void* ptr) {
  if (ptr) cudaFreeHost(ptr);
}

}  // extern "C"
