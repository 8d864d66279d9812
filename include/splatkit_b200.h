/* splatkit-b200: the C ABI of the B200 splat frame pipeline.
 *
 * The entry points mirror the reference's renderer surface, splatkit::SplatRenderer
 * (packages/splatkit-engine/include/splatkit/rendering/SplatRenderer.h:36-160), and the
 * components its GPU tests drive directly (MetalVisibilityPass, MetalRadixSort,
 * MetalLodSelection). Plain C types only: host arrays are caller-owned and only read during a
 * call; device pointers (sk_*_device entry points) are CUDA device addresses the caller owns.
 *
 * Threading: one context per host thread for render calls ("render thread only",
 * SplatRenderer.h:32). sk_get_stats may be called from any thread.
 *
 * Errors: every call returns an sk_status. After a CUDA error the context latches failed and
 * every later call returns SK_E_DEVICE (MetalFrameLoop's failure latch,
 * splatkit-ios/.../metal/presentation/MetalFrameLoop.h:51-55). sk_last_error gives the text.
 * A failed upload keeps the previous world (SplatRenderer.h:85-87).
 */
#ifndef SPLATKIT_B200_H
#define SPLATKIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t sk_status;
#define SK_OK 0
#define SK_E_INVALID 1     /* bad argument, range or world; nothing was changed */
#define SK_E_OOM 2         /* device allocation failed; the previous state is kept */
#define SK_E_ADMISSION 3   /* a request does not fit the memory budget */
#define SK_E_DEVICE 4      /* CUDA error; the context is latched failed */
#define SK_E_TIMEOUT 5     /* a bounded device wait gave up (the frame is wrong) */
#define SK_E_UNSUPPORTED 6 /* a feature this build leaves out */
#define SK_E_NO_WORLD 7    /* no world uploaded */
#define SK_E_LIMIT 8       /* a size is beyond a fixed limit of the call; nothing was enqueued */

#define SK_FORMAT_RGBA8 0   /* 4 bytes per pixel, row 0 on top */
#define SK_FORMAT_RGBA32F 1 /* 16 bytes per pixel, row 0 on top */
#define SK_FORMAT_BGRA8 2   /* the reference's capture layout (MetalFrameCaptureTest.mm:57) */

typedef struct sk_context sk_context;

typedef struct {
  int32_t device;                /* CUDA device ordinal */
  uint32_t width, height;        /* draw extent of the headless target */
  int32_t image_format;          /* SK_FORMAT_RGBA8 or SK_FORMAT_RGBA32F on the device */
  uint32_t time_stages;          /* 1: per-stage CUDA events (stats.*_ms) and fragment counts;
                                    2: frame events only (stats.gpu_ms; keeps the stage kernels
                                    chained); 0: none */
} sk_config;

/* A SplatCloud (packages/splat-core/include/splat/formats/SplatCloud.h:30-51), structure of
 * arrays: count positions (xyz), covariances (xx, xy, xz, yy, yz, zz), colours (rgb in [0,1]),
 * alphas, and for sh_degree > 0, 3 * ((d+1)^2 - 1) harmonics floats per splat, channel fastest. */
typedef struct {
  const float* positions;
  const float* covariances;
  const float* colors;
  const float* alphas;
  const float* sh;
  uint32_t count;
  int32_t sh_degree;
} sk_cloud_view;

/* LodNode (packages/splat-core/include/splat/lod/LodTree.h:13-23), 24 bytes. */
typedef struct {
  float position[3];
  float size;
  uint32_t child_start;
  uint32_t child_count;
} sk_lod_node;

/* LodCluster (LodTree.h:28-35), 64 bytes. */
typedef struct {
  float center[3], radius;
  float extent[3], error;
  float color_variance, opacity;
  uint32_t node, child_start, child_count, leaf_start, leaf_count, subtree_leaves;
} sk_lod_cluster;

/* A LodTree (LodTree.h:47-55): the nodes as a cloud in layout order, the BFS layout, and the
 * selection data (clusters + leaf references). cluster_count 0: the selection data is built
 * at upload (MetalLodSelection.mm:68-74). */
typedef struct {
  sk_cloud_view nodes;
  const sk_lod_node* layout;
  uint32_t node_count;
  uint32_t leaf_count;
  const sk_lod_cluster* clusters;
  uint32_t cluster_count;
  const uint32_t* leaves;
  uint32_t leaf_ref_count;
} sk_lod_view;

typedef struct {
  uint32_t offset;
  uint32_t count;
} sk_range;

/* SplatRenderer::Frame (SplatRenderer.h:111-131) for the GPU order source. */
typedef struct {
  float view[16];  /* column major */
  float proj[16];  /* [0,1] depth perspective (Mat4::perspective) */
  float camera_position[3];
  float reveal_level; /* +inf when idle */
  const sk_range* ranges;
  uint32_t range_count;
  int32_t sh_degree; /* capped by the world */
  /* RevealUniform (splatkit-engine/include/splatkit/reveal/Reveal.h:25-35): splats below the
   * reveal level within `band` of it glow toward `tint` (SplatProjection.metalh:177-189);
   * band 0: no glow */
  float reveal_band, reveal_tint_amount, reveal_brightness_boost;
  float reveal_tint[3];
} sk_frame;

/* PartStyle (splatkit-ios/.../metal/cull/SplatVisibility.metal:5-11). */
typedef struct {
  float tint[3];
  float tint_amount;
  float brightness;
  float opacity;
  float reserved[2];
} sk_part_style;

/* RenderPolicy (packages/splatkit-engine/include/splatkit/rendering/RenderPolicy.h:17-40). */
typedef struct {
  float lod_error_pixels;
  uint32_t lod_splat_limit;
  float alpha_threshold;
  float subpixel_threshold;
  uint32_t enable_frustum_culling;
  uint32_t enable_early_termination;
  uint32_t sort_depth_bits; /* 16 or 32 */
  double background[3];
} sk_policy;

/* DeviceCapabilities (RenderPolicy.h:42-62), the fields this backend reports. */
typedef struct {
  uint32_t max_lod_capacity_splats;
  uint32_t min_residency_capacity_splats;
  uint32_t max_residency_capacity_splats;
  uint32_t supports_subgroups;
  uint32_t max_texture_dimension;
  uint32_t sorts_on_gpu;
  uint32_t selects_lod_on_gpu;
  uint64_t total_memory;
} sk_capabilities;

/* Frame statistics: the SplatRenderer getters (SplatRenderer.h:135-149) plus counters. */
typedef struct {
  uint64_t submitted_frames;
  uint64_t completed_frames;
  double gpu_ms;     /* whole frame */
  double select_ms;  /* LOD cut */
  double cull_ms;    /* visibility */
  double sort_ms;    /* depth sort */
  double bin_ms;     /* binning + tile sort */
  double composite_ms;
  uint32_t draw_count;     /* survivors of the cull */
  uint32_t selected_count; /* LOD cut size */
  uint32_t lod_limited;
  uint32_t lod_evaluated;
  uint32_t instances;      /* tile instances */
  uint32_t device_error;   /* SK_DEVERR bits of the last frame */
  uint64_t fragments;      /* blended pixel x splat pairs (counted when time_stages is 1) */
  float lod_pixels;        /* the adapted LOD threshold in use */
  uint32_t instances_read; /* tile-list records the composite read before termination */
} sk_stats;

/* ---- context (SplatRenderer lifetime, deviceCapabilities, applyRenderPolicy) ---------- */
sk_status sk_create(const sk_config* config, sk_context** out);
void sk_destroy(sk_context* ctx);
const char* sk_last_error(const sk_context* ctx);
sk_status sk_resize(sk_context* ctx, uint32_t width, uint32_t height);         /* drawExtent */
sk_status sk_device_capabilities(sk_context* ctx, sk_capabilities* out);        /* :56 */
sk_status sk_apply_render_policy(sk_context* ctx, const sk_policy* policy);     /* :62 */
void sk_default_policy(sk_policy* out);                                         /* RenderPolicy{} */
sk_status sk_available_memory(sk_context* ctx, uint64_t* bytes);                /* :70 */
int32_t sk_gpu_failed(sk_context* ctx);                                         /* :74 */

/* ---- worlds (SplatRenderer.h:85-97) ----------------------------------------------- */
sk_status sk_upload_world(sk_context* ctx, const sk_cloud_view* cloud, int32_t max_sh_degree);
sk_status sk_upload_lod_world(sk_context* ctx, const sk_lod_view* tree, int32_t max_sh_degree,
                              uint32_t budget);
/* .lodsplat files (splat-core/include/splat/lod/LodFile.h:12-36): the LOD tree format the
 * reference's offline builder writes (version 1, or 2 with selection data). */
typedef struct {
  uint32_t version;
  uint32_t node_count, leaf_count;
  int32_t sh_degree;
  uint32_t depth;             /* refinement rounds (the tree's depth) */
  uint32_t cluster_count;     /* version 2 */
  uint32_t leaf_ref_count;    /* version 2 */
  float bounds_min[3], bounds_max[3];
} sk_lodsplat_header;
/* readLodSplatHeader (LodFile.cpp:335-360): the header, checked against the file length. */
sk_status sk_lodsplat_read_header(const void* data, size_t size, sk_lodsplat_header* out);
/* decodeLodSplat (LodFile.cpp:362-423) into caller arrays sized from the header (any may be
 * NULL): positions 3n, covariances 6n, colors 3n, alphas n, sh 3((d+1)^2-1)n for
 * d = min(file degree, max_sh_degree), layout n, clusters and leaves (version 2). Checks the
 * header, the topology and depth, and the attribute ranges. */
sk_status sk_lodsplat_decode(const void* data, size_t size, int32_t max_sh_degree, float* positions,
                             float* covariances, float* colors, float* alphas, float* sh,
                             sk_lod_node* layout, sk_lod_cluster* clusters, uint32_t* leaves);
/* The file (in memory, or mapped from `path`) decoded and uploaded as sk_upload_lod_world
 * would; a version-1 file gets its selection data built at upload. */
sk_status sk_upload_lodsplat(sk_context* ctx, const void* data, size_t size, int32_t max_sh_degree,
                             uint32_t budget);
sk_status sk_upload_lodsplat_file(sk_context* ctx, const char* path, int32_t max_sh_degree,
                                  uint32_t budget);
/* writeLodSplat (LodFile.cpp:425-458): version 2 when the tree has selection data, else 1;
 * refuses an existing path. */
sk_status sk_write_lodsplat(const sk_lod_view* tree, const float* bounds_min,
                            const float* bounds_max, const char* path);

/* buildLodTree (splat-core/src/lod/LodTree.cpp:308-330, LodTree.h:58-75), built on the GPU
 * (current device): the cloud's splats become the leaves of an octree of merged nodes, laid out
 * breadth first. Morton keys and a radix sort on the device, then the octree one pass per level,
 * and the merges deepest level first. Given the same bounds the layout (child ranges) is the
 * reference builder's exactly; node attributes agree to a few ulp (the eigen-solve's acos/cos and
 * the surface formula's powf are the device's, not the host library's). octree_depth 0: 21;
 * cluster_leaves 0: 32. bounds NULL: the positions' own box. build_selection: also build the
 * selection data (buildLodSelectionData). The tree is read through sk_lod_tree_view (pointers
 * valid until sk_lod_tree_free). SK_E_LIMIT above 2^31 - 1 splats; SK_E_DEVICE on a CUDA error
 * (out of device memory included). */
typedef struct sk_lod_tree sk_lod_tree;
sk_status sk_build_lod_tree_device(const sk_cloud_view* cloud, const float* bounds_min,
                                   const float* bounds_max, uint32_t octree_depth,
                                   uint32_t cluster_leaves, int32_t build_selection,
                                   sk_lod_tree** out);
sk_status sk_lod_tree_view(const sk_lod_tree* tree, sk_lod_view* out, float* bounds_min,
                           float* bounds_max);
void sk_lod_tree_free(sk_lod_tree* tree);
sk_status sk_create_slab(sk_context* ctx, uint32_t capacity, int32_t sh_degree);
sk_status sk_upload_tile(sk_context* ctx, uint32_t offset, const sk_cloud_view* cloud);
sk_status sk_world_info(sk_context* ctx, uint32_t* count, int32_t* sh_degree);
/* Part labels of the flat world's records [offset, offset + count) (SplatCloud::labels), kept
 * until the next world upload; labels start at 0. */
sk_status sk_upload_labels(sk_context* ctx, uint32_t offset, const uint16_t* labels, uint32_t count);
/* The styles labelled parts are drawn with (Frame::labelStyles): record r with label l uses
 * palette[states[l]] (10 palette entries, states[l] < 10; a label without a state draws
 * unstyled). state_count 0: no styling. Applied in the cull (SplatVisibility.metal:69-84):
 * colour = mix(colour, tint, tint_amount) * brightness, opacity *= opacity, dropped below 2/255. */
sk_status sk_set_part_styles(sk_context* ctx, const sk_part_style* palette, const uint32_t* states,
                             uint32_t state_count);

/* ---- the frame (SplatRenderer::draw, :134) ------------------------------------------- */
/* Enqueues LOD cut, cull, sort, binning and composite; returns without waiting. A flat world keeps
 * two frames in flight (MetalFrameSlots.h:8): with both slots busy the call first finishes the
 * older frame. A LOD world keeps one. */
sk_status sk_draw(sk_context* ctx, const sk_frame* frame);
/* Waits for the last frame and copies its image (captureNextFrame). */
sk_status sk_read_image(sk_context* ctx, void* host, size_t bytes, int32_t format);
sk_status sk_wait_idle(sk_context* ctx);
/* captureNextFrame (MetalSplatRenderer.mm:310-316): the next sk_draw also copies its image, in the
 * context's own pixel format, into `host` (at least width x height x 4 or 16 bytes) on a copy
 * stream of its own, so the copy overlaps the frames drawn after it; sk_wait_capture blocks until
 * the image is there (a frame that is drawn again because its lists overflowed is copied
 * again). From the first capture on, frames alternate between two device images. The host
 * buffer must be pinned (sk_server_alloc_host, cudaHostAlloc) for the copy to overlap, and must
 * stay untouched until the wait returns. One capture may wait for the next frame at a time. */
sk_status sk_capture_next_frame(sk_context* ctx, void* host, size_t bytes, int32_t format,
                                uint64_t* ticket);
sk_status sk_wait_capture(sk_context* ctx, uint64_t ticket);
sk_status sk_get_stats(sk_context* ctx, sk_stats* out);
/* Switches the event timing of later frames (sk_config.time_stages' values); waits for the
 * frame in flight first. */
sk_status sk_set_timing(sk_context* ctx, uint32_t time_stages);
/* How each binning cell's front-to-back list is built. SK_BINNING_AUTO: written in place from
 * per-block cell counts when the target has at most 4096 cells (32 x 32 pixels each), else by
 * a stable sort of (cell, splat) pairs; SK_BINNING_SORTED: always the sort. Both give the same
 * lists. Waits for the frame in flight first. */
#define SK_BINNING_AUTO 0u
#define SK_BINNING_SORTED 1u
sk_status sk_set_binning(sk_context* ctx, uint32_t mode);

/* Readbacks of the last frame for parity checks: the survivors in source order (keys and
 * 32-byte projected records), the depth order (indices into the projected records) and the
 * LOD cut. Each returns the element count in *count and copies min(count, capacity). */
sk_status sk_read_visible(sk_context* ctx, uint32_t* keys, void* projected, uint32_t capacity,
                          uint32_t* count);
sk_status sk_read_order(sk_context* ctx, uint32_t* order, uint32_t capacity, uint32_t* count);
sk_status sk_read_cut(sk_context* ctx, uint32_t* indices, uint32_t capacity, uint32_t* count,
                      uint32_t* lod_counters6);
/* The last frame's binning lists: ranges[2 * c], ranges[2 * c + 1] = [start, end) of 32x32
 * binning cell c (row major) in `values`, which holds projected-record indices front to back
 * per cell. ranges needs 2 * cells words; *count receives the number of list entries. */
sk_status sk_read_tile_lists(sk_context* ctx, uint32_t* ranges, uint32_t* values,
                             uint32_t capacity, uint32_t* count);

/* ---- batched multi-view rendering ---------------------------------------------------------
 * Many views, of one or several contexts' resident worlds and of different target sizes, drawn
 * together: each stage runs once over the whole batch. A view of a LOD world first selects its
 * cut on the batch's stream (with the context's current LOD threshold and splat limit, which the
 * batch reads but does not adapt) and is drawn from the cut. The same frame pipeline and
 * arithmetic as sk_draw, so every view's image and survivor count equal what sk_draw gives for
 * that view with 16-bit depth keys. Submissions go round robin to `lanes` CUDA streams and
 * overlap on the device; a submission's results (RGBA8 images, survivor counts) are copied to
 * pinned host memory by the same stream and stay readable until its lane is reused, `lanes`
 * submissions later. The contexts' worlds must not be replaced while a submission that draws
 * them is in flight. The batch keeps no reference to a context beyond the submit call.
 * A lane's device buffers grow stream-ordered (cudaMallocAsync on the lane's stream, at least
 * half again each time), so growing one lane never waits for the others. From the first batch or
 * server on, the device's default memory pool keeps the memory lanes give back, for later lanes
 * of any batch or server in the process; cudaMemPoolTrimTo on that pool returns it. */
typedef struct sk_batch sk_batch;

typedef struct {
  int32_t device;
  uint32_t lanes;      /* submissions in flight, >= 1 */
  uint32_t max_views;  /* most views one submission may hold, 1..65536 */
  uint32_t use_graphs; /* 1: each lane captures its stage sequence as a CUDA graph and replays it
                          while its views keep their worlds, ranges and sizes */
} sk_batch_config;

typedef struct {
  sk_context* world;   /* the context whose resident world this view draws */
  sk_frame frame;      /* camera; at most one range (none: the whole world; a LOD world: none) */
  uint32_t width, height;
} sk_batch_view;

typedef struct {
  uint32_t views;
  uint32_t visible;    /* survivors over all views */
  uint32_t instances;  /* tile instances over all views */
  uint32_t device_error;
  double gpu_ms;       /* the submission's stages, device time */
  uint64_t fragments;
} sk_batch_stats;

sk_status sk_batch_create(const sk_batch_config* config, sk_batch** out);
void sk_batch_destroy(sk_batch* batch);
const char* sk_batch_last_error(const sk_batch* batch);
/* The policy every view is drawn with; sort_depth_bits must be 16. */
sk_status sk_batch_apply_render_policy(sk_batch* batch, const sk_policy* policy);
/* Enqueues the views and returns at once with a ticket (waits only when the next lane is still
 * busy). All views must draw the same harmonics degree (min of the frame's and the world's). */
sk_status sk_batch_submit(sk_batch* batch, const sk_batch_view* views, uint32_t count,
                          uint64_t* ticket);
sk_status sk_batch_poll(sk_batch* batch, uint64_t ticket, int32_t* done);
sk_status sk_batch_wait(sk_batch* batch, uint64_t ticket);
/* View `view` of a completed submission as RGBA8 rows, top row first (waits if needed). */
sk_status sk_batch_read_image(sk_batch* batch, uint64_t ticket, uint32_t view, void* host,
                              size_t bytes);
sk_status sk_batch_view_visible(sk_batch* batch, uint64_t ticket, uint32_t view,
                                uint32_t* visible);
sk_status sk_batch_get_stats(sk_batch* batch, uint64_t ticket, sk_batch_stats* out);

/* Launch parameters the autotuner chooses among; none changes a result bit. */
typedef struct {
  uint32_t emission_balanced; /* tile binning: 0 walks each warp's splats one by one, 1 spreads
                                 each warp's tile instances evenly over its lanes */
  uint32_t sort_tile_keys;    /* keys per radix-sort scatter tile: 2048, 4096 or 6144 */
  uint32_t lanes;             /* submissions in flight (<= the batch's lanes) */
  uint32_t sorted_lists;      /* cell lists: 0 written in place per view where every view has at
                                 most 4096 binning cells, 1 always by the batch-wide stable sort
                                 of (cell, splat) pairs */
  double gpu_ms;              /* autotune: device time of the chosen kernels for the sample */
  double views_per_s;         /* autotune: throughput with `lanes` in flight, images read back */
} sk_batch_tuning;
/* Times the sample views under every cell-list construction, emission strategy and sort tile
 * size (device time), then with 1..lanes submissions in flight (host time, images read back),
 * and keeps the fastest.
 * Waits for submissions in flight first; their tickets stay readable until their lanes are
 * reused. */
sk_status sk_batch_autotune(sk_batch* batch, const sk_batch_view* views, uint32_t count,
                            sk_batch_tuning* out);
sk_status sk_batch_set_tuning(sk_batch* batch, const sk_batch_tuning* tuning);

/* ---- serving: continuous batching of render requests --------------------------------------
 * A server holds resident scenes (contexts with flat or LOD worlds, added once) and a scheduler
 * thread.
 * Requests are queued as they arrive; whenever one of the server's lanes is free the scheduler
 * takes the queued requests in arrival order (up to max_batch_views views and
 * max_batch_splats drawn records, within the memory budget) and runs them as one batch, so
 * requests that arrive while others are on the GPU join the next batch and their work overlaps
 * with the batches in flight. Each request's RGBA8 image is copied straight into the caller's
 * buffer. Admission: a request is priced like the reference's gpuWorldBytes (52 bytes per drawn
 * record plus its image) and waits until the priced bytes of the requests in flight leave room
 * for it under memory_budget minus the resident scenes; a request that can never fit, or that
 * has waited longer than max_queue_ms, completes with SK_E_ADMISSION. A request for a LOD scene
 * is priced at the scene's cut capacity; its cut is selected with the scene's LOD threshold,
 * which every completed request of the scene then adapts (LodThreshold::update,
 * splatkit-engine/include/splatkit/rendering/LodThreshold.h:27-36), as the scene's own frames
 * would. Results equal sk_draw's for the same view (16-bit depth keys, default policy).
 * At creation the server gives the device's memory pool its lanes' working size (about 192
 * bytes per drawn record of max_batch_splats per lane, at most a quarter of memory_budget), so
 * lanes that grow while requests wait take pooled memory instead of a driver allocation. */
typedef struct sk_server sk_server;

typedef struct {
  int32_t device;
  uint32_t lanes;            /* batches in flight, >= 1 */
  uint32_t max_batch_views;  /* 1..65536 */
  uint64_t max_batch_splats; /* drawn records per batch (bounds each lane's scratch) */
  uint64_t memory_budget;    /* bytes for resident scenes plus requests in flight */
  double max_queue_ms;       /* shed requests that waited longer; <= 0: never */
} sk_server_config;

typedef struct {
  uint32_t scene;  /* from sk_server_add_scene */
  sk_frame frame;  /* camera; at most one range (none: the whole scene) */
  uint32_t width, height;
  void* image;     /* caller host buffer of width * height * 4 bytes, or NULL; written when the
                      request completes; pinned memory (sk_server_alloc_host) copies fastest */
} sk_request;

typedef struct {
  uint64_t id;
  sk_status status;     /* SK_OK, SK_E_ADMISSION (shed or can never fit), SK_E_TIMEOUT */
  uint32_t visible;     /* survivors of the cull */
  uint32_t batch_views; /* views in the batch that drew it */
  double queue_ms;      /* arrival to batch start on the host */
  double latency_ms;    /* arrival to image on the host */
} sk_completion;

sk_status sk_server_create(const sk_server_config* config, sk_server** out);
void sk_server_destroy(sk_server* server);
const char* sk_server_last_error(const sk_server* server);
/* Adds the context's resident world (flat or LOD) as a scene; the context must outlive the
 * server and keep its world while the server runs, and is not drawn with directly meanwhile (the
 * server's thread adapts a LOD scene's threshold in it). */
sk_status sk_server_add_scene(sk_server* server, sk_context* world, uint32_t* scene);
/* Queues a request (any thread); its arrival time is now. */
sk_status sk_server_submit(sk_server* server, const sk_request* request, uint64_t* id);
/* Moves up to `capacity` completions out, oldest first. */
sk_status sk_server_take_completions(sk_server* server, sk_completion* out, uint32_t capacity,
                                     uint32_t* count);
/* Waits until every submitted request has completed. */
sk_status sk_server_drain(sk_server* server);
/* Replays an arrival trace: request i is submitted at arrival_us[i] microseconds after the call
 * starts (the calling thread sleeps between arrivals), then waits for all of them; out[i]
 * receives request i's completion. */
sk_status sk_server_replay(sk_server* server, const sk_request* requests, const double* arrival_us,
                           uint32_t count, sk_completion* out);
/* Pinned host memory for request images (sk_server_free_host releases it). */
void* sk_server_alloc_host(size_t bytes);
void sk_server_free_host(void* ptr);

/* ---- component operators over caller device memory ----------------------------------- */
/* MetalRadixSort (splatkit-ios/.../metal/sort/MetalRadixSort.h:13-54): stable ascending argsort
 * of min(*d_count, capacity) keys (d_count is a device word), 16 or 32 bits; d_keys is left
 * unchanged; d_order receives the key positions in sorted order. d_workspace holds
 * sk_sort_workspace_bytes(capacity) device bytes; calls on one workspace must be
 * stream-ordered. d_error (device word) receives SK_DEVERR bits. stream: a cudaStream_t. */
size_t sk_sort_workspace_bytes(uint32_t capacity);
sk_status sk_radix_argsort_device(const uint32_t* d_keys, const uint32_t* d_count,
                                  uint32_t capacity, int32_t bits, uint32_t* d_order,
                                  void* d_workspace, size_t workspace_bytes, uint32_t* d_error,
                                  void* stream);

/* The same argsort with no workspace argument and no allocation. No counterpart in the
 * reference: its Metal sort owns its buffers. For callers that may not allocate device memory
 * while they run (cudaMalloc/cudaFree synchronise the whole device, which a render callback
 * with a frame deadline cannot afford) and for code that owns no device allocator. The call
 * allocates nothing and calls no allocating library; it enqueues two small memsets and the
 * sort kernels on `stream` and returns.
 *
 * Limit: capacity <= SK_NOALLOC_SORT_MAX_KEYS (1,048,576 keys); a larger capacity returns
 * SK_E_LIMIT and enqueues nothing. The workspace is a 13,115,648-byte array of this library's
 * device module, zero when the module loads. The histogram accumulators and tile counters in
 * it must be zero when a sort starts; each sort leaves them at zero and each call clears them
 * again first, so the caller clears nothing. d_keys, d_count, d_order, d_error and bits mean
 * what they mean for sk_radix_argsort_device.
 *
 * Setup: the first call on each device (the device current on the calling thread) looks up the
 * array's device address, which may load the module; make that first call before any stream
 * capture. The address is kept for the life of the process: after cudaDeviceReset (or anything
 * else that destroys the device's primary context) the module reloads elsewhere, so do not call
 * this entry point on that device again. There is one array per device: calls on one device
 * whose sorts may overlap in time (different streams without an event between them, or several
 * host threads) race on it and give wrong orders. Keep them ordered on one stream. */
#define SK_NOALLOC_SORT_MAX_KEYS (1u << 20)
sk_status sk_radix_argsort_noalloc(const uint32_t* d_keys, const uint32_t* d_count,
                                   uint32_t capacity, int32_t bits, uint32_t* d_order,
                                   uint32_t* d_error, void* stream);

/* ---- host-side world preparation (no device needed) ----------------------------------- */
/* Harmonics words per splat in the device layout: the reference's packed stride
 * (GpuLayout.cpp:66-70) rounded up to whole 16-byte groups. */
uint32_t sk_sh_device_stride(int32_t degree);
/* packSplatRange (splatkit-engine/src/rendering/GpuLayout.cpp:122-137): records
 * [offset, offset + count) of the cloud as 32-byte GpuSplat records. */
sk_status sk_pack_splats(const sk_cloud_view* cloud, uint32_t offset, uint32_t count, void* out);
/* packShRange float16 (GpuLayout.cpp:92-113) at `stride` words per splat (>= packed stride). */
sk_status sk_pack_sh(const sk_cloud_view* cloud, int32_t degree, uint32_t offset, uint32_t count,
                     uint32_t* out, uint32_t stride);
/* buildLodSelectionData (splat-core/src/lod/LodSelection.cpp:47-133) of a breadth-first laid-out
 * tree (SK_E_INVALID otherwise). Pass null outputs to learn the counts first. */
sk_status sk_build_lod_selection(const sk_lod_view* tree, sk_lod_cluster* clusters,
                                 uint32_t cluster_capacity, uint32_t* cluster_count,
                                 uint32_t* leaves, uint32_t leaf_capacity, uint32_t* leaf_count);
/* The deepest node depth of a BFS-laid-out tree (validateLodTree's value,
 * splat-core/src/lod/LodFile.cpp:336-344), or -1 when the topology is invalid. */
int64_t sk_lod_depth(const sk_lod_node* layout, uint32_t node_count, uint32_t leaf_count);
/* gpuWorldBytes (GpuLayout.cpp:72-77): the device bytes a world of this shape is priced at. */
uint64_t sk_world_bytes(uint64_t records, int32_t sh_degree, uint64_t draw_capacity,
                        uint64_t clusters, uint64_t leaf_refs);
/* LodThreshold::update (splatkit-engine/include/splatkit/rendering/LodThreshold.h:27-36) on
 * state[0] = policy pixels, state[1] = current pixels; returns the new threshold. */
float sk_lod_threshold_update(float* state, uint32_t selected, uint32_t limited, uint32_t limit);

#ifdef __cplusplus
}
#endif

#endif /* SPLATKIT_B200_H */
