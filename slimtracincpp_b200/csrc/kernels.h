// Launchers of the trace kernels (implemented in kernels_*.cu).
#pragma once
#include <cuda_runtime.h>
#include "launch_count.h"
#include "device_scene.h"

namespace slim {

// Stages of a frame, for per-stage timing and work counters (16 counter
// slots per stage in DevFrame::counters).
enum Stage : int {
    STAGE_FUSED = 0, STAGE_EXTEND, STAGE_SHADOW_GEN, STAGE_SHADOW, STAGE_SHADE, STAGE_REFIT, STAGE_SHADOW_MESH,
    STAGE_CACHE, STAGE_CACHE_TRAIN, STAGE_CACHE_QUERY, STAGE_TAIL, STAGE_COUNT
};
constexpr int kCountersPerStage = 16;

// Optional CUDA-event timing around each stage launch.
struct StageTimer {
    virtual void begin(int stage, cudaStream_t stream) = 0;
    virtual void end(int stage, cudaStream_t stream) = 0;
    virtual ~StageTimer() = default;
};

// One thread per sample, the whole path in one kernel; `short_paths`: no
// path can bounce (the build with more blocks per SM than the one for
// bouncing paths).
cudaError_t launch_render_fused(const DevScene &S, const DevFrame &F, int block, cudaStream_t stream,
                                StageTimer *timer, bool short_paths = false);

// First closest hit of every primary ray.
cudaError_t launch_trace_primary(const DevScene &S, const SlimCameraRayProjection &P, uint32_t width, uint32_t height,
                                 int *geometry_ids, uint32_t *primitive_ids, float *distances, uint8_t *from_behind,
                                 uint32_t *error_flags, cudaStream_t stream);

// Single-ray pick behind a pixel (scene/selection.h:36-80) into device `out`.
cudaError_t launch_pick(const DevScene &S, const SlimCameraRayProjection &P, int x, int y, SlimPick *out,
                        uint32_t *error_flags, cudaStream_t stream);

// Wavefront form: stage kernels over compacted ray queues.
struct WavefrontBuffers {
    float4 *path_color;              // per sample: accumulated colour (xyz), depth (w)
    float4 *path_throughput;         // per sample: throughput (xyz)
    float4 *rays[2];                 // ping-pong ray queues, 2 float4 per ray
    uint32_t *queue_count;           // [0..1] ray queues, [2] shadow queue, [3] pairs, [4] pair cursor (8 slots)
    float4 *hits;                    // hit records: three planes of `capacity` float4
    float4 *shadow_rays;             // 2 float4 per shadow ray
    unsigned long long *shadow_mask; // per queue slot: occluded-light bits
    float4 *pairs;                   // shadow ray x mesh instance candidates, 3 float4 each
    uint32_t capacity;               // samples
    uint32_t shadow_capacity;        // shadow ray slots
    uint32_t pair_capacity;          // candidate pair slots
};

// Radiance cache in a wavefront frame (no counterpart in the reference).
// Paths stop at vertex `depth`: misses and emissive hits there finish as
// usual, every other hit becomes a query whose answer -- the network's
// (ON), nothing (TRUNCATE) or the tracer's own full-depth continuation
// (EXACT, a check of the plumbing) -- is added with the path throughput.
// With ON and a trainer, `train_capacity` queries (stratified over all of
// them) are traced on to max_depth from the same vertex; their radiance is
// the training target of the frame's Adam steps.
struct CacheTrainer {
    virtual cudaError_t step(const float4 *features, const float4 *targets, uint32_t samples, const uint32_t *count,
                             uint32_t offset, cudaStream_t stream) = 0;
    virtual ~CacheTrainer() = default;
};
struct CacheFrame {
    int mode = 0;                  // SLIM_CACHE_*
    uint32_t depth = 0;            // path vertex the cache answers at (>= 2)
    float4 *features = nullptr;    // 4 per query (capacity: one per sample)
    float4 *aux = nullptr;         // 2 per query: (ray origin, pixel) (ray direction, cone pixel)
    float4 *radiance = nullptr;    // 1 per query
    uint32_t *counts = nullptr;    // [0] queries, [1] training paths
    uint32_t train_capacity = 0;   // training paths per frame (every query in EXACT mode)
    float4 *t_features = nullptr, *t_targets = nullptr, *t_color = nullptr, *t_through = nullptr;
    uint32_t *frame_counter = nullptr;  // device: cache frames so far (moves the stratified
                                        // selection from frame to frame; counted on the device
                                        // so captured graphs replay correctly)
    uint32_t batch = 0;            // samples per training step
    const uint8_t *weights = nullptr;   // bf16 weight image
    CacheTrainer *trainer = nullptr;    // null: no training this frame
    // Overlapped training (ON mode with a trainer): the training paths of this
    // frame are traced and trained on `train_stream` with their own queues,
    // while the frame's stream answers the queries with the weights trained
    // through the previous frame.  The frame's stream waits for the previous
    // frame's training (`trained`) before it selects new training paths and
    // before it queries the network; `selected` hands the new set over.
    cudaStream_t train_stream = nullptr;      // null: train in order on the frame's stream
    cudaEvent_t selected = nullptr, trained = nullptr;
    const WavefrontBuffers *train_queues = nullptr;
    const uint8_t *train_weights = nullptr;   // image the training updates; copied into `weights`
                                              // (what the queries read) once per frame
    // Self-training (train_suffix > 0): the training paths stop train_suffix
    // bounces past the cache vertex and query the cache there; those queries
    // go to their own buffers (one slot per training path).
    uint32_t train_suffix = 0;
    float4 *s_features = nullptr, *s_aux = nullptr, *s_radiance = nullptr;
    uint32_t *s_count = nullptr;
    // Each query also keeps its path's state (colour + canvas depth,
    // throughput), so queries gathered by several row bands -- each with its
    // own path slots -- resolve together (null: read the path slots).
    float4 *q_color = nullptr, *q_through = nullptr;
    // Each query's hit record (3 float4), copied with the training selection
    // into the training queues, so training paths start at their cache vertex
    // without tracing the segment to it again (null: they retrace it).
    float4 *q_hit = nullptr;
    // Which part of a cache frame a launch runs: the whole frame, the rounds
    // up to the cache vertex and the gather only (a row band), or the cache
    // phase only (once the bands have joined).
    int part = 0;
};
constexpr int kCachePartWhole = 0, kCachePartGather = 1, kCachePartPhase = 2;

// Download of a frame's (or band's) canvas rows while its later bounces
// still run (no counterpart in the reference).  After the first round every
// path that ends at its first hit has its pixel, so the rows are copied to
// the host then, on copy_stream; the later rounds write the pixels they
// finish straight into the host canvas (pinned and mapped into the device's
// address space), once the copy has landed.
constexpr uint32_t kPixelChunks = 3;     // first-round shade launches, each followed by its rows' copy
struct FrameDownload {
    cudaStream_t copy_stream;
    cudaEvent_t depths_done, copied;      // recorded by the launcher
    cudaEvent_t pixels_done[kPixelChunks];
    void *host_pixels, *host_depths;      // destinations of the copies
    const void *dev_pixels, *dev_depths;  // sources of the copies
    size_t depth_bytes;
    size_t pixel_row_bytes;               // canvas pixel bytes per sample row
    float4 *mapped_pixels;                // the whole host canvas, as the device sees it
    float *mapped_depths;
};

cudaError_t launch_render_wavefront(const DevScene &S, const DevFrame &F, const WavefrontBuffers &B, int block,
                                    cudaStream_t stream, StageTimer *timer, const CacheFrame *cache = nullptr,
                                    const FrameDownload *download = nullptr);

// Batched requests (no counterpart in the reference): many requests, each
// with its own scene, camera and canvas, traced together over one set of
// queues.  Their pixels are cut into tiles; consecutive tiles fill waves of
// at most the queue capacity, and every wave is one multi-request frame
// whose stage kernels look up each path's scene and canvas by request.
struct BatchWave {
    uint32_t first_tile, tile_count;   // into BatchFrame::tiles
    uint32_t samples;                  // path slots of the wave
    uint32_t max_depth, max_lights;    // over the wave's requests
    uint32_t cache_paths;              // non-zero: a request of the wave uses the radiance cache
};
struct BatchFrame {
    DevScene shared;                   // mesh and texture arrays every request shares
    DevFrame frame;                    // error flags and counters every request shares
    const DevScene *scenes;            // device table, one entry per request
    const DevFrame *frames;            // device table, one entry per request
    const uint4 *tiles;                // device: (request, first pixel, pixel count, first slot in its wave)
    const BatchWave *waves;            // host
    uint32_t wave_count;
    const CacheFrame *cache;           // null: no request uses the cache
    // Waves without cache paths alternate between two lanes (the launching
    // stream with the first queue set, lane_stream with the second), so the
    // tail of one wave's persistent launches overlaps the next wave's work;
    // waves with cache paths stay on the first lane, which owns the cache's
    // buffers.  Null lane_stream or lane_queues: every wave on one lane.
    cudaStream_t lane_stream;
    const WavefrontBuffers *lane_queues;
    cudaEvent_t lane_fork, lane_join;
    // Requests without the cache in one persistent launch (plan.persistent):
    // their pixels are in no wave; the launch runs on the second lane (or
    // first, before the waves, with one lane) beside the cache requests' waves.
    const uint32_t *p_requests, *p_prefix;
    uint32_t p_count, p_total;
    uint32_t *p_cursor;
};
cudaError_t launch_render_batch(const BatchFrame &BF, const WavefrontBuffers &B, int block, cudaStream_t stream,
                                StageTimer *timer);
// Every pixel of the listed requests (prefix[k] = first pixel of request
// requests[k] in one flattened queue of `total` pixels) rendered by one
// persistent launch (kernels_fused.cu k_batch_persistent); `cursor` is a
// device counter the launch clears first.
cudaError_t launch_batch_persistent(const DevScene *scenes, const DevFrame *frames, const uint32_t *requests,
                                    const uint32_t *prefix, uint32_t count, uint32_t total, uint32_t *cursor,
                                    uint32_t *error_flags, unsigned long long *counters, cudaStream_t stream);

// GPU refit of the scene BVH: recomputes every node's bounds bottom-up from
// the geometries' world AABBs, keeping the uploaded topology.
cudaError_t launch_refit_scene_bvh(const DevScene &S, float4 *scene_nodes, const uint32_t *parent_order,
                                   uint32_t node_count, cudaStream_t stream, StageTimer *timer);

// bmp2texture's texel-quad baker on the device (kernels_bake.cu): the
// arguments and results of slimBakeTexture, on `stream`, synchronous.
int bake_texture_gpu(const uint8_t *bgr, uint32_t width, uint32_t height, uint32_t channels, uint32_t flags,
                     SlimTexture *texture, SlimTextureMip *mips, SlimTexelQuad *quads, uint32_t *mip_count,
                     uint32_t *quad_count, cudaStream_t stream);

}  // namespace slim
