// Launchers of the trace kernels (implemented in kernels_*.cu).
#pragma once
#include <cuda_runtime.h>
#include "device_scene.h"

namespace slim {

// Stages of a frame, for per-stage timing and work counters (16 counter
// slots per stage in DevFrame::counters).
enum Stage : int {
    STAGE_FUSED = 0, STAGE_EXTEND, STAGE_SHADOW_GEN, STAGE_SHADOW, STAGE_SHADE, STAGE_REFIT, STAGE_SHADOW_MESH, STAGE_COUNT
};
constexpr int kCountersPerStage = 16;

// Optional CUDA-event timing around each stage launch.
struct StageTimer {
    virtual void begin(int stage, cudaStream_t stream) = 0;
    virtual void end(int stage, cudaStream_t stream) = 0;
    virtual ~StageTimer() = default;
};

// One thread per sample, the whole path in one kernel.
cudaError_t launch_render_fused(const DevScene &S, const DevFrame &F, int block, cudaStream_t stream,
                                StageTimer *timer);

// First closest hit of every primary ray.
cudaError_t launch_trace_primary(const DevScene &S, const SlimCameraRayProjection &P, uint32_t width, uint32_t height,
                                 int *geometry_ids, uint32_t *primitive_ids, float *distances, uint8_t *from_behind,
                                 uint32_t *error_flags, cudaStream_t stream);

// Wavefront form: stage kernels over compacted ray queues.
struct WavefrontBuffers {
    float4 *path_color;              // per sample: accumulated colour (xyz), depth (w)
    float4 *path_throughput;         // per sample: throughput (xyz)
    float4 *rays[2];                 // ping-pong ray queues, 2 float4 per ray
    uint32_t *queue_count;           // [0..1] ray queues, [2] shadow queue, [3] pairs, [4] pair cursor
    float4 *hits;                    // 3 float4 per queue slot
    float4 *shadow_rays;             // 2 float4 per shadow ray
    unsigned long long *shadow_mask; // per queue slot: occluded-light bits
    float4 *pairs;                   // shadow ray x mesh instance candidates, 3 float4 each
    uint32_t capacity;               // samples
    uint32_t shadow_capacity;        // shadow ray slots
    uint32_t pair_capacity;          // candidate pair slots
};
cudaError_t launch_render_wavefront(const DevScene &S, const DevFrame &F, const WavefrontBuffers &B, int block,
                                    cudaStream_t stream, StageTimer *timer);

// GPU refit of the scene BVH: recomputes every node's bounds bottom-up from
// the geometries' world AABBs, keeping the uploaded topology.
cudaError_t launch_refit_scene_bvh(const DevScene &S, float4 *scene_nodes, const uint32_t *parent_order,
                                   uint32_t node_count, cudaStream_t stream, StageTimer *timer);

}  // namespace slim
