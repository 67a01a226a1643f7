// Launchers of the trace kernels (implemented in kernels_*.cu).
#pragma once
#include <cuda_runtime.h>
#include "device_scene.h"

namespace slim {

// One thread per sample, the whole path in one kernel.
cudaError_t launch_render_fused(const DevScene &S, const DevFrame &F, int block, cudaStream_t stream);

// First closest hit of every primary ray.
cudaError_t launch_trace_primary(const DevScene &S, const SlimCameraRayProjection &P, uint32_t width, uint32_t height,
                                 int *geometry_ids, uint32_t *primitive_ids, float *distances, uint8_t *from_behind,
                                 uint32_t *error_flags, cudaStream_t stream);

// Wavefront form: stage kernels over compacted ray queues.
struct WavefrontBuffers {
    // path state, one slot per sample
    float4 *path_color;        // accumulated color (xyz) | depth (w)
    float4 *path_throughput;   // throughput (xyz) | next throughput .x packed later
    float4 *path_next;         // next throughput (xyz)
    // ray queues (ping-pong): origin.xyz|pixel, direction.xyz|flags
    float4 *rays[2];
    uint32_t *queue_count;     // [0..1] ray queue sizes, [2] shadow queue size
    // per-ray hit records
    float4 *hits;              // 4 float4 per ray slot
    // shadow rays: origin.xyz|ray slot, direction.xyz|max distance
    float4 *shadow_rays;
    uint32_t *shadow_meta;     // (ray slot << 8) | light index
    uint32_t *shadow_mask;     // per ray slot: bit i set = light i occluded
    uint32_t capacity;         // samples
    uint32_t shadow_capacity;  // shadow ray slots
};
cudaError_t launch_render_wavefront(const DevScene &S, const DevFrame &F, const WavefrontBuffers &B, int block,
                                    cudaStream_t stream);

// GPU refit of the scene BVH: recomputes every node's bounds bottom-up from
// the geometries' world AABBs, keeping the uploaded topology.
cudaError_t launch_refit_scene_bvh(const DevScene &S, float4 *scene_nodes, const uint32_t *parent_order,
                                   uint32_t node_count, cudaStream_t stream);

}  // namespace slim
