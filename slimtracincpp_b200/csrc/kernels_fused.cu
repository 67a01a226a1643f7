// The fused (one thread per sample, whole path in one kernel) form of the
// trace path, plus the primary-hit kernel used for id/distance parity.
// Mirrors d_render (renderer/renderer_GPU.h:22-46) -> renderPixel
// (renderer/ray_tracer.h:19-161).
#include "kernels.h"
#include "tracer_core.cuh"

namespace slim {
namespace dev {

template <bool COUNT>
SLIM_D void flush_work(unsigned long long *counters, const Work &w) {
    if (!COUNT || !counters) return;
    // slots 0-8 as every stage counts them, 9-12 the any-hit parts
    uint32_t v[13] = {w.primary, w.shadow, w.bounce, w.scene_nodes, w.mesh_nodes, w.triangles,
                      w.geometries, w.mesh_fetches, w.taps, w.any_scene_nodes, w.any_mesh_nodes,
                      w.any_triangles, w.any_geometries};
#pragma unroll
    for (int k = 0; k < 13; k++) {
        unsigned long long s = v[k];
        for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
        if ((threadIdx.x & 31) == 0 && s) atomicAdd(counters + k, s);
    }
}

// renderPixelBeauty / renderPixelDebugMode for one sample.
template <bool COUNT>
SLIM_D void render_sample(const DevScene &S, const DevFrame &F, int x, int y, uint32_t *stack,
                          uint32_t *mesh_stack, uint32_t &err, Work &w, float3 &out_color, float &out_depth) {
    const SlimCameraRayProjection &P = F.projection;
    const SlimRayTracerSettings &st = F.settings;
    if (st.render_mode != SLIM_RENDER_BEAUTY) {
        float scaling = F.cones_per_pixel ? pixel_scaling(P, x, y) : 0.0f;
        float3 cam = f3(P.camera_position.x, P.camera_position.y, P.camera_position.z);
        Ray ray;
        reset(ray, cam, normalized(primary_direction(P, x, y)));
        Hit hit;
        bump<COUNT>(w.primary);
        float3 color = f3(0, 0, 0);
        float depth = INFINITY;
        Surface s;
        int g = scene_trace<COUNT>(S, ray, hit, false, INFINITY, stack, mesh_stack, err, w);
        if (g >= 0) {
            Geo geo = load_geo(S, (uint32_t)g);
            Mat m = load_mat(S, geo.material);
            prepare_for_shading<COUNT>(S, geo, m, ray, hit, scaling, s, w);
            depth = depth_at(P, hit.position);
            switch (st.render_mode) {
                case SLIM_RENDER_UVS: color = f3(hit.u, hit.v, 1.0f); break;
                case SLIM_RENDER_DEPTH: { float d = 4.0f / hit.distance; color = f3(d, d, d); } break;
                case SLIM_RENDER_NORMALS:
                    color = f3(fmaf(hit.normal.x, 0.5f, 0.5f), fmaf(hit.normal.y, 0.5f, 0.5f), fmaf(hit.normal.z, 0.5f, 0.5f));
                    break;
                case SLIM_RENDER_NORMAL_MAP: {
                    float3 n = sample_slot<COUNT>(S, m, 1, hit.u, hit.v, hit.uv_coverage, w);
                    color = f3(fmaf(n.x, 0.5f, 0.5f), fmaf(n.y, 0.5f, 0.5f), fmaf(n.z, 0.5f, 0.5f));
                } break;
                case SLIM_RENDER_MIP_LEVEL:
                    if (S.texture_count) {
                        DevTexture t0 = S.textures[0];
                        color = color_of_id(st.mip_level_colors[mip_level(hit.uv_coverage * (float)(t0.width * t0.height), t0.mip_count)]);
                    } else color = f3(0.5f, 0.5f, 0.5f);
                    break;
                default: break;
            }
        }
        out_color = color;
        out_depth = depth;
        return;
    }
    PathState p;
    path_start<COUNT>(F, x, y, p, w);
    while (p.depth_left && path_segment<COUNT>(S, F, p, stack, mesh_stack, err, w)) {}
    out_color = f3(tone_mapped_baked(p.color.x), tone_mapped_baked(p.color.y), tone_mapped_baked(p.color.z));
    out_depth = p.depth;
}

// Blocks per SM the fused kernel is compiled for (register caps with
// spills that mostly hit L1), one build for frames whose paths end at their
// first hit (no reflective or refractive material, or max depth 1) and one
// for the rest.  Measured on one B200, frames without refit, blocks per SM
// for short / long paths:
//   4 / 4 (128 registers):  config 1 640x360 0.035 ms, 1920x1080 0.201;
//                           config 3 (glass, depth 8) 320x180 0.075, 640x360 0.107
//   5 / 4:                  config 1 0.039, 0.215
//   6 / 4:                  config 1 0.041, 0.217
//   4 / 3 (170 registers):  config 3 0.071, 0.107
//   4 / 5:                  config 3 0.082, 0.123
// (uncapped, 220 registers and two blocks: config 1 0.045 ms).
#ifndef SLIM_FUSED_SHORT_BLOCKS
#define SLIM_FUSED_SHORT_BLOCKS 4
#endif
#ifndef SLIM_FUSED_LONG_BLOCKS
#define SLIM_FUSED_LONG_BLOCKS 3
#endif
constexpr int kFusedShortPathBlocks = SLIM_FUSED_SHORT_BLOCKS;
constexpr int kFusedLongPathBlocks = SLIM_FUSED_LONG_BLOCKS;
template <bool COUNT, int MIN_BLOCKS>
__global__ void __launch_bounds__(128, MIN_BLOCKS) k_render_fused(DevScene S, DevFrame F) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Work w = {};
    if (i < F.width * F.rows) {
        int x = (int)(i % F.width), y = (int)(F.row_begin + i / F.width);
        uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
        uint32_t err = 0;
        float3 color;
        float depth;
        render_sample<COUNT>(S, F, x, y, stack, mesh_stack, err, w, color, depth);
        set_pixel(F, x, y, color, depth);
        if (err) atomicOr(F.error_flags, err);
    }
    flush_work<COUNT>(F.counters, w);
}

// ---- batched requests in one persistent launch -------------------------------
// The pixels of the requests listed in `requests` form one work queue: pixel
// f of it belongs to request requests[k] with prefix[k] <= f < prefix[k + 1]
// (pixel f - prefix[k] of that request in 8 x 4 tile order).  Every warp
// keeps 32 paths in flight: each turn every live lane traces one path segment
// (closest hit, shading with its shadow rays, bounce), a lane whose path
// ended writes its pixel, and the idle lanes of the warp claim the next
// pixels of the queue together (one atomic per warp, ranks by ballot), so
// warps stay full until the queue is empty whatever the path lengths.
// Blocks per SM the persistent batch kernel is compiled for (a register cap:
// its walks wait on dependent loads, so warps beat registers; config 5's
// plain requests in one launch: 84.3 ms uncapped at 168 registers, 74.7 ms
// at 6 blocks, 77.0 ms at 8).
#ifndef SLIM_BATCH_PERSISTENT_MIN_BLOCKS
#define SLIM_BATCH_PERSISTENT_MIN_BLOCKS 6
#endif
template <bool COUNT>
__global__ void __launch_bounds__(128, SLIM_BATCH_PERSISTENT_MIN_BLOCKS)
k_batch_persistent(const DevScene *scenes, const DevFrame *frames,
                                                          const uint32_t *requests, const uint32_t *prefix,
                                                          uint32_t count, uint32_t total, uint32_t *cursor,
                                                          uint32_t *error_flags, unsigned long long *counters) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    PathState p;
    bool live = false;
    uint32_t req = 0, x = 0, y = 0;
    for (;;) {
        const unsigned idle = __ballot_sync(0xFFFFFFFFu, !live);
        if (idle) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(cursor, (uint32_t)__popc(idle));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (!live) {
                const uint32_t f = base + (uint32_t)__popc(idle & ((1u << lane) - 1u));
                if (base < total && f < total) {
                    uint32_t lo = 0, hi = count;          // last k with prefix[k] <= f
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (__ldg(prefix + mid) <= f) lo = mid; else hi = mid;
                    }
                    req = __ldg(requests + lo);
                    const DevFrame &F = frames[req];
                    const uint32_t pixel = pixel_of_slot(F.width, F.height, f - __ldg(prefix + lo));
                    x = pixel % F.width;
                    y = pixel / F.width;
                    path_start<COUNT>(F, (int)x, (int)y, p, w);
                    live = true;
                }
            }
            if (!__any_sync(0xFFFFFFFFu, live)) break;
        }
        if (live) {
            const DevFrame &F = frames[req];
            if (!p.depth_left || !path_segment<COUNT>(scenes[req], F, p, stack, mesh_stack, err, w)) {
                set_pixel(F, (int)x, (int)y,
                          f3(tone_mapped_baked(p.color.x), tone_mapped_baked(p.color.y), tone_mapped_baked(p.color.z)),
                          p.depth);
                live = false;
            }
        }
    }
    if (err) atomicOr(error_flags, err);
    flush_work<COUNT>(counters, w);
}

// First closest hit of each primary ray (renderer/ray_tracer.h:36-45).
__global__ void __launch_bounds__(128) k_trace_primary(DevScene S, SlimCameraRayProjection P, uint32_t width,
                                                       uint32_t height, int *geometry_ids, uint32_t *primitive_ids,
                                                       float *distances, uint8_t *from_behind, uint32_t *error_flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= width * height) return;
    int x = (int)(i % width), y = (int)(i / width);
    uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    Ray ray;
    reset(ray, f3(P.camera_position.x, P.camera_position.y, P.camera_position.z), normalized(primary_direction(P, x, y)));
    Hit hit;
    int g = scene_trace<false>(S, ray, hit, false, INFINITY, stack, mesh_stack, err, w);
    geometry_ids[i] = g;
    bool mesh = false;
    if (g >= 0) mesh = load_geo(S, (uint32_t)g).type == SLIM_GEOMETRY_MESH;
    primitive_ids[i] = mesh ? hit.id : 0u;
    distances[i] = g >= 0 ? hit.distance : INFINITY;
    from_behind[i] = g >= 0 ? (uint8_t)hit.from_behind : (uint8_t)0;
    if (err) atomicOr(error_flags, err);
}

// Selection::manipulate's pick (scene/selection.h:36-80): the closest
// geometry behind pixel (x, y), then every point light's selection sphere
// (radius intensity / 2 / 64) along the same -- already offset -- ray up to
// the hit distance, each hit shrinking that distance; the last light hit
// wins over the geometry.  One thread.
__global__ void k_pick(DevScene S, SlimCameraRayProjection P, int x, int y, SlimPick *out, uint32_t *error_flags) {
    if (blockIdx.x || threadIdx.x) return;
    uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    Ray ray;
    reset(ray, f3(P.camera_position.x, P.camera_position.y, P.camera_position.z), normalized(primary_direction(P, x, y)));
    Hit hit;
    int g = scene_trace<false>(S, ray, hit, false, INFINITY, stack, mesh_stack, err, w);
    float max_distance = hit.distance;
    int light = -1;
    for (uint32_t i = 0; i < S.light_count; i++) {
        LightRec l = load_light(S, i);
        if (l.flags & SLIM_LIGHT_IS_DIRECTIONAL) continue;
        // SphereTracer::hit (core/ray.h:317-336)
        float radius = l.intensity * 0.5f * kLightIntensityRadius;
        float orr = kLightRadiusIntensity / (l.intensity * 0.5f);
        float t_max = max_distance * orr;
        float3 rc = (l.pos - ray.o) * orr;
        float b = dot(ray.d, rc);
        float c = sqlen(rc) - 1;
        float h = b * b - c;
        if (h >= 0) {
            h = sqrtf(h);
            float t_near = b - h, t_far = b + h;
            if (t_far > 0 && t_near < t_max) {
                max_distance = t_max * radius;
                light = (int)i;
            }
        }
    }
    SlimPick r;
    r.geometry = g;
    r.light = light;
    r.triangle = (g >= 0 && load_geo(S, (uint32_t)g).type == SLIM_GEOMETRY_MESH) ? hit.id : 0u;
    r.distance = g >= 0 ? hit.distance : INFINITY;
    float3 pos = g >= 0 ? at(ray, hit.distance) : f3(0, 0, 0);
    r.position[0] = pos.x;
    r.position[1] = pos.y;
    r.position[2] = pos.z;
    r.from_behind = g >= 0 ? (uint32_t)hit.from_behind : 0u;
    *out = r;
    if (err) atomicOr(error_flags, err);
}

}  // namespace dev

cudaError_t launch_pick(const DevScene &S, const SlimCameraRayProjection &P, int x, int y, SlimPick *out,
                        uint32_t *error_flags, cudaStream_t stream) {
    dev::k_pick<<<1, 32, 0, stream>>>(S, P, x, y, out, error_flags);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_render_fused(const DevScene &S, const DevFrame &F, int block, cudaStream_t stream,
                                StageTimer *timer, bool short_paths) {
    uint32_t n = F.width * F.rows;
    if (block <= 0) block = 128;
    if (block > 128) block = 128;
    dim3 grid((n + block - 1) / block);
    if (timer) timer->begin(STAGE_FUSED, stream);
    constexpr int kShort = dev::kFusedShortPathBlocks, kLong = dev::kFusedLongPathBlocks;
    if (F.counters) {
        if (short_paths) dev::k_render_fused<true, kShort><<<grid, block, 0, stream>>>(S, F);
        else dev::k_render_fused<true, kLong><<<grid, block, 0, stream>>>(S, F);
    } else {
        if (short_paths) dev::k_render_fused<false, kShort><<<grid, block, 0, stream>>>(S, F);
        else dev::k_render_fused<false, kLong><<<grid, block, 0, stream>>>(S, F);
    }
    count_launch();
    if (timer) timer->end(STAGE_FUSED, stream);
    return cudaGetLastError();
}

cudaError_t launch_batch_persistent(const DevScene *scenes, const DevFrame *frames, const uint32_t *requests,
                                    const uint32_t *prefix, uint32_t count, uint32_t total, uint32_t *cursor,
                                    uint32_t *error_flags, unsigned long long *counters, cudaStream_t stream) {
    if (!count || !total) return cudaSuccess;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    if (counters) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_batch_persistent<true>, 128, 0);
        dev::k_batch_persistent<true><<<sms * (per_sm > 0 ? per_sm : 1), 128, 0, stream>>>(
            scenes, frames, requests, prefix, count, total, cursor, error_flags, counters);
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_batch_persistent<false>, 128, 0);
        dev::k_batch_persistent<false><<<sms * (per_sm > 0 ? per_sm : 1), 128, 0, stream>>>(
            scenes, frames, requests, prefix, count, total, cursor, error_flags, counters);
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_trace_primary(const DevScene &S, const SlimCameraRayProjection &P, uint32_t width, uint32_t height,
                                 int *geometry_ids, uint32_t *primitive_ids, float *distances, uint8_t *from_behind,
                                 uint32_t *error_flags, cudaStream_t stream) {
    uint32_t n = width * height;
    dim3 grid((n + 127) / 128);
    dev::k_trace_primary<<<grid, 128, 0, stream>>>(S, P, width, height, geometry_ids, primitive_ids, distances,
                                                  from_behind, error_flags);
    count_launch();
    return cudaGetLastError();
}

}  // namespace slim
