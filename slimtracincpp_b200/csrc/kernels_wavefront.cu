// Wavefront form of the trace path.
//
// The reference traces each pixel's whole path in one thread
// (renderer/renderer_GPU.h:22-46 -> renderer/ray_tracer.h:19-108).  Here a
// frame is a sequence of stage kernels over queues in HBM, one round per
// bounce:
//
//   extend      closest hit of every queued ray  -> hit record      (scene/scene_tracer.h:26-98)
//   shadow_gen  shading frame of every hit, one shadow ray per facing
//               shadowing light -> shadow queue                      (surface_shader.h:49-59,147-160)
//   shadow      any-hit test of every shadow ray -> per-path occlusion bits
//   shade       full shading with the occlusion bits, area lights, IBL,
//               glow, throughput; reflective/refractive hits append the
//               next bounce ray to the next queue; finished paths are tone
//               mapped and written to the canvas                    (ray_tracer.h:42-107)
//
// Each trace stage keeps only traversal state live, so it runs at a much
// higher occupancy than the fused kernel.  Queues are appended with one
// atomic per warp (ballot + popc prefix).  Shading applies the lights in
// the reference's order from the occlusion bits, so every colour is summed
// in the same order as the reference's per-pixel loop.
#include "kernels.h"
#include "nrc.h"
#include "tracer_core.cuh"

namespace slim {
namespace dev {

// Queue records.
//   ray:    float4 (origin.xyz, pixel)     float4 (direction.xyz, 0)
//   hit:    float4 (normal.xyz, distance)  float4 (u, v, uv_coverage, NdotRd)
//           float4 (geometry, from_behind, triangle id, 0)   -- ints as bits
//   shadow: float4 (origin.xyz, slot<<6 | light)  float4 (direction.xyz, max distance)

SLIM_D uint32_t lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated queue append: one atomicAdd per warp, slots handed out
// by the ballot's prefix popcount.  Returns the slot of a thread whose
// `want` is set.
SLIM_D uint32_t warp_append(uint32_t *counter, bool want) {
    uint32_t active = __activemask();
    uint32_t ballot = __ballot_sync(active, want);
    uint32_t base = 0;
    if (ballot) {
        int leader = __ffs(ballot) - 1;
        if ((int)lane_id() == leader) base = atomicAdd(counter, (uint32_t)__popc(ballot));
        base = __shfl_sync(active, base, leader);
    }
    return base + (uint32_t)__popc(ballot & ((1u << lane_id()) - 1u));
}

SLIM_D void store_hit(float4 *hits, uint32_t slot, int g, const Hit &h) {
    float4 *p = hits + 3 * (size_t)slot;
    p[0] = make_float4(h.normal.x, h.normal.y, h.normal.z, h.distance);
    p[1] = make_float4(h.u, h.v, h.uv_coverage, h.NdotRd);
    p[2] = make_float4(__int_as_float(g), __uint_as_float((uint32_t)h.from_behind), __uint_as_float(h.id), 0.0f);
}
SLIM_D int load_hit(const float4 *hits, uint32_t slot, Hit &h) {
    const float4 *p = hits + 3 * (size_t)slot;
    float4 a = p[0], b = p[1], c = p[2];
    h.normal = xyz(a);
    h.distance = a.w;
    h.u = b.x; h.v = b.y; h.uv_coverage = b.z; h.NdotRd = b.w;
    h.from_behind = __float_as_uint(c.y) != 0;
    h.id = __float_as_uint(c.z);
    return __float_as_int(c.x);
}

template <bool COUNT>
SLIM_D void flush_stage(unsigned long long *counters, const Work &w) {
    if (!COUNT || !counters) return;
    uint32_t v[9] = {w.primary, w.shadow, w.bounce, w.scene_nodes, w.mesh_nodes, w.triangles, w.geometries,
                     w.mesh_fetches, w.taps};
#pragma unroll
    for (int k = 0; k < 9; k++) {
        unsigned long long s = v[k];
        for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
        if (lane_id() == 0 && s) atomicAdd(counters + k, s);
    }
}

struct QueueArgs {
    const float4 *rays_in;        // null: primary rays generated from the slot (= sample index)
    float4 *rays_out;
    const uint32_t *count_in;     // null: count = samples
    uint32_t *count_out;
    float4 *hits;
    float4 *shadow_rays;
    uint32_t *shadow_count;
    unsigned long long *masks;    // per slot: bit i = light i occluded
    float4 *pairs;                // shadow ray x mesh instance candidates, 3 float4 each:
                                  // (local origin, aux distance) (local direction, tag) (nodes, triangles, first child)
    uint32_t *pair_count;
    uint32_t *pair_cursor;
    uint32_t pair_capacity;
    float4 *path_color;           // per sample: colour, depth
    float4 *path_throughput;      // per sample: throughput
    uint32_t samples;
    uint32_t depth;               // 1-based bounce of this round
    uint32_t light_begin, light_end;
    unsigned long long *counters; // this stage's counter slots, or null
    // radiance cache
    float4 *sink;                 // non-null: finished paths write their linear colour here
                                  // (indexed by the path slot) instead of the canvas
    uint32_t skip_glow_depth;     // no light glow on the segment of this depth (0 = none)
};

SLIM_D void primary_ray(const DevFrame &F, uint32_t i, float3 &o, float3 &d) {
    int x = (int)(i % F.width), y = (int)(i / F.width);
    const SlimCameraRayProjection &P = F.projection;
    o = f3(P.camera_position.x, P.camera_position.y, P.camera_position.z);
    d = normalized(primary_direction(P, x, y));
}

// `pixel` indexes the path state (and the canvas); `cone_pixel` is the canvas
// pixel whose ray-cone spread the path uses.  They differ only for the
// radiance cache's training paths, whose state lives in their own slots.
SLIM_D void load_ray(const DevFrame &F, const QueueArgs &A, uint32_t slot, float3 &o, float3 &d, uint32_t &pixel,
                     uint32_t &cone_pixel) {
    if (!A.rays_in) {
        pixel = cone_pixel = slot;
        primary_ray(F, slot, o, d);
        return;
    }
    float4 a = A.rays_in[2 * (size_t)slot], b = A.rays_in[2 * (size_t)slot + 1];
    o = xyz(a);
    pixel = __float_as_uint(a.w);
    d = xyz(b);
    cone_pixel = __float_as_uint(b.w);
}
SLIM_D void load_ray(const DevFrame &F, const QueueArgs &A, uint32_t slot, float3 &o, float3 &d, uint32_t &pixel) {
    uint32_t cone_pixel;
    load_ray(F, A, slot, o, d, pixel, cone_pixel);
}
SLIM_D float cone_scaling(const DevFrame &F, uint32_t cone_pixel) {
    return F.cones_per_pixel ? pixel_scaling(F.projection, (int)(cone_pixel % F.width), (int)(cone_pixel / F.width))
                             : 0.0f;
}

SLIM_D uint32_t queue_size(const QueueArgs &A) { return A.count_in ? *A.count_in : A.samples; }

// ---- extend: closest hit of every queued ray ----------------------------
template <bool COUNT>
__global__ void __launch_bounds__(256) k_extend(DevScene S, DevFrame F, QueueArgs A) {
    uint32_t n = queue_size(A);
    uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        float3 o, d;
        uint32_t pixel;
        load_ray(F, A, slot, o, d, pixel);
        if (!A.rays_in) bump<COUNT>(w.primary);
        Ray ray;
        reset(ray, o, d);
        Hit hit;
        int g = scene_trace<COUNT>(S, ray, hit, false, INFINITY, stack, mesh_stack, err, w);
        store_hit(A.hits, slot, g, hit);
    }
    if (err) atomicOr(F.error_flags, err);
    flush_stage<COUNT>(A.counters, w);
}

// ---- shadow_gen: one shadow ray per facing, shadowing light -------------
template <bool COUNT>
__global__ void __launch_bounds__(256) k_shadow_gen(DevScene S, DevFrame F, QueueArgs A) {
    uint32_t n = queue_size(A);
    Work w = {};
    uint32_t stride = gridDim.x * blockDim.x;
    // Every thread of a warp runs the same number of iterations so the
    // queue appends stay warp-uniform.
    uint32_t rounds = (n + stride - 1) / stride;
    for (uint32_t r = 0, slot = blockIdx.x * blockDim.x + threadIdx.x; r < rounds; r++, slot += stride) {
        bool live = slot < n;
        Surface s;
        bool shaded = false;
        if (live) {
            if (A.light_begin == 0) A.masks[slot] = 0ull;
            float3 o, d;
            uint32_t pixel, cone_pixel;
            load_ray(F, A, slot, o, d, pixel, cone_pixel);
            Hit hit;
            int g = load_hit(A.hits, slot, hit);
            if (g >= 0) {
                Geo geo = load_geo(S, (uint32_t)g);
                Mat m = load_mat(S, geo.material);
                if (!((m.flags & SLIM_MATERIAL_IS_EMISSIVE) && geo.type == SLIM_GEOMETRY_QUAD && !hit.from_behind)) {
                    Ray ray;
                    reset(ray, scale_add(d, kTraceOffset, o), d);
                    prepare_for_shading<COUNT>(S, geo, m, ray, hit, cone_scaling(F, cone_pixel), s, w);
                    shaded = true;
                }
            }
        }
        for (uint32_t li = A.light_begin; li < A.light_end; li++) {
            bool want = false;
            if (shaded) {
                LightRec l = load_light(S, li);
                want = is_facing_light(s, l) && (l.flags & SLIM_LIGHT_IS_SHADOWING);
            }
            uint32_t q = warp_append(A.shadow_count, want);
            if (want) {
                bump<COUNT>(w.shadow);
                A.shadow_rays[2 * (size_t)q] = make_float4(s.P.x, s.P.y, s.P.z, __uint_as_float((slot << 6) | li));
                A.shadow_rays[2 * (size_t)q + 1] = make_float4(s.L.x, s.L.y, s.L.z, s.Ld);
            }
        }
    }
    flush_stage<COUNT>(A.counters, w);
}

// ---- shadow: any-hit tests ------------------------------------------------
//
// An any-hit result is the OR, over every (scene leaf, geometry) the segment
// reaches, of that geometry's test with the leaf's aux distance
// min(leaf far + EPS, max distance) (scene/scene_tracer.h:111-136): the
// culling distance never shrinks before the first hit ends the search, so
// the result does not depend on the order the candidates are tested in.
// The shadow stage uses that freedom:
//   shadow_scene  walks the scene BVH per shadow ray, tests implicit
//                 primitives on the spot and appends one (ray, mesh
//                 instance, aux distance) pair per reached mesh instance;
//   shadow_mesh   a persistent kernel in which every lane runs one mesh BVH
//                 traversal step per loop turn and fetches the next pair as
//                 soon as its own finishes, so warps stay full although
//                 traversal lengths differ by orders of magnitude.

SLIM_D bool local_box_test(const DevScene &S, const Geo &g, const Ray &local) {
    float mn[3], mx[3], n, f;
    if (g.type == SLIM_GEOMETRY_MESH) {
        const DevMesh &m = S.meshes[g.mesh];
        for (int i = 0; i < 3; i++) { mn[i] = m.aabb_min[i]; mx[i] = m.aabb_max[i]; }
    } else {
        float e = g.type == SLIM_GEOMETRY_TET ? kTetMax : 1.0f;
        mx[0] = mx[1] = mx[2] = e;
        mn[0] = mn[1] = mn[2] = -e;
        if (g.type == SLIM_GEOMETRY_QUAD) { mn[1] = -kEps; mx[1] = kEps; }
    }
    return hit_aabb(local, mn[0], mn[1], mn[2], mx[0], mx[1], mx[2], n, f);
}

// Candidates of one scene leaf: implicit primitives are tested here, mesh
// instances whose BVH root the local ray reaches become pairs carrying the
// local ray, so the mesh pass starts at the root's children.  Returns true
// once the ray is known occluded.
template <bool COUNT>
SLIM_D bool shadow_leaf(const DevScene &S, const QueueArgs &A, uint32_t tag, uint32_t first, uint32_t count, float lf,
                        const Ray &ray, float max_distance, uint32_t *mesh_stack, uint32_t &err, Work &w) {
    float aux = minr(lf + kEps, max_distance);
    for (uint32_t i = 0; i < count; i++) {
        uint32_t gi = __ldg(S.leaf_geometry + first + i);
        Geo g = load_geo(S, gi);
        if (!(g.flags & SLIM_GEOMETRY_IS_SHADOWING)) continue;
        bump<COUNT>(w.geometries);
        Ray local;
        localize(local, ray.o, ray.d, g);
        if (!local_box_test(S, g, local)) continue;
        bool transparent = (g.flags & SLIM_GEOMETRY_IS_TRANSPARENT) != 0;
        Hit h;
        h.distance = aux;
        switch (g.type) {
            case SLIM_GEOMETRY_QUAD: if (hit_quad(local, h, transparent)) return true; break;
            case SLIM_GEOMETRY_BOX: if (hit_box(local, h, transparent)) return true; break;
            case SLIM_GEOMETRY_SPHERE: if (hit_sphere(local, h, transparent, nullptr)) return true; break;
            case SLIM_GEOMETRY_TET: if (hit_tet(local, h, transparent)) return true; break;
            case SLIM_GEOMETRY_MESH: {
                const DevMesh &m = S.meshes[g.mesh];
                const float4 *nodes = S.mesh_nodes + 2 * (size_t)m.node_offset;
                float ln, lf2;
                float4 ra, rb;
                load_node(nodes, 0, ra, rb);
                bump<COUNT>(w.mesh_nodes);
                if (!(hit_node(local, ra, rb, ln, lf2) && ln < aux)) break;
                if (node_leaf_count(rb)) {
                    if (hit_triangles<COUNT>(S.tri_hot, m.tri_offset, m.tri_count, lf2, local, h, true, w)) return true;
                    break;
                }
                uint32_t slot = warp_append(A.pair_count, true);
                if (slot < A.pair_capacity) {
                    float4 *p = A.pairs + 3 * (size_t)slot;
                    p[0] = make_float4(local.o.x, local.o.y, local.o.z, aux);
                    p[1] = make_float4(local.d.x, local.d.y, local.d.z, __uint_as_float(tag));
                    p[2] = make_float4(__uint_as_float(m.node_offset), __uint_as_float(m.tri_offset),
                                       __uint_as_float(node_first(rb)), 0.0f);
                } else if (mesh_trace<COUNT>(S, m, local, h, true, mesh_stack, err, w)) {
                    return true;   // pair queue full: trace the instance here
                }
            } break;
            default: break;
        }
    }
    return false;
}

template <bool COUNT>
__global__ void __launch_bounds__(256) k_shadow_scene(DevScene S, DevFrame F, QueueArgs A) {
    uint32_t n = *A.shadow_count;
    uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        float4 a = A.shadow_rays[2 * (size_t)q], b = A.shadow_rays[2 * (size_t)q + 1];
        uint32_t tag = __float_as_uint(a.w);
        Ray ray;
        float3 d = xyz(b);
        reset(ray, scale_add(d, kTraceOffset, xyz(a)), d);
        float Ld = b.w;
        bool occluded = false;
        float ln, rn, lf, rf;
        float4 ra, rb;
        load_node(S.scene_nodes, 0, ra, rb);
        bump<COUNT>(w.scene_nodes);
        if (hit_node(ray, ra, rb, ln, lf) && ln < Ld) {
            if (node_leaf_count(rb)) {
                occluded = shadow_leaf<COUNT>(S, A, tag, 0, S.geometry_count, lf, ray, Ld, mesh_stack, err, w);
            } else {
                uint32_t left = node_first(rb), top = 0;
                for (;;) {
                    float4 la, lb, xa, xb;
                    load_node(S.scene_nodes, left, la, lb);
                    load_node(S.scene_nodes, left + 1, xa, xb);
                    bump<COUNT>(w.scene_nodes, 2);
                    bool hl = hit_node(ray, la, lb, ln, lf) && ln < Ld;
                    bool hr = hit_node(ray, xa, xb, rn, rf) && rn < Ld;
                    uint32_t lc = node_first(lb), rc = node_first(xb);
                    bool go_left = hl && !node_leaf_count(lb), go_right = hr && !node_leaf_count(xb);
                    if (hl && node_leaf_count(lb) &&
                        shadow_leaf<COUNT>(S, A, tag, lc, node_leaf_count(lb), lf, ray, Ld, mesh_stack, err, w)) {
                        occluded = true;
                        break;
                    }
                    if (hr && node_leaf_count(xb) &&
                        shadow_leaf<COUNT>(S, A, tag, rc, node_leaf_count(xb), rf, ray, Ld, mesh_stack, err, w)) {
                        occluded = true;
                        break;
                    }
                    if (go_left) {
                        if (go_right) {
                            if (top >= (uint32_t)kStackCapacity) { err |= kErrStack; break; }
                            stack[top++] = rc;
                        }
                        left = lc;
                    } else if (go_right) {
                        left = rc;
                    } else {
                        if (top == 0) break;
                        left = stack[--top];
                    }
                }
            }
        }
        if (occluded) atomicOr(A.masks + (tag >> 6), 1ull << (tag & 63u));
    }
    if (err) atomicOr(F.error_flags, err);
    flush_stage<COUNT>(A.counters, w);
}

// One any-hit traversal step of a mesh BVH (MeshTracer::trace with
// any_hit, scene/mesh_tracer.h:51-114): test the child pair at `left`,
// triangles of hit leaves, then descend, or pop.  Returns 1 on a hit,
// -1 when the traversal is over without one, 0 to continue.
template <bool COUNT>
SLIM_D int mesh_any_step(const DevScene &S, const float4 *nodes, uint32_t tri_offset, const Ray &r, float aux,
                         uint32_t &left, uint32_t *stack, uint32_t &top, uint32_t &err, Work &w) {
    float ln, rn, lf, rf;
    float4 la, lb, xa, xb;
    load_node(nodes, left, la, lb);
    load_node(nodes, left + 1, xa, xb);
    bump<COUNT>(w.mesh_nodes, 2);
    bool hl = hit_node(r, la, lb, ln, lf) && ln < aux;
    bool hr = hit_node(r, xa, xb, rn, rf) && rn < aux;
    uint32_t lc = node_first(lb), rc = node_first(xb);
    uint32_t lcount = node_leaf_count(lb), rcount = node_leaf_count(xb);
    Hit h;
    h.distance = aux;
    if (hl && lcount && hit_triangles<COUNT>(S.tri_hot, tri_offset + lc, lcount, lf, r, h, true, w)) return 1;
    if (hr && rcount && hit_triangles<COUNT>(S.tri_hot, tri_offset + rc, rcount, rf, r, h, true, w)) return 1;
    bool go_left = hl && !lcount, go_right = hr && !rcount;
    if (go_left) {
        if (go_right) {
            if (top >= (uint32_t)kStackCapacity) { err |= kErrStack; return -1; }
            stack[top++] = rc;
        }
        left = lc;
    } else if (go_right) {
        left = rc;
    } else {
        if (top == 0) return -1;
        left = stack[--top];
    }
    return 0;
}

template <bool COUNT>
__global__ void __launch_bounds__(256) k_shadow_mesh(DevScene S, DevFrame F, QueueArgs A) {
    const uint32_t n = *A.pair_count < A.pair_capacity ? *A.pair_count : A.pair_capacity;
    uint32_t stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    bool busy = false;
    uint32_t tag = 0, left = 0, top = 0, tri_offset = 0;
    const float4 *nodes = nullptr;
    float aux = 0.0f;
    Ray r;
    for (;;) {
        if (!busy) {
            // idle lanes of the warp take consecutive pairs with one atomic
            uint32_t active = __activemask();
            int leader = __ffs(active) - 1;
            uint32_t base = 0;
            if ((int)lane_id() == leader) base = atomicAdd(A.pair_cursor, (uint32_t)__popc(active));
            base = __shfl_sync(active, base, leader);
            uint32_t idx = base + (uint32_t)__popc(active & ((1u << lane_id()) - 1u));
            if (idx >= n) break;
            const float4 *p = A.pairs + 3 * (size_t)idx;
            float4 p0 = p[0], p1 = p[1], p2 = p[2];
            tag = __float_as_uint(p1.w);
            if ((A.masks[tag >> 6] >> (tag & 63u)) & 1ull) continue;   // already known occluded
            reset(r, xyz(p0), xyz(p1));
            aux = p0.w;
            nodes = S.mesh_nodes + 2 * (size_t)__float_as_uint(p2.x);
            tri_offset = __float_as_uint(p2.y);
            left = __float_as_uint(p2.z);
            top = 0;
            busy = true;
        }
        int res = mesh_any_step<COUNT>(S, nodes, tri_offset, r, aux, left, stack, top, err, w);
        if (res) {
            if (res > 0) atomicOr(A.masks + (tag >> 6), 1ull << (tag & 63u));
            busy = false;
        }
    }
    if (err) atomicOr(F.error_flags, err);
    flush_stage<COUNT>(A.counters, w);
}

// ---- shade: colour of this segment, next bounce, finished paths --------
template <bool COUNT>
__global__ void __launch_bounds__(256) k_shade(DevScene S, DevFrame F, QueueArgs A) {
    uint32_t n = queue_size(A);
    const SlimRayTracerSettings &st = F.settings;
    Work w = {};
    uint32_t stride = gridDim.x * blockDim.x;
    uint32_t rounds = (n + stride - 1) / stride;
    for (uint32_t r = 0, slot = blockIdx.x * blockDim.x + threadIdx.x; r < rounds; r++, slot += stride) {
        bool live = slot < n;
        bool bounce = false;
        uint32_t pixel = 0, cone_pixel = 0;
        float3 bo = f3(0, 0, 0), bd = f3(0, 0, 0);
        if (live) {
            float3 o, d;
            load_ray(F, A, slot, o, d, pixel, cone_pixel);
            Ray ray;
            reset(ray, scale_add(d, kTraceOffset, o), d);
            Hit hit;
            int g = load_hit(A.hits, slot, hit);
            float4 pc = A.depth == 1 ? make_float4(0, 0, 0, INFINITY) : A.path_color[pixel];
            float3 color = xyz(pc), throughput = A.depth == 1 ? f3(1, 1, 1) : xyz(A.path_throughput[pixel]);
            float depth = pc.w;
            float3 current = f3(0, 0, 0), next_throughput = f3(0, 0, 0);
            float hit_distance = INFINITY;
            if (g >= 0) {
                hit_distance = hit.distance;
                Geo geo = load_geo(S, (uint32_t)g);
                Mat m = load_mat(S, geo.material);
                if ((m.flags & SLIM_MATERIAL_IS_EMISSIVE) && geo.type == SLIM_GEOMETRY_QUAD && !hit.from_behind) {
                    current = m.emission;
                } else {
                    Surface s;
                    prepare_for_shading<COUNT>(S, geo, m, ray, hit, cone_scaling(F, cone_pixel), s, w);
                    hit_distance = hit.distance;
                    if (A.depth == 1) depth = depth_at(F.projection, hit.position);
                    unsigned long long occluded = A.masks[slot];
                    for (uint32_t i = 0; i < S.light_count; i++) {
                        LightRec l = load_light(S, i);
                        if (!is_facing_light(s, l)) continue;
                        if ((l.flags & SLIM_LIGHT_IS_SHADOWING) && ((occluded >> i) & 1ull)) continue;
                        add_light(s, m, l, current);
                    }
                    if (S.flags & SLIM_SCENE_HAD_EMISSIVE_QUADS) shade_from_emissive_quads(S, g, s, m, current);
                    if (st.skybox_irradiance_texture_id >= 0 && st.skybox_radiance_texture_id >= 0) {
                        s.L = s.N;
                        s.NdotL = 1.0f;
                        float3 D = texture_sample_cube<COUNT>(S, (uint32_t)st.skybox_irradiance_texture_id, s.N.x, s.N.y, s.N.z, w);
                        float3 Sp = texture_sample_cube<COUNT>(S, (uint32_t)st.skybox_radiance_texture_id, s.R.x, s.R.y, s.R.z, w);
                        radiance_fraction(s, m);
                        current = mul_add(D, s.Fd, mul_add(s.Fs, Sp, current));
                    }
                    if ((m.flags & (SLIM_MATERIAL_IS_REFLECTIVE | SLIM_MATERIAL_IS_REFRACTIVE)) && A.depth < st.max_depth) {
                        float3 Fr = schlick_fresnel(clamp01(dot(s.N, s.R)), m.reflectivity);
                        next_throughput = s.refracted ? one_minus(Fr) : Fr;
                        bounce = true;
                        bo = hit.position;
                        bd = s.RF;
                        reset(ray, bo, bd);
                    }
                }
            } else if (st.skybox_color_texture_id >= 0) {
                current = texture_sample_cube<COUNT>(S, (uint32_t)st.skybox_color_texture_id, ray.d.x, ray.d.y, ray.d.z, w);
            }
            if (A.depth != A.skip_glow_depth) add_glow(S, ray, hit_distance, current);
            color = mul_add(current, throughput, color);
            throughput = throughput * next_throughput;
            if (bounce) {
                A.path_color[pixel] = make_float4(color.x, color.y, color.z, depth);
                A.path_throughput[pixel] = make_float4(throughput.x, throughput.y, throughput.z, 0.0f);
            } else if (A.sink) {
                A.sink[pixel] = make_float4(color.x, color.y, color.z, 0.0f);
            } else {
                float3 c = f3(tone_mapped_baked(color.x), tone_mapped_baked(color.y), tone_mapped_baked(color.z));
                set_pixel(F, (int)(pixel % F.width), (int)(pixel / F.width), c, depth);
            }
        }
        uint32_t q = warp_append(A.count_out, bounce);
        if (bounce) {
            bump<COUNT>(w.bounce);
            A.rays_out[2 * (size_t)q] = make_float4(bo.x, bo.y, bo.z, __uint_as_float(pixel));
            A.rays_out[2 * (size_t)q + 1] = make_float4(bd.x, bd.y, bd.z, __uint_as_float(cone_pixel));
        }
    }
    flush_stage<COUNT>(A.counters, w);
}

// ---- radiance cache ----------------------------------------------------------
struct CacheArgs {
    float4 *features, *aux, *radiance;
    uint32_t *count;               // queries
    uint32_t *train_count;         // training paths
    uint32_t train_capacity;
    float4 *t_features, *t_targets, *t_color, *t_through;
    float offset;
    int mode;
};

// Vertex-`depth` hits of the main paths.  Misses and emissive quads finish the
// path exactly as k_shade does; every other hit becomes a cache query: the
// segment's glow is added to the path colour now, the surface's features are
// appended for the network, and the path waits in path_color /
// path_throughput for the answer.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_cache_gather(DevScene S, DevFrame F, QueueArgs A, CacheArgs C) {
    uint32_t n = queue_size(A);
    const SlimRayTracerSettings &st = F.settings;
    Work w = {};
    // scene box -> [0,1]^3 (longest side), from the scene BVH root
    float4 r0 = make_float4(0, 0, 0, 1), r1 = make_float4(1, 1, 0, 0);
    if (S.scene_node_count) { r0 = S.scene_nodes[0]; r1 = S.scene_nodes[1]; }
    const float3 bmin = f3(r0.x, r0.y, r0.z);
    const float ext = fmaxf(fmaxf(r0.w - r0.x, r1.x - r0.y), r1.y - r0.z);
    const float inv = ext > 0.0f ? 1.0f / ext : 1.0f;
    uint32_t stride = gridDim.x * blockDim.x;
    uint32_t rounds = (n + stride - 1) / stride;
    for (uint32_t r = 0, slot = blockIdx.x * blockDim.x + threadIdx.x; r < rounds; r++, slot += stride) {
        bool query = false;
        uint32_t pixel = 0, cone_pixel = 0;
        float3 o = f3(0, 0, 0), d = f3(0, 0, 0);
        float4 f0 = make_float4(0, 0, 0, 0), f1 = f0, f2 = f0, f3v = f0;
        if (slot < n) {
            load_ray(F, A, slot, o, d, pixel, cone_pixel);
            Ray ray;
            reset(ray, scale_add(d, kTraceOffset, o), d);
            Hit hit;
            int g = load_hit(A.hits, slot, hit);
            float4 pc = A.path_color[pixel];
            float3 color = xyz(pc), throughput = xyz(A.path_throughput[pixel]);
            float3 current = f3(0, 0, 0);
            float hit_distance = INFINITY;
            if (g >= 0) {
                hit_distance = hit.distance;
                Geo geo = load_geo(S, (uint32_t)g);
                Mat m = load_mat(S, geo.material);
                if ((m.flags & SLIM_MATERIAL_IS_EMISSIVE) && geo.type == SLIM_GEOMETRY_QUAD && !hit.from_behind) {
                    current = m.emission;
                } else {
                    Surface s;
                    prepare_for_shading<COUNT>(S, geo, m, ray, hit, cone_scaling(F, cone_pixel), s, w);
                    hit_distance = hit.distance;
                    query = true;
                    float3 p = (s.P - bmin) * inv;
                    float3 al = m.albedo * s.albedo_from_map;
                    f0 = make_float4(p.x, p.y, p.z, m.roughness);
                    f1 = make_float4(ray.d.x, ray.d.y, ray.d.z, 0.0f);
                    f2 = make_float4(s.N.x, s.N.y, s.N.z, 0.0f);
                    f3v = make_float4(al.x, al.y, al.z, 0.0f);
                }
            } else if (st.skybox_color_texture_id >= 0) {
                current = texture_sample_cube<COUNT>(S, (uint32_t)st.skybox_color_texture_id, ray.d.x, ray.d.y, ray.d.z, w);
            }
            add_glow(S, ray, hit_distance, current);
            color = mul_add(current, throughput, color);
            if (query) {
                A.path_color[pixel] = make_float4(color.x, color.y, color.z, pc.w);
            } else {
                float3 c = f3(tone_mapped_baked(color.x), tone_mapped_baked(color.y), tone_mapped_baked(color.z));
                set_pixel(F, (int)(pixel % F.width), (int)(pixel / F.width), c, pc.w);
            }
        }
        uint32_t q = warp_append(C.count, query);
        if (query) {
            float4 *f = C.features + 4 * (size_t)q;
            f[0] = f0; f[1] = f1; f[2] = f2; f[3] = f3v;
            C.aux[2 * (size_t)q] = make_float4(o.x, o.y, o.z, __uint_as_float(pixel));
            C.aux[2 * (size_t)q + 1] = make_float4(d.x, d.y, d.z, __uint_as_float(cone_pixel));
        }
    }
    flush_stage<COUNT>(A.counters, w);
}

// Training paths: query j of the frame's training set restarts from the
// query's ray with zero colour and unit throughput in its own slot j.  With
// more queries than training paths the set is stratified: j takes query
// floor((j + offset) * queries / capacity).
__global__ void k_cache_select(CacheArgs C, float4 *rays, uint32_t *ray_count) {
    const uint32_t nq = *C.count, cap = C.train_capacity;
    const uint32_t n = nq < cap ? nq : cap;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        uint32_t idx = j;
        if (nq > cap) {
            idx = (uint32_t)(((double)j + (double)C.offset) * (double)nq / (double)cap);
            if (idx >= nq) idx = nq - 1;
        }
        if (C.t_features) {
            const float4 *f = C.features + 4 * (size_t)idx;
            float4 *t = C.t_features + 4 * (size_t)j;
            t[0] = f[0]; t[1] = f[1]; t[2] = f[2]; t[3] = f[3];
        }
        float4 a = C.aux[2 * (size_t)idx], b = C.aux[2 * (size_t)idx + 1];
        rays[2 * (size_t)j] = make_float4(a.x, a.y, a.z, __uint_as_float(j));
        rays[2 * (size_t)j + 1] = b;
        C.t_color[j] = make_float4(0.0f, 0.0f, 0.0f, INFINITY);
        C.t_through[j] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *C.train_count = n;
        *ray_count = n;
    }
}

// Waiting paths take the cache's answer: colour += throughput * radiance,
// then tone mapping and the canvas write of k_shade.
__global__ void k_cache_resolve(DevFrame F, CacheArgs C, const float4 *path_color, const float4 *path_throughput) {
    const uint32_t nq = *C.count;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        uint32_t pixel = __float_as_uint(C.aux[2 * (size_t)q].w);
        float4 pc = path_color[pixel];
        float3 thr = xyz(path_throughput[pixel]);
        float3 L = f3(0, 0, 0);
        if (C.mode == SLIM_CACHE_ON) L = xyz(C.radiance[q]);
        else if (C.mode == SLIM_CACHE_EXACT) L = xyz(C.t_targets[q]);
        float3 color = mul_add(L, thr, xyz(pc));
        float3 c = f3(tone_mapped_baked(color.x), tone_mapped_baked(color.y), tone_mapped_baked(color.z));
        set_pixel(F, (int)(pixel % F.width), (int)(pixel / F.width), c, pc.w);
    }
}

template <bool COUNT>
cudaError_t run_frame(const DevScene &S, const DevFrame &F, const WavefrontBuffers &B, int block, cudaStream_t stream,
                      StageTimer *timer, const CacheFrame *cache) {
    uint32_t samples = F.width * F.height;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (block <= 0) block = 256;
    // Persistent-style grids: enough resident blocks to fill every SM, the
    // threads stride over the device-side queue length.
    auto grid_for = [&](const void *kernel, uint32_t work) {
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
        uint32_t g = (uint32_t)(sms * (per_sm > 0 ? per_sm : 1));
        uint32_t need = (work + block - 1) / block;
        return need < g ? (need ? need : 1) : g;
    };
    uint32_t lights = S.light_count;
    unsigned long long *C = F.counters;
    auto stage_counters = [&](int stage) { return C ? C + kCountersPerStage * stage : nullptr; };
    cudaError_t e = cudaMemsetAsync(B.queue_count, 0, 8 * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    QueueArgs A{};
    A.hits = B.hits;
    A.shadow_rays = B.shadow_rays;
    A.masks = B.shadow_mask;
    A.pairs = B.pairs;
    A.pair_count = B.queue_count + 3;
    A.pair_cursor = B.queue_count + 4;
    A.pair_capacity = B.pair_capacity;
    A.path_color = B.path_color;
    A.path_throughput = B.path_throughput;
    A.samples = samples;
    const uint32_t max_depth = F.settings.max_depth;
    const bool use_cache = cache && cache->mode != SLIM_CACHE_OFF && cache->depth >= 2 && cache->depth <= max_depth;
    CacheArgs CA{};
    if (use_cache) {
        CA.features = cache->features;
        CA.aux = cache->aux;
        CA.radiance = cache->radiance;
        CA.count = cache->counts;
        CA.train_count = cache->counts + 1;
        CA.train_capacity = cache->train_capacity;
        CA.t_features = cache->mode == SLIM_CACHE_ON ? cache->t_features : nullptr;
        CA.t_targets = cache->t_targets;
        CA.t_color = cache->t_color;
        CA.t_through = cache->t_through;
        CA.offset = cache->select_offset;
        CA.mode = cache->mode;
        e = cudaMemsetAsync(cache->counts, 0, 2 * sizeof(uint32_t), stream);
        if (e != cudaSuccess) return e;
    }
    const uint32_t bound = samples;   // a queue holds at most one ray per sample

    // One bounce round over the queue `in` (primary rays at depth 1): extend,
    // then shadows and shading -- or, at the cache depth, the cache gather.
    uint32_t in = 0;
    auto round = [&](uint32_t depth, bool primary, bool gather) -> cudaError_t {
        uint32_t out = in ^ 1u;
        A.depth = depth;
        A.rays_in = primary ? nullptr : B.rays[in];
        A.count_in = primary ? nullptr : B.queue_count + in;
        A.rays_out = B.rays[out];
        A.count_out = B.queue_count + out;
        // the output queue of this round is the input of the next: clear it
        if (!primary) {
            cudaError_t r = cudaMemsetAsync(B.queue_count + out, 0, sizeof(uint32_t), stream);
            if (r != cudaSuccess) return r;
        }
        A.counters = stage_counters(STAGE_EXTEND);
        if (timer) timer->begin(STAGE_EXTEND, stream);
        k_extend<COUNT><<<grid_for((const void *)k_extend<COUNT>, bound), block, 0, stream>>>(S, F, A);
        if (timer) timer->end(STAGE_EXTEND, stream);
        if (gather) {
            A.counters = stage_counters(STAGE_CACHE);
            if (timer) timer->begin(STAGE_CACHE, stream);
            k_cache_gather<COUNT><<<grid_for((const void *)k_cache_gather<COUNT>, bound), block, 0, stream>>>(S, F, A, CA);
            if (timer) timer->end(STAGE_CACHE, stream);
            in = out;
            return cudaGetLastError();
        }
        // Shadow rays in light batches that fit the shadow queue.
        uint32_t per_batch = B.shadow_capacity / (samples ? samples : 1);
        if (per_batch < 1) per_batch = 1;
        for (uint32_t l0 = 0; l0 < lights; l0 += per_batch) {
            A.light_begin = l0;
            A.light_end = l0 + per_batch < lights ? l0 + per_batch : lights;
            cudaError_t r = cudaMemsetAsync(B.queue_count + 2, 0, sizeof(uint32_t), stream);
            if (r != cudaSuccess) return r;
            A.shadow_count = B.queue_count + 2;
            A.counters = stage_counters(STAGE_SHADOW_GEN);
            if (timer) timer->begin(STAGE_SHADOW_GEN, stream);
            k_shadow_gen<COUNT><<<grid_for((const void *)k_shadow_gen<COUNT>, bound), block, 0, stream>>>(S, F, A);
            if (timer) timer->end(STAGE_SHADOW_GEN, stream);
            r = cudaMemsetAsync(B.queue_count + 3, 0, 2 * sizeof(uint32_t), stream);
            if (r != cudaSuccess) return r;
            A.counters = stage_counters(STAGE_SHADOW);
            if (timer) timer->begin(STAGE_SHADOW, stream);
            k_shadow_scene<COUNT><<<grid_for((const void *)k_shadow_scene<COUNT>, bound * (A.light_end - A.light_begin)), block, 0, stream>>>(S, F, A);
            if (timer) timer->end(STAGE_SHADOW, stream);
            A.counters = stage_counters(STAGE_SHADOW_MESH);
            if (timer) timer->begin(STAGE_SHADOW_MESH, stream);
            k_shadow_mesh<COUNT><<<grid_for((const void *)k_shadow_mesh<COUNT>, B.pair_capacity), block, 0, stream>>>(S, F, A);
            if (timer) timer->end(STAGE_SHADOW_MESH, stream);
        }
        A.counters = stage_counters(STAGE_SHADE);
        if (timer) timer->begin(STAGE_SHADE, stream);
        k_shade<COUNT><<<grid_for((const void *)k_shade<COUNT>, bound), block, 0, stream>>>(S, F, A);
        if (timer) timer->end(STAGE_SHADE, stream);
        in = out;
        return cudaGetLastError();
    };

    const uint32_t last = use_cache ? cache->depth : max_depth;
    for (uint32_t depth = 1; depth <= last; depth++)
        if ((e = round(depth, depth == 1, use_cache && depth == last)) != cudaSuccess) return e;
    if (!use_cache) return cudaSuccess;

    const int mode = cache->mode;
    const bool train = mode == SLIM_CACHE_ON && cache->trainer && cache->batch && cache->train_capacity;
    if (mode == SLIM_CACHE_EXACT || train) {
        // training paths continue from the cache vertex in their own slots
        if (timer) timer->begin(STAGE_CACHE, stream);
        uint32_t g = (cache->train_capacity + 255) / 256;
        if (g > (uint32_t)(sms * 8)) g = (uint32_t)(sms * 8);
        k_cache_select<<<g ? g : 1, 256, 0, stream>>>(CA, B.rays[in], B.queue_count + in);
        if (timer) timer->end(STAGE_CACHE, stream);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        QueueArgs main = A;
        A.path_color = cache->t_color;
        A.path_throughput = cache->t_through;
        A.sink = cache->t_targets;
        A.skip_glow_depth = cache->depth;
        for (uint32_t depth = cache->depth; depth <= max_depth; depth++)
            if ((e = round(depth, false, false)) != cudaSuccess) return e;
        A = main;
    }
    if (train) {
        if (timer) timer->begin(STAGE_CACHE_TRAIN, stream);
        for (uint32_t off = 0; off < cache->train_capacity; off += cache->batch) {
            uint32_t n = cache->train_capacity - off < cache->batch ? cache->train_capacity - off : cache->batch;
            if ((e = cache->trainer->step(cache->t_features, cache->t_targets, n, cache->counts + 1, off, stream)) !=
                cudaSuccess)
                return e;
        }
        if (timer) timer->end(STAGE_CACHE_TRAIN, stream);
    }
    if (mode == SLIM_CACHE_ON) {
        if (timer) timer->begin(STAGE_CACHE_QUERY, stream);
        e = nrc::launch_infer(cache->features, cache->counts, 0, samples, cache->radiance, cache->weights,
                              F.error_flags, stream);
        if (timer) timer->end(STAGE_CACHE_QUERY, stream);
        if (e != cudaSuccess) return e;
    }
    if (timer) timer->begin(STAGE_CACHE, stream);
    k_cache_resolve<<<grid_for((const void *)k_cache_resolve, bound), block, 0, stream>>>(F, CA, B.path_color,
                                                                                          B.path_throughput);
    if (timer) timer->end(STAGE_CACHE, stream);
    return cudaGetLastError();
}

}  // namespace dev

cudaError_t launch_render_wavefront(const DevScene &S, const DevFrame &F, const WavefrontBuffers &B, int block,
                                    cudaStream_t stream, StageTimer *timer, const CacheFrame *cache) {
    if (F.settings.render_mode != SLIM_RENDER_BEAUTY)   // a single primary hit: nothing to queue
        return launch_render_fused(S, F, block, stream, timer);
    if (F.settings.max_depth == 0) return launch_render_fused(S, F, block, stream, timer);
    if (F.counters) return dev::run_frame<true>(S, F, B, block, stream, timer, cache);
    return dev::run_frame<false>(S, F, B, block, stream, timer, cache);
}

}  // namespace slim
