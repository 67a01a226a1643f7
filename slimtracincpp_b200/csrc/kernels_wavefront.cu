// Wavefront form of the trace path.
//
// The reference traces each pixel's whole path in one thread
// (renderer/renderer_GPU.h:22-46 -> renderer/ray_tracer.h:19-108).  Here a
// frame is a sequence of stage kernels over queues in HBM, one round per
// bounce:
//
//   extend      closest hit of every queued ray  -> hit record      (scene/scene_tracer.h:26-98);
//               with meshes: scene candidates, persistent mesh pass, resolve
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

// Hit records in three planes of `stride` float4 (one entry per queue slot):
//   plane 0 (normal.xyz, distance), plane 1 (u, v, uv coverage, N.Rd),
//   plane 2 (geometry, from behind, triangle, 0).
// A miss (geometry -1) writes and reads plane 2 only: most primary rays of
// an open scene miss, and their records then cost one 16-byte entry in
// the contiguous plane instead of 48 bytes.
SLIM_D void store_hit(float4 *hits, uint32_t stride, uint32_t slot, int g, const Hit &h) {
    hits[2 * (size_t)stride + slot] =
        make_float4(__int_as_float(g), __uint_as_float((uint32_t)h.from_behind), __uint_as_float(h.id), 0.0f);
    if (g < 0) return;
    hits[slot] = make_float4(h.normal.x, h.normal.y, h.normal.z, h.distance);
    hits[(size_t)stride + slot] = make_float4(h.u, h.v, h.uv_coverage, h.NdotRd);
}
SLIM_D int load_hit(const float4 *hits, uint32_t stride, uint32_t slot, Hit &h) {
    const float4 c = hits[2 * (size_t)stride + slot];
    const int g = __float_as_int(c.x);
    h.distance = INFINITY;
    if (g < 0) return g;
    const float4 a = hits[slot], b = hits[(size_t)stride + slot];
    h.normal = xyz(a);
    h.distance = a.w;
    h.u = b.x; h.v = b.y; h.uv_coverage = b.z; h.NdotRd = b.w;
    h.from_behind = __float_as_uint(c.y) != 0;
    h.id = __float_as_uint(c.z);
    return g;
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

// Radiance-cache state of a frame (see kernels.h CacheFrame).
struct CacheArgs {
    float4 *features, *aux, *radiance;
    uint32_t *count;               // queries
    uint32_t *train_count;         // training paths
    uint32_t train_capacity;
    float4 *t_features, *t_targets, *t_color, *t_through;
    uint32_t *frame_counter;
    int mode;
    float4 *q_color, *q_through;   // per query: path colour + depth, throughput (null: path slots)
    float4 *q_hit;                 // per query: its hit record, 3 float4 (null: not kept)
};

struct QueueArgs {
    const float4 *rays_in;        // null: primary rays generated from the slot (= sample index)
    float4 *rays_out;
    const uint32_t *count_in;     // null: count = samples
    uint32_t *count_out;
    float4 *hits;                 // hit records, three planes of hit_stride entries
    uint32_t hit_stride;
    float4 *shadow_rays;
    uint32_t *shadow_count;
    unsigned long long *masks;    // per slot: bit i = light i occluded
    float4 *pairs;                // shadow ray x mesh instance candidates, 3 float4 each:
                                  // (local origin, aux distance) (local direction, tag) (nodes, triangles, first child)
    uint32_t *pair_count;
    uint32_t *pair_cursor;
    uint32_t pair_capacity;
    float4 *path_color;           // per path: colour, depth
    float4 *path_throughput;      // per path: throughput
    uint32_t samples;
    uint32_t depth;               // 1-based bounce of this round
    uint32_t light_begin, light_end;
    uint32_t early_depth;         // non-zero: shadow_gen writes every path's canvas depth, shade only colours
    uint32_t slot_begin, slot_end;  // shade: the slots [begin, end) of the queue (end 0: all)
    unsigned long long *counters; // this stage's counter slots, or null
    // radiance cache
    float4 *sink;                 // non-null: finished paths write their linear colour here
                                  // (indexed by the path slot) instead of the canvas
    uint32_t skip_glow_depth;     // no light glow on the segment of this depth (0 = none)
    CacheArgs cache;              // batched frames: queries of requests using the cache
    // batched requests (null in a single-request frame)
    const DevScene *scenes;
    const DevFrame *frames;
};

// Ray records: (origin.xyz, path) (direction.xyz, pid).  `path` indexes the
// path state (colour, throughput); `pid` names the canvas pixel: the pixel
// index in a single-request frame, (request << 23) | pixel in a batch.  The
// two differ for the radiance cache's training paths, whose state lives in
// their own slots, and for batched paths, whose slots are per wave.
constexpr uint32_t kBatchPixelBits = 23;

template <bool BATCH> SLIM_D uint32_t req_of(uint32_t pid) { return BATCH ? pid >> kBatchPixelBits : 0u; }
template <bool BATCH> SLIM_D uint32_t pix_of(uint32_t pid) {
    return BATCH ? pid & ((1u << kBatchPixelBits) - 1u) : pid;
}
template <bool BATCH> SLIM_D const DevScene &scene_of(const DevScene &S, const QueueArgs &A, uint32_t pid) {
    if constexpr (BATCH) return A.scenes[req_of<true>(pid)];
    else return S;
}
template <bool BATCH> SLIM_D const DevFrame &frame_of(const DevFrame &F, const QueueArgs &A, uint32_t pid) {
    if constexpr (BATCH) return A.frames[req_of<true>(pid)];
    else return F;
}

SLIM_D void primary_ray(const DevFrame &F, uint32_t i, float3 &o, float3 &d) {
    int x = (int)(i % F.width), y = (int)(i / F.width);
    const SlimCameraRayProjection &P = F.projection;
    o = f3(P.camera_position.x, P.camera_position.y, P.camera_position.z);
    d = normalized(primary_direction(P, x, y));
}


SLIM_D void load_ray(const DevFrame &F, const QueueArgs &A, uint32_t slot, float3 &o, float3 &d, uint32_t &path,
                     uint32_t &pid) {
    if (!A.rays_in) {
        path = slot;
        pid = F.row_begin * F.width + pixel_of_slot(F.width, F.rows, slot);
        primary_ray(F, pid, o, d);
        return;
    }
    float4 a = A.rays_in[2 * (size_t)slot], b = A.rays_in[2 * (size_t)slot + 1];
    o = xyz(a);
    path = __float_as_uint(a.w);
    d = xyz(b);
    pid = __float_as_uint(b.w);
}
template <bool BATCH> SLIM_D float cone_scaling(const DevFrame &F, uint32_t pid) {
    uint32_t p = pix_of<BATCH>(pid);
    return F.cones_per_pixel ? pixel_scaling(F.projection, (int)(p % F.width), (int)(p / F.width)) : 0.0f;
}
template <bool BATCH>
SLIM_D void write_pixel(const DevFrame &F, uint32_t pid, float3 color, float depth, bool with_depth = true) {
    uint32_t p = pix_of<BATCH>(pid);
    float3 c = f3(tone_mapped_baked(color.x), tone_mapped_baked(color.y), tone_mapped_baked(color.z));
    if (with_depth) set_pixel(F, (int)(p % F.width), (int)(p / F.width), c, depth);
    else set_pixel_color(F, (int)(p % F.width), (int)(p / F.width), c);
}

SLIM_D uint32_t queue_size(const QueueArgs &A) { return A.count_in ? *A.count_in : A.samples; }

// ---- extend: closest hit of every queued ray ----------------------------
template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(256) k_extend(DevScene S0, DevFrame F0, QueueArgs A) {
    uint32_t n = queue_size(A);
    uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        float3 o, d;
        uint32_t path, pid;
        load_ray(F0, A, slot, o, d, path, pid);
        if (!A.rays_in) bump<COUNT>(w.primary);
        const DevScene &S = scene_of<BATCH>(S0, A, pid);
        Ray ray;
        reset(ray, o, d);
        Hit hit;
        int g = scene_trace<COUNT>(S, ray, hit, false, INFINITY, stack, mesh_stack, err, w);
        store_hit(A.hits, A.hit_stride, slot, g, hit);
    }
    if (err) atomicOr(F0.error_flags, err);
    flush_stage<COUNT>(A.counters, w);
}

// A batched request's path that reached its radiance-cache vertex: the
// cache answers there, so it is neither shaded nor lit (training paths,
// which carry a sink, are).
template <bool BATCH> SLIM_D bool at_cache_vertex(const DevFrame &F, const QueueArgs &A) {
    return BATCH && F.cache_depth == A.depth && !A.sink;
}

// ---- shadow_gen: one shadow ray per facing, shadowing light -------------
// In a single frame's first round it can also write the canvas depths (the
// shaded hit's depth, infinity where shade leaves none), which are final
// once the primary hits are: they download while the shadows are traced.
template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(256) k_shadow_gen(DevScene S0, DevFrame F0, QueueArgs A) {
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
        uint32_t lights = 0, pid = 0;
        if (live) {
            float3 o, d;
            uint32_t path;
            load_ray(F0, A, slot, o, d, path, pid);
            const DevScene &S = scene_of<BATCH>(S0, A, pid);
            const DevFrame &F = frame_of<BATCH>(F0, A, pid);
            lights = S.light_count;
            Hit hit;
            int g = load_hit(A.hits, A.hit_stride, slot, hit);
            if (g >= 0 && !at_cache_vertex<BATCH>(F, A)) {
                Geo geo = load_geo(S, (uint32_t)g);
                Mat m = load_mat(S, geo.material);
                if (!((m.flags & SLIM_MATERIAL_IS_EMISSIVE) && geo.type == SLIM_GEOMETRY_QUAD && !hit.from_behind)) {
                    Ray ray;
                    reset(ray, scale_add(d, kTraceOffset, o), d);
                    prepare_for_shading<COUNT>(S, geo, m, ray, hit, cone_scaling<BATCH>(F, pid), s, w);
                    shaded = true;
                    // occluded-light bits: read by shade for shaded hits only
                    if (A.light_begin == 0) A.masks[slot] = 0ull;
                }
            }
            if (!BATCH && A.early_depth && A.light_begin == 0) {
                uint32_t p = pix_of<BATCH>(pid);
                set_depth(F, (int)(p % F.width), (int)(p / F.width), shaded ? depth_at(F.projection, hit.position) : INFINITY);
            }
        }
        for (uint32_t li = A.light_begin; li < A.light_end; li++) {
            bool want = false;
            if (shaded && li < lights) {
                LightRec l = load_light(scene_of<BATCH>(S0, A, pid), li);
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
//   shadow_mesh   a persistent kernel (leaves parked, see PendingLeaves) in which every lane runs one mesh BVH
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

// Capped at 64 registers (4 blocks per SM instead of 3): latency-bound, the
// extra warps pay for the few spills (config 2: shadow 0.157 -> 0.149 ms;
// re-measured on the final build, 3 blocks at 78 registers without spills:
// 0.155 against 0.148 ms).
#ifndef SLIM_SHADOW_SCENE_BLOCKS
#define SLIM_SHADOW_SCENE_BLOCKS 4
#endif
template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(256, SLIM_SHADOW_SCENE_BLOCKS) k_shadow_scene(DevScene S0, DevFrame F, QueueArgs A) {
    uint32_t n = *A.shadow_count;
    uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        float4 a = A.shadow_rays[2 * (size_t)q], b = A.shadow_rays[2 * (size_t)q + 1];
        uint32_t tag = __float_as_uint(a.w);
        const DevScene &S = scene_of<BATCH>(S0, A, BATCH ? __float_as_uint(A.rays_in[2 * (size_t)(tag >> 6) + 1].w) : 0u);
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


// Leaves a walk reaches wait (up to three per lane, in visiting order) while
// the lane keeps stepping through inner nodes; the warp tests triangles only
// when enough of its lanes have a waiting leaf (kLeafFraction) or none can
// step, so the triangle code runs with many lanes busy instead of one or two.
// A lane keeps stepping through inner nodes while at most kStepWhileWaiting
// leaves wait (config 2: stepping with one leaf waiting 2.03 -> 1.94 ms).
constexpr uint32_t kStepWhileWaiting = 1;
// Inner steps a walking lane takes per loop turn: the turn's warp votes (new
// candidates? leaf tests?) are paid once per two steps (config 2: 1.55 ->
// 1.48 ms; three steps measured the same as two).
constexpr uint32_t kStepsPerTurn = 2;
// kStepWhileWaiting + 2 slots: a lane steps only with at most
// kStepWhileWaiting leaves waiting, and a step adds at most two.  A waiting
// leaf is packed into one word, first triangle | count << kLeafCountShift
// (mesh uploads are limited to fit), which frees registers for the walk
// (config 2: 1.45 -> 1.44 ms).
struct PendingLeaves {
    uint32_t leaf0, leaf1, leaf2;
    float clip0, clip1, clip2;
    uint32_t n;
    uint32_t first0, count0;            // slot 0 unpacked
    SLIM_D void push(uint32_t f, uint32_t c, float far) {
        const uint32_t v = f | (c << kLeafCountShift);
        if (n == 0) { leaf0 = v; clip0 = far; }
        else if (n == 1) { leaf1 = v; clip1 = far; }
        else { leaf2 = v; clip2 = far; }
        n++;
        unpack();
    }
    SLIM_D void pop() {
        leaf0 = leaf1; clip0 = clip1;
        leaf1 = leaf2; clip1 = clip2;
        n--;
        unpack();
    }
    SLIM_D void unpack() {
        first0 = leaf0 & ((1u << kLeafCountShift) - 1u);
        count0 = leaf0 >> kLeafCountShift;
    }
    SLIM_D bool can_step() const { return n <= kStepWhileWaiting; }
};
static_assert(kStepWhileWaiting + 2 <= 3, "PendingLeaves holds three leaves");

// Warp-uniform decision: should idle lanes take new candidates now?  Idle
// lanes wait until a quarter of the warp is idle (or nobody is busy) and
// then fetch together, so the fetch code -- one atomic, the candidate loads,
// the ray set-up -- runs for several lanes at once instead of for the one or
// two that finished this turn (config 2: 1.94 -> 1.82 ms).
constexpr uint32_t kFetchFraction = 4;   // fetch when idle lanes >= active lanes / kFetchFraction
SLIM_D bool fetch_round(bool idle) {
    const uint32_t act = __activemask();
    const uint32_t idle_mask = __ballot_sync(act, idle);
    return idle_mask && (kFetchFraction * (uint32_t)__popc(idle_mask) >= (uint32_t)__popc(act) || idle_mask == act);
}

// Warp-uniform decision: test waiting leaves now?  Once a third of the warp
// has a leaf waiting, or no lane can step (with two steps per turn, a third
// measured 1.49 -> 1.47 ms on config 2 against a half).
constexpr uint32_t kLeafFraction = 3;
SLIM_D bool leaf_round(bool waiting, bool can_step) {
    const uint32_t act = __activemask();
    const uint32_t wait_mask = __ballot_sync(act, waiting);
    const uint32_t step_mask = __ballot_sync(act, can_step);
    return wait_mask && (kLeafFraction * (uint32_t)__popc(wait_mask) >= (uint32_t)__popc(act) || !step_mask);
}

// The persistent mesh kernels run 128-thread blocks with a register cap
// that fits one more block per SM than their natural use (shadow: 61 -> 56
// registers, 32 -> 36 warps per SM; closest hit: 73 -> 70 registers, 24 -> 28
// warps): their walks wait on dependent loads, so warps beat registers
// (config 2: 1.61 -> 1.57 ms with the closest-hit pass, 1.59 with the any-hit
// pass alone).  With the later walk changes, config 2 at 9 / 7 blocks takes
// 1.437-1.443 ms; 10 or 12 any-hit blocks 1.54 / 1.68 ms (spills), 8 or 9
// closest-hit blocks 1.48-1.49 ms.
constexpr int kMeshBlock = 128;
#ifndef SLIM_SHADOW_MESH_BLOCKS
#define SLIM_SHADOW_MESH_BLOCKS 9
#endif
#ifndef SLIM_EXTEND_MESH_BLOCKS
#define SLIM_EXTEND_MESH_BLOCKS 7
#endif

// Drain phase of the persistent any-hit kernel.  Once the pair queue is
// empty, a lane with nothing left to walk takes the deepest pending subtree
// (the bottom entry of the stack) of a lane of its warp that is still
// walking, so the last long walks of a launch spread over the warp instead
// of running one lane each while the rest of the warp waits.  The i-th idle
// lane (in lane order) takes from the i-th lane with a pending subtree; the
// giver removes the entry from its stack.  Exact: an any-hit result is the
// OR over the leaves a walk reaches, whatever the order (config 2: 1.46 ->
// 1.45 ms; config 4's plain depth-8 frame, whose late rounds are almost all
// tail: 3.00 -> 2.91 ms).  The closest-hit walks do not share: a piece that
// does not know the best hit of the part before it in the reference's order
// could report a triangle the reference culls.
struct Steal {
    int from;           // giving lane for a taker, else -1
    uint32_t subtree;   // stack entry handed over (valid for a taker)
};
SLIM_D Steal steal_round(uint32_t act, uint32_t idle_mask, uint32_t donor_mask, bool idle, bool donor,
                         uint32_t *stack, uint32_t &bottom, uint32_t &top) {
    const uint32_t below = (1u << lane_id()) - 1u;
    const uint32_t pairs = min((uint32_t)__popc(idle_mask), (uint32_t)__popc(donor_mask));
    const uint32_t my_idle_rank = (uint32_t)__popc(idle_mask & below);
    const bool taker = idle && my_idle_rank < pairs;
    const bool giver = donor && (uint32_t)__popc(donor_mask & below) < pairs;
    uint32_t give = 0;
    if (giver) {
        give = stack[bottom++];
        if (bottom == top) bottom = top = 0;
    }
    uint32_t m = donor_mask;
    for (uint32_t j = 0; taker && j < my_idle_rank; j++) m &= m - 1u;
    const int src = taker ? __ffs(m) - 1 : (int)lane_id();
    Steal st;
    st.subtree = __shfl_sync(act, give, src);
    st.from = taker ? src : -1;
    return st;
}
// Stack push for walks that may give entries away from the bottom: the live
// entries are [bottom, top); when the top reaches the capacity they move
// down first.  Returns false on overflow.
SLIM_D bool push_entry(uint32_t *stack, uint32_t &bottom, uint32_t &top, uint32_t v) {
    if (top >= (uint32_t)kStackCapacity) {
        if (bottom == 0) return false;
        for (uint32_t i = bottom; i < top; i++) stack[i - bottom] = stack[i];
        top -= bottom;
        bottom = 0;
    }
    stack[top++] = v;
    return true;
}

template <bool COUNT>
__global__ void __launch_bounds__(kMeshBlock, SLIM_SHADOW_MESH_BLOCKS) k_shadow_mesh(DevScene S, DevFrame F, QueueArgs A) {
    const uint32_t n = *A.pair_count < A.pair_capacity ? *A.pair_count : A.pair_capacity;
    uint32_t stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    bool busy = false, walking = false, drained = false;
    uint32_t idx = 0, tag = 0, left = 0, top = 0, bottom = 0, tri_offset = 0;
    const float4 *nodes = nullptr;
    float aux = 0.0f;
    Ray r;
    PendingLeaves pend;
    pend.n = 0;
    // (shadow ray, instance) pair i from its root's children, or from `subtree`
    auto start = [&](uint32_t i, uint32_t subtree, bool whole) {
        const float4 *p = A.pairs + 3 * (size_t)i;
        float4 p0 = p[0], p1 = p[1], p2 = p[2];
        tag = __float_as_uint(p1.w);
        if ((A.masks[tag >> 6] >> (tag & 63u)) & 1ull) return;   // already known occluded
        idx = i;
        reset(r, xyz(p0), xyz(p1));
        aux = p0.w;
        nodes = S.mesh_nodes + 2 * (size_t)__float_as_uint(p2.x);
        tri_offset = __float_as_uint(p2.y);
        left = whole ? __float_as_uint(p2.z) : subtree;
        top = bottom = 0;
        pend.n = 0;
        busy = walking = true;
    };
    for (;;) {
        if (!drained) {
            const bool fetch = fetch_round(!busy);
            if (!busy && fetch) {
                uint32_t active = __activemask();
                int leader = __ffs(active) - 1;
                uint32_t base = 0;
                if ((int)lane_id() == leader) base = atomicAdd(A.pair_cursor, (uint32_t)__popc(active));
                base = __shfl_sync(active, base, leader);
                const uint32_t i = base + (uint32_t)__popc(active & ((1u << lane_id()) - 1u));
                if (i >= n) drained = true;
                else start(i, 0, true);
            }
        }
        {
            const uint32_t act = __activemask();
            if (__ballot_sync(act, drained)) {
                const uint32_t idle = __ballot_sync(act, drained && !busy);
                if (idle == act) break;
                const bool donor = walking && top > bottom;
                const uint32_t donors = __ballot_sync(act, donor);
                if (idle && donors) {
                    const Steal st = steal_round(act, idle, donors, drained && !busy, donor, stack, bottom, top);
                    const uint32_t from_idx = __shfl_sync(act, idx, st.from >= 0 ? st.from : (int)lane_id());
                    if (st.from >= 0) start(from_idx, st.subtree, false);
                }
            }
        }
#pragma unroll
        for (uint32_t sub = 0; sub < kStepsPerTurn; sub++) if (walking && pend.can_step()) {
            // one inner step of the any-hit walk (mesh_tracer.h:51-114); hit leaves wait
            float ln, rn, lf, rf;
            float4 la, lb, xa, xb;
            load_node(nodes, left, la, lb);
            load_node(nodes, left + 1, xa, xb);
            bump<COUNT>(w.mesh_nodes, 2);
            bool hl = hit_node(r, la, lb, ln, lf) && ln < aux;
            bool hr = hit_node(r, xa, xb, rn, rf) && rn < aux;
            uint32_t lc = node_first(lb), rc = node_first(xb);
            uint32_t lcount = node_leaf_count(lb), rcount = node_leaf_count(xb);
            if (hl && lcount) pend.push(lc, lcount, lf);
            if (hr && rcount) pend.push(rc, rcount, rf);
            bool go_left = hl && !lcount, go_right = hr && !rcount;
            if (go_left) {
                if (go_right) {
                    if (!push_entry(stack, bottom, top, rc)) { err |= kErrStack; walking = false; }
                }
                left = lc;
            } else if (go_right) {
                left = rc;
            } else if (top == bottom) {
                walking = false;
                top = bottom = 0;
            } else {
                left = stack[--top];
            }
        }
        if (leaf_round(pend.n > 0, walking && pend.can_step()) && pend.n) {
            Hit h;
            h.distance = aux;
            bool hit = hit_triangles<COUNT>(S.tri_hot, tri_offset + pend.first0, pend.count0, pend.clip0, r, h,
                                            true, w);
            pend.pop();
            if (hit) {
                atomicOr(A.masks + (tag >> 6), 1ull << (tag & 63u));
                walking = false;
                top = bottom = 0;
                pend.n = 0;
            }
        }
        if (busy && !walking && pend.n == 0) busy = false;
    }
    if (err) atomicOr(F.error_flags, err);
    flush_stage<COUNT>(A.counters, w);
}

// ---- extend, split: closest hit as scene candidates + a persistent mesh pass
//
// The closest hit the reference's SceneTracer::trace finds is the candidate
// with the smallest distance, ties going to the one it visits first: a later
// candidate replaces the current hit only when strictly closer
// (scene_tracer.h:129, mesh_tracer.h:37).  Culling by the current distance
// only skips candidates that cannot win, and a mesh walk started with a
// larger incoming distance finds a superset of hits in the same visiting
// order.  So the search splits exactly:
//   extend_scene   walks the scene BVH in the reference's order, numbering
//                  every geometry it visits (k), tests implicit primitives on
//                  the spot (culling by the best implicit hit so far) and
//                  appends one candidate per reached mesh instance;
//   extend_mesh    a persistent kernel: every lane takes one mesh-BVH step
//                  per loop turn in the reference's order and fetches the
//                  next candidate when its walk ends; finished candidates
//                  publish (distance, k) with a 64-bit atomicMin per ray;
//   extend_resolve the candidate whose (distance, k) is the ray's minimum
//                  writes the hit record.
// Cross-candidate culling keeps ties (<=), so the winner is the reference's.
// Candidate records (4 float4): (local origin, clip) (local direction, slot)
// (node offset, triangle offset, first child, 0) (geometry, mesh, k, found);
// a finished walk overwrites the third with (t, u, v, triangle | behind << 31)
// and sets `found`.  The ray keys live in the shadow-mask array, which is
// free until the shadow stage.

SLIM_D unsigned long long hit_key(float t, uint32_t k) {
    return ((unsigned long long)__float_as_uint(t) << 32) | k;
}
// No hit yet: distance +inf (the culling bound reads the high word as a float).
constexpr unsigned long long kNoHitKey = (0x7F800000ull << 32) | 0xFFFFFFFFull;

template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(256) k_extend_scene(DevScene S0, DevFrame F0, QueueArgs A) {
    uint32_t n = queue_size(A);
    uint32_t stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    const uint32_t cap = A.pair_capacity * 3u / 4u;
    uint32_t *overflow = reinterpret_cast<uint32_t *>(A.shadow_rays);   // free until shadow_gen
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        float3 o, d;
        uint32_t path, pid;
        load_ray(F0, A, slot, o, d, path, pid);
        if (!A.rays_in) bump<COUNT>(w.primary);
        const DevScene &S = scene_of<BATCH>(S0, A, pid);
        Ray r;
        reset(r, scale_add(d, kTraceOffset, o), d);
        Hit hit;
        hit.distance = INFINITY;
        int best_geo = -1;
        uint32_t best_k = 0, k = 0;
        bool full = false;
        // one scene leaf: [first, first + count) geometries, far distance lf
        auto leaf = [&](uint32_t first, uint32_t count, float lf) {
            Hit aux;
            aux.distance = minr(lf + kEps, hit.distance);
            const float clip = lf + kEps;
            Ray local;
            for (uint32_t i = 0; i < count; i++, k++) {
                uint32_t gi = __ldg(S.leaf_geometry + first + i);
                Geo g = load_geo(S, gi);
                if (!(g.flags & SLIM_GEOMETRY_IS_VISIBLE)) continue;
                if (g.type != SLIM_GEOMETRY_MESH) {
                    if (hit_geometry_local<COUNT>(S, g, r, local, aux, false, nullptr, err, w) &&
                        aux.distance < hit.distance) {
                        best_geo = (int)gi;
                        best_k = k;
                        hit = aux;
                        hit.NdotRd = -(dot(hit.normal, local.d));
                    }
                    continue;
                }
                bump<COUNT>(w.geometries);
                localize(local, r.o, r.d, g);
                const DevMesh &m = S.meshes[g.mesh];
                float bn, bf;
                if (!hit_aabb(local, m.aabb_min[0], m.aabb_min[1], m.aabb_min[2], m.aabb_max[0], m.aabb_max[1],
                              m.aabb_max[2], bn, bf))
                    continue;
                const float4 *nodes = S.mesh_nodes + 2 * (size_t)m.node_offset;
                float4 ra, rb;
                float rn, rf;
                load_node(nodes, 0, ra, rb);
                bump<COUNT>(w.mesh_nodes);
                // the root test with the largest distance the reference could have used
                if (!(hit_node(local, ra, rb, rn, rf) && rn < clip && rn <= hit.distance)) continue;
                if (node_leaf_count(rb)) {
                    // a single-leaf mesh (mesh_tracer.h:66-70): its triangles here
                    Hit mh;
                    mh.distance = clip;
                    if (hit_triangles<COUNT>(S.tri_hot, m.tri_offset, m.tri_count, rf, local, mh, false, w) &&
                        mh.distance < hit.distance) {
                        mh.uv_coverage = __ldg(&S.tri_cold[4 * (size_t)(m.tri_offset + mh.id) + 3].w);
                        best_geo = (int)gi;
                        best_k = k;
                        hit = mh;
                        hit.NdotRd = -(dot(hit.normal, local.d));
                    }
                    continue;
                }
                uint32_t q = warp_append(A.pair_count, true);
                if (q >= cap) { full = true; continue; }
                float4 *p = A.pairs + 4 * (size_t)q;
                p[0] = make_float4(local.o.x, local.o.y, local.o.z, clip);
                p[1] = make_float4(local.d.x, local.d.y, local.d.z, __uint_as_float(slot));
                p[2] = make_float4(__uint_as_float(m.node_offset), __uint_as_float(m.tri_offset),
                                   __uint_as_float(node_first(rb)), 0.0f);
                p[3] = make_float4(__uint_as_float(gi), __uint_as_float(g.mesh), __uint_as_float(k), 0.0f);
            }
        };
        float ln, rn, lf, rf;
        float4 a, b;
        load_node(S.scene_nodes, 0, a, b);
        bump<COUNT>(w.scene_nodes);
        if (hit_node(r, a, b, ln, lf) && ln < hit.distance) {
            if (node_leaf_count(b)) {
                leaf(0, S.geometry_count, lf);
            } else {
                uint32_t left = node_first(b), top = 0;
                for (;;) {
                    float4 la, lb, xa, xb;
                    load_node(S.scene_nodes, left, la, lb);
                    load_node(S.scene_nodes, left + 1, xa, xb);
                    bump<COUNT>(w.scene_nodes, 2);
                    bool hl = hit_node(r, la, lb, ln, lf) && ln < hit.distance;
                    bool hr = hit_node(r, xa, xb, rn, rf) && rn < hit.distance;
                    uint32_t lchild = node_first(lb), rchild = node_first(xb);
                    bool go_left = hl, go_right = hr;
                    if (hl && node_leaf_count(lb)) {
                        leaf(lchild, node_leaf_count(lb), lf);
                        go_left = false;
                    }
                    if (hr && node_leaf_count(xb)) {
                        leaf(rchild, node_leaf_count(xb), rf);
                        go_right = false;
                    }
                    if (go_left) {
                        if (go_right) {
                            if (ln > rn) { uint32_t t = lchild; lchild = rchild; rchild = t; }
                            if (top >= (uint32_t)kStackCapacity) { err |= kErrStack; break; }
                            stack[top++] = rchild;
                        }
                        left = lchild;
                    } else if (go_right) {
                        left = rchild;
                    } else {
                        if (top == 0) break;
                        left = stack[--top];
                    }
                }
            }
        }
        if (full) {
            // the candidate queue ran out: the ray is traced whole afterwards
            // (k_extend_overflow); key 0 matches no candidate (hit distances
            // are never 0: the plane test rejects an origin on the plane)
            A.masks[slot] = 0ull;
            overflow[atomicAdd(A.pair_count + 2, 1u)] = slot;
        } else {
            A.masks[slot] = best_geo >= 0 ? hit_key(hit.distance, best_k) : kNoHitKey;
            store_hit(A.hits, A.hit_stride, slot, best_geo, hit);
        }
    }
    if (err) atomicOr(F0.error_flags, err);
    flush_stage<COUNT>(A.counters, w);
}

// Rays whose candidates did not fit: the reference's whole closest-hit walk.
template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(256) k_extend_overflow(DevScene S0, DevFrame F0, QueueArgs A) {
    const uint32_t n = A.pair_count[2];
    const uint32_t *overflow = reinterpret_cast<const uint32_t *>(A.shadow_rays);
    uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = overflow[i];
        float3 o, d;
        uint32_t path, pid;
        load_ray(F0, A, slot, o, d, path, pid);
        const DevScene &S = scene_of<BATCH>(S0, A, pid);
        Ray ray;
        reset(ray, o, d);
        Hit hit;
        int g = scene_trace<COUNT>(S, ray, hit, false, INFINITY, stack, mesh_stack, err, w);
        store_hit(A.hits, A.hit_stride, slot, g, hit);
    }
    if (err) atomicOr(F0.error_flags, err);
    flush_stage<COUNT>(A.counters, w);
}

template <bool COUNT>
__global__ void __launch_bounds__(kMeshBlock, SLIM_EXTEND_MESH_BLOCKS) k_extend_mesh(DevScene S, DevFrame F, QueueArgs A) {
    const uint32_t cap = A.pair_capacity * 3u / 4u;
    const uint32_t n = *A.pair_count < cap ? *A.pair_count : cap;
    uint32_t stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    bool busy = false, walking = false;
    uint32_t idx = 0, slot = 0, left = 0, top = 0, tri_offset = 0, tri = 0, k = 0;
    const float4 *nodes = nullptr;
    float lc = 0.0f, bu = 0.0f, bv = 0.0f;
    bool found = false, behind = false;
    Ray r;
    PendingLeaves pend;
    pend.n = 0;
    for (;;) {
        const bool fetch = fetch_round(!busy);
        if (!busy && fetch) {
            uint32_t active = __activemask();
            int leader = __ffs(active) - 1;
            uint32_t base = 0;
            if ((int)lane_id() == leader) base = atomicAdd(A.pair_cursor, (uint32_t)__popc(active));
            base = __shfl_sync(active, base, leader);
            idx = base + (uint32_t)__popc(active & ((1u << lane_id()) - 1u));
            if (idx >= n) break;
            const float4 *p = A.pairs + 4 * (size_t)idx;
            float4 p0 = p[0], p1 = p[1], p2 = p[2];
            reset(r, xyz(p0), xyz(p1));
            lc = p0.w;
            slot = __float_as_uint(p1.w);
            k = __float_as_uint(p[3].z);
            nodes = S.mesh_nodes + 2 * (size_t)__float_as_uint(p2.x);
            tri_offset = __float_as_uint(p2.y);
            left = __float_as_uint(p2.z);
            top = 0;
            found = false;
            pend.n = 0;
            busy = walking = true;
        }
#pragma unroll
        for (uint32_t sub = 0; sub < kStepsPerTurn; sub++) if (walking && pend.can_step()) {
            // one inner step of MeshTracer::trace (mesh_tracer.h:51-114); hit leaves
            // wait and are tested in the order the walk reached them
            const float gb = __uint_as_float((uint32_t)(A.masks[slot] >> 32));
            float ln, rn, lf, rf;
            float4 la, lb, xa, xb;
            load_node(nodes, left, la, lb);
            load_node(nodes, left + 1, xa, xb);
            bump<COUNT>(w.mesh_nodes, 2);
            bool hl = hit_node(r, la, lb, ln, lf) && ln < lc && ln <= gb;
            bool hr = hit_node(r, xa, xb, rn, rf) && rn < lc && rn <= gb;
            uint32_t lchild = node_first(lb), rchild = node_first(xb);
            uint32_t lcount = node_leaf_count(lb), rcount = node_leaf_count(xb);
            if (hl && lcount) pend.push(lchild, lcount, lf);
            if (hr && rcount) pend.push(rchild, rcount, rf);
            bool go_left = hl && !lcount, go_right = hr && !rcount;
            if (go_left) {
                if (go_right) {
                    if (ln > rn) { uint32_t t = lchild; lchild = rchild; rchild = t; }
                    if (top >= (uint32_t)kStackCapacity) { err |= kErrStack; walking = false; }
                    else stack[top++] = rchild;
                }
                left = lchild;
            } else if (go_right) {
                left = rchild;
            } else if (top == 0) {
                walking = false;
            } else {
                left = stack[--top];
            }
        }
        if (leaf_round(pend.n > 0, walking && pend.can_step()) && pend.n) {
            // MeshTracer::hitTriangles (mesh_tracer.h:23-49) with the leaf's far clip
            const float gb = __uint_as_float((uint32_t)(A.masks[slot] >> 32));
            float closest = minr(pend.clip0, lc);
            for (uint32_t i = 0; i < pend.count0; i++) {
                bump<COUNT>(w.triangles);
                const uint32_t t_index = pend.first0 + i;
                const float4 *t4 = S.tri_hot + 3 * (size_t)(tri_offset + t_index);
                float4 a = __ldg(t4), b = __ldg(t4 + 1), c = __ldg(t4 + 2);
                float3 pp = xyz(a), nn = f3(a.w, b.x, b.y);
                float tt; float3 pos; bool bh;
                if (!hit_plane(r, pp, nn, tt, pos, bh)) continue;
                float3 q = pos - pp;
                float ux = b.z * q.x + c.x * q.y + c.z * q.z;
                float uy = b.w * q.x + c.y * q.y + c.w * q.z;
                if (ux < 0 || uy < 0 || (ux + uy) > 1 || tt >= closest || tt > gb) continue;
                closest = tt;
                lc = tt;
                bu = ux;
                bv = uy;
                behind = bh;
                tri = t_index;
                found = true;
            }
            pend.pop();
        }
        if (busy && !walking && pend.n == 0) {
            float4 *p = A.pairs + 4 * (size_t)idx;
            if (found) {
                p[2] = make_float4(lc, bu, bv, __uint_as_float(tri | ((uint32_t)behind << 31)));
                atomicMin(A.masks + slot, hit_key(lc, k));
            }
            p[3].w = found ? 1.0f : 0.0f;
            busy = false;
        }
    }
    if (err) atomicOr(F.error_flags, err);
    flush_stage<COUNT>(A.counters, w);
}

// The candidate holding its ray's minimum (distance, k) writes the hit
// record with the attributes MeshTracer::trace fills in.
template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(256) k_extend_resolve(DevScene S0, DevFrame F0, QueueArgs A) {
    const uint32_t cap = A.pair_capacity * 3u / 4u;
    const uint32_t n = *A.pair_count < cap ? *A.pair_count : cap;
    Work w = {};
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        const float4 *p = A.pairs + 4 * (size_t)idx;
        const float4 p3 = p[3];
        if (p3.w == 0.0f) continue;
        const float4 p1 = p[1], p2 = p[2];
        const uint32_t slot = __float_as_uint(p1.w);
        if (A.masks[slot] != hit_key(p2.x, __float_as_uint(p3.z))) continue;
        uint32_t pid = 0;
        if (BATCH) pid = __float_as_uint(A.rays_in[2 * (size_t)slot + 1].w);
        const DevScene &S = scene_of<BATCH>(S0, A, pid);
        const DevMesh &m = S.meshes[__float_as_uint(p3.y)];
        Hit h;
        h.distance = p2.x;
        h.u = p2.y;
        h.v = p2.z;
        const uint32_t tb = __float_as_uint(p2.w);
        h.id = tb & 0x7FFFFFFFu;
        h.from_behind = (tb >> 31) != 0;
        const float4 *t4 = S.tri_hot + 3 * (size_t)(m.tri_offset + h.id);
        const float4 a = __ldg(t4), b = __ldg(t4 + 1);
        h.normal = f3(a.w, b.x, b.y);
        h.position = f3(0, 0, 0);
        mesh_hit_attributes<COUNT>(S, m, h, w);
        h.NdotRd = -(dot(h.normal, xyz(p1)));
        store_hit(A.hits, A.hit_stride, slot, (int)__float_as_uint(p3.x), h);
    }
    flush_stage<COUNT>(A.counters, w);
}

// ---- fused tail: the rest of every queued path in one thread ------------------
//
// Late rounds hold few paths whose traversals are long, so each round's
// kernels wait on a handful of slow rays and the frame pays that wait once
// per remaining bounce.  From the tail depth on, one kernel walks every
// remaining path to its end -- the reference's per-pixel loop
// (ray_tracer.h:42-107) from the queued ray on, closest hits and shadow rays
// traced inline -- so the wait is paid once.  Per path the arithmetic is
// k_extend / k_shade's, in the same order: the frame is unchanged.
template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(128) k_finish_paths(DevScene S0, DevFrame F0, QueueArgs A) {
    const uint32_t n = queue_size(A);
    uint32_t stack[kStackCapacity], mesh_stack[kStackCapacity];
    uint32_t err = 0;
    Work w = {};
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        float3 o, d;
        uint32_t path, pid;
        load_ray(F0, A, slot, o, d, path, pid);
        const DevScene &S = scene_of<BATCH>(S0, A, pid);
        const DevFrame &F = frame_of<BATCH>(F0, A, pid);
        const SlimRayTracerSettings &st = F.settings;
        const float scaling = cone_scaling<BATCH>(F, pid);
        float4 pc = A.path_color[path];
        float3 color = xyz(pc), throughput = xyz(A.path_throughput[path]);
        const float depth = pc.w;
        Ray ray;
        reset(ray, o, d);
        for (uint32_t level = A.depth;; level++) {
            Hit hit;
            float3 current = f3(0, 0, 0), next_throughput = f3(0, 0, 0);
            bool bounce = false;
            int g = scene_trace<COUNT>(S, ray, hit, false, INFINITY, stack, mesh_stack, err, w);
            float hit_distance = INFINITY;
            if (g >= 0) {
                hit_distance = hit.distance;
                Geo geo = load_geo(S, (uint32_t)g);
                Mat m = load_mat(S, geo.material);
                if ((m.flags & SLIM_MATERIAL_IS_EMISSIVE) && geo.type == SLIM_GEOMETRY_QUAD && !hit.from_behind) {
                    current = m.emission;
                } else {
                    Surface s;
                    prepare_for_shading<COUNT>(S, geo, m, ray, hit, scaling, s, w);
                    hit_distance = hit.distance;
                    for (uint32_t i = 0; i < S.light_count; i++) {
                        LightRec l = load_light(S, i);
                        if (!is_facing_light(s, l)) continue;
                        if (l.flags & SLIM_LIGHT_IS_SHADOWING) {
                            Ray sr;
                            sr.o = s.P;
                            sr.d = s.L;
                            Hit sh;
                            bump<COUNT>(w.shadow);
                            if (scene_trace<COUNT>(S, sr, sh, true, s.Ld, stack, mesh_stack, err, w) >= 0) continue;
                        }
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
                    if ((m.flags & (SLIM_MATERIAL_IS_REFLECTIVE | SLIM_MATERIAL_IS_REFRACTIVE)) && level < st.max_depth) {
                        float3 Fr = schlick_fresnel(clamp01(dot(s.N, s.R)), m.reflectivity);
                        next_throughput = s.refracted ? one_minus(Fr) : Fr;
                        bounce = true;
                        reset(ray, hit.position, s.RF);
                        bump<COUNT>(w.bounce);
                    }
                }
            } else if (st.skybox_color_texture_id >= 0) {
                current = texture_sample_cube<COUNT>(S, (uint32_t)st.skybox_color_texture_id, ray.d.x, ray.d.y, ray.d.z, w);
            }
            if (level != A.skip_glow_depth) add_glow(S, ray, hit_distance, current);
            color = mul_add(current, throughput, color);
            throughput = throughput * next_throughput;
            if (!bounce) break;
        }
        if (A.sink) A.sink[path] = make_float4(color.x, color.y, color.z, 0.0f);
        else write_pixel<BATCH>(F, pid, color, depth);
    }
    if (err) atomicOr(F0.error_flags, err);
    flush_stage<COUNT>(A.counters, w);
}

// ---- radiance-cache vertex ---------------------------------------------------
// The network's inputs at a shaded surface: position in the scene box mapped
// to [0,1]^3 (longest side, from the scene BVH root), roughness, ray
// direction, shading normal, albedo x albedo map.
SLIM_D void query_features(const DevScene &S, const Mat &m, const Ray &ray, const Surface &s, float4 f[4]) {
    float4 r0 = make_float4(0, 0, 0, 1), r1 = make_float4(1, 1, 0, 0);
    if (S.scene_node_count) { r0 = S.scene_nodes[0]; r1 = S.scene_nodes[1]; }
    const float ext = fmaxf(fmaxf(r0.w - r0.x, r1.x - r0.y), r1.y - r0.z);
    const float inv = ext > 0.0f ? 1.0f / ext : 1.0f;
    float3 p = (s.P - f3(r0.x, r0.y, r0.z)) * inv;
    float3 al = m.albedo * s.albedo_from_map;
    f[0] = make_float4(p.x, p.y, p.z, m.roughness);
    f[1] = make_float4(ray.d.x, ray.d.y, ray.d.z, 0.0f);
    f[2] = make_float4(s.N.x, s.N.y, s.N.z, 0.0f);
    f[3] = make_float4(al.x, al.y, al.z, 0.0f);
}

// The path has reached the vertex the cache answers at.  Misses and emissive
// quads finish it exactly as k_shade does; every other hit turns it into a
// query: the segment's glow is added to the path colour now, the surface's
// features (position in the scene box, roughness, direction, shading normal,
// albedo) go to the network, and the path waits in path_color /
// path_throughput for the answer.  Returns true for a query.
template <bool COUNT, bool BATCH>
SLIM_D bool cache_vertex(const DevScene &S, const DevFrame &F, const QueueArgs &A, uint32_t slot, uint32_t path,
                         uint32_t pid, float3 o, float3 d, float4 f[4], Work &w, float4 &q_color, float4 &q_through) {
    const SlimRayTracerSettings &st = F.settings;
    Ray ray;
    reset(ray, scale_add(d, kTraceOffset, o), d);
    Hit hit;
    int g = load_hit(A.hits, A.hit_stride, slot, hit);
    float4 pc = A.path_color[path];
    float3 color = xyz(pc), throughput = xyz(A.path_throughput[path]);
    float3 current = f3(0, 0, 0);
    float hit_distance = INFINITY;
    bool query = false;
    if (g >= 0) {
        hit_distance = hit.distance;
        Geo geo = load_geo(S, (uint32_t)g);
        Mat m = load_mat(S, geo.material);
        if ((m.flags & SLIM_MATERIAL_IS_EMISSIVE) && geo.type == SLIM_GEOMETRY_QUAD && !hit.from_behind) {
            current = m.emission;
        } else {
            Surface s;
            prepare_for_shading<COUNT>(S, geo, m, ray, hit, cone_scaling<BATCH>(F, pid), s, w);
            hit_distance = hit.distance;
            query = true;
            query_features(S, m, ray, s, f);
        }
    } else if (st.skybox_color_texture_id >= 0) {
        current = texture_sample_cube<COUNT>(S, (uint32_t)st.skybox_color_texture_id, ray.d.x, ray.d.y, ray.d.z, w);
    }
    add_glow(S, ray, hit_distance, current);
    color = mul_add(current, throughput, color);
    q_color = make_float4(color.x, color.y, color.z, pc.w);
    q_through = make_float4(throughput.x, throughput.y, throughput.z, 0.0f);
    if (query) A.path_color[path] = q_color;
    else if (A.sink) A.sink[path] = make_float4(color.x, color.y, color.z, 0.0f);   // a self-training path ends
    else write_pixel<BATCH>(F, pid, color, pc.w);
    return query;
}

// `hits`: the round's hit planes (stride entries each), whose record of
// `slot` the query keeps (null: none kept).
SLIM_D void append_query(const CacheArgs &C, uint32_t q, const float4 f[4], float3 o, float3 d, uint32_t path,
                         uint32_t pid, float4 q_color, float4 q_through, const float4 *hits = nullptr,
                         uint32_t stride = 0, uint32_t slot = 0) {
    if (C.q_hit && hits) {
        float4 *h = C.q_hit + 3 * (size_t)q;
        h[0] = hits[slot]; h[1] = hits[(size_t)stride + slot]; h[2] = hits[2 * (size_t)stride + slot];
    }
    float4 *p = C.features + 4 * (size_t)q;
    p[0] = f[0]; p[1] = f[1]; p[2] = f[2]; p[3] = f[3];
    C.aux[2 * (size_t)q] = make_float4(o.x, o.y, o.z, __uint_as_float(path));
    C.aux[2 * (size_t)q + 1] = make_float4(d.x, d.y, d.z, __uint_as_float(pid));
    if (C.q_color) {
        C.q_color[q] = q_color;
        C.q_through[q] = q_through;
    }
}

// ---- shade: colour of this segment, next bounce, finished paths --------
// Capped at 80 registers (3 blocks per SM instead of 2): latency-bound, the
// extra warps pay for the spills (config 2: shade 0.180 -> 0.173 ms).  The
// spills are real traffic -- in round 1, 340 MB of local stores reach L2
// (ncu) -- but on the final build 2 blocks at 128 registers, without
// spills, measure the same (0.183 against 0.182 ms).
#ifndef SLIM_SHADE_BLOCKS
#define SLIM_SHADE_BLOCKS 3
#endif
template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(256, SLIM_SHADE_BLOCKS) k_shade(DevScene S0, DevFrame F0, QueueArgs A) {
    uint32_t n = queue_size(A);
    if (A.slot_end && A.slot_end < n) n = A.slot_end;
    const uint32_t first = A.slot_begin;
    Work w = {};
    uint32_t stride = gridDim.x * blockDim.x;
    uint32_t rounds = n > first ? (n - first + stride - 1) / stride : 0;
    for (uint32_t r = 0, slot = first + blockIdx.x * blockDim.x + threadIdx.x; r < rounds; r++, slot += stride) {
        bool live = slot < n;
        bool bounce = false, query = false;
        uint32_t path = 0, pid = 0;
        float3 o = f3(0, 0, 0), d = f3(0, 0, 0);
        float3 bo = f3(0, 0, 0), bd = f3(0, 0, 0);
        float4 feat[4], qc = make_float4(0, 0, 0, 0), qt = make_float4(0, 0, 0, 0);
        if (live) {
            load_ray(F0, A, slot, o, d, path, pid);
            const DevScene &S = scene_of<BATCH>(S0, A, pid);
            const DevFrame &F = frame_of<BATCH>(F0, A, pid);
            const SlimRayTracerSettings &st = F.settings;
            if (at_cache_vertex<BATCH>(F, A)) {
                query = cache_vertex<COUNT, BATCH>(S, F, A, slot, path, pid, o, d, feat, w, qc, qt);
            } else {
                Ray ray;
                reset(ray, scale_add(d, kTraceOffset, o), d);
                Hit hit;
                int g = load_hit(A.hits, A.hit_stride, slot, hit);
                float4 pc = A.depth == 1 ? make_float4(0, 0, 0, INFINITY) : A.path_color[path];
                float3 color = xyz(pc), throughput = A.depth == 1 ? f3(1, 1, 1) : xyz(A.path_throughput[path]);
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
                        prepare_for_shading<COUNT>(S, geo, m, ray, hit, cone_scaling<BATCH>(F, pid), s, w);
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
                    A.path_color[path] = make_float4(color.x, color.y, color.z, depth);
                    A.path_throughput[path] = make_float4(throughput.x, throughput.y, throughput.z, 0.0f);
                } else if (A.sink) {
                    A.sink[path] = make_float4(color.x, color.y, color.z, 0.0f);
                } else {
                    write_pixel<BATCH>(F, pid, color, depth, BATCH || !A.early_depth);
                }
            }
        }
        uint32_t q = warp_append(A.count_out, bounce);
        if (bounce) {
            bump<COUNT>(w.bounce);
            A.rays_out[2 * (size_t)q] = make_float4(bo.x, bo.y, bo.z, __uint_as_float(path));
            A.rays_out[2 * (size_t)q + 1] = make_float4(bd.x, bd.y, bd.z, __uint_as_float(pid));
        }
        if (BATCH) {
            uint32_t cq = warp_append(A.cache.count, query);
            if (query) append_query(A.cache, cq, feat, o, d, path, pid, qc, qt);
        }
    }
    flush_stage<COUNT>(A.counters, w);
}

// ---- radiance cache ----------------------------------------------------------
// Single-request frames: the round at the cache depth runs this instead of
// shadows and shading.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_cache_gather(DevScene S, DevFrame F, QueueArgs A, CacheArgs C) {
    uint32_t n = queue_size(A);
    Work w = {};
    uint32_t stride = gridDim.x * blockDim.x;
    uint32_t rounds = (n + stride - 1) / stride;
    for (uint32_t r = 0, slot = blockIdx.x * blockDim.x + threadIdx.x; r < rounds; r++, slot += stride) {
        bool query = false;
        uint32_t path = 0, pid = 0;
        float3 o = f3(0, 0, 0), d = f3(0, 0, 0);
        float4 feat[4], qc = make_float4(0, 0, 0, 0), qt = make_float4(0, 0, 0, 0);
        if (slot < n) {
            load_ray(F, A, slot, o, d, path, pid);
            query = cache_vertex<COUNT, false>(S, F, A, slot, path, pid, o, d, feat, w, qc, qt);
        }
        uint32_t q = warp_append(C.count, query);
        if (query) append_query(C, q, feat, o, d, path, pid, qc, qt, A.hits, A.hit_stride, slot);
    }
    flush_stage<COUNT>(A.counters, w);
}

// Training paths: query j of the frame's training set restarts from the
// query's ray with zero colour and unit throughput in its own slot j.  With
// more queries than training paths the set is stratified: j takes query
// floor((j + u) * queries / capacity), u = frac(0.618034 * frame) (a
// golden-ratio sequence, so consecutive frames train on different queries).
__global__ void k_cache_select(CacheArgs C, float4 *rays, uint32_t *ray_count, float4 *hits, uint32_t hit_stride) {
    const uint32_t nq = *C.count, cap = C.train_capacity;
    const uint32_t n = nq < cap ? nq : cap;
    const double f = (double)*C.frame_counter * 0.6180339887498949;
    const double u = f - floor(f);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        uint32_t idx = j;
        if (nq > cap) {
            idx = (uint32_t)(((double)j + u) * (double)nq / (double)cap);
            if (idx >= nq) idx = nq - 1;
        }
        if (C.t_features) {
            const float4 *f = C.features + 4 * (size_t)idx;
            float4 *t = C.t_features + 4 * (size_t)j;
            t[0] = f[0]; t[1] = f[1]; t[2] = f[2]; t[3] = f[3];
        }
        if (C.q_hit && hits) {   // the query's hit: the training path's first round needs no extend
            const float4 *h = C.q_hit + 3 * (size_t)idx;
            hits[j] = h[0];
            hits[(size_t)hit_stride + j] = h[1];
            hits[2 * (size_t)hit_stride + j] = h[2];
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

// Self-training targets: a training path that reached its cache vertex
// (query q of the self-training set) ends in the cache's answer there:
// target = colour so far + throughput * radiance.  Paths that ended earlier
// already wrote their targets.
__global__ void k_cache_train_targets(const float4 *aux, const uint32_t *count, const float4 *radiance,
                                      const float4 *t_color, const float4 *t_through, float4 *t_targets) {
    const uint32_t nq = *count;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        uint32_t path = __float_as_uint(aux[2 * (size_t)q].w);
        float3 c = mul_add(xyz(radiance[q]), xyz(t_through[path]), xyz(t_color[path]));
        t_targets[path] = make_float4(c.x, c.y, c.z, 0.0f);
    }
}

// Waiting paths take the cache's answer: colour += throughput * radiance,
// then tone mapping and the canvas write of k_shade.
template <bool BATCH>
__global__ void k_cache_resolve(DevFrame F0, QueueArgs A, const float4 *path_color, const float4 *path_throughput) {
    const CacheArgs &C = A.cache;
    const uint32_t nq = *C.count;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(C.frame_counter, 1u);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        uint32_t path = __float_as_uint(C.aux[2 * (size_t)q].w);
        uint32_t pid = __float_as_uint(C.aux[2 * (size_t)q + 1].w);
        float4 pc = C.q_color ? C.q_color[q] : path_color[path];
        float3 thr = xyz(C.q_color ? C.q_through[q] : path_throughput[path]);
        float3 L = f3(0, 0, 0);
        if (C.mode == SLIM_CACHE_ON) L = xyz(C.radiance[q]);
        else if (C.mode == SLIM_CACHE_EXACT) L = xyz(C.t_targets[q]);
        write_pixel<BATCH>(frame_of<BATCH>(F0, A, pid), pid, mul_add(L, thr, xyz(pc)), pc.w);
    }
}

// ---- batched requests: primary rays of a wave --------------------------------
// tiles[t] = (request, first pixel, pixel count, first slot), slots ascending.
__global__ void k_batch_generate(QueueArgs A, const uint4 *__restrict__ tiles, uint32_t tile_count, float4 *rays,
                                 uint32_t *ray_count, uint32_t wave_samples, unsigned long long *counters) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < wave_samples; s += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = tile_count;          // last tile with first slot <= s
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (__ldg(&tiles[mid].w) <= s) lo = mid; else hi = mid;
        }
        uint4 t = tiles[lo];
        const DevFrame &F = A.frames[t.x];
        uint32_t pixel = pixel_of_slot(F.width, F.height, t.y + (s - t.w));
        float3 o, d;
        primary_ray(F, pixel, o, d);
        rays[2 * (size_t)s] = make_float4(o.x, o.y, o.z, __uint_as_float(s));
        rays[2 * (size_t)s + 1] = make_float4(d.x, d.y, d.z, __uint_as_float((t.x << kBatchPixelBits) | pixel));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *ray_count = wave_samples;
        if (counters) atomicAdd(counters, (unsigned long long)wave_samples);   // primary rays
    }
}

// ---- frame orchestration ------------------------------------------------------
struct RoundLaunch {
    const DevScene *S;
    const DevFrame *F;
    const WavefrontBuffers *B;
    int block, sms;
    cudaStream_t stream;
    StageTimer *timer;
    unsigned long long *counters;
    uint32_t bound;      // queue capacity (one ray per path slot)
    uint32_t lights;     // most lights of any scene in the round
    bool split_extend;   // closest hits as scene candidates + the persistent mesh pass
    bool share_sms = false;  // leave a block's room per SM (overlapped cache training runs beside)
    cudaEvent_t pixel_wait = nullptr;  // kernels that write pixels wait for it (a download in flight)
    const FrameDownload *depth_download = nullptr;  // first round: the depths download after shadow_gen
    const FrameDownload *pixel_download = nullptr;  // first round: each shade chunk's rows download after it
    unsigned long long *stage(int st) const { return counters ? counters + kCountersPerStage * st : nullptr; }
    uint32_t grid(const void *kernel, uint32_t work) const { return grid_for(kernel, work, block); }
    // the persistent mesh kernels run 128-thread blocks (kMeshBlock)
    uint32_t mesh_grid(const void *kernel, uint32_t work) const { return grid_for(kernel, work, kMeshBlock); }
    uint32_t grid_for(const void *kernel, uint32_t work, int block) const {
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
        if (share_sms && per_sm > 1) per_sm--;
        uint32_t g = (uint32_t)(sms * (per_sm > 0 ? per_sm : 1));
        uint32_t need = (work + block - 1) / block;
        return need < g ? (need ? need : 1) : g;
    }
};

// One bounce round over the queue `in` (primary rays at depth 1 of a single
// frame): extend, then shadows and shading -- or, at a single frame's cache
// depth, the cache gather.  Leaves `in` at the round's output queue.
// Paths still bouncing at depth >= kTailDepth finish in the fused tail kernel
// when the scene has no meshes.  With meshes the rounds stay: one thread per
// remaining path would walk mesh BVHs and every light's shadow ray serially,
// which on the config-2 scene took 1.8 ms against 1.3 ms for rounds 3-8.
constexpr uint32_t kTailDepth = 3;

// The rest of the paths queued in `in` (depth `depth` on) in one fused kernel.
template <bool COUNT, bool BATCH>
cudaError_t tail_round(const RoundLaunch &L, QueueArgs &A, uint32_t in, uint32_t depth) {
    const WavefrontBuffers &B = *L.B;
    A.depth = depth;
    A.rays_in = B.rays[in];
    A.count_in = B.queue_count + in;
    if (L.pixel_wait) {
        cudaError_t r = cudaStreamWaitEvent(L.stream, L.pixel_wait, 0);
        if (r != cudaSuccess) return r;
    }
    A.counters = L.stage(STAGE_TAIL);
    if (L.timer) L.timer->begin(STAGE_TAIL, L.stream);
    RoundLaunch T = L;
    T.block = 128;
    k_finish_paths<COUNT, BATCH><<<T.grid((const void *)k_finish_paths<COUNT, BATCH>, L.bound), 128, 0, L.stream>>>(
        *L.S, *L.F, A);
    count_launch();
    if (L.timer) L.timer->end(STAGE_TAIL, L.stream);
    return cudaGetLastError();
}

template <bool COUNT, bool BATCH>
cudaError_t trace_round(const RoundLaunch &L, QueueArgs &A, const CacheArgs &CA, uint32_t &in, uint32_t depth,
                        bool primary, bool gather, bool hits_given = false) {
    const WavefrontBuffers &B = *L.B;
    const DevScene &S = *L.S;
    const DevFrame &F = *L.F;
    cudaStream_t stream = L.stream;
    StageTimer *timer = L.timer;
    uint32_t out = in ^ 1u;
    A.depth = depth;
    A.rays_in = primary ? nullptr : B.rays[in];
    A.count_in = primary ? nullptr : B.queue_count + in;
    A.rays_out = B.rays[out];
    A.count_out = B.queue_count + out;
    // the output queue of this round is the input of the next: clear it
    cudaError_t r = cudaMemsetAsync(B.queue_count + out, 0, sizeof(uint32_t), stream);
    if (r != cudaSuccess) return r;
    A.counters = L.stage(STAGE_EXTEND);
    if (timer) timer->begin(STAGE_EXTEND, stream);
    if (hits_given) {
        // the queued rays' hit records are in place already (training paths
        // that start at their cache vertex)
    } else if (L.split_extend && B.pair_capacity >= 4) {
        // [3] candidates, [4] candidate cursor, [5] overflowed rays
        r = cudaMemsetAsync(B.queue_count + 3, 0, 3 * sizeof(uint32_t), stream);
        if (r != cudaSuccess) return r;
        k_extend_scene<COUNT, BATCH><<<L.grid((const void *)k_extend_scene<COUNT, BATCH>, L.bound), L.block, 0, stream>>>(S, F, A);
        count_launch();
        k_extend_mesh<COUNT><<<L.mesh_grid((const void *)k_extend_mesh<COUNT>, B.pair_capacity), kMeshBlock, 0,
                               stream>>>(S, F, A);
        count_launch();
        k_extend_resolve<COUNT, BATCH><<<L.grid((const void *)k_extend_resolve<COUNT, BATCH>, B.pair_capacity), L.block, 0, stream>>>(S, F, A);
        count_launch();
        k_extend_overflow<COUNT, BATCH><<<L.grid((const void *)k_extend_overflow<COUNT, BATCH>, L.bound), L.block, 0, stream>>>(S, F, A);
        count_launch();
    } else {
        k_extend<COUNT, BATCH><<<L.grid((const void *)k_extend<COUNT, BATCH>, L.bound), L.block, 0, stream>>>(S, F, A);
        count_launch();
    }
    if (timer) timer->end(STAGE_EXTEND, stream);
    if (gather) {
        A.counters = L.stage(STAGE_CACHE);
        if (timer) timer->begin(STAGE_CACHE, stream);
        k_cache_gather<COUNT><<<L.grid((const void *)k_cache_gather<COUNT>, L.bound), L.block, 0, stream>>>(S, F, A, CA);
        count_launch();
        if (timer) timer->end(STAGE_CACHE, stream);
        in = out;
        return cudaGetLastError();
    }
    // Shadow rays in light batches that fit the shadow queue.
    uint32_t per_batch = B.shadow_capacity / (L.bound ? L.bound : 1);
    if (per_batch < 1) per_batch = 1;
    for (uint32_t l0 = 0; l0 < L.lights; l0 += per_batch) {
        A.light_begin = l0;
        A.light_end = l0 + per_batch < L.lights ? l0 + per_batch : L.lights;
        r = cudaMemsetAsync(B.queue_count + 2, 0, sizeof(uint32_t), stream);
        if (r != cudaSuccess) return r;
        A.shadow_count = B.queue_count + 2;
        A.counters = L.stage(STAGE_SHADOW_GEN);
        if (timer) timer->begin(STAGE_SHADOW_GEN, stream);
        k_shadow_gen<COUNT, BATCH><<<L.grid((const void *)k_shadow_gen<COUNT, BATCH>, L.bound), L.block, 0, stream>>>(S, F, A);
        count_launch();
        if (timer) timer->end(STAGE_SHADOW_GEN, stream);
        if (l0 == 0 && A.early_depth && L.depth_download) {
            const FrameDownload *dl = L.depth_download;
            if ((r = cudaEventRecord(dl->depths_done, stream)) != cudaSuccess) return r;
            if ((r = cudaStreamWaitEvent(dl->copy_stream, dl->depths_done, 0)) != cudaSuccess) return r;
            if ((r = cudaMemcpyAsync(dl->host_depths, dl->dev_depths, dl->depth_bytes, cudaMemcpyDeviceToHost,
                                     dl->copy_stream)) != cudaSuccess)
                return r;
        }
        // Scene arrays without meshes (split_extend is false exactly then)
        // append no (shadow ray, instance) pairs: no pair counters, no mesh pass
        // (config 3: 0.021 ms of a 0.56 ms whole-frame pass).
        if (L.split_extend && (r = cudaMemsetAsync(B.queue_count + 3, 0, 2 * sizeof(uint32_t), stream)) != cudaSuccess)
            return r;
        A.counters = L.stage(STAGE_SHADOW);
        if (timer) timer->begin(STAGE_SHADOW, stream);
        k_shadow_scene<COUNT, BATCH><<<L.grid((const void *)k_shadow_scene<COUNT, BATCH>, L.bound * (A.light_end - A.light_begin)),
                                      L.block, 0, stream>>>(S, F, A);
        count_launch();
        if (timer) timer->end(STAGE_SHADOW, stream);
        if (!L.split_extend) continue;
        A.counters = L.stage(STAGE_SHADOW_MESH);
        if (timer) timer->begin(STAGE_SHADOW_MESH, stream);
        k_shadow_mesh<COUNT><<<L.mesh_grid((const void *)k_shadow_mesh<COUNT>, B.pair_capacity), kMeshBlock, 0,
                               stream>>>(S, F, A);
        count_launch();
        if (timer) timer->end(STAGE_SHADOW_MESH, stream);
    }
    if (L.pixel_wait && (r = cudaStreamWaitEvent(stream, L.pixel_wait, 0)) != cudaSuccess) return r;
    A.counters = L.stage(STAGE_SHADE);
    if (timer) timer->begin(STAGE_SHADE, stream);
    // A downloaded frame's first round shades its primary paths (slot =
    // sample, in row order) in chunks of whole 4-row tiles; each chunk's rows
    // start crossing PCIe while the next chunk shades.
    const FrameDownload *dl = L.pixel_download;
    const uint32_t chunks = dl ? kPixelChunks : 1u, tiles = (F.rows + 3) / 4;
    for (uint32_t c = 0; c < chunks; c++) {
        const uint32_t r0 = 4 * (tiles * c / chunks), r1 = c + 1 == chunks ? F.rows : 4 * (tiles * (c + 1) / chunks);
        if (dl) {
            A.slot_begin = r0 * F.width;
            A.slot_end = r1 * F.width;
            if (r1 == r0) continue;
        }
        k_shade<COUNT, BATCH><<<L.grid((const void *)k_shade<COUNT, BATCH>, dl ? A.slot_end - A.slot_begin : L.bound),
                                L.block, 0, stream>>>(S, F, A);
        count_launch();
        if (dl) {
            if ((r = cudaEventRecord(dl->pixels_done[c], stream)) != cudaSuccess) return r;
            if ((r = cudaStreamWaitEvent(dl->copy_stream, dl->pixels_done[c], 0)) != cudaSuccess) return r;
            if ((r = cudaMemcpyAsync((char *)dl->host_pixels + r0 * dl->pixel_row_bytes,
                                     (const char *)dl->dev_pixels + r0 * dl->pixel_row_bytes,
                                     (r1 - r0) * dl->pixel_row_bytes, cudaMemcpyDeviceToHost, dl->copy_stream)) != cudaSuccess)
                return r;
        }
    }
    A.slot_begin = A.slot_end = 0;
    if (timer) timer->end(STAGE_SHADE, stream);
    in = out;
    return cudaGetLastError();
}

CacheArgs cache_args(const CacheFrame *cache) {
    CacheArgs CA{};
    if (!cache) return CA;
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
    CA.frame_counter = cache->frame_counter;
    CA.mode = cache->mode;
    CA.q_color = cache->q_color;
    CA.q_through = cache->q_through;
    CA.q_hit = cache->q_hit;
    return CA;
}

// The training paths queued in `in` (from the cache vertex on; A sinks
// their radiance into the training targets): traced to max_depth, or -- with
// a training suffix, in single-request frames -- `train_suffix` bounces on,
// where the paths still going query the cache (with the training's current
// weights, `weights`) and their targets take its answer.
template <bool COUNT, bool BATCH>
cudaError_t trace_training(const RoundLaunch &L, QueueArgs &A, const CacheArgs &CA, uint32_t in,
                           const CacheFrame *cache, uint32_t max_depth, const uint8_t *weights) {
    cudaError_t e;
    const uint32_t K = cache->depth;
    const bool short_paths = !BATCH && weights && cache->train_suffix && cache->s_count &&
                             K + cache->train_suffix <= max_depth;
    // the selection copied every training path's hit at the cache vertex
    const bool hits_given = !BATCH && cache->q_hit;
    if (!short_paths) {
        if (!L.split_extend && !hits_given) return tail_round<COUNT, BATCH>(L, A, in, K);
        for (uint32_t depth = K; depth <= max_depth; depth++) {
            if (!L.split_extend && depth >= kTailDepth && depth > K) return tail_round<COUNT, BATCH>(L, A, in, depth);
            if ((e = trace_round<COUNT, BATCH>(L, A, CA, in, depth, false, false, hits_given && depth == K)) != cudaSuccess)
                return e;
        }
        return cudaSuccess;
    }
    const uint32_t last = K + cache->train_suffix;
    CacheArgs SC = CA;
    SC.features = cache->s_features;
    SC.aux = cache->s_aux;
    SC.count = cache->s_count;
    SC.q_color = SC.q_through = SC.q_hit = nullptr;   // the frame's own query records stay untouched
    for (uint32_t depth = K; depth < last; depth++)
        if ((e = trace_round<COUNT, BATCH>(L, A, CA, in, depth, false, false, hits_given && depth == K)) != cudaSuccess)
            return e;
    if ((e = cudaMemsetAsync(cache->s_count, 0, sizeof(uint32_t), L.stream)) != cudaSuccess) return e;
    if ((e = trace_round<COUNT, BATCH>(L, A, SC, in, last, false, true)) != cudaSuccess) return e;
    if ((e = nrc::launch_infer(cache->s_features, cache->s_count, 0, cache->train_capacity, cache->s_radiance, weights,
                               L.F->error_flags, L.stream)) != cudaSuccess)
        return e;
    uint32_t g = (cache->train_capacity + 255) / 256;
    if (g > (uint32_t)(L.sms * 4)) g = (uint32_t)(L.sms * 4);
    k_cache_train_targets<<<g ? g : 1, 256, 0, L.stream>>>(cache->s_aux, cache->s_count, cache->s_radiance,
                                                            cache->t_color, cache->t_through, cache->t_targets);
    count_launch();
    return cudaGetLastError();
}

// After the queries of a frame (or wave) are gathered: the training paths
// traced on (to max_depth, or a few bounces into the cache's own answers),
// the Adam steps, the network's answers, and the waiting paths resolved.
template <bool COUNT, bool BATCH>
cudaError_t cache_phase(const RoundLaunch &L, QueueArgs &A, const CacheArgs &CA, uint32_t &in, const CacheFrame *cache,
                        uint32_t max_depth) {
    const WavefrontBuffers &B = *L.B;
    cudaStream_t stream = L.stream;
    StageTimer *timer = L.timer;
    cudaError_t e;
    const int mode = cache->mode;
    const bool train = mode == SLIM_CACHE_ON && cache->trainer && cache->batch && cache->train_capacity;
    if (train && cache->train_stream && cache->train_queues && !BATCH) {
        // Overlapped training.  The previous frame's training has finished
        // once `trained` completes: take its weights for this frame's
        // queries, then hand this frame's training paths to the training
        // stream, which traces them with its own queues while this stream
        // answers the queries and the next frame's primary rays run.
        const WavefrontBuffers &TB = *cache->train_queues;
        cudaStream_t ts = cache->train_stream;
        if ((e = cudaStreamWaitEvent(stream, cache->trained, 0)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync((void *)cache->weights, cache->train_weights, nrc::kImgBytes, cudaMemcpyDeviceToDevice,
                                 stream)) != cudaSuccess)
            return e;
        if ((e = cudaMemsetAsync(TB.queue_count, 0, 8 * sizeof(uint32_t), stream)) != cudaSuccess) return e;
        if (timer) timer->begin(STAGE_CACHE, stream);
        uint32_t g = (cache->train_capacity + 255) / 256;
        if (g > (uint32_t)(L.sms * 8)) g = (uint32_t)(L.sms * 8);
        k_cache_select<<<g ? g : 1, 256, 0, stream>>>(CA, TB.rays[0], TB.queue_count, TB.hits, TB.capacity);
        count_launch();
        if (timer) timer->end(STAGE_CACHE, stream);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = cudaEventRecord(cache->selected, stream)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(ts, cache->selected, 0)) != cudaSuccess) return e;
        RoundLaunch TL{L.S, L.F, &TB, L.block, L.sms, ts, nullptr, nullptr, TB.capacity, L.lights, L.split_extend};
        QueueArgs TA = A;
        TA.hits = TB.hits;
        TA.hit_stride = TB.capacity;
        TA.shadow_rays = TB.shadow_rays;
        TA.masks = TB.shadow_mask;
        TA.pairs = TB.pairs;
        TA.pair_count = TB.queue_count + 3;
        TA.pair_cursor = TB.queue_count + 4;
        TA.pair_capacity = TB.pair_capacity;
        TA.path_color = cache->t_color;
        TA.path_throughput = cache->t_through;
        TA.sink = cache->t_targets;
        TA.skip_glow_depth = cache->depth;
        TA.samples = TB.capacity;
        if ((e = trace_training<false, false>(TL, TA, CA, 0, cache, max_depth, cache->train_weights)) != cudaSuccess)
            return e;
        for (uint32_t off = 0; off < cache->train_capacity; off += cache->batch) {
            uint32_t n = cache->train_capacity - off < cache->batch ? cache->train_capacity - off : cache->batch;
            if ((e = cache->trainer->step(cache->t_features, cache->t_targets, n, cache->counts + 1, off, ts)) !=
                cudaSuccess)
                return e;
        }
        if ((e = cudaEventRecord(cache->trained, ts)) != cudaSuccess) return e;
    } else if (mode == SLIM_CACHE_EXACT || train) {
        if (timer) timer->begin(STAGE_CACHE, stream);
        uint32_t g = (cache->train_capacity + 255) / 256;
        if (g > (uint32_t)(L.sms * 8)) g = (uint32_t)(L.sms * 8);
        k_cache_select<<<g ? g : 1, 256, 0, stream>>>(CA, B.rays[in], B.queue_count + in, B.hits, B.capacity);
        count_launch();
        if (timer) timer->end(STAGE_CACHE, stream);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        QueueArgs main = A;
        A.path_color = cache->t_color;
        A.path_throughput = cache->t_through;
        A.sink = cache->t_targets;
        A.skip_glow_depth = cache->depth;
        if ((e = trace_training<COUNT, BATCH>(L, A, CA, in, cache, max_depth,
                                              mode == SLIM_CACHE_ON ? cache->weights : nullptr)) != cudaSuccess)
            return e;
        A = main;
    }
    if (train && !(cache->train_stream && cache->train_queues && !BATCH)) {
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
        e = nrc::launch_infer(cache->features, cache->counts, 0, L.bound, cache->radiance, cache->weights,
                              L.F->error_flags, stream);
        if (timer) timer->end(STAGE_CACHE_QUERY, stream);
        if (e != cudaSuccess) return e;
    }
    if (timer) timer->begin(STAGE_CACHE, stream);
    A.cache = CA;
    k_cache_resolve<BATCH><<<L.grid((const void *)k_cache_resolve<BATCH>, L.bound), L.block, 0, stream>>>(
        *L.F, A, B.path_color, B.path_throughput);
    count_launch();
    if (timer) timer->end(STAGE_CACHE, stream);
    return cudaGetLastError();
}

template <bool COUNT>
cudaError_t run_frame(const DevScene &S, const DevFrame &F, const WavefrontBuffers &B, int block, cudaStream_t stream,
                      StageTimer *timer, const CacheFrame *cache, const FrameDownload *dl) {
    uint32_t samples = F.width * F.rows;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    RoundLaunch L{&S, &F, &B, block <= 0 ? 256 : block, sms, stream, timer, F.counters, samples, S.light_count,
                  S.mesh_count > 0};
    // the cache's overlapped training runs beside this frame: leave it room
    // (config 4: 3.50 -> 3.37 ms per frame)
    L.share_sms = cache && cache->train_stream && cache->mode == SLIM_CACHE_ON && !cache->train_suffix;
    cudaError_t e = cudaMemsetAsync(B.queue_count, 0, 8 * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    QueueArgs A{};
    A.hits = B.hits;
    A.hit_stride = B.capacity;
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
    CacheArgs CA = use_cache ? cache_args(cache) : CacheArgs{};
    const int part = use_cache ? cache->part : kCachePartWhole;
    uint32_t in = 0;
    if (part == kCachePartPhase) {   // the bands have gathered every query of the frame
        A.cache = CA;
        return cache_phase<COUNT, false>(L, A, CA, in, cache, max_depth);
    }
    // Only the query count starts over: the training count belongs to the
    // training set, which the overlapped training stream may still be using;
    // the selection that replaces the set rewrites it.  (A banded frame
    // clears it once, before its bands.)
    if (use_cache && part == kCachePartWhole &&
        (e = cudaMemsetAsync(cache->counts, 0, sizeof(uint32_t), stream)) != cudaSuccess)
        return e;
    const uint32_t last = use_cache ? cache->depth : max_depth;
    DevFrame late = F;   // the frame as the rounds after a download see it
    for (uint32_t depth = 1; depth <= last; depth++) {
        if (!L.split_extend && depth >= kTailDepth && !(use_cache && depth == last)) {
            if ((e = tail_round<COUNT, false>(L, A, in, depth)) != cudaSuccess) return e;
            break;
        }
        // the depths are final after the first round's shadow_gen (which
        // needs a light to run): they download while the shadows are traced
        const bool early_depth = depth == 1 && dl && !use_cache && L.lights > 0;
        A.early_depth = early_depth;
        L.depth_download = early_depth ? dl : nullptr;
        // every path that ends at its first hit writes its pixel in this
        // round's shading: the rows go to the host chunk by chunk
        L.pixel_download = depth == 1 && !use_cache ? dl : nullptr;
        if ((e = trace_round<COUNT, false>(L, A, CA, in, depth, depth == 1, use_cache && depth == last)) != cudaSuccess)
            return e;
        A.early_depth = 0;
        L.depth_download = L.pixel_download = nullptr;
        if (depth == 1 && dl && !use_cache) {
            // the copy stream is past the round's last shade chunk: later
            // pixels go to the host canvas directly once the copies landed
            if (!early_depth && (e = cudaMemcpyAsync(dl->host_depths, dl->dev_depths, dl->depth_bytes,
                                                     cudaMemcpyDeviceToHost, dl->copy_stream)) != cudaSuccess)
                return e;
            if ((e = cudaEventRecord(dl->copied, dl->copy_stream)) != cudaSuccess) return e;
            late.pixels = dl->mapped_pixels;
            late.depths = dl->mapped_depths;
            L.F = &late;
            L.pixel_wait = dl->copied;
        }
    }
    if (!use_cache || part == kCachePartGather) return cudaSuccess;
    A.cache = CA;
    return cache_phase<COUNT, false>(L, A, CA, in, cache, max_depth);
}

// Batched requests: every wave is a full multi-request frame over its slots.
template <bool COUNT>
cudaError_t run_batch(const BatchFrame &BF, const WavefrontBuffers &B0, int block, cudaStream_t stream0,
                      StageTimer *timer) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const CacheFrame *cache = BF.cache;
    CacheArgs CA = cache_args(cache);
    cudaError_t e;
    const bool two_lanes = BF.lane_stream && BF.lane_queues;
    if (two_lanes) {
        if ((e = cudaEventRecord(BF.lane_fork, stream0)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(BF.lane_stream, BF.lane_fork, 0)) != cudaSuccess) return e;
    }
    uint32_t next_lane = 0;
    if (BF.p_count && BF.p_total) {
        // the persistent launch takes the second lane; the waves (the cache
        // requests') all stay on the first
        cudaStream_t ps = two_lanes ? BF.lane_stream : stream0;
        if (timer) timer->begin(STAGE_FUSED, ps);
        if ((e = launch_batch_persistent(BF.scenes, BF.frames, BF.p_requests, BF.p_prefix, BF.p_count, BF.p_total,
                                         BF.p_cursor, BF.frame.error_flags, BF.frame.counters, ps)) != cudaSuccess)
            return e;
        if (timer) timer->end(STAGE_FUSED, ps);
    }
    const bool one_lane_waves = BF.p_count && BF.p_total;
    for (uint32_t wi = 0; wi < BF.wave_count; wi++) {
        const BatchWave &wave = BF.waves[wi];
        uint32_t lane = 0;
        if (two_lanes && !one_lane_waves && !(cache && wave.cache_paths)) {
            lane = next_lane;
            next_lane ^= 1u;
        }
        const WavefrontBuffers &B = lane ? *BF.lane_queues : B0;
        const cudaStream_t stream = lane ? BF.lane_stream : stream0;
        RoundLaunch L{&BF.shared, &BF.frame, &B, block <= 0 ? 256 : block, sms, stream, timer, BF.frame.counters,
                      B.capacity, wave.max_lights, BF.shared.mesh_count > 0};
        if ((e = cudaMemsetAsync(B.queue_count, 0, 8 * sizeof(uint32_t), stream)) != cudaSuccess) return e;
        const bool use_cache = cache && wave.cache_paths;
        if (use_cache && (e = cudaMemsetAsync(cache->counts, 0, sizeof(uint32_t), stream)) != cudaSuccess)
            return e;
        QueueArgs A{};
        A.hits = B.hits;
        A.hit_stride = B.capacity;
        A.shadow_rays = B.shadow_rays;
        A.masks = B.shadow_mask;
        A.pairs = B.pairs;
        A.pair_count = B.queue_count + 3;
        A.pair_cursor = B.queue_count + 4;
        A.pair_capacity = B.pair_capacity;
        A.path_color = B.path_color;
        A.path_throughput = B.path_throughput;
        A.samples = wave.samples;
        A.scenes = BF.scenes;
        A.frames = BF.frames;
        A.cache = CA;
        if (timer) timer->begin(STAGE_EXTEND, stream);
        uint32_t g = (wave.samples + 255) / 256;
        if (g > (uint32_t)(sms * 8)) g = (uint32_t)(sms * 8);
        k_batch_generate<<<g ? g : 1, 256, 0, stream>>>(A, BF.tiles + wave.first_tile, wave.tile_count, B.rays[0],
                                                         B.queue_count, wave.samples, L.stage(STAGE_EXTEND));
        count_launch();
        if (timer) timer->end(STAGE_EXTEND, stream);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        uint32_t in = 0;
        const uint32_t tail_from = cache && cache->depth >= kTailDepth ? cache->depth + 1 : kTailDepth;
        for (uint32_t depth = 1; depth <= wave.max_depth; depth++) {
            if (!L.split_extend && depth >= tail_from) {
                if ((e = tail_round<COUNT, true>(L, A, in, depth)) != cudaSuccess) return e;
                break;
            }
            if ((e = trace_round<COUNT, true>(L, A, CA, in, depth, false, false)) != cudaSuccess) return e;
        }
        if (use_cache && (e = cache_phase<COUNT, true>(L, A, CA, in, cache, wave.max_depth)) != cudaSuccess) return e;
    }
    if (two_lanes) {
        if ((e = cudaEventRecord(BF.lane_join, BF.lane_stream)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(stream0, BF.lane_join, 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace dev

cudaError_t launch_render_wavefront(const DevScene &S, const DevFrame &F, const WavefrontBuffers &B, int block,
                                    cudaStream_t stream, StageTimer *timer, const CacheFrame *cache,
                                    const FrameDownload *download) {
    if (F.settings.render_mode != SLIM_RENDER_BEAUTY)   // a single primary hit: nothing to queue
        return launch_render_fused(S, F, block, stream, timer);
    if (F.settings.max_depth == 0) return launch_render_fused(S, F, block, stream, timer);
    if (F.counters) return dev::run_frame<true>(S, F, B, block, stream, timer, cache, download);
    return dev::run_frame<false>(S, F, B, block, stream, timer, cache, download);
}

cudaError_t launch_render_batch(const BatchFrame &BF, const WavefrontBuffers &B, int block, cudaStream_t stream,
                                StageTimer *timer) {
    if (BF.frame.counters) return dev::run_batch<true>(BF, B, block, stream, timer);
    return dev::run_batch<false>(BF, B, block, stream, timer);
}

}  // namespace slim
