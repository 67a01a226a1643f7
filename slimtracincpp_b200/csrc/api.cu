// C ABI of libslimtracer_b200: the drop-in hooks of renderer/renderer_GPU.h
// plus the device-resident extensions.  One process-wide render context,
// like the reference's module-global GPU mirror (renderer/renderer_GPU.h:
// 12-20); calls are serialised by a mutex.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "slimtracer_b200.h"
#include "device_scene.h"
#include "host_common.h"
#include "kernels.h"
#include "nrc.h"

namespace slim {

std::atomic<unsigned long long> g_kernel_launches{0};

namespace {
thread_local std::string g_error;
}
int set_error(int code, const char *message) {
    g_error = message ? message : "";
    return code;
}
const char *last_error() { return g_error.c_str(); }

namespace {

int cuda_fail(cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return set_error(SLIM_ERR_CUDA, m.c_str());
}
#define SLIM_CUDA(call, what) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return cuda_fail(e_, what); } while (0)

template <typename T>
struct DevArray {
    T *ptr = nullptr;
    size_t count = 0;
    int reserve(size_t n, const char *what) {
        if (n <= count && ptr) return SLIM_OK;
        // work in flight (the cache's overlapped training stream among it) may
        // still read the old array
        if (ptr) {
            cudaDeviceSynchronize();
            cudaFree(ptr);
        }
        ptr = nullptr;
        count = 0;
        if (!n) return SLIM_OK;
        SLIM_CUDA(cudaMalloc(&ptr, n * sizeof(T)), what);
        count = n;
        return SLIM_OK;
    }
    void release() { if (ptr) cudaFree(ptr); ptr = nullptr; count = 0; }
};

// Row bands of a frame in flight at once (queue sets and streams).
constexpr int kBandLanes = 2;

// Host threads that copy a finished frame from the pinned staging canvas
// into a pageable one: the driver's own download into pageable memory runs
// at about a third of the PCIe rate, one core copying from its bounce
// buffers.
class HostCopyPool {
  public:
    ~HostCopyPool() {
        {
            std::lock_guard<std::mutex> lock(m_);
            stop_ = true;
        }
        start_.notify_all();
        for (std::thread &t : threads_) t.join();
    }
    // dst[0, bytes) = src[0, bytes), split over the pool; returns when done.
    void copy(void *dst, const void *src, size_t bytes) {
        if (bytes < kChunk) {
            memcpy(dst, src, bytes);
            return;
        }
        std::unique_lock<std::mutex> lock(m_);
        if (threads_.empty()) {
            unsigned n = std::thread::hardware_concurrency();
            n = n < 2 ? 2 : (n > 16 ? 16 : n);
            for (unsigned i = 0; i < n; i++) threads_.emplace_back([this] { work(); });
        }
        dst_ = (char *)dst;
        src_ = (const char *)src;
        bytes_ = bytes;
        next_ = 0;
        busy_ = (uint32_t)threads_.size();
        generation_++;
        start_.notify_all();
        done_.wait(lock, [this] { return busy_ == 0; });
    }

  private:
    static constexpr size_t kChunk = 1 << 20;
    void work() {
        uint64_t seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lock(m_);
            start_.wait(lock, [&] { return stop_ || generation_ != seen; });
            if (stop_) return;
            seen = generation_;
            for (;;) {
                const size_t off = next_;
                if (off >= bytes_) break;
                next_ = off + kChunk;
                const size_t n = std::min(kChunk, bytes_ - off);
                lock.unlock();
                memcpy(dst_ + off, src_ + off, n);
                lock.lock();
            }
            if (--busy_ == 0) done_.notify_one();
        }
    }
    std::mutex m_;
    std::condition_variable start_, done_;
    std::vector<std::thread> threads_;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t bytes_ = 0, next_ = 0;
    uint32_t busy_ = 0;
    uint64_t generation_ = 0;
    bool stop_ = false;
};

// Pinned, device-mapped host memory.
struct PinnedBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t n) {
        if (n <= bytes) return cudaSuccess;
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
        cudaError_t e = cudaHostAlloc(&ptr, n, cudaHostAllocMapped | cudaHostAllocPortable);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
};

// The options a context starts with: every field zero, the engine chosen per
// frame (SLIM_ENGINE_AUTO).
SlimRenderOptions initial_options() {
    SlimRenderOptions o{};
    o.engine = SLIM_ENGINE_AUTO;
    return o;
}

struct Context {
    bool initialized = false;
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_streams[kBandLanes] = {};  // banded downloads, one per band lane
    PinnedBuffer stage_pixels, stage_depths;     // pageable canvases: the frame lands here first
    HostCopyPool copy_pool;
    cudaEvent_t refit_done = nullptr;            // the last scene BVH refit, on the caller's stream
    std::vector<cudaEvent_t> band_events;        // per band: depths, copies and one per pixel chunk; then one
                                                 // per lane marking the downloads' end
    SlimSceneCounts counts{};
    std::vector<SlimGeometry> geometries;
    std::vector<SlimMaterial> materials;
    uint32_t max_mesh_height = 0;

    DevArray<float4> d_geometries, d_scene_nodes, d_mesh_nodes, d_tri_hot, d_tri_cold;
    DevArray<SlimMaterial> d_materials;
    DevArray<SlimLight> d_lights;
    DevArray<uint32_t> d_leaf_geometry, d_emissive_quads, d_refit_order;
    DevArray<DevMesh> d_meshes;
    DevArray<DevTexture> d_textures;
    DevArray<DevMip> d_mips;
    DevArray<uint4> d_quads;
    DevArray<float4> d_pixels;
    DevArray<float> d_depths;
    DevArray<uint32_t> d_error;
    DevArray<unsigned long long> d_counters;
    std::vector<uint32_t> refit_order;
    uint32_t scene_node_count = 0;

    DevScene scene{};
    SlimRenderOptions options = initial_options();
    SlimWorkCounters last_counters{};
    // Queues of the wavefront engine: one set per band lane, so that many
    // row bands of a frame can be in flight at once (lane 0 on the caller's
    // stream, the others on band_streams).
    struct WaveSet {
        DevArray<float4> color, through, rays0, rays1, hits, shadow_rays, pairs;
        DevArray<uint32_t> counts;
        DevArray<unsigned long long> mask;
        WavefrontBuffers B{};
    } wave[kBandLanes];
    cudaStream_t band_streams[kBandLanes] = {};
    cudaEvent_t band_fork = nullptr, band_join[kBandLanes] = {};
    struct EventTimer *timer = nullptr;

    // neural radiance cache
    struct Cache : CacheTrainer {
        bool configured = false;
        SlimRadianceCacheConfig config{};
        DevArray<float> params, m, v, grad, partials, loss_partials, loss;
        DevArray<uint8_t> image;
        DevArray<float4> features, aux, radiance, t_features, t_targets, t_color, t_through;
        DevArray<float4> s_features, s_aux, s_radiance;   // self-training queries
        DevArray<uint32_t> s_count;
        DevArray<float4> q_color, q_through, q_hit;       // per-query path state and hit record
        DevArray<uint32_t> counts;
        DevArray<uint32_t> state;      // [0] Adam steps taken, [1] cache frames (training-set offsets)
        uint32_t *error_flags = nullptr;
        // overlapped training: second stream, its own queues, the queries' weight snapshot
        cudaStream_t stream_b = nullptr;
        cudaEvent_t ev_selected = nullptr, ev_trained = nullptr;
        DevArray<uint8_t> image_infer;
        DevArray<float4> tq_rays0, tq_rays1, tq_hits, tq_shadow, tq_pairs;
        DevArray<uint32_t> tq_counts;
        DevArray<unsigned long long> tq_masks;
        WavefrontBuffers tq{};
        cudaError_t step(const float4 *f, const float4 *t, uint32_t samples, const uint32_t *count, uint32_t offset,
                         cudaStream_t stream) override {
            nrc::AdamArgs a{};
            a.lr = config.learning_rate;
            a.beta1 = config.beta1;
            a.beta2 = config.beta2;
            a.eps = config.epsilon;
            a.step = state.ptr;
            return nrc::launch_train_step(f, t, samples, count, offset, params.ptr, m.ptr, v.ptr, image.ptr,
                                          partials.ptr, loss_partials.ptr, grad.ptr, loss.ptr, a, error_flags, stream);
        }
    } cache;
};

// CUDA-event pairs around stage launches, resolved lazily.
struct EventTimer : StageTimer {
    struct Pending { int stage; cudaEvent_t a, b; };
    std::vector<cudaEvent_t> pool;
    std::vector<Pending> pending;
    cudaEvent_t open[STAGE_COUNT] = {};
    uint32_t launches[STAGE_COUNT] = {};
    double total_ms[STAGE_COUNT] = {};
    cudaEvent_t take() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void begin(int stage, cudaStream_t stream) override {
        cudaEvent_t e = take();
        cudaEventRecord(e, stream);
        open[stage] = e;
    }
    void end(int stage, cudaStream_t stream) override {
        cudaEvent_t e = take();
        cudaEventRecord(e, stream);
        pending.push_back({stage, open[stage], e});
        open[stage] = nullptr;
    }
    void resolve() {
        for (auto &p : pending) {
            cudaEventSynchronize(p.b);
            float ms = 0;
            cudaEventElapsedTime(&ms, p.a, p.b);
            launches[p.stage]++;
            total_ms[p.stage] += ms;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    void reset() {
        resolve();
        for (int i = 0; i < STAGE_COUNT; i++) { launches[i] = 0; total_ms[i] = 0; }
    }
};
const char *kStageNames[STAGE_COUNT] = {"fused", "extend", "shadow_gen", "shadow", "shade", "refit", "shadow_mesh",
                                        "cache", "cache_train", "cache_query", "tail"};
SlimWorkCounters g_stage_work[STAGE_COUNT];

Context g_ctx;
std::mutex g_mutex;

int ensure_device(Context &c) {
    if (c.device >= 0) return SLIM_OK;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return set_error(SLIM_ERR_CUDA, "no CUDA device: libslimtracer_b200 has no CPU path");
    SLIM_CUDA(cudaGetDevice(&c.device), "cudaGetDevice");
    SLIM_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    int rc = c.d_error.reserve(1, "alloc error flags");
    if (rc) return rc;
    rc = c.d_counters.reserve(kCountersPerStage * STAGE_COUNT, "alloc counters");
    if (rc) return rc;
    SLIM_CUDA(cudaMemset(c.d_error.ptr, 0, sizeof(uint32_t)), "clear error flags");
    return SLIM_OK;
}

// Geometry record: rotation | position,type | scale,material | 1/scale,flags+mesh<<8.
// 1/scale is the IEEE quotient Ray::localize computes (core/ray.h:30).
void pack_geometry(const SlimGeometry &g, float4 out[4]) {
    const SlimTransform &t = g.transform;
    uint32_t type = (uint32_t)g.type, bits = (uint32_t)g.flags | ((g.type == SLIM_GEOMETRY_MESH ? g.id : 0u) << 8);
    float ft, fm, fb;
    memcpy(&ft, &type, 4);
    memcpy(&fm, &g.material_id, 4);
    memcpy(&fb, &bits, 4);
    out[0] = make_float4(t.orientation.axis.x, t.orientation.axis.y, t.orientation.axis.z, t.orientation.amount);
    out[1] = make_float4(t.position.x, t.position.y, t.position.z, ft);
    out[2] = make_float4(t.scale.x, t.scale.y, t.scale.z, fm);
    out[3] = make_float4(1.0f / t.scale.x, 1.0f / t.scale.y, 1.0f / t.scale.z, fb);
}

int check_scene_arrays(const SlimSceneData *s) {
    if (!s) return set_error(SLIM_ERR_ARGUMENT, "scene is null");
    const SlimSceneCounts &n = s->counts;
    if (!n.geometries || !s->geometries) return set_error(SLIM_ERR_ARGUMENT, "scene has no geometries");
    if (!n.materials || !s->materials) return set_error(SLIM_ERR_ARGUMENT, "scene has no materials");
    if (n.lights && !s->lights) return set_error(SLIM_ERR_ARGUMENT, "scene lights array missing");
    if (n.lights > (uint32_t)kMaxLights) return set_error(SLIM_ERR_LIMIT, "more lights than supported (64)");
    if (n.meshes && !s->meshes) return set_error(SLIM_ERR_ARGUMENT, "scene meshes array missing");
    if (n.textures && !s->textures) return set_error(SLIM_ERR_ARGUMENT, "scene textures array missing");
    if (n.geometries > (1u << 24)) return set_error(SLIM_ERR_LIMIT, "too many geometries");
    for (uint32_t g = 0; g < n.geometries; g++) {
        const SlimGeometry &geo = s->geometries[g];
        if (geo.material_id >= n.materials) return set_error(SLIM_ERR_ARGUMENT, "geometry material_id out of range");
        if (geo.type == SLIM_GEOMETRY_MESH && geo.id >= n.meshes) return set_error(SLIM_ERR_ARGUMENT, "geometry mesh id out of range");
    }
    for (uint32_t m = 0; m < n.materials; m++) {
        const SlimMaterial &mat = s->materials[m];
        for (uint32_t k = 0; k < mat.texture_count && k < 2; k++)
            if (mat.texture_ids[k] >= n.textures && (mat.flags & (SLIM_MATERIAL_HAS_ALBEDO_MAP | SLIM_MATERIAL_HAS_NORMAL_MAP)))
                return set_error(SLIM_ERR_ARGUMENT, "material texture id out of range");
    }
    return SLIM_OK;
}

// BVH topology checks that make every device traversal terminate and stay
// in bounds: inner nodes point strictly forward to an adjacent child pair,
// leaves point inside the primitive array, and the height fits the stack.
int check_bvh(const SlimBVHNode *nodes, uint32_t node_count, uint32_t primitive_count, uint32_t height, const char *what) {
    if (!nodes || !node_count) return set_error(SLIM_ERR_ARGUMENT, what);
    if (height + 2 > (uint32_t)kStackCapacity) return set_error(SLIM_ERR_LIMIT, "BVH deeper than the traversal stack (62 levels)");
    for (uint32_t i = 0; i < node_count; i++) {
        const SlimBVHNode &n = nodes[i];
        if (n.leaf_count) {
            if ((uint64_t)n.first_index + n.leaf_count > primitive_count) return set_error(SLIM_ERR_ARGUMENT, what);
        } else if (n.first_index <= i || (uint64_t)n.first_index + 1 >= node_count) {
            return set_error(SLIM_ERR_ARGUMENT, what);
        }
    }
    return SLIM_OK;
}

// Depth of the deepest node reachable from the root (the traversal stack
// bound) -- the stored height byte is not trusted.
uint32_t bvh_depth(const SlimBVHNode *nodes, uint32_t node_count) {
    std::vector<uint32_t> depth(node_count, 0);
    uint32_t deepest = 1;
    depth[0] = 1;
    for (uint32_t i = 0; i < node_count; i++) {
        if (!depth[i] || nodes[i].leaf_count) continue;
        uint32_t c = nodes[i].first_index;
        depth[c] = depth[c + 1] = depth[i] + 1;
        if (depth[i] + 1 > deepest) deepest = depth[i] + 1;
    }
    return deepest;
}

int upload_emissive(Context &c) {
    std::vector<uint32_t> list;
    for (uint32_t g = 0; g < c.counts.geometries; g++) {
        const SlimGeometry &geo = c.geometries[g];
        if (geo.type == SLIM_GEOMETRY_QUAD && (c.materials[geo.material_id].flags & SLIM_MATERIAL_IS_EMISSIVE))
            list.push_back(g);
    }
    c.scene.emissive_quad_count = (uint32_t)list.size();
    int rc = c.d_emissive_quads.reserve(list.size() ? list.size() : 1, "alloc emissive list");
    if (rc) return rc;
    if (!list.empty())
        SLIM_CUDA(cudaMemcpy(c.d_emissive_quads.ptr, list.data(), list.size() * 4, cudaMemcpyHostToDevice), "upload emissive list");
    c.scene.emissive_quads = c.d_emissive_quads.ptr;
    return SLIM_OK;
}

int upload_geometries(Context &c, const SlimSceneData *s) {
    uint32_t n = c.counts.geometries;
    for (uint32_t g = 0; g < n; g++) {
        const SlimGeometry &geo = s->geometries[g];
        if (geo.material_id >= c.counts.materials) return set_error(SLIM_ERR_ARGUMENT, "geometry material_id out of range");
        if (geo.type == SLIM_GEOMETRY_MESH && geo.id >= c.counts.meshes) return set_error(SLIM_ERR_ARGUMENT, "geometry mesh id out of range");
    }
    c.geometries.assign(s->geometries, s->geometries + n);
    std::vector<float4> packed(4 * (size_t)n);
    for (uint32_t g = 0; g < n; g++) pack_geometry(c.geometries[g], &packed[4 * (size_t)g]);
    int rc = c.d_geometries.reserve(packed.size(), "alloc geometries");
    if (rc) return rc;
    SLIM_CUDA(cudaMemcpy(c.d_geometries.ptr, packed.data(), packed.size() * sizeof(float4), cudaMemcpyHostToDevice),
              "upload geometries");
    c.scene.geometries = c.d_geometries.ptr;
    return upload_emissive(c);
}

int upload_materials(Context &c, const SlimSceneData *s) {
    uint32_t n = c.counts.materials;
    for (uint32_t m = 0; m < n; m++) {
        const SlimMaterial &mat = s->materials[m];
        for (uint32_t k = 0; k < mat.texture_count && k < 2; k++)
            if (mat.texture_ids[k] >= c.counts.textures && (mat.flags & (SLIM_MATERIAL_HAS_ALBEDO_MAP | SLIM_MATERIAL_HAS_NORMAL_MAP)))
                return set_error(SLIM_ERR_ARGUMENT, "material texture id out of range");
    }
    c.materials.assign(s->materials, s->materials + n);
    int rc = c.d_materials.reserve(n, "alloc materials");
    if (rc) return rc;
    SLIM_CUDA(cudaMemcpy(c.d_materials.ptr, s->materials, n * sizeof(SlimMaterial), cudaMemcpyHostToDevice), "upload materials");
    c.scene.materials = c.d_materials.ptr;
    return c.geometries.empty() ? SLIM_OK : upload_emissive(c);
}

int upload_lights(Context &c, const SlimSceneData *s) {
    uint32_t n = c.counts.lights;
    int rc = c.d_lights.reserve(n ? n : 1, "alloc lights");
    if (rc) return rc;
    if (n) SLIM_CUDA(cudaMemcpy(c.d_lights.ptr, s->lights, n * sizeof(SlimLight), cudaMemcpyHostToDevice), "upload lights");
    c.scene.lights = c.d_lights.ptr;
    c.scene.light_count = n;
    return SLIM_OK;
}

// Parent-before-child order of the scene BVH's inner nodes, reversed, so the
// refit kernel can process it level by level bottom-up in one launch.
void build_refit_order(Context &c, const SlimBVHNode *nodes, uint32_t node_count) {
    c.refit_order.clear();
    for (uint32_t i = 0; i < node_count; i++)
        if (!nodes[i].leaf_count) c.refit_order.push_back(i);
}

int upload_scene_bvh(Context &c, const SlimSceneData *s) {
    uint32_t n = s->bvh.node_count;
    int rc = check_bvh(s->bvh.nodes, n, c.counts.geometries, 0, "scene BVH malformed");
    if (rc) return rc;
    if (!s->bvh_leaf_geometry_indices) return set_error(SLIM_ERR_ARGUMENT, "scene BVH leaf indices missing");
    if (bvh_depth(s->bvh.nodes, n) + 2 > (uint32_t)kStackCapacity) return set_error(SLIM_ERR_LIMIT, "scene BVH deeper than the traversal stack");
    for (uint32_t g = 0; g < c.counts.geometries; g++)
        if (s->bvh_leaf_geometry_indices[g] >= c.counts.geometries) return set_error(SLIM_ERR_ARGUMENT, "scene BVH leaf index out of range");
    rc = c.d_scene_nodes.reserve(2 * (size_t)n, "alloc scene BVH");
    if (rc) return rc;
    rc = c.d_leaf_geometry.reserve(c.counts.geometries, "alloc leaf indices");
    if (rc) return rc;
    SLIM_CUDA(cudaMemcpy(c.d_scene_nodes.ptr, s->bvh.nodes, n * sizeof(SlimBVHNode), cudaMemcpyHostToDevice), "upload scene BVH");
    SLIM_CUDA(cudaMemcpy(c.d_leaf_geometry.ptr, s->bvh_leaf_geometry_indices, c.counts.geometries * 4, cudaMemcpyHostToDevice),
              "upload leaf indices");
    build_refit_order(c, s->bvh.nodes, n);
    rc = c.d_refit_order.reserve(c.refit_order.size() ? c.refit_order.size() : 1, "alloc refit order");
    if (rc) return rc;
    if (!c.refit_order.empty())
        SLIM_CUDA(cudaMemcpy(c.d_refit_order.ptr, c.refit_order.data(), c.refit_order.size() * 4, cudaMemcpyHostToDevice),
                  "upload refit order");
    c.scene_node_count = n;
    c.scene.scene_nodes = c.d_scene_nodes.ptr;
    c.scene.leaf_geometry = c.d_leaf_geometry.ptr;
    c.scene.scene_node_count = n;
    c.scene.flags = s->flags;
    return SLIM_OK;
}

int upload_meshes(Context &c, const SlimSceneData *s) {
    uint32_t n = c.counts.meshes;
    std::vector<DevMesh> metas(n ? n : 1);
    size_t total_nodes = 0, total_tris = 0;
    c.max_mesh_height = 0;
    for (uint32_t i = 0; i < n; i++) {
        const SlimMesh &m = s->meshes[i];
        if (!m.triangles || !m.triangle_count) return set_error(SLIM_ERR_ARGUMENT, "mesh has no triangles");
        int rc = check_bvh(m.bvh.nodes, m.bvh.node_count, m.triangle_count, 0, "mesh BVH malformed");
        if (rc) return rc;
        if (m.triangle_count >= (1u << kLeafCountShift))
            return set_error(SLIM_ERR_LIMIT, "mesh has 2^26 triangles or more");
        for (uint32_t k = 1; k < m.bvh.node_count; k++)   // a root leaf is tested without being packed
            if (m.bvh.nodes[k].leaf_count >= (1u << (32 - kLeafCountShift)))
                return set_error(SLIM_ERR_LIMIT, "mesh BVH leaf below the root holds 64 triangles or more");
        uint32_t d = bvh_depth(m.bvh.nodes, m.bvh.node_count);
        if (d + 2 > (uint32_t)kStackCapacity) return set_error(SLIM_ERR_LIMIT, "mesh BVH deeper than the traversal stack (62 levels)");
        if (d > c.max_mesh_height) c.max_mesh_height = d;
        DevMesh &dm = metas[i];
        memset(&dm, 0, sizeof(dm));
        dm.aabb_min[0] = m.aabb.min.x; dm.aabb_min[1] = m.aabb.min.y; dm.aabb_min[2] = m.aabb.min.z;
        dm.aabb_max[0] = m.aabb.max.x; dm.aabb_max[1] = m.aabb.max.y; dm.aabb_max[2] = m.aabb.max.z;
        // The reference's builder lays a mesh BVH out as the root followed by
        // child pairs, so every pair starts at an odd node index: an odd
        // absolute root index puts every pair on a 64-byte boundary and no
        // pair straddles two 128-byte cache lines (at most one node of
        // padding per mesh).
        if (total_nodes % 2 == 0) total_nodes++;
        dm.node_offset = (uint32_t)total_nodes;
        dm.tri_offset = (uint32_t)total_tris;
        dm.tri_count = m.triangle_count;
        dm.node_count = m.bvh.node_count;
        dm.has_normals = m.normals_count != 0;
        dm.has_uvs = m.uvs_count != 0;
        total_nodes += m.bvh.node_count;
        total_tris += m.triangle_count;
        if (total_nodes > 0xFFFFFFFFull / 2 || total_tris > 0xFFFFFFFFull / 4) return set_error(SLIM_ERR_LIMIT, "meshes too large");
    }

    int rc = c.d_meshes.reserve(metas.size(), "alloc meshes");
    if (rc) return rc;
    SLIM_CUDA(cudaMemcpy(c.d_meshes.ptr, metas.data(), metas.size() * sizeof(DevMesh), cudaMemcpyHostToDevice), "upload meshes");
    c.scene.meshes = c.d_meshes.ptr;
    c.scene.mesh_count = n;
    if (!n) {
        c.scene.mesh_nodes = nullptr;
        c.scene.tri_hot = c.scene.tri_cold = nullptr;
        return SLIM_OK;
    }
    rc = c.d_mesh_nodes.reserve(2 * total_nodes, "alloc mesh nodes");
    if (rc) return rc;
    rc = c.d_tri_hot.reserve(3 * total_tris, "alloc triangles");
    if (rc) return rc;
    rc = c.d_tri_cold.reserve(4 * total_tris, "alloc triangle attributes");
    if (rc) return rc;
    std::vector<float4> hot, cold;
    for (uint32_t i = 0; i < n; i++) {
        const SlimMesh &m = s->meshes[i];
        const DevMesh &dm = metas[i];
        SLIM_CUDA(cudaMemcpy(c.d_mesh_nodes.ptr + 2 * (size_t)dm.node_offset, m.bvh.nodes, m.bvh.node_count * sizeof(SlimBVHNode),
                             cudaMemcpyHostToDevice), "upload mesh nodes");
        hot.resize(3 * (size_t)m.triangle_count);
        cold.resize(4 * (size_t)m.triangle_count);
        for (uint32_t t = 0; t < m.triangle_count; t++) {
            const SlimTriangle &tr = m.triangles[t];
            const float *l = tr.local_to_tangent;
            hot[3 * t + 0] = make_float4(tr.position.x, tr.position.y, tr.position.z, tr.normal.x);
            hot[3 * t + 1] = make_float4(tr.normal.y, tr.normal.z, l[0], l[1]);
            hot[3 * t + 2] = make_float4(l[3], l[4], l[6], l[7]);
            cold[4 * t + 0] = make_float4(tr.n1.x, tr.n1.y, tr.n1.z, tr.n2.x);
            cold[4 * t + 1] = make_float4(tr.n2.y, tr.n2.z, tr.n3.x, tr.n3.y);
            cold[4 * t + 2] = make_float4(tr.n3.z, tr.uv1.x, tr.uv1.y, tr.uv2.x);
            cold[4 * t + 3] = make_float4(tr.uv2.y, tr.uv3.x, tr.uv3.y, tr.uv_coverage);
        }
        SLIM_CUDA(cudaMemcpy(c.d_tri_hot.ptr + 3 * (size_t)dm.tri_offset, hot.data(), hot.size() * sizeof(float4),
                             cudaMemcpyHostToDevice), "upload triangles");
        SLIM_CUDA(cudaMemcpy(c.d_tri_cold.ptr + 4 * (size_t)dm.tri_offset, cold.data(), cold.size() * sizeof(float4),
                             cudaMemcpyHostToDevice), "upload triangle attributes");
    }
    c.scene.mesh_nodes = c.d_mesh_nodes.ptr;
    c.scene.tri_hot = c.d_tri_hot.ptr;
    c.scene.tri_cold = c.d_tri_cold.ptr;
    return SLIM_OK;
}

int upload_textures(Context &c, const SlimSceneData *s) {
    uint32_t n = c.counts.textures;
    c.scene.texture_count = n;
    if (!n) {
        c.scene.textures = nullptr;
        c.scene.mips = nullptr;
        c.scene.quads = nullptr;
        return SLIM_OK;
    }
    std::vector<DevTexture> texs(n);
    std::vector<DevMip> mips;
    size_t total_quads = 0;
    for (uint32_t i = 0; i < n; i++) {
        const SlimTexture &t = s->textures[i];
        bool cube = (t.flags & SLIM_IMAGE_CUBEMAP) != 0;
        if (!t.mips || !t.mip_count || (cube && t.mip_count < 3)) return set_error(SLIM_ERR_ARGUMENT, "texture has no mips");
        DevTexture &dt = texs[i];
        memset(&dt, 0, sizeof(dt));
        dt.width = t.width; dt.height = t.height; dt.mip_count = t.mip_count; dt.flags = t.flags;
        dt.mip_base = (uint32_t)mips.size();
        for (uint32_t m = 0; m < t.mip_count; m++) {
            const SlimTextureMip &mip = t.mips[m];
            if (!mip.texel_quads || !mip.width || !mip.height) return set_error(SLIM_ERR_ARGUMENT, "texture mip empty");
            DevMip dm{mip.width, mip.height, (uint32_t)total_quads, 0};
            mips.push_back(dm);
            total_quads += (size_t)(mip.width + 1) * (mip.height + 1);
            if (total_quads > 0xFFFFFFFFull) return set_error(SLIM_ERR_LIMIT, "textures too large");
        }
    }
    int rc = c.d_textures.reserve(n, "alloc textures");
    if (rc) return rc;
    rc = c.d_mips.reserve(mips.size(), "alloc mips");
    if (rc) return rc;
    rc = c.d_quads.reserve(total_quads, "alloc texel quads");
    if (rc) return rc;
    SLIM_CUDA(cudaMemcpy(c.d_textures.ptr, texs.data(), n * sizeof(DevTexture), cudaMemcpyHostToDevice), "upload textures");
    SLIM_CUDA(cudaMemcpy(c.d_mips.ptr, mips.data(), mips.size() * sizeof(DevMip), cudaMemcpyHostToDevice), "upload mips");
    std::vector<uint4> quads;
    for (uint32_t i = 0; i < n; i++) {
        const SlimTexture &t = s->textures[i];
        for (uint32_t m = 0; m < t.mip_count; m++) {
            const SlimTextureMip &mip = t.mips[m];
            size_t q = (size_t)(mip.width + 1) * (mip.height + 1);
            quads.resize(q);
            for (size_t k = 0; k < q; k++) {
                const SlimTexelQuad &src = mip.texel_quads[k];
                uint4 v;
                memcpy(&v.x, src.R, 4);
                memcpy(&v.y, src.G, 4);
                memcpy(&v.z, src.B, 4);
                v.w = 0;
                quads[k] = v;
            }
            SLIM_CUDA(cudaMemcpy(c.d_quads.ptr + mips[texs[i].mip_base + m].quad_offset, quads.data(), q * sizeof(uint4),
                                 cudaMemcpyHostToDevice), "upload texel quads");
        }
    }
    c.scene.textures = c.d_textures.ptr;
    c.scene.mips = c.d_mips.ptr;
    c.scene.quads = c.d_quads.ptr;
    return SLIM_OK;
}

int require_init(Context &c, const SlimSceneData *s) {
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (!s) return set_error(SLIM_ERR_ARGUMENT, "scene is null");
    return SLIM_OK;
}

int check_settings(const Context &c, const SlimRayTracerSettings *st) {
    int8_t ids[3] = {st->skybox_color_texture_id, st->skybox_radiance_texture_id, st->skybox_irradiance_texture_id};
    for (int8_t id : ids) {
        if (id < 0) continue;
        if ((uint32_t)id >= c.counts.textures) return set_error(SLIM_ERR_ARGUMENT, "skybox texture id out of range");
    }
    if (st->render_mode == SLIM_RENDER_MIP_LEVEL)
        for (int k = 0; k < 9; k++)
            if (st->mip_level_colors[k] < 0 || st->mip_level_colors[k] > 35) return set_error(SLIM_ERR_ARGUMENT, "bad mip level color");
    return SLIM_OK;
}

int ensure_wavefront(Context &c, uint32_t samples, int set);


// Buffers and per-frame parameters of a radiance-cache frame.
int cache_frame(Context &c, uint32_t samples, CacheFrame &cf) {
    Context::Cache &k = c.cache;
    if (!k.configured) return set_error(SLIM_ERR_STATE, "radiance_cache is set but slimRadianceCacheConfigure was not called");
    const int mode = c.options.radiance_cache;
    const uint32_t cap = mode == SLIM_CACHE_EXACT ? samples : k.config.train_samples;
    int rc;
    if ((rc = k.features.reserve(4 * (size_t)samples, "alloc cache queries"))) return rc;
    if ((rc = k.aux.reserve(2 * (size_t)samples, "alloc cache query rays"))) return rc;
    if ((rc = k.radiance.reserve(samples, "alloc cache answers"))) return rc;
    if ((rc = k.counts.reserve(2, "alloc cache counters"))) return rc;
    if ((rc = k.q_color.reserve(samples, "alloc cache query paths"))) return rc;
    if ((rc = k.q_through.reserve(samples, "alloc cache query paths"))) return rc;
    if ((rc = k.q_hit.reserve(3 * (size_t)samples, "alloc cache query hits"))) return rc;
    if (cap) {
        if ((rc = k.t_targets.reserve(cap, "alloc training targets"))) return rc;
        if ((rc = k.t_color.reserve(cap, "alloc training paths"))) return rc;
        if ((rc = k.t_through.reserve(cap, "alloc training paths"))) return rc;
        if (mode == SLIM_CACHE_ON && (rc = k.t_features.reserve(4 * (size_t)cap, "alloc training samples"))) return rc;
        if (mode == SLIM_CACHE_ON && k.config.train_suffix) {
            if ((rc = k.s_features.reserve(4 * (size_t)cap, "alloc self-training queries"))) return rc;
            if ((rc = k.s_aux.reserve(2 * (size_t)cap, "alloc self-training queries"))) return rc;
            if ((rc = k.s_radiance.reserve(cap, "alloc self-training answers"))) return rc;
            if ((rc = k.s_count.reserve(1, "alloc self-training counter"))) return rc;
        }
    }
    cf.mode = mode;
    cf.depth = k.config.cache_depth;
    cf.features = k.features.ptr;
    cf.aux = k.aux.ptr;
    cf.radiance = k.radiance.ptr;
    cf.counts = k.counts.ptr;
    cf.q_color = k.q_color.ptr;
    cf.q_through = k.q_through.ptr;
    cf.q_hit = k.q_hit.ptr;
    cf.train_capacity = cap;
    cf.t_features = k.t_features.ptr;
    cf.t_targets = k.t_targets.ptr;
    cf.t_color = k.t_color.ptr;
    cf.t_through = k.t_through.ptr;
    cf.frame_counter = k.state.ptr + 1;
    cf.batch = k.config.batch;
    cf.weights = k.image.ptr;
    cf.trainer = (mode == SLIM_CACHE_ON && k.config.train) ? &k : nullptr;
    if (mode == SLIM_CACHE_ON && k.config.train_suffix && cap) {
        cf.train_suffix = k.config.train_suffix;
        cf.s_features = k.s_features.ptr;
        cf.s_aux = k.s_aux.ptr;
        cf.s_radiance = k.s_radiance.ptr;
        cf.s_count = k.s_count.ptr;
    }
    k.error_flags = c.d_error.ptr;
    // Overlapped training (not while counting work: the counters of a frame
    // must be complete when the frame's stream is).
    if (cf.trainer && k.config.overlap && !c.options.count_work && cap) {
        if (!k.stream_b) {
            // highest priority: the training rounds are long chains of small
            // launches that should take SMs as soon as the frame's blocks free
            // them (default and lowest priority measured the same)
            int least = 0, greatest = 0;
            cudaDeviceGetStreamPriorityRange(&least, &greatest);
            SLIM_CUDA(cudaStreamCreateWithPriority(&k.stream_b, cudaStreamNonBlocking, greatest), "cache training stream");
            SLIM_CUDA(cudaEventCreateWithFlags(&k.ev_selected, cudaEventDisableTiming), "cache event");
            SLIM_CUDA(cudaEventCreateWithFlags(&k.ev_trained, cudaEventDisableTiming), "cache event");
        }
        size_t lights = c.scene.light_count ? c.scene.light_count : 1;
        size_t instances = 0;
        for (const SlimGeometry &g : c.geometries) instances += g.type == SLIM_GEOMETRY_MESH;
        size_t shadow = (size_t)cap * lights, pairs = shadow * (instances < 4 ? (instances ? instances : 1) : 4);
        if ((rc = k.tq_rays0.reserve(2 * (size_t)cap, "alloc training queues"))) return rc;
        if ((rc = k.tq_rays1.reserve(2 * (size_t)cap, "alloc training queues"))) return rc;
        if ((rc = k.tq_hits.reserve(3 * (size_t)cap, "alloc training queues"))) return rc;
        if ((rc = k.tq_shadow.reserve(2 * shadow, "alloc training queues"))) return rc;
        if ((rc = k.tq_pairs.reserve(3 * pairs, "alloc training queues"))) return rc;
        if ((rc = k.tq_counts.reserve(8, "alloc training queues"))) return rc;
        if ((rc = k.tq_masks.reserve(cap, "alloc training queues"))) return rc;
        if ((rc = k.image_infer.reserve(nrc::kImgBytes, "alloc weight snapshot"))) return rc;
        WavefrontBuffers &T = k.tq;
        T.path_color = k.t_color.ptr;
        T.path_throughput = k.t_through.ptr;
        T.rays[0] = k.tq_rays0.ptr;
        T.rays[1] = k.tq_rays1.ptr;
        T.queue_count = k.tq_counts.ptr;
        T.hits = k.tq_hits.ptr;
        T.shadow_rays = k.tq_shadow.ptr;
        T.shadow_mask = k.tq_masks.ptr;
        T.pairs = k.tq_pairs.ptr;
        T.capacity = cap;
        T.shadow_capacity = (uint32_t)shadow;
        T.pair_capacity = (uint32_t)pairs;
        cf.train_stream = k.stream_b;
        cf.selected = k.ev_selected;
        cf.trained = k.ev_trained;
        cf.train_queues = &k.tq;
        cf.train_weights = k.image.ptr;
        cf.weights = k.image_infer.ptr;
    }
    return SLIM_OK;
}

StageTimer *timer_for(Context &c) {
    if (!c.options.profile_stages) return nullptr;
    if (!c.timer) c.timer = new EventTimer();
    return c.timer;
}

// A frame reads the scene BVH that the last slimRefitSceneBVH wrote, on
// whatever stream that ran.  A stream being captured into a graph is left
// alone: a captured wait on an event recorded outside the capture is an
// error, and the caller orders the graph's launch.
int wait_for_refit(Context &c, cudaStream_t stream) {
    if (!c.refit_done) return SLIM_OK;
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    SLIM_CUDA(cudaStreamIsCapturing(stream, &capture), "capture status");
    if (capture == cudaStreamCaptureStatusNone) SLIM_CUDA(cudaStreamWaitEvent(stream, c.refit_done, 0), "wait for the refit");
    return SLIM_OK;
}

// Frames of fewer samples than this in scenes without meshes run the fused
// kernel under SLIM_ENGINE_AUTO even when their paths bounce.  Measured on
// one B200, render only, the fused kernel against the wavefront engine:
// config 1's implicit scene (paths end at the first hit) 0.031 / 0.050 ms at
// 320x180, 0.036 / 0.069 at 640x360, 0.105 / 0.129 at 1280x720, 0.209 /
// 0.258 at 1920x1080; config 3's glass, mirror and texture scene at depth 8
// 0.075 / 0.163, 0.109 / 0.192, 0.274 / 0.260, 0.506 / 0.449 ms.
constexpr uint64_t kAutoFusedSamples = 1u << 19;

// The engine a frame runs on: the option, or under SLIM_ENGINE_AUTO the
// faster one for its scene and size (the pixels are the same).  Meshes and
// radiance-cache frames need the wavefront engine's split walks and queues.
// Can a path of this frame go past its first hit?  Only through a
// reflective or refractive material, with max depth above 1.
bool paths_bounce(const Context &c, const SlimRayTracerSettings *settings) {
    if (settings->max_depth <= 1) return false;
    for (const SlimMaterial &m : c.materials)
        if (m.flags & (SLIM_MATERIAL_IS_REFLECTIVE | SLIM_MATERIAL_IS_REFRACTIVE)) return true;
    return false;
}

int frame_engine(const Context &c, const SlimRayTracerSettings *settings, uint64_t samples) {
    if (c.options.engine != SLIM_ENGINE_AUTO) return c.options.engine;
    if (c.options.radiance_cache != SLIM_CACHE_OFF || c.scene.mesh_count) return SLIM_ENGINE_WAVEFRONT;
    return !paths_bounce(c, settings) || samples < kAutoFusedSamples ? SLIM_ENGINE_MEGAKERNEL : SLIM_ENGINE_WAVEFRONT;
}

// Renders the sample rows [row_begin, row_begin + rows) of the canvas (rows
// 0: all of them); `first` clears the work counters (the first band of a
// frame).
int render(Context &c, const SlimCanvasData *canvas, const SlimCameraRayProjection *projection,
           const SlimRayTracerSettings *settings, float4 *d_pixels, float *d_depths, cudaStream_t stream,
           uint32_t row_begin, uint32_t rows, bool first, int set = 0, const FrameDownload *download = nullptr,
           int cache_part = kCachePartWhole) {
    const SlimDimensions &dim = canvas->dimensions;
    if (!dim.width || !dim.height) return set_error(SLIM_ERR_ARGUMENT, "canvas has zero size");
    if (canvas->antialias < SLIM_AA_NONE || canvas->antialias > SLIM_AA_SSAA) return set_error(SLIM_ERR_ARGUMENT, "bad antialias mode");
    int rc = check_settings(c, settings);
    if (rc) return rc;
    if ((rc = wait_for_refit(c, stream))) return rc;
    uint32_t s = canvas->antialias == SLIM_AA_SSAA ? 2 : 1;
    DevFrame F;
    memset(&F, 0, sizeof(F));
    F.projection = *projection;
    F.settings = *settings;
    F.width = (uint32_t)dim.width * s;
    F.height = (uint32_t)dim.height * s;
    if (rows == 0) { row_begin = 0; rows = F.height; }
    if (row_begin >= F.height || rows > F.height - row_begin) return set_error(SLIM_ERR_ARGUMENT, "band outside the canvas");
    F.row_begin = row_begin;
    F.rows = rows;
    F.stride = dim.stride ? dim.stride : dim.width;
    if (F.stride < dim.width) return set_error(SLIM_ERR_ARGUMENT, "canvas stride below width");
    F.antialias = canvas->antialias;
    F.cones_per_pixel = c.options.ray_cones == SLIM_CONES_PER_PIXEL;
    F.pixels = d_pixels;
    F.depths = d_depths;
    F.error_flags = c.d_error.ptr;
    F.counters = c.options.count_work ? c.d_counters.ptr : nullptr;
    if (F.counters && first)
        SLIM_CUDA(cudaMemsetAsync(F.counters, 0, kCountersPerStage * STAGE_COUNT * sizeof(unsigned long long), stream),
                  "clear counters");
    StageTimer *timer = timer_for(c);
    cudaError_t e;
    if (frame_engine(c, settings, (uint64_t)F.width * F.height) == SLIM_ENGINE_MEGAKERNEL) {
        e = launch_render_fused(c.scene, F, c.options.block_size, stream, timer, !paths_bounce(c, settings));
    } else {
        // the cache phase of a banded frame needs no path queues of its own
        if (cache_part != kCachePartPhase && (rc = ensure_wavefront(c, F.width * F.rows, set))) return rc;
        CacheFrame cf;
        const CacheFrame *cache = nullptr;
        if (c.options.radiance_cache != SLIM_CACHE_OFF) {
            if ((rc = cache_frame(c, F.width * F.height, cf))) return rc;
            cf.part = cache_part;
            cache = &cf;
        }
        e = launch_render_wavefront(c.scene, F, c.wave[set].B, c.options.block_size, stream, timer, cache, download);
    }
    if (e != cudaSuccess) return cuda_fail(e, "render launch");
    return SLIM_OK;
}

int ensure_wavefront(Context &c, uint32_t samples, int set) {
    Context::WaveSet &W = c.wave[set];
    size_t lights = c.scene.light_count ? c.scene.light_count : 1;
    size_t budget = (size_t)(c.options.shadow_queue_mb > 0 ? c.options.shadow_queue_mb : 1024) << 20;
    size_t shadow = (size_t)samples * lights;
    size_t max_shadow = budget / (2 * sizeof(float4));
    if (shadow > max_shadow) shadow = max_shadow < samples ? samples : max_shadow;
    if (shadow > 0xFFFFFFFFull) shadow = 0xFFFFFFFFull;
    if ((uint64_t)samples << 6 > 0xFFFFFFFFull) return set_error(SLIM_ERR_LIMIT, "frame too large for the wavefront queues");
    size_t instances = 0;
    for (const SlimGeometry &g : c.geometries) instances += g.type == SLIM_GEOMETRY_MESH;
    size_t pairs = shadow * (instances < 4 ? (instances ? instances : 1) : 4);
    size_t max_pairs = budget / (3 * sizeof(float4));
    if (pairs > max_pairs) pairs = max_pairs;
    if (pairs > 0xFFFFFFFFull) pairs = 0xFFFFFFFFull;
    if (W.B.capacity >= samples && W.shadow_rays.count >= 2 * shadow && W.pairs.count >= 3 * (pairs ? pairs : 1)) {
        // the arrays are large enough; this frame's queue budget still sets
        // the capacities (overflow and light batches as a fresh context's)
        W.B.shadow_capacity = (uint32_t)shadow;
        W.B.pair_capacity = (uint32_t)pairs;
        return SLIM_OK;
    }
    uint32_t n = samples;
    int rc = 0;
    if ((rc = W.color.reserve(n, "alloc path colour"))) return rc;
    if ((rc = W.through.reserve(n, "alloc path throughput"))) return rc;
    if ((rc = W.rays0.reserve(2 * (size_t)n, "alloc ray queue"))) return rc;
    if ((rc = W.rays1.reserve(2 * (size_t)n, "alloc ray queue"))) return rc;
    if ((rc = W.hits.reserve(3 * (size_t)n, "alloc hit records"))) return rc;
    if ((rc = W.shadow_rays.reserve(2 * shadow, "alloc shadow queue"))) return rc;
    if ((rc = W.counts.reserve(8, "alloc queue counters"))) return rc;
    if ((rc = W.mask.reserve(n, "alloc shadow masks"))) return rc;
    if ((rc = W.pairs.reserve(3 * (pairs ? pairs : 1), "alloc shadow candidate pairs"))) return rc;
    WavefrontBuffers &B = W.B;
    B.path_color = W.color.ptr;
    B.path_throughput = W.through.ptr;
    B.rays[0] = W.rays0.ptr;
    B.rays[1] = W.rays1.ptr;
    B.queue_count = W.counts.ptr;
    B.hits = W.hits.ptr;
    B.shadow_rays = W.shadow_rays.ptr;
    B.shadow_mask = W.mask.ptr;
    B.capacity = n;
    B.shadow_capacity = (uint32_t)shadow;
    B.pairs = W.pairs.ptr;
    B.pair_capacity = (uint32_t)pairs;
    return SLIM_OK;
}

int read_errors(Context &c, cudaStream_t stream) {
    uint32_t flags = 0;
    SLIM_CUDA(cudaMemcpyAsync(&flags, c.d_error.ptr, 4, cudaMemcpyDeviceToHost, stream), "read error flags");
    SLIM_CUDA(cudaStreamSynchronize(stream), "render");
    if (flags) {
        SLIM_CUDA(cudaMemset(c.d_error.ptr, 0, 4), "clear error flags");
        if (flags & kErrStack) return set_error(SLIM_ERR_STACK, "a traversal stack overflowed on the device");
        if (flags & nrc::kErrTimeout) return set_error(SLIM_ERR_TIMEOUT, "a tensor-core wait timed out on the device");
        return set_error(SLIM_ERR_STATE, "device reported an index error");
    }
    return SLIM_OK;
}

int read_counters(Context &c, cudaStream_t stream) {
    if (!c.options.count_work) return SLIM_OK;
    unsigned long long v[kCountersPerStage * STAGE_COUNT];
    SLIM_CUDA(cudaMemcpyAsync(v, c.d_counters.ptr, sizeof(v), cudaMemcpyDeviceToHost, stream), "read counters");
    SLIM_CUDA(cudaStreamSynchronize(stream), "read counters");
    SlimWorkCounters &w = c.last_counters;
    memset(&w, 0, sizeof(w));
    for (int st = 0; st < STAGE_COUNT; st++) {
        const unsigned long long *p = v + kCountersPerStage * st;
        SlimWorkCounters &sw = g_stage_work[st];
        sw.primary_rays = p[0]; sw.shadow_rays = p[1]; sw.bounce_rays = p[2];
        sw.scene_node_tests = p[3]; sw.mesh_node_tests = p[4]; sw.triangle_tests = p[5];
        sw.geometry_tests = p[6]; sw.mesh_hit_fetches = p[7]; sw.texel_taps = p[8];
        sw.pixels = 0;
        sw.shadow_scene_node_tests = p[9]; sw.shadow_mesh_node_tests = p[10];
        sw.shadow_triangle_tests = p[11]; sw.shadow_geometry_tests = p[12];
        w.primary_rays += p[0]; w.shadow_rays += p[1]; w.bounce_rays += p[2];
        w.scene_node_tests += p[3]; w.mesh_node_tests += p[4]; w.triangle_tests += p[5];
        w.geometry_tests += p[6]; w.mesh_hit_fetches += p[7]; w.texel_taps += p[8];
        w.shadow_scene_node_tests += p[9]; w.shadow_mesh_node_tests += p[10];
        w.shadow_triangle_tests += p[11]; w.shadow_geometry_tests += p[12];
    }
    w.pixels = w.primary_rays;
    return SLIM_OK;
}

// Row bands of a wavefront frame.  Each band is a complete wavefront pass
// over its rows; bands take the kBandLanes queue sets in turn, the first on
// the caller's stream and the others on band_streams, so that many bands
// are in flight at once and the ends of one band's persistent launches, where most of the GPU
// waits on a few long walks, overlap the other band's work.  Into a pinned
// host canvas every band downloads as soon as it is done, while the next
// renders.  The pixels are the same for any band count.  Two bands, one
// per lane (config 2: 1.44 ms, 1.79 end to end); three, four or six bands
// queue behind each other on the two lanes: 1.82 / 1.79 / 1.95 ms (2.08 /
// 2.19 / 2.25 end to end).
constexpr uint32_t kDefaultRowBands = 2;
constexpr size_t kStagedDownloadBytes = 4u << 20;   // pageable canvases from here up go through staging
constexpr double kBandRatio = 2.0 / 3.0;
// A frame downloaded into a mapped pinned canvas ends when its pixels are on
// the host: a smaller second band finishes its first round sooner and its
// rows start crossing PCIe earlier (config 2 end to end: 67/33 1.79 ms,
// 60/40 1.84 ms, 70/30 1.80 ms; as the device-resident split 67/33 costs
// 1.51 against 1.45 ms).
constexpr double kDownloadBandRatio = 0.5;
constexpr uint32_t kMinBandedSamples = 1u << 18;

// Radiance-cache frames split into bands only when the cache trains
// overlapped on its own stream and queues (ON mode): the bands gather their
// queries into the frame's query buffers and one cache phase follows them.
bool banded_cache(const Context &c) {
    const Context::Cache &k = c.cache;
    return c.options.radiance_cache == SLIM_CACHE_ON && k.configured && k.config.train && k.config.overlap &&
           k.config.train_samples && !c.options.count_work;
}

uint32_t row_bands(const Context &c, const SlimRayTracerSettings *settings, uint32_t sample_rows, uint32_t samples) {
    if (frame_engine(c, settings, samples) == SLIM_ENGINE_MEGAKERNEL) return 1;
    if (c.options.radiance_cache != SLIM_CACHE_OFF && !banded_cache(c)) return 1;
    uint32_t bands = c.options.row_bands ? (uint32_t)c.options.row_bands
                                         : (samples >= kMinBandedSamples ? kDefaultRowBands : 1u);
    const uint32_t tiles = sample_rows / 4;
    if (bands > tiles) bands = tiles ? tiles : 1;
    return bands;
}

// The device's address of pinned host memory mapped into its address space.
bool mapped_host(const void *p, void **device_address) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type != cudaMemoryTypeHost || !a.devicePointer) return false;
    *device_address = a.devicePointer;
    return true;
}

bool pinned_host(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// The frame into d_pixels / d_depths on `stream`; with host_pixels set, it
// also downloads into the host canvas (ordered before the end of `stream`).
int render_frame(Context &c, const SlimCanvasData *canvas, const SlimCameraRayProjection *projection,
                 const SlimRayTracerSettings *settings, float4 *d_pixels, float *d_depths, cudaStream_t stream,
                 SlimPixel *host_pixels, float *host_depths, size_t pixel_count, size_t depth_count) {
    const SlimDimensions &dim = canvas->dimensions;
    if (!dim.width || !dim.height) return set_error(SLIM_ERR_ARGUMENT, "canvas has zero size");
    uint32_t stride = dim.stride ? dim.stride : dim.width;
    const bool ssaa = canvas->antialias == SLIM_AA_SSAA;
    const uint32_t sample_rows = (uint32_t)dim.height * (ssaa ? 2 : 1);
    const uint32_t bands = row_bands(c, settings, sample_rows, sample_rows * (uint32_t)dim.width * (ssaa ? 2 : 1));
    const bool download = host_pixels != nullptr;
    int rc;
    if (bands <= 1) {
        // A fused frame into a pinned canvas the device can address: the
        // kernel writes every pixel and depth once and reads none, so it
        // writes them there, over PCIe while it renders, and no copy follows
        // (config 1 end to end: 0.169 -> 0.141 ms).
        float4 *mapped_pixels = nullptr;
        float *mapped_depths = nullptr;
        if (download &&
            frame_engine(c, settings, (uint64_t)sample_rows * dim.width * (ssaa ? 2 : 1)) == SLIM_ENGINE_MEGAKERNEL &&
            mapped_host(host_pixels, (void **)&mapped_pixels) && mapped_host(host_depths, (void **)&mapped_depths))
            return render(c, canvas, projection, settings, mapped_pixels, mapped_depths, stream, 0, 0, true);
        if ((rc = render(c, canvas, projection, settings, d_pixels, d_depths, stream, 0, 0, true))) return rc;
        if (download) {
            SLIM_CUDA(cudaMemcpyAsync(host_pixels, d_pixels, pixel_count * sizeof(float4), cudaMemcpyDeviceToHost,
                                      stream), "download pixels");
            SLIM_CUDA(cudaMemcpyAsync(host_depths, d_depths, depth_count * sizeof(float), cudaMemcpyDeviceToHost,
                                      stream), "download depths");
        }
        return SLIM_OK;
    }
    // Canvas entries per sample row: a row of pixels (4 SSAA samples per
    // pixel, two sample rows per canvas row) and of depths (4 per pixel
    // under MSAA and SSAA).
    const size_t pix_per_row = ssaa ? (size_t)stride * 2 : stride;
    const size_t dep_per_row = ssaa ? (size_t)stride * 2 : (size_t)stride * (canvas->antialias == SLIM_AA_NONE ? 1 : 4);
    const bool cache_bands = c.options.radiance_cache != SLIM_CACHE_OFF;
    // a cache frame's query pixels are written by the cache phase after the
    // bands: it downloads whole, at the end
    const bool banded_download = download && !cache_bands && pinned_host(host_pixels) && pinned_host(host_depths);
    // Pinned canvases the device can address: each band's rows download as
    // soon as its first round is done, and later pixels go straight there.
    float4 *mapped_pixels = nullptr;
    float *mapped_depths = nullptr;
    const bool early = banded_download &&
                       frame_engine(c, settings, (uint64_t)sample_rows * dim.width * (ssaa ? 2 : 1)) == SLIM_ENGINE_WAVEFRONT &&
                       c.options.radiance_cache == SLIM_CACHE_OFF && settings->render_mode == SLIM_RENDER_BEAUTY &&
                       settings->max_depth >= 1 && mapped_host(host_pixels, (void **)&mapped_pixels) &&
                       mapped_host(host_depths, (void **)&mapped_depths);
    if (!c.band_fork) SLIM_CUDA(cudaEventCreateWithFlags(&c.band_fork, cudaEventDisableTiming), "band event");
    for (int l = 1; l < kBandLanes; l++) {
        if (!c.band_streams[l])
            SLIM_CUDA(cudaStreamCreateWithFlags(&c.band_streams[l], cudaStreamNonBlocking), "band stream");
        if (!c.band_join[l]) SLIM_CUDA(cudaEventCreateWithFlags(&c.band_join[l], cudaEventDisableTiming), "band event");
    }
    // one copy stream per lane: a band's copy waits for its own band only,
    // not for a band on another lane that finishes later
    for (int l = 0; banded_download && l < kBandLanes; l++)
        if (!c.copy_streams[l])
            SLIM_CUDA(cudaStreamCreateWithFlags(&c.copy_streams[l], cudaStreamNonBlocking), "copy stream");
    constexpr uint32_t kEventsPerBand = 2 + kPixelChunks;
    while (c.band_events.size() < kEventsPerBand * bands + kBandLanes) {
        cudaEvent_t e;
        SLIM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "band event");
        c.band_events.push_back(e);
    }
    // Work counters are cleared once, before the fork; the band stream
    // starts after everything the caller queued so far (the refit included).
    if (c.options.count_work)
        SLIM_CUDA(cudaMemsetAsync(c.d_counters.ptr, 0, kCountersPerStage * STAGE_COUNT * sizeof(unsigned long long),
                                  stream), "clear counters");
    if ((rc = wait_for_refit(c, stream))) return rc;
    if (cache_bands) {
        // the frame's query buffers, and its query count cleared once for all bands
        CacheFrame cf;
        if ((rc = cache_frame(c, sample_rows * (uint32_t)dim.width * (ssaa ? 2 : 1), cf))) return rc;
        SLIM_CUDA(cudaMemsetAsync(cf.counts, 0, sizeof(uint32_t), stream), "clear cache queries");
    }
    SLIM_CUDA(cudaEventRecord(c.band_fork, stream), "band fork");
    cudaStream_t lanes[kBandLanes];
    lanes[0] = stream;
    for (int l = 1; l < kBandLanes; l++) {
        lanes[l] = c.band_streams[l];
        SLIM_CUDA(cudaStreamWaitEvent(lanes[l], c.band_fork, 0), "band fork");
    }
    // Band b gets a share proportional to kBandRatio^b: unequal bands keep
    // the two pipelines out of step, so one's launch tails meet the other's
    // full launches (config 2, two bands: 60/40 1.62 ms, 50/50 1.67 ms).
    const uint32_t tiles = sample_rows / 4;
    const double ratio = early ? kDownloadBandRatio : kBandRatio;
    double total = 0.0, w = 1.0;
    for (uint32_t b = 0; b < bands; b++, w *= ratio) total += w;
    double cum = 0.0;
    w = 1.0;
    uint32_t r0 = 0;
    for (uint32_t b = 0; b < bands; b++, w *= ratio) {
        cum += w;
        uint32_t r1 = sample_rows;
        if (b + 1 < bands) {
            uint32_t t = (uint32_t)((double)tiles * cum / total);
            const uint32_t lo = r0 / 4 + 1, hi = tiles - (bands - 1 - b);   // at least one tile band each
            t = t < lo ? lo : (t > hi ? hi : t);
            r1 = 4 * t;
        }
        const int lane = (int)(b % kBandLanes);
        const cudaStream_t ls = lanes[lane];
        const size_t p0 = pix_per_row * r0, pn = pix_per_row * (r1 - r0);
        const size_t d0 = dep_per_row * r0, dn = dep_per_row * (r1 - r0);
        if (early) {
            FrameDownload dl{};
            dl.copy_stream = c.copy_streams[lane];
            dl.depths_done = c.band_events[kEventsPerBand * b];
            dl.copied = c.band_events[kEventsPerBand * b + 1];
            for (uint32_t k = 0; k < kPixelChunks; k++) dl.pixels_done[k] = c.band_events[kEventsPerBand * b + 2 + k];
            dl.host_pixels = host_pixels + p0;
            dl.host_depths = host_depths + d0;
            dl.dev_pixels = d_pixels + p0;
            dl.dev_depths = d_depths + d0;
            dl.depth_bytes = dn * sizeof(float);
            dl.pixel_row_bytes = pix_per_row * sizeof(float4);
            dl.mapped_pixels = mapped_pixels;
            dl.mapped_depths = mapped_depths;
            if ((rc = render(c, canvas, projection, settings, d_pixels, d_depths, ls, r0, r1 - r0, false, lane, &dl)))
                return rc;
            r0 = r1;
            continue;
        }
        if ((rc = render(c, canvas, projection, settings, d_pixels, d_depths, ls, r0, r1 - r0, false, lane, nullptr,
                         cache_bands ? kCachePartGather : kCachePartWhole)))
            return rc;
        if (banded_download) {
            SLIM_CUDA(cudaEventRecord(c.band_events[b], ls), "band event");
            SLIM_CUDA(cudaStreamWaitEvent(c.copy_streams[lane], c.band_events[b], 0), "band wait");
            SLIM_CUDA(cudaMemcpyAsync(host_pixels + p0, d_pixels + p0, pn * sizeof(float4), cudaMemcpyDeviceToHost,
                                      c.copy_streams[lane]), "download pixels");
            SLIM_CUDA(cudaMemcpyAsync(host_depths + d0, d_depths + d0, dn * sizeof(float), cudaMemcpyDeviceToHost,
                                      c.copy_streams[lane]), "download depths");
        }
        r0 = r1;
    }
    for (int l = 1; l < kBandLanes; l++) {
        SLIM_CUDA(cudaEventRecord(c.band_join[l], lanes[l]), "band join");
        SLIM_CUDA(cudaStreamWaitEvent(stream, c.band_join[l], 0), "band join");
    }
    // every band's queries are in: training-path selection, the network's
    // answers and the waiting paths of the whole frame
    if (cache_bands &&
        (rc = render(c, canvas, projection, settings, d_pixels, d_depths, stream, 0, 0, false, 0, nullptr, kCachePartPhase)))
        return rc;
    if (banded_download) {
        for (int l = 0; l < kBandLanes; l++) {
            SLIM_CUDA(cudaEventRecord(c.band_events[kEventsPerBand * bands + l], c.copy_streams[l]), "downloads done");
            SLIM_CUDA(cudaStreamWaitEvent(stream, c.band_events[kEventsPerBand * bands + l], 0), "downloads done");
        }
    } else if (download) {
        SLIM_CUDA(cudaMemcpyAsync(host_pixels, d_pixels, pixel_count * sizeof(float4), cudaMemcpyDeviceToHost, stream),
                  "download pixels");
        SLIM_CUDA(cudaMemcpyAsync(host_depths, d_depths, depth_count * sizeof(float), cudaMemcpyDeviceToHost, stream),
                  "download depths");
    }
    return SLIM_OK;
}

}  // namespace
}  // namespace slim

using namespace slim;

// A batch's tables point into the shared mesh and texture arrays and its
// graph into the cache's weights: re-initialising either drops the batch.
static void invalidate_batch();
// Forgets the cached device addresses of the no-alloc scratch (looked up
// again by the next no-alloc call).
static void noalloc_forget();

extern "C" {

int slimGetVersion(void) { return 1; }
const char *slimGetLastError(void) { return slim::last_error(); }

int slimInitDataOnGPU(const SlimSceneData *scene) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    int rc = ensure_device(c);
    if (rc) return rc;
    invalidate_batch();
    noalloc_forget();
    if ((rc = check_scene_arrays(scene))) return rc;
    c.initialized = false;
    c.counts = scene->counts;
    c.geometries.clear();
    c.materials.clear();
    if ((rc = upload_materials(c, scene))) return rc;
    if ((rc = upload_meshes(c, scene))) return rc;
    if ((rc = upload_textures(c, scene))) return rc;
    if ((rc = upload_lights(c, scene))) return rc;
    if ((rc = upload_geometries(c, scene))) return rc;
    c.scene.geometry_count = c.counts.geometries;
    c.scene.material_count = c.counts.materials;
    if ((rc = upload_scene_bvh(c, scene))) return rc;
    c.initialized = true;
    return SLIM_OK;
}

int slimUploadLights(const SlimSceneData *scene) {
    std::lock_guard<std::mutex> lock(g_mutex);
    int rc = require_init(g_ctx, scene);
    if (rc) return rc;
    if (scene->counts.lights != g_ctx.counts.lights || (scene->counts.lights && !scene->lights))
        return set_error(SLIM_ERR_STATE, "light count differs from slimInitDataOnGPU");
    return upload_lights(g_ctx, scene);
}

int slimUploadCameras(const SlimSceneData *scene) {
    std::lock_guard<std::mutex> lock(g_mutex);
    int rc = require_init(g_ctx, scene);
    if (rc) return rc;
    // Cameras are not read by the trace path (renderOnGPU takes the
    // projection); the hook exists for call compatibility.
    if (scene->counts.cameras != g_ctx.counts.cameras) return set_error(SLIM_ERR_STATE, "camera count differs");
    return SLIM_OK;
}

int slimUploadGeometries(const SlimSceneData *scene) {
    std::lock_guard<std::mutex> lock(g_mutex);
    int rc = require_init(g_ctx, scene);
    if (rc) return rc;
    if (scene->counts.geometries != g_ctx.counts.geometries || !scene->geometries)
        return set_error(SLIM_ERR_STATE, "geometry count differs from slimInitDataOnGPU");
    return upload_geometries(g_ctx, scene);
}

int slimUploadMaterials(const SlimSceneData *scene) {
    std::lock_guard<std::mutex> lock(g_mutex);
    int rc = require_init(g_ctx, scene);
    if (rc) return rc;
    if (scene->counts.materials != g_ctx.counts.materials || !scene->materials)
        return set_error(SLIM_ERR_STATE, "material count differs from slimInitDataOnGPU");
    return upload_materials(g_ctx, scene);
}

int slimUploadSceneBVH(const SlimSceneData *scene) {
    std::lock_guard<std::mutex> lock(g_mutex);
    int rc = require_init(g_ctx, scene);
    if (rc) return rc;
    if (scene->counts.geometries != g_ctx.counts.geometries) return set_error(SLIM_ERR_STATE, "geometry count differs");
    return upload_scene_bvh(g_ctx, scene);
}

int slimRenderOnGPU(const SlimCanvasData *canvas, const SlimCameraRayProjection *projection,
                    const SlimRayTracerSettings *settings) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (!canvas || !projection || !settings || !canvas->pixels || !canvas->depths)
        return set_error(SLIM_ERR_ARGUMENT, "slimRenderOnGPU: null argument");
    const SlimDimensions &dim = canvas->dimensions;
    uint32_t stride = dim.stride ? dim.stride : dim.width;
    size_t wth = (size_t)stride * dim.height;
    size_t pixel_count = wth * (canvas->antialias == SLIM_AA_SSAA ? 4 : 1);
    size_t depth_count = wth * (canvas->antialias == SLIM_AA_NONE ? 1 : 4);
    int rc = c.d_pixels.reserve(pixel_count, "alloc frame");
    if (rc) return rc;
    if ((rc = c.d_depths.reserve(depth_count, "alloc depths"))) return rc;
    // A pageable canvas of a large frame: the frame downloads into pinned
    // staging (banded, while it renders), then host threads copy it over.
    SlimPixel *host_pixels = canvas->pixels;
    float *host_depths = canvas->depths;
    const size_t pixel_bytes = pixel_count * sizeof(float4), depth_bytes = depth_count * sizeof(float);
    const bool staged = pixel_bytes >= kStagedDownloadBytes &&
                        !(pinned_host(canvas->pixels) && pinned_host(canvas->depths));
    if (staged) {
        SLIM_CUDA(c.stage_pixels.reserve(pixel_bytes), "pinned staging");
        SLIM_CUDA(c.stage_depths.reserve(depth_bytes), "pinned staging");
        host_pixels = (SlimPixel *)c.stage_pixels.ptr;
        host_depths = (float *)c.stage_depths.ptr;
    }
    if ((rc = render_frame(c, canvas, projection, settings, c.d_pixels.ptr, c.d_depths.ptr, c.stream, host_pixels,
                           host_depths, pixel_count, depth_count)))
        return rc;
    if ((rc = read_errors(c, c.stream))) return rc;
    if (staged) {
        c.copy_pool.copy(canvas->pixels, host_pixels, pixel_bytes);
        c.copy_pool.copy(canvas->depths, host_depths, depth_bytes);
    }
    return read_counters(c, c.stream);
}

int slimRenderToDevice(const SlimCanvasData *canvas, const SlimCameraRayProjection *projection,
                       const SlimRayTracerSettings *settings, void *d_pixels, void *d_depths, void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (!canvas || !projection || !settings || !d_pixels || !d_depths)
        return set_error(SLIM_ERR_ARGUMENT, "slimRenderToDevice: null argument");
    int rc = render_frame(c, canvas, projection, settings, (float4 *)d_pixels, (float *)d_depths, (cudaStream_t)stream,
                          nullptr, nullptr, 0, 0);
    if (rc) return rc;
    if (c.options.count_work) {
        if ((rc = read_errors(c, (cudaStream_t)stream))) return rc;
        return read_counters(c, (cudaStream_t)stream);
    }
    return SLIM_OK;
}

int slimTracePrimary(const SlimCameraRayProjection *projection, int width, int height, void *d_geometry_ids,
                     void *d_primitive_ids, void *d_distances, void *d_from_behind, void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (!projection || width <= 0 || height <= 0 || !d_geometry_ids || !d_primitive_ids || !d_distances || !d_from_behind)
        return set_error(SLIM_ERR_ARGUMENT, "slimTracePrimary: bad argument");
    cudaError_t e = launch_trace_primary(c.scene, *projection, (uint32_t)width, (uint32_t)height, (int *)d_geometry_ids,
                                         (uint32_t *)d_primitive_ids, (float *)d_distances, (uint8_t *)d_from_behind,
                                         c.d_error.ptr, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "trace primary launch");
    return read_errors(c, (cudaStream_t)stream);
}

int slimGetLaunchCount(uint64_t *count) {
    if (!count) return set_error(SLIM_ERR_ARGUMENT, "count is null");
    *count = g_kernel_launches.load();
    return SLIM_OK;
}

int slimSynchronize(void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (c.cache.ev_trained) SLIM_CUDA(cudaStreamWaitEvent((cudaStream_t)stream, c.cache.ev_trained, 0), "join training");
    SLIM_CUDA(cudaStreamSynchronize((cudaStream_t)stream), "synchronize");
    int rc = read_errors(c, (cudaStream_t)stream);
    if (rc) return rc;
    return read_counters(c, (cudaStream_t)stream);
}

int slimPick(const SlimCameraRayProjection *projection, int x, int y, SlimPick *out) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (!projection || !out) return set_error(SLIM_ERR_ARGUMENT, "slimPick: null argument");
    SlimPick *d = nullptr;
    SLIM_CUDA(cudaMalloc(&d, sizeof(SlimPick)), "pick buffer");
    cudaError_t e = launch_pick(c.scene, *projection, x, y, d, c.d_error.ptr, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, sizeof(SlimPick), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "pick");
    return read_errors(c, nullptr);
}

int slimSetRenderOptions(const SlimRenderOptions *options) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!options) return set_error(SLIM_ERR_ARGUMENT, "options is null");
    if (options->engine < SLIM_ENGINE_WAVEFRONT || options->engine > SLIM_ENGINE_AUTO || options->ray_cones < 0 || options->ray_cones > 1 ||
        options->scene_bvh < 0 || options->scene_bvh > 1 || options->block_size < 0 || options->block_size > 256 ||
        (options->block_size % 32) || options->radiance_cache < SLIM_CACHE_OFF ||
        options->radiance_cache > SLIM_CACHE_EXACT || options->row_bands < 0 || options->row_bands > 64)
        return set_error(SLIM_ERR_ARGUMENT, "bad render options");
    g_ctx.options = *options;
    return SLIM_OK;
}

int slimGetRenderOptions(SlimRenderOptions *options) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!options) return set_error(SLIM_ERR_ARGUMENT, "options is null");
    *options = g_ctx.options;
    return SLIM_OK;
}

int slimGetWorkCounters(SlimWorkCounters *counters) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!counters) return set_error(SLIM_ERR_ARGUMENT, "counters is null");
    *counters = g_ctx.last_counters;
    return SLIM_OK;
}

int slimDownloadSceneBVH(SlimSceneData *scene) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (!scene || !scene->bvh.nodes) return set_error(SLIM_ERR_ARGUMENT, "slimDownloadSceneBVH: null argument");
    if (scene->bvh.node_count != c.scene_node_count)
        return set_error(SLIM_ERR_STATE, "scene BVH node count differs from the uploaded one");
    if (c.refit_done) SLIM_CUDA(cudaEventSynchronize(c.refit_done), "wait for the refit");
    SLIM_CUDA(cudaMemcpy(scene->bvh.nodes, c.d_scene_nodes.ptr, c.scene_node_count * sizeof(SlimBVHNode),
                         cudaMemcpyDeviceToHost), "download scene BVH");
    return SLIM_OK;
}

int slimRefitSceneBVH(void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    cudaError_t e = launch_refit_scene_bvh(c.scene, c.d_scene_nodes.ptr, c.d_refit_order.ptr,
                                           (uint32_t)c.refit_order.size(), (cudaStream_t)stream, timer_for(c));
    if (e != cudaSuccess) return cuda_fail(e, "refit launch");
    // the next frame, on whatever stream, reads the refit nodes
    if (!c.refit_done) SLIM_CUDA(cudaEventCreateWithFlags(&c.refit_done, cudaEventDisableTiming), "refit event");
    SLIM_CUDA(cudaEventRecord(c.refit_done, (cudaStream_t)stream), "refit event");
    return SLIM_OK;
}

int slimGetStageStats(SlimStageStats *stats, int capacity, int *count) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!stats || capacity < 0 || !count) return set_error(SLIM_ERR_ARGUMENT, "slimGetStageStats: bad argument");
    Context &c = g_ctx;
    if (c.timer) c.timer->resolve();
    int n = 0;
    for (int st = 0; st < STAGE_COUNT && n < capacity; st++) {
        SlimStageStats &o = stats[n++];
        memset(&o, 0, sizeof(o));
        strncpy(o.name, kStageNames[st], sizeof(o.name) - 1);
        if (c.timer) {
            o.launches = c.timer->launches[st];
            o.total_ms = (float)c.timer->total_ms[st];
        }
        o.work = g_stage_work[st];
    }
    *count = n;
    return SLIM_OK;
}

int slimResetStageStats(void) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_ctx.timer) g_ctx.timer->reset();
    memset(g_stage_work, 0, sizeof(g_stage_work));
    return SLIM_OK;
}

int slimProjectionReset(const float orientation9[9], const float position3[3], float focal_length, int width, int height,
                        int antialias_ssaa, SlimCameraRayProjection *out) {
    return slim::projection_reset(orientation9, position3, focal_length, width, height, antialias_ssaa, out);
}

int slimBuildSceneBVH(SlimSceneData *scene) { return slim::build_scene_bvh(scene); }

int slimBuildMesh(float *positions, uint32_t vertex_count, const uint32_t *position_indices, uint32_t triangle_count,
                  const float *normals, uint32_t normals_count, const uint32_t *normal_indices, const float *uvs,
                  uint32_t uvs_count, const uint32_t *uv_indices, SlimTriangle *out_triangles, SlimBVHNode *out_nodes,
                  uint32_t *out_node_count, uint32_t *out_height, float out_aabb6[6]) {
    return slim::build_mesh(positions, vertex_count, position_indices, triangle_count, normals, normals_count,
                            normal_indices, uvs, uvs_count, uv_indices, out_triangles, out_nodes, out_node_count,
                            out_height, out_aabb6);
}

int slimReadMeshHeader(const char *path, SlimMesh *mesh) { return slim::read_mesh_header(path, mesh); }
int slimReadMesh(const char *path, SlimMesh *mesh) { return slim::read_mesh(path, mesh); }
int slimWriteMesh(const char *path, const SlimMesh *mesh) { return slim::write_mesh(path, mesh); }
int slimReadTextureHeader(const char *path, SlimTexture *texture, uint32_t *total_texel_quads) {
    return slim::read_texture_header(path, texture, total_texel_quads);
}
int slimReadTexture(const char *path, SlimTexture *texture, SlimTextureMip *mips, SlimTexelQuad *texel_quads) {
    return slim::read_texture(path, texture, mips, texel_quads);
}
int slimWriteTexture(const char *path, const SlimTexture *texture) { return slim::write_texture(path, texture); }
int slimSaveScene(const char *path, const SlimSceneFile *scene) { return slim::save_scene(path, scene); }
int slimReadSceneHeader(const char *path, SlimSceneFile *scene, uint32_t *texel_quad_counts) {
    return slim::read_scene_header(path, scene, texel_quad_counts);
}
int slimLoadScene(const char *path, SlimSceneFile *scene) { return slim::load_scene(path, scene); }
int slimBakeTexture(const uint8_t *bgr, uint32_t width, uint32_t height, uint32_t channels, uint32_t flags,
                    SlimTexture *texture, SlimTextureMip *mips, SlimTexelQuad *texel_quads, uint32_t *mip_count,
                    uint32_t *texel_quad_count) {
    return slim::bake_texture(bgr, width, height, channels, flags, texture, mips, texel_quads, mip_count, texel_quad_count);
}
int slimBakeTextureOnGPU(const uint8_t *bgr, uint32_t width, uint32_t height, uint32_t channels, uint32_t flags,
                         SlimTexture *texture, SlimTextureMip *mips, SlimTexelQuad *texel_quads, uint32_t *mip_count,
                         uint32_t *texel_quad_count) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (texel_quads && mips) {   // the sizing call needs no device
        int rc = ensure_device(g_ctx);
        if (rc) return rc;
    }
    return slim::bake_texture_gpu(bgr, width, height, channels, flags, texture, mips, texel_quads, mip_count,
                                  texel_quad_count, g_ctx.stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Frame rendering that allocates nothing.
//
// The ordinary entry points size the wavefront queues with cudaMalloc on
// the first frame of a size (hundreds of MiB at 1080p).  Some callers of a
// per-frame render hook cannot enter the CUDA allocator: an application
// whose other thread is capturing a CUDA graph in global capture mode (the
// runtime then refuses cudaMalloc/cudaFree from every thread), or a host
// engine that reserves the device memory up front and forbids allocation
// inside its frame loop.  slimRenderToDeviceNoAlloc gives them the
// wavefront render with its queues carved out of one file-scope device
// array of fixed size instead.
namespace slim {
namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;   // held by every GPU that loads the library
constexpr int kNoAllocMaxDevices = 64;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
unsigned char *g_noalloc_base[kNoAllocMaxDevices] = {};

// Device address of this device's copy of the array, looked up once per
// device (host code may only use the symbol through this address).  The
// calling thread's current device must be the one that holds the scene.
int noalloc_scratch(int scene_device, unsigned char **out) {
    int device = 0;
    SLIM_CUDA(cudaGetDevice(&device), "cudaGetDevice");
    if (device != scene_device)
        return set_error(SLIM_ERR_STATE, "slimRenderToDeviceNoAlloc: the current device is not the scene's device");
    if (device < 0 || device >= kNoAllocMaxDevices) return set_error(SLIM_ERR_LIMIT, "device index beyond 64");
    if (!g_noalloc_base[device]) {
        void *p = nullptr;
        SLIM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
        g_noalloc_base[device] = (unsigned char *)p;
    }
    *out = g_noalloc_base[device];
    return SLIM_OK;
}

// Carves the wavefront queues for `samples` out of the scratch: 152 bytes
// per sample of path state, ray queues, hit records and shadow masks, then
// the shadow-ray queue for as many lights per batch as fit (at least one)
// and the shadow candidate pairs in the rest.
int noalloc_layout(unsigned char *base, uint32_t samples, uint32_t lights, WavefrontBuffers &B) {
    auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
    size_t n = samples, off = 0;
    auto take = [&](size_t bytes) { unsigned char *p = base + off; off = up(off + bytes); return p; };
    B.path_color = (float4 *)take(16 * n);
    B.path_throughput = (float4 *)take(16 * n);
    B.rays[0] = (float4 *)take(32 * n);
    B.rays[1] = (float4 *)take(32 * n);
    B.hits = (float4 *)take(48 * n);
    B.shadow_mask = (unsigned long long *)take(8 * n);
    B.queue_count = (uint32_t *)take(8 * sizeof(uint32_t));
    if (off > kNoAllocScratchBytes) return set_error(SLIM_ERR_LIMIT, "frame larger than the no-alloc scratch (64 MiB)");
    size_t left = kNoAllocScratchBytes - off;
    size_t per_light = n * (32 + 48);           // one shadow ray + at least one candidate pair per sample and light
    size_t batch = per_light ? left / per_light : 0;
    if (batch < 1) return set_error(SLIM_ERR_LIMIT, "frame larger than the no-alloc scratch (64 MiB)");
    if (batch > lights) batch = lights ? lights : 1;
    size_t shadow = n * batch;
    B.shadow_rays = (float4 *)take(32 * shadow);
    size_t pairs = (kNoAllocScratchBytes - off) / 48;
    B.pairs = (float4 *)(base + off);
    if (shadow > 0xFFFFFFFFull) shadow = 0xFFFFFFFFull;
    if (pairs > 0xFFFFFFFFull) pairs = 0xFFFFFFFFull;
    B.capacity = samples;
    B.shadow_capacity = (uint32_t)shadow;
    B.pair_capacity = (uint32_t)pairs;
    return SLIM_OK;
}

}  // namespace
}  // namespace slim

static void noalloc_forget() {
    for (int i = 0; i < slim::kNoAllocMaxDevices; i++) slim::g_noalloc_base[i] = nullptr;
}

extern "C" int slimRenderToDeviceNoAlloc(const SlimCanvasData *canvas, const SlimCameraRayProjection *projection,
                                         const SlimRayTracerSettings *settings, void *d_pixels, void *d_depths,
                                         void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (!canvas || !projection || !settings || !d_pixels || !d_depths)
        return set_error(SLIM_ERR_ARGUMENT, "slimRenderToDeviceNoAlloc: null argument");
    const SlimDimensions &dim = canvas->dimensions;
    if (!dim.width || !dim.height) return set_error(SLIM_ERR_ARGUMENT, "canvas has zero size");
    if (canvas->antialias < SLIM_AA_NONE || canvas->antialias > SLIM_AA_SSAA) return set_error(SLIM_ERR_ARGUMENT, "bad antialias mode");
    int rc = check_settings(c, settings);
    if (rc) return rc;
    uint32_t s = canvas->antialias == SLIM_AA_SSAA ? 2 : 1;
    DevFrame F;
    memset(&F, 0, sizeof(F));
    F.projection = *projection;
    F.settings = *settings;
    F.width = (uint32_t)dim.width * s;
    F.height = (uint32_t)dim.height * s;
    F.rows = F.height;
    F.stride = dim.stride ? dim.stride : dim.width;
    if (F.stride < dim.width) return set_error(SLIM_ERR_ARGUMENT, "canvas stride below width");
    F.antialias = canvas->antialias;
    F.cones_per_pixel = c.options.ray_cones == SLIM_CONES_PER_PIXEL;
    F.pixels = (float4 *)d_pixels;
    F.depths = (float *)d_depths;
    F.error_flags = c.d_error.ptr;
    F.counters = nullptr;
    // The radiance cache keeps per-frame state and buffers of its own, and
    // work counting reads back device counters: neither fits a call that
    // allocates nothing, so both are refused rather than ignored.
    if (c.options.radiance_cache != SLIM_CACHE_OFF)
        return set_error(SLIM_ERR_STATE, "slimRenderToDeviceNoAlloc: the radiance cache is on");
    if (c.options.count_work)
        return set_error(SLIM_ERR_STATE, "slimRenderToDeviceNoAlloc: work counting is on");
    WavefrontBuffers B;
    memset(&B, 0, sizeof(B));
    // Debug render modes and max_depth 0 go to the fused kernel, which
    // queues nothing: no scratch, so no size limit either.
    if (settings->render_mode == SLIM_RENDER_BEAUTY && settings->max_depth != 0) {
        unsigned char *scratch = nullptr;
        if ((rc = noalloc_scratch(c.device, &scratch))) return rc;
        if ((rc = noalloc_layout(scratch, F.width * F.rows, c.scene.light_count, B))) return rc;
    }
    // The queue counters (after the per-sample arrays in the scratch) are
    // zeroed by the launcher (cudaMemsetAsync) before the first stage reads
    // them; every other region is written before it is read within the frame.
    if ((rc = wait_for_refit(c, (cudaStream_t)stream))) return rc;
    cudaError_t e = launch_render_wavefront(c.scene, F, B, c.options.block_size, (cudaStream_t)stream, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "no-alloc render launch");
    return SLIM_OK;
}

// ---- neural radiance cache --------------------------------------------------
namespace {

uint64_t splitmix64(uint64_t &state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// He-uniform weights (bound sqrt(6 / fan_in)); the output layer 10x smaller,
// so the untrained cache answers about exp(0) = 1.
void init_cache_weights(uint32_t seed, std::vector<float> &w) {
    w.assign(nrc::kParams, 0.0f);
    uint64_t state = 0x5EEDull ^ ((uint64_t)seed << 17);
    const int rows[5] = {nrc::kHidden, nrc::kHidden, nrc::kHidden, nrc::kHidden, nrc::kOutputs};
    const int cols[5] = {nrc::kInputs, nrc::kHidden, nrc::kHidden, nrc::kHidden, nrc::kHidden};
    size_t o = 0;
    for (int l = 0; l < 5; l++) {
        double bound = std::sqrt(6.0 / cols[l]) * (l == 4 ? 0.1 : 1.0);
        for (int i = 0; i < rows[l] * cols[l]; i++) {
            double u = (double)(splitmix64(state) >> 11) * (1.0 / 9007199254740992.0);
            w[o++] = (float)((2.0 * u - 1.0) * bound);
        }
    }
}

int cache_sync_errors(Context &c) {
    SLIM_CUDA(cudaDeviceSynchronize(), "radiance cache");
    return read_errors(c, nullptr);
}

int upload_cache_weights(Context &c, const float *params) {
    Context::Cache &k = c.cache;
    SLIM_CUDA(cudaDeviceSynchronize(), "wait for cache training");
    SLIM_CUDA(cudaMemcpy(k.params.ptr, params, nrc::kParams * sizeof(float), cudaMemcpyHostToDevice), "upload weights");
    SLIM_CUDA(cudaMemset(k.m.ptr, 0, nrc::kParams * sizeof(float)), "clear adam");
    SLIM_CUDA(cudaMemset(k.v.ptr, 0, nrc::kParams * sizeof(float)), "clear adam");
    SLIM_CUDA(cudaMemset(k.grad.ptr, 0, nrc::kParams * sizeof(float)), "clear gradient");
    SLIM_CUDA(cudaMemset(k.loss.ptr, 0, sizeof(float)), "clear loss");
    SLIM_CUDA(nrc::launch_pack_weights(k.params.ptr, k.image.ptr, nullptr), "pack weights");
    SLIM_CUDA(cudaMemset(k.state.ptr, 0, sizeof(uint32_t)), "clear step count");
    return cache_sync_errors(c);
}

// Validates `k`, allocates the cache's buffers, uploads `weights` and clears
// the Adam state and both counters.
int configure_cache(Context &c, const SlimRadianceCacheConfig &k, const float *weights) {
    if (k.cache_depth < 2 || k.cache_depth > 255 || !k.batch || !(k.learning_rate > 0.0f) || !(k.beta1 >= 0.0f) ||
        !(k.beta1 < 1.0f) || !(k.beta2 >= 0.0f) || !(k.beta2 < 1.0f) || !(k.epsilon > 0.0f) ||
        k.train_samples > (1u << 26) || k.train_suffix > 255)
        return set_error(SLIM_ERR_ARGUMENT, "bad radiance cache config");
    Context::Cache &st = c.cache;
    invalidate_batch();
    SLIM_CUDA(cudaDeviceSynchronize(), "wait for cache training");
    int rc;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    if ((rc = st.params.reserve(nrc::kParams, "alloc cache weights"))) return rc;
    if ((rc = st.m.reserve(nrc::kParams, "alloc adam"))) return rc;
    if ((rc = st.v.reserve(nrc::kParams, "alloc adam"))) return rc;
    if ((rc = st.grad.reserve(nrc::kParams, "alloc gradient"))) return rc;
    if ((rc = st.partials.reserve((size_t)sms * nrc::kParams, "alloc partial gradients"))) return rc;
    if ((rc = st.loss_partials.reserve((size_t)sms, "alloc partial losses"))) return rc;
    if ((rc = st.loss.reserve(1, "alloc loss"))) return rc;
    if ((rc = st.image.reserve(nrc::kImgBytes, "alloc weight image"))) return rc;
    if ((rc = st.state.reserve(2, "alloc cache counters"))) return rc;
    SLIM_CUDA(cudaMemset(st.state.ptr, 0, 2 * sizeof(uint32_t)), "clear cache counters");
    st.config = k;
    st.error_flags = c.d_error.ptr;
    SLIM_CUDA(nrc::prepare(), "radiance cache kernel attributes");
    if ((rc = upload_cache_weights(c, weights))) return rc;
    st.configured = true;
    return SLIM_OK;
}

}  // namespace

extern "C" {

int slimRadianceCacheConfigure(const SlimRadianceCacheConfig *config) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (!config) return set_error(SLIM_ERR_ARGUMENT, "config is null");
    std::vector<float> w;
    init_cache_weights(config->seed, w);
    return configure_cache(c, *config, w.data());
}

int slimRadianceCacheGetConfig(SlimRadianceCacheConfig *config) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!config) return set_error(SLIM_ERR_ARGUMENT, "config is null");
    if (!g_ctx.cache.configured) return set_error(SLIM_ERR_STATE, "radiance cache not configured");
    *config = g_ctx.cache.config;
    return SLIM_OK;
}

int slimRadianceCacheSetWeights(const float *params, uint32_t count) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.cache.configured) return set_error(SLIM_ERR_STATE, "radiance cache not configured");
    if (!params || count != (uint32_t)nrc::kParams) return set_error(SLIM_ERR_ARGUMENT, "expected SLIM_NRC_PARAMS weights");
    return upload_cache_weights(c, params);
}

int slimRadianceCacheGetWeights(float *params, uint32_t count) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.cache.configured) return set_error(SLIM_ERR_STATE, "radiance cache not configured");
    if (!params || count != (uint32_t)nrc::kParams) return set_error(SLIM_ERR_ARGUMENT, "expected SLIM_NRC_PARAMS weights");
    int rc = cache_sync_errors(c);
    if (rc) return rc;
    SLIM_CUDA(cudaMemcpy(params, c.cache.params.ptr, nrc::kParams * sizeof(float), cudaMemcpyDeviceToHost), "read weights");
    return SLIM_OK;
}

int slimRadianceCacheGetGradients(float *grad, uint32_t count) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.cache.configured) return set_error(SLIM_ERR_STATE, "radiance cache not configured");
    if (!grad || count != (uint32_t)nrc::kParams) return set_error(SLIM_ERR_ARGUMENT, "expected SLIM_NRC_PARAMS values");
    int rc = cache_sync_errors(c);
    if (rc) return rc;
    SLIM_CUDA(cudaMemcpy(grad, c.cache.grad.ptr, nrc::kParams * sizeof(float), cudaMemcpyDeviceToHost), "read gradient");
    return SLIM_OK;
}

int slimRadianceCacheSaveState(void *state, uint64_t bytes) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.cache.configured) return set_error(SLIM_ERR_STATE, "radiance cache not configured");
    if (!state || bytes < SLIM_NRC_STATE_BYTES) return set_error(SLIM_ERR_ARGUMENT, "state needs SLIM_NRC_STATE_BYTES");
    int rc = cache_sync_errors(c);
    if (rc) return rc;
    const Context::Cache &k = c.cache;
    SlimRadianceCacheStateHeader h{};
    uint32_t counters[2] = {0, 0};
    SLIM_CUDA(cudaMemcpy(counters, k.state.ptr, sizeof(counters), cudaMemcpyDeviceToHost), "read cache counters");
    h.magic = SLIM_NRC_STATE_MAGIC;
    h.params = (uint32_t)nrc::kParams;
    h.steps = counters[0];
    h.frames = counters[1];
    h.config = k.config;
    uint8_t *out = (uint8_t *)state;
    memcpy(out, &h, sizeof(h));
    float *f = (float *)(out + sizeof(h));
    const size_t n = (size_t)nrc::kParams * sizeof(float);
    SLIM_CUDA(cudaMemcpy(f, k.params.ptr, n, cudaMemcpyDeviceToHost), "read weights");
    SLIM_CUDA(cudaMemcpy(f + nrc::kParams, k.m.ptr, n, cudaMemcpyDeviceToHost), "read adam moments");
    SLIM_CUDA(cudaMemcpy(f + 2 * nrc::kParams, k.v.ptr, n, cudaMemcpyDeviceToHost), "read adam moments");
    return SLIM_OK;
}

int slimRadianceCacheLoadState(const void *state, uint64_t bytes) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called");
    if (!state || bytes < SLIM_NRC_STATE_BYTES) return set_error(SLIM_ERR_ARGUMENT, "state needs SLIM_NRC_STATE_BYTES");
    SlimRadianceCacheStateHeader h;
    memcpy(&h, state, sizeof(h));
    if (h.magic != SLIM_NRC_STATE_MAGIC || h.params != (uint32_t)nrc::kParams)
        return set_error(SLIM_ERR_ARGUMENT, "not a radiance cache state of this network");
    std::vector<float> f((size_t)3 * nrc::kParams);
    memcpy(f.data(), (const uint8_t *)state + sizeof(h), f.size() * sizeof(float));
    int rc = configure_cache(c, h.config, f.data());
    if (rc) return rc;
    const Context::Cache &k = c.cache;
    const size_t n = (size_t)nrc::kParams * sizeof(float);
    const uint32_t counters[2] = {h.steps, h.frames};
    SLIM_CUDA(cudaMemcpy(k.m.ptr, f.data() + nrc::kParams, n, cudaMemcpyHostToDevice), "restore adam moments");
    SLIM_CUDA(cudaMemcpy(k.v.ptr, f.data() + 2 * nrc::kParams, n, cudaMemcpyHostToDevice), "restore adam moments");
    SLIM_CUDA(cudaMemcpy(k.state.ptr, counters, sizeof(counters), cudaMemcpyHostToDevice), "restore cache counters");
    return cache_sync_errors(c);
}

int slimRadianceCacheQuery(const void *d_features, uint32_t count, void *d_radiance, void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.cache.configured) return set_error(SLIM_ERR_STATE, "radiance cache not configured");
    if ((!d_features || !d_radiance) && count) return set_error(SLIM_ERR_ARGUMENT, "null device buffer");
    if (c.cache.ev_trained) SLIM_CUDA(cudaStreamWaitEvent((cudaStream_t)stream, c.cache.ev_trained, 0), "join training");
    cudaError_t e = nrc::launch_infer((const float4 *)d_features, nullptr, count, count, (float4 *)d_radiance,
                                      c.cache.image.ptr, c.d_error.ptr, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "cache query launch");
    return SLIM_OK;
}

int slimRadianceCacheTrain(const void *d_features, const void *d_targets, uint32_t count, void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!c.cache.configured) return set_error(SLIM_ERR_STATE, "radiance cache not configured");
    if ((!d_features || !d_targets) && count) return set_error(SLIM_ERR_ARGUMENT, "null device buffer");
    if (!count) return SLIM_OK;
    c.cache.error_flags = c.d_error.ptr;
    cudaError_t e = c.cache.step((const float4 *)d_features, (const float4 *)d_targets, count, nullptr, 0,
                                 (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "cache train launch");
    return SLIM_OK;
}

int slimRadianceCacheJoin(void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (c.cache.ev_trained) SLIM_CUDA(cudaStreamWaitEvent((cudaStream_t)stream, c.cache.ev_trained, 0), "join training");
    return SLIM_OK;
}

int slimRadianceCacheGetStats(SlimRadianceCacheStats *stats) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    if (!stats) return set_error(SLIM_ERR_ARGUMENT, "stats is null");
    if (!c.cache.configured) return set_error(SLIM_ERR_STATE, "radiance cache not configured");
    int rc = cache_sync_errors(c);
    if (rc) return rc;
    memset(stats, 0, sizeof(*stats));
    uint32_t state[2] = {0, 0};
    SLIM_CUDA(cudaMemcpy(state, c.cache.state.ptr, sizeof(state), cudaMemcpyDeviceToHost), "read cache counters");
    stats->steps = state[0];
    stats->frames = state[1];
    SLIM_CUDA(cudaMemcpy(&stats->loss, c.cache.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost), "read loss");
    if (c.cache.counts.ptr) {
        uint32_t counts[2] = {0, 0};
        SLIM_CUDA(cudaMemcpy(counts, c.cache.counts.ptr, sizeof(counts), cudaMemcpyDeviceToHost), "read cache counts");
        stats->queries = counts[0];
        stats->train_samples = counts[1];
    }
    return SLIM_OK;
}

}  // extern "C"

// ---- batched requests -------------------------------------------------------
namespace {

struct BatchState {
    std::vector<SlimRenderRequest> requests;
    std::vector<DevScene> h_scenes;
    std::vector<DevFrame> h_frames;
    DevArray<float4> geometries, scene_nodes;
    DevArray<SlimMaterial> materials;
    DevArray<SlimLight> lights;
    DevArray<uint32_t> leaf_geometry, emissive;
    DevArray<DevScene> scenes;
    DevArray<DevFrame> frames;
    DevArray<uint4> tiles;
    std::vector<uint4> h_tiles;
    // persistent plan: the requests rendered by the persistent launch and the
    // first pixel of each in its flattened pixel queue
    DevArray<uint32_t> p_requests, p_prefix, p_cursor;
    uint32_t p_count = 0, p_total = 0;
    std::vector<BatchWave> waves;
    uint64_t pixels = 0;
    uint32_t max_lights = 0, max_instances = 0;
    bool any_cache = false;
    SlimBatchPlan plan{};
    // queues of a wave, one set per wave lane (waves alternate between the
    // launching stream and lane_stream)
    struct Queues {
        DevArray<float4> color, through, rays0, rays1, hits, shadow_rays, pairs;
        DevArray<uint32_t> counts;
        DevArray<unsigned long long> masks;
        WavefrontBuffers B{};
    } q[2];
    cudaStream_t lane_stream = nullptr;
    cudaEvent_t lane_fork = nullptr, lane_join = nullptr;
    // cache queries of a wave (the batch's own buffers, so single frames never
    // move what a captured batch graph points at)
    CacheFrame cache{};
    DevArray<float4> c_features, c_aux, c_radiance, c_targets, c_color, c_through, c_tfeatures;
    DevArray<uint32_t> c_counts;
    // captured batch
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graph_valid = false;
    size_t graph_nodes = 0;
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        graph_valid = false;
        graph_nodes = 0;
    }
};
BatchState g_batch;

}  // namespace

static void invalidate_batch() {
    g_batch.drop_graph();
    g_batch.requests.clear();
}

namespace {

constexpr uint32_t kBatchPixelBits = 23;

// Pixels of every request cut into tiles; consecutive tiles fill waves of at
// most queue_capacity slots.
int plan_waves(BatchState &b) {
    uint32_t Q = b.plan.queue_capacity, T = b.plan.tile_pixels;
    if (T > Q) T = Q;
    b.h_tiles.clear();
    b.waves.clear();
    BatchWave cur{};
    uint32_t slot = 0;
    auto close = [&]() {
        if (cur.tile_count) b.waves.push_back(cur);
        cur = BatchWave{};
        cur.first_tile = (uint32_t)b.h_tiles.size();
        slot = 0;
    };
    close();
    std::vector<uint32_t> preq, prefix;
    uint64_t ptotal = 0;
    for (uint32_t r = 0; r < b.requests.size(); r++) {
        const SlimRenderRequest &q = b.requests[r];
        const uint32_t n = q.width * q.height;
        if (b.plan.persistent && !b.h_frames[r].cache_depth) {   // the persistent launch renders it
            preq.push_back(r);
            prefix.push_back((uint32_t)ptotal);
            ptotal += n;
            continue;
        }
        for (uint32_t first = 0; first < n; first += T) {
            uint32_t count = n - first < T ? n - first : T;
            if (slot + count > Q) close();
            b.h_tiles.push_back(make_uint4(r, first, count, slot));
            cur.tile_count++;
            slot += count;
            cur.samples = slot;
            const DevFrame &f = b.h_frames[r];
            if (f.settings.max_depth > cur.max_depth) cur.max_depth = f.settings.max_depth;
            if (b.h_scenes[r].light_count > cur.max_lights) cur.max_lights = b.h_scenes[r].light_count;
            if (f.cache_depth) cur.cache_paths = 1;
        }
    }
    close();
    if (ptotal > 0xFFFFFFFFull - 4096) return set_error(SLIM_ERR_LIMIT, "persistent batch of 2^32 pixels or more");
    int rc = b.tiles.reserve(b.h_tiles.size() ? b.h_tiles.size() : 1, "alloc batch tiles");
    if (rc) return rc;
    b.p_count = (uint32_t)preq.size();
    b.p_total = (uint32_t)ptotal;
    if ((rc = b.p_requests.reserve(preq.size() ? preq.size() : 1, "alloc persistent batch table"))) return rc;
    if ((rc = b.p_prefix.reserve(prefix.size() ? prefix.size() : 1, "alloc persistent batch table"))) return rc;
    if ((rc = b.p_cursor.reserve(1, "alloc persistent batch cursor"))) return rc;
    if (!preq.empty()) {
        SLIM_CUDA(cudaMemcpy(b.p_requests.ptr, preq.data(), preq.size() * 4, cudaMemcpyHostToDevice), "upload persistent batch table");
        SLIM_CUDA(cudaMemcpy(b.p_prefix.ptr, prefix.data(), prefix.size() * 4, cudaMemcpyHostToDevice), "upload persistent batch table");
    }
    if (!b.h_tiles.empty())
        SLIM_CUDA(cudaMemcpy(b.tiles.ptr, b.h_tiles.data(), b.h_tiles.size() * sizeof(uint4), cudaMemcpyHostToDevice),
                  "upload batch tiles");
    b.plan.waves = (uint32_t)b.waves.size();
    return SLIM_OK;
}

// Queues for waves of queue_capacity paths (same sizing rule as a frame's).
int ensure_batch_queues(BatchState &b) {
    size_t Q = b.plan.queue_capacity;
    size_t lights = b.max_lights ? b.max_lights : 1;
    size_t budget = (size_t)1024 << 20;
    size_t shadow = Q * lights, max_shadow = budget / (2 * sizeof(float4));
    if (shadow > max_shadow) shadow = max_shadow < Q ? Q : max_shadow;
    size_t inst = b.max_instances ? (b.max_instances < 4 ? b.max_instances : 4) : 1;
    size_t pairs = shadow * inst, max_pairs = budget / (3 * sizeof(float4));
    if (pairs > max_pairs) pairs = max_pairs;
    int rc;
    for (BatchState::Queues &u : b.q) {
        if ((rc = u.color.reserve(Q, "alloc batch paths"))) return rc;
        if ((rc = u.through.reserve(Q, "alloc batch paths"))) return rc;
        if ((rc = u.rays0.reserve(2 * Q, "alloc batch rays"))) return rc;
        if ((rc = u.rays1.reserve(2 * Q, "alloc batch rays"))) return rc;
        if ((rc = u.hits.reserve(3 * Q, "alloc batch hits"))) return rc;
        if ((rc = u.shadow_rays.reserve(2 * shadow, "alloc batch shadow rays"))) return rc;
        if ((rc = u.pairs.reserve(3 * pairs, "alloc batch shadow pairs"))) return rc;
        if ((rc = u.counts.reserve(8, "alloc batch counters"))) return rc;
        if ((rc = u.masks.reserve(Q, "alloc batch masks"))) return rc;
        WavefrontBuffers &B = u.B;
        B.path_color = u.color.ptr;
        B.path_throughput = u.through.ptr;
        B.rays[0] = u.rays0.ptr;
        B.rays[1] = u.rays1.ptr;
        B.queue_count = u.counts.ptr;
        B.hits = u.hits.ptr;
        B.shadow_rays = u.shadow_rays.ptr;
        B.shadow_mask = u.masks.ptr;
        B.pairs = u.pairs.ptr;
        B.capacity = (uint32_t)Q;
        B.shadow_capacity = (uint32_t)shadow;
        B.pair_capacity = (uint32_t)pairs;
    }
    if (!b.lane_stream) SLIM_CUDA(cudaStreamCreateWithFlags(&b.lane_stream, cudaStreamNonBlocking), "batch lane stream");
    if (!b.lane_fork) SLIM_CUDA(cudaEventCreateWithFlags(&b.lane_fork, cudaEventDisableTiming), "batch lane event");
    if (!b.lane_join) SLIM_CUDA(cudaEventCreateWithFlags(&b.lane_join, cudaEventDisableTiming), "batch lane event");
    return SLIM_OK;
}

int batch_cache_frame(Context &c, BatchState &b) {
    if (!b.any_cache) return SLIM_OK;
    Context::Cache &k = c.cache;
    if (!k.configured) return set_error(SLIM_ERR_STATE, "a request uses the radiance cache but it is not configured");
    const uint32_t Q = b.plan.queue_capacity, cap = k.config.train_samples;
    int rc;
    if ((rc = b.c_features.reserve(4 * (size_t)Q, "alloc cache queries"))) return rc;
    if ((rc = b.c_aux.reserve(2 * (size_t)Q, "alloc cache query rays"))) return rc;
    if ((rc = b.c_radiance.reserve(Q, "alloc cache answers"))) return rc;
    if ((rc = b.c_counts.reserve(2, "alloc cache counters"))) return rc;
    if (cap) {
        if ((rc = b.c_targets.reserve(cap, "alloc training targets"))) return rc;
        if ((rc = b.c_color.reserve(cap, "alloc training paths"))) return rc;
        if ((rc = b.c_through.reserve(cap, "alloc training paths"))) return rc;
        if ((rc = b.c_tfeatures.reserve(4 * (size_t)cap, "alloc training samples"))) return rc;
    }
    CacheFrame &cf = b.cache;
    cf = CacheFrame{};
    cf.mode = SLIM_CACHE_ON;
    cf.depth = k.config.cache_depth;
    cf.features = b.c_features.ptr;
    cf.aux = b.c_aux.ptr;
    cf.radiance = b.c_radiance.ptr;
    cf.counts = b.c_counts.ptr;
    cf.train_capacity = cap;
    cf.t_features = b.c_tfeatures.ptr;
    cf.t_targets = b.c_targets.ptr;
    cf.t_color = b.c_color.ptr;
    cf.t_through = b.c_through.ptr;
    cf.frame_counter = k.state.ptr + 1;
    cf.batch = k.config.batch;
    cf.weights = k.image.ptr;
    cf.trainer = k.config.train ? &k : nullptr;
    k.error_flags = c.d_error.ptr;
    return SLIM_OK;
}

int batch_launch(Context &c, BatchState &b, cudaStream_t stream) {
    BatchFrame BF{};
    BF.shared = c.scene;
    memset(&BF.frame, 0, sizeof(BF.frame));
    BF.frame.error_flags = c.d_error.ptr;
    BF.frame.counters = c.options.count_work ? c.d_counters.ptr : nullptr;
    if (BF.frame.counters)
        SLIM_CUDA(cudaMemsetAsync(BF.frame.counters, 0, kCountersPerStage * STAGE_COUNT * sizeof(unsigned long long), stream),
                  "clear counters");
    BF.scenes = b.scenes.ptr;
    BF.frames = b.frames.ptr;
    BF.tiles = b.tiles.ptr;
    BF.waves = b.waves.data();
    BF.wave_count = (uint32_t)b.waves.size();
    BF.cache = b.any_cache ? &b.cache : nullptr;
    BF.lane_stream = b.lane_stream;
    BF.lane_queues = &b.q[1].B;
    BF.lane_fork = b.lane_fork;
    BF.lane_join = b.lane_join;
    BF.p_requests = b.p_requests.ptr;
    BF.p_prefix = b.p_prefix.ptr;
    BF.p_count = b.p_count;
    BF.p_total = b.p_total;
    BF.p_cursor = b.p_cursor.ptr;
    cudaError_t e = launch_render_batch(BF, b.q[0].B, b.plan.block_size, stream, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "batch launch");
    return SLIM_OK;
}

// (Re)plans waves and queues for the current plan.
int batch_prepare(Context &c, BatchState &b) {
    int rc;
    if ((rc = plan_waves(b))) return rc;
    if ((rc = ensure_batch_queues(b))) return rc;
    return batch_cache_frame(c, b);
}

int batch_time(Context &c, BatchState &b, cudaStream_t stream, int reps, float &ms) {
    int rc = batch_prepare(c, b);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if ((rc = batch_launch(c, b, stream))) return rc;     // warm-up
    cudaEventRecord(e0, stream);
    for (int i = 0; i < reps && !rc; i++) rc = batch_launch(c, b, stream);
    cudaEventRecord(e1, stream);
    cudaError_t e = cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= (float)(reps > 0 ? reps : 1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "batch tuning");
    return read_errors(c, stream);
}

}  // namespace

extern "C" {

int slimBatchSetRequests(const SlimRenderRequest *requests, uint32_t count) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    BatchState &b = g_batch;
    if (!c.initialized) return set_error(SLIM_ERR_STATE, "slimInitDataOnGPU has not been called (it uploads the shared assets)");
    if (!requests || !count) return set_error(SLIM_ERR_ARGUMENT, "no requests");
    if (count > (1u << (32 - kBatchPixelBits))) return set_error(SLIM_ERR_LIMIT, "more than 512 requests");
    b.drop_graph();
    b.requests.assign(requests, requests + count);
    b.h_scenes.assign(count, DevScene{});
    b.h_frames.assign(count, DevFrame{});
    b.pixels = 0;
    b.max_lights = b.max_instances = 0;
    b.any_cache = false;
    // validate and size the pools
    size_t n_geo = 0, n_mat = 0, n_light = 0, n_node = 0;
    for (uint32_t r = 0; r < count; r++) {
        const SlimRenderRequest &q = requests[r];
        const SlimSceneData *s = q.scene;
        int rc = check_scene_arrays(s);
        if (rc) return rc;
        if (!q.width || !q.height || (uint64_t)q.width * q.height > (1ull << kBatchPixelBits))
            return set_error(SLIM_ERR_LIMIT, "request canvas empty or above 2^23 pixels");
        if (!q.d_pixels || !q.d_depths) return set_error(SLIM_ERR_ARGUMENT, "request without device canvas");
        if (q.settings.render_mode != SLIM_RENDER_BEAUTY) return set_error(SLIM_ERR_ARGUMENT, "batched requests render beauty mode only");
        if (q.radiance_cache != SLIM_CACHE_OFF && q.radiance_cache != SLIM_CACHE_ON)
            return set_error(SLIM_ERR_ARGUMENT, "request radiance_cache must be OFF or ON");
        for (uint32_t g = 0; g < s->counts.geometries; g++)
            if (s->geometries[g].type == SLIM_GEOMETRY_MESH && s->geometries[g].id >= c.counts.meshes)
                return set_error(SLIM_ERR_ARGUMENT, "request geometry names a mesh the shared assets lack");
        for (uint32_t m = 0; m < s->counts.materials; m++) {
            const SlimMaterial &mat = s->materials[m];
            for (uint32_t k = 0; k < mat.texture_count && k < 2; k++)
                if (mat.texture_ids[k] >= c.counts.textures && (mat.flags & (SLIM_MATERIAL_HAS_ALBEDO_MAP | SLIM_MATERIAL_HAS_NORMAL_MAP)))
                    return set_error(SLIM_ERR_ARGUMENT, "request material names a texture the shared assets lack");
        }
        int8_t ids[3] = {q.settings.skybox_color_texture_id, q.settings.skybox_radiance_texture_id,
                         q.settings.skybox_irradiance_texture_id};
        for (int8_t id : ids)
            if (id >= 0 && (uint32_t)id >= c.counts.textures) return set_error(SLIM_ERR_ARGUMENT, "request skybox texture id out of range");
        if ((rc = check_bvh(s->bvh.nodes, s->bvh.node_count, s->counts.geometries, 0, "request scene BVH malformed"))) return rc;
        if (!s->bvh_leaf_geometry_indices) return set_error(SLIM_ERR_ARGUMENT, "request scene BVH leaf indices missing");
        if (bvh_depth(s->bvh.nodes, s->bvh.node_count) + 2 > (uint32_t)kStackCapacity)
            return set_error(SLIM_ERR_LIMIT, "request scene BVH deeper than the traversal stack");
        for (uint32_t g = 0; g < s->counts.geometries; g++)
            if (s->bvh_leaf_geometry_indices[g] >= s->counts.geometries) return set_error(SLIM_ERR_ARGUMENT, "request BVH leaf index out of range");
        n_geo += s->counts.geometries;
        n_mat += s->counts.materials;
        n_light += s->counts.lights;
        n_node += s->bvh.node_count;
    }
    int rc;
    if ((rc = b.geometries.reserve(4 * n_geo, "alloc batch geometries"))) return rc;
    if ((rc = b.materials.reserve(n_mat, "alloc batch materials"))) return rc;
    if ((rc = b.lights.reserve(n_light ? n_light : 1, "alloc batch lights"))) return rc;
    if ((rc = b.scene_nodes.reserve(2 * n_node, "alloc batch scene BVHs"))) return rc;
    if ((rc = b.leaf_geometry.reserve(n_geo, "alloc batch leaf indices"))) return rc;
    if ((rc = b.emissive.reserve(n_geo, "alloc batch emissive lists"))) return rc;
    if ((rc = b.scenes.reserve(count, "alloc batch scene table"))) return rc;
    if ((rc = b.frames.reserve(count, "alloc batch frame table"))) return rc;
    std::vector<float4> geo(4 * n_geo);
    std::vector<SlimMaterial> mat;
    std::vector<SlimLight> lig;
    std::vector<SlimBVHNode> nodes;
    std::vector<uint32_t> leaf, emis;
    mat.reserve(n_mat);
    lig.reserve(n_light);
    nodes.reserve(n_node);
    leaf.reserve(n_geo);
    emis.reserve(n_geo);
    size_t og = 0;
    const uint32_t cache_depth = c.cache.configured ? c.cache.config.cache_depth : 0;
    for (uint32_t r = 0; r < count; r++) {
        const SlimRenderRequest &q = requests[r];
        const SlimSceneData *s = q.scene;
        DevScene S = c.scene;                  // shared mesh and texture arrays
        S.geometries = b.geometries.ptr + 4 * og;
        S.materials = b.materials.ptr + mat.size();
        S.lights = b.lights.ptr + lig.size();
        S.scene_nodes = b.scene_nodes.ptr + 2 * nodes.size();
        S.leaf_geometry = b.leaf_geometry.ptr + leaf.size();
        S.emissive_quads = b.emissive.ptr + emis.size();
        S.geometry_count = s->counts.geometries;
        S.material_count = s->counts.materials;
        S.light_count = s->counts.lights;
        S.scene_node_count = s->bvh.node_count;
        S.flags = s->flags;
        uint32_t emissive = 0, instances = 0;
        for (uint32_t g = 0; g < s->counts.geometries; g++) {
            const SlimGeometry &G = s->geometries[g];
            pack_geometry(G, &geo[4 * (og + g)]);
            if (G.type == SLIM_GEOMETRY_QUAD && (s->materials[G.material_id].flags & SLIM_MATERIAL_IS_EMISSIVE)) {
                emis.push_back(g);
                emissive++;
            }
            instances += G.type == SLIM_GEOMETRY_MESH;
        }
        S.emissive_quad_count = emissive;
        og += s->counts.geometries;
        mat.insert(mat.end(), s->materials, s->materials + s->counts.materials);
        if (s->counts.lights) lig.insert(lig.end(), s->lights, s->lights + s->counts.lights);
        nodes.insert(nodes.end(), s->bvh.nodes, s->bvh.nodes + s->bvh.node_count);
        leaf.insert(leaf.end(), s->bvh_leaf_geometry_indices, s->bvh_leaf_geometry_indices + s->counts.geometries);
        b.h_scenes[r] = S;
        DevFrame F;
        memset(&F, 0, sizeof(F));
        F.projection = q.projection;
        F.settings = q.settings;
        F.width = q.width;
        F.height = q.height;
        F.rows = q.height;
        F.stride = q.width;
        F.antialias = SLIM_AA_NONE;
        F.cones_per_pixel = c.options.ray_cones == SLIM_CONES_PER_PIXEL;
        F.pixels = (float4 *)q.d_pixels;
        F.depths = (float *)q.d_depths;
        F.error_flags = c.d_error.ptr;
        F.cache_depth = (q.radiance_cache == SLIM_CACHE_ON && cache_depth && q.settings.max_depth >= cache_depth) ? cache_depth : 0;
        b.h_frames[r] = F;
        b.pixels += (uint64_t)q.width * q.height;
        if (s->counts.lights > b.max_lights) b.max_lights = s->counts.lights;
        if (instances > b.max_instances) b.max_instances = instances;
        b.any_cache |= F.cache_depth != 0;
    }
    SLIM_CUDA(cudaMemcpy(b.geometries.ptr, geo.data(), geo.size() * sizeof(float4), cudaMemcpyHostToDevice), "upload batch geometries");
    SLIM_CUDA(cudaMemcpy(b.materials.ptr, mat.data(), mat.size() * sizeof(SlimMaterial), cudaMemcpyHostToDevice), "upload batch materials");
    if (!lig.empty())
        SLIM_CUDA(cudaMemcpy(b.lights.ptr, lig.data(), lig.size() * sizeof(SlimLight), cudaMemcpyHostToDevice), "upload batch lights");
    SLIM_CUDA(cudaMemcpy(b.scene_nodes.ptr, nodes.data(), nodes.size() * sizeof(SlimBVHNode), cudaMemcpyHostToDevice), "upload batch BVHs");
    SLIM_CUDA(cudaMemcpy(b.leaf_geometry.ptr, leaf.data(), leaf.size() * 4, cudaMemcpyHostToDevice), "upload batch leaf indices");
    if (!emis.empty())
        SLIM_CUDA(cudaMemcpy(b.emissive.ptr, emis.data(), emis.size() * 4, cudaMemcpyHostToDevice), "upload batch emissive lists");
    SLIM_CUDA(cudaMemcpy(b.scenes.ptr, b.h_scenes.data(), count * sizeof(DevScene), cudaMemcpyHostToDevice), "upload batch scene table");
    SLIM_CUDA(cudaMemcpy(b.frames.ptr, b.h_frames.data(), count * sizeof(DevFrame), cudaMemcpyHostToDevice), "upload batch frame table");
    if (!b.plan.queue_capacity) {
        b.plan.queue_capacity = 4u << 20;
        b.plan.tile_pixels = 1u << 16;
        b.plan.block_size = 256;
    }
    return batch_prepare(c, b);
}

int slimBatchSetPlan(const SlimBatchPlan *plan) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!plan || plan->queue_capacity < 1024 || plan->queue_capacity > (1u << 26) || !plan->tile_pixels ||
        plan->block_size < 0 || plan->block_size > 256 || (plan->block_size % 32))
        return set_error(SLIM_ERR_ARGUMENT, "bad batch plan");
    BatchState &b = g_batch;
    b.drop_graph();
    b.plan.queue_capacity = plan->queue_capacity;
    b.plan.tile_pixels = plan->tile_pixels;
    b.plan.block_size = plan->block_size;
    b.plan.persistent = plan->persistent ? 1u : 0u;
    b.plan.tuned = 0;
    b.plan.batch_ms = 0;
    b.plan.candidates = 0;
    if (b.requests.empty()) return SLIM_OK;
    return batch_prepare(g_ctx, b);
}

int slimBatchGetPlan(SlimBatchPlan *plan) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!plan) return set_error(SLIM_ERR_ARGUMENT, "plan is null");
    *plan = g_batch.plan;
    plan->graph_nodes = (uint32_t)g_batch.graph_nodes;
    return SLIM_OK;
}

// Coordinate search: queue capacity first (the wave size sets the number of
// waves, the depth of the small late-bounce queues and the memory), then the
// block size, then the tile size that packs requests into waves.
int slimBatchTune(void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    BatchState &b = g_batch;
    if (b.requests.empty()) return set_error(SLIM_ERR_STATE, "slimBatchSetRequests has not been called");
    b.drop_graph();
    cudaStream_t s = (cudaStream_t)stream;
    SlimBatchPlan best = b.plan;
    if (!best.queue_capacity) { best.queue_capacity = 4u << 20; best.tile_pixels = 1u << 16; best.block_size = 256; }
    float best_ms = 1e30f;
    uint32_t tried = 0;
    auto attempt = [&](uint32_t Q, uint32_t T, int block, uint32_t persistent = 0) -> int {
        b.plan.queue_capacity = Q;
        b.plan.tile_pixels = T;
        b.plan.block_size = block;
        b.plan.persistent = persistent;
        float ms = 0;
        int rc = batch_time(c, b, s, 2, ms);
        if (rc) return rc;
        tried++;
        if (ms < best_ms) {
            best_ms = ms;
            best = b.plan;
        }
        return SLIM_OK;
    };
    uint64_t total = b.pixels;
    int rc;
    const SlimBatchPlan before = b.plan;
    auto fail = [&](int code) { b.plan = before; batch_prepare(c, b); return code; };
    for (uint32_t Q : {1u << 20, 2u << 20, 4u << 20, 8u << 20, 16u << 20}) {
        if (Q > 2 * total && Q != (1u << 20)) break;    // one wave already holds everything
        if ((rc = attempt(Q, best.tile_pixels, best.block_size))) return fail(rc);
    }
    for (int block : {128, 256})
        if (block != best.block_size && (rc = attempt(best.queue_capacity, best.tile_pixels, block))) return fail(rc);
    for (uint32_t T : {1u << 14, 1u << 18})
        if ((rc = attempt(best.queue_capacity, T, best.block_size))) return fail(rc);
    // the requests without the cache in one persistent launch instead of waves
    bool plain = false;
    for (const DevFrame &f : b.h_frames) plain = plain || !f.cache_depth;
    if (plain) {
        const SlimBatchPlan waves_best = best;
        if ((rc = attempt(waves_best.queue_capacity, waves_best.tile_pixels, waves_best.block_size, 1))) return fail(rc);
        for (uint32_t Q : {1u << 20, 4u << 20})   // the waves left are the cache requests' alone
            if (Q != waves_best.queue_capacity && (rc = attempt(Q, waves_best.tile_pixels, waves_best.block_size, 1)))
                return fail(rc);
    }
    b.plan = best;
    b.plan.batch_ms = best_ms;
    b.plan.candidates = tried;
    b.plan.tuned = 1;
    return batch_prepare(c, b);
}

int slimBatchRender(void *stream) {
    std::lock_guard<std::mutex> lock(g_mutex);
    Context &c = g_ctx;
    BatchState &b = g_batch;
    if (b.requests.empty()) return set_error(SLIM_ERR_STATE, "slimBatchSetRequests has not been called");
    cudaStream_t s = (cudaStream_t)stream;
    if (!b.graph_valid) {
        // a capture needs a non-default stream
        cudaStream_t cap = s;
        cudaStream_t own = nullptr;
        if (!cap) {
            SLIM_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking), "batch capture stream");
            cap = own;
        }
        SLIM_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin batch capture");
        const unsigned long long launched = g_kernel_launches.load();
        int rc = batch_launch(c, b, cap);
        g_kernel_launches.store(launched);    // recorded, not run: replays count the graph's kernels
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &graph);
        if (own) cudaStreamDestroy(own);
        if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
        if (e != cudaSuccess) return cuda_fail(e, "end batch capture");
        b.graph = graph;
        SLIM_CUDA(cudaGraphInstantiate(&b.exec, graph, 0), "instantiate batch graph");
        size_t nodes = 0;
        cudaGraphGetNodes(graph, nullptr, &nodes);
        std::vector<cudaGraphNode_t> list(nodes);
        if (nodes) cudaGraphGetNodes(graph, list.data(), &nodes);
        size_t kernels = 0;
        for (cudaGraphNode_t n : list) {
            cudaGraphNodeType type;
            if (cudaGraphNodeGetType(n, &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) kernels++;
        }
        b.graph_nodes = kernels;
        b.graph_valid = true;
    }
    SLIM_CUDA(cudaGraphLaunch(b.exec, s), "launch batch graph");
    count_launch(b.graph_nodes);
    return SLIM_OK;
}

}  // extern "C"
