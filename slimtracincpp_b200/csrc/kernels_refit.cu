// GPU refit of the scene BVH (per-frame update of instance bounds without a
// host rebuild).  The reference rebuilds the whole SAH tree on the host
// every frame (scene/scene.h:176-191); a refit keeps the uploaded topology
// and recomputes every node's bounds: leaves from their geometry's world
// AABB (Scene::updateAABB, scene/scene.h:165-174), inner nodes as the union
// of their two children (AABB::operator+, math/vec3.h:471-480).
#include "kernels.h"
#include "tracer_core.cuh"

namespace slim {
namespace dev {

SLIM_D void world_box(const DevScene &S, uint32_t gi, float mn[3], float mx[3]) {
    Geo g = load_geo(S, gi);
    float lo[3], hi[3];
    if (g.type == SLIM_GEOMETRY_MESH) {
        DevMesh m = S.meshes[g.mesh];
        for (int i = 0; i < 3; i++) { lo[i] = m.aabb_min[i]; hi[i] = m.aabb_max[i]; }
    } else {
        float e = g.type == SLIM_GEOMETRY_TET ? kTetMax : 1.0f;
        lo[0] = lo[1] = lo[2] = -e;
        hi[0] = hi[1] = hi[2] = e;
        if (g.type == SLIM_GEOMETRY_QUAD) lo[1] = hi[1] = 0.0f;
    }
    for (int i = 0; i < 3; i++) { mn[i] = INFINITY; mx[i] = -INFINITY; }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                float3 p = f3(i ? hi[0] : lo[0], j ? hi[1] : lo[1], k ? hi[2] : lo[2]);
                p = qrot(g.axis, g.w, g.s * p) + g.p;
                // minimum(min, pos) / maximum(max, pos) (math/vec3.h:403-417):
                // the running bound is the first operand, so an equal pair
                // (+0 against -0) keeps the corner's sign as the reference does
                mn[0] = mn[0] < p.x ? mn[0] : p.x; mn[1] = mn[1] < p.y ? mn[1] : p.y; mn[2] = mn[2] < p.z ? mn[2] : p.z;
                mx[0] = mx[0] > p.x ? mx[0] : p.x; mx[1] = mx[1] > p.y ? mx[1] : p.y; mx[2] = mx[2] > p.z ? mx[2] : p.z;
            }
}

SLIM_D void refit_leaf(const DevScene &S, float4 *nodes, uint32_t i) {
    float4 b = nodes[2 * i + 1];
    uint32_t count = __float_as_uint(b.w) & 0xFFFFu;
    if (!count) return;
    uint32_t first = __float_as_uint(b.z);
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t k = 0; k < count; k++) {
        float lo[3], hi[3];
        world_box(S, S.leaf_geometry[first + k], lo, hi);
        for (int a = 0; a < 3; a++) {
            mn[a] = lo[a] < mn[a] ? lo[a] : mn[a];
            mx[a] = hi[a] > mx[a] ? hi[a] : mx[a];
        }
    }
    nodes[2 * i] = make_float4(mn[0], mn[1], mn[2], mx[0]);
    nodes[2 * i + 1] = make_float4(mx[1], mx[2], b.z, b.w);
}

__global__ void k_refit_leaves(DevScene S, float4 *nodes, uint32_t node_count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < node_count) refit_leaf(S, nodes, i);
}

// Inner nodes: `order` lists them by increasing node index and every
// child pair sits after its parent (checked on upload), so walking the list
// backwards finishes both children before their parent.  The scene BVH has
// at most 2 x geometries nodes, so one thread does the whole sweep.
SLIM_D void refit_inner(float4 *nodes, const uint32_t *order, uint32_t count) {
    for (int32_t k = (int32_t)count - 1; k >= 0; k--) {
        uint32_t i = order[k];
        float4 b = nodes[2 * i + 1];
        uint32_t c = __float_as_uint(b.z);
        float4 la = nodes[2 * c], lb = nodes[2 * c + 1], ra = nodes[2 * c + 2], rb = nodes[2 * c + 3];
        float mnx = la.x < ra.x ? la.x : ra.x, mny = la.y < ra.y ? la.y : ra.y, mnz = la.z < ra.z ? la.z : ra.z;
        float mxx = la.w > ra.w ? la.w : ra.w, mxy = lb.x > rb.x ? lb.x : rb.x, mxz = lb.y > rb.y ? lb.y : rb.y;
        nodes[2 * i] = make_float4(mnx, mny, mnz, mxx);
        nodes[2 * i + 1] = make_float4(mxy, mxz, b.z, b.w);
    }
}
__global__ void k_refit_inner(float4 *nodes, const uint32_t *order, uint32_t count) {
    if (threadIdx.x == 0 && blockIdx.x == 0) refit_inner(nodes, order, count);
}

// Scenes of up to kRefitBlock nodes: both passes in one block, one launch.
constexpr uint32_t kRefitBlock = 1024;
__global__ void __launch_bounds__(kRefitBlock) k_refit_small(DevScene S, float4 *nodes, uint32_t node_count,
                                                             const uint32_t *order, uint32_t inner_count) {
    if (threadIdx.x < node_count) refit_leaf(S, nodes, threadIdx.x);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence_block();
        refit_inner(nodes, order, inner_count);
    }
}

}  // namespace dev

cudaError_t launch_refit_scene_bvh(const DevScene &S, float4 *scene_nodes, const uint32_t *order, uint32_t inner_count,
                                   cudaStream_t stream, StageTimer *timer) {
    uint32_t n = S.scene_node_count;
    if (!n) return cudaSuccess;
    if (timer) timer->begin(STAGE_REFIT, stream);
    if (n <= dev::kRefitBlock) {
        const uint32_t threads = (n + 31) / 32 * 32;
        dev::k_refit_small<<<1, threads, 0, stream>>>(S, scene_nodes, n, order, inner_count);
        count_launch();
        if (timer) timer->end(STAGE_REFIT, stream);
        return cudaGetLastError();
    }
    dev::k_refit_leaves<<<(n + 127) / 128, 128, 0, stream>>>(S, scene_nodes, n);
    count_launch();
    if (inner_count) {
        dev::k_refit_inner<<<1, 1, 0, stream>>>(scene_nodes, order, inner_count);
        count_launch();
    }
    if (timer) timer->end(STAGE_REFIT, stream);
    return cudaGetLastError();
}

}  // namespace slim
