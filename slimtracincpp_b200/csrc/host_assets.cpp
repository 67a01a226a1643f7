// Host-side algorithms of the trace path's boundary: camera projection,
// SAH BVH builds (scene and mesh), the native .mesh/.texture file formats
// and the texel-quad texture baker.  These restate the reference's own host
// code; the steps that decide bit-level output (sort order of the SAH
// quicksort, accumulation order of the prefix/suffix bounds, the triangle
// precompute) follow the reference step by step because the traversal
// order and the leaf-ordered triangle ids the GPU reports depend on them.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_set>
#include <vector>

#include "slimtracer_b200.h"
#include "host_common.h"

namespace slim {

namespace {

struct F3 { float x, y, z; };
inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
inline F3 sub(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 add(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 mul(F3 a, F3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline F3 scale(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
inline F3 cross(F3 a, F3 b) {
    return f3((a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x));
}
inline float length(F3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
inline F3 div(F3 a, float s) { float f = 1.0f / s; return scale(a, f); }
inline F3 fmin3(F3 a, F3 b) { return f3(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z); }
inline F3 fmax3(F3 a, F3 b) { return f3(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z); }
inline F3 from(const SlimVec3 &v) { return f3(v.x, v.y, v.z); }
inline SlimVec3 to(F3 v) { return SlimVec3{v.x, v.y, v.z}; }

// quat * vec3 (math/quat.h:37-43): v + 2(w (q x v) + q x (q x v)) with the
// reference's two fused steps.
inline F3 rotate(const SlimOrientation &q, F3 v) {
    F3 a = f3(q.axis.x, q.axis.y, q.axis.z);
    F3 out = cross(a, v);
    F3 qqv = cross(a, out);
    out = f3(fmaf(out.x, q.amount, qqv.x), fmaf(out.y, q.amount, qqv.y), fmaf(out.z, q.amount, qqv.z));
    return f3(fmaf(out.x, 2.0f, v.x), fmaf(out.y, 2.0f, v.y), fmaf(out.z, 2.0f, v.z));
}

struct Box { F3 mn, mx; };
inline Box merged(const Box &a, const Box &b) { return Box{fmin3(a.mn, b.mn), fmax3(a.mx, b.mx)}; }
// AABB::area (math/vec3.h:466-469): half the surface area.
inline float half_area(const Box &b) {
    F3 e = sub(b.mx, b.mn);
    return e.x * e.y + e.y * e.z + e.z * e.x;
}
inline float axis_max(const Box &b, int axis) { return axis == 0 ? b.mx.x : (axis == 1 ? b.mx.y : b.mx.z); }

// mat3::inverted (math/mat3.h:152-166) of the matrix with columns X, Y, Z,
// returned column-wise.
void inverted(F3 X, F3 Y, F3 Z, float out[9]) {
    float det = X.x * (Y.y * Z.z - Z.y * Y.z) - Y.x * (X.y * Z.z - Z.y * X.z) + Z.x * (X.y * Y.z - Y.y * X.z);
    float c[9] = {
        +(Y.y * Z.z - Z.y * Y.z), -(X.y * Z.z - Z.y * X.z), +(X.y * Y.z - Y.y * X.z),
        -(Y.x * Z.z - Z.x * Y.z), +(X.x * Z.z - Z.x * X.z), -(X.x * Y.z - Y.x * X.z),
        +(Y.x * Z.y - Z.x * Y.y), -(X.x * Z.y - Z.x * X.y), +(X.x * Y.y - Y.x * X.y)};
    float f = 1.0f / det;
    for (int i = 0; i < 9; i++) out[i] = c[i] * f;
}

// ---------------------------------------------------------------------------
// SAH builder.  One "item" per primitive (geometry or triangle) with its
// bounds; produces SlimBVHNode records with children adjacent at
// first_index / first_index + 1 and leaves indexing a leaf-ordered id list.
// Follows BVHPartition::partition / BVHBuilder::splitNode / build
// (scene/bvh_builder.h:15-263).
class SahBuilder {
public:
    explicit SahBuilder(uint32_t capacity)
        : items_(capacity), ids_(capacity), leaf_ids_(capacity), work_stack_(2 * capacity + 4) {
        for (auto &p : axes_) {
            p.sorted.resize(capacity);
            p.left_boxes.resize(capacity);
            p.right_boxes.resize(capacity);
            p.left_areas.resize(capacity);
            p.right_areas.resize(capacity);
        }
        tasks_.resize(capacity + 2);
    }

    void set_item(uint32_t i, const Box &b) { items_[i] = Item{b, i}; ids_[i] = i; }
    const std::vector<uint32_t> &leaf_ids() const { return leaf_ids_; }

    // Returns the node count; out has room for 2 * n nodes.
    uint32_t build(uint32_t n, uint32_t max_leaf, SlimBVHNode *out, uint8_t *height_out) {
        uint32_t node_count = 1;
        uint32_t height = 1;
        SlimBVHNode &root = out[0];
        root = blank_node();
        if (n <= max_leaf) {
            root.leaf_count = (uint16_t)n;
            Box b{f3(INFINITY, INFINITY, INFINITY), f3(-INFINITY, -INFINITY, -INFINITY)};
            for (uint32_t i = 0; i < n; i++) {
                leaf_ids_[i] = items_[i].first;
                b = merged(b, items_[i].box);
            }
            store_box(root, b);
            *height_out = (uint8_t)height;
            return node_count;
        }
        uint32_t middle = split(root, 0, n, out, node_count);
        Task left{0, middle, 1, 1}, right{middle, n, 2, 1};
        tasks_[0] = left;
        tasks_[1] = right;
        int32_t top = 1;
        uint32_t leaf_count = 0;
        while (top >= 0) {
            left = tasks_[top];
            SlimBVHNode &node = out[left.node_id];
            uint32_t count = left.end - left.start;
            if (count <= max_leaf) {
                node.depth = (uint8_t)left.depth;
                node.leaf_count = (uint16_t)count;
                node.first_index = leaf_count;
                for (uint32_t i = 0; i < count; i++) leaf_ids_[leaf_count + i] = items_[ids_[left.start + i]].first;
                leaf_count += count;
                top--;
            } else {
                middle = split(node, left.start, left.end, out, node_count);
                left.depth++;
                right.depth = left.depth;
                right.end = left.end;
                right.start = left.end = middle;
                left.node_id = node.first_index;
                right.node_id = node.first_index + 1;
                out[node_count - 1].depth = (uint8_t)left.depth;
                out[node_count - 2].depth = (uint8_t)right.depth;
                tasks_[top] = left;
                tasks_[++top] = right;
                if (left.depth > height) height = left.depth;
            }
        }
        out[1].depth = out[2].depth = 1;
        store_box(root, merged(load_box(out[1]), load_box(out[2])));
        *height_out = (uint8_t)height;
        return node_count;
    }

private:
    struct Item { Box box; uint32_t first; };
    struct Task { uint32_t start, end, node_id, depth; };
    struct Axis {
        std::vector<uint32_t> sorted;
        std::vector<Box> left_boxes, right_boxes;
        std::vector<float> left_areas, right_areas;
        uint32_t left_count;
        float cost;
    };

    static SlimBVHNode blank_node() {
        SlimBVHNode n;
        memset(&n, 0, sizeof(n));
        return n;
    }
    static void store_box(SlimBVHNode &n, const Box &b) { n.aabb.min = to(b.mn); n.aabb.max = to(b.mx); }
    static Box load_box(const SlimBVHNode &n) { return Box{from(n.aabb.min), from(n.aabb.max)}; }

    // Iterative quicksort by the bounds' max on one axis: Lomuto partition
    // around the last element, both halves pushed and the right one popped
    // first (scene/bvh_builder.h:22-78).  Ties keep this exact order.
    void sort_axis(Axis &a, int axis, uint32_t n) {
        int32_t top = -1;
        work_stack_[++top] = 0;
        work_stack_[++top] = (int32_t)n - 1;
        while (top >= 0) {
            int32_t end = work_stack_[top--];
            int32_t start = work_stack_[top--];
            int32_t p = start;
            float pivot = axis_max(items_[a.sorted[end]].box, axis);
            for (int32_t i = start; i < end; i++) {
                if (axis_max(items_[a.sorted[i]].box, axis) < pivot) {
                    uint32_t t = a.sorted[i];
                    a.sorted[i] = a.sorted[p];
                    a.sorted[p] = t;
                    p++;
                }
            }
            uint32_t t = a.sorted[end];
            a.sorted[end] = a.sorted[p];
            a.sorted[p] = t;
            if (p - 1 > start) { work_stack_[++top] = start; work_stack_[++top] = p - 1; }
            if (p + 1 < end) { work_stack_[++top] = p + 1; work_stack_[++top] = end; }
        }
    }

    // Prefix/suffix bounds and the SAH sweep (scene/bvh_builder.h:80-112).
    void evaluate(Axis &a, uint32_t n) {
        uint32_t li = 0, ri = n - 1;
        Box L = items_[a.sorted[li]].box, R = items_[a.sorted[ri]].box;
        a.left_boxes[li] = L;
        a.right_boxes[ri] = R;
        for (li = 0; li < n; li++, ri--) {
            if (li) {
                L = merged(L, items_[a.sorted[li]].box);
                R = merged(R, items_[a.sorted[ri]].box);
                a.left_boxes[li] = L;
                a.right_boxes[ri] = R;
            }
            a.left_areas[li] = half_area(L);
            a.right_areas[ri] = half_area(R);
        }
        uint32_t last = n - 1;
        ri = n - 1;
        a.left_count = li = 1;
        uint32_t next = 1;
        a.cost = INFINITY;
        for (uint32_t cur = 0; cur < last; cur++, next++, li++, ri--) {
            float c = a.left_areas[cur] * (float)li + a.right_areas[next] * (float)ri;
            if (a.cost > c) {
                a.cost = c;
                a.left_count = next;
            }
        }
    }

    uint32_t split(SlimBVHNode &node, uint32_t start, uint32_t end, SlimBVHNode *out, uint32_t &node_count) {
        uint32_t n = end - start;
        uint32_t *ids = ids_.data() + start;
        node.first_index = node_count;
        SlimBVHNode &left = out[node_count++];
        SlimBVHNode &right = out[node_count++];
        left = blank_node();
        right = blank_node();
        float best = INFINITY;
        int chosen = 0;
        for (int axis = 0; axis < 3; axis++) {
            Axis &a = axes_[axis];
            for (uint32_t i = 0; i < n; i++) a.sorted[i] = ids[i];
            sort_axis(a, axis, n);
            evaluate(a, n);
            if (a.cost < best) {
                best = a.cost;
                chosen = axis;
            }
        }
        Axis &c = axes_[chosen];
        store_box(left, c.left_boxes[c.left_count - 1]);
        store_box(right, c.right_boxes[c.left_count]);
        for (uint32_t i = 0; i < n; i++) ids[i] = c.sorted[i];
        return start + c.left_count;
    }

    std::vector<Item> items_;
    std::vector<uint32_t> ids_, leaf_ids_;
    std::vector<int32_t> work_stack_;
    std::vector<Task> tasks_;
    Axis axes_[3];
};

// Transform::externAABB over the 8 corners (core/transform.h:33-48).
Box extern_box(const SlimTransform &t, const Box &b) {
    F3 mn = f3(INFINITY, INFINITY, INFINITY), mx = f3(-INFINITY, -INFINITY, -INFINITY);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                F3 p = f3(i ? b.mx.x : b.mn.x, j ? b.mx.y : b.mn.y, k ? b.mx.z : b.mn.z);
                p = add(rotate(t.orientation, mul(from(t.scale), p)), from(t.position));
                mn = fmin3(mn, p);
                mx = fmax3(mx, p);
            }
    return Box{mn, mx};
}

}  // namespace

// Scene::updateAABB (scene/scene.h:165-174).
void geometry_world_box(const SlimSceneData &s, uint32_t g, float out_min[3], float out_max[3]) {
    const SlimGeometry &geo = s.geometries[g];
    Box b;
    if (geo.type == SLIM_GEOMETRY_MESH) {
        b = Box{from(s.meshes[geo.id].aabb.min), from(s.meshes[geo.id].aabb.max)};
    } else {
        float e = geo.type == SLIM_GEOMETRY_TET ? 0.577350259f : 1.0f;
        b = Box{f3(-e, -e, -e), f3(e, e, e)};
        if (geo.type == SLIM_GEOMETRY_QUAD) b.mn.y = b.mx.y = 0.0f;
    }
    b = extern_box(geo.transform, b);
    out_min[0] = b.mn.x; out_min[1] = b.mn.y; out_min[2] = b.mn.z;
    out_max[0] = b.mx.x; out_max[1] = b.mx.y; out_max[2] = b.mx.z;
}

int build_scene_bvh(SlimSceneData *s) {
    uint32_t n = s->counts.geometries;
    if (!n || !s->geometries || !s->materials || !s->bvh.nodes || !s->bvh_leaf_geometry_indices)
        return set_error(SLIM_ERR_ARGUMENT, "slimBuildSceneBVH: scene arrays missing");
    for (uint32_t g = 0; g < n; g++)
        if (s->geometries[g].type == SLIM_GEOMETRY_MESH && (!s->meshes || s->geometries[g].id >= s->counts.meshes))
            return set_error(SLIM_ERR_ARGUMENT, "slimBuildSceneBVH: geometry references a missing mesh");
    SahBuilder builder(n);
    for (uint32_t g = 0; g < n; g++) {
        Box b;
        geometry_world_box(*s, g, &b.mn.x, &b.mx.x);
        builder.set_item(g, b);
    }
    uint8_t height = 1;
    s->bvh.node_count = builder.build(n, 1, s->bvh.nodes, &height);
    s->bvh.height = height;
    for (uint32_t g = 0; g < n; g++) s->bvh_leaf_geometry_indices[g] = builder.leaf_ids()[g];
    s->flags = 0;
    for (uint32_t g = 0; g < n; g++)
        if (s->geometries[g].type == SLIM_GEOMETRY_QUAD &&
            (s->materials[s->geometries[g].material_id].flags & SLIM_MATERIAL_IS_EMISSIVE))
            s->flags = SLIM_SCENE_HAD_EMISSIVE_QUADS;
    return SLIM_OK;
}

int build_mesh(float *positions, uint32_t vertex_count, const uint32_t *pidx, uint32_t tri_count,
               const float *normals, uint32_t normals_count, const uint32_t *nidx, const float *uvs,
               uint32_t uvs_count, const uint32_t *uidx, SlimTriangle *out_tris, SlimBVHNode *out_nodes,
               uint32_t *out_node_count, uint32_t *out_height, float out_aabb6[6]) {
    if (!positions || !pidx || !tri_count || !vertex_count || !out_tris || !out_nodes || !out_node_count ||
        !out_height || !out_aabb6 || (normals_count && (!normals || !nidx)) || (uvs_count && (!uvs || !uidx)))
        return set_error(SLIM_ERR_ARGUMENT, "slimBuildMesh: missing arrays");
    for (uint64_t i = 0; i < 3ull * tri_count; i++)
        if (pidx[i] >= vertex_count || (normals_count && nidx[i] >= normals_count) || (uvs_count && uidx[i] >= uvs_count))
            return set_error(SLIM_ERR_ARGUMENT, "slimBuildMesh: index out of range");
    F3 *pos = reinterpret_cast<F3 *>(positions);
    // obj2mesh.cpp:211-226: AABB of the positions, recentred on its middle.
    F3 mn = f3(INFINITY, INFINITY, INFINITY), mx = f3(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t i = 0; i < vertex_count; i++) {
        pos[i] = scale(pos[i], 1.0f);
        mn = fmin3(mn, pos[i]);
        mx = fmax3(mx, pos[i]);
    }
    F3 centroid = div(add(mn, mx), 2.0f);
    if (centroid.x != 0.0f || centroid.y != 0.0f || centroid.z != 0.0f) {
        mn = sub(mn, centroid);
        mx = sub(mx, centroid);
        for (uint32_t i = 0; i < vertex_count; i++) pos[i] = sub(pos[i], centroid);
    }
    // BVHBuilder::buildMesh (scene/bvh_builder.h:265-341).
    const float eps = 0.0001f;
    SahBuilder builder(tri_count);
    for (uint32_t t = 0; t < tri_count; t++) {
        F3 v1 = pos[pidx[3 * t]], v2 = pos[pidx[3 * t + 1]], v3 = pos[pidx[3 * t + 2]];
        Box b{fmin3(fmin3(v1, v2), v3), fmax3(fmax3(v1, v2), v3)};
        float *bmn = &b.mn.x, *bmx = &b.mx.x;
        for (int a = 0; a < 3; a++) {
            float d = bmx[a] - bmn[a];
            if (d < 0) d = -d;
            if (d < eps) { bmn[a] -= eps; bmx[a] += eps; }
        }
        builder.set_item(t, b);
    }
    uint8_t height = 1;
    *out_node_count = builder.build(tri_count, 2, out_nodes, &height);
    *out_height = height;
    for (uint32_t i = 0; i < tri_count; i++) {
        uint32_t t = builder.leaf_ids()[i];
        F3 v1 = pos[pidx[3 * t]], v2 = pos[pidx[3 * t + 1]], v3 = pos[pidx[3 * t + 2]];
        SlimTriangle &tri = out_tris[i];
        memset(&tri, 0, sizeof(tri));
        F3 X = sub(v3, v1), Y = sub(v2, v1), Z = cross(X, Y);
        float area = length(Z);
        Z = div(Z, area);
        tri.normal = to(Z);
        tri.position = to(v1);
        inverted(X, Y, Z, tri.local_to_tangent);
        tri.uv_coverage = 1.0f;
        if (normals_count) {
            const F3 *nrm = reinterpret_cast<const F3 *>(normals);
            tri.n1 = to(nrm[nidx[3 * t]]);
            tri.n2 = to(nrm[nidx[3 * t + 1]]);
            tri.n3 = to(nrm[nidx[3 * t + 2]]);
        }
        if (uvs_count) {
            const SlimVec2 *uv = reinterpret_cast<const SlimVec2 *>(uvs);
            tri.uv1 = uv[uidx[3 * t]];
            tri.uv2 = uv[uidx[3 * t + 1]];
            tri.uv3 = uv[uidx[3 * t + 2]];
            float area_uv = (tri.uv2.x - tri.uv1.x) * (tri.uv3.y - tri.uv1.y) - (tri.uv3.x - tri.uv1.x) * (tri.uv2.y - tri.uv1.y);
            tri.uv_coverage = fabsf(area_uv / area);
        }
    }
    out_aabb6[0] = mn.x; out_aabb6[1] = mn.y; out_aabb6[2] = mn.z;
    out_aabb6[3] = mx.x; out_aabb6[4] = mx.y; out_aabb6[5] = mx.z;
    return SLIM_OK;
}

// CameraRayProjection::reset (scene/camera.h:69-83) with Dimensions::update
// (core/base.h:1312-1323).
int projection_reset(const float o[9], const float p[3], float focal_length, int width, int height,
                     int ssaa, SlimCameraRayProjection *out) {
    if (!o || !p || !out || width <= 0 || height <= 0 || width > 65535 || height > 65535)
        return set_error(SLIM_ERR_ARGUMENT, "slimProjectionReset: bad arguments");
    float f_width = (float)(uint16_t)width, f_height = (float)(uint16_t)height;
    float h_width = f_width * 0.5f, h_height = f_height * 0.5f;
    F3 X = f3(o[0], o[1], o[2]), Y = f3(o[3], o[4], o[5]), Z = f3(o[6], o[7], o[8]);
    SlimCameraRayProjection r;
    memset(&r, 0, sizeof(r));
    r.sample_size = ssaa ? 0.5f : 1.0f;
    r.squared_distance_to_projection_plane = h_height * focal_length;
    r.C_start.x = (r.sample_size * 0.5f) - h_width;
    r.C_start.y = h_height - (r.sample_size * 0.5f);
    inverted(X, Y, Z, r.inverted_camera_rotation);
    r.camera_position = SlimVec3{p[0], p[1], p[2]};
    r.down = to(scale(f3(-Y.x, -Y.y, -Y.z), r.sample_size));
    r.right = to(scale(X, r.sample_size));
    r.start = to(add(add(scale(X, r.C_start.x), scale(Y, r.C_start.y)), scale(Z, r.squared_distance_to_projection_plane)));
    r.squared_distance_to_projection_plane *= r.squared_distance_to_projection_plane;
    *out = r;
    return SLIM_OK;
}

// ---------------------------------------------------------------------------
// .mesh format (serialization/mesh.h:56-122, serialization/bvh.h:18-25):
// u32 vertex_count, triangle_count, edge_count, uvs_count, normals_count,
// bvh.node_count, 4 bytes of bvh.height; AABB min, max; Triangle[t];
// vec3 positions[v]; u32[3][t]; u32[2][e]; [vec2 uvs[u]; u32[3][t]];
// [vec3 normals[n]; u32[3][t]]; BVHNode[node_count].
namespace {
struct File {
    FILE *f;
    explicit File(const char *path, const char *mode) : f(fopen(path, mode)) {}
    ~File() { if (f) fclose(f); }
    bool read(void *p, size_t n) { return n == 0 || fread(p, 1, n, f) == n; }
    bool write(const void *p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }
};
}  // namespace

int read_mesh_header(const char *path, SlimMesh *m) {
    if (!path || !m) return set_error(SLIM_ERR_ARGUMENT, "slimReadMeshHeader: null argument");
    File file(path, "rb");
    if (!file.f) return set_error(SLIM_ERR_IO, "slimReadMeshHeader: cannot open file");
    uint32_t h[7];
    if (!file.read(h, sizeof(h))) return set_error(SLIM_ERR_IO, "slimReadMeshHeader: truncated header");
    memset(m, 0, sizeof(*m));
    m->vertex_count = h[0]; m->triangle_count = h[1]; m->edge_count = h[2];
    m->uvs_count = h[3]; m->normals_count = h[4];
    m->bvh.node_count = h[5]; m->bvh.height = (uint8_t)(h[6] & 0xFF);
    if (!m->triangle_count || !m->vertex_count || !m->bvh.node_count || m->bvh.node_count > 2 * m->triangle_count)
        return set_error(SLIM_ERR_IO, "slimReadMeshHeader: malformed counts");
    return SLIM_OK;
}

int read_mesh(const char *path, SlimMesh *m) {
    SlimMesh h;
    int rc = read_mesh_header(path, &h);
    if (rc) return rc;
    if (h.vertex_count != m->vertex_count || h.triangle_count != m->triangle_count || h.edge_count != m->edge_count ||
        h.uvs_count != m->uvs_count || h.normals_count != m->normals_count || h.bvh.node_count != m->bvh.node_count)
        return set_error(SLIM_ERR_ARGUMENT, "slimReadMesh: counts differ from the file's header");
    if (!m->triangles || !m->vertex_positions || !m->vertex_position_indices || !m->bvh.nodes ||
        (m->edge_count && !m->edge_vertex_indices) || (m->uvs_count && (!m->vertex_uvs || !m->vertex_uvs_indices)) ||
        (m->normals_count && (!m->vertex_normals || !m->vertex_normal_indices)))
        return set_error(SLIM_ERR_ARGUMENT, "slimReadMesh: destination arrays missing");
    File file(path, "rb");
    if (!file.f) return set_error(SLIM_ERR_IO, "slimReadMesh: cannot open file");
    uint32_t skip[7];
    bool ok = file.read(skip, sizeof(skip)) && file.read(&m->aabb, sizeof(SlimAABB)) &&
              file.read(m->triangles, sizeof(SlimTriangle) * (size_t)m->triangle_count) &&
              file.read(m->vertex_positions, sizeof(SlimVec3) * (size_t)m->vertex_count) &&
              file.read(m->vertex_position_indices, 12 * (size_t)m->triangle_count) &&
              file.read(m->edge_vertex_indices, 8 * (size_t)m->edge_count);
    if (ok && m->uvs_count)
        ok = file.read(m->vertex_uvs, sizeof(SlimVec2) * (size_t)m->uvs_count) &&
             file.read(m->vertex_uvs_indices, 12 * (size_t)m->triangle_count);
    if (ok && m->normals_count)
        ok = file.read(m->vertex_normals, sizeof(SlimVec3) * (size_t)m->normals_count) &&
             file.read(m->vertex_normal_indices, 12 * (size_t)m->triangle_count);
    if (ok) ok = file.read(m->bvh.nodes, sizeof(SlimBVHNode) * (size_t)m->bvh.node_count);
    if (!ok) return set_error(SLIM_ERR_IO, "slimReadMesh: truncated file");
    for (uint32_t i = 0; i < m->bvh.node_count; i++) {
        const SlimBVHNode &n = m->bvh.nodes[i];
        if (n.leaf_count ? (uint64_t)n.first_index + n.leaf_count > m->triangle_count
                         : (uint64_t)n.first_index + 1 >= m->bvh.node_count)
            return set_error(SLIM_ERR_IO, "slimReadMesh: BVH node index out of range");
    }
    return SLIM_OK;
}

int write_mesh(const char *path, const SlimMesh *m) {
    if (!path || !m || !m->triangles || !m->vertex_positions || !m->vertex_position_indices || !m->bvh.nodes ||
        (m->edge_count && !m->edge_vertex_indices))
        return set_error(SLIM_ERR_ARGUMENT, "slimWriteMesh: mesh arrays missing");
    File file(path, "wb");
    if (!file.f) return set_error(SLIM_ERR_IO, "slimWriteMesh: cannot open file");
    uint32_t h[7] = {m->vertex_count, m->triangle_count, m->edge_count, m->uvs_count, m->normals_count,
                     m->bvh.node_count, m->bvh.height};
    bool ok = file.write(h, sizeof(h)) && file.write(&m->aabb, sizeof(SlimAABB)) &&
              file.write(m->triangles, sizeof(SlimTriangle) * (size_t)m->triangle_count) &&
              file.write(m->vertex_positions, sizeof(SlimVec3) * (size_t)m->vertex_count) &&
              file.write(m->vertex_position_indices, 12 * (size_t)m->triangle_count) &&
              file.write(m->edge_vertex_indices, 8 * (size_t)m->edge_count);
    if (ok && m->uvs_count)
        ok = file.write(m->vertex_uvs, sizeof(SlimVec2) * (size_t)m->uvs_count) &&
             file.write(m->vertex_uvs_indices, 12 * (size_t)m->triangle_count);
    if (ok && m->normals_count)
        ok = file.write(m->vertex_normals, sizeof(SlimVec3) * (size_t)m->normals_count) &&
             file.write(m->vertex_normal_indices, 12 * (size_t)m->triangle_count);
    if (ok) ok = file.write(m->bvh.nodes, sizeof(SlimBVHNode) * (size_t)m->bvh.node_count);
    return ok ? SLIM_OK : set_error(SLIM_ERR_IO, "slimWriteMesh: write failed");
}

// .texture format (core/base.h:1544-1609, serialization/texture.h:55-62):
// ImageInfo (32 bytes) then per mip u32 width, u32 height and
// TexelQuad[(width + 1) * (height + 1)].
int read_texture_header(const char *path, SlimTexture *t, uint32_t *total_quads) {
    if (!path || !t || !total_quads) return set_error(SLIM_ERR_ARGUMENT, "slimReadTextureHeader: null argument");
    File file(path, "rb");
    if (!file.f) return set_error(SLIM_ERR_IO, "slimReadTextureHeader: cannot open file");
    memset(t, 0, sizeof(*t));
    if (!file.read(t, 32)) return set_error(SLIM_ERR_IO, "slimReadTextureHeader: truncated header");
    t->mips = nullptr;
    if (!t->mip_count || t->mip_count > 16) return set_error(SLIM_ERR_IO, "slimReadTextureHeader: bad mip count");
    uint64_t total = 0;
    for (uint32_t m = 0; m < t->mip_count; m++) {
        uint32_t wh[2];
        if (!file.read(wh, 8)) return set_error(SLIM_ERR_IO, "slimReadTextureHeader: truncated mip header");
        uint64_t q = (uint64_t)(wh[0] + 1ull) * (uint64_t)(wh[1] + 1ull);
        if (!wh[0] || !wh[1] || q > (1ull << 31)) return set_error(SLIM_ERR_IO, "slimReadTextureHeader: bad mip size");
        total += q;
        if (fseek(file.f, (long)(q * sizeof(SlimTexelQuad)), SEEK_CUR)) return set_error(SLIM_ERR_IO, "slimReadTextureHeader: truncated");
    }
    if (total > 0xFFFFFFFFull) return set_error(SLIM_ERR_LIMIT, "slimReadTextureHeader: too many texel quads");
    *total_quads = (uint32_t)total;
    return SLIM_OK;
}

int read_texture(const char *path, SlimTexture *t, SlimTextureMip *mips, SlimTexelQuad *quads) {
    uint32_t total = 0;
    SlimTexture h;
    int rc = read_texture_header(path, &h, &total);
    if (rc) return rc;
    if (!t || !mips || !quads) return set_error(SLIM_ERR_ARGUMENT, "slimReadTexture: null buffer");
    File file(path, "rb");
    if (!file.f) return set_error(SLIM_ERR_IO, "slimReadTexture: cannot open file");
    *t = h;
    t->mips = mips;
    file.read(t, 32);
    t->mips = mips;
    SlimTexelQuad *q = quads;
    for (uint32_t m = 0; m < t->mip_count; m++) {
        uint32_t wh[2];
        if (!file.read(wh, 8)) return set_error(SLIM_ERR_IO, "slimReadTexture: truncated");
        size_t n = (size_t)(wh[0] + 1) * (size_t)(wh[1] + 1);
        if (!file.read(q, n * sizeof(SlimTexelQuad))) return set_error(SLIM_ERR_IO, "slimReadTexture: truncated");
        mips[m].width = wh[0];
        mips[m].height = wh[1];
        mips[m].texel_quads = q;
        q += n;
    }
    return SLIM_OK;
}

int write_texture(const char *path, const SlimTexture *t) {
    if (!path || !t || !t->mips || !t->mip_count) return set_error(SLIM_ERR_ARGUMENT, "slimWriteTexture: bad texture");
    File file(path, "wb");
    if (!file.f) return set_error(SLIM_ERR_IO, "slimWriteTexture: cannot open file");
    SlimTexture h = *t;
    bool ok = file.write(&h, 32);
    for (uint32_t m = 0; ok && m < t->mip_count; m++) {
        const SlimTextureMip &mip = t->mips[m];
        ok = file.write(&mip.width, 4) && file.write(&mip.height, 4) &&
             file.write(mip.texel_quads, sizeof(SlimTexelQuad) * (size_t)(mip.width + 1) * (size_t)(mip.height + 1));
    }
    return ok ? SLIM_OK : set_error(SLIM_ERR_IO, "slimWriteTexture: write failed");
}

// ---- whole-scene files (serialization/scene.h:5-109) ------------------------
// Sections in file order: counts; mesh headers; texture ImageInfos; cameras;
// geometries; grids, boxes, curves; mesh contents; texture mips.
namespace {

constexpr size_t kCameraFileBytes = 4 * 4 + 12 + 12 + 48;   // the fields save() writes per camera

bool write_mesh_header(File &f, const SlimMesh &m) {
    uint32_t h[7] = {m.vertex_count, m.triangle_count, m.edge_count, m.uvs_count, m.normals_count, m.bvh.node_count,
                     m.bvh.height};
    return f.write(h, sizeof(h));
}

bool write_mesh_content(File &f, const SlimMesh &m) {
    bool ok = f.write(&m.aabb, sizeof(SlimAABB)) &&
              f.write(m.triangles, sizeof(SlimTriangle) * (size_t)m.triangle_count) &&
              f.write(m.vertex_positions, sizeof(SlimVec3) * (size_t)m.vertex_count) &&
              f.write(m.vertex_position_indices, 12 * (size_t)m.triangle_count) &&
              f.write(m.edge_vertex_indices, 8 * (size_t)m.edge_count);
    if (ok && m.uvs_count)
        ok = f.write(m.vertex_uvs, sizeof(SlimVec2) * (size_t)m.uvs_count) &&
             f.write(m.vertex_uvs_indices, 12 * (size_t)m.triangle_count);
    if (ok && m.normals_count)
        ok = f.write(m.vertex_normals, sizeof(SlimVec3) * (size_t)m.normals_count) &&
             f.write(m.vertex_normal_indices, 12 * (size_t)m.triangle_count);
    return ok && f.write(m.bvh.nodes, sizeof(SlimBVHNode) * (size_t)m.bvh.node_count);
}

bool read_mesh_content(File &f, SlimMesh &m) {
    bool ok = f.read(&m.aabb, sizeof(SlimAABB)) &&
              f.read(m.triangles, sizeof(SlimTriangle) * (size_t)m.triangle_count) &&
              f.read(m.vertex_positions, sizeof(SlimVec3) * (size_t)m.vertex_count) &&
              f.read(m.vertex_position_indices, 12 * (size_t)m.triangle_count) &&
              f.read(m.edge_vertex_indices, 8 * (size_t)m.edge_count);
    if (ok && m.uvs_count)
        ok = f.read(m.vertex_uvs, sizeof(SlimVec2) * (size_t)m.uvs_count) &&
             f.read(m.vertex_uvs_indices, 12 * (size_t)m.triangle_count);
    if (ok && m.normals_count)
        ok = f.read(m.vertex_normals, sizeof(SlimVec3) * (size_t)m.normals_count) &&
             f.read(m.vertex_normal_indices, 12 * (size_t)m.triangle_count);
    return ok && f.read(m.bvh.nodes, sizeof(SlimBVHNode) * (size_t)m.bvh.node_count);
}

size_t mesh_content_bytes(const SlimMesh &m) {
    size_t t = m.triangle_count;
    size_t b = sizeof(SlimAABB) + sizeof(SlimTriangle) * t + sizeof(SlimVec3) * (size_t)m.vertex_count + 12 * t +
               8 * (size_t)m.edge_count;
    if (m.uvs_count) b += sizeof(SlimVec2) * (size_t)m.uvs_count + 12 * t;
    if (m.normals_count) b += sizeof(SlimVec3) * (size_t)m.normals_count + 12 * t;
    return b + sizeof(SlimBVHNode) * (size_t)m.bvh.node_count;
}

bool write_camera(File &f, const SlimCamera &c) {
    float orientation[12];
    memcpy(orientation, c.orientation, 36);
    memcpy(orientation + 9, c.rotation, 12);
    return f.write(&c.focal_length, 4) && f.write(&c.zoom_amount, 4) && f.write(&c.dolly_amount, 4) &&
           f.write(&c.target_distance, 4) && f.write(&c.current_velocity, 12) && f.write(&c.position, 12) &&
           f.write(orientation, 48);
}

bool read_camera(File &f, SlimCamera &c) {
    float orientation[12];
    bool ok = f.read(&c.focal_length, 4) && f.read(&c.zoom_amount, 4) && f.read(&c.dolly_amount, 4) &&
              f.read(&c.target_distance, 4) && f.read(&c.current_velocity, 12) && f.read(&c.position, 12) &&
              f.read(orientation, 48);
    if (ok) {
        memcpy(c.orientation, orientation, 36);
        memcpy(c.rotation, orientation + 9, 12);
    }
    return ok;
}

bool check_counts(uint32_t n, const void *p) { return n == 0 || p != nullptr; }

// The counts a scene file's readers use, from its first 44 bytes.
bool read_counts(File &f, SlimSceneCounts &counts) {
    if (!f.read(&counts, sizeof(SlimSceneCounts))) return false;
    const uint32_t limit = 1u << 24;
    return counts.geometries < limit && counts.cameras < limit && counts.textures < 256 && counts.meshes < limit &&
           counts.grids < limit && counts.boxes < limit && counts.curves < limit;
}

bool skip(File &f, size_t bytes) { return bytes == 0 || fseek(f.f, (long)bytes, SEEK_CUR) == 0; }

}  // namespace

int save_scene(const char *path, const SlimSceneFile *sc) {
    if (!path || !sc) return set_error(SLIM_ERR_ARGUMENT, "slimSaveScene: null argument");
    const SlimSceneCounts &n = sc->counts;
    if (!check_counts(n.cameras, sc->cameras) || !check_counts(n.geometries, sc->geometries) ||
        !check_counts(n.meshes, sc->meshes) || !check_counts(n.textures, sc->textures) ||
        !check_counts(n.grids, sc->grids) || !check_counts(n.boxes, sc->boxes) || !check_counts(n.curves, sc->curves))
        return set_error(SLIM_ERR_ARGUMENT, "slimSaveScene: an array with a non-zero count is null");
    for (uint32_t i = 0; i < n.meshes; i++) {
        const SlimMesh &m = sc->meshes[i];
        if (!m.triangles || !m.vertex_positions || !m.vertex_position_indices || !m.bvh.nodes ||
            (m.edge_count && !m.edge_vertex_indices) || (m.uvs_count && (!m.vertex_uvs || !m.vertex_uvs_indices)) ||
            (m.normals_count && (!m.vertex_normals || !m.vertex_normal_indices)))
            return set_error(SLIM_ERR_ARGUMENT, "slimSaveScene: mesh arrays missing");
    }
    for (uint32_t i = 0; i < n.textures; i++)
        if (!sc->textures[i].mips || !sc->textures[i].mip_count)
            return set_error(SLIM_ERR_ARGUMENT, "slimSaveScene: texture without mips");
    File f(path, "wb");
    if (!f.f) return set_error(SLIM_ERR_IO, "slimSaveScene: cannot open file");
    bool ok = f.write(&n, sizeof(SlimSceneCounts));
    for (uint32_t i = 0; ok && i < n.meshes; i++) ok = write_mesh_header(f, sc->meshes[i]);
    for (uint32_t i = 0; ok && i < n.textures; i++) ok = f.write(&sc->textures[i], 32);
    for (uint32_t i = 0; ok && i < n.cameras; i++) ok = write_camera(f, sc->cameras[i]);
    ok = ok && f.write(sc->geometries, sizeof(SlimGeometry) * (size_t)n.geometries) &&
         f.write(sc->grids, (size_t)SLIM_GRID_BYTES * n.grids) && f.write(sc->boxes, (size_t)SLIM_BOX_BYTES * n.boxes) &&
         f.write(sc->curves, (size_t)SLIM_CURVE_BYTES * n.curves);
    for (uint32_t i = 0; ok && i < n.meshes; i++) ok = write_mesh_content(f, sc->meshes[i]);
    for (uint32_t i = 0; ok && i < n.textures; i++) {
        const SlimTexture &t = sc->textures[i];
        for (uint32_t m = 0; ok && m < t.mip_count; m++) {
            const SlimTextureMip &mip = t.mips[m];
            ok = f.write(&mip.width, 4) && f.write(&mip.height, 4) &&
                 f.write(mip.texel_quads, sizeof(SlimTexelQuad) * (size_t)(mip.width + 1) * (size_t)(mip.height + 1));
        }
    }
    return ok ? SLIM_OK : set_error(SLIM_ERR_IO, "slimSaveScene: write failed");
}

int read_scene_header(const char *path, SlimSceneFile *sc, uint32_t *texel_quad_counts) {
    if (!path || !sc) return set_error(SLIM_ERR_ARGUMENT, "slimReadSceneHeader: null argument");
    File f(path, "rb");
    if (!f.f) return set_error(SLIM_ERR_IO, "slimReadSceneHeader: cannot open file");
    if (!read_counts(f, sc->counts)) return set_error(SLIM_ERR_IO, "slimReadSceneHeader: truncated or bad counts");
    const SlimSceneCounts n = sc->counts;
    if ((n.meshes && !sc->meshes) || (n.textures && !sc->textures)) return SLIM_OK;   // counts only
    for (uint32_t i = 0; i < n.meshes; i++) {
        uint32_t h[7];
        if (!f.read(h, sizeof(h))) return set_error(SLIM_ERR_IO, "slimReadSceneHeader: truncated mesh header");
        SlimMesh &m = sc->meshes[i];
        m.vertex_count = h[0]; m.triangle_count = h[1]; m.edge_count = h[2];
        m.uvs_count = h[3]; m.normals_count = h[4];
        m.bvh.node_count = h[5]; m.bvh.height = (uint8_t)(h[6] & 0xFF);
        if (!m.triangle_count || !m.vertex_count || !m.bvh.node_count || m.bvh.node_count > 2 * m.triangle_count)
            return set_error(SLIM_ERR_IO, "slimReadSceneHeader: malformed mesh counts");
    }
    for (uint32_t i = 0; i < n.textures; i++) {
        SlimTexture &t = sc->textures[i];
        SlimTextureMip *mips = t.mips;
        if (!f.read(&t, 32)) return set_error(SLIM_ERR_IO, "slimReadSceneHeader: truncated texture header");
        t.mips = mips;
        if (!t.mip_count || t.mip_count > 16) return set_error(SLIM_ERR_IO, "slimReadSceneHeader: bad mip count");
    }
    if (!texel_quad_counts) return SLIM_OK;
    size_t fixed = kCameraFileBytes * n.cameras + sizeof(SlimGeometry) * (size_t)n.geometries +
                   (size_t)SLIM_GRID_BYTES * n.grids + (size_t)SLIM_BOX_BYTES * n.boxes + (size_t)SLIM_CURVE_BYTES * n.curves;
    for (uint32_t i = 0; i < n.meshes; i++) fixed += mesh_content_bytes(sc->meshes[i]);
    if (!skip(f, fixed)) return set_error(SLIM_ERR_IO, "slimReadSceneHeader: truncated");
    for (uint32_t i = 0; i < n.textures; i++) {
        uint64_t total = 0;
        for (uint32_t m = 0; m < sc->textures[i].mip_count; m++) {
            uint32_t wh[2];
            if (!f.read(wh, 8)) return set_error(SLIM_ERR_IO, "slimReadSceneHeader: truncated texture");
            uint64_t q = (uint64_t)(wh[0] + 1ull) * (uint64_t)(wh[1] + 1ull);
            if (!wh[0] || !wh[1] || q > (1ull << 31)) return set_error(SLIM_ERR_IO, "slimReadSceneHeader: bad mip size");
            total += q;
            if (!skip(f, q * sizeof(SlimTexelQuad))) return set_error(SLIM_ERR_IO, "slimReadSceneHeader: truncated");
        }
        if (total > 0xFFFFFFFFull) return set_error(SLIM_ERR_LIMIT, "slimReadSceneHeader: too many texel quads");
        texel_quad_counts[i] = (uint32_t)total;
    }
    return SLIM_OK;
}

int load_scene(const char *path, SlimSceneFile *sc) {
    if (!path || !sc) return set_error(SLIM_ERR_ARGUMENT, "slimLoadScene: null argument");
    File f(path, "rb");
    if (!f.f) return set_error(SLIM_ERR_IO, "slimLoadScene: cannot open file");
    SlimSceneCounts n;
    if (!read_counts(f, n)) return set_error(SLIM_ERR_IO, "slimLoadScene: truncated or bad counts");
    const SlimSceneCounts &c = sc->counts;
    if (n.geometries != c.geometries || n.cameras != c.cameras || n.textures != c.textures || n.meshes != c.meshes ||
        n.grids != c.grids || n.boxes != c.boxes || n.curves != c.curves)
        return set_error(SLIM_ERR_ARGUMENT, "slimLoadScene: counts differ from the file's");
    if (!check_counts(n.cameras, sc->cameras) || !check_counts(n.geometries, sc->geometries) ||
        !check_counts(n.meshes, sc->meshes) || !check_counts(n.textures, sc->textures) ||
        !check_counts(n.grids, sc->grids) || !check_counts(n.boxes, sc->boxes) || !check_counts(n.curves, sc->curves))
        return set_error(SLIM_ERR_ARGUMENT, "slimLoadScene: an array with a non-zero count is null");
    for (uint32_t i = 0; i < n.meshes; i++) {
        uint32_t h[7];
        if (!f.read(h, sizeof(h))) return set_error(SLIM_ERR_IO, "slimLoadScene: truncated mesh header");
        const SlimMesh &m = sc->meshes[i];
        if (h[0] != m.vertex_count || h[1] != m.triangle_count || h[2] != m.edge_count || h[3] != m.uvs_count ||
            h[4] != m.normals_count || h[5] != m.bvh.node_count)
            return set_error(SLIM_ERR_ARGUMENT, "slimLoadScene: mesh counts differ from the file's");
        if (!m.triangles || !m.vertex_positions || !m.vertex_position_indices || !m.bvh.nodes ||
            (m.edge_count && !m.edge_vertex_indices) || (m.uvs_count && (!m.vertex_uvs || !m.vertex_uvs_indices)) ||
            (m.normals_count && (!m.vertex_normals || !m.vertex_normal_indices)))
            return set_error(SLIM_ERR_ARGUMENT, "slimLoadScene: mesh arrays missing");
    }
    std::vector<SlimTexelQuad *> quads(n.textures, nullptr);
    for (uint32_t i = 0; i < n.textures; i++) {
        SlimTexture &t = sc->textures[i];
        SlimTextureMip *mips = t.mips;
        if (!mips || !mips[0].texel_quads) return set_error(SLIM_ERR_ARGUMENT, "slimLoadScene: texture buffers missing");
        quads[i] = mips[0].texel_quads;
        uint32_t mip_count = t.mip_count;
        if (!f.read(&t, 32)) return set_error(SLIM_ERR_IO, "slimLoadScene: truncated texture header");
        t.mips = mips;
        if (t.mip_count != mip_count) return set_error(SLIM_ERR_ARGUMENT, "slimLoadScene: mip count differs from the file's");
    }
    bool ok = true;
    for (uint32_t i = 0; ok && i < n.cameras; i++) ok = read_camera(f, sc->cameras[i]);
    ok = ok && f.read(sc->geometries, sizeof(SlimGeometry) * (size_t)n.geometries) &&
         f.read(sc->grids, (size_t)SLIM_GRID_BYTES * n.grids) && f.read(sc->boxes, (size_t)SLIM_BOX_BYTES * n.boxes) &&
         f.read(sc->curves, (size_t)SLIM_CURVE_BYTES * n.curves);
    for (uint32_t i = 0; ok && i < n.meshes; i++) ok = read_mesh_content(f, sc->meshes[i]);
    if (!ok) return set_error(SLIM_ERR_IO, "slimLoadScene: truncated file");
    for (uint32_t i = 0; i < n.meshes; i++) {
        const SlimMesh &m = sc->meshes[i];
        for (uint32_t k = 0; k < m.bvh.node_count; k++) {
            const SlimBVHNode &b = m.bvh.nodes[k];
            if (b.leaf_count ? (uint64_t)b.first_index + b.leaf_count > m.triangle_count
                             : (uint64_t)b.first_index + 1 >= m.bvh.node_count)
                return set_error(SLIM_ERR_IO, "slimLoadScene: BVH node index out of range");
        }
    }
    for (uint32_t i = 0; i < n.textures; i++) {
        SlimTexture &t = sc->textures[i];
        SlimTexelQuad *q = quads[i];
        for (uint32_t m = 0; m < t.mip_count; m++) {
            uint32_t wh[2];
            if (!f.read(wh, 8)) return set_error(SLIM_ERR_IO, "slimLoadScene: truncated texture");
            size_t count = (size_t)(wh[0] + 1) * (size_t)(wh[1] + 1);
            if (!f.read(q, count * sizeof(SlimTexelQuad))) return set_error(SLIM_ERR_IO, "slimLoadScene: truncated texture");
            t.mips[m].width = wh[0];
            t.mips[m].height = wh[1];
            t.mips[m].texel_quads = q;
            q += count;
        }
    }
    return SLIM_OK;
}

}  // namespace slim
