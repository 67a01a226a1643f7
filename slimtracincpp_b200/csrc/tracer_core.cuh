// Device functions of the per-pixel trace path, shared by the wavefront
// stage kernels and the fused kernel.
//
// Every floating-point expression keeps the reference's operation order:
// this translation unit is compiled with -fmad=false and fmaf() appears
// exactly where the reference writes fast_mul_add (core/base.h:94-99), so
// hit ids and distances match the reference bit for bit.  Comparisons keep
// the reference's ternary forms (Max/Min macros, core/base.h:115-116), whose
// NaN behaviour differs from fminf/fmaxf.
#pragma once
#include <cstdint>
#include "device_scene.h"

namespace slim {
namespace dev {

#define SLIM_D __device__ __forceinline__

constexpr float kEps = 0.0001f;
constexpr float kPi = 3.14159265f;
constexpr float kOneOverPi = 1.0f / 3.14159265f;
constexpr float kTetMax = 0.577350259f;
constexpr float kTetMin = 0.288675159f;
constexpr float kSqrt3 = 1.73205080757f;
constexpr float kTraceOffset = 0.0001f;
constexpr float kIorAir = 1.0003f;
constexpr float kLightRadiusIntensity = 64.0f;
constexpr float kLightIntensityRadius = 1.0f / 64.0f;
constexpr float kColorToFloat = 0.00392156862f;
constexpr float kUnitSphereAreaOverSix = (4.0f * 3.14159265f) / 6.0f;

enum : int { BoxNone = 0, BoxLeft = 1, BoxBottom = 2, BoxBack = 4, BoxRight = 8, BoxTop = 16, BoxFront = 32 };

SLIM_D float maxr(float a, float b) { return a > b ? a : b; }   // Max macro
SLIM_D float minr(float a, float b) { return a < b ? a : b; }   // Min macro
SLIM_D float clamp01(float v) { float mn = v < 1.0f ? v : 1.0f; return mn > 0.0f ? mn : 0.0f; }

// ---- vec3 (math/vec3.h) ---------------------------------------------------
SLIM_D float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
SLIM_D float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
SLIM_D float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
SLIM_D float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
SLIM_D float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
SLIM_D float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
SLIM_D float dot(float3 a, float3 b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
SLIM_D float3 cross(float3 a, float3 b) {
    return f3((a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x));
}
SLIM_D float sqlen(float3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
SLIM_D float3 divs(float3 a, float s) { float f = 1.0f / s; return a * f; }
SLIM_D float3 normalized(float3 a) { return divs(a, sqrtf(sqlen(a))); }
SLIM_D float3 scale_add(float3 a, float f, float3 b) { return f3(fmaf(a.x, f, b.x), fmaf(a.y, f, b.y), fmaf(a.z, f, b.z)); }
SLIM_D float3 mul_add(float3 a, float3 m, float3 b) { return f3(fmaf(a.x, m.x, b.x), fmaf(a.y, m.y, b.y), fmaf(a.z, m.z, b.z)); }
SLIM_D float3 one_minus(float3 a) { return f3(1.0f - a.x, 1.0f - a.y, 1.0f - a.z); }
SLIM_D float3 reflected(float3 d, float3 n) { return scale_add(n, -2.0f * dot(d, n), d); }
SLIM_D float3 ld3(const float *p) { return f3(__ldg(p), __ldg(p + 1), __ldg(p + 2)); }
SLIM_D float3 xyz(float4 v) { return f3(v.x, v.y, v.z); }

// quat * vec3 (math/quat.h:37-43)
SLIM_D float3 qrot(float3 axis, float w, float3 v) {
    float3 out = cross(axis, v);
    float3 qqv = cross(axis, out);
    out = scale_add(out, w, qqv);
    return scale_add(out, 2.0f, v);
}

// ---- rays and hits (core/ray.h) ------------------------------------------
struct Ray {
    float3 o, so, d, rcp;
    bool nx, ny, nz;        // sign bit of each direction component (octant shift 3)
};
struct Hit {
    float3 position, normal;
    float u, v;
    float distance, uv_coverage, NdotRd;
    uint32_t id;
    bool from_behind;
};

SLIM_D float3 at(const Ray &r, float t) { return scale_add(r.d, t, r.o); }
SLIM_D void reset(Ray &r, float3 o, float3 d) {                                    // ray.h:40-49
    r.o = o;
    r.d = d;
    r.rcp = f3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    r.so = (-o) * r.rcp;
    r.nx = signbit(d.x);
    r.ny = signbit(d.y);
    r.nz = signbit(d.z);
}

struct Geo {
    float3 axis; float w;           // rotation
    float3 p; int type;
    float3 s; uint32_t material;
    float3 inv_s; uint32_t flags;   // low 8 bits: geometry flags
    uint32_t mesh;
};
SLIM_D Geo load_geo(const DevScene &S, uint32_t g) {
    const float4 *r = S.geometries + 4 * (size_t)g;
    float4 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2), d = __ldg(r + 3);
    Geo o;
    o.axis = xyz(a); o.w = a.w;
    o.p = xyz(b); o.type = __float_as_int(b.w);
    o.s = xyz(c); o.material = __float_as_uint(c.w);
    o.inv_s = xyz(d);
    uint32_t bits = __float_as_uint(d.w);
    o.flags = bits & 0xFFu;
    o.mesh = bits >> 8;
    return o;
}
// Ray::localize (ray.h:29-34); inv_s is 1.0f / scale computed on upload.
SLIM_D void localize(Ray &out, float3 o, float3 d, const Geo &g) {
    float3 ia = -g.axis;
    reset(out, g.inv_s * qrot(ia, g.w, o - g.p), g.inv_s * qrot(ia, g.w, d));
}

// Ray::hitsAABB (ray.h:51-59): octant-selected slab test.
SLIM_D bool hit_aabb(const Ray &r, float mnx, float mny, float mnz, float mxx, float mxy, float mxz,
                     float &nearD, float &farD) {
    float lo_x = r.nx ? mxx : mnx, hi_x = r.nx ? mnx : mxx;
    float lo_y = r.ny ? mxy : mny, hi_y = r.ny ? mny : mxy;
    float lo_z = r.nz ? mxz : mnz, hi_z = r.nz ? mnz : mxz;
    float t0x = fmaf(lo_x, r.rcp.x, r.so.x), t0y = fmaf(lo_y, r.rcp.y, r.so.y), t0z = fmaf(lo_z, r.rcp.z, r.so.z);
    float t1x = fmaf(hi_x, r.rcp.x, r.so.x), t1y = fmaf(hi_y, r.rcp.y, r.so.y), t1z = fmaf(hi_z, r.rcp.z, r.so.z);
    float m = maxr(t0x, maxr(t0y, t0z));
    nearD = 0 > m ? 0.0f : m;
    farD = minr(t1x, minr(t1y, t1z));
    return nearD <= farD;
}
SLIM_D bool hit_node(const Ray &r, float4 a, float4 b, float &nearD, float &farD) {
    return hit_aabb(r, a.x, a.y, a.z, a.w, b.x, b.y, nearD, farD);
}

// Ray::hitsPlane (ray.h:61-82)
SLIM_D bool hit_plane(const Ray &r, float3 p, float3 n, float &t, float3 &pos, bool &from_behind) {
    float NdotRd = dot(n, r.d);
    if (NdotRd == 0) return false;
    float NdotRoP = dot(n, p - r.o);
    if (NdotRoP == 0) return false;
    bool facing = NdotRd < 0;
    from_behind = NdotRoP > 0;
    if (from_behind == facing) return false;
    t = NdotRoP / NdotRd;
    pos = at(r, t);
    return true;
}

SLIM_D bool checker(float u, float v) {                                             // base.h:277-279
    return (((int)(v * 4.0f)) & 1) == (((int)(u * 4.0f)) & 1);
}

// Ray::hitsDefaultQuad (ray.h:84-120)
SLIM_D bool hit_quad(const Ray &r, Hit &h, bool transparent) {
    if (r.d.y == 0) return false;
    if (r.o.y == 0) return false;
    h.from_behind = r.o.y < 0;
    if (h.from_behind == (r.d.y < 0)) return false;
    float t = fabsf(r.o.y * r.rcp.y);
    if (t > h.distance) return false;
    h.position = at(r, t);
    if (h.position.x < -1 || h.position.x > 1 || h.position.z < -1 || h.position.z > 1) return false;
    h.u = fmaf(h.position.x, 0.5f, 0.5f);
    h.v = fmaf(h.position.z, 0.5f, 0.5f);
    if (transparent && checker(h.u, h.v)) return false;
    h.distance = t;
    h.normal = f3(0.0f, 1.0f, 0.0f);
    h.uv_coverage = 0.25f;
    return true;
}

SLIM_D int octant_side(bool sx, bool sy, bool sz, int axis) {                      // base.h:532-538
    return (axis == 1) * (1 << (sx ? 3 : 0)) | (axis == 2) * (2 << (sy ? 3 : 0)) | (axis == 4) * (4 << (sz ? 3 : 0));
}
SLIM_D void uv_by_box_side(int side, float3 p, float &u, float &v) {               // base.h:424-454
    float a, b;
    switch (side) {
        case BoxTop: a = p.x; b = p.z; break;
        case BoxBottom: a = -p.x; b = -p.z; break;
        case BoxLeft: a = -p.z; b = p.y; break;
        case BoxRight: a = p.z; b = p.y; break;
        case BoxFront: a = p.x; b = p.y; break;
        default: a = -p.x; b = p.y; break;
    }
    u = fmaf(a, 0.5f, 0.5f);
    v = fmaf(b, 0.5f, 0.5f);
}
// Ray::hitsDefaultBox (ray.h:122-175)
SLIM_D bool hit_box(const Ray &r, Hit &h, bool transparent) {
    float3 sr = f3(1.0f - 2.0f * (float)r.nx, 1.0f - 2.0f * (float)r.ny, 1.0f - 2.0f * (float)r.nz) * r.rcp;
    float3 nt = r.so - sr, ft = r.so + sr;
    int near_axis = 1, far_axis = 1;
    float far_t = ft.x;
    if (ft.y < far_t) { far_t = ft.y; far_axis = 2; }
    if (ft.z < far_t) { far_t = ft.z; far_axis = 4; }
    if (far_t < 0) return false;
    float near_t = nt.x;
    if (nt.y > near_t) { near_t = nt.y; near_axis = 2; }
    if (nt.z > near_t) { near_t = nt.z; near_axis = 4; }
    if (near_t > h.distance || far_t < (near_t > 0 ? near_t : 0)) return false;
    float t = near_t;
    int side;
    h.from_behind = near_t < 0;
    if (h.from_behind) {
        if (far_t > h.distance) return false;
        t = far_t;
        side = octant_side(!r.nx, !r.ny, !r.nz, far_axis);
    } else
        side = octant_side(r.nx, r.ny, r.nz, near_axis);
    h.position = at(r, t);
    uv_by_box_side(side, h.position, h.u, h.v);
    if (transparent && checker(h.u, h.v)) {
        if (h.from_behind || far_t > h.distance) return false;
        side = octant_side(!r.nx, !r.ny, !r.nz, far_axis);
        h.from_behind = true;
        t = far_t;
        h.position = at(r, t);
        uv_by_box_side(side, h.position, h.u, h.v);
        if (checker(h.u, h.v)) return false;
    }
    h.distance = t;
    h.normal = f3((float)((int)(side == BoxRight) - (int)(side == BoxLeft)),
                  (float)((int)(side == BoxTop) - (int)(side == BoxBottom)),
                  (float)((int)(side == BoxFront) - (int)(side == BoxBack)));
    h.uv_coverage = 0.25f;
    return true;
}

SLIM_D void uv_by_sphere(float3 p, float &u, float &v) {                           // base.h:456-483
    float X = p.x, Y = p.y, Z = p.z, a, b;
    float zx = X ? (Z / X) : 2, yx = X ? (Y / X) : 2;
    if (zx <= 1 && zx >= -1 && yx <= 1 && yx >= -1) {
        a = zx;
        b = X > 0 ? yx : -yx;
    } else {
        float xz = Z ? (X / Z) : 2, yz = Z ? (Y / Z) : 2;
        if (xz <= 1 && xz >= -1 && yz <= 1 && yz >= -1) {
            a = -xz;
            b = Z > 0 ? yz : -yz;
        } else {
            a = X / (Y > 0 ? Y : -Y);
            b = Z / Y;
        }
    }
    u = fmaf(a, 0.5f, 0.5f);
    v = fmaf(b, 0.5f, 0.5f);
}
// Ray::hitsDefaultSphere (ray.h:177-215)
SLIM_D bool hit_sphere(const Ray &r, Hit &h, bool transparent, float *out_sq) {
    float tc = -(dot(r.o, r.d));
    if (tc <= 0) return false;
    float dsl = sqlen(r.d);
    float sq = sqlen(r.o) * dsl - tc * tc;
    if (sq > 1.0f) return false;
    float delta = sqrtf(dsl - sq);
    dsl = 1.0f / dsl;
    float t = (tc - delta) * dsl;
    if (t > h.distance) return false;
    h.normal = at(r, t);
    uv_by_sphere(h.normal, h.u, h.v);
    h.from_behind = t <= 0 || (transparent && checker(h.u, h.v));
    if (h.from_behind) {
        t = (tc + delta) * dsl;
        if (t <= 0 || t > h.distance) return false;
        h.normal = at(r, t);
        uv_by_sphere(h.normal, h.u, h.v);
        if (transparent && checker(h.u, h.v)) return false;
    }
    h.distance = t;
    h.uv_coverage = 1.0f / kUnitSphereAreaOverSix;
    if (out_sq) *out_sq = sq * dsl;
    return true;
}

// Ray::hitsDefaultTetrahedron (ray.h:217-311); rows: the two columns' x and
// y of each face's tangent matrix that the (u, v) test reads.
SLIM_D bool hit_tet(const Ray &r, Hit &h, bool transparent) {
    bool found = false;
    for (int f = 0; f < 4; f++) {
        float c = f == 3 ? kTetMax : -kTetMax;
        float3 tp = f3(c, c, c), fn = f3(c, c, c);
        if (f == 0) fn.y = kTetMax; else if (f == 1) fn.x = kTetMax; else if (f == 2) fn.z = kTetMax; else tp.y = -kTetMax;
        float t; float3 pos; bool behind;
        if (!hit_plane(r, tp, fn, t, pos, behind)) continue;
        float m[9];
        switch (f) {
            case 0: { float k[9] = {kTetMax, -kTetMin, -kTetMax, kTetMin, kTetMin, kTetMax, -kTetMin, kTetMax, -kTetMax};
                      for (int i = 0; i < 9; i++) m[i] = k[i]; } break;
            case 1: { float k[9] = {kTetMin, kTetMin, kTetMax, -kTetMin, kTetMax, -kTetMax, kTetMax, -kTetMin, -kTetMax};
                      for (int i = 0; i < 9; i++) m[i] = k[i]; } break;
            case 2: { float k[9] = {-kTetMin, kTetMax, -kTetMax, kTetMax, -kTetMin, -kTetMax, kTetMin, kTetMin, kTetMax};
                      for (int i = 0; i < 9; i++) m[i] = k[i]; } break;
            default: { float k[9] = {-kTetMax, kTetMin, kTetMax, kTetMin, kTetMin, kTetMax, kTetMin, -kTetMax, kTetMax};
                       for (int i = 0; i < 9; i++) m[i] = k[i]; } break;
        }
        float3 q = pos - tp;
        float tx = m[0] * q.x + m[3] * q.y + m[6] * q.z;
        float ty = m[1] * q.x + m[4] * q.y + m[7] * q.z;
        if (tx < 0 || ty < 0 || ty + tx > 1) continue;
        if (transparent && checker(tx, ty)) continue;
        if (t < h.distance) {
            h.distance = t;
            h.position = pos;
            h.normal = fn;
            h.from_behind = behind;
            h.u = tx;
            h.v = ty;
            h.uv_coverage = kSqrt3 / 4.0f;
            found = true;
        }
    }
    return found;
}

// ---- work counters (optional) --------------------------------------------
struct Work {
    uint32_t primary, shadow, bounce, scene_nodes, mesh_nodes, triangles, geometries, mesh_fetches, taps;
    // the parts of scene_nodes, mesh_nodes, triangles, geometries spent in
    // any-hit traversals (counted by the fused engine only)
    uint32_t any_scene_nodes, any_mesh_nodes, any_triangles, any_geometries;
};
template <bool COUNT> SLIM_D void bump(uint32_t &c, uint32_t n = 1) { if (COUNT) c += n; }

// ---- mesh BVH (scene/mesh_tracer.h) ----------------------------------------
SLIM_D void load_node(const float4 *nodes, uint32_t i, float4 &a, float4 &b) {
    a = __ldg(nodes + 2 * (size_t)i);
    b = __ldg(nodes + 2 * (size_t)i + 1);
}
SLIM_D uint32_t node_first(float4 b) { return __float_as_uint(b.z); }
SLIM_D uint32_t node_leaf_count(float4 b) { return __float_as_uint(b.w) & 0xFFFFu; }

// MeshTracer::hitTriangles (mesh_tracer.h:23-49) over triangles [first, first+count).
template <bool COUNT>
SLIM_D bool hit_triangles(const float4 *hot, uint32_t first, uint32_t count, float closest, const Ray &r,
                          Hit &h, bool any_hit, Work &w) {
    bool found = false;
    closest = minr(closest, h.distance);
    for (uint32_t i = 0; i < count; i++) {
        bump<COUNT>(w.triangles);
        const float4 *t = hot + 3 * (size_t)(first + i);
        float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
        float3 p = xyz(a), n = f3(a.w, b.x, b.y);
        float tt; float3 pos; bool behind;
        if (hit_plane(r, p, n, tt, pos, behind)) {
            float3 q = pos - p;
            // local_to_tangent * q: x = m0 q.x + m3 q.y + m6 q.z, y = m1 q.x + m4 q.y + m7 q.z
            float ux = b.z * q.x + c.x * q.y + c.z * q.z;
            float uy = b.w * q.x + c.y * q.y + c.w * q.z;
            if (ux < 0 || uy < 0 || (ux + uy) > 1 || tt >= closest) continue;
            closest = tt;
            h.distance = tt;
            h.position = pos;
            h.normal = n;
            h.from_behind = behind;
            h.u = ux;
            h.v = uy;
            h.id = i;
            found = true;
            if (any_hit) break;
        }
    }
    return found;
}

// The attributes MeshTracer::trace fills in for a closest hit (mesh_tracer.h:
// 116-133): the triangle's uv coverage and, with vertex normals / uvs, their
// barycentric blend.  h.id is the triangle's leaf-order index in the mesh.
template <bool COUNT>
SLIM_D void mesh_hit_attributes(const DevScene &S, const DevMesh &m, Hit &h, Work &w) {
    const float4 *c = S.tri_cold + 4 * (size_t)(m.tri_offset + h.id);
    float4 c3 = __ldg(c + 3);
    h.uv_coverage = c3.w;
    if (m.has_normals | m.has_uvs) {
        bump<COUNT>(w.mesh_fetches);
        float4 c0 = __ldg(c), c1 = __ldg(c + 1), c2 = __ldg(c + 2);
        float A = h.u, B = h.v, C = 1 - A - B;
        if (m.has_uvs) {
            // uv1 = (c2.y, c2.z), uv2 = (c2.w, c3.x), uv3 = (c3.y, c3.z)
            h.u = fmaf(c3.y, A, fmaf(c2.w, B, c2.y * C));
            h.v = fmaf(c3.z, A, fmaf(c3.x, B, c2.z * C));
        }
        if (m.has_normals) {
            // n1 = (c0.x, c0.y, c0.z), n2 = (c0.w, c1.x, c1.y), n3 = (c1.z, c1.w, c2.x)
            h.normal.x = fmaf(c1.z, A, fmaf(c0.w, B, c0.x * C));
            h.normal.y = fmaf(c1.w, A, fmaf(c1.x, B, c0.y * C));
            h.normal.z = fmaf(c2.x, A, fmaf(c1.y, B, c0.z * C));
        }
    }
}

// MeshTracer::trace (mesh_tracer.h:51-134).  `stack` holds kStackCapacity
// entries; overflow sets kErrStack and ends the traversal.
template <bool COUNT>
SLIM_D bool mesh_trace(const DevScene &S, const DevMesh &m, const Ray &r, Hit &h, bool any_hit,
                       uint32_t *stack, uint32_t &err, Work &w) {
    const float4 *nodes = S.mesh_nodes + 2 * (size_t)m.node_offset;
    const float4 *hot = S.tri_hot;
    float ln, rn, lf, rf;
    float4 a, b;
    load_node(nodes, 0, a, b);
    bump<COUNT>(w.mesh_nodes);
    if (!(hit_node(r, a, b, ln, lf) && ln < h.distance)) return false;
    if (node_leaf_count(b)) {
        bool f = hit_triangles<COUNT>(hot, m.tri_offset, m.tri_count, lf, r, h, any_hit, w);
        if (f) h.uv_coverage = __ldg(&S.tri_cold[4 * (size_t)(m.tri_offset + h.id) + 3].w);
        return f;
    }
    bool found = false;
    uint32_t left = node_first(b);
    uint32_t top = 0;
    for (;;) {
        float4 la, lb, ra, rb;
        load_node(nodes, left, la, lb);
        load_node(nodes, left + 1, ra, rb);
        bump<COUNT>(w.mesh_nodes, 2);
        bool hl = hit_node(r, la, lb, ln, lf) && ln < h.distance;
        bool hr = hit_node(r, ra, rb, rn, rf) && rn < h.distance;
        uint32_t lchild = node_first(lb), rchild = node_first(rb);
        bool go_left = hl, go_right = hr;
        if (hl) {
            uint32_t cnt = node_leaf_count(lb);
            if (cnt) {
                if (hit_triangles<COUNT>(hot, m.tri_offset + lchild, cnt, lf, r, h, any_hit, w)) {
                    h.id += lchild;
                    found = true;
                    if (any_hit) break;
                }
                go_left = false;
            }
        }
        if (hr) {
            uint32_t cnt = node_leaf_count(rb);
            if (cnt) {
                if (hit_triangles<COUNT>(hot, m.tri_offset + rchild, cnt, rf, r, h, any_hit, w)) {
                    h.id += rchild;
                    found = true;
                    if (any_hit) break;
                }
                go_right = false;
            }
        }
        if (go_left) {
            if (go_right) {
                if (!any_hit && ln > rn) { uint32_t t = lchild; lchild = rchild; rchild = t; }
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
    if (found && !any_hit) {
        mesh_hit_attributes<COUNT>(S, m, h, w);
    } else if (found) {
        h.uv_coverage = __ldg(&S.tri_cold[4 * (size_t)(m.tri_offset + h.id) + 3].w);
    }
    return found;
}

// SceneTracer::hitGeometryInLocalSpace (scene_tracer.h:138-165)
template <bool COUNT>
SLIM_D bool hit_geometry_local(const DevScene &S, const Geo &g, const Ray &r, Ray &local, Hit &h,
                               bool any_hit, uint32_t *mesh_stack, uint32_t &err, Work &w) {
    bump<COUNT>(w.geometries);
    localize(local, r.o, r.d, g);
    float mn[3], mx[3], n, f;
    DevMesh mesh;
    if (g.type == SLIM_GEOMETRY_MESH) {
        mesh = S.meshes[g.mesh];
        for (int i = 0; i < 3; i++) { mn[i] = mesh.aabb_min[i]; mx[i] = mesh.aabb_max[i]; }
    } else {
        float e = g.type == SLIM_GEOMETRY_TET ? kTetMax : 1.0f;
        mx[0] = mx[1] = mx[2] = e;
        mn[0] = mn[1] = mn[2] = -e;
        if (g.type == SLIM_GEOMETRY_QUAD) { mn[1] = -kEps; mx[1] = kEps; }
    }
    if (!hit_aabb(local, mn[0], mn[1], mn[2], mx[0], mx[1], mx[2], n, f)) return false;
    bool transparent = (g.flags & SLIM_GEOMETRY_IS_TRANSPARENT) != 0;
    switch (g.type) {
        case SLIM_GEOMETRY_QUAD: return hit_quad(local, h, transparent);
        case SLIM_GEOMETRY_BOX: return hit_box(local, h, transparent);
        case SLIM_GEOMETRY_SPHERE: return hit_sphere(local, h, transparent, nullptr);
        case SLIM_GEOMETRY_TET: return hit_tet(local, h, transparent);
        case SLIM_GEOMETRY_MESH: return mesh_trace<COUNT>(S, mesh, local, h, any_hit, mesh_stack, err, w);
        default: return false;
    }
}

// SceneTracer::hitGeometries (scene_tracer.h:111-136).  Returns the hit
// geometry index or -1; the closest hit lands in `hit` with NdotRd set.
template <bool COUNT>
SLIM_D int hit_geometries(const DevScene &S, uint32_t first, uint32_t count, float closest, const Ray &r,
                          Hit &hit, bool any_hit, uint32_t *mesh_stack, uint32_t &err, Work &w) {
    int hit_geo = -1;
    uint32_t vis = any_hit ? SLIM_GEOMETRY_IS_SHADOWING : SLIM_GEOMETRY_IS_VISIBLE;
    Hit aux;
    float cd = closest + kEps;
    aux.distance = minr(cd, hit.distance);
    Ray local;
    for (uint32_t i = 0; i < count; i++) {
        uint32_t gi = __ldg(S.leaf_geometry + first + i);
        Geo g = load_geo(S, gi);
        if (!(g.flags & vis)) continue;
        if (hit_geometry_local<COUNT>(S, g, r, local, aux, any_hit, mesh_stack, err, w)) {
            if (any_hit) return (int)gi;
            if (aux.distance < hit.distance) {
                hit_geo = (int)gi;
                hit = aux;
                hit.NdotRd = -(dot(hit.normal, local.d));
            }
        }
    }
    return hit_geo;
}

// SceneTracer::trace (scene_tracer.h:26-98): offsets the origin by
// TRACE_OFFSET along the direction, then walks the scene BVH near child
// first (both children tested per step, the far one pushed).
template <bool COUNT>
SLIM_D int scene_trace(const DevScene &S, Ray &r, Hit &hit, bool any_hit, float max_distance,
                       uint32_t *stack, uint32_t *mesh_stack, uint32_t &err, Work &w) {
    reset(r, scale_add(r.d, kTraceOffset, r.o), r.d);
    hit.distance = max_distance;
    float ln, rn, lf, rf;
    float4 a, b;
    load_node(S.scene_nodes, 0, a, b);
    bump<COUNT>(w.scene_nodes);
    if (!(hit_node(r, a, b, ln, lf) && ln < hit.distance)) return -1;
    if (node_leaf_count(b)) return hit_geometries<COUNT>(S, 0, S.geometry_count, lf, r, hit, any_hit, mesh_stack, err, w);
    int closest_geo = -1;
    uint32_t left = node_first(b);
    uint32_t top = 0;
    for (;;) {
        float4 la, lb, ra, rb;
        load_node(S.scene_nodes, left, la, lb);
        load_node(S.scene_nodes, left + 1, ra, rb);
        bump<COUNT>(w.scene_nodes, 2);
        bool hl = hit_node(r, la, lb, ln, lf) && ln < hit.distance;
        bool hr = hit_node(r, ra, rb, rn, rf) && rn < hit.distance;
        uint32_t lchild = node_first(lb), rchild = node_first(rb);
        bool go_left = hl, go_right = hr;
        if (hl) {
            uint32_t cnt = node_leaf_count(lb);
            if (cnt) {
                int g = hit_geometries<COUNT>(S, lchild, cnt, lf, r, hit, any_hit, mesh_stack, err, w);
                if (g >= 0) { closest_geo = g; if (any_hit) break; }
                go_left = false;
            }
        }
        if (hr) {
            uint32_t cnt = node_leaf_count(rb);
            if (cnt) {
                int g = hit_geometries<COUNT>(S, rchild, cnt, rf, r, hit, any_hit, mesh_stack, err, w);
                if (g >= 0) { closest_geo = g; if (any_hit) break; }
                go_right = false;
            }
        }
        if (go_left) {
            if (go_right) {
                if (!any_hit && ln > rn) { uint32_t t = lchild; lchild = rchild; rchild = t; }
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
    return closest_geo;
}

// ---- textures (core/texture.h) -------------------------------------------
template <bool COUNT>
SLIM_D float3 mip_sample(const DevScene &S, const DevMip &m, float u, float v, Work &w) {    // texture.h:17-41
    bump<COUNT>(w.taps);
    if (u > 1) u -= (float)((uint32_t)u);
    if (v > 1) v -= (float)((uint32_t)v);
    const float U = u * (float)m.width + 0.5f;
    const float V = v * (float)m.height + 0.5f;
    uint32_t x = (uint32_t)U, y = (uint32_t)V;
    const float r = U - (float)x, b = V - (float)y;
    const float l = 1 - r, t = 1 - b;
    const float tl = t * l * kColorToFloat, tr = t * r * kColorToFloat;
    const float bl = b * l * kColorToFloat, br = b * r * kColorToFloat;
    // Out-of-range coordinates (negative or non-finite uv) read the border
    // quad instead of memory outside the mip.
    x = x > m.width ? m.width : x;
    y = y > m.height ? m.height : y;
    uint4 q = __ldg(S.quads + m.quad_offset + (size_t)y * (m.width + 1) + x);
#define SLIM_TAP(word, k) ((float)(((word) >> (8 * (k))) & 0xFFu))
    return f3(fmaf(SLIM_TAP(q.x, 3), br, fmaf(SLIM_TAP(q.x, 2), bl, fmaf(SLIM_TAP(q.x, 1), tr, SLIM_TAP(q.x, 0) * tl))),
              fmaf(SLIM_TAP(q.y, 3), br, fmaf(SLIM_TAP(q.y, 2), bl, fmaf(SLIM_TAP(q.y, 1), tr, SLIM_TAP(q.y, 0) * tl))),
              fmaf(SLIM_TAP(q.z, 3), br, fmaf(SLIM_TAP(q.z, 2), bl, fmaf(SLIM_TAP(q.z, 1), tr, SLIM_TAP(q.z, 0) * tl))));
#undef SLIM_TAP
}
SLIM_D uint32_t mip_level(float area, uint32_t count) {                                      // texture.h:47-54
    uint32_t m = 0;
    while (area > 1 && ++m < count) area *= 0.25f;
    if (m >= count) m = count - 1;
    return m;
}
template <bool COUNT>
SLIM_D float3 texture_sample(const DevScene &S, uint32_t tex, float u, float v, float coverage, Work &w) {  // texture.h:68-70
    DevTexture t = S.textures[tex];
    uint32_t m = (t.flags & SLIM_IMAGE_MIPMAP) ? mip_level(coverage * (float)(t.width * t.height), t.mip_count) : 0;
    return mip_sample<COUNT>(S, S.mips[t.mip_base + m], u, v, w);
}
template <bool COUNT>
SLIM_D float3 texture_sample_cube(const DevScene &S, uint32_t tex, float X, float Y, float Z, Work &w) {  // texture.h:72-116
    float u, v;
    uint32_t mip = 0;
    float right = signbit(X) ? 0.0f : 1.0f, left = signbit(X) ? 1.0f : 0.0f;
    float zx = X ? (Z / X) : 2, yx = X ? (Y / X) : 2;
    if (zx <= 1 && zx >= -1 && yx <= 1 && yx >= -1) {
        u = fmaf(zx, -0.125f, fmaf(0.5f, right, 0.125f));
        v = fmaf(yx, left - 0.5f, 0.5f);
    } else {
        float xz = Z ? (X / Z) : 2, yz = Z ? (Y / Z) : 2;
        float sz = signbit(Z) ? 1.0f : 0.0f;
        if (xz <= 1 && xz >= -1 && yz <= 1 && yz >= -1) {
            v = fmaf(yz, sz - 0.5f, +0.5f);
            u = fmaf(xz, 0.125f, fmaf(sz, 0.5f, 0.375f));
        } else {
            u = fmaf(X / fabsf(Y), 0.5f, 0.5f);
            v = fmaf(Z / Y, 0.5f, 0.5f);
            mip = signbit(Y) ? 2u : 1u;
        }
    }
    DevTexture t = S.textures[tex];
    return mip_sample<COUNT>(S, S.mips[t.mip_base + mip], u, v, w);
}

// ---- materials (scene/material.h) ------------------------------------------
struct Mat {
    float3 albedo; float roughness;
    uint32_t flags, texture_count, tex0, tex1;
    int brdf;
    float normal_magnitude, rep_u, rep_v;
    float3 emission; float IOR;
    float3 reflectivity; float metalness;
};
SLIM_D Mat load_mat(const DevScene &S, uint32_t i) {
    const SlimMaterial *p = S.materials + i;
    Mat m;
    m.albedo = ld3(p->albedo);
    m.roughness = __ldg(&p->roughness);
    uint32_t packed = __ldg(reinterpret_cast<const uint32_t *>(&p->flags));
    m.flags = packed & 0xFFu;
    m.texture_count = (packed >> 8) & 0xFFu;
    m.tex0 = (packed >> 16) & 0xFFu;
    m.tex1 = packed >> 24;
    m.brdf = __ldg(&p->brdf);
    m.normal_magnitude = __ldg(&p->normal_magnitude);
    m.rep_u = __ldg(&p->uv_repeat.x);
    m.rep_v = __ldg(&p->uv_repeat.y);
    m.emission = ld3(p->emission);
    m.IOR = __ldg(&p->IOR);
    m.reflectivity = ld3(p->reflectivity);
    m.metalness = __ldg(&p->metalness);
    return m;
}
SLIM_D float3 schlick_fresnel(float HdotL, float3 F0) {                              // material.h:57-59
    float p = powf(1.0f - HdotL, 5.0f);
    return F0 + one_minus(F0) * p;
}
SLIM_D float ggx_d(float roughness, float NdotH) {                                   // material.h:27-36
    float a = roughness * roughness;
    float denom = NdotH * NdotH * (a - 1.0f) + 1.0f;
    return a / (kPi * denom * denom);
}
SLIM_D float ggx_g(float roughness, float NdotL, float NdotV) {                      // material.h:38-55
    float a = roughness * roughness;
    float k = a * 0.5f;
    float omk = 1.0f - k;
    float denom = fmaf(NdotV, omk, k);
    float result = NdotV / fmaxf(denom, kEps);
    denom = fmaf(NdotL, omk, k);
    result *= NdotL / fmaxf(denom, kEps);
    return result;
}

// SurfaceShader state (renderer/surface_shader.h:33-42)
struct Surface {
    float3 P, N, V, L, R, RF;
    float3 albedo_from_map, Fs, Fd;
    float Ld, Ld2, NdotL, NdotV;
    bool refracted;
};

// SurfaceShader::radianceFraction (surface_shader.h:109-145)
SLIM_D void radiance_fraction(Surface &s, const Mat &m) {
    s.Fs = f3(0, 0, 0);
    s.Fd = m.albedo * s.albedo_from_map;
    if (m.brdf == SLIM_BRDF_COOK_TORRANCE) {
        s.Fd = s.Fd * ((1.0f - m.metalness) * kOneOverPi);
        if (s.NdotV > 0.0f && m.roughness > 0.0f) {
            float3 H = normalized(s.L + s.V);
            float NdotH = clamp01(dot(s.N, H));
            float HdotL = clamp01(dot(H, s.L));
            float3 F = schlick_fresnel(HdotL, m.reflectivity);
            float D = ggx_d(m.roughness, NdotH);
            float G = ggx_g(m.roughness, s.NdotL, s.NdotV);
            s.Fs = F * (D * G / (4.0f * s.NdotL * s.NdotV));
            s.Fd = s.Fd * one_minus(F);
        }
    } else {
        s.Fd = s.Fd * (m.roughness * kOneOverPi);
        if (m.brdf != SLIM_BRDF_LAMBERT) {
            float spec, exponent;
            if (m.brdf == SLIM_BRDF_PHONG) {
                exponent = 4.0f;
                spec = clamp01(dot(s.R, s.L));
            } else {
                exponent = 16.0f;
                spec = clamp01(dot(s.N, normalized(s.L + s.V)));
            }
            if (spec > 0.0f) s.Fs = m.reflectivity * (powf(spec, exponent) * (1.0f - m.roughness));
        }
    }
}

// rotateNormal (material.h:83-86)
SLIM_D float3 rotate_normal(float3 normal, float3 sample, float magnitude) {
    float3 N = normalized(f3(fmaf(sample.x, 2.0f, -1.0f), fmaf(sample.z, 2.0f, -1.0f), fmaf(sample.y, 2.0f, -1.0f)));
    float3 axis = normalized(f3(N.z, 0, -N.x));
    float radians = acosf(N.y) * magnitude;
    radians *= 0.5f;
    float3 qa = axis * sinf(radians);
    float qw = cosf(radians);
    float len = sqrtf(qa.x * qa.x + qa.y * qa.y + qa.z * qa.z + qw * qw);
    float f = 1.0f / len;
    return qrot(qa * f, qw * f, normal);
}

template <bool COUNT>
SLIM_D float3 sample_slot(const DevScene &S, const Mat &m, uint32_t slot, float u, float v, float coverage, Work &w) {
    if (!S.texture_count || m.texture_count <= slot) return f3(0, 0, 0);
    return texture_sample<COUNT>(S, slot ? m.tex1 : m.tex0, u, v, coverage, w);
}

// SurfaceShader::prepareForShading (surface_shader.h:61-107).  `ray` is the
// traced world-space ray (origin already offset), `hit` the local-space hit.
template <bool COUNT>
SLIM_D void prepare_for_shading(const DevScene &S, const Geo &g, const Mat &m, const Ray &ray, Hit &hit,
                                float scaling, Surface &s, Work &w) {
    hit.u *= m.rep_u;
    hit.v *= m.rep_v;
    if (hit.from_behind) hit.normal = -hit.normal;
    float cone = hit.distance * scaling;
    cone *= cone;
    cone *= cone;
    hit.uv_coverage *= cone / (m.rep_u * m.rep_v * hit.NdotRd * fabsf(dot(one_minus(hit.normal), g.s)));
    hit.position = at(ray, hit.distance);
    hit.normal = normalized(qrot(g.axis, g.w, g.s * hit.normal));
    bool has_maps = m.texture_count != 0;
    if (has_maps && (m.flags & SLIM_MATERIAL_HAS_NORMAL_MAP))
        hit.normal = rotate_normal(hit.normal, sample_slot<COUNT>(S, m, 1, hit.u, hit.v, hit.uv_coverage, w), m.normal_magnitude);
    s.P = hit.position;
    s.N = hit.normal;
    s.R = s.RF = reflected(ray.d, s.N);
    s.V = -ray.d;
    s.NdotV = clamp01(dot(s.N, s.V));
    s.albedo_from_map = (has_maps && (m.flags & SLIM_MATERIAL_HAS_ALBEDO_MAP))
        ? sample_slot<COUNT>(S, m, 0, hit.u, hit.v, hit.uv_coverage, w) : f3(1, 1, 1);
    s.refracted = (m.flags & SLIM_MATERIAL_IS_REFRACTIVE) != 0;
    if (s.refracted) {
        float ior = hit.from_behind ? (m.IOR / kIorAir) : (kIorAir / m.IOR);
        float c = ior * ior * (1.0f - (s.NdotV * s.NdotV));
        s.refracted = c < 1.0f;
        if (s.refracted) s.RF = normalized(scale_add(s.N, ior * s.NdotV - sqrtf(1 - c), ray.d * ior));
    }
}

struct LightRec { float3 color, pos; float intensity; uint32_t flags; };
SLIM_D LightRec load_light(const DevScene &S, uint32_t i) {
    const SlimLight *p = S.lights + i;
    LightRec l;
    l.color = ld3(p->color);
    l.pos = ld3(&p->position_or_direction.x);
    l.intensity = __ldg(&p->intensity);
    l.flags = __ldg(reinterpret_cast<const uint32_t *>(&p->flags)) & 0xFFu;
    return l;
}

// SurfaceShader::isFacingLight (surface_shader.h:147-160)
SLIM_D bool is_facing_light(Surface &s, const LightRec &l) {
    if (l.flags & SLIM_LIGHT_IS_DIRECTIONAL) {
        s.Ld = INFINITY;
        s.Ld2 = 1.0f;
        s.L = -l.pos;
    } else {
        s.L = l.pos - s.P;
        s.Ld2 = sqlen(s.L);
        s.Ld = sqrtf(s.Ld2);
        s.L = divs(s.L, s.Ld);
    }
    s.NdotL = clamp01(dot(s.L, s.N));
    return s.NdotL > 0.0f;
}

// Light contribution once the shadow test passed (surface_shader.h:57-58).
SLIM_D void add_light(Surface &s, const Mat &m, const LightRec &l, float3 &color) {
    radiance_fraction(s, m);
    color = mul_add(s.Fs + s.Fd, l.color * (s.NdotL * l.intensity / s.Ld2), color);
}

// SurfaceShader::getAreaLightVector (surface_shader.h:162-186)
SLIM_D float3 area_light_vector(const Surface &s, const Geo &q, float3 verts[4]) {
    const float sx = q.s.x, sz = q.s.z;
    if (sx == 0 || sz == 0) return f3(0, 0, 0);
    float3 U = qrot(q.axis, q.w, f3(sx < 0 ? -sx : sx, 0.0f, 0.0f));
    float3 V = qrot(q.axis, q.w, f3(0.0f, 0.0f, sz < 0 ? -sz : sz));
    verts[0] = (q.p - U) - V;
    verts[1] = (q.p + U) - V;
    verts[2] = (q.p + U) + V;
    verts[3] = (q.p - U) + V;
    float3 u1 = normalized(verts[0] - s.P), u2 = normalized(verts[1] - s.P);
    float3 u3 = normalized(verts[2] - s.P), u4 = normalized(verts[3] - s.P);
    return ((cross(u1, u2) * (acosf(dot(u1, u2)) * 0.5f) + cross(u2, u3) * (acosf(dot(u2, u3)) * 0.5f)) +
            cross(u3, u4) * (acosf(dot(u3, u4)) * 0.5f)) + cross(u4, u1) * (acosf(dot(u4, u1)) * 0.5f);
}

// SurfaceShader::shadeFromEmissiveQuads (surface_shader.h:188-264): the
// analytic soft shadow only ever tests sphere and quad occluders; other
// geometries leave the running minimum as Min(shaded, 1) does.
SLIM_D void shade_from_emissive_quads(const DevScene &S, int self, Surface &s, const Mat &m, float3 &color) {
    for (uint32_t e = 0; e < S.emissive_quad_count; e++) {
        uint32_t qi = __ldg(S.emissive_quads + e);
        if ((int)qi == self) continue;
        Geo q = load_geo(S, qi);
        s.L = q.p - s.P;
        s.NdotL = dot(s.N, s.L);
        if (s.NdotL <= 0.0f) continue;
        s.Ld2 = sqlen(s.L);
        s.Ld = sqrtf(s.Ld2);
        float Ld_rcp = 1.0f / s.Ld;
        s.L = s.L * Ld_rcp;
        s.NdotL *= Ld_rcp;
        float3 Ro = scale_add(s.L, kTraceOffset, s.P);
        float3 verts[4];
        float ei = dot(s.N, area_light_vector(s, q, verts));
        if (!(ei > 0)) continue;
        bool skip = true;
        for (int k = 0; k < 4; k++)
            if (dot(s.N, verts[k] - s.P) >= 0) { skip = false; break; }
        if (skip) continue;
        float shaded = 1.0f;
        for (uint32_t j = 0; j < S.geometry_count; j++) {
            if (j == qi || (int)j == self) continue;
            Geo o = load_geo(S, j);
            float d = 1.0f;
            if (o.type == SLIM_GEOMETRY_SPHERE || o.type == SLIM_GEOMETRY_QUAD) {
                Ray sr;
                localize(sr, Ro, s.L, o);
                // The reference normalises the direction after reset(), so the
                // reciprocal and scaled origin stay those of the raw direction.
                sr.d = normalized(sr.d);
                Hit sh;
                sh.distance = INFINITY;
                bool tr = (o.flags & SLIM_GEOMETRY_IS_TRANSPARENT) != 0;
                if (o.type == SLIM_GEOMETRY_SPHERE) {
                    float sq;
                    if (hit_sphere(sr, sh, tr, &sq)) d -= (1.0f - sqrtf(sq)) / (sh.distance * ei * 3.0f);
                } else if (hit_quad(sr, sh, tr)) {
                    float ax = fabsf(sh.position.x), az = fabsf(sh.position.z);
                    d -= 3.0f * (1.0f - maxr(ax, az)) / (sh.distance * ei);
                }
            }
            shaded = minr(shaded, d);
        }
        if (shaded > 0.0f) {
            radiance_fraction(s, m);
            Mat em = load_mat(S, q.material);
            color = mul_add(s.Fd + s.Fs, em.emission * (ei * shaded * 7.0f), color);
        }
    }
}

// Light glow (renderer/ray_tracer.h:98-101, core/ray.h:314-347).
SLIM_D void add_glow(const DevScene &S, const Ray &ray, float &hit_distance, float3 &color) {
    for (uint32_t i = 0; i < S.light_count; i++) {
        LightRec l = load_light(S, i);
        if (l.flags & SLIM_LIGHT_IS_DIRECTIONAL) continue;
        float radius = l.intensity * kLightIntensityRadius;
        float orr = kLightRadiusIntensity / l.intensity;
        float t_max = hit_distance * orr;
        float3 rc = (l.pos - ray.o) * orr;
        float b = dot(ray.d, rc);
        float c = sqlen(rc) - 1;
        float h = b * b - c;
        if (h >= 0) {
            h = sqrtf(h);
            float t_near = b - h, t_far = b + h;
            if (t_far > 0 && t_near < t_max) {
                hit_distance = t_max * radius;
                float tn = maxr(t_near, 0), tf = minr(t_far, t_max);
                float tn2 = tn * tn, tf2 = tf * tf;
                float density = (c * tn - b * tn2 + tn * tn2 / 3.0f - (c * tf - b * tf2 + tf * tf2 / 3.0f)) * (3.0f / 4.0f);
                color = scale_add(l.color, powf(density, 8.0f) * 4, color);
            }
        }
    }
}

SLIM_D float tone_mapped_baked(float c) {                                            // base.h:777-786
    float x = c - 0.004f;
    if (x < 0.0f) x = 0.0f;
    float x2s = x * x * 6.2f;
    return (x2s + x * 0.5f) / (x2s + x * 1.7f + 0.06f);
}

SLIM_D float3 color_of_id(int id) {                                                  // base.h:806-855
    switch (id) {
        case 1: return f3(1, 1, 1);
        case 2: return f3(0.5f, 0.5f, 0.5f);
        case 3: return f3(1, 0, 0);
        case 4: return f3(0, 1, 0);
        case 5: return f3(0, 0, 1);
        case 6: return f3(0, 1, 1);
        case 7: return f3(1, 0, 1);
        case 8: return f3(1, 1, 0);
        case 9: return f3(0.5f, 0, 0);
        case 10: return f3(0, 0.5f, 0);
        case 11: return f3(0, 0, 0.5f);
        case 12: return f3(0.25f, 0.25f, 0.25f);
        case 13: return f3(1, 0.5f, 0.5f);
        case 14: return f3(0.5f, 1, 0.5f);
        case 15: return f3(0.5f, 0.5f, 1);
        case 16: return f3(0.75f, 0.75f, 0.75f);
        case 17: return f3(0, 0.75f, 0.75f);
        case 18: return f3(0.75f, 0, 0.75f);
        case 19: return f3(0.75f, 0.75f, 0);
        case 20: return f3(0, 0.5f, 0.5f);
        case 21: return f3(0.5f, 0, 0.5f);
        case 22: return f3(0.5f, 0.5f, 0);
        case 23: return f3(0.04f, 0.04f, 0.04f);
        case 24: return f3(0.02f, 0.02f, 0.02f);
        case 25: return f3(0.03f, 0.03f, 0.03f);
        case 26: return f3(0.08f, 0.08f, 0.08f);
        case 27: return f3(0.03f, 0.03f, 0.03f);
        case 28: return f3(0.05f, 0.05f, 0.05f);
        case 29: return f3(0.08f, 0.08f, 0.08f);
        case 30: return f3(0.17f, 0.17f, 0.17f);
        case 31: return f3(0.56f, 0.57f, 0.58f);
        case 32: return f3(0.95f, 0.64f, 0.54f);
        case 33: return f3(1.0f, 0.71f, 0.29f);
        case 34: return f3(0.91f, 0.92f, 0.92f);
        case 35: return f3(0.95f, 0.93f, 0.88f);
        default: return f3(0, 0, 0);
    }
}

// Primary ray of sample (x, y): getRayDirectionAt (scene/camera.h:67) and
// d_render's per-pixel cone spread (renderer/renderer_GPU.h:38-40).
SLIM_D float3 primary_direction(const SlimCameraRayProjection &p, int x, int y) {
    float3 start = f3(p.start.x, p.start.y, p.start.z);
    float3 down = f3(p.down.x, p.down.y, p.down.z);
    float3 right = f3(p.right.x, p.right.y, p.right.z);
    return (start + down * (float)y) + right * (float)x;
}
// Primary rays are numbered in 8 x 4 pixel tiles, so the 32 rays of a warp
// (and the shadow rays and hits that follow them through the queues) cover
// a compact patch instead of a 32-pixel row strip: within every band of 4
// rows the slots run through 8-column groups; the columns past the last
// full group, and a last band shorter than 4 rows, keep row order.  A
// bijection of [0, width * height); config 2: 2.08 -> 2.03 ms.
SLIM_D uint32_t pixel_of_slot(uint32_t W, uint32_t H, uint32_t slot) {
    const uint32_t band = 4u * W;
    const uint32_t b = slot / band;
    if (b >= H / 4u) return slot;
    const uint32_t j = slot - b * band;
    const uint32_t groups = W / 8u, g = j / 32u;
    uint32_t x, y;
    if (g < groups) {
        x = g * 8u + (j & 7u);
        y = b * 4u + ((j & 31u) >> 3);
    } else {
        const uint32_t r = j - groups * 32u, rest = W - groups * 8u;
        x = groups * 8u + r % rest;
        y = b * 4u + r / rest;
    }
    return y * W + x;
}

SLIM_D float pixel_scaling(const SlimCameraRayProjection &p, int x, int y) {
    float cx = fmaf((float)x, p.sample_size, p.C_start.x);
    float cy = fmaf((float)-y, p.sample_size, p.C_start.y);
    return 1.0f / sqrtf(p.squared_distance_to_projection_plane + (cx * cx + cy * cy));
}
SLIM_D float depth_at(const SlimCameraRayProjection &p, float3 pos) {               // camera.h:66
    float3 v = pos - f3(p.camera_position.x, p.camera_position.y, p.camera_position.z);
    const float *m = p.inverted_camera_rotation;
    return m[2] * v.x + m[5] * v.y + m[8] * v.z;
}

// Canvas::setPixel(x, y, color, -1, depth) (draw/canvas.h:128-165), in two
// halves so a frame can write its depths before its colours are final.
// Canvas entry of a sample: SSAA keeps a pixel's four samples together.
SLIM_D uint32_t canvas_offset(const DevFrame &F, int x, int y) {
    return F.antialias == SLIM_AA_SSAA
        ? ((F.stride * (uint32_t)(y >> 1) + (uint32_t)(x >> 1)) * 4 + 2 * (uint32_t)(y & 1) + (uint32_t)(x & 1))
        : (F.stride * (uint32_t)y + (uint32_t)x);
}
SLIM_D void set_pixel_color(const DevFrame &F, int x, int y, float3 c) {
    c = f3(clamp01(c.x), clamp01(c.y), clamp01(c.z));
    c = c * (c * 1.0f);
    F.pixels[canvas_offset(F, x, y)] = make_float4(c.x, c.y, c.z, 1.0f);
}
SLIM_D void set_depth(const DevFrame &F, int x, int y, float depth) {
    uint32_t offset = canvas_offset(F, x, y);
    if (F.antialias == SLIM_AA_MSAA) {
        F.depths[offset * 4] = depth;
        F.depths[offset * 4 + 1] = 0;
        F.depths[offset * 4 + 2] = 0;
        F.depths[offset * 4 + 3] = 0;
    } else {
        F.depths[offset] = depth;
    }
}
SLIM_D void set_pixel(const DevFrame &F, int x, int y, float3 c, float depth) {
    set_pixel_color(F, x, y, c);
    set_depth(F, x, y, depth);
}

// renderPixelBeauty (renderer/ray_tracer.h:19-108) as a sequence of path
// segments: a path's state between two segments is the ray of the next one,
// the colour and throughput so far, the canvas depth and the bounces left.
struct PathState {
    float3 o, d;
    float3 color, throughput;
    float depth, scaling;
    uint32_t depth_left;
};

template <bool COUNT>
SLIM_D void path_start(const DevFrame &F, int x, int y, PathState &p, Work &w) {
    const SlimCameraRayProjection &P = F.projection;
    p.scaling = F.cones_per_pixel ? pixel_scaling(P, x, y) : 0.0f;
    p.o = f3(P.camera_position.x, P.camera_position.y, P.camera_position.z);
    p.d = normalized(primary_direction(P, x, y));
    bump<COUNT>(w.primary);
    p.color = f3(0, 0, 0);
    p.throughput = f3(1, 1, 1);
    p.depth = INFINITY;
    p.depth_left = F.settings.max_depth;
}

// One segment: closest hit, shading (point lights with their shadow rays,
// area lights, IBL), the bounce decision, the light glow of the segment.
// Returns whether the path goes on.
template <bool COUNT>
SLIM_D bool path_segment(const DevScene &S, const DevFrame &F, PathState &p, uint32_t *stack, uint32_t *mesh_stack,
                         uint32_t &err, Work &w, bool glow = true) {
    const SlimRayTracerSettings &st = F.settings;
    Ray ray;
    reset(ray, p.o, p.d);
    Hit hit;
    Surface s;
    float3 current = f3(0, 0, 0), next_throughput = f3(0, 0, 0);
    int g = scene_trace<COUNT>(S, ray, hit, false, INFINITY, stack, mesh_stack, err, w);
    if (g >= 0) {
        Geo geo = load_geo(S, (uint32_t)g);
        Mat m = load_mat(S, geo.material);
        if ((m.flags & SLIM_MATERIAL_IS_EMISSIVE) && geo.type == SLIM_GEOMETRY_QUAD && !hit.from_behind) {
            p.depth_left = 0;
            current = m.emission;
        } else {
            prepare_for_shading<COUNT>(S, geo, m, ray, hit, p.scaling, s, w);
            if (p.depth_left == st.max_depth) p.depth = depth_at(F.projection, hit.position);
            for (uint32_t i = 0; i < S.light_count; i++) {
                LightRec l = load_light(S, i);
                if (!is_facing_light(s, l)) continue;
                if (l.flags & SLIM_LIGHT_IS_SHADOWING) {
                    Ray sr;
                    sr.o = s.P;
                    sr.d = s.L;
                    Hit sh;
                    bump<COUNT>(w.shadow);
                    const uint32_t sn = w.scene_nodes, mn = w.mesh_nodes, tr = w.triangles, ge = w.geometries;
                    const bool occluded = scene_trace<COUNT>(S, sr, sh, true, s.Ld, stack, mesh_stack, err, w) >= 0;
                    bump<COUNT>(w.any_scene_nodes, w.scene_nodes - sn);
                    bump<COUNT>(w.any_mesh_nodes, w.mesh_nodes - mn);
                    bump<COUNT>(w.any_triangles, w.triangles - tr);
                    bump<COUNT>(w.any_geometries, w.geometries - ge);
                    if (occluded) continue;
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
            if ((m.flags & (SLIM_MATERIAL_IS_REFLECTIVE | SLIM_MATERIAL_IS_REFRACTIVE)) && --p.depth_left) {
                float3 Fr = schlick_fresnel(clamp01(dot(s.N, s.R)), m.reflectivity);
                next_throughput = s.refracted ? one_minus(Fr) : Fr;
                reset(ray, hit.position, s.RF);
                bump<COUNT>(w.bounce);
            } else p.depth_left = 0;
        }
    } else {
        p.depth_left = 0;
        if (st.skybox_color_texture_id >= 0)
            current = texture_sample_cube<COUNT>(S, (uint32_t)st.skybox_color_texture_id, ray.d.x, ray.d.y, ray.d.z, w);
    }
    if (glow) add_glow(S, ray, hit.distance, current);
    p.color = mul_add(current, p.throughput, p.color);
    p.throughput = p.throughput * next_throughput;
    p.o = ray.o;
    p.d = ray.d;
    return p.depth_left != 0;
}

}  // namespace dev
}  // namespace slim
