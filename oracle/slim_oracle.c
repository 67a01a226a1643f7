/*
 * oracle/slim_oracle.c -- TEST INFRASTRUCTURE: the CPU oracle.
 *
 * A scalar plain-C restatement of SlimTracin's per-pixel trace path
 * (HardCoreCodin/SlimTracinCpp), used only as the checker by tests/,
 * __graft_entry__.smoke() and as bench.py's CPU baseline ("port").  The
 * product never links or calls it.  Each function names the reference
 * lines it follows.  Floating-point policy (identical to oracle/_ref and to
 * the CUDA kernels): the reference's fast_mul_add sites are fmaf, nothing
 * else is contracted (-ffp-contract=off), IEEE division and square root.
 *
 * It is pinned against the reference itself (oracle/_ref/libslimref.so,
 * built from the reference sources by oracle/build_ref.sh) and against the
 * committed golden frames in tests/golden/ that the reference produced.
 *
 * State semantics: the reference keeps tracer/shader state in structs whose
 * never-written members read as zero (value-initialised app object); the
 * restatement zero-initialises the same state for every pixel, as d_render
 * creates it per pixel (renderer/renderer_GPU.h:28-33).  Stale-state reads
 * the reference relies on are reproduced: RayHit copies carry the aux hit's
 * scaling_factor (always 0), the emissive-quad shadow ray keeps the
 * reciprocal of its un-normalised direction, and the light glow reads the
 * ray after the bounce was set up.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

#include "../include/slimtracer_b200.h"

typedef struct { float x, y, z; } v3;
typedef struct { float u, v; } v2;

#define EPS_ 0.0001f
#define PI_ 3.14159265f
#define ONE_OVER_PI_ (1.0f / PI_)
#define UNIT_SPHERE_AREA_OVER_SIX_ ((4.0f * PI_) / 6.0f)
#define TET_MAX_ 0.577350259f
#define TET_MIN_ 0.288675159f
#define SQRT3_ 1.73205080757f
#define TRACE_OFFSET_ 0.0001f
#define IOR_AIR_ 1.0003f
#define LIGHT_RADIUS_INTENSITY_FACTOR_ 64.0f
#define LIGHT_INTENSITY_RADIUS_FACTOR_ (1.0f / LIGHT_RADIUS_INTENSITY_FACTOR_)
#define COLOR_COMPONENT_TO_FLOAT_ 0.00392156862f
#define MAXF(a, b) ((a) > (b) ? (a) : (b))
#define MINF(a, b) ((a) < (b) ? (a) : (b))

enum { BOX_NONE = 0, BOX_LEFT = 1, BOX_BOTTOM = 2, BOX_BACK = 4, BOX_RIGHT = 8, BOX_TOP = 16, BOX_FRONT = 32 };

/* ---- vector helpers: math/vec3.h, math/vec2.h, math/quat.h ------------- */
static inline v3 V3(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmul(v3 a, v3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 vscale(v3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline v3 vneg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline float vdot(v3 a, v3 b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }           /* vec3.h:285 */
static inline v3 vcross(v3 a, v3 b) {                                                               /* vec3.h:289 */
    return V3((a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x));
}
static inline float vsqlen(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }                   /* vec3.h:297 */
static inline v3 vdivs(v3 a, float s) { float f = 1.0f / s; return vscale(a, f); }                 /* vec3.h:154 */
static inline v3 vnormalized(v3 a) { return vdivs(a, sqrtf(vsqlen(a))); }                          /* vec3.h:305 */
static inline v3 vscaleadd(v3 a, float f, v3 b) {                                                   /* vec3.h:356 */
    return V3(fmaf(a.x, f, b.x), fmaf(a.y, f, b.y), fmaf(a.z, f, b.z));
}
static inline v3 vmuladd(v3 a, v3 m, v3 b) {                                                        /* vec3.h:372 */
    return V3(fmaf(a.x, m.x, b.x), fmaf(a.y, m.y, b.y), fmaf(a.z, m.z, b.z));
}
static inline v3 vrcp(v3 a) { return V3(1.0f / a.x, 1.0f / a.y, 1.0f / a.z); }                    /* vec3.h:452 */
static inline v3 vreflect(v3 d, v3 n) { return vscaleadd(n, -2.0f * vdot(d, n), d); }              /* vec3.h:309 */
static inline float clamp01(float v) { float mn = v < 1.0f ? v : 1.0f; return mn > 0.0f ? mn : 0.0f; }  /* base.h:208 */
static inline float vmaxc(v3 a) { float yz = MAXF(a.y, a.z); return MAXF(a.x, yz); }               /* vec3.h:262 */
static inline float vminc(v3 a) { float yz = MINF(a.y, a.z); return MINF(a.x, yz); }               /* vec3.h:247 */
static inline float vmaxc_axis(v3 a, int *axis) {                                                   /* vec3.h:264-277 */
    float r = a.x; *axis = 1;
    if (a.y > r) { r = a.y; *axis = 2; }
    if (a.z > r) { r = a.z; *axis = 4; }
    return r;
}
static inline float vminc_axis(v3 a, int *axis) {                                                   /* vec3.h:249-260 */
    float r = a.x; *axis = 1;
    if (a.y < r) { r = a.y; *axis = 2; }
    if (a.z < r) { r = a.z; *axis = 4; }
    return r;
}
typedef struct { v3 axis; float w; } quat_;
static inline v3 qrot(quat_ q, v3 v) {                                                              /* quat.h:37-43 */
    v3 out = vcross(q.axis, v);
    v3 qqv = vcross(q.axis, out);
    out = vscaleadd(out, q.w, qqv);
    return vscaleadd(out, 2.0f, v);
}
static inline quat_ qconj(quat_ q) { quat_ r = {vneg(q.axis), q.w}; return r; }
static inline quat_ qnormalized(quat_ q) {                                                          /* quat.h:17-24 */
    float len = sqrtf(q.axis.x * q.axis.x + q.axis.y * q.axis.y + q.axis.z * q.axis.z + q.w * q.w);
    float f = 1.0f / len;
    quat_ r = {vscale(q.axis, f), q.w * f};
    return r;
}
static inline quat_ qaxisangle(v3 axis, float radians) {                                            /* quat.h:86-92 */
    radians *= 0.5f;
    quat_ q = {vscale(axis, sinf(radians)), cosf(radians)};
    return qnormalized(q);
}
static inline int checker(float u, float v) {                                                       /* base.h:277-279 */
    return (((int)(v * 4.0f)) & 1) == (((int)(u * 4.0f)) & 1);
}
static inline v3 mat3_mul(const float m[9], v3 v) {                                                 /* mat3.h:277-283 */
    return V3(m[0] * v.x + m[3] * v.y + m[6] * v.z,
              m[1] * v.x + m[4] * v.y + m[7] * v.z,
              m[2] * v.x + m[5] * v.y + m[8] * v.z);
}

/* ---- ray / hit: core/ray.h --------------------------------------------- */
typedef struct {
    v3 position, normal;
    v2 uv;
    float distance, uv_coverage, cone_width, NdotRd, scaling_factor;
    uint32_t id;
    int from_behind;
} Hit;
typedef struct {
    v3 origin, scaled_origin, direction, rcp;
    int sx, sy, sz;      /* octant shifts: 3 when the component's sign bit is set */
    int left, bottom, back;
} Ray;

static inline v3 ray_at(const Ray *r, float t) { return vscaleadd(r->direction, t, r->origin); }   /* ray.h:26 */
static inline void ray_reset(Ray *r, v3 o, v3 d) {                                                  /* ray.h:40-49 */
    r->origin = o;
    r->direction = d;
    r->rcp = vrcp(d);
    r->scaled_origin = vmul(vneg(o), r->rcp);
    r->left = signbit(d.x) != 0; r->bottom = signbit(d.y) != 0; r->back = signbit(d.z) != 0;
    r->sx = 3 * r->left; r->sy = 3 * r->bottom; r->sz = 3 * r->back;
}
static inline void ray_localize(Ray *r, v3 ro, v3 rd, const SlimTransform *t) {                    /* ray.h:29-34 */
    v3 inv_scale = V3(1.0f / t->scale.x, 1.0f / t->scale.y, 1.0f / t->scale.z);
    quat_ inv = {V3(-t->orientation.axis.x, -t->orientation.axis.y, -t->orientation.axis.z), t->orientation.amount};
    v3 p = V3(t->position.x, t->position.y, t->position.z);
    ray_reset(r, vmul(inv_scale, qrot(inv, vsub(ro, p))), vmul(inv_scale, qrot(inv, rd)));
}
static inline int ray_hits_aabb(const Ray *r, const float *mn, const float *mx, float *nearD, float *farD) {  /* ray.h:51-59 */
    /* aabb.min + shift reads aabb.max when the ray component is negative */
    v3 min_t = V3(r->sx ? mx[0] : mn[0], r->sy ? mx[1] : mn[1], r->sz ? mx[2] : mn[2]);
    v3 max_t = V3(r->sx ? mn[0] : mx[0], r->sy ? mn[1] : mx[1], r->sz ? mn[2] : mx[2]);
    min_t = vmuladd(min_t, r->rcp, r->scaled_origin);
    max_t = vmuladd(max_t, r->rcp, r->scaled_origin);
    float m = vmaxc(min_t);
    *nearD = 0 > m ? 0.0f : m;
    *farD = vminc(max_t);
    return *nearD <= *farD;
}
static inline int ray_hits_plane(const Ray *r, v3 p, v3 n, Hit *hit) {                             /* ray.h:61-82 */
    float NdotRd = vdot(n, r->direction);
    if (NdotRd == 0) return 0;
    float NdotRoP = vdot(n, vsub(p, r->origin));
    if (NdotRoP == 0) return 0;
    int facing = NdotRd < 0;
    hit->from_behind = NdotRoP > 0;
    if (hit->from_behind == facing) return 0;
    float t = NdotRoP / NdotRd;
    hit->distance = t;
    hit->position = ray_at(r, t);
    hit->normal = n;
    return 1;
}
static int ray_hits_quad(const Ray *r, Hit *hit, int transparent) {                               /* ray.h:84-120 */
    if (r->direction.y == 0) return 0;
    if (r->origin.y == 0) return 0;
    hit->from_behind = r->origin.y < 0;
    if (hit->from_behind == (r->direction.y < 0)) return 0;
    float t = fabsf(r->origin.y * r->rcp.y);
    if (t > hit->distance) return 0;
    hit->position = ray_at(r, t);
    if (hit->position.x < -1 || hit->position.x > 1 || hit->position.z < -1 || hit->position.z > 1) return 0;
    hit->uv.u = fmaf(hit->position.x, 0.5f, 0.5f);
    hit->uv.v = fmaf(hit->position.z, 0.5f, 0.5f);
    if (transparent && checker(hit->uv.u, hit->uv.v)) return 0;
    hit->distance = t;
    hit->normal = V3(0.0f, 1.0f, 0.0f);
    hit->uv_coverage = 0.25f;
    return 1;
}
static inline int octant_side(int shift_x, int shift_y, int shift_z, int axis) {                   /* base.h:532-538 */
    return (axis == 1) * (1 << shift_x) | (axis == 2) * (2 << shift_y) | (axis == 4) * (4 << shift_z);
}
static inline void uv_by_box_side(int side, v3 p, v2 *uv) {                                        /* base.h:424-454 */
    float u, v;
    switch (side) {
        case BOX_TOP: u = p.x; v = p.z; break;
        case BOX_BOTTOM: u = -p.x; v = -p.z; break;
        case BOX_LEFT: u = -p.z; v = p.y; break;
        case BOX_RIGHT: u = p.z; v = p.y; break;
        case BOX_FRONT: u = p.x; v = p.y; break;
        default: u = -p.x; v = p.y; break;
    }
    uv->u = fmaf(u, 0.5f, 0.5f);
    uv->v = fmaf(v, 0.5f, 0.5f);
}
static int ray_hits_box(const Ray *r, Hit *hit, int transparent) {                                 /* ray.h:122-175 */
    v3 signed_rcp = V3(1.0f - 2.0f * (float)r->left, 1.0f - 2.0f * (float)r->bottom, 1.0f - 2.0f * (float)r->back);
    signed_rcp = vmul(signed_rcp, r->rcp);
    v3 near_t = vsub(r->scaled_origin, signed_rcp);
    v3 far_t = vadd(r->scaled_origin, signed_rcp);
    int near_axis, far_axis, side;
    float far_hit_t = vminc_axis(far_t, &far_axis);
    if (far_hit_t < 0) return BOX_NONE;
    float near_hit_t = vmaxc_axis(near_t, &near_axis);
    if (near_hit_t > hit->distance || far_hit_t < (near_hit_t > 0 ? near_hit_t : 0)) return BOX_NONE;
    float t = near_hit_t;
    /* flipped faces: the opposite octant */
    int fsx = 3 * !r->left, fsy = 3 * !r->bottom, fsz = 3 * !r->back;
    hit->from_behind = near_hit_t < 0;
    if (hit->from_behind) {
        if (far_hit_t > hit->distance) return BOX_NONE;
        t = far_hit_t;
        side = octant_side(fsx, fsy, fsz, far_axis);
    } else
        side = octant_side(r->sx, r->sy, r->sz, near_axis);
    hit->position = ray_at(r, t);
    uv_by_box_side(side, hit->position, &hit->uv);
    if (transparent && checker(hit->uv.u, hit->uv.v)) {
        if (hit->from_behind || far_hit_t > hit->distance) return BOX_NONE;
        side = octant_side(fsx, fsy, fsz, far_axis);
        hit->from_behind = 1;
        t = far_hit_t;
        hit->position = ray_at(r, t);
        uv_by_box_side(side, hit->position, &hit->uv);
        if (checker(hit->uv.u, hit->uv.v)) return BOX_NONE;
    }
    hit->distance = t;
    hit->normal.x = (float)((int)(side == BOX_RIGHT) - (int)(side == BOX_LEFT));
    hit->normal.y = (float)((int)(side == BOX_TOP) - (int)(side == BOX_BOTTOM));
    hit->normal.z = (float)((int)(side == BOX_FRONT) - (int)(side == BOX_BACK));
    hit->uv_coverage = 0.25f;
    return side;
}
static inline void uv_by_sphere(v3 p, v2 *uv) {                                                    /* base.h:456-483 */
    float X = p.x, Y = p.y, Z = p.z, u, v;
    float z_over_x = X ? (Z / X) : 2;
    float y_over_x = X ? (Y / X) : 2;
    if (z_over_x <= 1 && z_over_x >= -1 && y_over_x <= 1 && y_over_x >= -1) {
        u = z_over_x;
        v = X > 0 ? y_over_x : -y_over_x;
    } else {
        float x_over_z = Z ? (X / Z) : 2;
        float y_over_z = Z ? (Y / Z) : 2;
        if (x_over_z <= 1 && x_over_z >= -1 && y_over_z <= 1 && y_over_z >= -1) {
            u = -x_over_z;
            v = Z > 0 ? y_over_z : -y_over_z;
        } else {
            u = X / (Y > 0 ? Y : -Y);
            v = Z / Y;
        }
    }
    uv->u = fmaf(u, 0.5f, 0.5f);
    uv->v = fmaf(v, 0.5f, 0.5f);
}
static int ray_hits_sphere(const Ray *r, Hit *hit, int transparent, float *out_sq) {               /* ray.h:177-215 */
    float t_to_closest = -(vdot(r->origin, r->direction));
    if (t_to_closest <= 0) return 0;
    float dsl = vsqlen(r->direction);
    float sq = vsqlen(r->origin) * dsl - t_to_closest * t_to_closest;
    if (sq > 1.0f) return 0;
    float delta = sqrtf(dsl - sq);
    dsl = 1.0f / dsl;
    float t = (t_to_closest - delta) * dsl;
    if (t > hit->distance) return 0;
    hit->normal = ray_at(r, t);
    uv_by_sphere(hit->normal, &hit->uv);
    hit->from_behind = t <= 0 || (transparent && checker(hit->uv.u, hit->uv.v));
    if (hit->from_behind) {
        t = (t_to_closest + delta) * dsl;
        if (t <= 0 || t > hit->distance) return 0;
        hit->normal = ray_at(r, t);
        uv_by_sphere(hit->normal, &hit->uv);
        if (transparent && checker(hit->uv.u, hit->uv.v)) return 0;
    }
    hit->distance = t;
    hit->uv_coverage = 1.0f / UNIT_SPHERE_AREA_OVER_SIX_;
    if (out_sq) *out_sq = sq * dsl;
    return 1;
}
static const float TET_TANGENT[4][9] = {                                                            /* ray.h:239-292 */
    { TET_MAX_, -TET_MIN_, -TET_MAX_,  TET_MIN_,  TET_MIN_,  TET_MAX_, -TET_MIN_,  TET_MAX_, -TET_MAX_},
    { TET_MIN_,  TET_MIN_,  TET_MAX_, -TET_MIN_,  TET_MAX_, -TET_MAX_,  TET_MAX_, -TET_MIN_, -TET_MAX_},
    {-TET_MIN_,  TET_MAX_, -TET_MAX_,  TET_MAX_, -TET_MIN_, -TET_MAX_,  TET_MIN_,  TET_MIN_,  TET_MAX_},
    {-TET_MAX_,  TET_MIN_,  TET_MAX_,  TET_MIN_,  TET_MIN_,  TET_MAX_,  TET_MIN_, -TET_MAX_,  TET_MAX_},
};
static int ray_hits_tet(const Ray *r, Hit *hit, int transparent) {                                 /* ray.h:217-311 */
    int found = 0;
    Hit cur; memset(&cur, 0, sizeof(cur));   /* a fresh local RayHit; never-written fields read 0 */
    cur.uv.u = cur.uv.v = 1.0f;
    cur.uv_coverage = SQRT3_ / 4.0f;
    for (int t = 0; t < 4; t++) {
        float c = t == 3 ? TET_MAX_ : -TET_MAX_;
        v3 tangent_pos = V3(c, c, c), face_normal = V3(c, c, c);
        switch (t) {
            case 0: face_normal.y = TET_MAX_; break;
            case 1: face_normal.x = TET_MAX_; break;
            case 2: face_normal.z = TET_MAX_; break;
            case 3: tangent_pos.y = -TET_MAX_; break;
        }
        cur.distance = hit->distance;
        if (!ray_hits_plane(r, tangent_pos, face_normal, &cur)) continue;
        tangent_pos = mat3_mul(TET_TANGENT[t], vsub(cur.position, tangent_pos));
        if (tangent_pos.x < 0 || tangent_pos.y < 0 || tangent_pos.y + tangent_pos.x > 1) continue;
        cur.uv.u = tangent_pos.x;
        cur.uv.v = tangent_pos.y;
        if (transparent && checker(cur.uv.u, cur.uv.v)) continue;
        if (cur.distance < hit->distance) { *hit = cur; found = 1; }
    }
    return found;
}

/* ---- tracers: scene/scene_tracer.h, scene/mesh_tracer.h ----------------- */
typedef struct {
    float b, c, t_near, t_far, t_max;
} SphereTracer;
typedef struct {
    Ray aux_ray;
    Hit aux_hit, triangle_hit;
    SphereTracer light;
    uint32_t scene_stack[256], mesh_stack[256];
    SlimWorkCounters *counters;
} Tracer;

#define COUNT(field) do { if (tr->counters) tr->counters->field++; } while (0)

static int hit_triangles(Tracer *tr, const SlimTriangle *tris, uint32_t count, float closest,
                         const Ray *r, Hit *hit, int any_hit) {                                     /* mesh_tracer.h:23-49 */
    int found = 0;
    closest = MINF(closest, hit->distance);
    for (uint32_t i = 0; i < count; i++) {
        const SlimTriangle *t = tris + i;
        COUNT(triangle_tests);
        v3 tp = V3(t->position.x, t->position.y, t->position.z);
        v3 tn = V3(t->normal.x, t->normal.y, t->normal.z);
        if (ray_hits_plane(r, tp, tn, &tr->triangle_hit)) {
            v3 uvw = mat3_mul(t->local_to_tangent, vsub(tr->triangle_hit.position, tp));
            if (uvw.x < 0 || uvw.y < 0 || (uvw.x + uvw.y) > 1 || tr->triangle_hit.distance >= closest) continue;
            closest = tr->triangle_hit.distance;
            *hit = tr->triangle_hit;
            hit->uv.u = uvw.x;
            hit->uv.v = uvw.y;
            hit->uv_coverage = t->uv_coverage;
            hit->id = i;
            found = 1;
            if (any_hit) break;
        }
    }
    return found;
}

static int mesh_trace(Tracer *tr, const SlimMesh *mesh, Ray *r, Hit *hit, int any_hit) {           /* mesh_tracer.h:51-134 */
    float ln, rn, lf, rf;
    const SlimBVHNode *nodes = mesh->bvh.nodes;
    int found = 0;
    COUNT(mesh_node_tests);
    if (!(ray_hits_aabb(r, &nodes->aabb.min.x, &nodes->aabb.max.x, &ln, &lf) && ln < hit->distance)) return 0;
    if (nodes->leaf_count) return hit_triangles(tr, mesh->triangles, mesh->triangle_count, lf, r, hit, any_hit);
    const SlimBVHNode *left = nodes + nodes->first_index, *right;
    uint32_t top = 0;
    for (;;) {
        right = left + 1;
        COUNT(mesh_node_tests); COUNT(mesh_node_tests);
        int hl = ray_hits_aabb(r, &left->aabb.min.x, &left->aabb.max.x, &ln, &lf) && ln < hit->distance;
        int hr = ray_hits_aabb(r, &right->aabb.min.x, &right->aabb.max.x, &rn, &rf) && rn < hit->distance;
        if (hl) {
            if (left->leaf_count) {
                if (hit_triangles(tr, mesh->triangles + left->first_index, left->leaf_count, lf, r, hit, any_hit)) {
                    hit->id += left->first_index;
                    found = 1;
                    if (any_hit) break;
                }
                left = NULL;
            }
        } else left = NULL;
        if (hr) {
            if (right->leaf_count) {
                if (hit_triangles(tr, mesh->triangles + right->first_index, right->leaf_count, rf, r, hit, any_hit)) {
                    hit->id += right->first_index;
                    found = 1;
                    if (any_hit) break;
                }
                right = NULL;
            }
        } else right = NULL;
        if (left) {
            if (right) {
                if (!any_hit && ln > rn) { const SlimBVHNode *tmp = left; left = right; right = tmp; }
                tr->mesh_stack[top++] = right->first_index;
            }
            left = nodes + left->first_index;
        } else if (right) {
            left = nodes + right->first_index;
        } else {
            if (top == 0) break;
            left = nodes + tr->mesh_stack[--top];
        }
    }
    if (found && !any_hit && (mesh->normals_count | mesh->uvs_count)) {
        const SlimTriangle *t = mesh->triangles + hit->id;
        COUNT(mesh_hit_fetches);
        float a = hit->uv.u, b = hit->uv.v, c = 1 - a - b;
        if (mesh->uvs_count) {
            hit->uv.u = fmaf(t->uv3.x, a, fmaf(t->uv2.x, b, t->uv1.x * c));
            hit->uv.v = fmaf(t->uv3.y, a, fmaf(t->uv2.y, b, t->uv1.y * c));
        }
        if (mesh->normals_count) {
            hit->normal.x = fmaf(t->n3.x, a, fmaf(t->n2.x, b, t->n1.x * c));
            hit->normal.y = fmaf(t->n3.y, a, fmaf(t->n2.y, b, t->n1.y * c));
            hit->normal.z = fmaf(t->n3.z, a, fmaf(t->n2.z, b, t->n1.z * c));
        }
    }
    return found;
}

static int hit_geometry_local(Tracer *tr, const SlimGeometry *geo, const SlimMesh *meshes,
                              const Ray *r, Hit *hit, int any_hit) {                               /* scene_tracer.h:138-165 */
    COUNT(geometry_tests);
    ray_localize(&tr->aux_ray, r->origin, r->direction, &geo->transform);
    float mn[3], mx[3], n, f;
    if (geo->type == SLIM_GEOMETRY_MESH) {
        const SlimMesh *m = meshes + geo->id;
        mn[0] = m->aabb.min.x; mn[1] = m->aabb.min.y; mn[2] = m->aabb.min.z;
        mx[0] = m->aabb.max.x; mx[1] = m->aabb.max.y; mx[2] = m->aabb.max.z;
    } else {
        float e = geo->type == SLIM_GEOMETRY_TET ? TET_MAX_ : 1.0f;
        mx[0] = mx[1] = mx[2] = e;
        mn[0] = mn[1] = mn[2] = -e;
        if (geo->type == SLIM_GEOMETRY_QUAD) { mn[1] = -EPS_; mx[1] = EPS_; }
    }
    if (!ray_hits_aabb(&tr->aux_ray, mn, mx, &n, &f)) return 0;
    int transparent = (geo->flags & SLIM_GEOMETRY_IS_TRANSPARENT) != 0;
    switch (geo->type) {
        case SLIM_GEOMETRY_QUAD: return ray_hits_quad(&tr->aux_ray, hit, transparent);
        case SLIM_GEOMETRY_BOX: return ray_hits_box(&tr->aux_ray, hit, transparent) != BOX_NONE;
        case SLIM_GEOMETRY_SPHERE: return ray_hits_sphere(&tr->aux_ray, hit, transparent, NULL);
        case SLIM_GEOMETRY_TET: return ray_hits_tet(&tr->aux_ray, hit, transparent);
        case SLIM_GEOMETRY_MESH: return mesh_trace(tr, meshes + geo->id, &tr->aux_ray, hit, any_hit);
        default: return 0;
    }
}

static int hit_geometries(Tracer *tr, const uint32_t *ids, uint32_t count, const SlimSceneData *s,
                          float closest, const Ray *r, Hit *hit, int any_hit) {                    /* scene_tracer.h:111-136 */
    int hit_geo = -1;
    uint8_t vis = any_hit ? SLIM_GEOMETRY_IS_SHADOWING : SLIM_GEOMETRY_IS_VISIBLE;
    float cd = closest + EPS_;
    tr->aux_hit.distance = MINF(cd, hit->distance);
    for (uint32_t i = 0; i < count; i++) {
        const SlimGeometry *geo = s->geometries + ids[i];
        if (!(geo->flags & vis)) continue;
        if (hit_geometry_local(tr, geo, s->meshes, r, &tr->aux_hit, any_hit)) {
            if (any_hit) return (int)ids[i];
            if (tr->aux_hit.distance < hit->distance) {
                hit_geo = (int)ids[i];
                *hit = tr->aux_hit;
                hit->NdotRd = -(vdot(hit->normal, tr->aux_ray.direction));
            }
        }
    }
    return hit_geo;
}

/* SceneTracer::trace (scene_tracer.h:26-98); returns the geometry index or -1. */
static int scene_trace(Tracer *tr, Ray *r, Hit *hit, const SlimSceneData *s, int any_hit, float max_distance) {
    ray_reset(r, vscaleadd(r->direction, TRACE_OFFSET_, r->origin), r->direction);
    hit->distance = max_distance;
    float ln, rn, lf, rf;
    const SlimBVHNode *nodes = s->bvh.nodes;
    COUNT(scene_node_tests);
    if (!(ray_hits_aabb(r, &nodes->aabb.min.x, &nodes->aabb.max.x, &ln, &lf) && ln < hit->distance)) return -1;
    const uint32_t *indices = s->bvh_leaf_geometry_indices;
    if (nodes->leaf_count) return hit_geometries(tr, indices, s->counts.geometries, s, lf, r, hit, any_hit);
    const SlimBVHNode *left = nodes + nodes->first_index, *right;
    int hit_geo, closest_geo = -1;
    uint32_t top = 0;
    for (;;) {
        right = left + 1;
        COUNT(scene_node_tests); COUNT(scene_node_tests);
        int hl = ray_hits_aabb(r, &left->aabb.min.x, &left->aabb.max.x, &ln, &lf) && ln < hit->distance;
        int hr = ray_hits_aabb(r, &right->aabb.min.x, &right->aabb.max.x, &rn, &rf) && rn < hit->distance;
        if (hl) {
            if (left->leaf_count) {
                hit_geo = hit_geometries(tr, indices + left->first_index, left->leaf_count, s, lf, r, hit, any_hit);
                if (hit_geo >= 0) { closest_geo = hit_geo; if (any_hit) break; }
                left = NULL;
            }
        } else left = NULL;
        if (hr) {
            if (right->leaf_count) {
                hit_geo = hit_geometries(tr, indices + right->first_index, right->leaf_count, s, rf, r, hit, any_hit);
                if (hit_geo >= 0) { closest_geo = hit_geo; if (any_hit) break; }
                right = NULL;
            }
        } else right = NULL;
        if (left) {
            if (right) {
                if (!any_hit && ln > rn) { const SlimBVHNode *tmp = left; left = right; right = tmp; }
                tr->scene_stack[top++] = right->first_index;
            }
            left = nodes + left->first_index;
        } else if (right) {
            left = nodes + right->first_index;
        } else {
            if (top == 0) break;
            left = nodes + tr->scene_stack[--top];
        }
    }
    return closest_geo;
}

static int sphere_tracer_hit(SphereTracer *st, v3 center, float radius, float one_over_radius,
                             v3 Ro, v3 Rd, float *max_distance) {                                  /* ray.h:317-336 */
    st->t_max = *max_distance * one_over_radius;
    v3 rc = vscale(vsub(center, Ro), one_over_radius);
    st->b = vdot(Rd, rc);
    st->c = vsqlen(rc) - 1;
    float h = st->b * st->b - st->c;
    if (h >= 0) {
        h = sqrtf(h);
        st->t_near = st->b - h;
        st->t_far = st->b + h;
        if (st->t_far > 0 && st->t_near < st->t_max) {
            *max_distance = st->t_max * radius;
            return 1;
        }
    }
    return 0;
}
static float sphere_tracer_density(const SphereTracer *st) {                                       /* ray.h:338-346 */
    float tn = MAXF(st->t_near, 0);
    float tf = MINF(st->t_far, st->t_max);
    float tn2 = tn * tn, tf2 = tf * tf;
    return (st->c * tn - st->b * tn2 + tn * tn2 / 3.0f - (st->c * tf - st->b * tf2 + tf * tf2 / 3.0f)) * (3.0f / 4.0f);
}

/* ---- textures: core/texture.h ------------------------------------------ */
static v3 mip_sample(const SlimTextureMip *mip, float u, float v, SlimWorkCounters *counters) {    /* texture.h:17-41 */
    if (counters) counters->texel_taps++;
    if (u > 1) u -= (float)((uint32_t)u);
    if (v > 1) v -= (float)((uint32_t)v);
    const float U = u * (float)mip->width + 0.5f;
    const float V = v * (float)mip->height + 0.5f;
    const uint32_t x = (uint32_t)U;
    const uint32_t y = (uint32_t)V;
    const float r = U - (float)x, b = V - (float)y;
    const float l = 1 - r, t = 1 - b;
    const float tl = t * l * COLOR_COMPONENT_TO_FLOAT_;
    const float tr = t * r * COLOR_COMPONENT_TO_FLOAT_;
    const float bl = b * l * COLOR_COMPONENT_TO_FLOAT_;
    const float br = b * r * COLOR_COMPONENT_TO_FLOAT_;
    const SlimTexelQuad q = mip->texel_quads[y * (mip->width + 1) + x];
    return V3(fmaf((float)q.R[3], br, fmaf((float)q.R[2], bl, fmaf((float)q.R[1], tr, (float)q.R[0] * tl))),
              fmaf((float)q.G[3], br, fmaf((float)q.G[2], bl, fmaf((float)q.G[1], tr, (float)q.G[0] * tl))),
              fmaf((float)q.B[3], br, fmaf((float)q.B[2], bl, fmaf((float)q.B[1], tr, (float)q.B[0] * tl))));
}
static uint32_t mip_level(float texel_area, uint32_t mip_count) {                                  /* texture.h:47-54 */
    uint32_t m = 0;
    while (texel_area > 1 && ++m < mip_count) texel_area *= 0.25f;
    if (m >= mip_count) m = mip_count - 1;
    return m;
}
static v3 texture_sample(const SlimTexture *t, float u, float v, float coverage, SlimWorkCounters *c) {  /* texture.h:68-70 */
    uint32_t m = (t->flags & SLIM_IMAGE_MIPMAP) ? mip_level(coverage * (float)(t->width * t->height), t->mip_count) : 0;
    return mip_sample(t->mips + m, u, v, c);
}
static v3 texture_sample_cube(const SlimTexture *t, float X, float Y, float Z, SlimWorkCounters *c) {  /* texture.h:72-116 */
    float u, v;
    int mip = 0;
    float right = signbit(X) ? 0.0f : 1.0f, left = signbit(X) ? 1.0f : 0.0f;
    float z_over_x = X ? (Z / X) : 2;
    float y_over_x = X ? (Y / X) : 2;
    if (z_over_x <= 1 && z_over_x >= -1 && y_over_x <= 1 && y_over_x >= -1) {
        u = fmaf(z_over_x, -0.125f, fmaf(0.5f, right, 0.125f));
        v = fmaf(y_over_x, left - 0.5f, 0.5f);
    } else {
        float x_over_z = Z ? (X / Z) : 2;
        float y_over_z = Z ? (Y / Z) : 2;
        float sz = signbit(Z) ? 1.0f : 0.0f;
        if (x_over_z <= 1 && x_over_z >= -1 && y_over_z <= 1 && y_over_z >= -1) {
            v = fmaf(y_over_z, sz - 0.5f, +0.5f);
            u = fmaf(x_over_z, 0.125f, fmaf(sz, 0.5f, 0.375f));
        } else {
            u = fmaf(X / fabsf(Y), 0.5f, 0.5f);
            v = fmaf(Z / Y, 0.5f, 0.5f);
            mip = 2 - !signbit(Y);
        }
    }
    return mip_sample(t->mips + mip, u, v, c);
}

/* ---- shading: renderer/surface_shader.h, scene/material.h --------------- */
typedef struct {
    int geometry;
    const SlimMaterial *material;
    v3 F, albedo_from_map, Fs, Fd;
    Ray shadow_ray;
    Hit shadow_hit;
    v3 P, N, V, L, R, RF, H, quad[4];
    float Ld, Ld2, NdotL, NdotV, NdotH, HdotL, IOR;
    int refracted;
} Shader;

static inline v3 mat_vec(const float *c) { return V3(c[0], c[1], c[2]); }
static v3 schlick_fresnel(float HdotL, v3 F0) {                                                     /* material.h:57-59 */
    float p = powf(1.0f - HdotL, 5.0f);
    return vadd(F0, vscale(V3(1.0f - F0.x, 1.0f - F0.y, 1.0f - F0.z), p));
}
static float ggx_d(float roughness, float NdotH) {                                                  /* material.h:27-36 */
    float a = roughness * roughness;
    float denom = NdotH * NdotH * (a - 1.0f) + 1.0f;
    return a / (PI_ * denom * denom);
}
static float ggx_g(float roughness, float NdotL, float NdotV) {                                     /* material.h:38-55 */
    float a = roughness * roughness;
    float k = a * 0.5f;
    float omk = 1.0f - k;
    float denom = fmaf(NdotV, omk, k);
    float result = NdotV / fmaxf(denom, EPS_);
    denom = fmaf(NdotL, omk, k);
    result *= NdotL / fmaxf(denom, EPS_);
    return result;
}
static v3 cook_torrance(float r, float NdotL, float NdotV, float HdotL, float NdotH, v3 F0, v3 *F) {  /* material.h:61-70 */
    *F = schlick_fresnel(HdotL, F0);
    float D = ggx_d(r, NdotH);
    float G = ggx_g(r, NdotL, NdotV);
    return vscale(*F, D * G / (4.0f * NdotL * NdotV));
}
static void radiance_fraction(Shader *sh) {                                                         /* surface_shader.h:109-145 */
    const SlimMaterial *m = sh->material;
    sh->Fs = V3(0, 0, 0);
    sh->Fd = vmul(mat_vec(m->albedo), sh->albedo_from_map);
    if (m->brdf == SLIM_BRDF_COOK_TORRANCE) {
        sh->Fd = vscale(sh->Fd, (1.0f - m->metalness) * ONE_OVER_PI_);
        if (sh->NdotV > 0.0f) {
            if (m->roughness > 0.0f) {
                sh->H = vnormalized(vadd(sh->L, sh->V));
                sh->NdotH = clamp01(vdot(sh->N, sh->H));
                sh->HdotL = clamp01(vdot(sh->H, sh->L));
                sh->Fs = cook_torrance(m->roughness, sh->NdotL, sh->NdotV, sh->HdotL, sh->NdotH, mat_vec(m->reflectivity), &sh->F);
                sh->Fd = vmul(sh->Fd, V3(1.0f - sh->F.x, 1.0f - sh->F.y, 1.0f - sh->F.z));
            }
        }
    } else {
        sh->Fd = vscale(sh->Fd, m->roughness * ONE_OVER_PI_);
        if (m->brdf != SLIM_BRDF_LAMBERT) {
            float spec, exponent;
            if (m->brdf == SLIM_BRDF_PHONG) {
                exponent = 4.0f;
                spec = clamp01(vdot(sh->R, sh->L));
            } else {
                exponent = 16.0f;
                spec = clamp01(vdot(sh->N, vnormalized(vadd(sh->L, sh->V))));
            }
            if (spec > 0.0f) sh->Fs = vscale(mat_vec(m->reflectivity), powf(spec, exponent) * (1.0f - m->roughness));
        }
    }
}

static v3 rotate_normal(v3 normal, v3 sample, float magnitude) {                                   /* material.h:83-86 */
    v3 N = vnormalized(V3(fmaf(sample.x, 2.0f, -1.0f), fmaf(sample.z, 2.0f, -1.0f), fmaf(sample.y, 2.0f, -1.0f)));
    quat_ q = qaxisangle(vnormalized(V3(N.z, 0, -N.x)), acosf(N.y) * magnitude);
    return qrot(q, normal);
}
static v3 sample_slot(const SlimMaterial *m, int slot, const SlimTexture *textures, v2 uv, float coverage,
                      SlimWorkCounters *c) {                                                         /* surface_shader.h:9-11 */
    return (textures && m->texture_count > slot)
        ? texture_sample(textures + m->texture_ids[slot], uv.u, uv.v, coverage, c) : V3(0, 0, 0);
}

typedef struct {
    const SlimSceneData *scene;
    const SlimCameraRayProjection *proj;
    const SlimRayTracerSettings *settings;
    int cones_per_pixel;   /* 0: reference semantics (aux-hit scaling factor) */
} Frame;

static void prepare_for_shading(Shader *sh, const Frame *fr, Ray *ray, Hit *hit, float pixel_scaling,
                                SlimWorkCounters *c) {                                               /* surface_shader.h:61-107 */
    const SlimSceneData *s = fr->scene;
    const SlimGeometry *geo = s->geometries + sh->geometry;
    const SlimMaterial *mat = s->materials + geo->material_id;
    v2 rep = {mat->uv_repeat.x, mat->uv_repeat.y};
    hit->uv.u *= rep.u;
    hit->uv.v *= rep.v;
    if (hit->from_behind) hit->normal = vneg(hit->normal);
    float scaling = fr->cones_per_pixel ? pixel_scaling : hit->scaling_factor;
    hit->cone_width = hit->distance * scaling;
    hit->cone_width *= hit->cone_width;
    hit->cone_width *= hit->cone_width;
    v3 scale = V3(geo->transform.scale.x, geo->transform.scale.y, geo->transform.scale.z);
    hit->uv_coverage *= hit->cone_width / (rep.u * rep.v * hit->NdotRd *
                                           fabsf(vdot(V3(1.0f - hit->normal.x, 1.0f - hit->normal.y, 1.0f - hit->normal.z), scale)));
    hit->position = ray_at(ray, hit->distance);
    quat_ rot = {V3(geo->transform.orientation.axis.x, geo->transform.orientation.axis.y, geo->transform.orientation.axis.z),
                 geo->transform.orientation.amount};
    hit->normal = vnormalized(qrot(rot, vmul(scale, hit->normal)));
    sh->material = mat;
    int has_maps = mat->texture_count != 0;
    if (has_maps && (mat->flags & SLIM_MATERIAL_HAS_NORMAL_MAP))
        hit->normal = rotate_normal(hit->normal, sample_slot(mat, 1, s->textures, hit->uv, hit->uv_coverage, c), mat->normal_magnitude);
    sh->P = hit->position;
    sh->N = hit->normal;
    sh->R = sh->RF = vreflect(ray->direction, sh->N);
    sh->V = vneg(ray->direction);
    sh->NdotV = clamp01(vdot(sh->N, sh->V));
    sh->albedo_from_map = (has_maps && (mat->flags & SLIM_MATERIAL_HAS_ALBEDO_MAP))
        ? sample_slot(mat, 0, s->textures, hit->uv, hit->uv_coverage, c) : V3(1, 1, 1);
    sh->refracted = (mat->flags & SLIM_MATERIAL_IS_REFRACTIVE) != 0;
    if (sh->refracted) {
        sh->IOR = hit->from_behind ? (mat->IOR / IOR_AIR_) : (IOR_AIR_ / mat->IOR);
        float cc = sh->IOR * sh->IOR * (1.0f - (sh->NdotV * sh->NdotV));
        sh->refracted = cc < 1.0f;
        if (sh->refracted)
            sh->RF = vnormalized(vscaleadd(sh->N, sh->IOR * sh->NdotV - sqrtf(1 - cc), vscale(ray->direction, sh->IOR)));
    }
}

static int is_facing_light(Shader *sh, const SlimLight *light) {                                   /* surface_shader.h:147-160 */
    v3 pod = V3(light->position_or_direction.x, light->position_or_direction.y, light->position_or_direction.z);
    if (light->flags & SLIM_LIGHT_IS_DIRECTIONAL) {
        sh->Ld = INFINITY;
        sh->Ld2 = 1.0f;
        sh->L = vneg(pod);
    } else {
        sh->L = vsub(pod, sh->P);
        sh->Ld2 = vsqlen(sh->L);
        sh->Ld = sqrtf(sh->Ld2);
        sh->L = vdivs(sh->L, sh->Ld);
    }
    sh->NdotL = clamp01(vdot(sh->L, sh->N));
    return sh->NdotL > 0.0f;
}

static void shade_from_light(Shader *sh, Tracer *tr, const Frame *fr, const SlimLight *light, v3 *color) {  /* surface_shader.h:49-59 */
    if (!is_facing_light(sh, light)) return;
    if (light->flags & SLIM_LIGHT_IS_SHADOWING) {
        sh->shadow_ray.origin = sh->P;
        sh->shadow_ray.direction = sh->L;
        COUNT(shadow_rays);
        if (scene_trace(tr, &sh->shadow_ray, &sh->shadow_hit, fr->scene, 1, sh->Ld) >= 0) return;
    }
    radiance_fraction(sh);
    v3 lc = vscale(mat_vec(light->color), sh->NdotL * light->intensity / sh->Ld2);
    *color = vmuladd(vadd(sh->Fs, sh->Fd), lc, *color);
}

static v3 area_light_vector(Shader *sh, const SlimTransform *t) {                                  /* surface_shader.h:162-186 */
    const float sx = t->scale.x, sz = t->scale.z;
    if (sx == 0 || sz == 0) return V3(0, 0, 0);
    quat_ q = {V3(t->orientation.axis.x, t->orientation.axis.y, t->orientation.axis.z), t->orientation.amount};
    v3 U = qrot(q, V3(sx < 0 ? -sx : sx, 0.0f, 0.0f));
    v3 Vv = qrot(q, V3(0.0f, 0.0f, sz < 0 ? -sz : sz));
    v3 p = V3(t->position.x, t->position.y, t->position.z);
    sh->quad[0] = vsub(vsub(p, U), Vv);
    sh->quad[1] = vsub(vadd(p, U), Vv);
    sh->quad[2] = vadd(vadd(p, U), Vv);
    sh->quad[3] = vadd(vsub(p, U), Vv);
    v3 u1 = vnormalized(vsub(sh->quad[0], sh->P));
    v3 u2 = vnormalized(vsub(sh->quad[1], sh->P));
    v3 u3 = vnormalized(vsub(sh->quad[2], sh->P));
    v3 u4 = vnormalized(vsub(sh->quad[3], sh->P));
    return vadd(vadd(vadd(vscale(vcross(u1, u2), acosf(vdot(u1, u2)) * 0.5f),
                          vscale(vcross(u2, u3), acosf(vdot(u2, u3)) * 0.5f)),
                     vscale(vcross(u3, u4), acosf(vdot(u3, u4)) * 0.5f)),
                vscale(vcross(u4, u1), acosf(vdot(u4, u1)) * 0.5f));
}

static void shade_from_emissive_quads(Shader *sh, const Frame *fr, v3 *color) {                    /* surface_shader.h:188-264 */
    const SlimSceneData *s = fr->scene;
    float sq_to_center = 0;
    for (uint32_t i = 0; i < s->counts.geometries; i++) {
        const SlimGeometry *eq = s->geometries + i;
        if ((int)i == sh->geometry || eq->type != SLIM_GEOMETRY_QUAD ||
            !(s->materials[eq->material_id].flags & SLIM_MATERIAL_IS_EMISSIVE)) continue;
        const SlimTransform *xf = &eq->transform;
        sh->L = vsub(V3(xf->position.x, xf->position.y, xf->position.z), sh->P);
        sh->NdotL = vdot(sh->N, sh->L);
        if (sh->NdotL <= 0.0f) continue;
        sh->Ld2 = vsqlen(sh->L);
        sh->Ld = sqrtf(sh->Ld2);
        float Ld_rcp = 1.0f / sh->Ld;
        sh->L = vscale(sh->L, Ld_rcp);
        sh->NdotL *= Ld_rcp;
        v3 Ro = vscaleadd(sh->L, TRACE_OFFSET_, sh->P);
        ray_localize(&sh->shadow_ray, Ro, sh->L, xf);
        sh->shadow_hit.distance = INFINITY;
        sh->shadow_ray.direction = vnormalized(sh->shadow_ray.direction);
        ray_hits_quad(&sh->shadow_ray, &sh->shadow_hit, (eq->flags & SLIM_GEOMETRY_IS_TRANSPARENT) != 0);
        float ei = vdot(sh->N, area_light_vector(sh, xf));
        if (ei > 0) {
            int skip = 1;
            for (int k = 0; k < 4; k++)
                if (vdot(sh->N, vsub(sh->quad[k], sh->P)) >= 0) { skip = 0; break; }
            if (skip) continue;
            float shaded = 1.0f;
            for (uint32_t j = 0; j < s->counts.geometries; j++) {
                if (j == i || (int)j == sh->geometry) continue;
                const SlimGeometry *sg = s->geometries + j;
                ray_localize(&sh->shadow_ray, Ro, sh->L, &sg->transform);
                sh->shadow_hit.distance = INFINITY;
                sh->shadow_ray.direction = vnormalized(sh->shadow_ray.direction);
                float d = 1.0f;
                int tr_ = (sg->flags & SLIM_GEOMETRY_IS_TRANSPARENT) != 0;
                if (sg->type == SLIM_GEOMETRY_SPHERE) {
                    if (ray_hits_sphere(&sh->shadow_ray, &sh->shadow_hit, tr_, &sq_to_center))
                        d -= (1.0f - sqrtf(sq_to_center)) / (sh->shadow_hit.distance * ei * 3.0f);
                } else if (sg->type == SLIM_GEOMETRY_QUAD) {
                    if (ray_hits_quad(&sh->shadow_ray, &sh->shadow_hit, tr_)) {
                        float ax = fabsf(sh->shadow_hit.position.x), az = fabsf(sh->shadow_hit.position.z);
                        d -= 3.0f * (1.0f - MAXF(ax, az)) / (sh->shadow_hit.distance * ei);
                    }
                }
                shaded = MINF(shaded, d);
            }
            if (shaded > 0.0f) {
                radiance_fraction(sh);
                v3 e = vscale(mat_vec(s->materials[eq->material_id].emission), ei * shaded * 7.0f);
                *color = vmuladd(vadd(sh->Fd, sh->Fs), e, *color);
            }
        }
    }
}

static float tone_mapped_baked(float c) {                                                          /* base.h:777-786 */
    float x = c - 0.004f;
    if (x < 0.0f) x = 0.0f;
    float x2s = x * x * 6.2f;
    return (x2s + x * 0.5f) / (x2s + x * 1.7f + 0.06f);
}
static v3 color_of_id(int id) {                                                                    /* base.h:806-855 */
    switch (id) {
        case 1: return V3(1, 1, 1);
        case 2: return V3(0.5f, 0.5f, 0.5f);
        case 3: return V3(1, 0, 0);
        case 4: return V3(0, 1, 0);
        case 5: return V3(0, 0, 1);
        case 6: return V3(0, 1, 1);
        case 7: return V3(1, 0, 1);
        case 8: return V3(1, 1, 0);
        case 9: return V3(0.5f, 0, 0);
        case 10: return V3(0, 0.5f, 0);
        case 11: return V3(0, 0, 0.5f);
        case 12: return V3(0.25f, 0.25f, 0.25f);
        case 13: return V3(1, 0.5f, 0.5f);
        case 14: return V3(0.5f, 1, 0.5f);
        case 15: return V3(0.5f, 0.5f, 1);
        case 16: return V3(0.75f, 0.75f, 0.75f);
        case 17: return V3(0, 0.75f, 0.75f);
        case 18: return V3(0.75f, 0, 0.75f);
        case 19: return V3(0.75f, 0.75f, 0);
        case 20: return V3(0, 0.5f, 0.5f);
        case 21: return V3(0.5f, 0, 0.5f);
        case 22: return V3(0.5f, 0.5f, 0);
        case 23: return V3(0.04f, 0.04f, 0.04f);
        case 24: return V3(0.02f, 0.02f, 0.02f);
        case 25: return V3(0.03f, 0.03f, 0.03f);
        case 26: return V3(0.08f, 0.08f, 0.08f);
        case 27: return V3(0.03f, 0.03f, 0.03f);
        case 28: return V3(0.05f, 0.05f, 0.05f);
        case 29: return V3(0.08f, 0.08f, 0.08f);
        case 30: return V3(0.17f, 0.17f, 0.17f);
        case 31: return V3(0.56f, 0.57f, 0.58f);
        case 32: return V3(0.95f, 0.64f, 0.54f);
        case 33: return V3(1.0f, 0.71f, 0.29f);
        case 34: return V3(0.91f, 0.92f, 0.92f);
        case 35: return V3(0.95f, 0.93f, 0.88f);
        default: return V3(0, 0, 0);
    }
}

/* renderPixelBeauty / renderPixelDebugMode (renderer/ray_tracer.h:19-142). */
static void render_pixel(const Frame *fr, Tracer *tr, Shader *sh, Ray *ray, Hit *hit, v3 direction,
                         float pixel_scaling, v3 *out_color, float *out_depth) {
    const SlimSceneData *s = fr->scene;
    const SlimRayTracerSettings *st = fr->settings;
    const SlimCameraRayProjection *pj = fr->proj;
    v3 color = V3(0, 0, 0);
    float depth = INFINITY;
    v3 cam = V3(pj->camera_position.x, pj->camera_position.y, pj->camera_position.z);
    ray_reset(ray, cam, vnormalized(direction));
    if (tr->counters) tr->counters->primary_rays++;
    if (st->render_mode != SLIM_RENDER_BEAUTY) {
        int g = scene_trace(tr, ray, hit, s, 0, INFINITY);
        if (g >= 0) {
            sh->geometry = g;
            prepare_for_shading(sh, fr, ray, hit, pixel_scaling, tr->counters);
            depth = mat3_mul(pj->inverted_camera_rotation, vsub(hit->position, cam)).z;
            switch (st->render_mode) {
                case SLIM_RENDER_UVS: color = V3(hit->uv.u, hit->uv.v, 1.0f); break;
                case SLIM_RENDER_DEPTH: { float d = 4.0f / hit->distance; color = V3(d, d, d); } break;
                case SLIM_RENDER_NORMALS:
                    color = V3(fmaf(hit->normal.x, 0.5f, 0.5f), fmaf(hit->normal.y, 0.5f, 0.5f), fmaf(hit->normal.z, 0.5f, 0.5f));
                    break;
                case SLIM_RENDER_NORMAL_MAP: {
                    v3 n = sample_slot(sh->material, 1, s->textures, hit->uv, hit->uv_coverage, tr->counters);
                    color = V3(fmaf(n.x, 0.5f, 0.5f), fmaf(n.y, 0.5f, 0.5f), fmaf(n.z, 0.5f, 0.5f));
                } break;
                case SLIM_RENDER_MIP_LEVEL:
                    if (s->counts.textures) {
                        const SlimTexture *t0 = s->textures;
                        color = color_of_id(st->mip_level_colors[mip_level(hit->uv_coverage * (float)(t0->width * t0->height), t0->mip_count)]);
                    } else color = V3(0.5f, 0.5f, 0.5f);
                    break;
                default: break;
            }
        }
        *out_color = color;
        *out_depth = depth;
        return;
    }
    v3 current, next_throughput = V3(0, 0, 0), throughput = V3(1, 1, 1);
    uint32_t depth_left = st->max_depth;
    while (depth_left) {
        current = V3(0, 0, 0);
        int g = scene_trace(tr, ray, hit, s, 0, INFINITY);
        if (g >= 0) {
            sh->geometry = g;
            const SlimGeometry *geo = s->geometries + g;
            const SlimMaterial *mat = s->materials + geo->material_id;
            sh->material = mat;
            if ((mat->flags & SLIM_MATERIAL_IS_EMISSIVE) && geo->type == SLIM_GEOMETRY_QUAD && !hit->from_behind) {
                depth_left = 0;
                current = mat_vec(mat->emission);
            } else {
                prepare_for_shading(sh, fr, ray, hit, pixel_scaling, tr->counters);
                if (depth_left == st->max_depth) depth = mat3_mul(pj->inverted_camera_rotation, vsub(hit->position, cam)).z;
                if (s->lights)
                    for (uint32_t i = 0; i < s->counts.lights; i++) shade_from_light(sh, tr, fr, s->lights + i, &current);
                if (s->flags & SLIM_SCENE_HAD_EMISSIVE_QUADS) shade_from_emissive_quads(sh, fr, &current);
                if (st->skybox_irradiance_texture_id >= 0 && st->skybox_radiance_texture_id >= 0) {
                    sh->L = sh->N;
                    sh->NdotL = 1.0f;
                    v3 D = texture_sample_cube(s->textures + st->skybox_irradiance_texture_id, sh->N.x, sh->N.y, sh->N.z, tr->counters);
                    v3 S = texture_sample_cube(s->textures + st->skybox_radiance_texture_id, sh->R.x, sh->R.y, sh->R.z, tr->counters);
                    radiance_fraction(sh);
                    current = vmuladd(D, sh->Fd, vmuladd(sh->Fs, S, current));
                }
                if ((mat->flags & (SLIM_MATERIAL_IS_REFLECTIVE | SLIM_MATERIAL_IS_REFRACTIVE)) && --depth_left) {
                    sh->F = schlick_fresnel(clamp01(vdot(sh->N, sh->R)), mat_vec(mat->reflectivity));
                    next_throughput = sh->refracted ? V3(1.0f - sh->F.x, 1.0f - sh->F.y, 1.0f - sh->F.z) : sh->F;
                    ray_reset(ray, hit->position, sh->RF);
                    if (tr->counters) tr->counters->bounce_rays++;
                } else depth_left = 0;
            }
        } else {
            depth_left = 0;
            if (st->skybox_color_texture_id >= 0)
                current = texture_sample_cube(s->textures + st->skybox_color_texture_id, ray->direction.x, ray->direction.y,
                                              ray->direction.z, tr->counters);
        }
        if (s->lights)
            for (uint32_t i = 0; i < s->counts.lights; i++) {
                const SlimLight *l = s->lights + i;
                if (!(l->flags & SLIM_LIGHT_IS_DIRECTIONAL) &&
                    sphere_tracer_hit(&tr->light, V3(l->position_or_direction.x, l->position_or_direction.y, l->position_or_direction.z),
                                      l->intensity * LIGHT_INTENSITY_RADIUS_FACTOR_, LIGHT_RADIUS_INTENSITY_FACTOR_ / l->intensity,
                                      ray->origin, ray->direction, &hit->distance))
                    current = vscaleadd(mat_vec(l->color), powf(sphere_tracer_density(&tr->light), 8.0f) * 4, current);
            }
        color = vmuladd(current, throughput, color);
        throughput = vmul(throughput, next_throughput);
    }
    color = V3(tone_mapped_baked(color.x), tone_mapped_baked(color.y), tone_mapped_baked(color.z));
    *out_color = color;
    *out_depth = depth;
}

/* Canvas::setPixel(x, y, color, -1, depth) (draw/canvas.h:128-165). */
static void set_pixel(const SlimCanvasData *cv, int x, int y, v3 c, float depth) {
    int w = cv->dimensions.width, h = cv->dimensions.height;
    if (cv->antialias == SLIM_AA_SSAA) { w <<= 1; h <<= 1; }
    if (x < 0 || y < 0 || x >= w || y >= h) return;
    c = V3(clamp01(c.x), clamp01(c.y), clamp01(c.z));
    c = vmul(c, vscale(c, 1.0f));
    uint32_t offset = cv->antialias == SLIM_AA_SSAA
        ? ((cv->dimensions.stride * (uint32_t)(y >> 1) + (uint32_t)(x >> 1)) * 4 + 2 * (uint32_t)(y & 1) + (uint32_t)(x & 1))
        : (cv->dimensions.stride * (uint32_t)y + (uint32_t)x);
    SlimPixel *px = cv->pixels + offset;
    px->r = c.x; px->g = c.y; px->b = c.z; px->opacity = 1.0f;
    float *dp = cv->depths + (cv->antialias == SLIM_AA_MSAA ? offset * 4 : offset);
    dp[0] = depth;
    if (cv->antialias == SLIM_AA_MSAA) dp[1] = dp[2] = dp[3] = 0;
}

/* ---- C ABI --------------------------------------------------------------- */
int oracle_abi_version(void) { return 1; }

/* Renders rows [row_begin, row_end) of the sample grid the way d_render
 * does per pixel (renderer/renderer_GPU.h:22-46).  counters may be NULL. */
int oracle_render(const SlimSceneData *scene, const SlimCanvasData *canvas, const SlimCameraRayProjection *proj,
                  const SlimRayTracerSettings *settings, int row_begin, int row_end, int cones_per_pixel,
                  SlimWorkCounters *counters) {
    if (!scene || !canvas || !proj || !settings) return SLIM_ERR_ARGUMENT;
    Frame fr = {scene, proj, settings, cones_per_pixel};
    int s = canvas->antialias == SLIM_AA_SSAA ? 2 : 1;
    int width = canvas->dimensions.width * s, height = canvas->dimensions.height * s;
    if (row_end > height) row_end = height;
    Tracer *tr = (Tracer*)malloc(sizeof(Tracer));
    Shader *sh = (Shader*)malloc(sizeof(Shader));
    if (!tr || !sh) { free(tr); free(sh); return SLIM_ERR_LIMIT; }
    v3 start = V3(proj->start.x, proj->start.y, proj->start.z);
    v3 down = V3(proj->down.x, proj->down.y, proj->down.z);
    v3 right = V3(proj->right.x, proj->right.y, proj->right.z);
    for (int y = row_begin < 0 ? 0 : row_begin; y < row_end; y++)
        for (int x = 0; x < width; x++) {
            Ray ray; Hit hit; v3 color; float depth;
            memset(tr, 0, sizeof(Tracer)); memset(sh, 0, sizeof(Shader));
            memset(&ray, 0, sizeof(ray)); memset(&hit, 0, sizeof(hit));
            tr->aux_hit.uv.u = tr->aux_hit.uv.v = 1.0f;
            tr->triangle_hit.uv.u = tr->triangle_hit.uv.v = 1.0f;
            tr->counters = counters;
            /* getRayDirectionAt (scene/camera.h:67): start + down*y + right*x */
            v3 dir = vadd(vadd(start, vscale(down, (float)y)), vscale(right, (float)x));
            float cx = fmaf((float)x, proj->sample_size, proj->C_start.x);
            float cy = fmaf((float)-y, proj->sample_size, proj->C_start.y);
            float pixel_scaling = 1.0f / sqrtf(proj->squared_distance_to_projection_plane + (cx * cx + cy * cy));
            hit.scaling_factor = pixel_scaling;
            render_pixel(&fr, tr, sh, &ray, &hit, dir, pixel_scaling, &color, &depth);
            set_pixel(canvas, x, y, color, depth);
            if (counters) counters->pixels++;
        }
    free(tr); free(sh);
    return SLIM_OK;
}

/* First closest hit of each primary ray (renderer/ray_tracer.h:36-45) of
 * rows [row_begin, row_end); outputs are indexed y * width + x. */
int oracle_trace_primary_rows(const SlimSceneData *scene, const SlimCameraRayProjection *proj, int width,
                              int row_begin, int row_end, int32_t *geometry_ids, uint32_t *primitive_ids,
                              float *distances, uint8_t *from_behind) {
    Tracer *tr = (Tracer*)calloc(1, sizeof(Tracer));
    if (!tr) return SLIM_ERR_LIMIT;
    v3 start = V3(proj->start.x, proj->start.y, proj->start.z);
    v3 down = V3(proj->down.x, proj->down.y, proj->down.z);
    v3 right = V3(proj->right.x, proj->right.y, proj->right.z);
    v3 cam = V3(proj->camera_position.x, proj->camera_position.y, proj->camera_position.z);
    for (int y = row_begin; y < row_end; y++)
        for (int x = 0; x < width; x++) {
            Ray ray; Hit hit;
            memset(tr, 0, sizeof(Tracer)); memset(&ray, 0, sizeof(ray)); memset(&hit, 0, sizeof(hit));
            v3 dir = vadd(vadd(start, vscale(down, (float)y)), vscale(right, (float)x));
            ray_reset(&ray, cam, vnormalized(dir));
            int g = scene_trace(tr, &ray, &hit, scene, 0, INFINITY);
            size_t o = (size_t)y * (size_t)width + (size_t)x;
            geometry_ids[o] = g;
            primitive_ids[o] = (g >= 0 && scene->geometries[g].type == SLIM_GEOMETRY_MESH) ? hit.id : 0;
            distances[o] = g >= 0 ? hit.distance : INFINITY;
            from_behind[o] = g >= 0 ? (uint8_t)hit.from_behind : 0;
        }
    free(tr);
    return SLIM_OK;
}

int oracle_trace_primary(const SlimSceneData *scene, const SlimCameraRayProjection *proj, int width, int height,
                         int32_t *geometry_ids, uint32_t *primitive_ids, float *distances, uint8_t *from_behind) {
    return oracle_trace_primary_rows(scene, proj, width, 0, height, geometry_ids, primitive_ids, distances,
                                     from_behind);
}
