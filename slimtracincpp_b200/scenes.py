"""Seeded synthetic scenes for the workloads the trace path is measured on.

There is no public dataset: every scene is generated from a seed with the
shapes, sizes and value ranges of the workload it stands for.

  config 1  implicit scene, 640x360, depth 1: 20x20 quad floor, 3 spheres,
            2 boxes, 1 tetrahedron, Lambert/Blinn/Phong, 2 point lights.
  config 2  mesh PBR scene, 1920x1080, depth 2: an icosphere (6 subdivisions,
            81,920 triangles, smooth normals) and a 256x256 value-noise
            heightfield (130,050 triangles), 8 instances, Cook-Torrance,
            4 point lights and 1 emissive quad area light.
  config 3  config 1 plus 4 glass spheres and 2 mirror quads, value-noise
            albedo and normal textures, sky cube maps, 1920x1080, depth 8.
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

from . import layout as L
from .scene import Camera, MeshAsset, Scene, TextureAsset, geometry, light, quat_y

ROOT = Path(__file__).resolve().parent.parent
ASSET_CACHE = Path(os.environ.get("SLIM_ASSET_CACHE", ROOT / "_build" / "assets"))

TET_MAX = np.float32(0.577350259)


# ---- procedural meshes ----------------------------------------------------
def icosphere(subdivisions: int):
    """Unit icosphere: positions, triangle indices facing outwards, smooth
    normals = normalised positions."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.array(verts, np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(faces, np.int64)
    for _ in range(subdivisions):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.minimum(edges[:, 0], edges[:, 1]) * len(v) + np.maximum(edges[:, 0], edges[:, 1])
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // len(v), uniq % len(v)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        m = inv.reshape(3, -1).T + base   # midpoints of edges (0,1), (1,2), (2,0)
        f = np.concatenate([
            np.stack([f[:, 0], m[:, 0], m[:, 2]], 1),
            np.stack([f[:, 1], m[:, 1], m[:, 0]], 1),
            np.stack([f[:, 2], m[:, 2], m[:, 1]], 1),
            np.stack([m[:, 0], m[:, 1], m[:, 2]], 1)])
    pos = v.astype(np.float32)
    # The reference's triangle normal is (v3 - v1) x (v2 - v1)
    # (scene/bvh_builder.h:315-319): clockwise seen from the front.
    return pos, f[:, [0, 2, 1]].astype(np.uint32), pos.copy()


def value_noise_2d(rng, n, cells, octaves=4):
    """Seeded value noise on an n x n grid in [0, 1]: smoothstep-interpolated
    random lattices, `octaves` octaves of halving amplitude."""
    out = np.zeros((n, n), np.float64)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        c = cells * (2 ** o)
        lattice = rng.random((c + 1, c + 1))
        x = np.linspace(0, c, n, endpoint=False) if o else np.linspace(0, c, n)
        i = np.minimum(x.astype(np.int64), c - 1)
        f = x - i
        s = f * f * (3 - 2 * f)
        row0 = lattice[i][:, i] * (1 - s)[None, :] + lattice[i][:, i + 1] * s[None, :]
        row1 = lattice[i + 1][:, i] * (1 - s)[None, :] + lattice[i + 1][:, i + 1] * s[None, :]
        out += amp * (row0 * (1 - s)[:, None] + row1 * s[:, None])
        total += amp
        amp *= 0.5
    return out / total


def heightfield(rng, n=256, amplitude=0.3):
    """n x n grid over [-1, 1]^2 displaced in y by value noise of the given
    amplitude; smooth area-weighted vertex normals."""
    h = (value_noise_2d(rng, n, 8) - 0.5) * 2.0 * amplitude
    xs = np.linspace(-1.0, 1.0, n)
    X, Z = np.meshgrid(xs, xs, indexing="xy")
    pos = np.stack([X, h, Z], -1).reshape(-1, 3)
    idx = np.arange(n * n).reshape(n, n)
    a, b, c, d = idx[:-1, :-1], idx[:-1, 1:], idx[1:, :-1], idx[1:, 1:]
    # winding so the geometric normal faces +y
    t1 = np.stack([a, c, b], -1).reshape(-1, 3)
    t2 = np.stack([b, c, d], -1).reshape(-1, 3)
    tris = np.concatenate([t1, t2])
    fn = np.cross(pos[tris[:, 1]] - pos[tris[:, 0]], pos[tris[:, 2]] - pos[tris[:, 0]])
    vn = np.zeros_like(pos)
    for k in range(3):
        np.add.at(vn, tris[:, k], fn)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    if vn[:, 1].mean() < 0:
        vn = -vn
    # clockwise seen from +y, the reference's front (see icosphere)
    return pos.astype(np.float32), tris[:, [0, 2, 1]].astype(np.uint32), vn.astype(np.float32)


def cached_mesh(name, builder):
    """Builds a mesh asset once per machine and reuses its .mesh file (read
    and written by this library; a caller-supplied mesh builder builds it
    afresh instead)."""
    from .scene import HOST_BUILDERS
    if "mesh" in HOST_BUILDERS:
        pos, idx, nrm = builder()
        return MeshAsset.build(pos, idx, normals=nrm, normal_indices=idx)
    ASSET_CACHE.mkdir(parents=True, exist_ok=True)
    path = ASSET_CACHE / f"{name}.mesh"
    if path.exists():
        try:
            return MeshAsset.load(path)
        except Exception:
            path.unlink()
    pos, idx, nrm = builder()
    mesh = MeshAsset.build(pos, idx, normals=nrm, normal_indices=idx)
    tmp = path.with_suffix(".mesh.tmp")
    mesh.save(tmp)
    os.replace(tmp, path)
    return mesh


def random_quat(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    return tuple(np.float32(x) for x in q[:3]), np.float32(q[3])


# ---- configs ---------------------------------------------------------------
class Workload:
    def __init__(self, name, scene, camera, width, height, settings, antialias=L.AA_NONE):
        self.name, self.scene, self.camera = name, scene, camera
        self.width, self.height, self.settings, self.antialias = width, height, settings, antialias

    @property
    def samples(self):
        s = 2 if self.antialias == L.AA_SSAA else 1
        return self.width * self.height * s * s

    def projection(self):
        return self.camera.projection(self.width, self.height, self.antialias == L.AA_SSAA)


def _implicit_objects(rng, materials):
    """config 1's objects: 3 spheres, 2 boxes, 1 tetrahedron resting on the
    floor at random positions, random Y rotation, Lambert/Blinn/Phong."""
    geos = []
    shapes = [L.GEOMETRY_SPHERE] * 3 + [L.GEOMETRY_BOX] * 2 + [L.GEOMETRY_TET]
    for kind in shapes:
        brdf = int(rng.integers(0, 3))   # Lambert, Blinn, Phong
        _shininess = rng.uniform(4, 128)  # no slot in the reference's Material (exponents are fixed)
        mat = L.default_material(albedo=0, roughness=float(rng.uniform(0.2, 0.8)), brdf=brdf,
                                 reflectivity=float(rng.uniform(0.2, 1.0)))
        mat["albedo"] = rng.uniform(0, 1, 3).astype(np.float32)
        materials.append(mat)
        mid = len(materials) - 1
        x, z = rng.uniform(-5, 5, 2)
        if kind == L.GEOMETRY_SPHERE:
            r = np.float32(rng.uniform(0.5, 1.5))
            geos.append(geometry(kind, mid, (x, r, z), (r, r, r)))
        else:
            s = np.float32(rng.uniform(0.5, 2.0))
            axis, amount = quat_y(rng.uniform(0, 2 * np.pi))
            y = s if kind == L.GEOMETRY_BOX else np.float32(s * TET_MAX)
            geos.append(geometry(kind, mid, (x, y, z), (s, s, s), axis, amount))
    return geos


def config1(seed=0, width=640, height=360):
    rng = np.random.default_rng(seed)
    materials = [L.default_material(albedo=0.8, roughness=0.8, brdf=L.BRDF_LAMBERT)]
    geos = [geometry(L.GEOMETRY_QUAD, 0, (0, 0, 0), (10, 1, 10))]
    geos += _implicit_objects(rng, materials)
    lights = [light(rng.uniform(0.5, 1.0, 3), (rng.uniform(-5, 5), rng.uniform(3, 6), rng.uniform(-5, 5)),
                    rng.uniform(5, 20)) for _ in range(2)]
    scene = Scene(np.array(geos), np.array(materials), np.array(lights))
    cam = Camera.look_at((0.0, 6.0, -14.0), (0.0, 0.5, 0.0), 60.0)
    return Workload("config1_implicit_640x360_d1", scene, cam, width, height, L.default_settings(max_depth=1))


def config2_meshes():
    ico = cached_mesh("icosphere6", lambda: icosphere(6))
    hf = cached_mesh("heightfield256_s7", lambda: heightfield(np.random.default_rng(7), 256, 0.3))
    return [ico, hf]


def config2(seed=0, width=1920, height=1080, meshes=None):
    rng = np.random.default_rng(seed)
    meshes = meshes if meshes is not None else config2_meshes()
    materials, geos = [], []
    for i in range(8):
        metallic = int(rng.integers(0, 2))
        mat = L.default_material(albedo=0, roughness=float(rng.uniform(0.05, 1.0)), brdf=L.BRDF_COOK_TORRANCE,
                                 reflectivity=0.04, metalness=float(metallic),
                                 flags=L.MATERIAL_IS_REFLECTIVE if metallic else 0)
        mat["albedo"] = rng.uniform(0.2, 1.0, 3).astype(np.float32)
        materials.append(mat)
        axis, amount = random_quat(rng)
        s = np.float32(rng.uniform(0.5, 3.0))
        # a jittered 4 x 2 layout keeps the instances spread over the frame
        col, row = i % 4, i // 4
        pos = (-6.0 + 4.0 * col + rng.uniform(-1, 1), rng.uniform(0.5, 3.0), -2.0 + 4.5 * row + rng.uniform(-1, 1))
        geos.append(geometry(L.GEOMETRY_MESH, i, pos, (s, s, s), axis, amount, mesh_id=i % 2))
    materials.append(L.default_material(albedo=0, roughness=0, flags=L.MATERIAL_IS_EMISSIVE, emission=(1.0, 0.9, 0.8)))
    # quad normal +y rotated 180 degrees about X: the area light faces down
    geos.append(geometry(L.GEOMETRY_QUAD, len(materials) - 1, (0, 9, 1), (5, 1, 5), (1, 0, 0), 0.0,
                         flags=L.GEOMETRY_IS_VISIBLE))
    lights = [light(rng.uniform(0.6, 1.0, 3), (rng.uniform(-8, 8), rng.uniform(4, 8), rng.uniform(-8, 2)),
                    rng.uniform(20, 60)) for _ in range(4)]
    scene = Scene(np.array(geos), np.array(materials), np.array(lights), meshes=meshes)
    cam = Camera.look_at((0.0, 6.0, -11.0), (0.0, 1.0, 1.5), 60.0)
    return Workload("config2_mesh_pbr_1920x1080_d2", scene, cam, width, height, L.default_settings(max_depth=2))


def small_mesh_scene(seed=0, width=160, height=90, subdivisions=2, grid=16):
    """A config-2-shaped scene with small meshes, sized for the oracle."""
    rng = np.random.default_rng(seed)
    meshes = [MeshAsset.build(*_with_normals(icosphere(subdivisions))),
              MeshAsset.build(*_with_normals(heightfield(np.random.default_rng(seed + 1), grid, 0.3)))]
    return config2(seed, width, height, meshes=meshes)


def _with_normals(mesh):
    pos, idx, nrm = mesh
    return pos, idx, nrm, idx


def feature_scene(seed=0, width=96, height=54, max_depth=4):
    """Every branch of the reference's per-pixel path in one small scene:
    checkerboard-transparent quad/box/sphere/tet, glass (refraction and total
    internal reflection), mirrors, two emissive-quad area lights with sphere
    and quad occluders, point, directional and non-shadowing lights, all four
    BRDFs, meshes with and without normals."""
    rng = np.random.default_rng(seed)
    M = L.default_material
    materials = [
        M(albedo=0.8, roughness=0.6, brdf=L.BRDF_LAMBERT),                                           # 0 floor
        M(albedo=0.9, roughness=0.3, brdf=L.BRDF_PHONG, reflectivity=(1.0, 1.0, 0.4)),                # 1
        M(albedo=0.7, roughness=0.4, brdf=L.BRDF_BLINN, reflectivity=(1.0, 0.4, 1.0)),                # 2
        M(albedo=0.8, roughness=0.3, brdf=L.BRDF_COOK_TORRANCE, metalness=0.5),                       # 3
        M(albedo=0.05, roughness=0.25, flags=L.MATERIAL_IS_REFRACTIVE, ior=1.5, reflectivity=0.03),   # 4 glass
        M(albedo=0.0, roughness=0.02, flags=L.MATERIAL_IS_REFLECTIVE, reflectivity=(0.91, 0.92, 0.92)),  # 5 mirror
        M(albedo=0, roughness=0, flags=L.MATERIAL_IS_EMISSIVE, emission=(0.9, 0.5, 0.5)),           # 6 emissive
        M(albedo=0, roughness=0, flags=L.MATERIAL_IS_EMISSIVE, emission=(0.5, 0.5, 0.9)),           # 7 emissive
        M(albedo=0.6, roughness=0.0, brdf=L.BRDF_COOK_TORRANCE),                                      # 8 roughness 0
    ]
    V, S, T = L.GEOMETRY_IS_VISIBLE, L.GEOMETRY_IS_SHADOWING, L.GEOMETRY_IS_TRANSPARENT
    def jitter(p):
        return tuple(np.float32(c + rng.uniform(-0.3, 0.3)) for c in p)
    ay = lambda: quat_y(rng.uniform(0, 2 * np.pi))
    geos = [geometry(L.GEOMETRY_QUAD, 0, (0, 0, 0), (12, 1, 12))]
    a, w = ay(); geos.append(geometry(L.GEOMETRY_BOX, 1, jitter((-4, 1, 1)), (1, 1, 1), a, w, flags=V | S | T))
    geos.append(geometry(L.GEOMETRY_SPHERE, 2, jitter((-1.5, 1.2, 2)), (1.2, 1.2, 1.2), flags=V | S | T))
    a, w = ay(); geos.append(geometry(L.GEOMETRY_TET, 3, jitter((1.5, 0.9, 3)), (1.5, 1.5, 1.5), a, w, flags=V | S | T))
    geos.append(geometry(L.GEOMETRY_SPHERE, 4, jitter((0.5, 1.0, -1)), (1.0, 1.0, 1.0), flags=V))       # glass
    a, w = ay(); geos.append(geometry(L.GEOMETRY_BOX, 4, jitter((3.5, 0.8, -0.5)), (0.8, 0.8, 0.8), a, w, flags=V))
    geos.append(geometry(L.GEOMETRY_QUAD, 5, jitter((0, 3, 6)), (5, 1, 3), (0.70710678, 0, 0), 0.70710678))  # mirror
    geos.append(geometry(L.GEOMETRY_QUAD, 3, jitter((-2, 2.5, 4)), (1, 1, 1), (0, 0, 0.70710678), 0.70710678,
                         flags=V | S | T))
    geos.append(geometry(L.GEOMETRY_QUAD, 6, (-7, 4, 2), (2, 1, 3), (0, 0, -0.70710678), 0.70710678, flags=V))
    geos.append(geometry(L.GEOMETRY_QUAD, 7, (7, 3, 1), (2, 1, 2), (0, 0, 0.70710678), 0.70710678, flags=V))
    geos.append(geometry(L.GEOMETRY_SPHERE, 8, jitter((5, 0.6, 3)), (0.6, 0.6, 0.6)))
    meshes = [MeshAsset.build(*_with_normals(icosphere(1))),
              MeshAsset.build(*heightfield(np.random.default_rng(seed + 9), 6, 0.3)[:2])]
    a, w = random_quat(rng); geos.append(geometry(L.GEOMETRY_MESH, 3, jitter((-3.5, 1.0, -1.5)), (0.9, 0.9, 0.9), a, w,
                                                  mesh_id=0))
    geos.append(geometry(L.GEOMETRY_MESH, 4, jitter((2.0, 2.2, 1.0)), (0.8, 0.8, 0.8), mesh_id=0, flags=V))
    a, w = random_quat(rng); geos.append(geometry(L.GEOMETRY_MESH, 2, jitter((-0.5, 2.8, 4.0)), (1.5, 1.5, 1.5), a, w,
                                                  mesh_id=1))
    lights = [light((1.0, 0.9, 0.8), jitter((-3, 6, -3)), 30.0),
              light((0.4, 0.6, 1.0), (0.3, -1.0, 0.4), 1.5, flags=L.LIGHT_IS_DIRECTIONAL | L.LIGHT_IS_SHADOWING),
              light((0.3, 1.0, 0.3), jitter((2, 1.5, -2)), 8.0, flags=0)]
    scene = Scene(np.array(geos), np.array(materials), np.array(lights), meshes=meshes)
    cam = Camera.look_at((1.0, 5.0, -9.0), (0.0, 1.2, 1.5), 60.0)
    return Workload(f"features_{width}x{height}_d{max_depth}", scene, cam, width, height,
                    L.default_settings(max_depth=max_depth))


# ---- textures and sky -------------------------------------------------------
def albedo_texture(rng, size):
    """Value-noise RGBA8 albedo (sRGB bytes, B,G,R,A as a BMP stores them),
    baked with a full mip chain and wrap addressing."""
    base = rng.uniform(0.15, 0.95, 3)
    n = value_noise_2d(rng, size, max(2, size // 64))
    tint = rng.uniform(0.5, 1.0, 3)
    rgb = np.clip(base[None, None, :] * (0.55 + 0.9 * (n[..., None] - 0.5)) * tint[None, None, :], 0, 1)
    bgra = np.empty((size, size, 4), np.uint8)
    bgra[..., 0] = (rgb[..., 2] * 255).astype(np.uint8)
    bgra[..., 1] = (rgb[..., 1] * 255).astype(np.uint8)
    bgra[..., 2] = (rgb[..., 0] * 255).astype(np.uint8)
    bgra[..., 3] = 255
    return TextureAsset.bake(bgra, L.IMAGE_MIPMAP | L.IMAGE_WRAP)


def normal_texture(rng, size, strength=2.0):
    """Tangent-space normal map of a value-noise height field: X and Y stored
    in R and G, Z derived by the baker (bmp2texture's -n)."""
    hgt = value_noise_2d(rng, size, max(2, size // 32)) * strength
    gy, gx = np.gradient(hgt * size / 16.0)
    x, y = -gx, -gy
    inv = 1.0 / np.sqrt(x * x + y * y + 1.0)
    bgr = np.zeros((size, size, 3), np.uint8)
    bgr[..., 2] = np.clip((x * inv * 0.5 + 0.5) * 255, 0, 255).astype(np.uint8)
    bgr[..., 1] = np.clip((y * inv * 0.5 + 0.5) * 255, 0, 255).astype(np.uint8)
    bgr[..., 0] = 255
    return TextureAsset.bake(bgr, L.IMAGE_MIPMAP | L.IMAGE_WRAP | L.IMAGE_NORMAL | L.IMAGE_LINEAR)


def cube_directions(h):
    """Unit directions of the texel centres of a 6h x h cube strip laid out
    as the reference samples it (core/texture.h:72-116): four side faces
    (left, front, right, back) across the first 4h columns, then the top and
    bottom faces."""
    ys = (np.arange(h) + 0.5) / h
    dirs = np.zeros((h, 6 * h, 3))
    u4 = (np.arange(4 * h) + 0.5) / (4 * h)
    U, V = np.meshgrid(u4, ys)
    face = np.minimum((U * 4).astype(int), 3)
    d = np.zeros((h, 4 * h, 3))
    left, front, right, back = face == 0, face == 1, face == 2, face == 3
    d[left] = np.stack([-np.ones(left.sum()), -(2 * V[left] - 1), -(1 - 8 * U[left])], -1)
    d[front] = np.stack([8 * U[front] - 3, 1 - 2 * V[front], np.ones(front.sum())], -1)
    d[right] = np.stack([np.ones(right.sum()), 1 - 2 * V[right], 5 - 8 * U[right]], -1)
    d[back] = np.stack([7 - 8 * U[back], 1 - 2 * V[back], -np.ones(back.sum())], -1)
    dirs[:, :4 * h] = d
    u1 = (np.arange(h) + 0.5) / h
    U1, V1 = np.meshgrid(u1, ys)
    dirs[:, 4 * h:5 * h] = np.stack([2 * U1 - 1, np.ones_like(U1), 2 * V1 - 1], -1)
    dirs[:, 5 * h:] = np.stack([2 * U1 - 1, -np.ones_like(U1), 1 - 2 * V1], -1)
    return dirs / np.linalg.norm(dirs, axis=-1, keepdims=True)


def sky_radiance(dirs, rng):
    """Procedural sky: zenith/horizon gradient, dark ground, three Gaussian
    sun lobes; linear RGB in [0, 1]."""
    y = dirs[..., 1:2]
    zenith, horizon, ground = np.array([0.18, 0.32, 0.62]), np.array([0.75, 0.78, 0.82]), np.array([0.16, 0.14, 0.12])
    t = np.clip(y, 0, 1) ** 0.45
    col = np.where(y >= 0, horizon * (1 - t) + zenith * t, ground + (horizon - ground) * np.exp(8 * y))
    for _ in range(3):
        elev = rng.uniform(0.15, 1.0)
        az = rng.uniform(0, 2 * np.pi)
        sd = np.array([np.cos(az) * np.sqrt(1 - elev ** 2), elev, np.sin(az) * np.sqrt(1 - elev ** 2)])
        cosang = np.clip(dirs @ sd, -1, 1)
        sharp = rng.uniform(200, 900)
        col = col + rng.uniform(0.5, 0.9) * np.exp(-(1 - cosang)[..., None] * sharp) * rng.uniform(0.8, 1.0, 3)
    return np.clip(col, 0, 1)


def to_bgr8(rgb):
    out = np.empty(rgb.shape[:2] + (3,), np.uint8)
    out[..., 0] = (rgb[..., 2] * 255).astype(np.uint8)
    out[..., 1] = (rgb[..., 1] * 255).astype(np.uint8)
    out[..., 2] = (rgb[..., 0] * 255).astype(np.uint8)
    return out


def sky_cubes(rng, size=512, irradiance_size=32):
    """Radiance cube (size) and its cosine-convolved irradiance cube
    (irradiance_size), both baked as linear 8-bit cube strips (-c -l)."""
    dirs = cube_directions(size)
    radiance = sky_radiance(dirs, rng)
    # irradiance: cosine-weighted average over a coarse copy of the sky
    coarse = max(8, min(size, 32))
    cd = cube_directions(coarse).reshape(-1, 3)
    cr = sky_radiance(cube_directions(coarse), np.random.default_rng(rng.integers(1 << 31)))
    step = size // coarse
    cr = radiance[step // 2::step, step // 2::step][:coarse, :6 * coarse].reshape(-1, 3)
    idirs = cube_directions(irradiance_size).reshape(-1, 3)
    w = np.clip(idirs @ cd.T, 0, None)
    irr = (w @ cr) / np.maximum(w.sum(1, keepdims=True), 1e-9)
    irr = irr.reshape(irradiance_size, 6 * irradiance_size, 3)
    flags = L.IMAGE_CUBEMAP | L.IMAGE_LINEAR
    return TextureAsset.bake(to_bgr8(radiance), flags), TextureAsset.bake(to_bgr8(irr), flags)


def config3(seed=0, width=1920, height=1080, tex_size=1024, cube_size=512, irradiance_size=32, max_depth=8):
    """config 1's objects + 4 glass spheres + 2 mirror quads, albedo and
    normal textures, sky cube IBL."""
    rng = np.random.default_rng(seed)
    trng = np.random.default_rng(seed + 1000)
    textures = [albedo_texture(trng, tex_size) for _ in range(4)] + [normal_texture(trng, tex_size) for _ in range(2)]
    sky, irr = sky_cubes(trng, cube_size, irradiance_size)
    textures += [sky, irr]
    SKY, IRR = 6, 7
    floor = L.default_material(albedo=0.9, roughness=0.7, brdf=L.BRDF_LAMBERT,
                               flags=L.MATERIAL_HAS_ALBEDO_MAP | L.MATERIAL_HAS_NORMAL_MAP, texture_ids=(0, 4),
                               uv_repeat=(4.0, 4.0), normal_magnitude=0.8)
    materials = [floor]
    geos = [geometry(L.GEOMETRY_QUAD, 0, (0, 0, 0), (10, 1, 10))]
    geos += _implicit_objects(rng, materials)
    # texture the implicit objects (the tetrahedron stays untextured)
    for k, mid in enumerate(range(1, 6)):
        m = materials[mid]
        m["flags"] |= L.MATERIAL_HAS_ALBEDO_MAP | (L.MATERIAL_HAS_NORMAL_MAP if k % 2 == 0 else 0)
        m["texture_count"] = 2
        m["texture_ids"] = (1 + k % 3, 4 + k % 2)
        m["albedo"] = np.float32(1.0)
    glass = L.default_material(albedo=0.05, roughness=0.25, flags=L.MATERIAL_IS_REFRACTIVE, ior=1.5, reflectivity=0.04)
    mirror = L.default_material(albedo=0.0, roughness=0.02, flags=L.MATERIAL_IS_REFLECTIVE,
                                reflectivity=(0.91, 0.92, 0.92))
    materials += [glass, mirror]
    GLASS, MIRROR = len(materials) - 2, len(materials) - 1
    for _ in range(4):
        r = np.float32(rng.uniform(0.5, 1.2))
        x, z = rng.uniform(-5, 5, 2)
        geos.append(geometry(L.GEOMETRY_SPHERE, GLASS, (x, r, z), (r, r, r), flags=L.GEOMETRY_IS_VISIBLE))
    for sx in (-1, 1):
        ang = rng.uniform(-0.6, 0.6) + (0.35 if sx > 0 else -0.35)
        a, w_ = quat_y(ang)
        # stand the quad up: rotate +y normal to face -z, then turn about y
        qx = np.array([np.sin(-np.pi / 4), 0, 0, np.cos(-np.pi / 4)])
        qy = np.array([a[0], a[1], a[2], w_], np.float64)
        q = _qmul(qy, qx)
        geos.append(geometry(L.GEOMETRY_QUAD, MIRROR, (sx * 4.5, 2.5, 6.5), (2.5, 1, 2.5), q[:3], q[3]))
    lights = [light(rng.uniform(0.5, 1.0, 3), (rng.uniform(-5, 5), rng.uniform(3, 6), rng.uniform(-5, 5)),
                    rng.uniform(5, 20)) for _ in range(2)]
    scene = Scene(np.array(geos), np.array(materials), np.array(lights), textures=textures)
    cam = Camera.look_at((0.0, 5.0, -13.0), (0.0, 1.0, 1.0), 60.0)
    return Workload(f"config3_glass_mirror_textures_ibl_{width}x{height}_d{max_depth}", scene, cam, width, height,
                    L.default_settings(max_depth=max_depth, skybox_color=SKY, skybox_radiance=SKY,
                                       skybox_irradiance=IRR))


def _qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz], np.float32)


def small_textured_scene(seed=0, width=160, height=90, max_depth=8):
    """config 3's shape at oracle-friendly size (64^2 textures, 32^2 sky)."""
    return config3(seed, width, height, tex_size=64, cube_size=32, irradiance_size=8, max_depth=max_depth)


def config4(seed=0, width=1920, height=1080, meshes=None):
    """The radiance-cache workload: config 2's scene with bounce depth 8 (the
    plain depth-8 frame is the reference image for the cache frame, whose
    paths stop at vertex 2 and take the cache's answer)."""
    w = config2(seed, width, height, meshes)
    w.name = f"config4_cache_mesh_pbr_{width}x{height}_d8_cache2"
    w.settings = L.default_settings(max_depth=8)
    return w


CONFIGS = {"config1": config1, "config2": config2, "config3": config3, "config4": config4}


# ---- config 5: batched requests ------------------------------------------------
BATCH_RESOLUTIONS = [(320, 180), (640, 360), (1280, 720), (1920, 1080), (3840, 2160)]


class Request:
    """One render request of a batch: its own scene (mesh ids refer to the
    shared assets), camera, canvas size, bounce depth and cache use."""

    def __init__(self, name, scene, camera, width, height, settings, radiance_cache):
        self.name, self.scene, self.camera = name, scene, camera
        self.width, self.height, self.settings, self.radiance_cache = width, height, settings, radiance_cache

    @property
    def samples(self):
        return self.width * self.height

    def projection(self):
        return self.camera.projection(self.width, self.height, False)

    def workload(self):
        return Workload(self.name, self.scene, self.camera, self.width, self.height, self.settings)


def batch_request(rng, meshes, width, height, max_depth, radiance_cache, index=0):
    """A seeded scene of 1-16 instances of the shared meshes and 0-8 implicit
    primitives on a floor, with Cook-Torrance, glass and mirror materials
    and 2-4 point lights."""
    pbr = []
    for _ in range(4):
        metallic = int(rng.integers(0, 2))
        m = L.default_material(albedo=0, roughness=float(rng.uniform(0.05, 1.0)), brdf=L.BRDF_COOK_TORRANCE,
                               reflectivity=0.04, metalness=float(metallic),
                               flags=L.MATERIAL_IS_REFLECTIVE if metallic else 0)
        m["albedo"] = rng.uniform(0.2, 1.0, 3).astype(np.float32)
        pbr.append(m)
    glass = L.default_material(albedo=0.05, roughness=0.25, flags=L.MATERIAL_IS_REFRACTIVE, ior=1.5, reflectivity=0.04)
    mirror = L.default_material(albedo=0.0, roughness=0.02, flags=L.MATERIAL_IS_REFLECTIVE,
                                reflectivity=(0.91, 0.92, 0.92))
    floor = L.default_material(albedo=0.8, roughness=0.8, brdf=L.BRDF_LAMBERT)
    materials = [floor] + pbr + [glass, mirror]
    GLASS, MIRROR = 5, 6
    geos = [geometry(L.GEOMETRY_QUAD, 0, (0, 0, 0), (12, 1, 12))]
    for _ in range(int(rng.integers(1, 17))):
        axis, amount = random_quat(rng)
        s = np.float32(rng.uniform(0.5, 2.0))
        pos = (rng.uniform(-7, 7), rng.uniform(0.5, 3.0), rng.uniform(-4, 8))
        r = rng.uniform()
        mid = GLASS if r < 0.15 else MIRROR if r < 0.3 else int(rng.integers(1, 5))
        flags = L.GEOMETRY_IS_VISIBLE if mid == GLASS else L.GEOMETRY_IS_VISIBLE | L.GEOMETRY_IS_SHADOWING
        geos.append(geometry(L.GEOMETRY_MESH, mid, pos, (s, s, s), axis, amount, mesh_id=int(rng.integers(0, len(meshes))),
                             flags=flags))
    kinds = [L.GEOMETRY_SPHERE, L.GEOMETRY_BOX, L.GEOMETRY_TET, L.GEOMETRY_QUAD]
    for _ in range(int(rng.integers(0, 9))):
        kind = kinds[int(rng.integers(0, 4))]
        r = rng.uniform()
        mid = GLASS if (r < 0.25 and kind == L.GEOMETRY_SPHERE) else MIRROR if r < 0.4 else int(rng.integers(1, 5))
        flags = L.GEOMETRY_IS_VISIBLE if mid == GLASS else L.GEOMETRY_IS_VISIBLE | L.GEOMETRY_IS_SHADOWING
        s = np.float32(rng.uniform(0.5, 1.5))
        x, z = rng.uniform(-6, 6), rng.uniform(-4, 8)
        axis, amount = quat_y(rng.uniform(0, 2 * np.pi))
        y = s if kind != L.GEOMETRY_TET else np.float32(s * TET_MAX)
        geos.append(geometry(kind, mid, (x, y, z), (s, s, s), axis, amount, flags=flags))
    lights = [light(rng.uniform(0.6, 1.0, 3), (rng.uniform(-8, 8), rng.uniform(4, 8), rng.uniform(-8, 4)),
                    rng.uniform(15, 50)) for _ in range(int(rng.integers(2, 5)))]
    scene = Scene(np.array(geos), np.array(materials), np.array(lights), meshes=meshes)
    eye = (rng.uniform(-3, 3), rng.uniform(4, 7), rng.uniform(-15, -11))
    cam = Camera.look_at(eye, (0.0, 1.0, 2.0), 60.0)
    return Request(f"request{index}_{width}x{height}_d{max_depth}{'_cache' if radiance_cache else ''}", scene, cam,
                   width, height, L.default_settings(max_depth=max_depth), radiance_cache)


def config5(seed=0, count=64, meshes=None, resolutions=None):
    """64 requests: resolutions drawn uniformly from 320x180 ... 3840x2160,
    bounce depth 1-8, every other request with the radiance cache."""
    rng = np.random.default_rng(seed)
    meshes = meshes if meshes is not None else config2_meshes()
    resolutions = resolutions or BATCH_RESOLUTIONS
    out = []
    for i in range(count):
        w, h = resolutions[int(rng.integers(0, len(resolutions)))]
        depth = int(rng.integers(1, 9))
        out.append(batch_request(rng, meshes, w, h, depth, L.CACHE_ON if i % 2 == 0 else L.CACHE_OFF, i))
    return out
