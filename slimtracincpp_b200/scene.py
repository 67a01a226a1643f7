"""Host-side scene containers mirroring the reference's Scene
(scene/scene.h:35-192), Mesh (scene/mesh.h:25-41) and Texture
(core/texture.h:44-45), backed by numpy arrays in the reference's binary
layouts so the C ABI can read them in place.
"""
from __future__ import annotations

import numpy as np

from . import layout as L
from .native import check, lib, ptr

# Host-side builders the containers below call: the library's own
# restatements by default.  A caller may put other implementations of the
# same algorithms here (same arguments, same outputs), e.g. to build a scene
# for another renderer without loading this library:
#   "scene_bvh"   f(scene_data_record)          Scene::updateAABBs + updateBVH
#   "mesh"        f(positions, indices, normals, normal_indices, uvs, uv_indices)
#                   -> (triangles, nodes, height, aabb6, recentred positions)
#   "projection"  f(camera, width, height, ssaa) -> CameraRayProjection record
#   "texture"     f(bgr rows, flags) -> (Texture record, mip sizes, texel quads)
HOST_BUILDERS = {}


class MeshAsset:
    """A mesh with its leaf-ordered Triangle records and SAH BVH, as the
    reference's obj2mesh produces them (obj2mesh.cpp:125-231)."""

    def __init__(self, triangles, nodes, aabb_min, aabb_max, height, positions, position_indices,
                 normals=None, normal_indices=None, uvs=None, uv_indices=None, edges=None):
        self.triangles = np.ascontiguousarray(triangles, dtype=L.TRIANGLE)
        self.nodes = np.ascontiguousarray(nodes, dtype=L.BVH_NODE)
        self.aabb_min = np.asarray(aabb_min, np.float32)
        self.aabb_max = np.asarray(aabb_max, np.float32)
        self.height = int(height)
        self.positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        self.position_indices = np.ascontiguousarray(position_indices, np.uint32).reshape(-1, 3)
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        self.normal_indices = None if normal_indices is None else np.ascontiguousarray(normal_indices, np.uint32).reshape(-1, 3)
        self.uvs = None if uvs is None else np.ascontiguousarray(uvs, np.float32).reshape(-1, 2)
        self.uv_indices = None if uv_indices is None else np.ascontiguousarray(uv_indices, np.uint32).reshape(-1, 3)
        self.edges = np.zeros((0, 2), np.uint32) if edges is None else np.ascontiguousarray(edges, np.uint32).reshape(-1, 2)

    @property
    def triangle_count(self):
        return len(self.triangles)

    @classmethod
    def build(cls, positions, indices, normals=None, normal_indices=None, uvs=None, uv_indices=None):
        """obj2mesh's build step (recentre, SAH BVH, Triangle precompute) via
        slimBuildMesh; `positions` are copied, the copy is recentred."""
        pos = np.array(positions, dtype=np.float32).reshape(-1, 3).copy()
        idx = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
        t = len(idx)
        nrm = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        nidx = None if normal_indices is None else np.ascontiguousarray(normal_indices, np.uint32).reshape(-1, 3)
        uv = None if uvs is None else np.ascontiguousarray(uvs, np.float32).reshape(-1, 2)
        uidx = None if uv_indices is None else np.ascontiguousarray(uv_indices, np.uint32).reshape(-1, 3)
        if "mesh" in HOST_BUILDERS:
            tris, nodes, height, aabb, pos = HOST_BUILDERS["mesh"](pos, idx, nrm, nidx, uv, uidx)
            return cls(tris, nodes, aabb[:3], aabb[3:], height, pos, idx, nrm, nidx, uv, uidx, _edges(idx))
        tris = np.zeros(t, L.TRIANGLE)
        nodes = np.zeros(2 * t, L.BVH_NODE)
        node_count = np.zeros(1, np.uint32)
        height = np.zeros(1, np.uint32)
        aabb = np.zeros(6, np.float32)
        check(lib().slimBuildMesh(ptr(pos), len(pos), ptr(idx), t, ptr(nrm), 0 if nrm is None else len(nrm), ptr(nidx),
                                  ptr(uv), 0 if uv is None else len(uv), ptr(uidx), ptr(tris), ptr(nodes),
                                  ptr(node_count), ptr(height), ptr(aabb)))
        edges = _edges(idx)
        return cls(tris, nodes[:int(node_count[0])].copy(), aabb[:3], aabb[3:], int(height[0]), pos, idx, nrm, nidx,
                   uv, uidx, edges)

    def record(self):
        """The Mesh struct (128 bytes) pointing at this asset's arrays."""
        m = np.zeros((), L.MESH)
        m["aabb_min"], m["aabb_max"] = self.aabb_min, self.aabb_max
        m["bvh_nodes"], m["bvh_node_count"], m["bvh_height"] = ptr(self.nodes), len(self.nodes), min(self.height, 255)
        m["triangles"] = ptr(self.triangles)
        m["vertex_positions"] = ptr(self.positions)
        m["vertex_position_indices"] = ptr(self.position_indices)
        m["vertex_normals"] = ptr(self.normals)
        m["vertex_normal_indices"] = ptr(self.normal_indices)
        m["vertex_uvs"] = ptr(self.uvs)
        m["vertex_uvs_indices"] = ptr(self.uv_indices)
        m["edge_vertex_indices"] = ptr(self.edges)
        m["triangle_count"] = len(self.triangles)
        m["vertex_count"] = len(self.positions)
        m["edge_count"] = len(self.edges)
        m["normals_count"] = 0 if self.normals is None else len(self.normals)
        m["uvs_count"] = 0 if self.uvs is None else len(self.uvs)
        return m

    def save(self, path):
        """Writes the native .mesh format (serialization/mesh.h:56-122)."""
        rec = self.record()
        check(lib().slimWriteMesh(str(path).encode(), ptr(rec)))

    @classmethod
    def load(cls, path):
        """Reads a .mesh file (serialization/mesh.h:149-163)."""
        h = np.zeros((), L.MESH)
        check(lib().slimReadMeshHeader(str(path).encode(), ptr(h)))
        t, v, e = int(h["triangle_count"]), int(h["vertex_count"]), int(h["edge_count"])
        nn, nu = int(h["normals_count"]), int(h["uvs_count"])
        tris = np.zeros(t, L.TRIANGLE)
        nodes = np.zeros(int(h["bvh_node_count"]), L.BVH_NODE)
        pos = np.zeros((v, 3), np.float32)
        pidx = np.zeros((t, 3), np.uint32)
        edges = np.zeros((e, 2), np.uint32)
        nrm = np.zeros((nn, 3), np.float32) if nn else None
        nidx = np.zeros((t, 3), np.uint32) if nn else None
        uv = np.zeros((nu, 2), np.float32) if nu else None
        uidx = np.zeros((t, 3), np.uint32) if nu else None
        rec = np.zeros((), L.MESH)
        for k in ("triangle_count", "vertex_count", "edge_count", "normals_count", "uvs_count", "bvh_node_count"):
            rec[k] = h[k]
        rec["triangles"], rec["bvh_nodes"] = ptr(tris), ptr(nodes)
        rec["vertex_positions"], rec["vertex_position_indices"] = ptr(pos), ptr(pidx)
        rec["edge_vertex_indices"] = ptr(edges)
        rec["vertex_normals"], rec["vertex_normal_indices"] = ptr(nrm), ptr(nidx)
        rec["vertex_uvs"], rec["vertex_uvs_indices"] = ptr(uv), ptr(uidx)
        check(lib().slimReadMesh(str(path).encode(), ptr(rec)))
        return cls(tris, nodes, rec["aabb_min"], rec["aabb_max"], int(h["bvh_height"]), pos, pidx, nrm, nidx, uv, uidx,
                   edges)


def _edges(idx):
    """Unique undirected edges of a triangle list (the .mesh edge table)."""
    a = np.concatenate([idx[:, [0, 1]], idx[:, [1, 2]], idx[:, [2, 0]]]).astype(np.uint64)
    lo, hi = np.minimum(a[:, 0], a[:, 1]), np.maximum(a[:, 0], a[:, 1])
    key = np.unique(lo | (hi << np.uint64(32)))
    return np.stack([(key & np.uint64(0xFFFFFFFF)).astype(np.uint32), (key >> np.uint64(32)).astype(np.uint32)], 1)


class TextureAsset:
    """A texture in the texel-quad layout (core/texture.h:5-45)."""

    def __init__(self, header, mip_sizes, quads):
        self.header = np.array(header, dtype=L.TEXTURE)
        self.mip_sizes = [(int(w), int(h)) for w, h in mip_sizes]
        self.quads = np.ascontiguousarray(quads, dtype=L.TEXEL_QUAD)
        self.mips = np.zeros(len(self.mip_sizes), L.TEXTURE_MIP)
        off = 0
        for i, (w, h) in enumerate(self.mip_sizes):
            self.mips[i]["width"], self.mips[i]["height"] = w, h
            self.mips[i]["texel_quads"] = self.quads.ctypes.data + off * L.TEXEL_QUAD.itemsize
            off += (w + 1) * (h + 1)
        assert off == len(self.quads)
        self.header["mip_count"] = len(self.mip_sizes)
        self.header["mips"] = ptr(self.mips)

    def record(self):
        return self.header

    def mip_quads(self, m):
        off = sum((w + 1) * (h + 1) for w, h in self.mip_sizes[:m])
        w, h = self.mip_sizes[m]
        return self.quads[off:off + (w + 1) * (h + 1)].reshape(h + 1, w + 1)

    @classmethod
    def bake(cls, bgr, flags, on_gpu=False):
        """bmp2texture's baker (bmp2texture.cpp:24-335) on 8-bit BGR(A) rows,
        on the host or (on_gpu) on the device: the same bytes."""
        img = np.ascontiguousarray(bgr, dtype=np.uint8)
        if "texture" in HOST_BUILDERS and not on_gpu:
            header, sizes, quads = HOST_BUILDERS["texture"](img, flags)
            return cls(header, sizes, quads)
        h, w, ch = img.shape
        mip_count = np.zeros(1, np.uint32)
        quad_count = np.zeros(1, np.uint32)
        header = np.zeros((), L.TEXTURE)
        baker = lib().slimBakeTextureOnGPU if on_gpu else lib().slimBakeTexture
        check(baker(ptr(img), w, h, ch, flags, ptr(header), 0, 0, ptr(mip_count), ptr(quad_count)))
        mips = np.zeros(int(mip_count[0]), L.TEXTURE_MIP)
        quads = np.zeros(int(quad_count[0]), L.TEXEL_QUAD)
        check(baker(ptr(img), w, h, ch, flags, ptr(header), ptr(mips), ptr(quads), ptr(mip_count), ptr(quad_count)))
        return cls(header, [(m["width"], m["height"]) for m in mips], quads)

    def save(self, path):
        check(lib().slimWriteTexture(str(path).encode(), ptr(self.header)))

    @classmethod
    def load(cls, path):
        header = np.zeros((), L.TEXTURE)
        total = np.zeros(1, np.uint32)
        check(lib().slimReadTextureHeader(str(path).encode(), ptr(header), ptr(total)))
        mips = np.zeros(int(header["mip_count"]), L.TEXTURE_MIP)
        quads = np.zeros(int(total[0]), L.TEXEL_QUAD)
        check(lib().slimReadTexture(str(path).encode(), ptr(header), ptr(mips), ptr(quads)))
        return cls(header, [(m["width"], m["height"]) for m in mips], quads)


class Camera:
    """Camera pose as the reference's Camera holds it (scene/camera.h:6-13):
    orientation matrix columns right (X), up (Y), forward (Z), position and
    focal length (1/tan(fov_y/2))."""

    def __init__(self, orientation, position, focal_length=2.0):
        self.orientation = np.asarray(orientation, np.float32).reshape(9)
        self.position = np.asarray(position, np.float32).reshape(3)
        self.focal_length = float(np.float32(focal_length))

    @classmethod
    def look_at(cls, position, target, fov_y_degrees=60.0):
        p = np.asarray(position, np.float64)
        fwd = np.asarray(target, np.float64) - p
        fwd /= np.linalg.norm(fwd)
        right = np.cross([0.0, 1.0, 0.0], fwd)
        right /= np.linalg.norm(right)
        up = np.cross(fwd, right)
        focal = 1.0 / np.tan(np.radians(fov_y_degrees) * 0.5)
        return cls(np.concatenate([right, up, fwd]).astype(np.float32), p.astype(np.float32), focal)

    def projection(self, width, height, ssaa=False):
        if "projection" in HOST_BUILDERS:
            return HOST_BUILDERS["projection"](self, width, height, ssaa)
        from .native import projection_reset
        return projection_reset(self.orientation, self.position, self.focal_length, width, height, ssaa)


class Scene:
    """Geometries, materials, lights, meshes and textures plus the scene BVH,
    laid out as the reference's SceneData (scene/scene.h:35-56)."""

    def __init__(self, geometries, materials, lights=None, meshes=(), textures=(), cameras=None):
        self.geometries = np.ascontiguousarray(geometries, dtype=L.GEOMETRY)
        self.materials = np.ascontiguousarray(materials, dtype=L.MATERIAL)
        self.lights = np.ascontiguousarray(lights if lights is not None else np.zeros(0, L.LIGHT), dtype=L.LIGHT)
        self.meshes = list(meshes)
        self.textures = list(textures)
        self.cameras = cameras
        self.mesh_records = np.zeros(max(1, len(self.meshes)), L.MESH)
        self.texture_records = np.zeros(max(1, len(self.textures)), L.TEXTURE)
        self.refresh_assets()
        g = len(self.geometries)
        self.bvh_nodes = np.zeros(max(2 * g, 1), L.BVH_NODE)
        self.leaf_ids = np.zeros(max(g, 1), np.uint32)
        self.data = np.zeros((), L.SCENE_DATA)
        self._fill()
        self.build_bvh()

    def refresh_assets(self):
        for i, m in enumerate(self.meshes):
            self.mesh_records[i] = m.record()
        for i, t in enumerate(self.textures):
            self.texture_records[i] = t.record()

    def _fill(self):
        d = self.data
        d["counts"] = [len(self.geometries), 0 if self.cameras is None else 1, len(self.lights), len(self.materials),
                       len(self.textures), len(self.meshes), 0, 0, 0, 0, 0]
        d["geometries"] = ptr(self.geometries)
        d["lights"] = ptr(self.lights) if len(self.lights) else 0
        d["materials"] = ptr(self.materials)
        d["textures"] = ptr(self.texture_records) if self.textures else 0
        d["meshes"] = ptr(self.mesh_records) if self.meshes else 0
        d["bvh_leaf_geometry_indices"] = ptr(self.leaf_ids)
        d["bvh_nodes"] = ptr(self.bvh_nodes)
        d["mesh_stack_size"] = (max(m.height for m in self.meshes) + 2) if self.meshes else 0

    def build_bvh(self):
        """Scene::updateAABBs + updateBVH (scene/scene.h:176-191) on the host."""
        if "scene_bvh" in HOST_BUILDERS:
            HOST_BUILDERS["scene_bvh"](self.data)
            return
        check(lib().slimBuildSceneBVH(ptr(self.data)))

    @property
    def ptr(self):
        return ptr(self.data)


def geometry(kind, material_id, position=(0, 0, 0), scale=(1, 1, 1), axis=(0, 0, 0), amount=1.0, mesh_id=0,
             flags=L.GEOMETRY_IS_VISIBLE | L.GEOMETRY_IS_SHADOWING):
    g = np.zeros((), L.GEOMETRY)
    g["axis"], g["amount"] = axis, amount
    g["position"], g["scale"] = position, np.broadcast_to(np.float32(scale), 3) if np.ndim(scale) == 0 else scale
    g["type"], g["material_id"], g["id"], g["flags"], g["color"] = kind, material_id, mesh_id, flags, 1
    return g


def light(color, position, intensity, flags=L.LIGHT_IS_SHADOWING):
    li = np.zeros((), L.LIGHT)
    li["color"], li["position"], li["intensity"], li["flags"] = color, position, intensity, flags
    return li


def quat_y(radians):
    """quat::AxisAngle(Y, radians) components (math/quat.h:86-92), float32."""
    h = np.float32(radians) * np.float32(0.5)
    s, c = np.float32(np.sin(h)), np.float32(np.cos(h))
    inv = np.float32(1.0) / np.float32(np.sqrt(np.float32(s * s) + np.float32(c * c)))
    return (np.float32(0), np.float32(s * inv), np.float32(0)), np.float32(c * inv)
