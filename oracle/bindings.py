"""ctypes access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

  liboracle.so        plain-C restatement of the reference's trace path
                      (oracle/slim_oracle.c), built by oracle/Makefile.
  _ref/libslimref.so  the reference's own CPU code, compiled from its
                      sources by oracle/build_ref.sh (present when it was
                      built on a machine holding the reference sources).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs use this module, as the checker and the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libslimref.so"
# The reference built for timing: -O3 -DNDEBUG with the host's ISA level
# (x86-64-v4 where the CPU has AVX-512, else x86-64-v3), no parity flags.
REF_TIMED_LIBS = {"x86-64-v4": HERE / "_ref" / "libslimref_timed_v4.so",
                  "x86-64-v3": HERE / "_ref" / "libslimref_timed_v3.so"}

P = C.c_void_p
WORK_FIELDS = ["primary_rays", "shadow_rays", "bounce_rays", "scene_node_tests", "mesh_node_tests",
               "triangle_tests", "geometry_tests", "mesh_hit_fetches", "texel_taps", "pixels"]

_oracle = None
_ref = None
_ref_timed = None


def _ptr(a):
    return 0 if a is None else (a.ctypes.data if isinstance(a, np.ndarray) else int(a))


def oracle():
    global _oracle
    if _oracle is None:
        if not ORACLE_LIB.exists():
            import subprocess
            subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
        h = C.CDLL(str(ORACLE_LIB))
        h.oracle_render.argtypes = [P, P, P, P, C.c_int, C.c_int, C.c_int, P]
        h.oracle_render.restype = C.c_int
        h.oracle_trace_primary.argtypes = [P, P, C.c_int, C.c_int, P, P, P, P]
        h.oracle_trace_primary.restype = C.c_int
        h.oracle_trace_primary_rows.argtypes = [P, P, C.c_int, C.c_int, C.c_int, P, P, P, P]
        h.oracle_trace_primary_rows.restype = C.c_int
        _oracle = h
    return _oracle


def reference_available():
    return REF_LIB.exists()


def _bind_reference(path):
    h = C.CDLL(str(path))
    h.ref_projection_reset.argtypes = [P, P, C.c_float, C.c_int, C.c_int, C.c_int, P]
    h.ref_build_scene_bvh.argtypes = [P]
    h.ref_build_mesh.argtypes = [P, C.c_uint32, P, C.c_uint32, P, C.c_uint32, P, P, C.c_uint32, P, P, P, P, P, P, P]
    h.ref_render.argtypes = [P, P, P, P, C.c_int, C.c_int, C.c_int]
    h.ref_render_cpu.argtypes = [P, P, P, P]
    h.ref_trace_primary.argtypes = [P, P, C.c_int, C.c_int, P, P, P, P, C.c_int]
    for n in ["ref_projection_reset", "ref_build_scene_bvh", "ref_build_mesh", "ref_render", "ref_render_cpu",
              "ref_trace_primary"]:
        getattr(h, n).restype = C.c_int
    return h


def reference():
    """The reference built with the parity flags (bit-exact checker)."""
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (oracle/build_ref.sh needs the reference sources)")
        _ref = _bind_reference(REF_LIB)
    return _ref


def host_isa_level():
    """x86-64-v4 when this CPU has the AVX-512 subsets that level requires,
    else x86-64-v3 (AVX2 + FMA)."""
    try:
        flags = set()
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                flags = set(line.split(":", 1)[1].split())
                break
        if {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags:
            return "x86-64-v4"
    except OSError:
        pass
    return "x86-64-v3"


def reference_timed():
    """The reference built for timing (-O3 -DNDEBUG, the host's ISA level);
    returns (library, description).  Falls back to the parity build when the
    timing build is absent, and says so."""
    global _ref_timed
    if _ref_timed is None:
        level = host_isa_level()
        path = REF_TIMED_LIBS[level]
        if path.exists():
            _ref_timed = (_bind_reference(path), f"-O3 -DNDEBUG -march={level}")
        else:
            _ref_timed = (reference(), "parity build (-O3 -march=x86-64-v3 -ffp-contract=off): timing build absent")
    return _ref_timed


def reference_host_builders(layout, lib=None):
    """Host builders for slimtracincpp_b200.scene.HOST_BUILDERS that run the
    reference's own code (scene BVH, obj2mesh build, camera projection), so
    a scene can be built without loading libslimtracer_b200."""
    h = lib or reference()

    def scene_bvh(sd):
        rc = h.ref_build_scene_bvh(sd.ctypes.data)
        assert rc == 0, rc

    def mesh(pos, idx, nrm, nidx, uv, uidx):
        tris, nodes, height, aabb, out_pos = reference_build_mesh(pos, idx, nrm, nidx, uv, uidx, layout=layout, lib=h)
        return tris, nodes, height, aabb, out_pos

    def projection(camera, width, height, ssaa):
        return reference_projection(camera, width, height, ssaa, layout, lib=h)

    out = {"scene_bvh": scene_bvh, "mesh": mesh, "projection": projection}
    if BMP2TEXTURE.exists():
        out["texture"] = lambda bgr, flags: reference_bake_texture(bgr, flags, layout)
    return out


BMP2TEXTURE = HERE / "_ref" / "bmp2texture"


def write_bmp(path, bgr, top_down=True):
    """A BMP of 8-bit B,G,R(,A) rows as the reference's loader reads them
    (rows read back to back: 24-bit rows must be 4-byte multiples)."""
    import struct
    h, w, ch = bgr.shape
    rows = bgr if top_down else bgr[::-1]
    data = np.ascontiguousarray(rows).tobytes()
    off = 14 + 40
    head = struct.pack("<2sIHHI", b"BM", off + len(data), 0, 0, off)
    info = struct.pack("<IiiHHIIiiII", 40, w, -h if top_down else h, 1, 8 * ch, 0, len(data), 2835, 2835, 0, 0)
    Path(path).write_bytes(head + info + data)


def read_texture_file(path, layout):
    """A .texture file (ImageInfo, then per mip u32 width, height and its
    texel quads) as (Texture record, mip sizes, texel quads)."""
    b = Path(path).read_bytes()
    buf = np.zeros(1, layout.TEXTURE)
    buf.view(np.uint8)[:32] = np.frombuffer(b[:32], np.uint8)
    header = buf[0]
    off, sizes, chunks = 32, [], []
    for _ in range(int(header["mip_count"])):
        w, h = np.frombuffer(b[off:off + 8], np.uint32)
        off += 8
        n = (int(w) + 1) * (int(h) + 1) * layout.TEXEL_QUAD.itemsize
        chunks.append(np.frombuffer(b[off:off + n], layout.TEXEL_QUAD))
        off += n
        sizes.append((int(w), int(h)))
    return header, sizes, np.concatenate(chunks)


def reference_bake_texture(bgr, flags, layout):
    """The reference's own converter (oracle/_ref/bmp2texture) on 8-bit
    BGR(A) rows: the image goes through a BMP file and the switches the
    flags name (-l -m -w -n -c)."""
    import subprocess
    import tempfile
    img = np.ascontiguousarray(bgr, dtype=np.uint8)
    if (img.shape[1] * img.shape[2]) % 4:
        raise ValueError("the reference's BMP loader needs rows of a multiple of 4 bytes")
    switches = [s for bit, s in ((layout.IMAGE_LINEAR, "-l"), (layout.IMAGE_MIPMAP, "-m"), (layout.IMAGE_WRAP, "-w"),
                                 (layout.IMAGE_NORMAL, "-n"), (layout.IMAGE_CUBEMAP, "-c")) if flags & bit]
    with tempfile.TemporaryDirectory() as d:
        bmp, tex = Path(d) / "t.bmp", Path(d) / "t.texture"
        write_bmp(bmp, img)
        subprocess.run([str(BMP2TEXTURE), str(bmp), str(tex), *switches], check=True, timeout=600)
        return read_texture_file(tex, layout)


def make_canvas(width, height, antialias, layout):
    """Host framebuffer + CanvasData record (draw/canvas.h:11-17)."""
    s = 2 if antialias == 2 else 1
    pixels = np.zeros((height * s * width * s, 4), np.float32)
    depths = np.full(height * width * (1 if antialias == 0 else 4), np.inf, np.float32)
    cv = np.zeros((), layout.CANVAS_DATA)
    cv["width_times_height"] = width * height
    cv["f_width"], cv["f_height"] = width, height
    cv["h_width"], cv["h_height"] = width * 0.5, height * 0.5
    cv["width_over_height"], cv["height_over_width"] = width / height, height / width
    cv["width"], cv["height"], cv["stride"] = width, height, width
    cv["antialias"] = antialias
    cv["pixels"], cv["depths"] = pixels.ctypes.data, depths.ctypes.data
    return cv, pixels, depths


def oracle_render(scene, projection, settings, width, height, antialias=0, rows=None, cones_per_pixel=False,
                  count=False, layout=None, threads=1):
    """Renders with the C restatement; returns (pixels, depths, counters).

    threads > 1 (or 0: every host core) renders 8-row chunks of the rows on
    that many host threads (ctypes releases the GIL around the call; the
    oracle keeps all state per call and every pixel is written by the call
    that owns its row), each with its own counters, summed at the end."""
    cv, pixels, depths = make_canvas(width, height, antialias, layout)
    s = 2 if antialias == 2 else 1
    r0, r1 = (0, height * s) if rows is None else rows
    threads = threads or os.cpu_count() or 1
    h = oracle()
    if threads <= 1 or r1 - r0 <= 8:
        counters = np.zeros(14, np.uint64) if count else None
        rc = h.oracle_render(scene.ptr, _ptr(cv), _ptr(projection), _ptr(settings), r0, r1, int(cones_per_pixel),
                             _ptr(counters))
        assert rc == 0, rc
        work = None if counters is None else dict(zip(WORK_FIELDS, (int(c) for c in counters)))
        return pixels, depths, work
    from concurrent.futures import ThreadPoolExecutor
    chunks = [(y, min(r1, y + 8)) for y in range(r0, r1, 8)]
    per = [np.zeros(14, np.uint64) if count else None for _ in chunks]

    def run(k):
        a, b = chunks[k]
        return h.oracle_render(scene.ptr, _ptr(cv), _ptr(projection), _ptr(settings), a, b, int(cones_per_pixel),
                               _ptr(per[k]))

    with ThreadPoolExecutor(max_workers=threads) as ex:
        rcs = list(ex.map(run, range(len(chunks))))
    assert all(rc == 0 for rc in rcs), rcs
    work = None
    if count:
        total = np.sum(np.stack(per), axis=0, dtype=np.uint64)
        work = dict(zip(WORK_FIELDS, (int(c) for c in total)))
    return pixels, depths, work


def reference_render(scene, projection, settings, width, height, antialias=0, rows=None, threads=None, layout=None,
                     lib=None):
    cv, pixels, depths = make_canvas(width, height, antialias, layout)
    s = 2 if antialias == 2 else 1
    r0, r1 = (0, height * s) if rows is None else rows
    threads = threads or os.cpu_count() or 1
    rc = (lib or reference()).ref_render(scene.ptr, _ptr(cv), _ptr(projection), _ptr(settings), r0, r1, threads)
    assert rc == 0, rc
    return pixels, depths


def reference_render_cpu(scene, projection, settings, width, height, layout=None, lib=None):
    """The reference's unmodified single-threaded renderOnCPU."""
    cv, pixels, depths = make_canvas(width, height, 0, layout)
    rc = (lib or reference()).ref_render_cpu(scene.ptr, _ptr(cv), _ptr(projection), _ptr(settings))
    assert rc == 0, rc
    return pixels, depths


def _primary(fn, scene, projection, width, height, *extra):
    n = width * height
    g = np.zeros(n, np.int32)
    p = np.zeros(n, np.uint32)
    d = np.zeros(n, np.float32)
    b = np.zeros(n, np.uint8)
    rc = fn(scene.ptr, _ptr(projection), width, height, _ptr(g), _ptr(p), _ptr(d), _ptr(b), *extra)
    assert rc == 0, rc
    return g, p, d, b


def oracle_trace_primary(scene, projection, width, height, threads=1):
    """Closest primary hits by the C restatement; threads > 1 (0: every host
    core) traces 8-row chunks concurrently."""
    threads = threads or os.cpu_count() or 1
    if threads <= 1:
        return _primary(oracle().oracle_trace_primary, scene, projection, width, height)
    from concurrent.futures import ThreadPoolExecutor
    n = width * height
    g, p, d, b = np.zeros(n, np.int32), np.zeros(n, np.uint32), np.zeros(n, np.float32), np.zeros(n, np.uint8)
    h = oracle()

    def run(y):
        return h.oracle_trace_primary_rows(scene.ptr, _ptr(projection), width, y, min(height, y + 8), _ptr(g), _ptr(p),
                                           _ptr(d), _ptr(b))

    with ThreadPoolExecutor(max_workers=threads) as ex:
        rcs = list(ex.map(run, range(0, height, 8)))
    assert all(rc == 0 for rc in rcs), rcs
    return g, p, d, b


def reference_trace_primary(scene, projection, width, height, threads=None):
    return _primary(reference().ref_trace_primary, scene, projection, width, height, threads or os.cpu_count() or 1)


def reference_projection(camera, width, height, ssaa, layout, lib=None):
    out = np.zeros((), layout.PROJECTION)
    o = np.ascontiguousarray(camera.orientation, np.float32)
    p = np.ascontiguousarray(camera.position, np.float32)
    rc = (lib or reference()).ref_projection_reset(_ptr(o), _ptr(p), C.c_float(camera.focal_length), width, height,
                                                   int(ssaa), _ptr(out))
    assert rc == 0
    return out


def reference_scene_bvh(scene, layout):
    """Runs the reference's Scene BVH build on a copy of the scene data;
    returns (nodes, leaf_ids, flags, height)."""
    g = int(scene.data["counts"][0])
    nodes = np.zeros(2 * g, layout.BVH_NODE)
    leaf = np.zeros(g, np.uint32)
    sd = scene.data.copy()
    sd["bvh_nodes"], sd["bvh_leaf_geometry_indices"] = nodes.ctypes.data, leaf.ctypes.data
    rc = reference().ref_build_scene_bvh(_ptr(sd))
    assert rc == 0
    return nodes[:int(sd["bvh_node_count"])], leaf, int(sd["flags"]), int(sd["bvh_height"])


def reference_build_mesh(positions, indices, normals=None, normal_indices=None, uvs=None, uv_indices=None,
                         layout=None, lib=None):
    pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    idx = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
    t = len(idx)
    nrm = None if normals is None else np.ascontiguousarray(normals, np.float32)
    nidx = None if normal_indices is None else np.ascontiguousarray(normal_indices, np.uint32)
    uv = None if uvs is None else np.ascontiguousarray(uvs, np.float32)
    uidx = None if uv_indices is None else np.ascontiguousarray(uv_indices, np.uint32)
    tris = np.zeros(t, layout.TRIANGLE)
    nodes = np.zeros(2 * t + 2, layout.BVH_NODE)
    nc = np.zeros(1, np.uint32)
    ht = np.zeros(1, np.uint32)
    aabb = np.zeros(6, np.float32)
    out_pos = np.zeros_like(pos)
    rc = (lib or reference()).ref_build_mesh(_ptr(pos), len(pos), _ptr(idx), t, _ptr(nrm), 0 if nrm is None else len(nrm),
                                    _ptr(nidx), _ptr(uv), 0 if uv is None else len(uv), _ptr(uidx), _ptr(tris),
                                    _ptr(nodes), _ptr(nc), _ptr(ht), _ptr(aabb), _ptr(out_pos))
    assert rc == 0
    return tris, nodes[:int(nc[0])], int(ht[0]), aabb, out_pos


def reference_scene_record_sizes():
    """sizeof Camera, OrientationUsing3x3Matrix, Grid, Box, Curve,
    SceneCounts, ImageInfo, Geometry in the reference build."""
    h = reference()
    out = np.zeros(8, np.uint32)
    h.ref_scene_record_sizes.argtypes = [P]
    h.ref_scene_record_sizes(_ptr(out))
    return [int(x) for x in out]


def _reference_scene_data(scene_file_record, layout):
    """A reference SceneData pointing at the arrays of a SlimSceneFile record
    (the members save/load read: counts, cameras, geometries, meshes,
    textures, grids, boxes, curves)."""
    sd = np.zeros((), layout.SCENE_DATA)
    sd["counts"] = scene_file_record["counts"]
    for k in ("cameras", "geometries", "meshes", "textures", "grids", "boxes", "curves"):
        sd[k] = scene_file_record[k]
    return sd


def reference_save_scene(scene_file, path, layout):
    """The reference's save(Scene&, SceneIO&) on a SceneFile's arrays."""
    h = reference()
    h.ref_save_scene.argtypes = [P, C.c_char_p]
    rec = scene_file.record()
    sd = _reference_scene_data(rec, layout)
    rc = h.ref_save_scene(_ptr(sd), str(path).encode())
    assert rc == 0


def reference_load_scene(path, like, layout):
    """The reference's load(Scene&, SceneIO&) into fresh arrays shaped like
    the SceneFile `like` (its counts, mesh counts and mip sizes), returned
    as a SceneFile.  The reference sizes these arrays from the mesh and
    texture files its app loads before the scene file."""
    import copy
    from slimtracincpp_b200.scene import MeshAsset, TextureAsset
    from slimtracincpp_b200.scene_file import SceneFile
    meshes = []
    for m in like.meshes:
        z = lambda a: None if a is None else np.zeros_like(a)
        meshes.append(MeshAsset(np.zeros_like(m.triangles), np.zeros_like(m.nodes), np.zeros(3), np.zeros(3), 0,
                                np.zeros_like(m.positions), np.zeros_like(m.position_indices), z(m.normals),
                                z(m.normal_indices), z(m.uvs), z(m.uv_indices), np.zeros_like(m.edges)))
    textures = [TextureAsset(np.zeros((), layout.TEXTURE), t.mip_sizes, np.zeros_like(t.quads)) for t in like.textures]
    out = SceneFile(np.zeros_like(like.geometries), meshes, textures, np.zeros_like(like.cameras),
                    np.zeros_like(like.grids), np.zeros_like(like.boxes), np.zeros_like(like.curves))
    rec = out.record()
    sd = _reference_scene_data(rec, layout)
    h = reference()
    h.ref_load_scene.argtypes = [P, C.c_char_p]
    rc = h.ref_load_scene(_ptr(sd), str(path).encode())
    assert rc == 0
    # the reference wrote the headers into the records: carry them back
    for i, m in enumerate(out.meshes):
        r = out._mesh_records[i]
        m.aabb_min, m.aabb_max, m.height = r["aabb_min"].copy(), r["aabb_max"].copy(), int(r["bvh_height"])
    for i, t in enumerate(out.textures):
        r = out._texture_records[i]
        for k in ("width", "height", "size", "stride", "tile_width", "tile_height", "mip_count", "flags"):
            t.header[k] = r[k]
    return out
