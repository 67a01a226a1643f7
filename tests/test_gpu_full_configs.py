"""GPU parity at the full sizes of the measured workloads, through the C ABI,
against the CPU oracle run on every host core.

  config 1  640x360, depth 1, implicit primitives;
  config 2  1920x1080, depth 2, 8 mesh instances (81,920- and 130,050-triangle
            meshes, BVH heights 17-19), rendered after every instance moved
            and the device scene BVH was refit on the GPU (the frame the
            benchmark times), both through slimRenderOnGPU (host canvas) and
            slimRenderToDevice (device canvas, row bands in flight);
  config 3  1920x1080, depth 8, glass/mirror, 1024^2 albedo and normal maps
            with full mip chains, 512^2 sky cube IBL.

The reference rebuilds the scene BVH on the host every frame
(scene/scene.h:176-191); the GPU frame keeps the uploaded topology and refits
its bounds.  Closest hits keep the first of equally distant candidates in
visiting order (scene/scene_tracer.h:129, mesh_tracer.h:37), so a different
topology may only change which of two EQUALLY distant surfaces wins: primary
ids must match except at such ties, on at most 0.01% of pixels, and every
mismatch must be a tie (same distance).

Bars: ids bit-exact (ties as above), distances within 1e-5 relative, 8-bit
pixels within 1 LSB on >= 99.9% of pixels.
"""
import numpy as np
import pytest

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200 import native, scenes
from slimtracincpp_b200.renderer import RayTracingRenderer, Viewport, make_canvas
from slimtracincpp_b200.scene import quat_y
from oracle import bindings as O

from test_gpu_parity import (ENGINES, assert_depths_close, assert_float_pixels_close, assert_pixels_close,
                             gpu_primary, renderer_for)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def oracle_frame(w, proj=None):
    return O.oracle_render(w.scene, proj if proj is not None else w.projection(), w.settings, w.width, w.height,
                           layout=L, threads=0)


def assert_primary_ids_match(w, proj, allow_ties=False):
    g, p, d, b = gpu_primary(w.scene, proj, w.width, w.height)
    og, op, od, ob = O.oracle_trace_primary(w.scene, proj, w.width, w.height, threads=0)
    differ = (g != og) | (p != op)
    if not allow_ties:
        assert not differ.any(), f"{int(differ.sum())} primary ids differ"
        assert np.array_equal(b, ob)
        assert np.array_equal(d.view(np.uint32), od.view(np.uint32))
        return
    assert differ.mean() <= 1e-4, f"{int(differ.sum())} primary ids differ ({differ.mean():.2e} of pixels)"
    # every differing id is a tie: the same distance
    assert np.array_equal(d[differ].view(np.uint32), od[differ].view(np.uint32))
    same = ~differ
    assert np.array_equal(d[same].view(np.uint32), od[same].view(np.uint32))
    assert np.array_equal(b[same], ob[same])


@pytest.mark.parametrize("engine", ENGINES)
def test_config1_full_size(engine):
    native.set_render_options(engine=engine)
    w = scenes.config1(0)
    assert (w.width, w.height) == (640, 360)
    r = renderer_for(w)
    pix, dep = r.render(Viewport(w.camera, w.width, w.height))
    opix, odep, _ = oracle_frame(w)
    assert_pixels_close(pix, opix, w.width, w.height)
    assert_depths_close(dep, odep)
    assert_float_pixels_close(pix, opix)
    assert_primary_ids_match(w, w.projection())
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)


def move_instances(scene, seed):
    """Every geometry of the scene gets a new seeded rigid transform and
    scale, as an app moving its instances between frames would."""
    rng = np.random.default_rng(seed)
    geos = scene.geometries
    for i in range(len(geos)):
        if geos[i]["type"] != L.GEOMETRY_MESH:
            continue
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        geos[i]["axis"], geos[i]["amount"] = q[:3].astype(np.float32), np.float32(q[3])
        geos[i]["position"] = geos[i]["position"] + rng.uniform(-1.0, 1.0, 3).astype(np.float32)
        geos[i]["scale"] = geos[i]["scale"] * np.float32(rng.uniform(0.8, 1.25))


@pytest.fixture(scope="module")
def config2_workload():
    return scenes.config2(0)


def refit_expected(scene, old_nodes, old_leaf_ids):
    """The bounds a refit of the OLD topology must give for the scene's
    current geometries: every leaf gets its geometry's world AABB as
    Scene::updateAABB computes it (scene/scene.h:165-174; read here from the
    leaves of the reference's own rebuild of the moved scene), every inner
    node the union of its children (AABB::operator+, math/vec3.h:471-480)."""
    nodes, leaf_ids, _, _ = O.reference_scene_bvh(scene, L) if O.reference_available() else _host_rebuild(scene)
    box = {}
    for n in nodes:
        if n["leaf_count"]:
            gi = int(leaf_ids[n["first_index"]])
            box[gi] = (n["min"].copy(), n["max"].copy())
    assert len(box) == len(scene.geometries)
    out = old_nodes.copy()
    for i in range(len(out) - 1, -1, -1):
        if out[i]["leaf_count"]:
            out[i]["min"], out[i]["max"] = box[int(old_leaf_ids[out[i]["first_index"]])]
        else:
            c = int(out[i]["first_index"])
            out[i]["min"] = np.where(out[c]["min"] < out[c + 1]["min"], out[c]["min"], out[c + 1]["min"])
            out[i]["max"] = np.where(out[c]["max"] > out[c + 1]["max"], out[c]["max"], out[c + 1]["max"])
    return out


def _host_rebuild(scene):
    """The library's host restatement of the reference's rebuild (bit-exact
    against it) on a copy of the scene's BVH arrays."""
    saved = scene.bvh_nodes.copy(), scene.leaf_ids.copy(), scene.data.copy()
    scene.build_bvh()
    out = scene.bvh_nodes[:int(scene.data["bvh_node_count"])].copy(), scene.leaf_ids.copy(), 0, 0
    scene.bvh_nodes[:], scene.leaf_ids[:] = saved[0], saved[1]
    scene.data[...] = saved[2]
    return out


def download_scene_bvh(scene):
    sd = scene.data.copy()
    nodes = np.zeros(int(sd["bvh_node_count"]), L.BVH_NODE)
    sd["bvh_nodes"] = nodes.ctypes.data
    native.check(native.lib().slimDownloadSceneBVH(native.ptr(sd)))
    return nodes


def test_refit_bounds_match_reference_aabbs(config2_workload):
    """slimRefitSceneBVH's node bounds equal Scene::updateAABBs' world AABBs
    (transform.h:33-48) on the uploaded topology: unmoved, and after every
    instance moved twice."""
    w = config2_workload
    scene = w.scene
    RayTracingRenderer(scene, max_depth=2)
    n = int(scene.data["bvh_node_count"])
    old_nodes, old_leaf = scene.bvh_nodes[:n].copy(), scene.leaf_ids.copy()
    saved = scene.geometries.copy()
    try:
        native.check(native.lib().slimRefitSceneBVH(None))
        got = download_scene_bvh(scene)
        for k in ("min", "max", "first_index", "leaf_count"):
            assert np.array_equal(got[k], old_nodes[k]), k
        for seed in (11, 12):
            move_instances(scene, seed)
            native.check(native.lib().slimUploadGeometries(scene.ptr))
            native.check(native.lib().slimRefitSceneBVH(None))
            got = download_scene_bvh(scene)
            want = refit_expected(scene, old_nodes, old_leaf)
            for k in ("min", "max", "first_index", "leaf_count"):
                assert np.array_equal(got[k], want[k]), k
    finally:
        scene.geometries[:] = saved
        scene.build_bvh()


@pytest.mark.parametrize("entry", ["render_on_gpu", "render_to_device"])
def test_config2_full_size_after_moves_and_gpu_refit(config2_workload, entry):
    """The benchmark's frame: instances moved, geometries uploaded, the scene
    BVH refit on the GPU, the 1080p frame rendered (wavefront engine, the
    library default); the oracle renders the same moved scene with the
    reference's host rebuild of the scene BVH."""
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    w = config2_workload
    scene = w.scene
    assert (w.width, w.height, int(w.settings["max_depth"])) == (1920, 1080, 2)
    assert sum(m.triangle_count for m in scene.meshes) == 211970
    r = renderer_for(w)                       # uploads the unmoved scene and its host-built BVH
    saved = scene.geometries.copy()
    try:
        move_instances(scene, 21)
        lib = native.lib()
        native.check(lib.slimUploadGeometries(scene.ptr))
        native.check(lib.slimRefitSceneBVH(None))
        proj = w.projection()
        if entry == "render_on_gpu":
            cv, pix, dep = make_canvas(w.width, w.height, L.AA_NONE)
            native.check(lib.slimRenderOnGPU(native.ptr(cv), native.ptr(proj), native.ptr(r.settings)))
        else:
            n = w.width * w.height
            dp = torch.empty((n, 4), dtype=torch.float32, device="cuda")
            dd = torch.empty(n, dtype=torch.float32, device="cuda")
            r.render_to_device(Viewport(w.camera, w.width, w.height), dp.data_ptr(), dd.data_ptr(), 0)
            torch.cuda.synchronize()
            pix, dep = dp.cpu().numpy(), dd.cpu().numpy()
        gpu_ids = gpu_primary(scene, proj, w.width, w.height)
        scene.build_bvh()                      # the reference's per-frame host rebuild, for the oracle
        opix, odep, _ = oracle_frame(w, proj)
        assert_pixels_close(pix, opix, w.width, w.height)
        assert_depths_close(dep, odep)
        assert_float_pixels_close(pix, opix)
        og, op, od, ob = O.oracle_trace_primary(scene, proj, w.width, w.height, threads=0)
        g, p, d, b = gpu_ids
        differ = (g != og) | (p != op)
        assert differ.mean() <= 1e-4, f"{int(differ.sum())} primary ids differ"
        assert np.array_equal(d.view(np.uint32), od.view(np.uint32))
        assert np.array_equal(b[~differ], ob[~differ])
        assert (og >= 0).mean() > 0.1           # the moved instances still cover a good part of the frame
    finally:
        scene.geometries[:] = saved
        scene.build_bvh()


@pytest.fixture(scope="module")
def config3_workload():
    return scenes.config3(0)


@pytest.mark.parametrize("engine", ENGINES)
def test_config3_full_size(config3_workload, engine):
    """1080p glass/mirror + 1024^2 textures + sky IBL at bounce depth 8."""
    native.set_render_options(engine=engine)
    w = config3_workload
    assert (w.width, w.height, int(w.settings["max_depth"])) == (1920, 1080, 8)
    assert [t.mip_sizes[0] for t in w.scene.textures[:6]] == [(1024, 1024)] * 6
    assert len(w.scene.textures[0].mip_sizes) == 9
    r = renderer_for(w)
    pix, dep = r.render(Viewport(w.camera, w.width, w.height))
    opix, odep, _ = oracle_frame(w)
    assert_pixels_close(pix, opix, w.width, w.height)
    assert_depths_close(dep, odep)
    assert_float_pixels_close(pix, opix)
    if engine == L.ENGINE_WAVEFRONT:
        assert_primary_ids_match(w, w.projection())
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)


def test_config4_plain_depth8_full_size(config2_workload):
    """The radiance cache's reference image: config 2's scene at depth 8,
    1080p, plain wavefront frame."""
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    w = config2_workload
    r = RayTracingRenderer(w.scene, max_depth=8)
    pix, dep = r.render(Viewport(w.camera, w.width, w.height))
    st = L.default_settings(max_depth=8)
    opix, odep, _ = O.oracle_render(w.scene, w.projection(), st, w.width, w.height, layout=L, threads=0)
    assert_pixels_close(pix, opix, w.width, w.height)
    assert_depths_close(dep, odep)
    assert_float_pixels_close(pix, opix)


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("antialias", [L.AA_MSAA, L.AA_SSAA])
def test_config1_full_size_antialiased(engine, antialias):
    """Config 1 at 640x360 with the canvas's MSAA (depths for four samples
    per pixel, draw/canvas.h:128-185) and SSAA (four samples per pixel,
    renderer_GPU.h:23-25) layouts, against the oracle."""
    native.set_render_options(engine=engine)
    w = scenes.config1(0)
    r = renderer_for(w)
    pix, dep = r.render(Viewport(w.camera, w.width, w.height, antialias))
    ssaa = antialias == L.AA_SSAA
    proj = w.camera.projection(w.width, w.height, ssaa)
    opix, odep, _ = O.oracle_render(w.scene, proj, w.settings, w.width, w.height, antialias=antialias, layout=L,
                                    threads=0)
    s = 2 if ssaa else 1
    assert_pixels_close(pix, opix, s * w.width, s * w.height)
    assert_depths_close(dep, odep)
    assert_float_pixels_close(pix, opix)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)


def test_queue_overflow_and_light_batches_match_oracle():
    """Config 2's scene at 640x360 with a 1 MiB queue budget: the shadow queue
    holds one ray per sample, so the 4 lights go in 4 batches; the candidate
    queue holds 21,845 pairs (closest-hit candidates stop at three quarters of
    that), far fewer than the primary rays that reach a mesh instance, so
    most rays are traced whole by k_extend_overflow and the shadow rays whose
    pairs do not fit walk their instances inline.  The frame is bit-identical
    to the one with the default budget and matches the oracle."""
    w = scenes.config2(0, 640, 360)
    r = renderer_for(w)
    vp = Viewport(w.camera, w.width, w.height)
    def shadow_launches():
        return {s["name"]: s["launches"] for s in native.stage_stats()}["shadow"]

    try:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, row_bands=1, profile_stages=True)
        native.reset_stage_stats()
        pix, dep = r.render(vp)
        plain = shadow_launches()
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, row_bands=1, shadow_queue_mb=1, profile_stages=True)
        native.reset_stage_stats()
        spix, sdep = r.render(vp, update_scene=False)
        batched = shadow_launches()
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    assert batched == 4 * plain                 # one light per batch
    assert np.array_equal(spix, pix) and np.array_equal(sdep, dep)
    opix, odep, _ = oracle_frame(w)
    assert_pixels_close(spix, opix, w.width, w.height)
    assert_depths_close(sdep, odep)
    assert_float_pixels_close(spix, opix)
