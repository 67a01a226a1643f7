"""GPU: batched requests (slimBatch*) against rendering every request on its
own through the single-frame path.

Bars:
  * a request without the radiance cache renders bit-identically (pixels and
    depths) in a batch and alone: the stage kernels run the same per-path
    arithmetic, only the queues are shared;
  * the wave split (queue capacity, tile size) and the graph replay change
    nothing in the output;
  * the project autotuner returns a timed plan that renders the same frame;
  * requests with the radiance cache stay close to their plain frames.
"""
import numpy as np
import pytest

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200 import native, scenes
from slimtracincpp_b200.batch import BatchRenderer
from slimtracincpp_b200.radiance_cache import RadianceCache
from slimtracincpp_b200.renderer import RayTracingRenderer, Viewport
from slimtracincpp_b200.scene import MeshAsset, Scene, geometry

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SIZES = [(80, 45), (160, 90), (96, 54), (240, 135), (64, 36)]


@pytest.fixture(scope="module")
def meshes():
    pos, idx, nrm = scenes.icosphere(3)
    ico = MeshAsset.build(pos, idx, nrm, idx)
    pos, idx, nrm = scenes.heightfield(np.random.default_rng(7), 48, 0.3)
    hf = MeshAsset.build(pos, idx, nrm, idx)
    return [ico, hf]


def make_requests(meshes, seed, count, cache_every=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        w, h = SIZES[i % len(SIZES)]
        depth = int(rng.integers(1, 7))
        use = L.CACHE_ON if cache_every and i % cache_every == 0 and depth >= 2 else L.CACHE_OFF
        out.append(scenes.batch_request(rng, meshes, w, h, depth, use, i))
    return out


def assets(meshes):
    return Scene(np.array([geometry(L.GEOMETRY_SPHERE, 0)]), np.array([L.default_material()]), meshes=meshes)


def outputs(reqs):
    return [(torch.zeros((q.samples, 4), dtype=torch.float32, device="cuda"),
             torch.full((q.samples,), float("inf"), dtype=torch.float32, device="cuda")) for q in reqs]


def render_batch(batch, reqs, plan=None, repeats=1):
    outs = outputs(reqs)
    batch.set_requests(reqs, [(p.data_ptr(), d.data_ptr()) for p, d in outs])
    if plan:
        batch.set_plan(*plan)
    for _ in range(repeats):
        batch.render()
    batch.synchronize()
    return [(p.cpu().numpy(), d.cpu().numpy()) for p, d in outs]


def render_alone(q):
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    r = RayTracingRenderer(q.scene, int(q.settings["max_depth"]))
    return r.render(Viewport(q.camera, q.width, q.height))


def test_batch_matches_single_frames(meshes):
    reqs = make_requests(meshes, 0, 7)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    got = render_batch(BatchRenderer(assets(meshes)), reqs)
    for q, (pix, dep) in zip(reqs, got):
        spix, sdep = render_alone(q)
        assert np.array_equal(pix.view(np.uint32), spix.view(np.uint32)), q.name
        assert np.array_equal(dep.view(np.uint32), sdep.view(np.uint32)), q.name


def test_wave_split_and_graph_replay_change_nothing(meshes):
    reqs = make_requests(meshes, 1, 5)
    batch = BatchRenderer(assets(meshes))
    big = render_batch(batch, reqs, plan=(1 << 20, 1 << 16, 256))
    assert batch.plan()["waves"] == 1
    small = render_batch(batch, reqs, plan=(8192, 1000, 128), repeats=3)
    plan = batch.plan()
    assert plan["waves"] > 5 and plan["graph_nodes"] > 0
    for (a, da), (b, db) in zip(big, small):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        assert np.array_equal(da.view(np.uint32), db.view(np.uint32))


def test_autotuner_picks_a_timed_plan(meshes):
    reqs = make_requests(meshes, 2, 6)
    batch = BatchRenderer(assets(meshes))
    ref = render_batch(batch, reqs, plan=(1 << 20, 1 << 16, 256))
    outs = outputs(reqs)
    batch.set_requests(reqs, [(p.data_ptr(), d.data_ptr()) for p, d in outs])
    plan = batch.tune()
    assert plan["tuned"] and plan["candidates"] >= 3 and plan["batch_ms"] > 0
    batch.render()
    batch.synchronize()
    for (p, d), (rp, rd) in zip(outs, ref):
        assert np.array_equal(p.cpu().numpy().view(np.uint32), rp.view(np.uint32))


def test_cache_requests_in_a_batch(meshes):
    reqs = make_requests(meshes, 3, 6, cache_every=2)
    batch = BatchRenderer(assets(meshes))
    RadianceCache.configure(cache_depth=2, train_samples=4096, batch=1024, seed=2)
    outs = outputs(reqs)
    batch.set_requests(reqs, [(p.data_ptr(), d.data_ptr()) for p, d in outs])
    for _ in range(20):
        batch.render()
    batch.synchronize()
    got = [(p.cpu().numpy(), d.cpu().numpy()) for p, d in outs]
    for q, (pix, dep) in zip(reqs, got):
        spix, sdep = render_alone(q)
        assert np.isfinite(pix).all()
        assert np.array_equal(dep.view(np.uint32), sdep.view(np.uint32)), q.name   # depth comes from vertex 1
        if q.radiance_cache == L.CACHE_OFF:
            assert np.array_equal(pix.view(np.uint32), spix.view(np.uint32)), q.name
        else:
            a = RayTracingRenderer.to_content(pix, q.width, q.height).astype(np.float64)
            b = RayTracingRenderer.to_content(spix, q.width, q.height).astype(np.float64)
            mse = np.mean((a - b) ** 2)
            assert mse == 0 or 10 * np.log10(255.0 ** 2 / mse) > 20.0, q.name


def _assert_matches_oracle(q, pix, dep):
    from oracle import bindings as O
    opix, odep, _ = O.oracle_render(q.scene, q.projection(), q.settings, q.width, q.height, layout=L, threads=0)
    a = RayTracingRenderer.to_content(pix, q.width, q.height).astype(np.int32)
    b = RayTracingRenderer.to_content(opix, q.width, q.height).astype(np.int32)
    within = (np.abs(a - b) <= 1).all(axis=-1).mean()
    assert within >= 0.999, f"{q.name}: only {within:.5f} of pixels within 1 LSB of the oracle"
    finite = np.isfinite(odep)
    assert np.array_equal(np.isfinite(dep), finite), q.name
    np.testing.assert_allclose(dep[finite], odep[finite], rtol=1e-5, atol=0, err_msg=q.name)


def test_batch_matches_oracle(meshes):
    """Every request of a batch against the CPU oracle on its own scene (the
    reference's per-pixel path, renderer/ray_tracer.h:144-161): 8-bit pixels
    within 1 LSB on >= 99.9% of pixels, depths within 1e-5 relative."""
    reqs = make_requests(meshes, 4, 8)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    got = render_batch(BatchRenderer(assets(meshes)), reqs, plan=(1 << 16, 4096, 256))
    for q, (pix, dep) in zip(reqs, got):
        _assert_matches_oracle(q, pix, dep)


def test_config5_shaped_batch_matches_oracle():
    """config 5's request generator with the full config-2 meshes (81,920
    and 130,050 triangles), at the two smallest resolutions; the requests
    without the radiance cache are checked against the oracle."""
    mesh_assets = scenes.config2_meshes()
    reqs = scenes.config5(5, count=8, meshes=mesh_assets, resolutions=[(320, 180), (640, 360)])
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    plain = [q for q in reqs if q.radiance_cache == L.CACHE_OFF]
    got = render_batch(BatchRenderer(assets(mesh_assets)), plain)
    for q, (pix, dep) in zip(plain, got):
        _assert_matches_oracle(q, pix, dep)


def test_persistent_batch_matches_oracle_and_fused_frames(meshes):
    """The persistent plan: every request without the cache is rendered by
    one persistent launch fed by a device pixel queue (warps refill lanes
    whose paths ended).  Its per-path arithmetic is the fused engine's, so
    each request equals its single frame rendered by the fused engine bit
    for bit, and the oracle within the usual bars; two replays of the
    captured graph change nothing."""
    reqs = make_requests(meshes, 6, 9)
    batch = BatchRenderer(assets(meshes))
    got = render_batch(batch, reqs, plan=(1 << 16, 4096, 256, True), repeats=2)
    plan = batch.plan()
    assert plan["persistent"] == 1 and plan["waves"] == 0
    for q, (pix, dep) in zip(reqs, got):
        native.set_render_options(engine=L.ENGINE_MEGAKERNEL)
        r = RayTracingRenderer(q.scene, int(q.settings["max_depth"]))
        spix, sdep = r.render(Viewport(q.camera, q.width, q.height))
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
        assert np.array_equal(pix.view(np.uint32), spix.view(np.uint32)), q.name
        assert np.array_equal(dep.view(np.uint32), sdep.view(np.uint32)), q.name
        _assert_matches_oracle(q, pix, dep)


def test_persistent_plan_beside_cache_waves(meshes):
    """Cache requests keep their waves while the plain requests run in the
    persistent launch on the second lane: the plain requests still match
    the wave plan's output bit for bit."""
    reqs = make_requests(meshes, 7, 6, cache_every=2)
    RadianceCache.configure(cache_depth=2, train_samples=2048, batch=1024, seed=3)
    batch = BatchRenderer(assets(meshes))
    a = render_batch(batch, reqs, plan=(1 << 16, 4096, 256, True))
    assert batch.plan()["waves"] >= 1
    for q, (pix, dep) in zip(reqs, a):
        assert np.isfinite(pix).all()
        if q.radiance_cache == L.CACHE_OFF:
            native.set_render_options(engine=L.ENGINE_MEGAKERNEL)
            r = RayTracingRenderer(q.scene, int(q.settings["max_depth"]))
            spix, _ = r.render(Viewport(q.camera, q.width, q.height))
            native.set_render_options(engine=L.ENGINE_WAVEFRONT)
            assert np.array_equal(pix.view(np.uint32), spix.view(np.uint32)), q.name
