"""GPU: the radiance cache's tcgen05 kernels (through the C ABI) against the
CPU oracle (oracle/nrc_oracle.py), and the cache inside a wavefront frame.

Bars:
  * forward: the output z = log(radiance + 0.01) within 0.05 of the oracle's
    on every sample and within 5e-3 on 99 % (bf16 activations: an f32
    accumulation that lands on a bf16 rounding boundary may round the other
    way than the oracle's);
  * gradients: relative error of every layer's gradient below 2 %;
  * Adam: the update of the GPU gradient within f32 rounding of the oracle's;
  * EXACT cache mode (every query traced on by the tracer): the plain frame
    within 1 LSB on every pixel;
  * ablation: after online training the cache beats truncating the paths at
    the cache depth, in PSNR against the plain full-depth frame.
"""
import numpy as np
import pytest

from oracle import nrc_oracle as N
from slimtracincpp_b200 import layout as L
from slimtracincpp_b200 import native, scenes
from slimtracincpp_b200.radiance_cache import RadianceCache
from slimtracincpp_b200.renderer import RayTracingRenderer, Viewport

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def rand_features(rng, n):
    f = np.zeros((n, 16), np.float32)
    f[:, 0:3] = rng.uniform(0, 1, (n, 3))
    f[:, 3] = rng.uniform(0.05, 1, n)
    d = rng.normal(size=(n, 3))
    f[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nrm = rng.normal(size=(n, 3))
    f[:, 8:11] = nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    f[:, 12:15] = rng.uniform(0, 1, (n, 3))
    return f


def rand_params(rng, out_scale=0.5):
    mats = [rng.uniform(-1, 1, s) * np.sqrt(6.0 / s[1]) for s in N.SHAPES]
    mats[4] = mats[4] * out_scale
    return N.pack(mats).astype(np.float32)


def smooth_targets(f):
    p, n = f[:, 0:3], f[:, 8:11]
    t = np.zeros((len(f), 4), np.float32)
    t[:, 0] = 0.6 + 0.4 * np.sin(2 * np.pi * p[:, 0]) * np.cos(2 * np.pi * p[:, 2])
    t[:, 1] = 0.5 + 0.3 * n[:, 1] + 0.1 * p[:, 1]
    t[:, 2] = 0.3 + 0.25 * np.cos(3 * np.pi * p[:, 1]) * f[:, 12]
    return t


@pytest.fixture(scope="module")
def cache():
    w = scenes.feature_scene(0, 32, 18)
    RayTracingRenderer(w.scene, max_depth=2)
    return RadianceCache.configure(seed=1)


def gpu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def query(cache, f):
    df = gpu(f)
    out = torch.zeros((len(f), 4), dtype=torch.float32, device="cuda")
    cache.query(df.data_ptr(), len(f), out.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy()[:, :3]


@pytest.mark.parametrize("n", [1, 1000, 5000])
def test_query_matches_oracle(cache, n):
    rng = np.random.default_rng(n)
    params = rand_params(rng)
    cache.weights = params
    f = rand_features(rng, n)
    got = query(cache, f)
    ref = N.infer(params, f)
    # compared in the network's output space: log(radiance + 0.01) = z
    err = np.abs(np.log(got + N.LOG_OFFSET) - np.log(ref + N.LOG_OFFSET))
    assert err.max() < 0.05, err.max()
    assert np.quantile(err, 0.99) < 5e-3


@pytest.mark.parametrize("n", [1000, 16384])
def test_gradients_match_oracle(cache, n):
    rng = np.random.default_rng(10 + n)
    params = rand_params(rng)
    cache.weights = params
    f = rand_features(rng, n)
    t = rng.uniform(0, 2, (n, 4)).astype(np.float32)
    df, dt = gpu(f), gpu(t)
    cache.train(df.data_ptr(), dt.data_ptr(), n)
    torch.cuda.synchronize()
    g = cache.gradients()
    ref, loss = N.gradients(params, f, t)
    o = 0
    for r, c in N.SHAPES:
        a, b = g[o:o + r * c], ref[o:o + r * c]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel < 2e-2, (r, c, rel)
        o += r * c
    assert abs(cache.stats()["loss"] - loss) <= 1e-3 * loss


def test_adam_steps_match_oracle(cache):
    rng = np.random.default_rng(7)
    params = rand_params(rng)
    cache.weights = params               # also clears the moments
    f = rand_features(rng, 2048)
    t = rng.uniform(0, 2, (2048, 4)).astype(np.float32)
    df, dt = gpu(f), gpu(t)
    p, m, v = params.copy(), np.zeros_like(params), np.zeros_like(params)
    for step in (1, 2, 3):
        cache.train(df.data_ptr(), dt.data_ptr(), 2048)
        g = cache.gradients().astype(np.float64)
        p, m, v = N.adam(p, m, v, g, step)
        np.testing.assert_allclose(cache.weights, p, rtol=2e-5, atol=1e-7)


def test_online_training_fits_a_smooth_radiance(cache):
    rng = np.random.default_rng(3)
    cache.weights = rand_params(rng, out_scale=0.1)
    f = rand_features(rng, 65536)
    t = smooth_targets(f)
    df, dt = gpu(f), gpu(t)
    fv = rand_features(rng, 4096)
    tv = smooth_targets(fv)

    def val_loss():
        y = query(cache, fv)
        return float(np.mean((np.log(y + N.LOG_OFFSET) - np.log(tv[:, :3] + N.LOG_OFFSET)) ** 2))

    before = val_loss()
    for it in range(300):
        o = (it % 16) * 4096
        cache.train(df[o:].data_ptr(), dt[o:].data_ptr(), 4096)
    after = val_loss()
    assert after < 0.05 * before, (before, after)
    assert after < 5e-3


def renderer_for(w):
    st = w.settings
    return RayTracingRenderer(w.scene, int(st["max_depth"]), int(st["skybox_color_texture_id"]),
                              int(st["skybox_radiance_texture_id"]), int(st["skybox_irradiance_texture_id"]))


def to8(pixels, w, h):
    return RayTracingRenderer.to_content(pixels, w, h).astype(np.int32)


def psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 99.0 if mse == 0 else 10 * np.log10(255.0 ** 2 / mse)


@pytest.mark.parametrize("depth", [2, 3])
def test_exact_cache_mode_reproduces_the_plain_frame(depth):
    """Every query traced on from the cache vertex in its own slot and added
    back with the path throughput: only the summation order changes."""
    w = scenes.small_textured_scene(0, 96, 54, max_depth=6)
    r = renderer_for(w)
    vp = Viewport(w.camera, w.width, w.height)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    plain, pdep = r.render(vp)
    cache = RadianceCache.configure(cache_depth=depth, train=False)
    try:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_EXACT)
        exact, edep = r.render(vp)
        st = cache.stats()
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    assert st["queries"] > 20 and st["train_samples"] == st["queries"]
    assert np.array_equal(edep.view(np.uint32), pdep.view(np.uint32))
    a, b = to8(exact, w.width, w.height), to8(plain, w.width, w.height)
    assert np.abs(a - b).max() <= 1
    assert (np.abs(exact - plain) <= 1e-5).all(axis=1).mean() >= 0.999


def test_cache_beats_truncation_after_online_training():
    """Ablation: the same frame with the paths cut at vertex 2 and nothing
    added (TRUNCATE) against the trained cache's answer (ON), both measured
    against the plain depth-6 frame."""
    w = scenes.small_textured_scene(1, 128, 72, max_depth=6)
    r = renderer_for(w)
    vp = Viewport(w.camera, w.width, w.height)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    plain, _ = r.render(vp)
    ref = to8(plain, w.width, w.height)
    RadianceCache.configure(cache_depth=2, train_samples=4096, batch=512, seed=5)
    try:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_TRUNCATE)
        trunc, _ = r.render(vp)
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_ON)
        scores = []
        for frame in range(120):
            img, _ = r.render(vp, update_scene=False)
            scores.append(psnr(to8(img, w.width, w.height), ref))
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    p_trunc = psnr(to8(trunc, w.width, w.height), ref)
    assert scores[-1] > p_trunc + 3.0, (p_trunc, scores[0], scores[-1])
    assert scores[-1] > scores[0]


@pytest.mark.parametrize("suffix", [1, 2])
def test_self_training_cache_beats_truncation(suffix):
    """Training paths traced `suffix` bounces past the cache vertex that end
    in the cache's own answer there (the self-training targets): after online
    training the cache frame is closer to the plain frame than cutting the
    paths at vertex 2, and it improves as it trains."""
    w = scenes.small_textured_scene(1, 128, 72, max_depth=6)
    r = renderer_for(w)
    vp = Viewport(w.camera, w.width, w.height)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    plain, _ = r.render(vp)
    ref = to8(plain, w.width, w.height)
    cache = RadianceCache.configure(cache_depth=2, train_samples=4096, batch=512, seed=5, train_suffix=suffix)
    assert int(cache.config()["train_suffix"]) == suffix
    try:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_TRUNCATE)
        trunc, _ = r.render(vp)
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_ON)
        scores = []
        for frame in range(120):
            img, _ = r.render(vp, update_scene=False)
            scores.append(psnr(to8(img, w.width, w.height), ref))
        st = cache.stats()
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    assert st["train_samples"] > 0 and np.isfinite(st["loss"])
    p_trunc = psnr(to8(trunc, w.width, w.height), ref)
    assert scores[-1] > p_trunc + 3.0, (p_trunc, scores[0], scores[-1])
    assert scores[-1] > scores[0]


def test_banded_cache_frames_gather_every_band():
    """A 1080p-sized cache frame renders as two row bands whose queries meet
    in one cache phase (the query records carry their paths' colour and
    throughput).  Against the same frames rendered as one band: every depth
    and every pixel whose path ends before the cache vertex are bit-identical,
    all queries are answered (finite pixels, every pixel written), and both
    trained caches stay above 40 dB against the plain frame."""
    w = scenes.small_mesh_scene(2, 512, 512)
    w.settings = L.default_settings(max_depth=6)
    r = renderer_for(w)
    vp = Viewport(w.camera, w.width, w.height)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    plain, _ = r.render(vp)
    ref = to8(plain, w.width, w.height)
    out = {}
    try:
        for bands in (1, 2):
            cache = RadianceCache.configure(cache_depth=2, train_samples=8192, batch=2048, seed=4, train_suffix=1)
            native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_ON, row_bands=bands)
            for _ in range(40):
                img, dep = r.render(vp, update_scene=False)
            cache.join()
            img, dep = r.render(vp, update_scene=False)
            out[bands] = (img, dep, cache.stats()["queries"])
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    (a, da, qa), (b, db, qb) = out[1], out[2]
    assert qa == qb and qa > 100
    assert np.array_equal(da.view(np.uint32), db.view(np.uint32))
    assert np.isfinite(b).all() and (b[:, 3] == 1.0).all()
    same = (a.view(np.uint32) == b.view(np.uint32)).all(axis=1).mean()
    assert same >= 1.0 - qa / (w.width * w.height) - 1e-3, same
    # the bands gather queries in another order, so the training sets (and
    # weights) differ: both must still be well trained
    pa, pb = psnr(to8(a, w.width, w.height), ref), psnr(to8(b, w.width, w.height), ref)
    assert min(pa, pb) > 40.0, (pa, pb)


def test_checkpoint_resumes_training_exactly(cache):
    """slimRadianceCacheSaveState / LoadState: training continued from a
    restored checkpoint takes the same Adam steps, bit for bit, as training
    that never stopped; restoring the weights alone (moments cleared) does
    not."""
    rng = np.random.default_rng(11)
    c = RadianceCache.configure(seed=3, batch=4096, learning_rate=5e-3, train=False)
    f = [gpu(rand_features(rng, 4096)) for _ in range(5)]
    t = [gpu(rng.uniform(0, 2, (4096, 4)).astype(np.float32)) for _ in range(5)]
    for i in range(3):
        c.train(f[i].data_ptr(), t[i].data_ptr(), 4096)
    state = c.save_state()
    assert len(state) == L.NRC_STATE_BYTES
    h, w, m, v = RadianceCache.parse_state(state)
    assert h["magic"] == L.NRC_STATE_MAGIC and h["params"] == L.NRC_PARAMS and h["steps"] == 3
    assert h["config"]["seed"] == 3 and h["config"]["batch"] == 4096 and h["config"]["train"] == 0
    assert np.array_equal(w, c.weights) and np.any(m != 0) and np.all(v >= 0) and np.any(v > 0)

    def two_more_steps(cc):
        for i in (3, 4):
            cc.train(f[i].data_ptr(), t[i].data_ptr(), 4096)
        return cc.weights

    resumed_without_stop = two_more_steps(c)
    c2 = RadianceCache.load_state(state)
    assert c2.stats()["steps"] == 3 and np.array_equal(c2.weights, w)
    assert c2.config()["learning_rate"] == np.float32(5e-3)
    assert np.array_equal(two_more_steps(c2), resumed_without_stop)
    c2.weights = w                          # same weights, Adam state cleared
    assert not np.array_equal(two_more_steps(c2), resumed_without_stop)


def test_checkpoint_keeps_the_frame_counter():
    """Online training picks each frame's training set from the cache-frame
    counter; a restored checkpoint continues the count."""
    w = scenes.small_textured_scene(1, 64, 36, max_depth=4)
    r = renderer_for(w)
    vp = Viewport(w.camera, w.width, w.height)
    c = RadianceCache.configure(cache_depth=2, train_samples=1024, batch=256, seed=2, train_suffix=1, overlap=False)
    try:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_ON)
        for _ in range(3):
            r.render(vp, update_scene=False)
        s = c.stats()
        state = c.save_state()
        assert s["frames"] == 3 and s["steps"] > 0
        r.render(vp, update_scene=False)
        c2 = RadianceCache.load_state(state)
        assert c2.stats()["frames"] == 3 and c2.stats()["steps"] == s["steps"]
        assert c2.config()["train_suffix"] == 1 and c2.config()["overlap"] == 0
        img, _ = r.render(vp, update_scene=False)
        assert c2.stats()["frames"] == 4 and np.isfinite(img).all()
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
