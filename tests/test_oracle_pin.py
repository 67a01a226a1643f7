"""Pins the CPU oracle (oracle/slim_oracle.c) to the reference.

  * against the committed golden cases, which the reference's own code
    produced (tests/golden/make_golden.py): bit-exact pixels, depths and
    primary-hit ids/distances;
  * against the reference compiled here (oracle/_ref), when present, on
    more seeded scenes: bit-exact as well (same compiler, same flags).
"""
from pathlib import Path

import numpy as np
import pytest

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200 import scenes
from oracle import bindings as O

GOLDEN = Path(__file__).resolve().parent / "golden"
RENDER_CASES = sorted(p.stem for p in GOLDEN.glob("render_*.npz"))


def _golden_scene(name):
    import sys
    sys.path.insert(0, str(GOLDEN))
    from golden_io import load_scene
    z = np.load(GOLDEN / f"{name}.npz")
    scene, cam = load_scene(z)
    return z, scene, cam


def test_golden_cases_exist():
    assert len(RENDER_CASES) >= 6


@pytest.mark.parametrize("name", RENDER_CASES)
def test_oracle_matches_reference_golden(name):
    z, scene, cam = _golden_scene(name)
    settings = z["settings"].view(L.SETTINGS).reshape(())
    proj = z["projection"].view(L.PROJECTION).reshape(())
    w, h, aa = int(z["width"]), int(z["height"]), int(z["antialias"])
    pix, dep, _ = O.oracle_render(scene, proj, settings, w, h, antialias=aa, layout=L)
    assert np.array_equal(pix.view(np.uint32), z["pixels"].view(np.uint32))
    assert np.array_equal(dep.view(np.uint32), z["depths"].view(np.uint32))
    s = 2 if aa == L.AA_SSAA else 1
    g, p, d, b = O.oracle_trace_primary(scene, proj, w * s, h * s)
    assert np.array_equal(g, z["geometry_ids"])
    assert np.array_equal(p, z["primitive_ids"])
    assert np.array_equal(d.view(np.uint32), z["distances"].view(np.uint32))
    assert np.array_equal(b, z["from_behind"])


def test_golden_frames_are_not_trivial():
    z, _, _ = _golden_scene("render_features")
    pix = z["pixels"][:, :3]
    assert (pix > 0).any(axis=1).mean() > 0.3
    assert len(np.unique(z["geometry_ids"])) >= 8


needs_ref = pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (needs reference sources)")


@needs_ref
@pytest.mark.parametrize("make", [
    lambda: scenes.config1(0, 160, 90),
    lambda: scenes.config1(5, 96, 54),
    lambda: scenes.small_mesh_scene(3, 96, 54),
    lambda: scenes.feature_scene(1, 96, 54),
    lambda: scenes.feature_scene(2, 64, 36, max_depth=8),
    lambda: scenes.small_textured_scene(3, 96, 54),
], ids=["config1", "config1_s5", "mesh", "features", "features_d8", "textured_ibl"])
def test_oracle_matches_reference_live(make):
    w = make()
    proj = w.projection()
    rp, rd = O.reference_render(w.scene, proj, w.settings, w.width, w.height, layout=L)
    op, od, _ = O.oracle_render(w.scene, proj, w.settings, w.width, w.height, layout=L)
    assert np.array_equal(rp.view(np.uint32), op.view(np.uint32))
    assert np.array_equal(rd.view(np.uint32), od.view(np.uint32))


@needs_ref
@pytest.mark.parametrize("mode", [L.RENDER_NORMALS, L.RENDER_DEPTH, L.RENDER_UVS, L.RENDER_MIP_LEVEL,
                                  L.RENDER_NORMAL_MAP])
def test_oracle_debug_modes_match_reference(mode):
    w = scenes.small_textured_scene(3, 64, 36)
    st = L.default_settings(max_depth=4, render_mode=mode)
    proj = w.projection()
    rp, rd = O.reference_render(w.scene, proj, st, w.width, w.height, layout=L)
    op, od, _ = O.oracle_render(w.scene, proj, st, w.width, w.height, layout=L)
    assert np.array_equal(rp.view(np.uint32), op.view(np.uint32))
    assert np.array_equal(rd.view(np.uint32), od.view(np.uint32))


@needs_ref
def test_ssaa_matches_reference():
    w = scenes.feature_scene(4, 48, 27)
    proj = w.camera.projection(w.width, w.height, True)
    rp, rd = O.reference_render(w.scene, proj, w.settings, w.width, w.height, antialias=L.AA_SSAA, layout=L)
    op, od, _ = O.oracle_render(w.scene, proj, w.settings, w.width, w.height, antialias=L.AA_SSAA, layout=L)
    assert np.array_equal(rp.view(np.uint32), op.view(np.uint32))
    assert np.array_equal(rd.view(np.uint32), od.view(np.uint32))


@needs_ref
def test_reference_cpu_loop_close_to_per_pixel_directions():
    """renderOnCPU steps directions incrementally (renderer/renderer.h:91-94)
    while d_render computes start + down*y + right*x; the two differ only by
    rounding, so the 8-bit frames agree almost everywhere."""
    w = scenes.config1(2, 96, 54)
    proj = w.projection()
    a, _ = O.reference_render_cpu(w.scene, proj, w.settings, w.width, w.height, layout=L)
    b, _ = O.reference_render(w.scene, proj, w.settings, w.width, w.height, layout=L)
    to8 = lambda p: (np.float32(255) * np.sqrt(np.clip(p[:, :3], 0, 1))).astype(np.int32)
    assert (np.abs(to8(a) - to8(b)) <= 1).all(axis=1).mean() > 0.99
