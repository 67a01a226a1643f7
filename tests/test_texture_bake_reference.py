"""The texture bakers against the reference's own converter: the unmodified
src/bmp2texture.cpp (bmp2texture.cpp:24-335), compiled by
oracle/build_ref.sh into oracle/_ref/bmp2texture, run on BMP files written
here.  The host baker (slimBakeTexture) must write the same .texture bytes
for every switch the converter takes for 2D images and cube strips:
gamma (no switch), -l linear, -w wrap, -m mip chain, -n normal map (Z
derived), -c cube map, on 24- and 32-bit BMPs stored bottom-up and top-down,
sizes down to 1 pixel.  The GPU baker (slimBakeTextureOnGPU) is checked
against the same files where a GPU is present."""
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200.scene import TextureAsset

TOOL = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "bmp2texture"
needs_tool = pytest.mark.skipif(not TOOL.exists(), reason="oracle/_ref/bmp2texture not built (needs the reference)")

SWITCHES = {
    "gamma": ([], 0),
    "linear": (["-l"], L.IMAGE_LINEAR),
    "wrap": (["-w"], L.IMAGE_WRAP),
    "mip": (["-m"], L.IMAGE_MIPMAP),
    "mip_wrap": (["-m", "-w"], L.IMAGE_MIPMAP | L.IMAGE_WRAP),
    "mip_linear": (["-m", "-l"], L.IMAGE_MIPMAP | L.IMAGE_LINEAR),
    "normal": (["-n", "-l"], L.IMAGE_NORMAL | L.IMAGE_LINEAR),
    "normal_mip_wrap": (["-n", "-m", "-w", "-l"], L.IMAGE_NORMAL | L.IMAGE_MIPMAP | L.IMAGE_WRAP | L.IMAGE_LINEAR),
}
SIZES = [(1, 1), (3, 2), (5, 7), (16, 16), (33, 17), (64, 48), (128, 128)]


def write_bmp(path, bgr, top_down=False):
    """A BMP of 8-bit B,G,R(,A) components (rows padded to 4 bytes only for
    24-bit images, as the format requires)."""
    h, w, ch = bgr.shape
    rows = bgr if top_down else bgr[::-1]
    stride = (w * ch + 3) // 4 * 4
    data = bytearray()
    for r in rows:
        line = r.tobytes()
        data += line + b"\0" * (stride - len(line))
    off = 14 + 40
    head = struct.pack("<2sIHHI", b"BM", off + len(data), 0, 0, off)
    info = struct.pack("<IiiHHIIiiII", 40, w, -h if top_down else h, 1, 8 * ch, 0, len(data), 2835, 2835, 0, 0)
    Path(path).write_bytes(head + info + bytes(data))


def reference_texture(tmp_path, bgr, switches, top_down=False, name="t"):
    bmp = tmp_path / f"{name}.bmp"
    out = tmp_path / f"{name}.texture"
    write_bmp(bmp, bgr, top_down)
    if out.exists():
        out.unlink()
    subprocess.run([str(TOOL), str(bmp), str(out), *switches], check=True, timeout=120)
    return out.read_bytes()


def ours(bgr, flags, on_gpu=False, tmp_path=None, name="o"):
    t = TextureAsset.bake(bgr, flags, on_gpu=on_gpu)
    p = tmp_path / f"{name}.texture"
    t.save(p)
    return p.read_bytes()


def row_padding_free(w, ch):
    """The reference reads width * channels bytes per row with no row
    padding, so 24-bit rows must already be 4-byte multiples."""
    return (w * ch) % 4 == 0


@needs_tool
@pytest.mark.parametrize("name", list(SWITCHES))
def test_host_baker_matches_reference_converter(name, tmp_path):
    switches, flags = SWITCHES[name]
    rng = np.random.default_rng(abs(hash(name)) % 1000)
    checked = 0
    for (w, h) in SIZES:
        for ch in (3, 4):
            if not row_padding_free(w, ch):
                continue
            img = rng.integers(0, 256, (h, w, ch), dtype=np.uint8)
            for top_down in (False, True):
                ref = reference_texture(tmp_path, img, switches, top_down)
                assert ours(img, flags | (L.IMAGE_ALPHA if ch == 4 else 0), tmp_path=tmp_path) == ref, \
                    (name, w, h, ch, top_down)
                checked += 1
    assert checked >= 8


# Cube strips of these heights.  The converter writes two texel quads past
# the end of the main strip's quad array when it fills the seams
# (bmp2texture.cpp:100,126 size a quad row as (w + 1) * 4 where the strip has
# 4w + 1 quads), a heap overflow whose effect depends on the allocator: with
# glibc at h = 16 it lands on texel 10 of the top face's texel array, which
# the converter has already allocated, and changes that texel's four
# corners.  The bakers here keep their writes in bounds, so heights whose
# overflow reaches a live array are not comparable; 4, 8, 12, 24 and 32 are.
CUBE_HEIGHTS = [4, 8, 12, 24, 32]


@needs_tool
@pytest.mark.parametrize("h", CUBE_HEIGHTS)
def test_cube_strip_matches_reference_converter(h, tmp_path):
    rng = np.random.default_rng(h)
    img = rng.integers(0, 256, (h, 6 * h, 3), dtype=np.uint8)
    for switches, flags in ((["-c", "-l"], L.IMAGE_CUBEMAP | L.IMAGE_LINEAR), (["-c"], L.IMAGE_CUBEMAP),
                            (["-c", "-l", "-m", "-w"], L.IMAGE_CUBEMAP | L.IMAGE_LINEAR | L.IMAGE_MIPMAP | L.IMAGE_WRAP)):
        ref = reference_texture(tmp_path, img, switches)
        assert ours(img, flags, tmp_path=tmp_path) == ref, (h, switches)


@needs_tool
@pytest.mark.gpu
@pytest.mark.parametrize("name", ["gamma", "mip_wrap", "normal_mip_wrap"])
def test_gpu_baker_matches_reference_converter(name, tmp_path):
    switches, flags = SWITCHES[name]
    rng = np.random.default_rng(7)
    for (w, h), ch in (((64, 48), 3), ((33, 17), 4), ((128, 128), 3), ((1, 1), 4)):
        img = rng.integers(0, 256, (h, w, ch), dtype=np.uint8)
        ref = reference_texture(tmp_path, img, switches)
        got = ours(img, flags | (L.IMAGE_ALPHA if ch == 4 else 0), on_gpu=True, tmp_path=tmp_path)
        assert got == ref, (name, w, h, ch)
    for h in (8, 32):
        cube = rng.integers(0, 256, (h, 6 * h, 3), dtype=np.uint8)
        assert ours(cube, L.IMAGE_CUBEMAP | L.IMAGE_LINEAR, on_gpu=True, tmp_path=tmp_path) == \
            reference_texture(tmp_path, cube, ["-c", "-l"])
