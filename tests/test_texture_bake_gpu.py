"""bmp2texture's texel-quad baker on the GPU (slimBakeTextureOnGPU) against
the host baker (slimBakeTexture, itself byte-identical to the reference's
shipped .texture files in test_host.py): the same header, mip chain and
texel-quad bytes for every flag set, channel count and size, down to 1-pixel
images whose border writes overlap, and cube strips whose seam pass writes
past the strip."""
import numpy as np
import pytest

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200 import native
from slimtracincpp_b200.scene import TextureAsset

FLAG_SETS = {
    "gamma": 0,
    "linear": L.IMAGE_LINEAR,
    "wrap": L.IMAGE_LINEAR | L.IMAGE_WRAP,
    "mip_wrap": L.IMAGE_MIPMAP | L.IMAGE_WRAP,
    "mip_clamp": L.IMAGE_MIPMAP | L.IMAGE_LINEAR,
    "normal_mip": L.IMAGE_NORMAL | L.IMAGE_MIPMAP | L.IMAGE_LINEAR | L.IMAGE_WRAP,
    "normal_clamp": L.IMAGE_NORMAL,
}
SIZES = [(1, 1), (1, 3), (3, 1), (2, 2), (5, 3), (33, 17), (64, 48), (96, 160)]


def _header(t):
    h = t.header.copy()
    h["mips"] = 0
    return h.tobytes()


def _same(a, b):
    assert _header(a) == _header(b)
    assert a.mip_sizes == b.mip_sizes
    assert a.quads.tobytes() == b.quads.tobytes()


def test_gpu_baker_sizing_call_matches_the_host_baker():
    """The sizing call (no buffers) runs on the host: same header and counts."""
    rng = np.random.default_rng(3)
    for (w, h), flags, ch in [((64, 48), L.IMAGE_MIPMAP, 3), ((7, 5), L.IMAGE_WRAP, 4),
                              ((48, 8), L.IMAGE_CUBEMAP | L.IMAGE_WRAP | L.IMAGE_MIPMAP, 3)]:
        img = rng.integers(0, 256, (h, w, ch), dtype=np.uint8)
        counts = []
        for fn in (native.lib().slimBakeTexture, native.lib().slimBakeTextureOnGPU):
            mip_count = np.zeros(1, np.uint32)
            quad_count = np.zeros(1, np.uint32)
            header = np.zeros((), L.TEXTURE)
            native.check(fn(native.ptr(img), w, h, ch, flags, native.ptr(header), 0, 0, native.ptr(mip_count),
                            native.ptr(quad_count)))
            counts.append((header.tobytes(), int(mip_count[0]), int(quad_count[0])))
        assert counts[0] == counts[1]


def test_gpu_baker_refuses_what_the_host_baker_refuses():
    img = np.zeros((4, 20, 3), np.uint8)
    header = np.zeros((), L.TEXTURE)
    mc = np.zeros(1, np.uint32)
    qc = np.zeros(1, np.uint32)
    # a cube strip must be 6h x h
    rc = native.lib().slimBakeTextureOnGPU(native.ptr(img), 20, 4, 3, L.IMAGE_CUBEMAP, native.ptr(header), 0, 0,
                                           native.ptr(mc), native.ptr(qc))
    assert rc == 1
    rc = native.lib().slimBakeTextureOnGPU(native.ptr(img), 20, 4, 2, 0, native.ptr(header), 0, 0,
                                           native.ptr(mc), native.ptr(qc))
    assert rc == 1


@pytest.mark.gpu
@pytest.mark.parametrize("flags", list(FLAG_SETS))
@pytest.mark.parametrize("channels", [3, 4])
def test_gpu_baker_matches_the_host_baker(flags, channels):
    rng = np.random.default_rng(11)
    for w, h in SIZES:
        img = rng.integers(0, 256, (h, w, channels), dtype=np.uint8)
        _same(TextureAsset.bake(img, FLAG_SETS[flags], on_gpu=True), TextureAsset.bake(img, FLAG_SETS[flags]))


@pytest.mark.gpu
@pytest.mark.parametrize("face", [1, 2, 3, 8, 32])
@pytest.mark.parametrize("linear", [False, True])
def test_gpu_baker_matches_the_host_baker_on_cube_strips(face, linear):
    """6h x h strips: the main strip, top and bottom faces and their seams
    (bmp2texture -c, with and without -l); wrap, mip and normal flags are
    dropped for cube maps on both sides."""
    rng = np.random.default_rng(face)
    img = rng.integers(0, 256, (face, 6 * face, 3), dtype=np.uint8)
    flags = L.IMAGE_CUBEMAP | L.IMAGE_WRAP | (L.IMAGE_LINEAR if linear else 0)
    gpu = TextureAsset.bake(img, flags, on_gpu=True)
    _same(gpu, TextureAsset.bake(img, flags))
    assert gpu.mip_sizes == [(4 * face, face), (face, face), (face, face)]


@pytest.mark.gpu
def test_gpu_baker_on_a_1024_texture_with_mips():
    """A texture of the 1080p glass/mirror workload's size: 1024^2, wrapped,
    mip chain down to 4 x 4, albedo and normal map."""
    rng = np.random.default_rng(5)
    img = rng.integers(0, 256, (1024, 1024, 3), dtype=np.uint8)
    for flags in (L.IMAGE_MIPMAP | L.IMAGE_WRAP, L.IMAGE_MIPMAP | L.IMAGE_WRAP | L.IMAGE_NORMAL | L.IMAGE_LINEAR):
        gpu = TextureAsset.bake(img, flags, on_gpu=True)
        _same(gpu, TextureAsset.bake(img, flags))
        assert len(gpu.mip_sizes) == 9
