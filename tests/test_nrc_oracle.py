"""The radiance cache's CPU restatement (oracle/nrc_oracle.py) checked on its
own: its analytic backward pass against finite differences, its encoding's
spherical harmonics against their orthonormality, and the C-ABI record sizes.
The GPU kernels are checked against this oracle in test_gpu_nrc.py."""
import numpy as np
import pytest

from oracle import nrc_oracle as N
from slimtracincpp_b200 import layout as L


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
    return N.pack(mats)


def test_param_count_matches_the_abi():
    assert N.N_PARAMS == L.NRC_PARAMS == 18624
    assert L.CACHE_CONFIG.itemsize == 48 and L.CACHE_STATS.itemsize == 32 and L.RENDER_OPTIONS.itemsize == 36


def test_backward_matches_finite_differences():
    """Exact (unrounded) mode: the analytic gradient of the log-radiance L2
    loss against central differences, for parameters of every layer."""
    rng = np.random.default_rng(0)
    params = rand_params(rng).astype(np.float64)
    f = rand_features(rng, 48)
    X = N.encode(f).astype(np.float64)
    target = rng.uniform(0.0, 2.0, (48, 4))
    grad, _ = N.gradients(params, f, target, rounding=False, X=X)
    logt = np.log(target[:, :3] + N.LOG_OFFSET)

    def surrogate(p):
        z = N.forward(p, X, rounding=False)["z"]
        return np.mean((z - logt) ** 2)

    bounds = np.cumsum([0] + [a * b for a, b in N.SHAPES])
    idx = np.concatenate([rng.choice(np.arange(bounds[i], bounds[i + 1]), 8, replace=False) for i in range(5)])
    for i in idx:
        e = 1e-6
        p1, p0 = params.copy(), params.copy()
        p1[i] += e
        p0[i] -= e
        fd = (surrogate(p1) - surrogate(p0)) / (2 * e)
        assert abs(fd - grad[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, grad[i])


def test_spherical_harmonics_are_orthonormal():
    rng = np.random.default_rng(1)
    d = rng.normal(size=(400000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    Y = N.sh_bands4(d)
    gram = 4 * np.pi * (Y.T @ Y) / len(d)
    assert np.abs(gram - np.eye(16)).max() < 0.03


def test_encoding_layout():
    f = np.zeros((1, 16), np.float32)
    f[0, 0:3] = [0.25, 0.5, 0.125]
    f[0, 3] = 0.7
    f[0, 4:7] = [0, 0, 1]
    f[0, 8:11] = [0, 1, 0]
    f[0, 12:15] = [0.1, 0.2, 0.3]
    X = N.encode(f)[0]
    # axis x = 0.25: octave 0 -> sin(pi/4), cos(pi/4); octave 1 -> sin(pi/2) = 1, cos(pi/2) = 0
    assert X[0] == X[1] == N.bf16(np.float32(np.sqrt(0.5)))
    assert X[2] == 1.0 and abs(X[3]) < 1e-7
    # axis y = 0.5 starts at column 24: octave 1 -> sin(pi) = 0, cos(pi) = -1
    assert X[24] == 1.0 and abs(X[27 - 1]) < 1e-7 and X[27] == -1.0
    assert X[72] == N.bf16(np.float32(0.28209479177387814))       # band 0
    assert X[74] == N.bf16(np.float32(0.48860251190291987))       # band 1, z
    assert X[95] == 1.0 and X[91] == N.bf16(np.float32(0.7))
    assert np.array_equal(X[88:91], [0, 1, 0]) and np.array_equal(X[92:95], N.bf16(np.float32([0.1, 0.2, 0.3])))
