"""Neural radiance cache over the library's slimRadianceCache* entry points.

    cache = RadianceCache.configure(cache_depth=2, train_samples=65536, batch=16384)
    native.set_render_options(radiance_cache=L.CACHE_ON)
    renderer.render(viewport)          # paths stop at vertex 2 and ask the cache

Queries and training steps take device pointers (e.g. torch tensors): 16
floats of features per sample in, a float4 (rgb, 0) per sample out.  The
network runs only on the GPU; there is no CPU path.
"""
from __future__ import annotations

import numpy as np

from . import layout as L
from .native import check, lib, ptr


class RadianceCache:
    @staticmethod
    def configure(cache_depth=2, train_samples=65536, batch=16384, seed=0, learning_rate=1e-2, beta1=0.9,
                  beta2=0.99, epsilon=1e-8, train=True, overlap=True, train_suffix=0):
        """train_suffix 0: training targets are full-depth paths traced by the
        tracer; k > 0: training paths are traced k bounces on and end in the
        cache's own answer (self-training)."""
        c = np.zeros((), L.CACHE_CONFIG)
        c["cache_depth"], c["train_samples"], c["batch"], c["seed"] = cache_depth, train_samples, batch, seed
        c["learning_rate"], c["beta1"], c["beta2"], c["epsilon"] = learning_rate, beta1, beta2, epsilon
        c["train"], c["overlap"] = int(bool(train)), int(bool(overlap))
        c["train_suffix"] = int(train_suffix)
        check(lib().slimRadianceCacheConfigure(ptr(c)))
        return RadianceCache()

    def config(self):
        c = np.zeros((), L.CACHE_CONFIG)
        check(lib().slimRadianceCacheGetConfig(ptr(c)))
        return c

    @property
    def weights(self):
        w = np.zeros(L.NRC_PARAMS, np.float32)
        check(lib().slimRadianceCacheGetWeights(ptr(w), L.NRC_PARAMS))
        return w

    @weights.setter
    def weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        check(lib().slimRadianceCacheSetWeights(ptr(w), len(w)))

    def save_state(self) -> bytes:
        """Checkpoint: header (magic, params, Adam steps, cache frames,
        config), then weights, first and second Adam moments."""
        buf = np.zeros(L.NRC_STATE_BYTES, np.uint8)
        check(lib().slimRadianceCacheSaveState(ptr(buf), buf.nbytes))
        return buf.tobytes()

    @staticmethod
    def load_state(state: bytes) -> "RadianceCache":
        """Configures the cache from a checkpoint and resumes its training."""
        buf = np.frombuffer(bytes(state), np.uint8).copy()
        check(lib().slimRadianceCacheLoadState(ptr(buf), buf.nbytes))
        return RadianceCache()

    @staticmethod
    def parse_state(state: bytes):
        """(header record, weights, first moments, second moments) of a checkpoint."""
        buf = np.frombuffer(bytes(state), np.uint8)
        h = buf[:L.CACHE_STATE_HEADER.itemsize].view(L.CACHE_STATE_HEADER)[0]
        f = buf[L.CACHE_STATE_HEADER.itemsize:L.NRC_STATE_BYTES].view(np.float32)
        n = L.NRC_PARAMS
        return h, f[:n], f[n:2 * n], f[2 * n:3 * n]

    def gradients(self):
        g = np.zeros(L.NRC_PARAMS, np.float32)
        check(lib().slimRadianceCacheGetGradients(ptr(g), L.NRC_PARAMS))
        return g

    def query(self, d_features, count, d_radiance, stream=0):
        check(lib().slimRadianceCacheQuery(int(d_features), int(count), int(d_radiance), int(stream)))

    def train(self, d_features, d_targets, count, stream=0):
        check(lib().slimRadianceCacheTrain(int(d_features), int(d_targets), int(count), int(stream)))

    def join(self, stream=0):
        """Make `stream` wait for the overlapped training."""
        check(lib().slimRadianceCacheJoin(int(stream)))

    def stats(self):
        s = np.zeros((), L.CACHE_STATS)
        check(lib().slimRadianceCacheGetStats(ptr(s)))
        return {k: s[k].item() for k in ("frames", "steps", "queries", "train_samples", "loss")}
