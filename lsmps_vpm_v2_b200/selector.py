"""Learned (leaf caps, p) selector of the mixed 2D form (host side).

The network, its training and its inference run in libvpm_fmm.so
(include/vpm_fmm.h, "Learned (leaf caps, p) selector"); this module holds
the data plumbing: features, normalisation statistics, the weights file and
the choice of parameters for a particle set.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import Params, default_params, lib

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "selector_weights.npz")
N_FEAT = 228
N_CAND = 35
N_OUT = 2 * N_CAND
REFERENCE_PAIR = (50, 75, 10)   # global.cpp:311-313


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def candidates():
    """The 35 (cap, p) pairs in output order; max_src = cap, max_par = 3 cap / 2."""
    caps = np.zeros(N_CAND, np.int32)
    ps = np.zeros(N_CAND, np.int32)
    st = lib().vpm_selector_candidates(_p(caps), _p(ps), N_CAND)
    if st:
        raise RuntimeError("vpm_selector_candidates failed")
    return [(int(c), int(c) * 3 // 2, int(p)) for c, p in zip(caps, ps)]


def param_count() -> int:
    return int(lib().vpm_mlp_param_count())


class Selector:
    """The network of one context plus its normalisation statistics."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.in_mean = np.zeros(N_FEAT, np.float32)
        self.in_std = np.ones(N_FEAT, np.float32)
        self.out_mean = np.zeros(N_OUT, np.float32)
        self.out_std = np.ones(N_OUT, np.float32)

    # ---- parameters ----------------------------------------------------------
    def init(self, seed: int = 0):
        self.ctx._check(lib().vpm_mlp_init(self.ctx._h, seed))

    def set_params(self, params):
        w = np.ascontiguousarray(params, dtype=np.float32)
        self.ctx._check(lib().vpm_mlp_set_params(self.ctx._h, _p(w), w.size))

    def get_params(self) -> np.ndarray:
        w = np.zeros(param_count(), np.float32)
        self.ctx._check(lib().vpm_mlp_get_params(self.ctx._h, _p(w), w.size))
        return w

    def set_norm(self, in_mean, in_std, out_mean, out_std):
        self.in_mean, self.in_std = (np.ascontiguousarray(v, dtype=np.float32) for v in (in_mean, in_std))
        self.out_mean, self.out_std = (np.ascontiguousarray(v, dtype=np.float32) for v in (out_mean, out_std))
        self.ctx._check(lib().vpm_mlp_set_norm(self.ctx._h, _p(self.in_mean), _p(self.in_std), _p(self.out_mean),
                                               _p(self.out_std)))

    def save(self, path: str = WEIGHTS, **extra):
        np.savez(path, params=self.get_params(), in_mean=self.in_mean, in_std=self.in_std, out_mean=self.out_mean,
                 out_std=self.out_std, **extra)

    def load(self, path: str = WEIGHTS) -> bool:
        if not os.path.exists(path):
            return False
        f = np.load(path)
        self.set_params(f["params"])
        self.set_norm(f["in_mean"], f["in_std"], f["out_mean"], f["out_std"])
        return True

    # ---- kernels -------------------------------------------------------------
    def forward(self, X, bf16: bool = False) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((X.shape[0], N_OUT), np.float32)
        self.ctx._check(lib().vpm_mlp_forward(self.ctx._h, _p(X), X.shape[0], _p(Y), int(bf16)))
        return Y

    def grads(self, X, Y, mask=None):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        M = None if mask is None else np.ascontiguousarray(mask, dtype=np.float32)
        g = np.zeros(param_count(), np.float32)
        loss = C.c_float()
        self.ctx._check(lib().vpm_mlp_grads(self.ctx._h, _p(X), _p(Y), None if M is None else _p(M), X.shape[0],
                                            _p(g), C.byref(loss)))
        return float(loss.value), g

    def train(self, X, Y, mask=None, batch: int = 256, steps: int = 2000, lr: float = 1e-3, seed: int = 0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        M = None if mask is None else np.ascontiguousarray(mask, dtype=np.float32)
        hist = np.zeros(max(steps, 1), np.float32)
        self.ctx._check(lib().vpm_mlp_train(self.ctx._h, _p(X), _p(Y), None if M is None else _p(M), X.shape[0],
                                            min(batch, X.shape[0]), steps, lr, seed, _p(hist)))
        return hist[:steps]

    # ---- features and choice -------------------------------------------------
    def features(self, x, y, q, active, target_err: float) -> np.ndarray:
        x, y, q = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, q))
        a = np.ascontiguousarray(active, dtype=np.uint8)
        f = np.zeros(N_FEAT, np.float32)
        self.ctx._check(lib().vpm_selector_features2d(self.ctx._h, _p(x), _p(y), _p(q), _p(a), x.size,
                                                      float(target_err), _p(f)))
        return f

    def features_device(self, x, y, q, active, target_err: float) -> np.ndarray:
        """The same features from device arrays (torch CUDA tensors: float64
        x, y, q and uint8 active): the particles are not copied to the host;
        the 228 floats come back."""
        f = np.zeros(N_FEAT, np.float32)
        self.ctx._check(lib().vpm_selector_features2d_device(
            self.ctx._h, *[C.c_void_p(v.data_ptr()) for v in (x, y, q, active)], x.numel(), float(target_err), _p(f)))
        return f

    def choose(self, feat, target_err: float, margin: float = 0.3):
        """(max_src, max_par, p) and the 70 predictions for a feature vector."""
        f = np.ascontiguousarray(feat, dtype=np.float32)
        ms, mp, p = C.c_int32(), C.c_int32(), C.c_int32()
        pred = np.zeros(N_OUT, np.float32)
        self.ctx._check(lib().vpm_select2d(self.ctx._h, _p(f), float(target_err), float(margin), C.byref(ms),
                                           C.byref(mp), C.byref(p), _p(pred)))
        return (ms.value, mp.value, p.value), pred

    def params_for(self, x, y, q, active, target_err: float = 1e-4, margin: float = 0.3, **over) -> Params:
        """vpm_fmm_params of the mixed form with the chosen caps and order
        (host arrays, or torch CUDA tensors: the features are then computed
        from the device buffers)."""
        feat = (self.features_device(x, y, q, active, target_err) if hasattr(x, "data_ptr")
                else self.features(x, y, q, active, target_err))
        (ms, mp, p), _ = self.choose(feat, target_err, margin)
        prm = default_params(max_src=ms, max_par=mp, p=p, precision=1, binom=1)
        for k, v in over.items():
            setattr(prm, k, v)
        return prm
