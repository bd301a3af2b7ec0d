"""Stage entry points of the pipeline (the parity harness and callers that run part of it)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, _check, _CConfig, Configuration
from ._abi import ptr


def preprocess(x, device: int = 0):
    """preprocess_x non-PCA branch (lib.rs:485-511) -> (x', min, max, column mean)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, d = x.shape
    out = np.zeros_like(x)
    mn, mx = C.c_float(0), C.c_float(0)
    mean = np.zeros(d, np.float32)
    _check(_abi.lib().pacmap_preprocess(ptr(x), n, d, device, ptr(out), C.byref(mn), C.byref(mx), ptr(mean)))
    return out, mn.value, mx.value, mean


def pca_axes(cov, k: int):
    """Initialization::Pca's eigen-step (host): the k leading eigenvectors of a symmetric matrix (d x k)."""
    cov = np.ascontiguousarray(cov, dtype=np.float64)
    d = cov.shape[0]
    out = np.zeros((d, k), np.float64)
    _check(_abi.lib().pacmap_pca_axes(ptr(cov), d, k, ptr(out)))
    return out


def generate_pairs(x, config: Configuration):
    """sample_pairs with Generate (lib.rs:641-648 -> neighbors.rs:56-108) -> (pair_nn, pair_mn, pair_fp)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, d = x.shape
    cc = _CConfig(config, n)
    counts = np.zeros(3, np.uint64)
    _check(_abi.lib().pacmap_generate_pairs(ptr(x), n, d, C.byref(cc.c), ptr(counts), None, None, None))
    k, n_mn, n_fp = (int(v) for v in counts)
    pnn = np.zeros((n * k, 2), np.uint32)
    pmn = np.zeros((n * n_mn, 2), np.uint32)
    pfp = np.zeros((n * n_fp, 2), np.uint32)
    _check(_abi.lib().pacmap_generate_pairs(ptr(x), n, d, C.byref(cc.c), ptr(counts), ptr(pnn), ptr(pmn), ptr(pfp)))
    return pnn, pmn, pfp


def reselect_neighbors(knn_idx, knn_dist, k: int, device: int = 0):
    """sigma + scale_dist + sample_neighbors_pair (neighbors.rs:79-89) -> (pair_neighbors, sigma)."""
    ki = np.ascontiguousarray(knn_idx, dtype=np.uint32)
    kd = np.ascontiguousarray(knn_dist, dtype=np.float32)
    n, kp = ki.shape
    out = np.zeros((n * k, 2), np.uint32)
    sig = np.zeros(n, np.float32)
    _check(_abi.lib().pacmap_reselect_neighbors(ptr(ki), ptr(kd), n, kp, k, device, ptr(out), ptr(sig)))
    return out, sig


def sample_pairs(xp, pair_neighbors, k: int, n_mn: int, n_fp: int, seed: int, device: int = 0):
    """MN and FP sampling (sampling.rs:77-142) on the library's Philox stream -> (pair_mn, pair_fp)."""
    xp = np.ascontiguousarray(xp, dtype=np.float32)
    n, d = xp.shape
    pn = np.ascontiguousarray(pair_neighbors, dtype=np.uint32)
    pmn = np.zeros((n * n_mn, 2), np.uint32)
    pfp = np.zeros((n * n_fp, 2), np.uint32)
    _check(_abi.lib().pacmap_sample_pairs(ptr(xp), n, d, ptr(pn), k, n_mn, n_fp, seed & (2**64 - 1), device,
                                          ptr(pmn) if n_mn else None, ptr(pfp) if n_fp else None))
    return pmn, pfp


def optimize_steps(y, m, v, pnn, pmn, pfp, lr: float, p1: int, p2: int, itr_begin: int, itr_end: int,
                   device: int = 0, want_grad: bool = True):
    """Iterations [itr_begin, itr_end) of the optimiser from (y, m, v), updated in place.

    Returns the (n+1) x dim gradient of the last iteration (loss at [n, 0]) when want_grad.
    """
    n, dim = y.shape
    for a in (y, m, v):
        assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    pnn, pmn, pfp = (np.ascontiguousarray(p, dtype=np.uint32).reshape(-1, 2) for p in (pnn, pmn, pfp))
    g = np.zeros((n + 1, dim), np.float32) if want_grad else None
    _check(_abi.lib().pacmap_optimize_steps(ptr(y), ptr(m), ptr(v), n, dim, ptr(pnn), pnn.shape[0], ptr(pmn),
                                            pmn.shape[0], ptr(pfp), pfp.shape[0], lr, p1, p2, itr_begin, itr_end,
                                            device, ptr(g)))
    return g


def init_value(v, device: int = 0):
    """Initialization::Value normalisation (lib.rs:753-766) on the device."""
    v = np.ascontiguousarray(v, dtype=np.float32)
    out = np.zeros_like(v)
    _check(_abi.lib().pacmap_init_value(ptr(v), v.shape[0], v.shape[1], device, ptr(out)))
    return out


def init_random(n: int, dim: int, seed: int, device: int = 0):
    """Initialization::Random(seed) on the library's Philox stream."""
    out = np.zeros((n, dim), np.float32)
    _check(_abi.lib().pacmap_init_random(n, dim, seed & (2**64 - 1), device, ptr(out)))
    return out


def gradient(y, pnn, pmn, pfp, w_nn: float, w_mn: float, w_fp: float, device: int = 0):
    """pacmap_grad (gradient.rs:35-74) with explicit weights -> (n+1) x dim, loss at [n, 0]."""
    y = np.ascontiguousarray(y, dtype=np.float32)
    n, dim = y.shape
    pnn, pmn, pfp = (np.ascontiguousarray(p, dtype=np.uint32).reshape(-1, 2) for p in (pnn, pmn, pfp))
    g = np.zeros((n + 1, dim), np.float32)
    _check(_abi.lib().pacmap_gradient(ptr(y), n, dim, ptr(pnn), pnn.shape[0], ptr(pmn), pmn.shape[0], ptr(pfp),
                                      pfp.shape[0], w_nn, w_mn, w_fp, device, ptr(g)))
    return g
