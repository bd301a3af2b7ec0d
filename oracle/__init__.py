"""CPU oracle for the PaCMAP hot path -- TEST INFRASTRUCTURE ONLY.

numpy wrappers around ``oracle/pacmap_oracle.cpp`` (a C++ restatement of beamform/pacmap-rs v0.2.6;
each C function cites the reference file:line it follows). Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg import this package, and only as the checker: the product in
``pacmap-rs_b200/`` never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64 = C.c_uint64
_vp = C.c_void_p


class OracleError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"oracle {what} failed with status {code}")
        self.code = code


def _host_has_avx2() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " avx2 " in f" {line.strip()} " and " fma " in f" {line.strip()} "
    except OSError:
        pass
    return False


def build() -> None:
    """Compile the oracle libraries (make; no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    names = (["liboracle_avx2.so"] if _host_has_avx2() else []) + ["liboracle.so"]
    path = next((os.path.join(_HERE, n) for n in names if os.path.exists(os.path.join(_HERE, n))), None)
    if path is None:
        build()
        path = os.path.join(_HERE, names[0])
    L = C.CDLL(path)
    sig = {
        "orc_distance": (C.c_float, [_f32p, _f32p, _u64]),
        "orc_powi": (C.c_float, [C.c_float, C.c_int]),
        "orc_total_key": (C.c_uint32, [C.c_float]),
        "orc_philox4x32_10": (None, [_u32p, C.c_uint32, C.c_uint32, _u32p]),
        "orc_sample_stream": (None, [_u64, _u64, C.c_uint32, _u32p]),
        "orc_set_threads": (C.c_int, [C.c_int]),
        "orc_decide_num_pairs": (C.c_int, [_u64, C.c_int64, C.c_float, C.c_float, _u64p]),
        "orc_preprocess": (C.c_int, [_f32p, _u64, _u64, _f32p, _vp, _vp, _vp]),
        "orc_knn_exact": (C.c_int, [_f32p, _u64, _u64, _u64, _u32p, _f32p]),
        "orc_knn_exact_allpairs": (C.c_int, [_f32p, _u64, _u64, _u64, _u32p, _f32p]),
        "orc_knn_rows": (C.c_int, [_f32p, _u64, _u64, _u32p, _u64, _u64, _u32p, _f32p]),
        "orc_sigma": (None, [_f32p, _u64, _u64, _f32p]),
        "orc_scale_dist": (None, [_f32p, _f32p, _u32p, _u64, _u64, _f32p]),
        "orc_sample_neighbors_pair": (None, [_f32p, _u32p, _u64, _u64, _u64, _u32p]),
        "orc_sample_fp_pairs": (C.c_int, [_u32p, _u64, _u64, _u64, _u64, _u32p]),
        "orc_sample_mn_pairs": (C.c_int, [_f32p, _u64, _u64, _u64, _u64, _u32p]),
        "orc_weights": (None, [_u64, _u64, _u64, C.c_float, _f32p]),
        "orc_lr_t": (C.c_float, [C.c_float, _u64]),
        "orc_grad": (C.c_int, [_f32p, _u64, _u64, _u32p, _u64, _u32p, _u64, _u32p, _u64,
                               C.c_float, C.c_float, C.c_float, _f32p, _vp, _vp]),
        "orc_adam": (None, [_f32p, _f32p, _f32p, _f32p, _u64, C.c_float, _u64]),
        "orc_init_value": (C.c_int, [_f32p, _u64, _u64, _f32p]),
        "orc_init_random": (None, [_u64, _u64, _u64, _f32p]),
        "orc_optimize": (C.c_int, [_f32p, _u64, _u64, _u32p, _u64, _u32p, _u64, _u32p, _u64, C.c_float,
                                   _u64, _u64, _u64, _vp, _u64, _vp, _vp]),
        "orc_optimize_parallel": (C.c_int, [_f32p, _u64, _u64, _u32p, _u64, _u32p, _u64, _u32p, _u64, C.c_float,
                                            _u64, _u64, _u64]),
        "orc_step": (C.c_int, [_f32p, _f32p, _f32p, _u64, _u64, _u32p, _u64, _u32p, _u64, _u32p, _u64,
                               C.c_float, _u64, _u64, _u64, _vp, _vp, _vp]),
        "orc_generate_pairs": (C.c_int, [_f32p, _u64, _u64, _u64, _u64, _u64, _u64, _u32p, _u32p, _u32p]),
        "orc_knn_preservation": (C.c_double, [_f32p, _u64, _u64, _f32p, _u64, _u32p, _u64, _u64]),
        "orc_triplet_accuracy": (C.c_double, [_f32p, _u64, _f32p, _u64, _u32p, _u64]),
        "orc_fit_transform": (C.c_int, [_f32p, _u64, _u64, _u64, C.c_int, _vp, _u64, C.c_float, C.c_float,
                                        C.c_int64, _u64, C.c_float, _u64, _u64, _u64, _f32p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc, what):
    if rc != 0:
        raise OracleError(rc, what)


def set_threads(t: int) -> int:
    return lib().orc_set_threads(int(t))


def distance(a, b) -> float:
    a, b = _f32(a), _f32(b)
    return float(lib().orc_distance(a, b, a.size))


def powi(a: float, b: int) -> float:
    return float(lib().orc_powi(a, b))


def philox4x32_10(ctr, k0: int, k1: int) -> np.ndarray:
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(_u32(ctr), k0 & 0xFFFFFFFF, k1 & 0xFFFFFFFF, out)
    return out


def sample_stream(seed: int, point: int, count: int) -> np.ndarray:
    out = np.zeros(count, np.uint32)
    lib().orc_sample_stream(seed, point, count, out)
    return out


def decide_num_pairs(n: int, override=None, mn_ratio=0.5, fp_ratio=2.0):
    out = np.zeros(3, np.uint64)
    rc = lib().orc_decide_num_pairs(n, -1 if override is None else int(override), mn_ratio, fp_ratio, out)
    return rc, tuple(int(v) for v in out)


def preprocess(x):
    x = _f32(x)
    n, d = x.shape
    out = np.empty_like(x)
    mn = np.zeros(1, np.float32)
    mx = np.zeros(1, np.float32)
    mean = np.zeros(d, np.float32)
    _check(lib().orc_preprocess(x, n, d, out, _ptr(mn), _ptr(mx), _ptr(mean)), "preprocess")
    return out, float(mn[0]), float(mx[0]), mean


def knn_exact(x, k: int, allpairs: bool = False):
    x = _f32(x)
    n, d = x.shape
    kp = min(k, n - 1) if n > 0 else 0
    idx = np.zeros((n, kp), np.uint32)
    dist = np.zeros((n, kp), np.float32)
    fn = lib().orc_knn_exact_allpairs if allpairs else lib().orc_knn_exact
    _check(fn(x, n, d, k, idx, dist), "knn_exact")
    return idx, dist


def knn_rows(x, rows, k: int):
    """Rows ``rows`` of ``knn_exact(x, k)`` (same indices and f32 distances), without the full matrix."""
    x = _f32(x)
    n, d = x.shape
    rows = _u32(rows)
    kp = min(k, n - 1) if n > 0 else 0
    idx = np.zeros((rows.size, kp), np.uint32)
    dist = np.zeros((rows.size, kp), np.float32)
    _check(lib().orc_knn_rows(x, n, d, rows, rows.size, k, idx, dist), "knn_rows")
    return idx, dist


def sigma(knn_dist):
    kd = _f32(knn_dist)
    n, kp = kd.shape
    sig = np.zeros(n, np.float32)
    lib().orc_sigma(kd, n, kp, sig)
    return sig


def scale_dist(knn_dist, sig, nbrs):
    kd = _f32(knn_dist)
    n, kp = kd.shape
    out = np.zeros_like(kd)
    lib().orc_scale_dist(kd, _f32(sig), _u32(nbrs), n, kp, out)
    return out


def sample_neighbors_pair(scaled, nbrs, k: int):
    sc = _f32(scaled)
    n, kp = sc.shape
    out = np.zeros((n * k, 2), np.uint32)
    lib().orc_sample_neighbors_pair(sc, _u32(nbrs), n, kp, k, out)
    return out


def sample_fp_pairs(pair_neighbors, n: int, k: int, n_fp: int, seed: int):
    out = np.zeros((n * n_fp, 2), np.uint32)
    _check(lib().orc_sample_fp_pairs(_u32(pair_neighbors), n, k, n_fp, seed, out), "sample_fp_pairs")
    return out


def sample_mn_pairs(x, n_mn: int, seed: int):
    x = _f32(x)
    n, d = x.shape
    out = np.zeros((n * n_mn, 2), np.uint32)
    _check(lib().orc_sample_mn_pairs(x, n, d, n_mn, seed, out), "sample_mn_pairs")
    return out


def weights(itr: int, p1: int, p2: int, w_mn_init: float = 1000.0):
    out = np.zeros(3, np.float32)
    lib().orc_weights(itr, p1, p2, w_mn_init, out)
    return tuple(float(v) for v in out)  # (w_mn, w_nn, w_fp)


def lr_t(lr: float, itr: int) -> float:
    return float(lib().orc_lr_t(lr, itr))


def grad(y, pnn, pmn, pfp, w_nn, w_mn, w_fp, with64=False):
    y = _f32(y)
    n, dim = y.shape
    pnn, pmn, pfp = _u32(pnn).reshape(-1, 2), _u32(pmn).reshape(-1, 2), _u32(pfp).reshape(-1, 2)
    g = np.zeros((n + 1, dim), np.float32)
    g64 = np.zeros((n + 1, dim), np.float64) if with64 else None
    ab = np.zeros((n, dim), np.float32) if with64 else None
    _check(lib().orc_grad(y, n, dim, pnn, len(pnn), pmn, len(pmn), pfp, len(pfp), w_nn, w_mn, w_fp, g,
                          _ptr(g64), _ptr(ab)), "grad")
    return (g, g64, ab) if with64 else g


def adam(y, g, m, v, lr: float, itr: int):
    """In-place Adam step on float32 arrays y, m, v (g has >= n rows)."""
    n, dim = y.shape
    gg = _f32(g)[:n]
    lib().orc_adam(y, np.ascontiguousarray(gg), m, v, n * dim, lr, itr)


def init_value(v):
    v = _f32(v)
    n, dim = v.shape
    y = np.zeros_like(v)
    _check(lib().orc_init_value(v, n, dim, y), "init_value")
    return y


def init_random(n: int, dim: int, seed: int):
    y = np.zeros((n, dim), np.float32)
    lib().orc_init_random(n, dim, seed, y)
    return y


def optimize(y0, pnn, pmn, pfp, lr=1.0, num_iters=(100, 100, 250), snapshots=None, with_loss=False):
    y = np.array(y0, dtype=np.float32, copy=True, order="C")
    n, dim = y.shape
    pnn, pmn, pfp = _u32(pnn).reshape(-1, 2), _u32(pmn).reshape(-1, 2), _u32(pfp).reshape(-1, 2)
    snaps = None if snapshots is None else np.ascontiguousarray(snapshots, dtype=np.uint64)
    sout = None if snaps is None else np.zeros((len(snaps), n, dim), np.float32)
    loss = np.zeros(sum(num_iters), np.float32) if with_loss else None
    _check(lib().orc_optimize(y, n, dim, pnn, len(pnn), pmn, len(pmn), pfp, len(pfp), lr, *num_iters,
                              _ptr(snaps), 0 if snaps is None else len(snaps), _ptr(sout), _ptr(loss)), "optimize")
    return y, sout, loss


def optimize_parallel(y0, pnn, pmn, pfp, lr=1.0, num_iters=(100, 100, 250)):
    """The reference's parallel optimiser loop (gradient.rs:35-151 chunked private arrays + adam.rs) for the
    timed CPU baseline; its sums are ordered by thread, not pinned (use ``optimize`` for parity)."""
    y = np.array(y0, dtype=np.float32, copy=True, order="C")
    n, dim = y.shape
    pnn, pmn, pfp = _u32(pnn).reshape(-1, 2), _u32(pmn).reshape(-1, 2), _u32(pfp).reshape(-1, 2)
    _check(lib().orc_optimize_parallel(y, n, dim, pnn, len(pnn), pmn, len(pmn), pfp, len(pfp), lr, *num_iters),
           "optimize_parallel")
    return y


def step(y, m, v, pnn, pmn, pfp, lr, p1, p2, itr, with_grad=True):
    """One optimiser step in place on (y, m, v); returns (grad, grad64, abs_sum)."""
    n, dim = y.shape
    pnn, pmn, pfp = _u32(pnn).reshape(-1, 2), _u32(pmn).reshape(-1, 2), _u32(pfp).reshape(-1, 2)
    g = np.zeros((n + 1, dim), np.float32) if with_grad else None
    g64 = np.zeros((n + 1, dim), np.float64) if with_grad else None
    ab = np.zeros((n, dim), np.float32) if with_grad else None
    _check(lib().orc_step(y, m, v, n, dim, pnn, len(pnn), pmn, len(pmn), pfp, len(pfp), lr, p1, p2, itr,
                          _ptr(g), _ptr(g64), _ptr(ab)), "step")
    return g, g64, ab


def generate_pairs(xp, n_neighbors: int, n_mn: int, n_fp: int, seed: int):
    xp = _f32(xp)
    n, d = xp.shape
    k = min(n_neighbors, n - 1)
    pnn = np.zeros((n * k, 2), np.uint32)
    pmn = np.zeros((n * n_mn, 2), np.uint32)
    pfp = np.zeros((n * n_fp, 2), np.uint32)
    _check(lib().orc_generate_pairs(xp, n, d, n_neighbors, n_mn, n_fp, seed, pnn, pmn, pfp), "generate_pairs")
    return pnn, pmn, pfp


def knn_preservation(xh, yl, sample, k=10) -> float:
    xh, yl = _f32(xh), _f32(yl)
    n, d = xh.shape
    return float(lib().orc_knn_preservation(xh, n, d, yl, yl.shape[1], _u32(sample), len(sample), k))


def triplet_accuracy(xh, yl, triplets) -> float:
    xh, yl = _f32(xh), _f32(yl)
    t = _u32(triplets).reshape(-1, 3)
    return float(lib().orc_triplet_accuracy(xh, xh.shape[1], yl, yl.shape[1], t, len(t)))


def fit_transform(x, dim=2, init="random", init_value=None, init_seed=0, mn_ratio=0.5, fp_ratio=2.0,
                  override_neighbors=None, seed=0, lr=1.0, num_iters=(100, 100, 250)):
    x = _f32(x)
    n, d = x.shape
    out = np.zeros((n, dim), np.float32)
    kind = 1 if init == "value" else 2
    iv = None if init_value is None else _f32(init_value)
    _check(lib().orc_fit_transform(x, n, d, dim, kind, _ptr(iv), init_seed, mn_ratio, fp_ratio,
                                   -1 if override_neighbors is None else int(override_neighbors), seed, lr,
                                   *num_iters, out), "fit_transform")
    return out
