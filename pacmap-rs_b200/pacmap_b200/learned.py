"""The learned initialiser: an MLP d -> 512 -> 512 -> dim from preprocessed data to an embedding.

No counterpart in beamform/pacmap-rs. The reference accepts any starting embedding through
``Initialization::Value`` (src/lib.rs:753-766, z-scored to std 1e-4); this module trains a network on
the (x, embedding) pairs that a plain fit produces for one data generator, and starts new fits of the
same generator from its prediction, so that a shortened schedule (``SHORT_SCHEDULE``) replaces the
plain one (``PLAIN_SCHEDULE``). Training, inference and the gradient check all run on the GPU
(tcgen05 BF16 GEMMs with FP32 accumulation, AdamW) through the C ABI (include/pacmap.h).

``LearnedModel`` bundles a trained network with its training data's preprocessing constants and the
training embedding's scale: it is saved to and loaded from a file, and ``transform`` embeds points the
fit never saw into that embedding's coordinates (the reference cannot, README.md:165).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np

from . import Configuration, Initialization, _abi, _check, _CConfig, stages
from ._abi import ptr

PLAIN_SCHEDULE = (100, 100, 250)
SHORT_SCHEDULE = (0, 50, 150)
HIDDEN = 512


def param_count(d: int, dim: int) -> int:
    return int(_abi.lib().pacmap_mlp_param_count(d, dim))


def init_params(d: int, dim: int, seed: int = 0) -> np.ndarray:
    """Seeded U(-1/sqrt(fan_in), 1/sqrt(fan_in)) parameters in the flat layout
    [W1 (512 x d), b1, W2 (512 x 512), b2, W3 (dim x 512), b3]."""
    p = np.zeros(param_count(d, dim), np.float32)
    _check(_abi.lib().pacmap_mlp_init(d, dim, seed & (2**64 - 1), ptr(p)))
    return p


def train(params, xp, target, epochs: int = 20, batch: int = 4096, lr: float = 1e-3, weight_decay: float = 1e-4,
          seed: int = 0, device: int = 0):
    """AdamW on the mean-squared error between MLP(xp) and the per-dimension z-scored target.

    Returns (trained parameters, loss of each epoch)."""
    xp = np.ascontiguousarray(xp, dtype=np.float32)
    t = np.ascontiguousarray(target, dtype=np.float32)
    n, d = xp.shape
    dim = t.shape[1]
    p = np.array(params, dtype=np.float32, copy=True)
    assert p.size == param_count(d, dim), "parameter count does not match (d, dim)"
    losses = np.zeros(max(epochs, 1), np.float32)
    _check(_abi.lib().pacmap_mlp_train(ptr(xp), ptr(t), n, d, dim, epochs, batch, lr, weight_decay,
                                       seed & (2**64 - 1), device, ptr(p), ptr(losses)))
    return p, losses[:epochs]


def apply(params, xp, dim: int, device: int = 0) -> np.ndarray:
    """MLP(xp) (n x dim)."""
    xp = np.ascontiguousarray(xp, dtype=np.float32)
    n, d = xp.shape
    p = np.ascontiguousarray(params, dtype=np.float32)
    out = np.zeros((n, dim), np.float32)
    _check(_abi.lib().pacmap_mlp_apply(ptr(p), d, dim, ptr(xp), n, device, ptr(out)))
    return out


def gradient(params, xp, target, device: int = 0):
    """(loss, flat gradient) of the mean-squared error on one batch (rows a multiple of 128)."""
    xp = np.ascontiguousarray(xp, dtype=np.float32)
    t = np.ascontiguousarray(target, dtype=np.float32)
    B, d = xp.shape
    dim = t.shape[1]
    p = np.ascontiguousarray(params, dtype=np.float32)
    g = np.zeros(p.size, np.float32)
    loss = C.c_float(0)
    _check(_abi.lib().pacmap_mlp_grad(ptr(p), d, dim, ptr(xp), ptr(t), B, device, ptr(g), C.byref(loss)))
    return loss.value, g


def _stats_ptrs(target_stats):
    if target_stats is None:
        return None, None, ()
    mean, std = (np.ascontiguousarray(v, dtype=np.float32) for v in target_stats)
    return ptr(mean), ptr(std), (mean, std)


def fit_transform_learned(x, params, config: Optional[Configuration] = None, target_stats=None):
    """fit_transform (lib.rs:294-367) starting from the network's prediction.

    ``target_stats`` = (mean, std) of the training embedding (``target_stats(y_train)``): the fit starts from
    MLP(x') in that embedding's coordinates, so the predicted layout survives the first Adam steps. Without
    it, from MLP(x') through Initialization::Value (z-scored to std 1e-4, lib.rs:753-766).
    ``config.initialization`` is ignored; pass a shortened ``num_iters`` (``SHORT_SCHEDULE``)."""
    config = config or dataclasses.replace(Configuration(), num_iters=SHORT_SCHEDULE)
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, d = x.shape
    dim = int(config.embedding_dimensions)
    p = np.ascontiguousarray(params, dtype=np.float32)
    cc = _CConfig(dataclasses.replace(config, initialization=Initialization.Random(0)), n)
    out = np.zeros((n, dim), np.float32)
    snaps = None
    if config.snapshots is not None:
        snaps = np.zeros((len(config.snapshots), n, dim), np.float32)
    pm_, ps_, _keep = _stats_ptrs(target_stats)
    _check(_abi.lib().pacmap_fit_transform_learned(ptr(x), n, d, C.byref(cc.c), ptr(p), pm_, ps_, ptr(out),
                                                   ptr(snaps)))
    return out, snaps


def fit_transform_learned_device(x_ptr: int, n: int, d: int, out_ptr: int, params, config: Configuration,
                                 snapshots_ptr: Optional[int] = None, target_stats=None) -> None:
    """fit_transform_learned on device memory (raw CUDA pointers); params and target_stats stay host arrays."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    cc = _CConfig(dataclasses.replace(config, initialization=Initialization.Random(0)), n)
    pm_, ps_, _keep = _stats_ptrs(target_stats)
    _check(_abi.lib().pacmap_fit_transform_learned_device(C.c_void_p(x_ptr), n, d, C.byref(cc.c), ptr(p), pm_, ps_,
                                                          C.c_void_p(out_ptr),
                                                          C.c_void_p(snapshots_ptr) if snapshots_ptr else None))


@dataclasses.dataclass
class LearnedModel:
    """A trained initialiser plus what ``transform`` needs: ``params`` (flat MLP layout), the training
    data's preprocessing constants (``pre_min``, ``pre_max``, ``pre_mean``: preprocess_x's min, max and
    column means) and the training embedding's per-dimension ``target_mean`` / ``target_std``."""

    params: np.ndarray
    d: int
    dim: int
    pre_min: float
    pre_max: float
    pre_mean: np.ndarray
    target_mean: np.ndarray
    target_std: np.ndarray

    def save(self, path: str) -> None:
        _check(_abi.lib().pacmap_model_save(str(path).encode(), self.d, self.dim, ptr(_f32(self.params)),
                                            float(self.pre_min), float(self.pre_max), ptr(_f32(self.pre_mean)),
                                            ptr(_f32(self.target_mean)), ptr(_f32(self.target_std))))

    @classmethod
    def load(cls, path: str) -> "LearnedModel":
        L = _abi.lib()
        d, dim = C.c_uint64(0), C.c_uint64(0)
        _check(L.pacmap_model_load(str(path).encode(), C.byref(d), C.byref(dim), None, None, None, None, None, None))
        d, dim = int(d.value), int(dim.value)
        params = np.zeros(param_count(d, dim), np.float32)
        pre_mean = np.zeros(d, np.float32)
        t_mean, t_std = np.zeros(dim, np.float32), np.zeros(dim, np.float32)
        mn, mx = C.c_float(0), C.c_float(0)
        _check(L.pacmap_model_load(str(path).encode(), None, None, ptr(params), C.byref(mn), C.byref(mx),
                                   ptr(pre_mean), ptr(t_mean), ptr(t_std)))
        return cls(params, d, dim, mn.value, mx.value, pre_mean, t_mean, t_std)

    def transform(self, x, device: int = 0) -> np.ndarray:
        """Embeds new points (raw data like the training data) into the training embedding's coordinates."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        n, d = x.shape
        assert d == self.d, f"the model expects {self.d} columns, got {d}"
        out = np.zeros((n, self.dim), np.float32)
        _check(_abi.lib().pacmap_transform(ptr(x), n, d, self.dim, ptr(_f32(self.params)), float(self.pre_min),
                                           float(self.pre_max), ptr(_f32(self.pre_mean)),
                                           ptr(_f32(self.target_mean)), ptr(_f32(self.target_std)), device,
                                           ptr(out)))
        return out


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def target_stats(y):
    """Per-dimension (mean, population std) of an embedding: the standardisation of the MLP's targets."""
    y = _f32(y)
    n, dim = y.shape
    mean, std = np.zeros(dim, np.float32), np.zeros(dim, np.float32)
    _check(_abi.lib().pacmap_model_target_stats(ptr(y), n, dim, ptr(mean), ptr(std)))
    return mean, std


def fit_model(x, embedding, epochs: int = 20, batch: int = 4096, lr: float = 1e-3, weight_decay: float = 1e-4,
              seed: int = 0, device: int = 0):
    """Trains a ``LearnedModel`` on raw data x and its embedding (e.g. the plain fit of x).

    Returns (model, loss of each epoch)."""
    x = _f32(x)
    y = _f32(embedding)
    n, d = x.shape
    dim = y.shape[1]
    xp, mn, mx, mean = stages.preprocess(x, device)
    batch = min(batch, n // 128 * 128)
    params, losses = train(init_params(d, dim, seed), xp, y, epochs=epochs, batch=batch, lr=lr,
                           weight_decay=weight_decay, seed=seed, device=device)
    t_mean, t_std = target_stats(y)
    return LearnedModel(params, d, dim, float(mn), float(mx), _f32(mean), t_mean, t_std), losses
