"""B200-native PaCMAP with the calling contract of beamform/pacmap-rs v0.2.6 (crate ``pacmap``).

Mirrors the reference's public Rust API (src/lib.rs:159-367, src/knn.rs:137) over the C ABI of
``libpacmap_b200.so`` (include/pacmap.h):

    Configuration (builder + defaults)   lib.rs:159-224
    Initialization.{Pca, Value, Random}  lib.rs:226-239
    PairConfiguration.{Generate, NeighborsProvided, AllProvided}   lib.rs:241-267
    fit_transform(x, config) -> (embedding, snapshots | None)     lib.rs:294-367
    PaCMapError and its variants         lib.rs:870-922
    knn.find_k_nearest_neighbors         knn.rs:137-194

Every computation runs on the GPU through hand-written sm_100a kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _abi
from ._abi import ptr

__all__ = [
    "Configuration", "Initialization", "PairConfiguration", "fit_transform", "fit_transform_device",
    "PaCMapError", "KnnMode", "Metric", "knn", "quality", "last_launch_count", "learned",
]

# ---------------------------------------------------------------------------------------------
# Errors: one class per PaCMapError / KnnError variant (lib.rs:870-922, knn.rs:196-206).
# ---------------------------------------------------------------------------------------------


class PaCMapError(RuntimeError):
    """Base of every failure; ``code`` is the C status (include/pacmap.h)."""

    code = -1

    def __init__(self, message: str = ""):
        super().__init__(message or type(self).__name__)


def _variant(name: str, code: int, doc: str):
    cls = type(name, (PaCMapError,), {"code": code, "__doc__": doc})
    globals()[name] = cls
    __all__.append(name)
    return cls


_ERRORS = {
    1: _variant("SampleSize", 1, "Input has <= 1 samples (lib.rs:875)."),
    2: _variant("InvalidNearestNeighborShape", 2, "Provided neighbour pairs have the wrong shape (lib.rs:879)."),
    3: _variant("EmptyArrayMean", 3, "Mean of an empty array (lib.rs:888)."),
    4: _variant("Normal", 4, "Normal distribution construction failed (lib.rs:892)."),
    5: _variant("InvalidNeighborCount", 5, "Neighbour count below 1 (lib.rs:896)."),
    6: _variant("InvalidFarPointCount", 6, "Far-pair count below 1 (lib.rs:900)."),
    7: _variant("EmptyArrayMinMax", 7, "Min/max of an empty array (lib.rs:904)."),
    8: _variant("ZeroRange", 8, "Zero data range (lib.rs:908; never raised, as in the reference)."),
    9: _variant("Pca", 9, "PCA failure (lib.rs:912)."),
    10: _variant("KnnConstruction", 10, "KnnError::Construction (knn.rs:200)."),
    11: _variant("KnnReservation", 11, "KnnError::Reservation (knn.rs:204)."),
    12: _variant("MissingTransform", 12, "PCA transform missing (lib.rs:920)."),
    20: _variant("InvalidArgument", 20, "A NULL pointer, bad enum or size overflow."),
    21: _variant("PairIndexOutOfRange", 21, "A provided pair names a point >= n (the reference panics)."),
    22: _variant("SamplingFailed", 22, "Distinct partners cannot be drawn (the reference loops forever)."),
    23: _variant("Unsupported", 23, "A size beyond a kernel limit."),
    24: _variant("ModelFileError", 24, "A model file cannot be read or written, or is damaged."),
    30: _variant("CudaError", 30, "CUDA runtime error."),
    31: _variant("OutOfMemory", 31, "Device allocation failed."),
    32: _variant("NoDevice", 32, "No CUDA device of compute capability 10.x."),
    33: _variant("DeviceInvariant", 33, "A kernel's own check failed."),
}


def _check(rc: int) -> None:
    if rc != 0:
        cls = _ERRORS.get(rc, PaCMapError)
        raise cls(_abi.last_error())


# ---------------------------------------------------------------------------------------------
# Initialization / PairConfiguration (Rust enums as small classes).
# ---------------------------------------------------------------------------------------------


class Initialization:
    """Initialization::{Pca, Value(Array2<f32>), Random(Option<u64>)} (lib.rs:226-239)."""

    @dataclass(frozen=True)
    class Pca:
        kind = 0

    @dataclass(frozen=True)
    class Value:
        value: np.ndarray
        kind = 1

    @dataclass(frozen=True)
    class Random:
        seed: Optional[int] = None
        kind = 2


class PairConfiguration:
    """PairConfiguration::{Generate, NeighborsProvided, AllProvided} (lib.rs:241-267)."""

    @dataclass(frozen=True)
    class Generate:
        kind = 0

    @dataclass(frozen=True)
    class NeighborsProvided:
        pair_neighbors: np.ndarray
        kind = 1

    @dataclass(frozen=True)
    class AllProvided:
        pair_neighbors: np.ndarray
        pair_mn: np.ndarray
        pair_fp: np.ndarray
        kind = 2


class KnnMode:
    """How the kNN is computed (engine switch). Modes 0-3 and 5 return identical exact indices and
    distances; mode 4 (APPROX) is approximate from ``approx_threshold`` rows on. From 32,768 rows the
    tensor-core modes 0-2 skip column tiles that provably hold no neighbour; mode 5 computes every tile."""

    AUTO = 0
    TENSOR_F16 = 1
    TENSOR_BF16 = 2
    SIMT_EXACT = 3
    APPROX = 4  # approximate at n >= approx_threshold (16 of 256 pivot cells per row block); exact below
    TENSOR_F16_FULL = 5  # TENSOR_F16 without tile pruning


class Metric:
    """The distance the pairs are drawn with (engine switch; the reference is Euclidean only,
    README.md:164). ANGULAR: the preprocessed rows are scaled to unit norm, so distances become
    sqrt(2 - 2 cos)."""

    EUCLIDEAN = 0
    ANGULAR = 1


@dataclass
class Configuration:
    """Configuration (lib.rs:159-224) with the reference's defaults, plus engine switches."""

    embedding_dimensions: int = 2
    initialization: object = field(default_factory=Initialization.Pca)
    mid_near_ratio: float = 0.5
    far_pair_ratio: float = 2.0
    override_neighbors: Optional[int] = None
    seed: Optional[int] = None
    pair_configuration: object = field(default_factory=PairConfiguration.Generate)
    learning_rate: float = 1.0
    num_iters: Tuple[int, int, int] = (100, 100, 250)
    snapshots: Optional[Sequence[int]] = None
    approx_threshold: int = 8_000
    # engine switches (no reference analogue)
    knn_mode: int = KnnMode.AUTO
    device: int = 0
    metric: int = Metric.EUCLIDEAN

    @staticmethod
    def builder() -> "_Builder":
        """The reference's bon builder: Configuration.builder().learning_rate(0.8).build()."""
        return _Builder()


class _Builder:
    def __init__(self):
        self._kw = {}

    def __getattr__(self, name):
        if name.startswith("_") or name not in Configuration.__dataclass_fields__:
            raise AttributeError(name)

        def setter(value):
            self._kw[name] = value
            return self

        return setter

    def build(self) -> Configuration:
        return Configuration(**self._kw)


def _pairs_u32(a, what: str) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    if a.ndim != 2 or a.shape[1] != 2:
        raise InvalidArgument(f"{what} must be an (rows, 2) array")  # noqa: F821
    return a


class _CConfig:
    """Builds struct pacmap_config and keeps the numpy buffers it points at alive."""

    def __init__(self, config: Configuration, n: int, loss_trace: Optional[np.ndarray] = None):
        c = _abi.lib().pacmap_config_default()
        self.keep = []
        c.embedding_dimensions = int(config.embedding_dimensions)
        init = config.initialization
        c.init_kind = init.kind
        if isinstance(init, Initialization.Value):
            v = np.ascontiguousarray(init.value, dtype=np.float32)
            if v.shape != (n, config.embedding_dimensions):
                raise InvalidArgument(  # noqa: F821
                    f"Initialization.Value must be {(n, config.embedding_dimensions)}, got {v.shape}")
            self.keep.append(v)
            c.init_value = v.ctypes.data
        elif isinstance(init, Initialization.Random):
            c.init_has_seed = 0 if init.seed is None else 1
            c.init_seed = 0 if init.seed is None else int(init.seed) & (2**64 - 1)
        c.mid_near_ratio = float(config.mid_near_ratio)
        c.far_pair_ratio = float(config.far_pair_ratio)
        if config.override_neighbors is not None:
            c.has_override_neighbors = 1
            c.override_neighbors = int(config.override_neighbors)
        if config.seed is not None:
            c.has_seed = 1
            c.seed = int(config.seed) & (2**64 - 1)
        pc = config.pair_configuration
        c.pair_kind = pc.kind
        if isinstance(pc, (PairConfiguration.NeighborsProvided, PairConfiguration.AllProvided)):
            pn = _pairs_u32(pc.pair_neighbors, "pair_neighbors")
            self.keep.append(pn)
            c.pair_neighbors, c.pair_neighbors_rows = pn.ctypes.data, pn.shape[0]
        if isinstance(pc, PairConfiguration.AllProvided):
            pm, pf = _pairs_u32(pc.pair_mn, "pair_mn"), _pairs_u32(pc.pair_fp, "pair_fp")
            self.keep += [pm, pf]
            c.pair_mn, c.pair_mn_rows = pm.ctypes.data, pm.shape[0]
            c.pair_fp, c.pair_fp_rows = pf.ctypes.data, pf.shape[0]
        c.learning_rate = float(config.learning_rate)
        for t in range(3):
            c.num_iters[t] = int(config.num_iters[t])
        if config.snapshots is not None:
            s = np.ascontiguousarray(config.snapshots, dtype=np.uint64)
            self.keep.append(s)
            c.snapshots, c.n_snapshots = (s.ctypes.data if s.size else None), s.size
        c.approx_threshold = int(config.approx_threshold)
        c.knn_mode = int(config.knn_mode)
        c.device = int(config.device)
        c.metric = int(config.metric)
        if loss_trace is not None:
            self.keep.append(loss_trace)
            c.loss_trace = loss_trace.ctypes.data
        self.c = c


def fit_transform(x, config: Optional[Configuration] = None, loss_trace: bool = False):
    """fit_transform (lib.rs:294-367): returns (embedding n x dim, snapshots or None).

    With ``loss_trace=True`` a third value holds the loss of every iteration (the reference logs it).
    """
    config = config or Configuration()
    x = np.ascontiguousarray(x, dtype=np.float32)
    if x.ndim != 2:
        raise InvalidArgument("x must be 2-D")  # noqa: F821
    n, d = x.shape
    dim = int(config.embedding_dimensions)
    total = sum(int(t) for t in config.num_iters)
    lt = np.zeros(max(total, 1), np.float32) if loss_trace else None
    cc = _CConfig(config, n, lt)
    out = np.zeros((n, dim), np.float32)
    snaps = None
    if config.snapshots is not None:
        snaps = np.zeros((len(config.snapshots), n, dim), np.float32)
    _check(_abi.lib().pacmap_fit_transform(ptr(x), n, d, C.byref(cc.c), ptr(out), ptr(snaps)))
    if loss_trace:
        return out, snaps, lt[:total]
    return out, snaps


def fit_transform_device(x_ptr: int, n: int, d: int, out_ptr: int, config: Optional[Configuration] = None,
                         snapshots_ptr: Optional[int] = None) -> None:
    """fit_transform on device memory (raw CUDA pointers, e.g. torch.Tensor.data_ptr())."""
    config = config or Configuration()
    cc = _CConfig(config, n)
    _check(_abi.lib().pacmap_fit_transform_device(C.c_void_p(x_ptr), n, d, C.byref(cc.c), C.c_void_p(out_ptr),
                                                  C.c_void_p(snapshots_ptr) if snapshots_ptr else None))


def decide_num_pairs(n: int, config: Optional[Configuration] = None):
    """(k, n_mn, n_fp) of ``decide_num_pairs`` (lib.rs:565-597) as the library computes it for n points
    (k clamped to n - 1), through ``pacmap_generate_pairs`` with no output buffers: no device is needed."""
    cfg = config if config is not None else Configuration()
    cc = _CConfig(cfg, n)
    counts = np.zeros(3, np.uint64)
    dummy = np.zeros(1, np.float32)  # not read when only the counts are asked for
    _check(_abi.lib().pacmap_generate_pairs(ptr(dummy), n, 1, C.byref(cc.c), ptr(counts), None, None, None))
    return tuple(int(v) for v in counts)


def quality(x, y, sample, triplets, k: int = 10, device: int = 0):
    """(k-NN preservation over `sample`, triplet-order accuracy over `triplets`) on the GPU."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    s = np.ascontiguousarray(sample, dtype=np.uint32)
    t = np.ascontiguousarray(triplets, dtype=np.uint32).reshape(-1, 3)
    p, a = C.c_double(0), C.c_double(0)
    _check(_abi.lib().pacmap_quality(ptr(x), x.shape[0], x.shape[1], ptr(y), y.shape[1], ptr(s), s.size, k, ptr(t),
                                     t.shape[0], device, C.byref(p), C.byref(a)))
    return p.value, a.value


STAGES = ("preprocess", "knn", "reselect", "sample_mn", "sample_fp", "csr", "init", "optimize", "knn_filter",
          "knn_fallback_rows", "knn_bound", "knn_tiles_visited", "knn_tiles_full", "knn_tiles_bound",
          "knn_insertions_per_row", "knn_compactions_per_row", "knn_band_per_row", "optimize_graph_setup")


def set_stage_timing(enabled: bool) -> None:
    """Record per-stage device times (CUDA events) in each later fit_transform on this thread."""
    _abi.lib().pacmap_set_stage_timing(1 if enabled else 0)


def stage_times() -> dict:
    """Device milliseconds per stage of the last timed fit_transform on this thread."""
    buf = np.zeros(len(STAGES), np.float64)
    k = int(_abi.lib().pacmap_stage_times(ptr(buf), len(STAGES)))
    return {name: float(buf[i]) for i, name in enumerate(STAGES[:k])}


def gather_rate(device: int = 0) -> float:
    """Random 8-byte loads per second from an L2-resident 8 MB array on the device: the ceiling of the
    gradient's partner gathers (one such load per CSR entry)."""
    v = C.c_double(0.0)
    _check(_abi.lib().pacmap_gather_rate(int(device), C.byref(v)))
    return v.value


def last_launch_count() -> int:
    """Kernel launches issued by this thread since the previous call."""
    return int(_abi.lib().pacmap_take_launch_count())


from . import knn  # noqa: E402  (submodule mirrors `pacmap::knn`)
from . import stages  # noqa: E402
from . import learned  # noqa: E402  (the learned initialiser; no reference counterpart)
