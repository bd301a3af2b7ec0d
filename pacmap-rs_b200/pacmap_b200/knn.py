"""`pacmap::knn` (src/knn.rs): exact k-nearest neighbours on the GPU."""
from __future__ import annotations

import numpy as np

from . import _abi, _check
from ._abi import ptr


def find_k_nearest_neighbors(data, k: int, knn_mode: int = 0, device: int = 0):
    """knn::find_k_nearest_neighbors (knn.rs:137-194).

    Returns (indices u32, distances f32), each n x min(k, n-1), rows in ascending (distance, index)
    order, self excluded; an empty input gives (0, 0) arrays (knn.rs:141-143).
    """
    x = np.ascontiguousarray(data, dtype=np.float32)
    if x.ndim != 2:
        raise ValueError("data must be 2-D")
    n, d = x.shape
    if n == 0:
        return np.zeros((0, 0), np.uint32), np.zeros((0, 0), np.float32)
    kp = min(int(k), n - 1)
    idx = np.zeros((n, kp), np.uint32)
    dist = np.zeros((n, kp), np.float32)
    if kp > 0:
        _check(_abi.lib().pacmap_knn_exact(ptr(x), n, d, int(k), int(knn_mode), int(device), ptr(idx), ptr(dist)))
    return idx, dist
