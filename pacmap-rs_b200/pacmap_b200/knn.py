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


def find_k_nearest_neighbors_shard(data, k: int, shard: int, n_shards: int, knn_mode: int = 0, device: int = 0):
    """One shard of ``find_k_nearest_neighbors`` (no reference analogue; multi-GPU use).

    Returns (indices, distances, owned): the full-size arrays with this shard's rows filled (others 0)
    and the boolean mask of those rows. The shards partition the rows; their union is the full result
    bit for bit.
    """
    x = np.ascontiguousarray(data, dtype=np.float32)
    n, d = x.shape
    if n == 0:
        return np.zeros((0, 0), np.uint32), np.zeros((0, 0), np.float32), np.zeros(0, bool)
    kp = min(int(k), n - 1)
    idx = np.zeros((n, kp), np.uint32)
    dist = np.zeros((n, kp), np.float32)
    owned = np.zeros(n, np.uint8)
    _check(_abi.lib().pacmap_knn_exact_shard(ptr(x), n, d, int(k), int(knn_mode), int(shard), int(n_shards),
                                             int(device), ptr(idx), ptr(dist), ptr(owned)))
    return idx, dist, owned.astype(bool)


def find_k_nearest_neighbors_distributed(data, k: int, knn_mode: int = 0, device: int = 0, group=None,
                                         shard_fn=None):
    """``find_k_nearest_neighbors`` split over the ranks of a torch.distributed group: every rank holds
    all points and computes its shard of the rows; one all-reduce of the masked results (each row has
    exactly one owner, so the sums are the owner's values) gives every rank the full result.

    ``shard_fn(data, k, shard, n_shards, knn_mode, device)`` replaces the GPU shard (tests on CPU ranks).
    Works with the nccl backend (CUDA tensors) and gloo (CPU tensors).
    """
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    fn = shard_fn or find_k_nearest_neighbors_shard
    idx, dst, owned = fn(data, k, rank, world, knn_mode, device)
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", device) if on_gpu else torch.device("cpu")
    own = torch.from_numpy(owned.astype(np.int32)).to(dev)
    ti = torch.from_numpy(idx.astype(np.int64) * owned[:, None]).to(dev)
    td = torch.from_numpy(np.where(owned[:, None], dst, np.float32(0))).to(dev)
    for t in (own, ti, td):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    if not bool((own == 1).all()):
        raise RuntimeError("kNN shards do not partition the rows")
    return ti.cpu().numpy().astype(np.uint32), td.cpu().numpy().astype(np.float32)
