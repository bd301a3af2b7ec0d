"""`pacmap::knn` (src/knn.rs): exact k-nearest neighbours on the GPU."""
from __future__ import annotations

from typing import Optional

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


def _shard_device(x, k: int, shard: int, n_shards: int, knn_mode: int, device: int):
    """The GPU shard into device tensors (pacmap_knn_exact_shard_device): (idx int32 view of u32, dist, owned)."""
    import torch

    n, d = x.shape
    kp = min(int(k), n - 1)
    dev = torch.device("cuda", device)
    dx = torch.from_numpy(x).to(dev)
    idx = torch.empty((n, kp), dtype=torch.int32, device=dev)
    dst = torch.empty((n, kp), dtype=torch.float32, device=dev)
    owned = torch.empty(n, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)  # the library computes on its own stream; the upload must be complete
    _check(_abi.lib().pacmap_knn_exact_shard_device(dx.data_ptr(), n, d, int(k), int(knn_mode), int(shard),
                                                    int(n_shards), int(device), idx.data_ptr(), dst.data_ptr(),
                                                    owned.data_ptr()))
    return idx, dst, owned.bool()


def find_k_nearest_neighbors_distributed(data, k: int, knn_mode: int = 0, device: int = 0, group=None,
                                         shard_fn=None, stats: Optional[dict] = None):
    """``find_k_nearest_neighbors`` split over the ranks of a torch.distributed group (no reference analogue).

    Every rank holds all points and computes its shard of the rows. Each rank packs its owned rows as
    records (row, k' indices, k' distances) into one int32 tensor, padded to the largest shard; one
    all-gather of those records (after one of the record counts) and a scatter into place give every rank
    the full result. With the nccl backend the shard is computed into device buffers and stays on the GPU
    through the collective; with gloo it is computed on the host side.

    ``shard_fn(data, k, shard, n_shards, knn_mode, device)`` (numpy arrays) replaces the GPU shard (tests
    on CPU ranks). ``stats`` (a dict, optional) receives ``bytes_sent``, this rank's payload.
    """
    import torch
    import torch.distributed as dist

    x = np.ascontiguousarray(data, dtype=np.float32)
    n = x.shape[0]
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    kp = min(int(k), n - 1) if n > 0 else 0
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", device) if on_gpu else torch.device("cpu")
    if shard_fn is None and on_gpu:
        idx, dst, owned = _shard_device(x, k, rank, world, knn_mode, device)
    else:
        fn = shard_fn or find_k_nearest_neighbors_shard
        i_np, d_np, o_np = fn(x, k, rank, world, knn_mode, device)
        idx = torch.from_numpy(np.ascontiguousarray(i_np, dtype=np.uint32).view(np.int32)).to(dev)
        dst = torch.from_numpy(np.ascontiguousarray(d_np, dtype=np.float32)).to(dev)
        owned = torch.from_numpy(np.asarray(o_np, dtype=bool)).to(dev)
    rows = torch.nonzero(owned).squeeze(1)
    rec = torch.cat([rows.to(torch.int32)[:, None], idx[rows], dst[rows].view(torch.int32)], 1)
    width = 1 + 2 * kp
    counts = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(counts, torch.tensor([rec.shape[0]], dtype=torch.int64, device=dev), group=group)
    counts = [int(c.item()) for c in counts]
    m = max(counts) if counts else 0
    send = torch.zeros((m, width), dtype=torch.int32, device=dev)
    send[: rec.shape[0]] = rec
    recv = [torch.empty((m, width), dtype=torch.int32, device=dev) for _ in range(world)]
    dist.all_gather(recv, send, group=group)
    if stats is not None:
        stats["bytes_sent"] = int(send.numel() * 4 + 8)
    if sum(counts) != n:
        raise RuntimeError("kNN shards do not partition the rows")
    out_i = torch.zeros((n, kp), dtype=torch.int32, device=dev)
    out_d = torch.zeros((n, kp), dtype=torch.int32, device=dev)
    seen = torch.zeros(n, dtype=torch.int32, device=dev)
    for r in range(world):
        g = recv[r][: counts[r]]
        rr = g[:, 0].long()
        out_i[rr] = g[:, 1:1 + kp]
        out_d[rr] = g[:, 1 + kp:]
        seen[rr] += 1
    if not bool((seen == 1).all()):
        raise RuntimeError("kNN shards do not partition the rows")
    return (out_i.cpu().numpy().view(np.uint32).copy(), out_d.view(torch.float32).cpu().numpy().copy())
