"""The multi-GPU kNN's collective assembly (knn.find_k_nearest_neighbors_distributed) on CPU ranks: two
gloo processes, each computing its shard of the rows (here from the CPU oracle, as the GPU shard would),
must both end with the full exact kNN. The GPU shard itself is tested in test_gpu_knn_tc.py."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _paths():
    for p in (ROOT, os.path.join(ROOT, "pacmap-rs_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)


def _data():
    rng = np.random.default_rng(4)
    return (rng.normal(size=(600, 12)) + rng.integers(0, 5, size=(600, 1))).astype(np.float32)


def _oracle_shard(data, k, shard, n_shards, knn_mode, device):
    import oracle

    idx, dist = oracle.knn_exact(data, k)
    n = data.shape[0]
    owned = np.zeros(n, bool)
    owned[n * shard // n_shards: n * (shard + 1) // n_shards] = True
    return np.where(owned[:, None], idx, 0).astype(np.uint32), np.where(owned[:, None], dist, 0).astype(np.float32), owned


def _worker(rank, world, port, q):
    _paths()
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pacmap_b200 import knn
        import oracle

        x = _data()
        st = {}
        idx, d = knn.find_k_nearest_neighbors_distributed(x, 15, shard_fn=_oracle_shard, stats=st)
        ei, ed = oracle.knn_exact(x, 15)
        # each rank sends only its owned rows' records (300 rows x (1 + 2 * 15) int32 + the count), not the
        # full n x k' arrays
        small = st["bytes_sent"] <= 300 * 31 * 4 + 8
        q.put((rank, bool(np.array_equal(idx, ei) and np.array_equal(d, ed) and small)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_distributed_knn_assembles_the_full_result_on_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0, p.exitcode
    results = sorted(q.get(timeout=10) for _ in range(2))
    assert results == [(0, True), (1, True)]
