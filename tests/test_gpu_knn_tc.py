"""The tensor-core kNN (tcgen05 FP16/BF16 distance GEMM filter + exact FP32 re-rank) against the oracle.

Bar: indices AND f32 distances bit-exact with the reference algorithm (knn.rs:137-194, ties -> lower
index) at every size, including rows that overflow the candidate buffer (exact fallback).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F16, BF16, AUTO = 1, 2, 0


def _mix(n, d, seed):
    from pacmap_b200 import datasets

    return datasets.isotropic_mixture(n=n, d=d, k=10, seed=seed)[0]


@pytest.mark.parametrize("mode", [F16, BF16])
@pytest.mark.parametrize("n,d,k", [(3001, 128, 90), (2000, 100, 60), (4096, 32, 17), (777, 13, 90), (300, 64, 10),
                                   (1024, 128, 1), (513, 65, 200),
                                   # fewer columns than one chunk of the reference's eight distance lanes
                                   (900, 5, 20),
                                   # resident A, one K block per stage (d 129..256)
                                   (700, 130, 17), (4100, 192, 99), (2000, 256, 90),
                                   # A and B streamed per K block (d > 256), ragged last block included
                                   (1000, 300, 60), (1500, 784, 72), (600, 1024, 30), (257, 333, 256)])
def test_tc_knn_bit_exact(lib, orc, mode, n, d, k):
    x = _mix(n, d, seed=n + d)
    gi, gd = lib.knn.find_k_nearest_neighbors(x, k, knn_mode=mode)
    ei, ed = orc.knn_exact(x, k)
    assert np.array_equal(gd, ed)
    assert np.array_equal(gi, ei)


def test_tc_knn_preprocessed_anisotropic(lib, orc):
    # the fit_transform path: preprocessed data of the 1M x 128 generator, a 20k slice
    from pacmap_b200 import datasets

    x, _ = datasets.anisotropic_mixture(n=20000, d=128, k=50, seed=1)
    xp, *_ = orc.preprocess(x)
    gi, gd = lib.knn.find_k_nearest_neighbors(xp, 90, knn_mode=AUTO)
    ei, ed = orc.knn_exact(xp, 90)
    assert np.array_equal(gd, ed) and np.array_equal(gi, ei)


def test_tc_knn_duplicates_overflow_to_exact_fallback(lib, orc):
    # 700 identical points: each has ~700 candidates at distance 0, more than the candidate buffer,
    # so those rows take the exact SIMT fallback; the result must still be the oracle's.
    x = _mix(3000, 24, seed=9)
    x[1000:1700] = x[5]
    x[2000:2010] = x[6]
    for mode in (F16, BF16):
        gi, gd = lib.knn.find_k_nearest_neighbors(x, 60, knn_mode=mode)
        ei, ed = orc.knn_exact(x, 60)
        assert np.array_equal(gd, ed) and np.array_equal(gi, ei)


def test_tc_knn_quantised_ties(lib, orc):
    # image-like data quantised to 1/255: many exactly tied distances
    from pacmap_b200 import datasets

    x, _ = datasets.image_like(n=2500, d=784, seed=3)
    x = x[:, :128].copy()
    gi, gd = lib.knn.find_k_nearest_neighbors(x, 72, knn_mode=F16)
    ei, ed = orc.knn_exact(x, 72)
    assert np.array_equal(gd, ed) and np.array_equal(gi, ei)


def _sampled_rows_vs_oracle(lib, orc, x, k, n_rows, seed=0, knn_mode=AUTO):
    """The GPU's full kNN (AUTO: the tensor-core path at n >= 16384) against the oracle on a seeded sample
    of query rows (knn.rs:137-194 restated row by row): indices and f32 distances bit-exact."""
    gi, gd = lib.knn.find_k_nearest_neighbors(x, k, knn_mode=knn_mode)
    n = x.shape[0]
    rows = np.sort(np.random.default_rng(seed).choice(n, size=min(n_rows, n), replace=False)).astype(np.uint32)
    ei, ed = orc.knn_rows(x, rows, k)
    bad = np.nonzero(~(np.all(gi[rows] == ei, axis=1) & np.all(gd[rows] == ed, axis=1)))[0]
    assert bad.size == 0, f"{bad.size} of {rows.size} sampled rows differ, first row {rows[bad[0]]}"
    return gi, gd


def test_tc_knn_anisotropic_100k_slice(lib, orc):
    # a 100,000-row slice of the 1M x 128 generator, preprocessed, k' = 90: 2,000 sampled rows
    from pacmap_b200 import datasets

    x, _ = datasets.anisotropic_mixture(n=100000, d=128, k=50, seed=0, draw_seed=5)
    xp = lib.stages.preprocess(x)[0]
    _sampled_rows_vs_oracle(lib, orc, xp, 90, 2000)


def test_tc_knn_image_like_60k_x_784(lib, orc):
    # the 60,000 x 784 image-like configuration (quantised to 1/255, many ties), k' = 22 + 50: 5,000 rows
    from pacmap_b200 import datasets

    x, _ = datasets.image_like(n=60000, d=784, seed=0)
    xp = lib.stages.preprocess(x)[0]
    _sampled_rows_vs_oracle(lib, orc, xp, 72, 5000)


def test_tc_knn_subspace_mixture_slice_256(lib, orc):
    # a 100,000-row draw of the 4M x 256 subspace-mixture generator, k' = 49 + 50: 2,000 rows
    from pacmap_b200 import datasets

    x, _ = datasets.subspace_mixture(n=100000, d=256, seed=2)
    xp = lib.stages.preprocess(x)[0]
    _sampled_rows_vs_oracle(lib, orc, xp, 99, 2000)


def test_tc_knn_full_1m_x_128(lib, orc):
    # the benchmarked size: a full 1,000,000 x 128 draw of its generator, preprocessed, k' = 40 + 50,
    # AUTO mode; 600 sampled rows against the oracle
    from pacmap_b200 import datasets

    x, _ = datasets.anisotropic_mixture(n=1_000_000, d=128, k=50, seed=0, draw_seed=1000)
    xp = lib.stages.preprocess(x)[0]
    gi, gd = _sampled_rows_vs_oracle(lib, orc, xp, 90, 600, seed=1)
    # size-independent properties over every row: ascending distances, no self, indices in range
    assert (np.diff(gd, axis=1) >= 0).all()
    assert (gi < x.shape[0]).all() and not (gi == np.arange(x.shape[0], dtype=np.uint32)[:, None]).any()


F16_FULL = 5


def _pruned_stats(lib, x, k):
    """One fit_transform of one iteration with stage timing on: the kNN stage's tile counters."""
    lib.set_stage_timing(True)
    try:
        lib.fit_transform(x, lib.Configuration(seed=3, initialization=lib.Initialization.Random(1),
                                               override_neighbors=k, num_iters=(0, 0, 1)))
        return lib.stage_times()
    finally:
        lib.set_stage_timing(False)


@pytest.mark.parametrize("gen,n,d,k", [("aniso", 60000, 128, 90), ("subspace", 50000, 256, 99),
                                       ("iso", 40000, 64, 60), ("uniform", 40000, 32, 30),
                                       ("dups", 40000, 24, 60)])
def test_tile_pruning_equals_full_sweep(lib, orc, gen, n, d, k):
    """From 32,768 rows the tensor-core kNN skips column tiles that provably hold no neighbour; the result
    must equal the full sweep (mode 5) bit for bit, and the oracle on sampled rows, on clustered data
    (much pruned), uniform data (little pruned) and exact duplicates (overflow rows)."""
    from pacmap_b200 import datasets

    if gen == "aniso":
        x, _ = datasets.anisotropic_mixture(n=n, d=d, k=50, seed=4)
    elif gen == "subspace":
        x, _ = datasets.subspace_mixture(n=n, d=d, k=200, seed=4)
    elif gen == "iso":
        x = _mix(n, d, seed=4)
    elif gen == "uniform":
        x = np.random.default_rng(4).random((n, d), dtype=np.float32)
    else:
        x = _mix(n, d, seed=5)
        x[1000:1700] = x[5]
    xp = lib.stages.preprocess(x)[0]
    fi, fd = lib.knn.find_k_nearest_neighbors(xp, k, knn_mode=F16_FULL)
    gi, gd = _sampled_rows_vs_oracle(lib, orc, xp, k, 300, seed=2, knn_mode=AUTO)
    assert np.array_equal(gd, fd)
    assert np.array_equal(gi, fi)


def test_tile_pruning_skips_most_tiles_on_clustered_data(lib):
    # 100,000 x 128 of the 1M x 128 generator (50 clusters): most (row block, tile) pairs are skipped
    from pacmap_b200 import datasets

    x, _ = datasets.anisotropic_mixture(n=100000, d=128, k=50, seed=0, draw_seed=6)
    st = _pruned_stats(lib, x, 40)
    frac = st["knn_tiles_visited"] / st["knn_tiles_full"]
    print(f"tiles visited {st['knn_tiles_visited']:.0f} of {st['knn_tiles_full']:.0f} ({frac:.3f}); bound pass "
          f"{st['knn_tiles_bound']:.0f}; filter {st['knn_filter']:.2f} ms, bound {st['knn_bound']:.2f} ms")
    assert 0 < frac < 0.25


def test_bounded_wait_runs_out_with_a_status_and_the_next_call_succeeds(lib, orc):
    """Failure detection without a GPU fault: with the test hook on, the filter's operand copies are never
    issued, so its bounded mbarrier wait runs out; the call returns DEVICE_INVARIANT (a timeout), the block
    releases its tensor memory, and the next call on the same context is exact again."""
    x = _mix(3000, 64, seed=12)
    stall = lib._abi.lib().pacmap_debug_stall_knn_loads
    try:
        assert stall(0, 1) == 0
        with pytest.raises(lib.DeviceInvariant) as e:
            lib.knn.find_k_nearest_neighbors(x, 30, knn_mode=F16)
        assert "timed out" in str(e.value)
    finally:
        assert stall(0, 0) == 0
    gi, gd = lib.knn.find_k_nearest_neighbors(x, 30, knn_mode=F16)
    ei, ed = orc.knn_exact(x, 30)
    assert np.array_equal(gd, ed) and np.array_equal(gi, ei)


def test_simt_knn_key_slices(lib, orc):
    # 9,000 rows on the exact SIMT path: the keys are split into two slices whose lists are merged
    x = _mix(9000, 16, seed=4)
    gi, gd = lib.knn.find_k_nearest_neighbors(x, 30, knn_mode=3)
    ei, ed = orc.knn_exact(x, 30)
    assert np.array_equal(gd, ed) and np.array_equal(gi, ei)


def test_tc_knn_fallback_rows_over_key_slices(lib, orc):
    # 700 duplicates overflow the filter's buffers; those few rows are recomputed over ~9 key slices
    x = _mix(40000, 24, seed=8)
    x[1000:1700] = x[5]
    gi, gd = lib.knn.find_k_nearest_neighbors(x, 60, knn_mode=F16)
    ei, ed = orc.knn_exact(x, 60)
    assert np.array_equal(gd, ed) and np.array_equal(gi, ei)


@pytest.mark.parametrize("mode,n,d,k", [(F16, 3000, 40, 60), (AUTO, 20000, 24, 30), (3, 2500, 17, 12)])
def test_knn_shards_partition_rows_and_reproduce_the_full_result(lib, mode, n, d, k):
    # the multi-GPU primitive on one GPU: shards of the tensor-core path (row blocks in its locality
    # order) and of the SIMT path (rows in order) partition the rows and rebuild the full kNN exactly
    x = _mix(n, d, seed=n)
    gi, gd = lib.knn.find_k_nearest_neighbors(x, k, knn_mode=mode)
    cover = np.zeros(n, int)
    ui, ud = np.zeros_like(gi), np.zeros_like(gd)
    for s in range(3):
        si, sd, own = lib.knn.find_k_nearest_neighbors_shard(x, k, s, 3, knn_mode=mode)
        cover += own
        ui[own], ud[own] = si[own], sd[own]
        assert not si[~own].any() and not sd[~own].any()
    assert (cover == 1).all()
    assert np.array_equal(ui, gi) and np.array_equal(ud, gd)
    # the device-buffer shard entry point (the NCCL assembly's input) writes the same rows
    for s in range(3):
        di, dd, down = lib.knn._shard_device(x, k, s, 3, mode, 0)
        own = down.cpu().numpy()
        assert np.array_equal(di.cpu().numpy().view(np.uint32)[own], gi[own])
        assert np.array_equal(dd.cpu().numpy()[own], gd[own])


APPROX = 4


def test_approximate_knn_recall_and_exact_distances(lib, orc):
    """knn_mode APPROX: each row block searches the 16 pivot cells nearest its own. Most true neighbours
    are found, every returned distance is the reference's exact f32 distance of that pair, and rank by
    rank the returned distances are never below the exact ones."""
    from pacmap_b200 import datasets

    x, _ = datasets.anisotropic_mixture(n=60000, d=32, k=20, seed=3)
    xp = lib.stages.preprocess(x)[0]
    k = 30
    ei, ed = lib.knn.find_k_nearest_neighbors(xp, k)
    ai, ad = lib.knn.find_k_nearest_neighbors(xp, k, knn_mode=APPROX)
    recall = np.mean([len(np.intersect1d(ai[r], ei[r])) / k for r in range(0, 60000, 7)])
    print(f"approximate kNN recall {recall:.4f}")
    assert recall >= 0.95
    assert (ad >= ed).all() and (np.diff(ad, axis=1) >= 0).all()
    rows = np.arange(0, 60000, 997)
    for r in rows:
        for c in range(0, k, 7):
            assert ad[r, c] == np.float32(orc.distance(xp[r], xp[ai[r, c]]))


def test_approximate_mode_is_exact_below_the_threshold(lib):
    x = _mix(3000, 20, seed=5)
    cfg = lambda thr: lib.Configuration(seed=7, initialization=lib.Initialization.Random(1), knn_mode=APPROX,  # noqa
                                        approx_threshold=thr)
    exact = lib.stages.generate_pairs(x, lib.Configuration(seed=7, initialization=lib.Initialization.Random(1)))
    below = lib.stages.generate_pairs(x, cfg(8000))
    assert all(np.array_equal(a, b) for a, b in zip(exact, below))
    y, _ = lib.fit_transform(x, cfg(1000))  # above the threshold (SIMT at this n: still exact)
    assert np.all(np.isfinite(y))
