"""The stage statistics a fit reports (pacmap_stage_times): device times of every stage and, for the
tensor-core kNN, its pair counts and per-row candidate counts, consistent with each other."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_stage_times_and_knn_counters(lib):
    from pacmap_b200 import datasets

    x, _ = datasets.anisotropic_mixture(n=40_000, d=32, k=12, seed=5)
    lib.set_stage_timing(True)
    try:
        lib.fit_transform(x, lib.Configuration(initialization=lib.Initialization.Random(1), seed=1,
                                               num_iters=(2, 2, 2)))
        st = lib.stage_times()
    finally:
        lib.set_stage_timing(False)
    for name in ("preprocess", "knn", "reselect", "sample_mn", "sample_fp", "csr", "init", "optimize"):
        assert st[name] >= 0.0 and np.isfinite(st[name]), name
    assert st["knn_filter"] > 0.0 and st["knn_filter"] <= st["knn"]
    # pruning ran (40,000 rows): the pairs computed are a part of the full sweep
    assert 0 < st["knn_tiles_bound"] + st["knn_tiles_visited"] <= st["knn_tiles_full"]
    kp = min(lib.decide_num_pairs(40_000)[0] + 50, 39_999)
    # a settled row keeps at least its k' + 1 candidates (itself included) through to the re-rank (rows
    # left to the exact fallback count none), and every kept candidate was inserted by the filter
    assert st["knn_band_per_row"] > 0.5 * kp and st["knn_insertions_per_row"] >= st["knn_band_per_row"]
    assert st["knn_compactions_per_row"] >= 0.0
