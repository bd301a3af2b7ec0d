"""Pins the CPU oracle against the reference's own golden vectors and known answers (no GPU)."""
import numpy as np
import pytest

from conftest import gaussian_mixture


def test_gradient_golden(orc, golden):
    g = golden["gradient"]
    y = np.array(g["y"], np.float32)
    got = orc.grad(y, np.array(g["pair_neighbors"]), np.array(g["pair_mn"]), np.array(g["pair_fp"]),
                   g["w_neighbors"], g["w_mn"], g["w_fp"])
    np.testing.assert_allclose(got, np.array(g["expected"], np.float32), atol=g["eps"], rtol=0)


def test_adam_golden(orc, golden):
    a = golden["adam"]
    y = np.array(a["y"], np.float32)
    m = np.zeros_like(y)
    v = np.zeros_like(y)
    orc.adam(y, np.array(a["grad"], np.float32), m, v, a["lr"], a["itr"])
    np.testing.assert_allclose(y, np.array(a["y_expected"], np.float32), atol=a["eps"], rtol=0)
    np.testing.assert_allclose(m, np.array(a["m_expected"], np.float32), atol=a["eps"], rtol=0)
    np.testing.assert_allclose(v, np.array(a["v_expected"], np.float32), atol=a["eps"], rtol=0)


def test_weights_known_answers(orc, golden):
    w = golden["weights"]
    assert len(w["cases"]) == 4
    for c in w["cases"]:
        w_mn, w_nn, w_fp = orc.weights(c["itr"], c["p1"], c["p2"], w["w_mn_init"])
        assert w_mn == pytest.approx(c["w_mn"], abs=1e-6)
        assert w_nn == pytest.approx(c["w_neighbors"], abs=1e-6)
        assert w_fp == pytest.approx(c["w_fp"], abs=1e-6)


def test_scale_dist_golden(orc, golden):
    s = golden["scale_dist_small"]
    got = orc.scale_dist(np.array(s["knn_distances"]), np.array(s["sig"]), np.array(s["neighbors"]))
    assert np.array_equal(got, np.array(s["expected"], np.float32))
    s = golden["scale_dist_large"]
    got = orc.scale_dist(np.array(s["knn_distances"]), np.array(s["sig"]), np.array(s["neighbors"]))
    np.testing.assert_allclose(got, np.array(s["expected"], np.float32), atol=s["eps"], rtol=0)


@pytest.mark.parametrize("allpairs", [False, True])
def test_knn_known_answers(orc, golden, allpairs):
    for name, case in golden["knn"]["cases"].items():
        x = np.array(case["embeddings"], np.float32)
        idx, dist = orc.knn_exact(x, case["k"], allpairs=allpairs)
        for point, exp in case["expected"]:
            got = sorted(zip(idx[point].tolist(), dist[point].tolist()))
            exp = sorted((int(i), float(v)) for i, v in exp)
            assert [g[0] for g in got] == [e[0] for e in exp], name
            np.testing.assert_allclose([g[1] for g in got], [e[1] for e in exp], atol=1e-4, rtol=1e-4)


def test_knn_edge_shapes(orc):
    # knn.rs:215-255: empty input, single point, k = 0, k > n-1.
    idx, dist = orc.knn_exact(np.zeros((0, 128), np.float32), 5)
    assert idx.shape == (0, 0)
    idx, dist = orc.knn_exact(np.array([[1.0, 0.0, 0.0]], np.float32), 1)
    assert idx.shape == (1, 0)
    idx, dist = orc.knn_exact(np.array([[1.0, 0.0], [0.0, 1.0], [0.0, 0.0]], np.float32), 0)
    assert idx.shape == (3, 0)
    idx, dist = orc.knn_exact(np.array([[1.0], [2.0], [3.0]], np.float32), 5)
    assert idx.shape == (3, 2) and (idx < 3).all() and (dist >= 0).all()


def test_knn_per_row_equals_reference_allpairs(orc):
    # The per-row oracle equals the reference's literal all-pairs + global sort algorithm
    # (knn.rs:149-191) with ties broken by (distance, i, j) -- including exact duplicates.
    x, _ = gaussian_mixture(300, 20, seed=3)
    x[50] = x[7]
    x[51] = x[7]
    x = np.round(x, 1).astype(np.float32)  # many exact distance ties
    for k in (1, 6, 60):
        a = orc.knn_exact(x, k)
        b = orc.knn_exact(x, k, allpairs=True)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_knn_rows_equals_full_matrix_rows(orc):
    # The sampled-row oracle (used at sizes where the full matrix is too slow) returns exactly the rows
    # of the full per-row oracle, ties included; the allpairs test above pins that one to knn.rs.
    x, _ = gaussian_mixture(5000, 37, seed=4)
    x[100:140] = x[7]
    x = np.round(x, 1).astype(np.float32)
    rows = np.array([0, 7, 100, 139, 140, 2047, 2048, 4999, 3333, 120], np.uint32)
    for k in (1, 90, 4999, 6000):
        full = orc.knn_exact(x, k)
        got = orc.knn_rows(x, rows, k)
        assert np.array_equal(got[0], full[0][rows]) and np.array_equal(got[1], full[1][rows])


def test_distance_properties(orc):
    # distance.rs:192-268 quickcheck properties: non-negative, zero when equal, symmetric, and equal to
    # the serial sum within f32::EPSILON absolute.
    rng = np.random.default_rng(0)
    for length in [0, 1, 7, 8, 9, 64, 100, 255]:
        for _ in range(20):
            a = rng.normal(0, 1, length).astype(np.float32)
            b = rng.normal(0, 1, length).astype(np.float32)
            d1, d2 = orc.distance(a, b), orc.distance(b, a)
            assert d1 >= 0 and orc.distance(a, a) == 0.0 and abs(d1 - d2) <= np.finfo(np.float32).eps
            serial = np.float32(0)
            for u, v in zip(a, b):
                serial = np.float32(serial + np.float32(u - v) * np.float32(u - v))
            assert abs(d1 - np.sqrt(serial, dtype=np.float32)) <= 4 * np.finfo(np.float32).eps * max(1, d1)


def test_decide_num_pairs(orc):
    # lib.rs:565-597 at the configurations' sizes.
    assert orc.decide_num_pairs(2000)[1] == (10, 5, 20)
    assert orc.decide_num_pairs(60000)[1] == (22, 11, 44)
    assert orc.decide_num_pairs(200000)[1] == (30, 15, 60)
    assert orc.decide_num_pairs(1000000)[1] == (40, 20, 80)
    assert orc.decide_num_pairs(4000000)[1] == (49, 25, 98)
    assert orc.decide_num_pairs(1000, override=0)[0] == 5      # InvalidNeighborCount
    assert orc.decide_num_pairs(1000, fp_ratio=0.0)[0] == 6    # InvalidFarPointCount


def test_preprocess_semantics(orc):
    # lib.rs:485-511: divide by max (not the range), then subtract the sequential column mean.
    rng = np.random.default_rng(1)
    x = rng.uniform(-3, 5, size=(257, 13)).astype(np.float32)
    out, mn, mx, mean = orc.preprocess(x)
    assert mn == x.min() and mx == x.max()
    y = ((x - np.float32(mn)) / np.float32(mx)).astype(np.float32)
    s = np.zeros(13, np.float32)
    for r in range(257):
        s = (s + y[r]).astype(np.float32)
    exp_mean = (s / np.float32(257)).astype(np.float32)
    assert np.array_equal(mean, exp_mean)
    assert np.array_equal(out, (y - exp_mean).astype(np.float32))


def test_philox_known_answer(orc):
    # Random123 philox4x32-10 known-answer vectors (kat_vectors): zero and all-ones inputs.
    assert orc.philox4x32_10([0, 0, 0, 0], 0, 0).tolist() == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert orc.philox4x32_10([0xFFFFFFFF] * 4, 0xFFFFFFFF, 0xFFFFFFFF).tolist() == \
        [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]


def test_sampling_rules(orc):
    # sampling.rs:468-568 properties, on the Philox stream: shape, exclusion of NN and self,
    # uniqueness, determinism for one seed.
    n, k, n_fp = 100, 10, 5
    pn = np.stack([np.repeat(np.arange(n), k), np.tile(np.arange(k), n)], 1).astype(np.uint32)
    fp = orc.sample_fp_pairs(pn, n, k, n_fp, 42)
    assert fp.shape == (n * n_fp, 2)
    for i in range(n):
        blk = fp[i * n_fp:(i + 1) * n_fp]
        assert (blk[:, 0] == i).all()
        assert not np.isin(blk[:, 1], np.arange(k)).any()
        assert len(set(blk[:, 1].tolist())) == n_fp and i not in blk[:, 1]
    assert np.array_equal(fp, orc.sample_fp_pairs(pn, n, k, n_fp, 42))
    x = np.random.default_rng(0).uniform(-1, 1, (1000, 20)).astype(np.float32)
    mn = orc.sample_mn_pairs(x, 5, 42)
    assert mn.shape == (5000, 2) and (mn < 1000).all() and (mn[:, 0] != mn[:, 1]).all()
    assert np.array_equal(mn, orc.sample_mn_pairs(x, 5, 42))
