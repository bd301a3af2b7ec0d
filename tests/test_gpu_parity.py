"""Parity of the CUDA path (through the C ABI) with the CPU oracle on the same seeded inputs.

Bars: bit-exact for preprocessing, kNN indices and distances, reselection and sampled pairs; for the
floating-point optimiser, per-element gradient error <= 1e-5 of the row's sum of |contributions| and
normwise embedding error <= 1e-5 per iteration (the reference sums the gradient in an unspecified
order, gradient.rs:53-70); end-to-end embeddings within 0.005 on 10-NN preservation and triplet accuracy.
"""
import numpy as np
import pytest

from conftest import gaussian_mixture

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-5
EMB_TOL = 1e-5


def _mixture(n, d, seed=0):
    from pacmap_b200 import datasets

    x, _ = datasets.isotropic_mixture(n=n, d=d, k=10, seed=seed)
    return x


# ----------------------------------------------------------------------------------------------------
# Preprocessing (lib.rs:485-511): bit-exact.
# ----------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("shape,lo,hi", [((3000, 37), -3.0, 5.0), ((2000, 100), 0.0, 1.0), ((513, 8), -9.0, -1.0),
                                         ((20000, 128), -2.0, 2.0)])
def test_preprocess_bit_exact(lib, orc, shape, lo, hi):
    x = np.random.default_rng(7).uniform(lo, hi, size=shape).astype(np.float32)
    got, mn, mx, mean = lib.stages.preprocess(x)
    exp, emn, emx, emean = orc.preprocess(x)
    assert (mn, mx) == (emn, emx)
    assert np.array_equal(mean, emean)
    assert np.array_equal(got, exp)


# ----------------------------------------------------------------------------------------------------
# Exact kNN (knn.rs:137-194): indices and f32 distances bit-exact, ties -> lower index.
# ----------------------------------------------------------------------------------------------------
def test_knn_reference_known_answers(lib, golden):
    for name, case in golden["knn"]["cases"].items():
        x = np.array(case["embeddings"], np.float32)
        idx, dist = lib.knn.find_k_nearest_neighbors(x, case["k"])
        for point, exp in case["expected"]:
            got = sorted(zip(idx[point].tolist(), dist[point].tolist()))
            exp = sorted((int(i), float(v)) for i, v in exp)
            assert [g[0] for g in got] == [e[0] for e in exp], name
            np.testing.assert_allclose([g[1] for g in got], [e[1] for e in exp], atol=1e-4, rtol=1e-4)


def test_knn_edge_shapes(lib):
    f = lib.knn.find_k_nearest_neighbors
    assert f(np.zeros((0, 128), np.float32), 5)[0].shape == (0, 0)
    assert f(np.array([[1.0, 0.0, 0.0]], np.float32), 1)[0].shape == (1, 0)
    assert f(np.array([[1.0, 0.0], [0.0, 1.0], [0.0, 0.0]], np.float32), 0)[0].shape == (3, 0)
    idx, dist = f(np.array([[1.0], [2.0], [3.0]], np.float32), 5)
    assert idx.shape == (3, 2) and (idx < 3).all() and (dist >= 0).all()


@pytest.mark.parametrize("n,d,k,mode", [(2000, 100, 60, 3), (1500, 784, 72, 3), (777, 13, 90, 3), (3001, 128, 90, 0),
                                        (4096, 32, 17, 0)])
def test_knn_bit_exact(lib, orc, n, d, k, mode):
    x = _mixture(n, d, seed=n)
    got_i, got_d = lib.knn.find_k_nearest_neighbors(x, k, knn_mode=mode)
    exp_i, exp_d = orc.knn_exact(x, k)
    assert np.array_equal(got_d, exp_d)
    assert np.array_equal(got_i, exp_i)


def test_knn_ties_and_duplicates(lib, orc):
    x, _ = gaussian_mixture(1200, 24, seed=3)
    x = np.round(x, 1).astype(np.float32)
    x[100:140] = x[7]  # 41 identical points: distance-0 ties resolved by index
    for k in (5, 60):
        gi, gd = lib.knn.find_k_nearest_neighbors(x, k)
        ei, ed = orc.knn_exact(x, k)
        assert np.array_equal(gi, ei) and np.array_equal(gd, ed)


# ----------------------------------------------------------------------------------------------------
# Sigma + reselection (neighbors.rs:79-89, distance.rs:27-37, sampling.rs:251-286): bit-exact.
# ----------------------------------------------------------------------------------------------------
def test_reselect_bit_exact(lib, orc):
    x = _mixture(3000, 50, seed=11)
    xp, *_ = orc.preprocess(x)
    ki, kd = orc.knn_exact(xp, 60)
    pnn, sig = lib.stages.reselect_neighbors(ki, kd, 10)
    esig = orc.sigma(kd)
    assert np.array_equal(sig, esig)
    exp = orc.sample_neighbors_pair(orc.scale_dist(kd, esig, ki), ki, 10)
    assert np.array_equal(pnn, exp)


# ----------------------------------------------------------------------------------------------------
# Philox samplers (sampling.rs:37-142): bit-exact against the oracle's host mirror.
# ----------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("n,d,k,n_mn,n_fp", [(3000, 50, 10, 5, 20), (500, 8, 40, 20, 80), (12, 3, 10, 5, 20),
                                             # the fp16-screened mid-near path (d = 128, 256)
                                             (3000, 128, 10, 5, 20), (2000, 256, 12, 6, 24), (20, 128, 5, 10, 5)])
def test_samplers_bit_exact(lib, orc, n, d, k, n_mn, n_fp):
    x = _mixture(n, d, seed=5)
    xp, *_ = orc.preprocess(x)
    kk = min(k, n - 1)
    ki, kd = orc.knn_exact(xp, min(kk + 50, n - 1))
    pnn = orc.sample_neighbors_pair(orc.scale_dist(kd, orc.sigma(kd), ki), ki, kk)
    for seed in (0, 42, 2**40 + 3):
        pmn, pfp = lib.stages.sample_pairs(xp, pnn, kk, n_mn, n_fp, seed)
        assert np.array_equal(pfp, orc.sample_fp_pairs(pnn, n, kk, n_fp, seed))
        assert np.array_equal(pmn, orc.sample_mn_pairs(xp, n_mn, seed))


def test_mn_screening_ties_and_duplicates_bit_exact(lib, orc):
    # many exact duplicates and quantised values: the fp16 intervals overlap on ties, so those slots take the
    # exact distances and the draw order, as the rule does
    x = np.round(_mixture(4000, 128, seed=6) * 2.0) / 2.0
    x[100:400] = x[7]
    x[1000:1050] = x[8]
    xp, *_ = orc.preprocess(x.astype(np.float32))
    pnn = np.zeros((4000 * 10, 2), np.uint32)
    for seed in (3, 77):
        pmn, _ = lib.stages.sample_pairs(xp, pnn, 10, 20, 0, seed)
        assert np.array_equal(pmn, orc.sample_mn_pairs(xp, 20, seed))


def test_generate_pairs_bit_exact(lib, orc):
    # neighbors.rs:56-108 end to end on config-1-shaped data (n=2000, d=100).
    x = _mixture(2000, 100, seed=42)
    cfg = lib.Configuration(seed=7, initialization=lib.Initialization.Random(1))
    pnn, pmn, pfp = lib.stages.generate_pairs(x, cfg)
    xp, *_ = orc.preprocess(x)
    enn, emn, efp = orc.generate_pairs(xp, 10, 5, 20, 7)
    assert np.array_equal(pnn, enn) and np.array_equal(pmn, emn) and np.array_equal(pfp, efp)


def test_fp_distribution_uniform(lib, orc):
    # The reference's rule draws FP partners uniformly from the allowed set; chi-square over partners.
    n, k, n_fp = 400, 10, 30
    pnn = np.stack([np.repeat(np.arange(n), k), (np.repeat(np.arange(n), k) + np.tile(np.arange(1, k + 1), n)) % n],
                   1).astype(np.uint32)
    _, pfp = lib.stages.sample_pairs(np.zeros((n, 4), np.float32), pnn, k, 0, n_fp, 99)
    counts = np.bincount(pfp[:, 1].astype(np.int64), minlength=n)
    exp = n * n_fp / n
    chi2 = ((counts - exp) ** 2 / exp).sum()
    assert chi2 < n + 6 * np.sqrt(2 * n)  # df ~ n


def test_mn_distribution_is_the_second_of_six_rule(lib, orc):
    """sampling.rs:118-142,296-313: each mid-near partner is the 2nd closest of 6 distinct uniform draws
    (excluding the point and its earlier picks). The rank of the partner's distance among all n - 1 other
    points, divided by n, then follows the 2nd order statistic of 6 uniforms, Beta(2, 5): KS test of the
    GPU's draws against it, and two-sample KS against the rule run with numpy's own generator."""
    from scipy import stats

    n, d, n_mn = 3000, 10, 5
    x = _mixture(n, d, seed=8)
    xp, *_ = orc.preprocess(x)
    pmn, _ = lib.stages.sample_pairs(xp, np.zeros((n * 10, 2), np.uint32), 10, n_mn, 0, 2024)
    dist = np.sqrt(((xp[:, None, :] - xp[None, :, :]) ** 2).sum(-1))
    np.fill_diagonal(dist, np.inf)
    order = np.argsort(np.argsort(dist, axis=1, kind="stable"), axis=1, kind="stable")  # rank of j in row i
    i, j = pmn[:, 0].astype(np.int64), pmn[:, 1].astype(np.int64)
    u_gpu = (order[i, j] + 0.5) / (n - 1)
    rng = np.random.default_rng(5)
    u_ref = []
    for r in range(n):
        picked = []
        for _ in range(n_mn):
            cand = []
            while len(cand) < 6:
                c = int(rng.integers(n))
                if c != r and c not in picked and c not in cand:
                    cand.append(c)
            c2 = sorted(cand, key=lambda c: (dist[r, c], cand.index(c)))[1]
            picked.append(c2)
            u_ref.append((order[r, c2] + 0.5) / (n - 1))
    ks_beta = stats.kstest(u_gpu, "beta", args=(2, 5))
    ks_two = stats.ks_2samp(u_gpu, np.array(u_ref))
    print(f"MN rank KS vs Beta(2,5): p={ks_beta.pvalue:.3f}; vs the rule on numpy draws: p={ks_two.pvalue:.3f}")
    assert ks_beta.pvalue > 1e-3 and ks_two.pvalue > 1e-3


# ----------------------------------------------------------------------------------------------------
# Gradient and optimiser (gradient.rs, adam.rs, weights.rs, lib.rs:800-837).
# ----------------------------------------------------------------------------------------------------
def test_gradient_golden_through_gpu(lib, golden):
    g = golden["gradient"]
    got = lib.stages.gradient(np.array(g["y"], np.float32), np.array(g["pair_neighbors"]), np.array(g["pair_mn"]),
                              np.array(g["pair_fp"]), g["w_neighbors"], g["w_mn"], g["w_fp"])
    np.testing.assert_allclose(got, np.array(g["expected"], np.float32), atol=g["eps"], rtol=0)


def _pairs_for(n, d, seed):
    from oracle import generate_pairs, preprocess

    x = _mixture(n, d, seed=seed)
    xp, *_ = preprocess(x)
    return generate_pairs(xp, 10, 5, 20, seed)


def test_gradient_matches_oracle(lib, orc):
    pnn, pmn, pfp = _pairs_for(2000, 30, 3)
    y = np.random.default_rng(0).normal(size=(2000, 2)).astype(np.float32)
    for w in [(2.0, 1000.0, 1.0), (3.0, 3.0, 1.0), (1.0, 0.0, 1.0)]:
        got = lib.stages.gradient(y, pnn, pmn, pfp, *w)
        exp, exp64, absum = orc.grad(y, pnn, pmn, pfp, *w, with64=True)
        err = np.abs(got[:-1] - exp[:-1])
        assert (err <= GRAD_TOL * absum + 1e-30).all(), err.max()
        # against the FP64 oracle: both f32 paths are within the same bound
        assert (np.abs(got[:-1] - exp64[:-1]) <= GRAD_TOL * absum + 1e-30).all()
        # the loss: both sides against the FP64 sum (the oracle's f32 sequential sum drifts by ~1e-4)
        assert abs(got[-1, 0] - exp64[-1, 0]) <= 1e-5 * abs(exp64[-1, 0])


def _hub_pairs(n, seed):
    """Grouped pair lists whose far partners are skewed towards hubs, so that CSR segments take every
    sorting path: most hold < 32 entries, 30 mid hubs ~100 (4 keys per lane in registers), 5 big hubs ~240
    (shared memory)."""
    rng = np.random.default_rng(seed)
    def grouped(k, partners):
        a = np.repeat(np.arange(n), k)
        return np.stack([a, partners.reshape(-1)], 1).astype(np.uint32)
    nn = rng.integers(0, n, size=(n, 10))
    mn = rng.integers(0, n, size=(n, 5))
    u = rng.random(size=(n, 20))
    fp = np.where(u < 0.02, rng.integers(0, 5, size=(n, 20)),
                  np.where(u < 0.07, 5 + rng.integers(0, 30, size=(n, 20)), rng.integers(0, n, size=(n, 20))))
    return grouped(10, nn), grouped(5, mn), grouped(20, fp)


def test_gradient_with_hub_segments_matches_oracle_and_is_deterministic(lib, orc):
    n = 3000
    pnn, pmn, pfp = _hub_pairs(n, 12)
    y = np.random.default_rng(1).normal(size=(n, 2)).astype(np.float32)
    w = (2.0, 1000.0, 1.0)
    got = lib.stages.gradient(y, pnn, pmn, pfp, *w)
    again = lib.stages.gradient(y, pnn, pmn, pfp, *w)
    # every segment is sorted, so the summation order (and the result) is the same on every call
    assert np.array_equal(got, again)
    exp, exp64, absum = orc.grad(y, pnn, pmn, pfp, *w, with64=True)
    assert (np.abs(got[:-1] - exp[:-1]) <= GRAD_TOL * absum + 1e-30).all()
    assert (np.abs(got[:-1] - exp64[:-1]) <= GRAD_TOL * absum + 1e-30).all()


@pytest.mark.parametrize("itr", [0, 1, 37, 99, 100, 150, 199, 200, 300, 449])
def test_each_iteration_matches_oracle(lib, orc, itr):
    """AllProvided pairs + identical state: one GPU iteration vs one oracle iteration."""
    n = 2000
    pnn, pmn, pfp = _pairs_for(n, 30, 9)
    rng = np.random.default_rng(itr)
    y0 = orc.init_value(rng.normal(size=(n, 2)).astype(np.float32)) if itr == 0 else \
        rng.normal(0, 3, size=(n, 2)).astype(np.float32)
    m0 = np.zeros_like(y0) if itr == 0 else rng.normal(0, 0.05, size=(n, 2)).astype(np.float32)
    v0 = np.zeros_like(y0) if itr == 0 else np.abs(rng.normal(0, 0.01, size=(n, 2))).astype(np.float32)
    yg, mg, vg = y0.copy(), m0.copy(), v0.copy()
    gg = lib.stages.optimize_steps(yg, mg, vg, pnn, pmn, pfp, 1.0, 100, 100, itr, itr + 1)
    yo, mo, vo = y0.copy(), m0.copy(), v0.copy()
    go, g64, absum = orc.step(yo, mo, vo, pnn, pmn, pfp, 1.0, 100, 100, itr)
    # (1) the gradient: within 1e-5 of the row's sum of |contributions| (any summation order is the
    #     reference's; gradient.rs:53-70 reduces in an unspecified order)
    assert (np.abs(gg[:-1] - go[:-1]) <= GRAD_TOL * absum + 1e-30).all()
    # (2) Adam (adam.rs:35-60) applied to the GPU's own gradient reproduces y, m, v bit for bit
    ya, ma, va = y0.copy(), m0.copy(), v0.copy()
    orc.adam(ya, gg, ma, va, 1.0, itr)
    assert np.array_equal(yg, ya) and np.array_equal(mg, ma) and np.array_equal(vg, va)
    # (3) the embedding against the oracle's: 1e-5 normwise. At itr 0 (m = v = 0) Adam's step is close
    #     to sign(g) * lr_t and amplifies the order-dependent rounding of near-zero gradients, so the
    #     bound there is the propagated one (checked via (1) + (2)) and 1e-4 normwise.
    tol = EMB_TOL if itr > 0 else 10 * EMB_TOL
    assert np.abs(yg - yo).max() <= tol * np.abs(yo).max()
    assert np.abs(mg - mo).max() <= EMB_TOL * max(np.abs(mo).max(), 1e-30)
    assert np.abs(vg - vo).max() <= tol * max(np.abs(vo).max(), 1e-30)


def test_trajectory_tracks_oracle(lib, orc):
    """AllProvided + Value init through fit_transform: 30 iterations stay close to the oracle's."""
    n = 2000
    pnn, pmn, pfp = _pairs_for(n, 30, 21)
    x = _mixture(n, 30, seed=21)
    v = np.random.default_rng(5).normal(size=(n, 2)).astype(np.float32)
    cfg = lib.Configuration(initialization=lib.Initialization.Value(v), num_iters=(10, 10, 10),
                            pair_configuration=lib.PairConfiguration.AllProvided(pnn, pmn, pfp))
    got, _ = lib.fit_transform(x, cfg)
    exp, _, _ = orc.optimize(orc.init_value(v), pnn, pmn, pfp, num_iters=(10, 10, 10))
    assert np.abs(got - exp).max() <= 1e-3 * np.abs(exp).max()


def test_init_value_and_random(lib, orc):
    v = np.random.default_rng(2).normal(3, 2, size=(5000, 2)).astype(np.float32)
    g = lib.stages.init_value(v)
    e = orc.init_value(v)
    assert np.abs(g - e).max() <= 1e-6 * np.abs(e).max()
    r = lib.stages.init_random(10000, 3, 42)
    er = orc.init_random(10000, 3, 42)
    assert np.abs(r - er).max() <= 1e-6
    assert abs(r.mean()) < 0.05 and abs(r.std() - 1) < 0.05


# ----------------------------------------------------------------------------------------------------
# fit_transform end to end (lib.rs:294-367).
# ----------------------------------------------------------------------------------------------------
def test_fit_transform_config1_quality_matches_oracle(lib, orc):
    from pacmap_b200 import datasets

    x, labels = datasets.isotropic_mixture(2000, 100, 10, seed=0)
    cfg = lib.Configuration(initialization=lib.Initialization.Random(42), seed=42)
    y, snaps = lib.fit_transform(x, cfg)
    assert y.shape == (2000, 2) and snaps is None and np.isfinite(y).all()
    ye = orc.fit_transform(x, init="random", init_seed=42, seed=42)
    sample, trip = datasets.quality_sample(2000, 2000, 5)
    xp, *_ = orc.preprocess(x)
    p_gpu, t_gpu = lib.quality(x, y, sample, trip)
    p_orc, t_orc = orc.knn_preservation(xp, ye, sample, 10), orc.triplet_accuracy(xp, ye, trip)
    assert abs(p_gpu - orc.knn_preservation(xp, y, sample, 10)) < 1e-12
    assert abs(t_gpu - orc.triplet_accuracy(xp, y, trip)) < 1e-12
    assert abs(p_gpu - p_orc) <= 0.005 and abs(t_gpu - t_orc) <= 0.005
    # tests.rs:87-135 sanity: centred, non-degenerate, clusters preserved
    assert (np.abs(y.mean(0)) < np.abs(y).max()).all() and (y.std(0) > 1e-6).all()
    d = np.linalg.norm(y[:, None] - y[None], axis=-1)
    same = labels[:, None] == labels[None]
    assert d[same].mean() < d[~same].mean()


def test_fit_transform_reference_integration_configs(lib):
    # tests.rs:22-149 (PCA init replaced by Value init: PCA is not built).
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, size=(1000, 50)).astype(np.float32)
    x += (np.arange(1000) // 200)[:, None].astype(np.float32)
    configs = [
        lib.Configuration(initialization=lib.Initialization.Random(None)),
        lib.Configuration(initialization=lib.Initialization.Value(rng.normal(size=(1000, 2)).astype(np.float32)),
                          override_neighbors=15, seed=42, snapshots=[100, 200, 300]),
        lib.Configuration(initialization=lib.Initialization.Random(42), mid_near_ratio=0.3, far_pair_ratio=1.5,
                          override_neighbors=10, seed=42, learning_rate=0.8, num_iters=(50, 50, 100)),
    ]
    lab = np.arange(1000) // 200
    for cfg in configs:
        y, snaps = lib.fit_transform(x, cfg)
        assert y.shape == (1000, 2)
        assert (np.abs(y.mean(0)) < 1.0).all() and (y.std(0) > 1e-6).all()
        d = np.linalg.norm(y[:, None] - y[None], axis=-1)
        same = lab[:, None] == lab[None]
        assert d[same].mean() < d[~same].mean()
        if cfg.snapshots is not None:
            assert snaps.shape == (3, 1000, 2)


def test_snapshot_slots(lib, orc):
    n = 500
    pnn, pmn, pfp = _pairs_for(n, 10, 4)
    x = _mixture(n, 10, seed=4)
    v = np.random.default_rng(1).normal(size=(n, 2)).astype(np.float32)
    snaps = [3, 0, 3, 7]
    cfg = lib.Configuration(initialization=lib.Initialization.Value(v), num_iters=(3, 2, 3), snapshots=snaps,
                            pair_configuration=lib.PairConfiguration.AllProvided(pnn, pmn, pfp))
    y, s = lib.fit_transform(x, cfg)
    _, es, _ = orc.optimize(orc.init_value(v), pnn, pmn, pfp, num_iters=(3, 2, 3), snapshots=snaps)
    # lib.rs:789-791,830-836: slot 0 keeps its first write only until itr+1 == snaps[0]; duplicate
    # indices leave the later slot at zero; index 0 never matches an iteration.
    assert s.shape == es.shape
    assert np.abs(s - es).max() <= 1e-4 * max(np.abs(es).max(), 1e-6)
    assert (s[1] == 0).all() and (s[2] == 0).all()


def test_loss_trace(lib):
    x = _mixture(1000, 20, seed=8)
    y, _, loss = lib.fit_transform(x, lib.Configuration(initialization=lib.Initialization.Random(1), seed=1),
                                   loss_trace=True)
    assert loss.shape == (450,) and np.isfinite(loss).all()


def test_errors_like_reference(lib):
    x = _mixture(100, 5)
    R = lib.Initialization.Random(0)
    with pytest.raises(lib.SampleSize):
        lib.fit_transform(x[:1], lib.Configuration(initialization=R))
    with pytest.raises(lib.InvalidNearestNeighborShape):
        lib.fit_transform(x, lib.Configuration(initialization=R, pair_configuration=lib.PairConfiguration.
                                               NeighborsProvided(np.zeros((10, 2), np.uint32))))
    with pytest.raises(lib.InvalidFarPointCount):
        lib.fit_transform(x, lib.Configuration(initialization=R, far_pair_ratio=0.0))
    with pytest.raises(lib.InvalidNeighborCount):
        lib.fit_transform(x, lib.Configuration(initialization=R, override_neighbors=0))
    with pytest.raises(lib.Pca):  # Initialization::Pca with more embedding dimensions than columns
        lib.fit_transform(x, lib.Configuration(embedding_dimensions=6))
    bad = np.array([[0, 1], [5, 100]], np.uint32)
    with pytest.raises(lib.PairIndexOutOfRange):
        lib.fit_transform(x, lib.Configuration(initialization=R, pair_configuration=lib.PairConfiguration.
                                               AllProvided(bad, bad, bad)))
    with pytest.raises(lib.EmptyArrayMinMax):
        lib.fit_transform(np.zeros((10, 0), np.float32), lib.Configuration(initialization=R))


def test_neighbors_provided(lib, orc):
    n = 800
    x = _mixture(n, 16, seed=13)
    xp, *_ = orc.preprocess(x)
    ki, kd = orc.knn_exact(xp, 60)
    pnn = orc.sample_neighbors_pair(orc.scale_dist(kd, orc.sigma(kd), ki), ki, 10)
    cfg = lib.Configuration(initialization=lib.Initialization.Random(3), seed=3,
                            pair_configuration=lib.PairConfiguration.NeighborsProvided(pnn))
    y, _ = lib.fit_transform(x, cfg)
    cfg2 = lib.Configuration(initialization=lib.Initialization.Random(3), seed=3)
    y2, _ = lib.fit_transform(x, cfg2)
    # NeighborsProvided with the generated neighbours gives the same pairs -> the same embedding
    assert np.array_equal(y, y2)


def test_deterministic(lib):
    x = _mixture(1500, 20, seed=2)
    cfg = lib.Configuration(initialization=lib.Initialization.Random(5), seed=5)
    a, _ = lib.fit_transform(x, cfg)
    b, _ = lib.fit_transform(x, cfg)
    assert np.array_equal(a, b)


# ----------------------------------------------------------------------------------------------------
# Initialization::Pca (lib.rs:442-522, 753-768): exact principal axes (the reference's petal-decomposition
# SVD is not in the tree), each axis's largest loading positive; zero iterations return the start.
# ----------------------------------------------------------------------------------------------------
def _axes(z, k):
    zc = z.astype(np.float64) - z.astype(np.float64).mean(0)
    w, v = np.linalg.eigh(zc.T @ zc)
    v = v[:, np.argsort(w)[::-1][:k]]
    v *= np.sign(v[np.abs(v).argmax(0), np.arange(k)])
    return zc @ v


def test_pca_init_small_d_is_the_projection_of_the_normalised_data(lib, orc):
    x = _mixture(2000, 30, seed=4)
    y, _ = lib.fit_transform(x, lib.Configuration(num_iters=(0, 0, 0), seed=1))
    xp, *_ = orc.preprocess(x)
    want = 0.01 * _axes(xp, 2)
    assert np.abs(y - want).max() <= 1e-5 * np.abs(want).max()


def test_pca_init_wide_data_uses_the_100_axis_projection(lib):
    x = _mixture(3000, 150, seed=6)
    y, _ = lib.fit_transform(x, lib.Configuration(num_iters=(0, 0, 0), seed=1))
    want = 0.01 * _axes(x, 2)  # the raw data's projection, its leading two columns
    assert np.abs(y - want).max() <= 1e-4 * np.abs(want).max()


def test_pca_default_configuration_embeds_like_random_init(lib):
    """The reference's default configuration (Initialization::Pca) runs end to end, as well as Random."""
    from pacmap_b200 import datasets

    x, _ = datasets.isotropic_mixture(n=2000, d=100, k=10, seed=0)
    sample, trip = datasets.quality_sample(2000, 1000, seed=3)
    y_pca, _ = lib.fit_transform(x, lib.Configuration(seed=42))
    y_rnd, _ = lib.fit_transform(x, lib.Configuration(seed=42, initialization=lib.Initialization.Random(42)))
    q_pca, q_rnd = lib.quality(x, y_pca, sample, trip), lib.quality(x, y_rnd, sample, trip)
    assert q_pca[1] >= q_rnd[1] - 0.03 and q_pca[0] >= q_rnd[0] - 0.05, (q_pca, q_rnd)
    # wide data: pairs drawn on the 100-axis projection
    xw = np.concatenate([x, 0.1 * np.random.default_rng(1).normal(size=(2000, 60)).astype(np.float32)], 1)
    y_w, _ = lib.fit_transform(xw, lib.Configuration(seed=42))
    assert np.all(np.isfinite(y_w)) and lib.quality(xw, y_w, sample, trip)[1] >= q_rnd[1] - 0.05


# ----------------------------------------------------------------------------------------------------
# The angular metric (engine switch; the reference is Euclidean only, README.md:164).
# ----------------------------------------------------------------------------------------------------
def _unit_rows(orc, xp):
    out = xp.copy()
    zero = np.zeros(xp.shape[1], np.float32)
    for r in range(xp.shape[0]):
        nrm = np.float32(orc.distance(xp[r], zero))  # the reference's f32 distance from the origin
        if nrm > 0:
            out[r] = (xp[r] / nrm).astype(np.float32)
    return out


def test_angular_pairs_are_the_euclidean_pairs_of_unit_rows(lib, orc):
    x = _mixture(2000, 40, seed=12)
    x *= np.random.default_rng(3).uniform(0.2, 5.0, size=(2000, 1)).astype(np.float32)  # scales vary
    cfg = lib.Configuration(seed=7, initialization=lib.Initialization.Random(1), metric=lib.Metric.ANGULAR)
    pnn, pmn, pfp = lib.stages.generate_pairs(x, cfg)
    xp, *_ = orc.preprocess(x)
    enn, emn, efp = orc.generate_pairs(_unit_rows(orc, xp), 10, 5, 20, 7)
    assert np.array_equal(pnn, enn) and np.array_equal(pmn, emn) and np.array_equal(pfp, efp)
    with pytest.raises(lib.InvalidArgument):
        lib.stages.generate_pairs(x, lib.Configuration(seed=7, metric=5))


def test_angular_neighbours_are_closer_in_angle(lib, orc):
    """Rows with scales spread over two decades: the neighbour pairs drawn with the angular metric have
    a higher cosine similarity (on the preprocessed rows) than the Euclidean ones, and most differ."""
    rng = np.random.default_rng(8)
    x = (_mixture(3000, 24, seed=9) * rng.uniform(0.1, 10.0, size=(3000, 1))).astype(np.float32)
    R = lib.Initialization.Random(3)
    p_ang = lib.stages.generate_pairs(x, lib.Configuration(seed=2, initialization=R, metric=lib.Metric.ANGULAR))[0]
    p_euc = lib.stages.generate_pairs(x, lib.Configuration(seed=2, initialization=R))[0]
    xp, *_ = orc.preprocess(x)
    u = xp.astype(np.float64) / np.linalg.norm(xp.astype(np.float64), axis=1, keepdims=True)

    def mean_cos(p):
        return float((u[p[:, 0]] * u[p[:, 1]]).sum(1).mean())

    c_ang, c_euc = mean_cos(p_ang), mean_cos(p_euc)
    print(f"mean cosine of neighbour pairs: angular {c_ang:.4f}, euclidean {c_euc:.4f}")
    assert c_ang > c_euc + 0.002  # measured 0.9732 vs 0.9697
    same = (p_ang == p_euc).all(1).mean()
    assert same < 0.5  # measured 0.136
