"""The learned initialiser on the GPU: tcgen05 MLP gradients against the CPU oracle (oracle/mlp.py), one
AdamW step, training, inference, the learned fit_transform path, and what the trained network gains.
"""
import numpy as np
import pytest

from oracle import mlp as om

pytestmark = pytest.mark.gpu

TENSORS = ("W1", "b1", "W2", "b2", "W3", "b3")


def _split(g, d, dim):
    return dict(zip(TENSORS, om.unflatten(g, d, dim)))


@pytest.mark.parametrize("d,dim,B", [(128, 2, 256), (37, 3, 128), (200, 2, 384), (64, 8, 128)])
def test_mlp_gradient_matches_oracle(lib, d, dim, B):
    rng = np.random.default_rng(d * 31 + dim)
    p = lib.learned.init_params(d, dim, seed=d)
    x = rng.normal(scale=0.7, size=(B, d)).astype(np.float32)
    t = rng.normal(size=(B, dim)).astype(np.float32)
    loss, g = lib.learned.gradient(p, x, t)
    loss_o, g_o = om.loss_and_grad(p, x, t, d, dim, bf16_ops=True)
    # same BF16 rounding points; only the FP32 accumulation order differs (tensor cores vs float64)
    assert abs(loss - loss_o) <= 1e-4 * loss_o
    gs, gos = _split(g, d, dim), _split(g_o, d, dim)
    for name in TENSORS:
        rel = np.linalg.norm(gs[name] - gos[name]) / max(np.linalg.norm(gos[name]), 1e-30)
        assert rel < 5e-3, f"{name}: relative error {rel:.2e}"


def test_mlp_apply_matches_oracle_across_padding_and_chunks(lib):
    d, dim = 16, 2
    rng = np.random.default_rng(4)
    p = lib.learned.init_params(d, dim, seed=9)
    n = (1 << 18) + 300  # two inference chunks, the second ragged
    x = rng.normal(size=(n, d)).astype(np.float32)
    y = lib.learned.apply(p, x, dim)
    rows = np.concatenate([np.arange(0, 200), np.arange((1 << 18) - 100, n)])
    want = om.apply(p, x[rows], d, dim, bf16_ops=True)
    scale = np.abs(want).max()
    assert np.abs(y[rows] - want).max() <= 2e-3 * scale
    # rows are independent: applying a slice gives the same rows bit for bit
    assert np.array_equal(lib.learned.apply(p, x[:1000], dim), y[:1000])


def _zscore(t):
    t = t.astype(np.float64)
    return ((t - t.mean(0)) / t.std(0)).astype(np.float32)


def test_mlp_training_step_is_adamw_on_the_oracle_gradient(lib):
    d, dim, B = 64, 2, 256
    rng = np.random.default_rng(5)
    p0 = lib.learned.init_params(d, dim, seed=3)
    x = rng.normal(size=(B, d)).astype(np.float32)
    t = rng.normal(size=(B, dim)).astype(np.float32)
    lr, wd = 1e-3, 1e-2
    p1, losses = lib.learned.train(p0, x, t, epochs=1, batch=B, lr=lr, weight_decay=wd, seed=1)
    _, g_o = om.loss_and_grad(p0, x, _zscore(t), d, dim, bf16_ops=True)
    p1_o, _, _ = om.adamw(p0.astype(np.float64), g_o, np.zeros_like(g_o), np.zeros_like(g_o), 1, lr, wd, d, dim)
    # step 1 of Adam moves every weight by about lr * sign(g): only near-zero gradients may disagree
    bad = np.abs((p1 - p0) - (p1_o - p0)) > 0.05 * lr
    assert bad.mean() < 0.01, f"{bad.mean():.4f} of the parameters moved differently"
    assert losses.shape == (1,) and np.isfinite(losses[0])


def test_mlp_training_reduces_loss_and_generalises(lib):
    d, dim = 16, 2
    rng = np.random.default_rng(6)

    def target(x):
        return np.stack([np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2], np.tanh(x[:, 3] - x[:, 4]) + 0.5 * x[:, 5]], 1)

    x = rng.normal(size=(16384, d)).astype(np.float32)
    xt = rng.normal(size=(4096, d)).astype(np.float32)
    p0 = lib.learned.init_params(d, dim, seed=0)
    p, losses = lib.learned.train(p0, x, target(x), epochs=12, batch=512, lr=2e-3, weight_decay=1e-4, seed=2)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.15 * losses[0], losses
    # held-out rows, against the same z-scoring of the training targets
    t = target(x).astype(np.float64)
    tt = (target(xt) - t.mean(0)) / t.std(0)
    mse = np.mean((lib.learned.apply(p, xt, dim) - tt) ** 2)
    assert mse < 0.1, mse


def test_learned_fit_transform_is_value_init_from_the_network(lib):
    from pacmap_b200 import datasets

    x, _ = datasets.anisotropic_mixture(3000, 32, 6, seed=2)
    p = lib.learned.init_params(32, 2, seed=4)
    cfg = lib.Configuration(seed=3, num_iters=(0, 20, 30))
    y_learned, _ = lib.learned.fit_transform_learned(x, p, cfg)
    xp, *_ = lib.stages.preprocess(x)
    init = lib.learned.apply(p, xp, 2)
    y_value, _ = lib.fit_transform(x, lib.Configuration(seed=3, num_iters=(0, 20, 30),
                                                        initialization=lib.Initialization.Value(init)))
    assert np.array_equal(y_learned, y_value)


def test_learned_init_gains_over_random_init_on_the_short_schedule(lib):
    """What the trained network buys: from its prediction the shortened schedule (0, 50, 150) reaches the
    plain schedule's 10-NN preservation (within 0.005) and beats the same short schedule from Random init."""
    from pacmap_b200 import datasets

    n, d, k = 20000, 32, 12
    x_train, _ = datasets.anisotropic_mixture(n, d, k, seed=11)
    x_new, _ = datasets.anisotropic_mixture(n, d, k, seed=11, draw_seed=99)
    plain = lib.Configuration(seed=1, initialization=lib.Initialization.Random(7))
    y_train, _ = lib.fit_transform(x_train, plain)
    xp_train, *_ = lib.stages.preprocess(x_train)
    p, losses = lib.learned.train(lib.learned.init_params(d, 2, seed=0), xp_train, y_train, epochs=20, batch=1024,
                                  lr=1e-3, weight_decay=1e-4, seed=0)
    assert losses[-1] < losses[0]

    sample, trip = datasets.quality_sample(n, 5000, seed=5)
    y_plain, _ = lib.fit_transform(x_new, plain)
    short = lib.Configuration(seed=1, num_iters=lib.learned.SHORT_SCHEDULE, initialization=lib.Initialization.Random(7))
    y_short, _ = lib.fit_transform(x_new, short)
    y_learned, _ = lib.learned.fit_transform_learned(x_new, p, short)
    y_scaled, _ = lib.learned.fit_transform_learned(x_new, p, short, target_stats=lib.learned.target_stats(y_train))
    q_plain = lib.quality(x_new, y_plain, sample, trip)
    q_short = lib.quality(x_new, y_short, sample, trip)
    q_learned = lib.quality(x_new, y_learned, sample, trip)
    q_scaled = lib.quality(x_new, y_scaled, sample, trip)
    print(f"plain {q_plain}, random+short {q_short}, learned+short {q_learned}, learned (own scale)+short {q_scaled}")
    assert q_learned[0] >= q_plain[0] - 0.005
    assert q_learned[1] >= q_short[1] + 0.02
    # started in the training embedding's coordinates, the short schedule keeps more of the predicted layout
    # than through the 1e-4 Value z-scoring (0.728 vs 0.718 here, plain 0.734; the benchmark's gate is
    # measured at 1M x 128)
    assert q_scaled[1] > q_learned[1]
    assert q_scaled[0] >= q_plain[0] - 0.005 and q_scaled[1] >= q_plain[1] - 0.01


def test_learned_start_in_training_coordinates_is_the_destandardised_prediction(lib):
    # with target statistics the fit starts from MLP(x') * std + mean: zero iterations return exactly that
    from pacmap_b200 import datasets

    x, _ = datasets.anisotropic_mixture(3000, 32, 6, seed=2)
    p = lib.learned.init_params(32, 2, seed=4)
    mean, std = np.array([3.0, -2.0], np.float32), np.array([10.0, 20.0], np.float32)
    y0, _ = lib.learned.fit_transform_learned(x, p, lib.Configuration(seed=3, num_iters=(0, 0, 0)),
                                              target_stats=(mean, std))
    xp, *_ = lib.stages.preprocess(x)
    z = lib.learned.apply(p, xp, 2)
    assert np.array_equal(y0, (z * std + mean).astype(np.float32))


def test_transform_is_the_training_preprocessing_the_network_and_the_embedding_scale(lib, tmp_path):
    """model.transform(x) = MLP((x - min) / max - mean) * std + mean_t, with the training data's constants:
    bit for bit on the training points (their x' is pacmap_preprocess's), within BF16 tolerance of the
    CPU oracle on new points, and the same after a save / load round trip."""
    from pacmap_b200 import datasets

    d, dim = 32, 2
    x, _ = datasets.anisotropic_mixture(4000, d, 6, seed=5)
    y = np.random.default_rng(1).normal(size=(4000, dim)).astype(np.float32) * [3.0, 0.5] + [1.0, -2.0]
    model, losses = lib.learned.fit_model(x, y.astype(np.float32), epochs=2, batch=1024)
    assert np.all(np.isfinite(losses))
    xp, *_ = lib.stages.preprocess(x)
    z = lib.learned.apply(model.params, xp, dim)
    got = model.transform(x)
    assert np.array_equal(got, z * model.target_std + model.target_mean)
    path = tmp_path / "model.bin"
    model.save(path)
    assert np.array_equal(lib.learned.LearnedModel.load(path).transform(x), got)
    # new draws of the generator against the oracle: preprocessing with the stored constants in f32
    x_new, _ = datasets.anisotropic_mixture(3000, d, 6, seed=5, draw_seed=77)
    f = np.float32
    xn = ((x_new - f(model.pre_min)).astype(f) / f(model.pre_max)).astype(f) - model.pre_mean
    want = (om.apply(model.params, xn.astype(f), d, dim, bf16_ops=True) * model.target_std
            + model.target_mean).astype(f)
    got_new = model.transform(x_new)
    assert np.abs(got_new - want).max() <= 2e-3 * np.abs(want).max()


def test_transform_places_new_draws_like_a_fit_of_them(lib):
    """What the saved model buys: fresh draws embedded by transform alone (no optimisation at all) keep
    the triplet order of a full plain fit of those draws and about half of its 10-NN preservation, far
    above chance (measured: triplets 0.738 vs 0.731, 10-NN 0.059 vs 0.119, random 0.498 / 0.002)."""
    from pacmap_b200 import datasets

    n, d, k = 20000, 32, 12
    x_train, _ = datasets.anisotropic_mixture(n, d, k, seed=11)
    y_train, _ = lib.fit_transform(x_train, lib.Configuration(seed=1, initialization=lib.Initialization.Random(7)))
    model, _ = lib.learned.fit_model(x_train, y_train, epochs=20, batch=1024)
    x_new, _ = datasets.anisotropic_mixture(5000, d, k, seed=11, draw_seed=99)
    y_new = model.transform(x_new)
    y_fit, _ = lib.fit_transform(x_new, lib.Configuration(seed=1, initialization=lib.Initialization.Random(7)))
    sample, trip = datasets.quality_sample(5000, 2000, seed=5)
    q_tr = lib.quality(x_new, y_new, sample, trip)
    q_fit = lib.quality(x_new, y_fit, sample, trip)
    y_rand = np.random.default_rng(0).normal(size=y_new.shape).astype(np.float32)
    q_rand = lib.quality(x_new, y_rand, sample, trip)
    print(f"transform {q_tr}, plain fit {q_fit}, random {q_rand}")
    assert q_tr[1] >= q_fit[1] - 0.05
    assert q_tr[0] >= 0.35 * q_fit[0] and q_tr[0] > 10 * q_rand[0]
