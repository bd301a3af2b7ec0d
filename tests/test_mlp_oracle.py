"""The learned initialiser's CPU oracle (oracle/mlp.py), pinned without a GPU.

The MLP has no counterpart in the reference, so there are no golden vectors: the float64 backward pass
is pinned by central differences, and the BF16 rounding by torch's own bfloat16 conversion.
"""
import numpy as np
import pytest

from oracle import mlp as om


def _problem(d=7, dim=2, B=16, seed=0):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-0.1, 0.1, size=om.param_count(d, dim))
    x = rng.normal(size=(B, d))
    t = rng.normal(size=(B, dim))
    return p, x, t


def test_backward_matches_finite_differences():
    d, dim = 7, 2
    p, x, t = _problem(d, dim)
    _, g = om.loss_and_grad(p, x, t, d, dim, bf16_ops=False)
    sizes = [512 * d, 512, 512 * 512, 512, dim * 512, dim]
    starts = np.cumsum([0] + sizes[:-1])
    rng = np.random.default_rng(1)
    # a few entries of every tensor (W1, b1, W2, b2, W3, b3)
    idx = np.concatenate([s + rng.choice(n, size=min(n, 6), replace=False) for s, n in zip(starts, sizes)])
    fd = om.finite_difference(p, x, t, d, dim, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=1e-5, atol=1e-9)


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2)
    a = np.concatenate([rng.normal(scale=s, size=4000) for s in (1e-30, 1e-3, 1.0, 1e6)]).astype(np.float32)
    # exact ties (the low 16 bits 0x8000) and values just around them
    u = rng.integers(0, 2**31, size=2000, dtype=np.uint64).astype(np.uint32) & np.uint32(0xFFFF0000)
    ties = np.concatenate([(u | 0x8000), (u | 0x7FFF), (u | 0x8001)]).view(np.float32)
    a = np.concatenate([a, ties[np.isfinite(ties)]])
    want = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(om.bf16(a), want)


def test_bf16_gradient_stays_close_to_float64():
    # the rounding points cost accuracy at the BF16 level, amplified by the cancellation in the batch sums
    d, dim = 32, 2
    p, x, t = _problem(d, dim, B=256, seed=3)
    _, g64 = om.loss_and_grad(p, x, t, d, dim, bf16_ops=False)
    _, g16 = om.loss_and_grad(p.astype(np.float32), x.astype(np.float32), t.astype(np.float32), d, dim, bf16_ops=True)
    rel = np.linalg.norm(g16 - g64) / np.linalg.norm(g64)
    assert rel < 5e-2


def test_adamw_first_step_is_signed_learning_rate():
    d, dim = 3, 2
    p, x, t = _problem(d, dim)
    _, g = om.loss_and_grad(p, x, t, d, dim, bf16_ops=False)
    lr, wd = 1e-3, 0.1
    p1, m, v = om.adamw(p, g, np.zeros_like(p), np.zeros_like(p), 1, lr, wd, d, dim)
    decay = np.concatenate([np.full(s.size, wd if s.ndim == 2 else 0.0) for s in om.unflatten(p, d, dim)])
    big = np.abs(g) > 1e-5
    np.testing.assert_allclose((p1 - p * (1 - lr * decay))[big], -lr * np.sign(g[big]), rtol=1e-3)


def test_library_parameter_layout_and_init(lib):
    d, dim = 37, 3
    assert lib.learned.param_count(d, dim) == om.param_count(d, dim)
    p = lib.learned.init_params(d, dim, seed=5)
    assert np.array_equal(p, lib.learned.init_params(d, dim, seed=5))
    assert not np.array_equal(p, lib.learned.init_params(d, dim, seed=6))
    W1, b1, W2, b2, W3, b3 = om.unflatten(p, d, dim)
    for w, fan_in in ((W1, d), (b1, d), (W2, 512), (b2, 512), (W3, 512), (b3, 512)):
        bound = 1 / np.sqrt(fan_in)
        assert np.all(np.abs(w) <= bound)
        if w.size >= 100:
            assert np.abs(w).max() > 0.9 * bound
