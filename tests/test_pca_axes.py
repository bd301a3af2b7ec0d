"""Initialization::Pca's eigen-step on the host (pacmap_pca_axes; no GPU): the leading eigenvectors of a
symmetric matrix against numpy's f64 eigh, with the sign convention (largest loading positive), on
both paths (cyclic Jacobi for d <= 160, subspace iteration + Rayleigh-Ritz above)."""
import numpy as np
import pytest


@pytest.mark.parametrize("d,k,decay", [(30, 2, 0.8), (100, 8, 0.9), (160, 3, 0.95), (300, 100, 0.93), (784, 100, 0.97)])
def test_pca_axes_match_numpy(lib, d, k, decay):
    rng = np.random.default_rng(d)
    q, _ = np.linalg.qr(rng.normal(size=(d, d)))
    lam = 10.0 * decay ** np.arange(d)
    cov = (q * lam) @ q.T
    cov = 0.5 * (cov + cov.T)
    got = lib.stages.pca_axes(cov, k)
    w, v = np.linalg.eigh(cov)
    v = v[:, np.argsort(w)[::-1][:k]]
    v *= np.sign(v[np.abs(v).argmax(0), np.arange(k)])
    assert np.abs(got - v).max() < 1e-6
    assert np.allclose(got.T @ got, np.eye(k), atol=1e-9)


def test_pca_axes_rejects_bad_shapes(lib):
    with pytest.raises(lib.Unsupported):
        lib.stages.pca_axes(np.eye(4), 5)
