"""Seeded synthetic datasets with the shapes and distributions of the benchmark configurations.

No public dataset is used; these generators stand in for them (float32, row-major):

* ``isotropic_mixture``: n x d, k isotropic Gaussians, centres ~ N(0, centre_std^2 I), within-cluster
  sigma, equal weights (2,000 x 100, 10 clusters, centre_std 5, sigma 1 for the CPU-runnable case).
* ``image_like``: n x 784 in [0, 1] quantised to multiples of 1/255: 10 classes, each with a rank-20
  basis W_c (entries U(0, 0.15)) and latent z ~ N(mu_c, I), x = clip(W_c z + 0.1 eps, 0, 1).
* ``anisotropic_mixture``: n x d, k Gaussians with a random rotation per cluster, axis scales
  log-uniform in [0.3, 3], centres ~ N(0, 16 I), cluster sizes ~ Dirichlet(2) (1,000,000 x 128, 50).
* ``subspace_mixture``: n x d, k Gaussians on a random 32-dim subspace plus isotropic noise 0.05 in
  the other d - 32 dims (4,000,000 x 256, 200 clusters).
"""
from __future__ import annotations

import numpy as np


def isotropic_mixture(n=2000, d=100, k=10, centre_std=5.0, sigma=1.0, seed=0):
    rng = np.random.default_rng(seed)
    centres = rng.normal(0.0, centre_std, size=(k, d))
    labels = np.repeat(np.arange(k), -(-n // k))[:n]
    rng.shuffle(labels)
    x = centres[labels] + rng.normal(0.0, sigma, size=(n, d))
    return x.astype(np.float32), labels


def image_like(n=60000, d=784, classes=10, rank=20, seed=0):
    rng = np.random.default_rng(seed)
    W = rng.uniform(0.0, 0.15, size=(classes, d, rank))
    mu = rng.normal(0.0, 1.0, size=(classes, rank))
    labels = rng.integers(0, classes, size=n)
    x = np.empty((n, d), np.float32)
    for c in range(classes):
        idx = np.nonzero(labels == c)[0]
        if idx.size == 0:
            continue
        z = mu[c] + rng.normal(0.0, 1.0, size=(idx.size, rank))
        v = z @ W[c].T + 0.1 * rng.normal(0.0, 1.0, size=(idx.size, d))
        x[idx] = (np.round(np.clip(v, 0.0, 1.0) * 255.0) / 255.0).astype(np.float32)
    return x, labels


def _rotation(rng, d):
    q, r = np.linalg.qr(rng.normal(size=(d, d)))
    return q * np.sign(np.diag(r))


def anisotropic_mixture(n=1_000_000, d=128, k=50, seed=0, chunk=1 << 16, draw_seed=None):
    """``seed`` fixes the mixture (centres, weights, rotations, scales); ``draw_seed`` (default: the
    same stream) the points drawn from it, so two draw seeds give fresh samples of one generator."""
    rng = np.random.default_rng(seed)
    rd = rng if draw_seed is None else np.random.default_rng(draw_seed)
    centres = rng.normal(0.0, 4.0, size=(k, d))
    weights = rng.dirichlet(np.full(k, 2.0))
    sizes = rd.multinomial(n, weights)
    x = np.empty((n, d), np.float32)
    labels = np.empty(n, np.int32)
    row = 0
    for c in range(k):
        rot = _rotation(rng, d)
        scales = np.exp(rng.uniform(np.log(0.3), np.log(3.0), size=d))
        a = (rot * scales).astype(np.float64)  # x = centre + rot @ diag(scales) @ z
        m = int(sizes[c])
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            z = rd.normal(size=(e - s, d))
            x[row + s:row + e] = (centres[c] + z @ a.T).astype(np.float32)
        labels[row:row + m] = c
        row += m
    perm = rd.permutation(n)
    return x[perm], labels[perm]


def subspace_mixture(n=4_000_000, d=256, k=200, sub=32, noise=0.05, seed=0, chunk=1 << 16, draw_seed=None):
    """``seed`` fixes the subspace and the centres; ``draw_seed`` (default: the same stream) the points."""
    rng = np.random.default_rng(seed)
    rd = rng if draw_seed is None else np.random.default_rng(draw_seed)
    basis = _rotation(rng, d)
    on, off = basis[:, :sub], basis[:, sub:]
    centres = rng.normal(0.0, 4.0, size=(k, sub))
    labels = rd.integers(0, k, size=n).astype(np.int32)
    x = np.empty((n, d), np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        z = centres[labels[s:e]] + rd.normal(size=(e - s, sub))
        w = noise * rd.normal(size=(e - s, d - sub))
        x[s:e] = (z @ on.T + w @ off.T).astype(np.float32)
    return x, labels


def quality_sample(n, n_sample=10_000, n_triplets_per_point=5, seed=1234):
    """Seeded query sample and random triplets (i, j, l) for the quality metrics."""
    rng = np.random.default_rng(seed)
    sample = rng.choice(n, size=min(n_sample, n), replace=False).astype(np.uint32)
    i = np.repeat(sample, n_triplets_per_point)
    j = rng.integers(0, n, size=i.size)
    l = rng.integers(0, n, size=i.size)
    keep = (j != i) & (l != i) & (j != l)
    trip = np.stack([i[keep], j[keep], l[keep]], 1).astype(np.uint32)
    return sample, trip
