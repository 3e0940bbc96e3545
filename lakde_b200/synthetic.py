"""Seeded synthetic data sets with the shapes of the lakde workloads.

The reference evaluates on the MAF tabular sets (GAS d=8, HEPMASS d=21,
MINIBOONE d=43, BSDS300 d=63; lakde/datasets/*.py) and 2-d toy data.  None of
those files ship with it, so these generators stand in for them with the same
dimensionality, size and character (full-covariance clusters, heavy tails,
near-singular embeddings, near-duplicate points).  Everything is drawn from
``numpy.random.default_rng(seed)`` and returned as float32 arrays.
"""

import math

import numpy as np


def _rotation(rng, d):
    """Haar-distributed orthogonal matrix (QR of a Gaussian with sign fix)."""
    q, r = np.linalg.qr(rng.standard_normal((d, d)))
    return q * np.sign(np.diag(r))[None, :]


def _full_cov_factor(rng, d, eig_lo, eig_hi):
    eig = np.exp(rng.uniform(math.log(eig_lo), math.log(eig_hi), size=d))
    return _rotation(rng, d) * np.sqrt(eig)[None, :]


def _sample_gmm(rng, n, means, factors, weights):
    comp = rng.choice(len(means), size=n, p=weights)
    d = means.shape[1]
    out = np.empty((n, d))
    for c in range(len(means)):
        idx = np.nonzero(comp == c)[0]
        out[idx] = means[c] + rng.standard_normal((len(idx), d)) @ factors[c].T
    return out


def circle_gmm(seed=0, n_train=2000, n_test=1000):
    """d=2: 8 isotropic Gaussians (sd 0.2) with means evenly spaced on a circle of radius 2."""
    rng = np.random.default_rng(seed)

    def draw(n):
        lab = rng.integers(0, 8, size=n)
        ang = 2 * np.pi * lab / 8
        mu = np.stack([2 * np.cos(ang), 2 * np.sin(ang)], axis=1)
        return (mu + 0.2 * rng.standard_normal((n, 2))).astype(np.float32)

    return draw(n_train), draw(n_test)


def heavy_tail_mixture(seed=0, n_train=200_000, n_test=20_000, d=8):
    """d=8: 9 full-covariance Gaussians (eigenvalues log-uniform in [1e-2, 1],
    Haar rotations, means N(0, 4I)) plus one Student-t (nu=3) component, each of
    weight 0.1; standardised with the training mean and standard deviation."""
    rng = np.random.default_rng(seed)
    means = 2.0 * rng.standard_normal((9, d))
    factors = [_full_cov_factor(rng, d, 1e-2, 1.0) for _ in range(9)]
    t_factor = _full_cov_factor(rng, d, 1e-2, 1.0)

    def draw(n):
        comp = rng.integers(0, 10, size=n)
        out = np.empty((n, d))
        for c in range(9):
            idx = np.nonzero(comp == c)[0]
            out[idx] = means[c] + rng.standard_normal((len(idx), d)) @ factors[c].T
        idx = np.nonzero(comp == 9)[0]
        z = rng.standard_normal((len(idx), d)) @ t_factor.T
        u = rng.chisquare(3, size=len(idx))
        out[idx] = z / np.sqrt(u / 3)[:, None]
        return out

    tr, te = draw(n_train), draw(n_test)
    mu, sd = tr.mean(0), tr.std(0)
    return ((tr - mu) / sd).astype(np.float32), ((te - mu) / sd).astype(np.float32)


def embedded_mixture(seed=0, n_train=30_000, n_test=3_000, d=43, d_latent=10, noise=1e-3):
    """d=43: a 6-component full-covariance GMM in 10 dims embedded linearly
    (orthonormal columns) in 43 dims plus isotropic noise of sd 1e-3, giving
    near-singular local covariances."""
    rng = np.random.default_rng(seed)
    means = 2.0 * rng.standard_normal((6, d_latent))
    factors = [_full_cov_factor(rng, d_latent, 1e-2, 1.0) for _ in range(6)]
    emb = _rotation(rng, d)[:, :d_latent]
    w = np.full(6, 1 / 6)

    def draw(n):
        z = _sample_gmm(rng, n, means, factors, w)
        return (z @ emb.T + noise * rng.standard_normal((n, d))).astype(np.float32)

    return draw(n_train), draw(n_test)


def lognormal_neighbourhood_sizes(n, seed=0, median=64, sigma=1.0, cap=4096, floor=2):
    """Per-point candidate counts, lognormal with the given median and sigma, capped."""
    rng = np.random.default_rng(seed + 7919)
    k = np.exp(math.log(median) + sigma * rng.standard_normal(n))
    return np.clip(np.round(k), floor, cap).astype(np.int64)


def wide_spectrum_mixture(seed=0, n_train=300_000, n_test=4_096, d=21, n_comp=12):
    """d=21: 12-component GMM with random full covariances, eigenvalues log-uniform in [1e-3, 1]."""
    rng = np.random.default_rng(seed)
    means = 2.0 * rng.standard_normal((n_comp, d))
    factors = [_full_cov_factor(rng, d, 1e-3, 1.0) for _ in range(n_comp)]
    w = np.full(n_comp, 1 / n_comp)
    tr = _sample_gmm(rng, n_train, means, factors, w)
    te = _sample_gmm(rng, n_test, means, factors, w)
    return tr.astype(np.float32), te.astype(np.float32)


def decaying_spectrum_mixture(seed=0, n_train=1_000_000, n_test=50_000, d=63, n_comp=20, n_dup=1000):
    """d=63: 20-component GMM whose covariance spectra decay as k^-1.5 with
    random rotations, plus one near-duplicate cluster of 1,000 points (sd 1e-4)."""
    rng = np.random.default_rng(seed)
    means = 2.0 * rng.standard_normal((n_comp, d))
    spec = np.arange(1, d + 1, dtype=np.float64) ** -1.5
    factors = [_rotation(rng, d) * np.sqrt(spec)[None, :] for _ in range(n_comp)]
    w = np.full(n_comp, 1 / n_comp)
    tr = _sample_gmm(rng, n_train - n_dup, means, factors, w)
    base = tr[rng.integers(0, len(tr))]
    dup = base + 1e-4 * rng.standard_normal((n_dup, d))
    tr = np.concatenate([tr, dup])[rng.permutation(n_train)]
    te = _sample_gmm(rng, n_test, means, factors, w)
    return tr.astype(np.float32), te.astype(np.float32)


WORKLOADS = {
    "circle2d": dict(make=circle_gmm, k=20, iterations=10, model="knn"),
    "gas8": dict(make=heavy_tail_mixture, k=50, iterations=20, model="knn"),
    "embed43": dict(make=embedded_mixture, k=None, iterations=10, model="hierarchical"),
    "spec21": dict(make=wide_spectrum_mixture, k=64, iterations=10, model="knn"),
    "bsds63": dict(make=decaying_spectrum_mixture, k=100, iterations=10, model="knn"),
}
