"""Seeded synthetic inputs for tests and benchmarks.

The reference benchmarks and tests run on synthetic data only
(tests/commons/mod.rs, tests/umap_gpu_bench.rs); these generators produce
Gaussian mixtures of the shapes the benchmark workloads name, and the exact
kNN graph the hot path starts from (self excluded, squared Euclidean
distances ascending -- the form the reference's ANN backends return,
src/lib.rs:434-436).
"""
from __future__ import annotations

import numpy as np


def isotropic_mixture(n, dim, n_clusters, seed, mean_sd=5.0, sd=1.0):
    """n x dim f32 from n_clusters isotropic Gaussians, means ~ N(0, mean_sd^2 I),
    within-cluster sd, equal weights. Returns (X, labels)."""
    rng = np.random.default_rng(seed)
    means = rng.normal(0.0, mean_sd, (n_clusters, dim))
    lab = rng.integers(0, n_clusters, n)
    X = means[lab] + rng.normal(0.0, sd, (n, dim))
    return X.astype(np.float32), lab.astype(np.int32)


def anisotropic_mixture(n, dim, n_clusters, seed, mean_sd=5.0, eig_lo=0.1, eig_hi=4.0):
    """Mixture with random anisotropic covariances (eigenvalues log-uniform in
    [eig_lo, eig_hi], random orthogonal basis) and Dirichlet(1) weights."""
    rng = np.random.default_rng(seed)
    means = rng.normal(0.0, mean_sd, (n_clusters, dim))
    w = rng.dirichlet(np.ones(n_clusters))
    lab = rng.choice(n_clusters, size=n, p=w)
    X = np.empty((n, dim), np.float32)
    for c in range(n_clusters):
        idx = np.nonzero(lab == c)[0]
        if idx.size == 0:
            continue
        q, _ = np.linalg.qr(rng.normal(size=(dim, dim)))
        ev = np.exp(rng.uniform(np.log(eig_lo), np.log(eig_hi), dim))
        A = q * np.sqrt(ev)
        z = rng.normal(size=(idx.size, dim))
        X[idx] = (means[c] + z @ A.T).astype(np.float32)
    return X, lab.astype(np.int32)


def variable_density_mixture(n, dim, n_clusters, seed, sd_lo=0.2, sd_hi=3.0, mean_sd=8.0):
    """Isotropic clusters whose within-cluster sd is log-uniform in
    [sd_lo, sd_hi], so local radii differ (densMAP workload)."""
    rng = np.random.default_rng(seed)
    means = rng.normal(0.0, mean_sd, (n_clusters, dim))
    sds = np.exp(rng.uniform(np.log(sd_lo), np.log(sd_hi), n_clusters))
    lab = rng.integers(0, n_clusters, n)
    X = means[lab] + rng.normal(size=(n, dim)) * sds[lab, None]
    return X.astype(np.float32), lab.astype(np.int32)


def subspace_mixture(n, dim, n_clusters, seed, sub_dim=3, mean_sd=6.0, sd=1.0, noise=0.05):
    """Clusters that live in random sub_dim-dimensional subspaces of the dim-D
    space (plus small isotropic noise): data with low intrinsic dimension,
    whose neighbourhoods a 2-D layout can preserve."""
    rng = np.random.default_rng(seed)
    means = rng.normal(0.0, mean_sd, (n_clusters, dim))
    lab = rng.integers(0, n_clusters, n)
    X = means[lab] + rng.normal(0.0, noise, (n, dim))
    for c in range(n_clusters):
        idx = np.nonzero(lab == c)[0]
        q, _ = np.linalg.qr(rng.normal(size=(dim, sub_dim)))
        X[idx] += rng.normal(0.0, sd, (idx.size, sub_dim)) @ q.T
    return X.astype(np.float32), lab.astype(np.int32)


def random_layout(n_samples, n_comp, seed, init_range=10.0):
    """U(-range, range) initial embedding from numpy's PCG64 stream seeded
    with `seed` (the values umapcu.random_layout returns)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-init_range, init_range, (n_samples, n_comp)).astype(np.float32)


def _finish(i_idx, d2, k):
    """Drop self (or the farthest if self is absent), sort ascending."""
    n = i_idx.shape[0]
    rows = np.arange(n)[:, None]
    is_self = i_idx == rows
    drop = np.where(is_self.any(1), is_self.argmax(1), k)
    keep = np.ones_like(i_idx, dtype=bool)
    keep[np.arange(n), drop] = False
    idx = i_idx[keep].reshape(n, k)
    dd = d2[keep].reshape(n, k)
    o = np.argsort(dd, axis=1, kind="stable")
    return np.take_along_axis(idx, o, 1).astype(np.int32), np.take_along_axis(dd, o, 1).astype(np.float32)


def exact_knn_cpu(X, k, chunk=2048):
    """Exact kNN (self excluded), squared Euclidean in f64 cast to f32."""
    X64 = np.asarray(X, np.float64)
    n = X64.shape[0]
    sq = (X64 * X64).sum(1)
    out_i = np.empty((n, k + 1), np.int64)
    for s in range(0, n, chunk):
        q = X64[s:s + chunk]
        d = sq[s:s + chunk, None] + sq[None, :] - 2.0 * q @ X64.T
        part = np.argpartition(d, k, axis=1)[:, :k + 1]
        out_i[s:s + chunk] = part
    d2 = ((X64[:, None, :] - X64[out_i]) ** 2).sum(-1)
    return _finish(out_i, d2, k)


def exact_knn_torch(X, k, device="cuda", chunk=2048):
    """Exact kNN on the GPU with torch (input preparation only): candidate
    k+1 neighbours from an fp32 distance matrix per query chunk, distances
    of the candidates recomputed exactly in f64."""
    import torch
    Xt = torch.as_tensor(np.asarray(X, np.float32), device=device)
    n = Xt.shape[0]
    sq = (Xt * Xt).sum(1)
    cand = torch.empty((n, k + 1), dtype=torch.int64, device=device)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for s in range(0, n, chunk):
            q = Xt[s:s + chunk]
            d = sq[s:s + chunk, None] + sq[None, :] - 2.0 * (q @ Xt.T)
            cand[s:s + chunk] = torch.topk(d, k + 1, dim=1, largest=False).indices
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    X64 = Xt.double()
    d2 = torch.empty((n, k + 1), dtype=torch.float64, device=device)
    for s in range(0, n, chunk):
        c = cand[s:s + chunk]
        d2[s:s + chunk] = ((X64[s:s + chunk, None, :] - X64[c]) ** 2).sum(-1)
    out = _finish(cand.cpu().numpy(), d2.cpu().numpy(), k)
    del Xt, X64, sq, cand, d2
    torch.cuda.empty_cache()
    return out


def exact_knn(X, k):
    try:
        import torch
        if torch.cuda.is_available() and X.shape[0] > 20000:
            return exact_knn_torch(X, k)
    except ImportError:
        pass
    return exact_knn_cpu(X, k)
