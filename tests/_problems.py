"""Shared seeded test problems: data -> exact kNN -> oracle graph."""
import functools

import numpy as np

from oracle import oracle as O


@functools.lru_cache(maxsize=8)
def knn_problem(n=3000, dim=50, k=15, clusters=10, seed=0, kind="isotropic"):
    import umapdata.synth as S
    if kind == "subspace":
        X, lab = S.subspace_mixture(n, dim, clusters, seed)
    else:
        X, lab = S.isotropic_mixture(n, dim, clusters, seed)
    idx, dist = S.exact_knn_cpu(X, k)
    return X, lab, idx, dist


@functools.lru_cache(maxsize=8)
def oracle_graph(n=3000, dim=50, k=15, clusters=10, seed=0, n_epochs=200, kind="isotropic"):
    X, lab, idx, dist = knn_problem(n, dim, k, clusters, seed, kind)
    (r, c, v), sig, rho = O.construct_umap_graph(idx, dist, n_epochs)
    ptr = O.coo_to_adj_ptr(n, r)
    return dict(X=X, lab=lab, idx=idx, dist=dist, row=r, col=c, val=v, ptr=ptr, sigma=sig, rho=rho)


def init_embedding(n, d=2, seed=7):
    return np.random.default_rng(seed).uniform(-10, 10, (n, d)).astype(np.float32)


def knn_preservation(X_idx, Y, k=15):
    """mean |kNN_X(i) & kNN_Y(i)| / k over all points (exact, small n)."""
    import umapdata.synth as S
    yi, _ = S.exact_knn_cpu(Y, k)
    return float(np.mean([len(set(a[:k]) & set(b)) / k for a, b in zip(X_idx, yi)]))


def fuzzy_cross_entropy(row, col, w, Y, a, b):
    """sum over graph entries of w log(w/q) + (1-w) log((1-w)/(1-q)),
    q = 1 / (1 + a d^2b) clamped to [1e-12, 1 - 1e-12]."""
    d2 = ((Y[row].astype(np.float64) - Y[col]) ** 2).sum(1)
    q = np.clip(1.0 / (1.0 + a * d2 ** b), 1e-12, 1 - 1e-12)
    w = np.clip(w.astype(np.float64), 1e-12, 1 - 1e-12)
    return float(np.sum(w * np.log(w / q) + (1 - w) * np.log((1 - w) / (1 - q))))


def oracle_adam_gpu_run(args):
    """One oracle run of the reference's GPU optimiser (process-pool worker):
    (init, ptr, col, val, params dict, seed, sampler) -> final embedding."""
    init, ptr, col, val, pd, seed, sampler = args
    st, yo = O.optimise_adam_gpu(init, init.shape[0], ptr, col, val, pd, seed, sampler=sampler)
    if st != O.OK:
        raise RuntimeError(f"oracle status {st}")
    return yo
