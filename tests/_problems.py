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


# The benchmark workloads' inputs (the shapes BASELINE's configurations name):
# name -> (n, dim, clusters, k, n_epochs, generator), data seed 2024.
CONFIGS = {
    "c1": (10_000, 50, 10, 15, 500, "isotropic"),
    "c2": (1_000_000, 50, 30, 15, 200, "anisotropic"),
    "c3": (200_000, 30, 20, 30, 200, "variable"),
}


@functools.lru_cache(maxsize=3)
def config_inputs(name, seed=2024):
    """(X, knn_idx, knn_dist) of a benchmark workload. The exact kNN comes
    from the library's GPU brute force (bit-exact with the oracle's, see
    test_gpu_knn.py) and is kept in a kNN cache file under the temp
    directory (UMAPCU_TEST_KNN_CACHE overrides), written and read with the
    NumPy cache reader."""
    import os
    import tempfile

    import umapcu
    import umapdata.synth as S
    from umapdata import knn_cache
    n, dim, clusters, k, _, kind = CONFIGS[name]
    gen = {"isotropic": S.isotropic_mixture, "anisotropic": S.anisotropic_mixture,
           "variable": S.variable_density_mixture}[kind]
    X, _ = gen(n, dim, clusters, seed)
    d = os.environ.get("UMAPCU_TEST_KNN_CACHE") or os.path.join(tempfile.gettempdir(), "umapcu_test_knn")
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, f"{name}_s{seed}_exact.knn")
    if os.path.exists(path):
        try:
            idx, dist, _ = knn_cache.load(path)
            if idx.shape == (n, k):
                return X, idx, dist
        except ValueError:
            pass
    idx, dist = umapcu.knn_exact(X, k)
    tmp = f"{path}.{os.getpid()}.tmp"
    knn_cache.save(tmp, idx, dist)
    os.replace(tmp, path)
    return X, idx, dist


@functools.lru_cache(maxsize=3)
def config_oracle_graph(name, seed=2024):
    """The oracle's fuzzy graph of a benchmark workload, with its sigma/rho
    and adjacency row pointers."""
    X, idx, dist = config_inputs(name, seed)
    n, _, _, _, n_epochs, _ = CONFIGS[name]
    (r, c, v), sig, rho = O.construct_umap_graph(idx, dist, n_epochs)
    return dict(X=X, idx=idx, dist=dist, row=r, col=c, val=v, sigma=sig, rho=rho, ptr=O.coo_to_adj_ptr(n, r),
                n=n, n_epochs=n_epochs)
