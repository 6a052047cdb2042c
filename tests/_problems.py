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


# Unit roundoff of f32 (2^-24): the scale of one rounding of an f32 sum,
# relative to the magnitude of its terms.
F32_U = 2.0 ** -24


def adam_step64(g, m0, v0, fused, epsc, beta1, beta2):
    """The Adam step of umap_adam_update (umap_optimiser_gpu.rs:912-922) in
    f64 from the epoch's starting moments, and its derivative by g."""
    g = np.asarray(g, np.float64)
    m0 = np.asarray(m0, np.float64)
    v0 = np.asarray(v0, np.float64)
    m = m0 + (1.0 - beta1) * (g - m0)
    v = v0 + (1.0 - beta2) * (g * g - v0)
    sv = np.sqrt(v)
    den = sv + np.float64(epsc)
    step = np.float64(fused) * m / den
    dv = 2.0 * (1.0 - beta2) * g
    dsv = np.where(sv > 0, dv / (2.0 * np.maximum(sv, 1e-300)), 0.0)
    dstep = np.float64(fused) * ((1.0 - beta1) / den - m * dsv / (den * den))
    return step, dstep


def update_errors(go, gg, abs_sum, m0, v0, fused, epsc, beta1, beta2, active, floor=0.1, units=64.0):
    """Per-element comparison of the Adam steps two gradients imply (the
    reference's go, the device's gg), over the active nodes' elements.
    -> dict with
      rel      : |s_dev - s_ref| / |s_ref| per element;
      bound_ok : every element within 1e-5 |s_ref| + units * u * S * |ds/dg|,
                 S = the sum of |terms| of the element's gradient (the scale
                 of the reference's own f32 rounding of that sum, u = 2^-24):
                 1e-5 relative, up to what cancellation in the gradient sum
                 leaves undetermined;
      floor_max: the largest rel among elements whose step is at least
                 `floor` of the largest and whose gradient sum does not
                 cancel (S <= 30 |g|)."""
    act = np.asarray(active, bool)
    s_ref, ds = adam_step64(go, m0, v0, fused, epsc, beta1, beta2)
    s_dev, _ = adam_step64(gg, m0, v0, fused, epsc, beta1, beta2)
    s_ref, ds, s_dev, S, g = s_ref[act], ds[act], s_dev[act], np.asarray(abs_sum)[act], np.asarray(go, np.float64)[act]
    err = np.abs(s_dev - s_ref)
    rel = err / np.maximum(np.abs(s_ref), 1e-300)
    bound = 1e-5 * np.abs(s_ref) + units * F32_U * S * np.abs(ds)
    sel = (np.abs(s_ref) >= floor * np.abs(s_ref).max()) & (S <= 30.0 * np.abs(g))
    return dict(rel=rel.ravel(), bound_ok=bool((err <= bound).all()), worst_over_bound=float((err / bound).max()),
                floor_max=float(rel[sel].max()) if sel.any() else 0.0, floor_count=int(sel.sum()),
                count=int(rel.size))
