"""ctypes binding of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py`` as the checker / baseline. The
product (the CUDA library under ``manifolds-rs_b200/``) never imports it.

Each wrapper names the reference function it restates; the C source cites
file:line for each.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

OK, NO_DATA, NO_GRAPH_EDGES, DEGENERATE_LOCAL_RADII, BAD_ARG = 0, 1, 2, 3, 7
SAMPLER_HASH, SAMPLER_PHILOX = 0, 1

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
u8 = C.c_uint8


def build() -> str:
    """Compile liboracle.so with the committed Makefile (no-op when fresh)."""
    src = os.path.join(_HERE, "umap_oracle.c")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        L.orc_set_exp_mode.argtypes = [C.c_int]
        L.orc_set_exp_mode.restype = None
        L.orc_local_connectivity_distance.restype = C.c_float
        L.orc_local_connectivity_distance.argtypes = [f32p, C.c_uint32, C.c_float]
        L.orc_smooth_knn_dist.argtypes = [f32p, C.c_uint32, C.c_uint32, C.c_float, C.c_float,
                                          C.c_uint32, f32p, f32p]
        L.orc_knn_to_coo.restype = C.c_uint64
        L.orc_knn_to_coo.argtypes = [i32p, f32p, C.c_uint32, C.c_uint32, f32p, f32p, u32p, u32p, f32p]
        L.orc_symmetrise.restype = C.c_uint64
        L.orc_symmetrise.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, f32p, C.c_float, u32p, u32p, f32p]
        L.orc_filter_weak_edges.restype = C.c_uint64
        L.orc_filter_weak_edges.argtypes = [C.c_uint64, u32p, u32p, f32p, C.c_uint32, u32p, u32p, f32p]
        L.orc_csr_from_graph.restype = C.c_int
        L.orc_csr_from_graph.argtypes = [C.c_uint32, u64p, u32p, f32p, u32p, u32p, u32p, f32p, f32p,
                                         C.POINTER(C.c_uint64)]
        L.orc_fit_params_f32.argtypes = [C.c_float, C.c_float, C.c_uint32, C.POINTER(C.c_float),
                                         C.POINTER(C.c_float)]
        L.orc_fit_params_f64.argtypes = [C.c_double, C.c_double, C.c_uint32, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]
        L.orc_adam_epoch_scalars.argtypes = [C.c_float] * 4 + [C.c_uint32, C.c_uint32,
                                                               C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_hash_neg.restype = C.c_uint32
        L.orc_hash_neg.argtypes = [C.c_uint32] * 6
        L.orc_philox_neg.restype = C.c_uint32
        L.orc_philox_neg.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_dens_radii.argtypes = [f32p, C.c_uint32, C.c_uint32, u32p, u32p, C.c_float, C.c_float,
                                     f32p, f32p]
        L.orc_correlation_stats.argtypes = [f32p, f32p, C.c_uint64, C.c_float, C.POINTER(C.c_float),
                                            C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_dens_weights.restype = C.c_float
        L.orc_dens_weights.argtypes = [f32p, f32p, C.c_uint32, C.c_float, C.c_float, C.c_float, f32p]
        L.orc_grad_accum.argtypes = [f32p, C.c_uint32, C.c_uint32, u32p, u32p, u32p, f32p, C.c_uint32,
                                     C.c_uint64, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float,
                                     vp, vp, vp, vp, C.c_float, vp, f32p, vp]
        L.orc_set_grad_abs_sum.argtypes = [C.c_void_p]
        L.orc_set_grad_abs_sum.restype = None
        L.orc_adam_update.argtypes = [f32p, u32p, f32p, f32p, f32p, C.c_uint32, C.c_uint32, C.c_float,
                                      C.c_float, C.c_float, C.c_float]
        L.orc_schedule_update.argtypes = [f32p, f32p, C.c_uint64, C.c_uint32]
        L.orc_dens_is_active.restype = C.c_int
        L.orc_dens_is_active.argtypes = [C.c_float, C.c_float, C.c_uint32, C.c_uint32]
        L.orc_optimise_adam_gpu.restype = C.c_int
        L.orc_optimise_adam_gpu.argtypes = [f32p, C.c_uint32, C.c_uint32, u64p, u32p, f32p,
                                            C.c_float, C.c_float, C.c_float, C.c_float, C.c_uint32,
                                            C.c_uint32, C.c_float, C.c_float, C.c_float, vp, C.c_float,
                                            C.c_float, C.c_float, C.c_float, C.c_uint64, C.c_uint32,
                                            C.c_uint32]
        L.orc_edge_distances_from_knn.argtypes = [C.c_uint64, u32p, u32p, i32p, f32p, C.c_uint32, C.c_int, f32p]
        L.orc_original_log_radii.restype = C.c_int
        L.orc_original_log_radii.argtypes = [C.c_uint32, C.c_uint64, u32p, f32p, f32p, f32p, f32p]
        L.orc_dens_state_new.restype = C.c_int
        L.orc_dens_state_new.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, f32p, i32p, f32p, C.c_uint32,
                                         C.c_int, f32p, f32p, C.POINTER(C.c_float)]
        L.orc_optimise_adam_parallel.restype = C.c_int
        L.orc_optimise_adam_parallel.argtypes = [f32p, C.c_uint32, C.c_uint32, u64p, u32p, f32p,
                                                 C.c_float, C.c_float, C.c_float, C.c_float, C.c_uint32,
                                                 C.c_uint32, C.c_float, C.c_float, C.c_float, vp, C.c_float,
                                                 C.c_float, C.c_float, C.c_float, C.c_uint64, C.c_int,
                                                 C.c_uint32, C.c_uint32, C.POINTER(C.c_double)]
        L.orc_optimise_sequential.restype = C.c_int
        L.orc_optimise_sequential.argtypes = [C.c_int, f32p, C.c_uint32, C.c_uint32, u64p, u32p, f32p,
                                              C.c_float, C.c_float, C.c_float, C.c_float, C.c_uint32,
                                              C.c_uint32, C.c_float, C.c_float, C.c_float, vp, C.c_float,
                                              C.c_float, C.c_float, C.c_float, C.c_uint64]
        L.orc_active_edges_per_epoch.argtypes = [f32p, C.c_uint64, C.c_uint32, u64p]
        L.orc_knn_exact.restype = C.c_int
        L.orc_knn_exact.argtypes = [f32p, C.c_uint32, C.c_uint32, vp, C.c_uint32, C.c_uint32, C.c_int, u32p, f32p]
        L.orc_rank_counts.restype = C.c_int
        L.orc_rank_counts.argtypes = [f32p, C.c_uint32, C.c_uint32, vp, C.c_uint32, u32p, C.c_uint32, C.c_int,
                                      u32p]
        _lib = L
    return _lib


def _f32(x):
    return np.ascontiguousarray(x, dtype=np.float32)


def _u32(x):
    return np.ascontiguousarray(x, dtype=np.uint32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- graph

EXP_GLIBC, EXP_FROM_DOUBLE = 0, 1


def set_exp_mode(mode):
    """The graph stage's exp: EXP_GLIBC (glibc expf, the reference's; the
    default) or EXP_FROM_DOUBLE ((float)exp((double)x), the device's form),
    for attributing a difference to the last bit of expf."""
    lib().orc_set_exp_mode(int(mode))

def local_connectivity_distance(dists, local_connectivity):
    d = _f32(dists)
    return float(lib().orc_local_connectivity_distance(d, d.size, local_connectivity))


def smooth_knn_dist(knn_dist, local_connectivity=1.0, bandwidth=1e-5, n_iter=64):
    """graph.rs:499-565. knn_dist [n, k] -> (sigma[n], rho[n])."""
    d = _f32(knn_dist)
    n, k = d.shape
    sig = np.zeros(n, np.float32)
    rho = np.zeros(n, np.float32)
    lib().orc_smooth_knn_dist(d, n, k, local_connectivity, bandwidth, n_iter, sig, rho)
    return sig, rho


def knn_to_coo(knn_idx, knn_dist, sigma, rho):
    """graph.rs:585-662 -> (row, col, val)."""
    idx = np.ascontiguousarray(knn_idx, dtype=np.int32)
    d = _f32(knn_dist)
    n, k = idx.shape
    row = np.zeros(n * k, np.uint32)
    col = np.zeros(n * k, np.uint32)
    val = np.zeros(n * k, np.float32)
    m = lib().orc_knn_to_coo(idx, d, n, k, _f32(sigma), _f32(rho), row, col, val)
    return row[:m], col[:m], val[:m]


def symmetrise_graph(n, row, col, val, mix_weight=1.0):
    """graph.rs:684-694 (+ symmetrise_csr :387-468)."""
    row, col, val = _u32(row), _u32(col), _f32(val)
    cap = max(2 * row.size, 1)
    orow = np.zeros(cap, np.uint32)
    ocol = np.zeros(cap, np.uint32)
    oval = np.zeros(cap, np.float32)
    m = lib().orc_symmetrise(n, row.size, row, col, val, mix_weight, orow, ocol, oval)
    return orow[:m], ocol[:m], oval[:m]


def filter_weak_edges(row, col, val, n_epochs):
    """graph.rs:776-853."""
    row, col, val = _u32(row), _u32(col), _f32(val)
    orow = np.zeros(max(row.size, 1), np.uint32)
    ocol = np.zeros(max(row.size, 1), np.uint32)
    oval = np.zeros(max(row.size, 1), np.float32)
    m = lib().orc_filter_weak_edges(row.size, row, col, val, n_epochs, orow, ocol, oval)
    return orow[:m], ocol[:m], oval[:m]


def construct_umap_graph(knn_idx, knn_dist, n_epochs, local_connectivity=1.0, bandwidth=1e-5,
                         mix_weight=1.0):
    """lib.rs:296-306 stage chain: sigma/rho -> COO -> symmetrise -> filter."""
    n = knn_dist.shape[0]
    sig, rho = smooth_knn_dist(knn_dist, local_connectivity, bandwidth, 64)
    r, c, v = knn_to_coo(knn_idx, knn_dist, sig, rho)
    r, c, v = symmetrise_graph(n, r, c, v, mix_weight)
    r, c, v = filter_weak_edges(r, c, v, n_epochs)
    return (r, c, v), sig, rho


def coo_to_adj_ptr(n, row):
    """Row pointer of a row-grouped COO (graph.rs:709-758 fast path)."""
    cnt = np.bincount(np.asarray(row, dtype=np.int64), minlength=n)
    ptr = np.zeros(n + 1, np.uint64)
    np.cumsum(cnt, out=ptr[1:])
    return ptr


def csr_from_graph(n, adj_ptr, adj_col, adj_w):
    """umap_optimiser_gpu.rs:132-209 UmapCsrGraph::from_graph."""
    adj_ptr = np.ascontiguousarray(adj_ptr, dtype=np.uint64)
    adj_col, adj_w = _u32(adj_col), _f32(adj_w)
    cap = int(adj_ptr[-1]) if n else 0
    offsets = np.zeros(n + 1, np.uint32)
    edge_idx = np.zeros(2 * cap + 2, np.uint32)
    other = np.zeros(2 * cap + 2, np.uint32)
    eps = np.zeros(cap + 1, np.float32)
    mu = np.zeros(cap + 1, np.float32)
    ne = C.c_uint64(0)
    st = lib().orc_csr_from_graph(n, adj_ptr if n else np.zeros(1, np.uint64), adj_col, adj_w,
                                  offsets, edge_idx, other, eps, mu, C.byref(ne))
    if st != OK:
        return st, None
    e = ne.value
    return OK, dict(n=n, n_edges=e, offsets=offsets, edge_idx=edge_idx[:2 * e].copy(),
                    other=other[:2 * e].copy(), eps=eps[:e].copy(), mu=mu[:e].copy())


# ---------------------------------------------------------------- params

def fit_params(min_dist, spread, n_iter=300, dtype=np.float32):
    """umap_optimisers.rs:139-209."""
    if dtype == np.float64:
        a, b = C.c_double(), C.c_double()
        lib().orc_fit_params_f64(min_dist, spread, n_iter, C.byref(a), C.byref(b))
    else:
        a, b = C.c_float(), C.c_float()
        lib().orc_fit_params_f32(min_dist, spread, n_iter, C.byref(a), C.byref(b))
    return a.value, b.value


def adam_epoch_scalars(lr, beta1, beta2, eps, epoch, n_epochs):
    """umap_optimiser_gpu.rs:1168-1175 -> (lr_alpha*ad_scale, epsc) in f32."""
    f, e = C.c_float(), C.c_float()
    lib().orc_adam_epoch_scalars(lr, beta1, beta2, eps, epoch, n_epochs, C.byref(f), C.byref(e))
    return np.float32(f.value), np.float32(e.value)


# ---------------------------------------------------------------- kernels

def hash_neg(seed, node, epoch, edge_local, neg, n):
    return int(lib().orc_hash_neg(seed & 0xFFFFFFFF, node, epoch, edge_local, neg, n))


def philox_neg(seed, entry, epoch, neg, n):
    return int(lib().orc_philox_neg(seed, entry, epoch, neg, n))


def dens_radii(embd, csr, a, b):
    """umap_optimiser_gpu.rs:1409-1453."""
    e = _f32(embd)
    n, d = e.shape
    re = np.zeros(n, np.float32)
    phi = np.zeros(n, np.float32)
    lib().orc_dens_radii(e, n, d, csr["offsets"], _u32(csr["other"]), a, b, re, phi)
    return re, phi


def correlation_stats(re, r, var_shift):
    """density.rs:464-508 (T = f32)."""
    m, s, c = C.c_float(), C.c_float(), C.c_float()
    re, r = _f32(re), _f32(r)
    lib().orc_correlation_stats(re, r, re.size, var_shift, C.byref(m), C.byref(s), C.byref(c))
    return np.float32(m.value), np.float32(s.value), np.float32(c.value)


def dens_weights(r, re, var_shift, lam, mu_tot):
    r, re = _f32(r), _f32(re)
    w = np.zeros(r.size, np.float32)
    coeff = lib().orc_dens_weights(r, re, r.size, var_shift, lam, mu_tot, w)
    return w, np.float32(coeff)


def grad_accum(embd, csr, cursor, epoch, seed, neg_rate, a, b, gamma, sampler=SAMPLER_HASH,
               dens=None, injected=None, abs_sum=None):
    """umap_optimiser_gpu.rs:1461-1579 (+ has_update of :737-742, :859).

    dens: None or dict(re, phi_sum, weight, coeff). injected: None or
    uint32 [2E, neg_rate] of negative nodes per CSR entry. abs_sum: None or a
    float64 [n, n_dim] array that receives the sum of |term| per node and
    coordinate (the scale of the f32 sum's own rounding)."""
    e = _f32(embd)
    n, d = e.shape
    grad = np.zeros((n, d), np.float32)
    hu = np.zeros(n, np.uint32)
    cur = _f32(cursor)
    if dens is not None:
        re, phi, wt = _f32(dens["re"]), _f32(dens["phi_sum"]), _f32(dens["weight"])
        mu = _f32(csr["mu"])
        coeff = float(dens["coeff"])
    else:
        re = phi = wt = mu = None
        coeff = 0.0
    inj = None if injected is None else np.ascontiguousarray(injected, dtype=np.uint32)
    if abs_sum is not None:
        assert abs_sum.dtype == np.float64 and abs_sum.shape == (n, d) and abs_sum.flags.c_contiguous
    lib().orc_set_grad_abs_sum(_ptr(abs_sum))
    try:
        lib().orc_grad_accum(e, n, d, csr["offsets"], _u32(csr["edge_idx"]), _u32(csr["other"]), cur,
                             epoch, seed, sampler, neg_rate, a, b, gamma, _ptr(mu), _ptr(re), _ptr(phi),
                             _ptr(wt), coeff, _ptr(inj), grad, hu.ctypes.data_as(C.c_void_p))
    finally:
        lib().orc_set_grad_abs_sum(None)
    return grad, hu


def adam_update(grad, has_update, m, v, embd, fused, epsc, beta1, beta2):
    """umap_optimiser_gpu.rs:1584-1627 (in place on m, v, embd)."""
    n, d = embd.shape
    lib().orc_adam_update(_f32(grad), _u32(has_update), m, v, embd, n, d, fused, epsc, beta1, beta2)


def schedule_update(eps, cursor, epoch):
    """umap_optimiser_gpu.rs:940-955 (in place on cursor)."""
    lib().orc_schedule_update(_f32(eps), cursor, cursor.size, epoch)


def dens_is_active(lam, frac, epoch, n_epochs):
    return bool(lib().orc_dens_is_active(lam, frac, epoch, n_epochs))


def _dens_args(dens):
    if dens is None:
        return None, 0.0, 0.0, 0.0, 0.0, None
    r = _f32(dens["r"])
    return _ptr(r), dens["lambda"], dens["frac"], dens["var_shift"], dens["mu_tot"], r


def optimise_adam_gpu(embd, n, adj_ptr, adj_col, adj_w, p, seed, dens=None, sampler=SAMPLER_HASH,
                      epochs_to_run=0):
    """umap_optimiser_gpu.rs:1302-1369 restated over the CPU mirrors."""
    e = np.array(embd, dtype=np.float32, order="C")
    rp, lam, frac, vs, mt, keep = _dens_args(dens)
    st = lib().orc_optimise_adam_gpu(e, n, e.shape[1], np.ascontiguousarray(adj_ptr, np.uint64),
                                     _u32(adj_col), _f32(adj_w), p["a"], p["b"], p["lr"], p["gamma"],
                                     p["n_epochs"], p["neg_sample_rate"], p["beta1"], p["beta2"],
                                     p["eps"], rp, lam, frac, vs, mt, seed, sampler, epochs_to_run)
    return st, e


def optimise_adam_parallel(embd, n, adj_ptr, adj_col, adj_w, p, seed, dens=None, n_threads=0,
                           epochs_to_run=0, first_epoch=0, return_seconds=False):
    """umap_optimisers.rs:1170-1492 (the timed CPU baseline). Runs epochs
    [first_epoch, first_epoch + epochs_to_run) after fast-forwarding the
    schedule; return_seconds adds the epoch loop's wall time."""
    e = np.array(embd, dtype=np.float32, order="C")
    rp, lam, frac, vs, mt, keep = _dens_args(dens)
    secs = C.c_double(0.0)
    st = lib().orc_optimise_adam_parallel(e, n, e.shape[1], np.ascontiguousarray(adj_ptr, np.uint64),
                                          _u32(adj_col), _f32(adj_w), p["a"], p["b"], p["lr"],
                                          p["gamma"], p["n_epochs"], p["neg_sample_rate"], p["beta1"],
                                          p["beta2"], p["eps"], rp, lam, frac, vs, mt, seed, n_threads,
                                          first_epoch, epochs_to_run, C.byref(secs))
    return (st, e, secs.value) if return_seconds else (st, e)


def optimise_sequential(algo, embd, n, adj_ptr, adj_col, adj_w, p, seed, dens=None):
    """umap_optimisers.rs:653-865 (algo 'sgd') and :907-1142 (algo 'adam')."""
    e = np.array(embd, dtype=np.float32, order="C")
    rp, lam, frac, vs, mt, keep = _dens_args(dens)
    st = lib().orc_optimise_sequential(0 if algo == "sgd" else 1, e, n, e.shape[1],
                                       np.ascontiguousarray(adj_ptr, np.uint64), _u32(adj_col),
                                       _f32(adj_w), p["a"], p["b"], p["lr"], p["gamma"], p["n_epochs"],
                                       p["neg_sample_rate"], p["beta1"], p["beta2"], p["eps"], rp, lam,
                                       frac, vs, mt, seed)
    return st, e


def edge_distances_from_knn(row, col, knn_idx, knn_dist, distances_squared=True):
    row, col = _u32(row), _u32(col)
    idx = np.ascontiguousarray(knn_idx, dtype=np.int32)
    out = np.zeros(row.size, np.float32)
    lib().orc_edge_distances_from_knn(row.size, row, col, idx, _f32(knn_dist), idx.shape[1],
                                      int(distances_squared), out)
    return out


def original_log_radii(n, row, val, edge_d_sq):
    r = np.zeros(n, np.float32)
    ms = np.zeros(n, np.float32)
    row, val, ed = _u32(row), _f32(val), _f32(edge_d_sq)
    st = lib().orc_original_log_radii(n, row.size, row, val, ed, r, ms)
    return st, r, ms


def dens_state_new(n, row, col, val, knn_idx, knn_dist, distances_squared=True, lam=2.0, frac=0.3,
                   var_shift=0.1):
    """density.rs:181-201 -> dict(r, mu_sum, mu_tot, lambda, frac, var_shift)."""
    row, col, val = _u32(row), _u32(col), _f32(val)
    idx = np.ascontiguousarray(knn_idx, dtype=np.int32)
    r = np.zeros(n, np.float32)
    ms = np.zeros(n, np.float32)
    mt = C.c_float()
    st = lib().orc_dens_state_new(n, row.size, row, col, val, idx, _f32(knn_dist), idx.shape[1],
                                  int(distances_squared), r, ms, C.byref(mt))
    if st != OK:
        return st, None
    return OK, dict(r=r, mu_sum=ms, mu_tot=np.float32(mt.value), **{"lambda": lam}, frac=frac,
                    var_shift=var_shift)


def active_edges_per_epoch(eps, n_epochs):
    """Per-epoch count of edges with cursor <= epoch (the edge-update unit)."""
    e = _f32(eps)
    out = np.zeros(n_epochs, np.uint64)
    lib().orc_active_edges_per_epoch(e, e.size, n_epochs, out)
    return out


# ------------------------------------------------------- kNN and metrics

def knn_exact(X, k, queries=None, metric=0):
    """Exact kNN restatement (ann-search-rs exhaustive search as called by
    nearest_neighbours.rs:313-361): self excluded, sequential-FMA f32
    distances, ties by index. -> (idx u32 [nq, k], dist f32 [nq, k])."""
    X = _f32(X)
    n, dim = X.shape
    q = None if queries is None else np.ascontiguousarray(queries, np.uint32)
    nq = n if q is None else q.size
    idx = np.empty((nq, k), np.uint32)
    dist = np.empty((nq, k), np.float32)
    st = lib().orc_knn_exact(X, n, dim, None if q is None else q.ctypes.data, nq, k, metric, idx, dist)
    if st != OK:
        raise ValueError(f"orc_knn_exact: status {st}")
    return idx, dist


def rank_counts(X, nbr, queries=None, metric=0):
    """0-based rank of each given neighbour in its query's (distance, index)
    order over all other points."""
    X = _f32(X)
    n, dim = X.shape
    nbr = np.ascontiguousarray(nbr, np.uint32)
    q = None if queries is None else np.ascontiguousarray(queries, np.uint32)
    nq, k = nbr.shape
    out = np.empty((nq, k), np.uint32)
    lib().orc_rank_counts(X, n, dim, None if q is None else q.ctypes.data, nq, nbr, k, metric, out)
    return out


def trustworthiness(X, Y, k=15, queries=None, metric=0):
    """sklearn.manifold.trustworthiness's definition, restated on the exact
    kNN above (over a query subset: the same sum over those queries, the
    normalisation with their count)."""
    n = X.shape[0]
    ynbr, _ = knn_exact(Y, k, queries)
    c = rank_counts(X, ynbr, queries, metric).astype(np.float64)
    nq = ynbr.shape[0]
    pen = np.maximum(0.0, c + 1.0 - k).sum()
    return 1.0 - pen * (2.0 / (nq * k * (2.0 * n - 3.0 * k - 1.0)))


def knn_preservation(knn_idx, Y, k=15, queries=None):
    ynbr, _ = knn_exact(Y, k, queries)
    rows = np.arange(Y.shape[0]) if queries is None else np.asarray(queries)
    kx = np.asarray(knn_idx)[rows, :k]
    return float(np.mean([len(set(a.tolist()) & set(b.tolist())) / k for a, b in zip(kx, ynbr)]))


# ------------------------------------------------------- spectral init

def splitmix_start(n, seed):
    """The library's Lanczos start vector: uniform in [-0.5, 0.5) from the
    counter-based SplitMix64 stream (the reference draws it from StdRng)."""
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15) * i
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z ^= z >> np.uint64(31)
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) - 0.5


def lanczos_smallest(M, k, start):
    """lanczos_eigendecomp + select_eigenpairs (src/utils/math.rs:401-616),
    restated with numpy: min(4 k + 30, n) steps from `start`, modified
    Gram-Schmidt against the whole basis, stop when beta < 1e-12; Ritz
    values ascending and unit Ritz vectors [n, k]. M: dense or scipy."""
    n = M.shape[0]
    n_iter = min(4 * k + 30, n)
    v = start / np.linalg.norm(start)
    basis, alpha, beta = [], [], []
    v_old = np.zeros(n)
    for j in range(n_iter):
        basis.append(v.copy())
        w = M @ v
        a = float(w @ v)
        alpha.append(a)
        w = w - a * v - (beta[j - 1] * v_old if j else 0.0)
        for b in basis:
            w = w - float(w @ b) * b
        bt = float(np.linalg.norm(w))
        beta.append(bt)
        if bt < 1e-12:
            break
        v_old, v = v, w / bt
    m = len(alpha)
    T = np.diag(alpha) + np.diag(beta[:m - 1], 1) + np.diag(beta[:m - 1], -1)
    tw, tv = np.linalg.eigh(T)
    sel = np.argsort(tw, kind="stable")[:min(k, m)]
    V = np.array(basis).T @ tv[:, sel]
    V /= np.linalg.norm(V, axis=0, keepdims=True)
    return tw[sel], V
