"""Pins the CPU oracle to the known-answer tests the reference itself holds.

Each test restates one reference test (cited file:line, paths relative to
the manifolds-rs crate root) and runs it against the oracle. The reference's
Rust code cannot be built here, so these known answers are the oracle's pin.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O


# ------------------------------------------------------------ graph.rs


def test_smooth_knn_dist_basic():
    # graph.rs:1442-1460
    dist = np.array([[1.0, 2.0], [1.5, 3.0], [0.5, 1.5]], np.float32)
    sig, rho = O.smooth_knn_dist(dist, 1.0, 1e-5, 64)
    assert rho == pytest.approx([1.0, 1.5, 0.5], abs=1e-4)
    assert (sig > 0).all()


def test_smooth_knn_dist_zero_local_connectivity():
    # graph.rs:1463-1471
    dist = np.array([[0.0, 1.0, 2.0], [0.0, 1.0, 2.0]], np.float32)
    sig, rho = O.smooth_knn_dist(dist, 0.0, 1e-5, 64)
    assert (rho == 0).all() and sig.size == 2


def test_local_connectivity_interpolates():
    # graph.rs:107-125: fractional local_connectivity interpolates linearly
    d = [1.0, 3.0, 5.0]
    assert O.local_connectivity_distance(d, 1.0) == 1.0
    assert O.local_connectivity_distance(d, 1.5) == pytest.approx(2.0)
    assert O.local_connectivity_distance(d, 7.0) == 5.0
    assert O.local_connectivity_distance(d, -1.0) == 0.0


def test_sigma_hits_log_k_target():
    # graph.rs:536-557: the bisection stops once sum exp(-adj/sigma) ~ ln(k)
    rng = np.random.default_rng(0)
    d = np.sort(rng.uniform(0.1, 4.0, (64, 15)).astype(np.float32), axis=1)
    sig, rho = O.smooth_knn_dist(d)
    adj = np.maximum(d - rho[:, None], 0)
    val = np.exp(-adj / sig[:, None]).sum(1)
    assert np.abs(val - math.log(15)).max() < 1e-4


def test_knn_to_coo_basic():
    # graph.rs:1474-1491
    idx = np.array([[1, 2], [0, 2], [0, 1]], np.int32)
    d = np.array([[1.0, 2.0], [1.0, 1.5], [2.0, 1.5]], np.float32)
    r, c, v = O.knn_to_coo(idx, d, np.ones(3, np.float32), np.zeros(3, np.float32))
    assert r.size == 6 and c.size == 6 and v.size == 6
    assert ((v >= 0) & (v <= 1)).all()


def test_knn_to_coo_self_loop_excluded():
    # graph.rs:1494-1510
    idx = np.array([[0, 1], [1, 0]], np.int32)
    d = np.array([[0.0, 1.0], [0.0, 1.0]], np.float32)
    r, c, v = O.knn_to_coo(idx, d, np.ones(2, np.float32), np.zeros(2, np.float32))
    assert v.size == 2 and (r != c).all()


def test_knn_to_coo_degenerate_sigma():
    # graph.rs:640-647: sigma <= 0 gives 1 at rho and 0 beyond
    idx = np.array([[1, 2]], np.int32)
    d = np.array([[1.0, 2.0]], np.float32)
    r, c, v = O.knn_to_coo(idx, d, np.zeros(1, np.float32), np.ones(1, np.float32))
    assert list(v) == [1.0, 0.0]


def test_symmetrise_graph_full_union():
    # graph.rs:1513-1539 (mix 0.5)
    r, c, v = O.symmetrise_graph(2, [0, 1], [1, 0], [0.8, 0.6], 0.5)
    e = {(int(a), int(b)): float(w) for a, b, w in zip(r, c, v)}
    assert len(e) == 2
    assert e[(0, 1)] == pytest.approx(0.86, abs=1e-6)
    assert e[(1, 0)] == pytest.approx(0.76, abs=1e-6)


def test_symmetrise_graph_directed():
    # graph.rs:1542-1563 (mix 1.0)
    r, c, v = O.symmetrise_graph(2, [0, 1], [1, 0], [0.8, 0.6], 1.0)
    assert v.size == 2
    assert np.allclose(v, 0.8 + 0.6 - 0.8 * 0.6, atol=1e-6)


def test_symmetrise_adds_missing_direction_sorted():
    # graph.rs:373-375: output grouped by row, columns ascending; a missing
    # direction contributes zero (graph.rs:303-305)
    r, c, v = O.symmetrise_graph(3, [0, 0, 2], [2, 1, 0], [0.5, 0.25, 0.5], 1.0)
    assert list(zip(r.tolist(), c.tolist())) == [(0, 1), (0, 2), (1, 0), (2, 0)]
    assert v.tolist() == pytest.approx([0.25, 0.75, 0.25, 0.75])


def test_filter_weak_edges_threshold():
    # graph.rs:786-809: keep w >= max/n_epochs, order preserved
    r, c, v = O.filter_weak_edges([0, 0, 1, 1], [1, 2, 0, 2], [1.0, 0.004, 0.005, 0.5], 200)
    assert v.tolist() == pytest.approx([1.0, 0.005, 0.5])
    assert r.tolist() == [0, 1, 1] and c.tolist() == [1, 0, 2]


def test_coo_to_adjacency_ptr():
    # graph.rs:1566-1602 (row pointer form of the adjacency list)
    ptr = O.coo_to_adj_ptr(3, np.array([0, 0, 1, 2]))
    assert ptr.tolist() == [0, 2, 3, 4]
    assert O.coo_to_adj_ptr(3, np.array([], np.int64)).tolist() == [0, 0, 0, 0]


# ------------------------------------------------------ CSR (optimiser)

TRI = ([0, 2, 4, 6], [1, 2, 0, 2, 0, 1], [1.0, 0.5, 1.0, 1.0, 0.5, 1.0])


def _tri_csr():
    ptr, col, w = TRI
    st, csr = O.csr_from_graph(3, np.array(ptr, np.uint64), col, w)
    assert st == O.OK
    return csr


def test_csr_triangle_layout():
    # umap_optimiser_gpu.rs:1716-1728
    csr = _tri_csr()
    assert csr["n_edges"] == 3
    assert csr["offsets"].tolist() == [0, 2, 4, 6]
    assert csr["edge_idx"].tolist() == [0, 1, 0, 2, 1, 2]
    assert csr["other"].tolist() == [1, 2, 0, 2, 0, 1]


def test_csr_triangle_sampling_periods():
    # umap_optimiser_gpu.rs:1730-1737
    assert _tri_csr()["eps"].tolist() == [1.0, 2.0, 1.0]


def test_csr_offsets_sum_to_2x_edges():
    # umap_optimiser_gpu.rs:1741-1749
    csr = _tri_csr()
    assert csr["offsets"][-1] == 2 * csr["n_edges"]


def test_csr_zero_nodes_and_no_edges():
    # umap_optimiser_gpu.rs:1751-1767
    st, _ = O.csr_from_graph(0, np.zeros(1, np.uint64), [], [])
    assert st == O.NO_DATA
    st, _ = O.csr_from_graph(3, np.zeros(4, np.uint64), [], [])
    assert st == O.NO_GRAPH_EDGES


def test_csr_drops_self_loops():
    # umap_optimiser_gpu.rs:1769-1776
    st, csr = O.csr_from_graph(2, np.array([0, 2, 4], np.uint64), [0, 1, 1, 0], [1, 1, 1, 1])
    assert csr["n_edges"] == 1 and csr["other"].tolist() == [1, 0]


def test_csr_asymmetric_input():
    # umap_optimiser_gpu.rs:1778-1785
    st, csr = O.csr_from_graph(3, np.array([0, 2, 2, 2], np.uint64), [1, 2], [1.0, 0.5])
    assert csr["n_edges"] == 2 and csr["offsets"].tolist() == [0, 2, 3, 4]


def _adj(rows):
    ptr = np.zeros(len(rows) + 1, np.uint64)
    ptr[1:] = np.cumsum([len(r) for r in rows])
    return ptr, [c for r in rows for c, _ in r], [w for r in rows for _, w in r]


def test_csr_other_adjacency_forms():
    """from_graph (umap_optimiser_gpu.rs:132-209) on the adjacency forms the
    device build is also tested on, with the results its definition gives:
    edges are the i < j entries in adjacency order, each node's CSR row lists
    its edges in edge order, periods are 1 / (w / max_w) or 1e8."""
    # an unsorted row, and lower entries whose weights differ from their mirrors'
    st, c = O.csr_from_graph(3, *_adj([[(2, 0.5), (1, 1.0)], [(0, 0.3)], [(0, 0.9), (1, 0.25)]]))
    assert st == O.OK and c["n_edges"] == 2
    assert c["offsets"].tolist() == [0, 2, 3, 4]
    assert c["edge_idx"].tolist() == [0, 1, 1, 0] and c["other"].tolist() == [2, 1, 0, 0]
    assert c["eps"].tolist() == [2.0, 1.0] and c["mu"].tolist() == [0.5, 1.0]
    # a repeated entry is a second edge; a self entry is dropped
    st, c = O.csr_from_graph(2, *_adj([[(0, 1.0), (1, 0.5), (1, 0.5)], [(0, 0.5)]]))
    assert st == O.OK and c["n_edges"] == 2
    assert c["offsets"].tolist() == [0, 2, 4]
    assert c["edge_idx"].tolist() == [0, 1, 0, 1] and c["other"].tolist() == [1, 1, 0, 0]
    assert c["eps"].tolist() == [1.0, 1.0]
    # only lower entries: no edge
    st, _ = O.csr_from_graph(3, *_adj([[], [(0, 0.7)], [(1, 0.4)]]))
    assert st == O.NO_GRAPH_EDGES
    # a zero weight gets the 1e8 period
    st, c = O.csr_from_graph(3, *_adj([[(1, 0.0), (2, 1.0)], [], []]))
    assert st == O.OK and c["eps"].tolist() == [np.float32(1e8), 1.0]


# ------------------------------------------------- kernels (CPU mirrors)

def _tri_params():
    # umap_optimiser_gpu.rs:1651-1671
    return dict(a=1.5, b=0.9, lr=1.0, gamma=1.0, n_epochs=10, neg_sample_rate=5, min_dist=0.1,
                beta1=0.9, beta2=0.999, eps=1e-7)


TRI_EMBD = np.array([[0, 0], [1, 0], [0, 1]], np.float32)


def test_grad_empty_epoch():
    # umap_optimiser_gpu.rs:1995-2003
    csr = _tri_csr()
    g, hu = O.grad_accum(TRI_EMBD, csr, csr["eps"], 0, 42, 5, 1.5, 0.9, 1.0)
    assert (g == 0).all() and (hu == 0).all()


def test_grad_single_edge_hand_computed():
    # umap_optimiser_gpu.rs:2060-2092
    st, csr = O.csr_from_graph(2, np.array([0, 1, 2], np.uint64), [1, 0], [1.0, 1.0])
    e = np.array([[0, 0], [3, 0]], np.float32)
    g, hu = O.grad_accum(e, csr, csr["eps"], 5, 42, 0, 1.0, 1.0, 1.0)
    assert g.ravel().tolist() == pytest.approx([1.2, 0.0, -1.2, 0.0], abs=1e-5)
    assert hu.tolist() == [1, 1]


def test_grad_deterministic():
    # umap_optimiser_gpu.rs:2094-2104
    csr = _tri_csr()
    g1, _ = O.grad_accum(TRI_EMBD, csr, csr["eps"], 5, 42, 5, 1.5, 0.9, 1.0)
    g2, _ = O.grad_accum(TRI_EMBD, csr, csr["eps"], 5, 42, 5, 1.5, 0.9, 1.0)
    assert (g1 == g2).all()


def test_grad_injected_negatives_equal_hash():
    # umap_optimiser_gpu.rs:806-815: the hash draws k per (node, edge_local,
    # neg); injecting exactly those k must reproduce the sampled gradient
    csr = _tri_csr()
    n, nr = 3, 5
    inj = np.zeros((6, nr), np.uint32)
    for node in range(n):
        for el, pos in enumerate(range(csr["offsets"][node], csr["offsets"][node + 1])):
            for k in range(nr):
                inj[pos, k] = O.hash_neg(42, node, 5, el, k, n)
    g1, _ = O.grad_accum(TRI_EMBD, csr, csr["eps"], 5, 42, nr, 1.5, 0.9, 1.0)
    g2, _ = O.grad_accum(TRI_EMBD, csr, csr["eps"], 5, 42, nr, 1.5, 0.9, 1.0, injected=inj)
    assert (g1 == g2).all()


def test_hash_matches_reference_formula():
    # umap_optimiser_gpu.rs:1379-1391, written out independently in Python
    def h(seed, node, epoch, el, neg, n):
        M = 0xFFFFFFFF
        x = seed ^ (node * 0x9E3779B1 & M) ^ (epoch * 0x85EBCA77 & M) ^ (el * 0xC2B2AE3D & M) ^ (neg * 0x27D4EB2F & M)
        x ^= x >> 16
        x = x * 0x7FEB352D & M
        x ^= x >> 15
        x = x * 0x846CA68B & M
        x ^= x >> 16
        return x % n
    for args in [(42, 0, 5, 0, 0, 3), (7, 123456, 199, 17, 4, 1000000), (0xDEADBEEF, 9, 0, 3, 2, 97)]:
        assert O.hash_neg(*args) == h(*args)


def test_philox_known_answer():
    # Philox4x32-10 known-answer vector from the Random123 distribution
    # (kat_vectors: counter 0, key 0 -> 6627e8d5 e169c58d bc57ac4c 9b00dbd8)
    import ctypes as C
    c = (C.c_uint32 * 4)(0, 0, 0, 0)
    O.lib().orc_philox4x32_10.argtypes = [C.c_uint32 * 4, C.c_uint32, C.c_uint32]
    O.lib().orc_philox4x32_10(c, 0, 0)
    assert [hex(x) for x in c] == ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]


def test_adam_single_step_hand_computed():
    # umap_optimiser_gpu.rs:2211-2242
    fused, epsc = O.adam_epoch_scalars(1.0, 0.9, 0.999, 1e-7, 0, 10)
    m = np.zeros((1, 1), np.float32)
    v = np.zeros((1, 1), np.float32)
    e = np.zeros((1, 1), np.float32)
    O.adam_update(np.ones((1, 1), np.float32), np.ones(1, np.uint32), m, v, e, fused, epsc, 0.9, 0.999)
    assert m[0, 0] == pytest.approx(0.1, abs=1e-6)
    assert v[0, 0] == pytest.approx(0.001, abs=1e-6)
    assert e[0, 0] == pytest.approx(1.0, abs=1e-4)


def test_adam_inactive_node_preserved():
    # umap_optimiser_gpu.rs:2192-2209
    fused, epsc = O.adam_epoch_scalars(1.0, 0.9, 0.999, 1e-7, 3, 10)
    e = np.array([[1.5, -2.5], [7.0, 8.0]], np.float32)
    m = np.array([[0.1, 0.2], [0.3, 0.4]], np.float32)
    v = np.array([[0.01, 0.02], [0.03, 0.04]], np.float32)
    e0, m0, v0 = e.copy(), m.copy(), v.copy()
    O.adam_update(np.full((2, 2), 5.0, np.float32), np.zeros(2, np.uint32), m, v, e, fused, epsc, 0.9, 0.999)
    assert (e == e0).all() and (m == m0).all() and (v == v0).all()


def test_schedule_updates():
    # umap_optimiser_gpu.rs:2342-2379
    csr = _tri_csr()
    c = csr["eps"].copy()
    O.schedule_update(csr["eps"], c, 5)
    assert c.tolist() == [2.0, 4.0, 2.0]
    c = csr["eps"].copy()
    O.schedule_update(csr["eps"], c, 0)
    assert c.tolist() == csr["eps"].tolist()
    c = csr["eps"].copy()
    O.schedule_update(csr["eps"], c, 1)
    assert c.tolist() == [2.0, 2.0, 2.0]


def test_dens_radii_known_value():
    # umap_optimiser_gpu.rs:1409-1453 on the triangle: node 0 sees d^2 = 1, 1
    csr = _tri_csr()
    re, phi = O.dens_radii(TRI_EMBD, csr, 1.5, 0.9)
    phi1 = 1.0 / (1.0 + 1.5 * 1.0)
    assert phi[0] == pytest.approx(2 * phi1, rel=1e-6)
    assert re[0] == pytest.approx(math.log(1e-8 + (2 * phi1) / (2 * phi1)), abs=1e-6)


# ------------------------------------------------------------ density.rs


def test_edge_distances_squared_passthrough():
    # density.rs:560-577
    d = O.edge_distances_from_knn([0, 1], [1, 0], [[1], [0]], [[9.0], [9.0]], True)
    assert d.tolist() == [9.0, 9.0]
    d = O.edge_distances_from_knn([0, 1], [1, 0], [[1], [0]], [[9.0], [9.0]], False)
    assert d.tolist() == [81.0, 81.0]


def test_edge_distances_reverse_row():
    # density.rs:579-591
    d = O.edge_distances_from_knn([0, 1], [1, 0], [[7], [0]], [[1.0], [4.0]], True)
    assert d.tolist() == [4.0, 4.0]


def test_original_log_radii_known_value():
    # density.rs:593-623
    st, r, ms = O.original_log_radii(3, [0, 0, 1, 2], [1.0, 3.0, 1.0, 3.0], [4.0, 8.0, 4.0, 8.0])
    assert st == O.OK
    assert ms.tolist() == [4.0, 1.0, 3.0]
    raw = np.log(1e-8 + np.array([7.0, 4.0, 8.0]))
    want = (raw - raw.mean()) / raw.std(ddof=1)
    assert r == pytest.approx(want, abs=1e-6)


def test_original_log_radii_degenerate_and_isolated():
    # density.rs:625-650
    st, _, _ = O.original_log_radii(2, [0, 1], [1.0, 1.0], [4.0, 4.0])
    assert st == O.DEGENERATE_LOCAL_RADII
    st, r, ms = O.original_log_radii(3, [0, 1], [1.0, 2.0], [4.0, 9.0])
    assert st == O.OK and ms[2] == 0.0 and np.isfinite(r).all()


def test_correlation_stats():
    # density.rs:652-677
    r = np.array([-1.0, 0.0, 1.0], np.float32)
    mean, sd, cov = O.correlation_stats(3 * r + 5, r, 0.0)
    assert (mean, sd, cov) == pytest.approx((5.0, 3.0, 3.0), abs=1e-6)
    _, sd0, _ = O.correlation_stats(r, r, 0.0)
    _, sd1, _ = O.correlation_stats(r, r, 0.1)
    assert sd0 == pytest.approx(1.0, abs=1e-6)
    assert sd1 == pytest.approx(math.sqrt(1.1), abs=1e-6)


def test_dens_is_active():
    # density.rs:692-718
    assert not O.dens_is_active(2.0, 0.3, 69, 100)
    assert O.dens_is_active(2.0, 0.3, 70, 100)
    assert O.dens_is_active(2.0, 0.3, 99, 100)
    assert not O.dens_is_active(0.0, 1.0, 99, 100)
    # 200 epochs, frac 0.3: active exactly for epochs 140..199 in f32
    act = [O.dens_is_active(2.0, 0.3, e, 200) for e in range(200)]
    assert act.index(True) == 140 and sum(act) == 60


# --------------------------------------------------- optimiser parameters


def test_fit_params_constraints_and_curve():
    # umap_optimisers.rs:1559-1593
    for dt in (np.float32, np.float64):
        a, b = O.fit_params(0.1, 1.0, 300, dt)
        assert 0.001 <= a <= 10 and 0.1 <= b <= 2
        f = lambda x: 1 / (1 + a * x ** (2 * b))
        assert f(0.1) > 0.9 and f(3.0) < 0.1 and f(0.1) > f(1.5) > f(3.0)


# ------------------------------------------------------- full optimisers

TWO_TRI = [[(1, 1.0), (2, 1.0)], [(0, 1.0), (2, 1.0)], [(0, 1.0), (1, 1.0), (3, 0.1)],
           [(2, 0.1), (4, 1.0), (5, 1.0)], [(3, 1.0), (5, 1.0)], [(3, 1.0), (4, 1.0)]]
TWO_TRI_EMBD = np.array([[0, 0], [10, 0], [0, 10], [10, 10], [-5, -5], [15, 15]], np.float32)


def _adj(g):
    ptr = np.zeros(len(g) + 1, np.uint64)
    ptr[1:] = np.cumsum([len(r) for r in g])
    col = np.array([j for r in g for j, _ in r], np.uint32)
    w = np.array([w for r in g for _, w in r], np.float32)
    return ptr, col, w


def default_2d(**kw):
    # umap_optimisers.rs:56-69 with training/mod.rs:15-24 constants
    p = dict(a=1.5, b=0.9, lr=1.0, gamma=1.0, n_epochs=500, neg_sample_rate=5, min_dist=0.1,
             beta1=0.5, beta2=0.9, eps=1e-7)
    p.update(kw)
    return p


def _inter_intra(e):
    d = lambda i, j: float(np.linalg.norm(e[i] - e[j]))
    intra = ((d(0, 1) + d(0, 2) + d(1, 2)) / 3 + (d(3, 4) + d(3, 5) + d(4, 5)) / 3) / 2
    inter = np.mean([d(0, 3), d(0, 4), d(0, 5), d(1, 3), d(1, 4), d(1, 5)])
    return inter, intra


@pytest.mark.parametrize("algo", ["adam_gpu", "adam_parallel", "adam", "sgd"])
def test_optimisers_preserve_graph_structure(algo):
    # umap_optimiser_gpu.rs:2383-2448; umap_optimisers.rs:1923-2085
    ptr, col, w = _adj(TWO_TRI)
    p = default_2d(n_epochs=200)
    if algo == "adam_gpu":
        st, e = O.optimise_adam_gpu(TWO_TRI_EMBD, 6, ptr, col, w, p, 42)
    elif algo == "adam_parallel":
        st, e = O.optimise_adam_parallel(TWO_TRI_EMBD, 6, ptr, col, w, p, 42)
    else:
        st, e = O.optimise_sequential(algo, TWO_TRI_EMBD, 6, ptr, col, w, p, 42)
    assert st == O.OK and np.isfinite(e).all()
    inter, intra = _inter_intra(e)
    assert inter > 1.5 * intra


def test_adam_gpu_driver_deterministic_and_finite():
    # umap_optimiser_gpu.rs:2450-2505
    ptr, col, w = _adj([[(1, 1.0), (2, 0.5)], [(0, 1.0), (2, 1.0)], [(0, 0.5), (1, 1.0)]])
    p = _tri_params()
    st, e1 = O.optimise_adam_gpu(TRI_EMBD, 3, ptr, col, w, p, 42)
    st, e2 = O.optimise_adam_gpu(TRI_EMBD, 3, ptr, col, w, p, 42)
    assert np.isfinite(e1).all() and (e1 == e2).all()


def test_cpu_optimisers_reproducible():
    # umap_optimisers.rs:1693-1741, :1898-1921
    ptr, col, w = _adj([[(1, 1.0)], [(0, 1.0)]])
    p = default_2d(a=1.0, b=1.0, n_epochs=50)
    e0 = np.array([[0, 0], [1, 0]], np.float32)
    for fn in (lambda: O.optimise_adam_parallel(e0, 2, ptr, col, w, p, 42),
               lambda: O.optimise_sequential("adam", e0, 2, ptr, col, w, p, 42),
               lambda: O.optimise_sequential("sgd", e0, 2, ptr, col, w, p, 42)):
        (s1, a1), (s2, a2) = fn(), fn()
        assert (a1 == a2).all()


def test_empty_graph_errors():
    # umap_optimisers.rs:1677-1691; umap_optimiser_gpu.rs:151-153
    ptr = np.zeros(4, np.uint64)
    e = np.zeros((3, 2), np.float32)
    st, _ = O.optimise_adam_gpu(e, 3, ptr, np.zeros(0, np.uint32), np.zeros(0, np.float32), default_2d(), 1)
    assert st == O.NO_GRAPH_EDGES
