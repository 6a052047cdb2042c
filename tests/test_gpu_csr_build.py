"""The optimiser CSR build against the oracle's restatement of
UmapCsrGraph::from_graph (umap_optimiser_gpu.rs:132-209), through the C ABI
(needs a B200), on adjacencies of every form the reference accepts: the
fuzzy graph, weights that differ between an entry and its mirror, missing or
extra mirrors, unsorted and repeated rows, self entries, empty rows and hub
rows longer than a warp. Offsets, edge indices, other endpoints, periods and
weights must equal the reference's bit for bit; row pointers out of order
are refused.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._problems import init_embedding, oracle_graph

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")


def _rows(ptr, col, val):
    return [list(zip(col[ptr[i]:ptr[i + 1]].tolist(), val[ptr[i]:ptr[i + 1]].tolist()))
            for i in range(ptr.size - 1)]


def _adj(rows):
    a = umapcu.Adjacency.from_lists(rows)
    return a.ptr, a.col, a.w


def _check(ptr, col, val, dens=None, epochs=6):
    n = ptr.size - 1
    st = umapcu.UmapGpuState(init_embedding(n), umapcu.Adjacency(ptr, col, val),
                             umapcu.UmapOptimParams(n_epochs=max(epochs, 40)), dens, 42)
    ok, ref = O.csr_from_graph(n, ptr, col, val)
    assert ok == O.OK
    c = st.csr()
    assert c["n_edges"] == ref["n_edges"]
    for key in ("offsets", "edge_idx", "other", "eps", "mu"):
        assert (c[key] == ref[key]).all(), key
    st.run(0, epochs)
    assert np.isfinite(st.read()[0]).all()
    st.close()


def test_fuzzy_graph():
    g = oracle_graph()
    _check(g["ptr"], g["col"], g["val"])


def test_asymmetric_weights_take_the_upper_entry():
    # mirrored structure, lower entries' weights changed: from_graph reads
    # the i < j entries only
    g = oracle_graph()
    ptr, col, val = g["ptr"], g["col"], g["val"].copy()
    row = np.repeat(np.arange(ptr.size - 1), np.diff(ptr).astype(np.int64))
    low = col < row
    val[low] = val[low] * np.float32(0.5) + np.float32(0.25)
    _check(ptr, col, val)


def test_self_loops_empty_rows_and_hubs():
    rng = np.random.default_rng(3)
    n = 700
    edges = set()
    for i in range(1, 500):  # node 0: a hub with 499 neighbours
        edges.add((0, i))
    for i in range(1, 600):  # node 699: a hub whose row is all lower entries
        edges.add((i, 699))
    for _ in range(1500):
        i, j = sorted(rng.integers(1, 650, 2).tolist())
        if i != j:
            edges.add((i, j))
    rows = [[] for _ in range(n)]
    for i, j in edges:
        w = float(rng.uniform(0.05, 1.0))
        rows[i].append((j, w))
        rows[j].append((i, w))
    for v in (5, 17, 699):
        rows[v].append((v, 0.7))  # self entries are dropped
    rows = [sorted(r) for r in rows]
    assert any(len(r) == 0 for r in rows)
    _check(*_adj(rows))


def test_missing_and_moved_mirrors():
    g = oracle_graph()
    rows = _rows(g["ptr"], g["col"], g["val"])
    v = next(i for i, r in enumerate(rows) if any(c < i for c, _ in r))
    c = next(c for c, _ in rows[v] if c < v)
    rows[c] = [(j, w) for j, w in rows[c] if j != v]  # (c, v) gone, (v, c) kept
    _check(*_adj(rows))
    have = {j for j, _ in rows[5]}
    v2 = next(j for j in range(2999, 5, -1) if j not in have and j != v)
    rows[5] = sorted(rows[5] + [(v2, 0.75)])  # (5, v2) without (v2, 5)
    _check(*_adj(rows))


def test_unsorted_and_repeated_rows():
    g = oracle_graph()
    rows = _rows(g["ptr"], g["col"], g["val"])
    rows[10] = rows[10][::-1]
    rows[20] = rows[20] + [rows[20][-1]]
    _check(*_adj(rows))


def test_row_pointers_out_of_order_refused():
    ptr = np.array([0, 2, 1, 3], np.uint64)
    col = np.array([1, 2, 0], np.uint32)
    w = np.ones(3, np.float32)
    with pytest.raises(umapcu.ManifoldsError):
        umapcu.UmapGpuState(init_embedding(3), umapcu.Adjacency(ptr, col, w), umapcu.UmapOptimParams(n_epochs=10))


def test_densmap_graph():
    import umapdata.synth as S
    X, _ = S.variable_density_mixture(2000, 30, 6, seed=5)
    idx, dist = S.exact_knn_cpu(X, 30)
    (r, c, v), _, _ = O.construct_umap_graph(idx, dist, 40)
    ptr = O.coo_to_adj_ptr(2000, r)
    cl = umapcu.CoordinateList(r, c, v, 2000)
    dens = umapcu.DensState.new(umapcu.DensParams(2.0, 0.5, 0.1), cl, idx, dist, True)
    _check(ptr, c, v, dens=dens, epochs=40)
