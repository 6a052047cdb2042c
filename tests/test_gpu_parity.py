"""CUDA path vs the oracle, through the C ABI (needs a B200).

Tolerances are the hot path's parity bar:
* graph: edge index structure bit-exact; sigma, rho, weights within 1e-6
  relative (the device evaluates exp as (float)exp((double)x), glibc's
  expf is not correctly rounded in every case);
* one epoch with the reference's negatives injected: the update within 1e-5
  relative of the reference's own (oracle gradient through oracle Adam), per
  element on the steps of at least a tenth of the largest (f64 steps);
* samplers, CSR, Adam-from-identical-gradient, schedule: bit-exact.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._problems import init_embedding, oracle_graph, update_errors

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")


def _tri():
    return umapcu.Adjacency.from_lists([[(1, 1.0), (2, 0.5)], [(0, 1.0), (2, 1.0)], [(0, 0.5), (1, 1.0)]])


TRI_EMBD = np.array([[0, 0], [1, 0], [0, 1]], np.float32)


def _tri_params(**kw):
    p = umapcu.UmapOptimParams(a=1.5, b=0.9, lr=1.0, gamma=1.0, n_epochs=10, neg_sample_rate=5, min_dist=0.1,
                               beta1=0.9, beta2=0.999, eps=1e-7)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


# ------------------------------------------------------------- graph stage

def test_smooth_knn_dist_parity():
    g = oracle_graph()
    sig, rho = umapcu.smooth_knn_dist(g["dist"])
    assert (rho == g["rho"]).all()
    rel = np.abs(sig - g["sigma"]) / np.abs(g["sigma"])
    assert rel.max() <= 1e-6, rel.max()


def test_smooth_knn_dist_kats():
    # graph.rs:1442-1471
    sig, rho = umapcu.smooth_knn_dist(np.array([[1.0, 2.0], [1.5, 3.0], [0.5, 1.5]], np.float32))
    assert rho.tolist() == pytest.approx([1.0, 1.5, 0.5], abs=1e-4) and (sig > 0).all()
    _, rho = umapcu.smooth_knn_dist(np.array([[0.0, 1.0, 2.0], [0.0, 1.0, 2.0]], np.float32), local_connectivity=0.0)
    assert (rho == 0).all()


def test_graph_structure_bit_exact_and_weights():
    g = oracle_graph()
    G, sig, rho = umapcu.construct_umap_graph(g["idx"], g["dist"], n_epochs=200, return_sigma_rho=True)
    assert G.row_indices.size == g["row"].size
    assert (G.row_indices == g["row"]).all() and (G.col_indices == g["col"]).all()
    rel = np.abs(G.values - g["val"]) / g["val"]
    assert rel.max() <= 1e-6, rel.max()


@pytest.mark.parametrize("mix,lc", [(0.5, 1.0), (1.0, 2.5), (0.0, 0.0)])
def test_graph_params_variants(mix, lc):
    g = oracle_graph()
    (r, c, v), _, _ = O.construct_umap_graph(g["idx"], g["dist"], 100, local_connectivity=lc, mix_weight=mix)
    G = umapcu.construct_umap_graph(g["idx"], g["dist"], umapcu.UmapGraphParams(1e-5, lc, mix), n_epochs=100)
    assert (G.row_indices == r).all() and (G.col_indices == c).all()
    assert np.abs(G.values - v).max() <= 1e-6 * np.abs(v).max()


def test_graph_with_self_entries_and_duplicates_edge_cases():
    # kNN lists that contain self (graph.rs:635-637 skips it) and a node
    # referenced by nobody
    idx = np.array([[0, 1, 2], [1, 0, 2], [0, 1, 3], [2, 0, 1]], np.int32)
    dist = np.array([[0.0, 1.0, 2.0], [0.0, 1.0, 3.0], [2.0, 3.0, 4.0], [4.0, 5.0, 6.0]], np.float32)
    (r, c, v), _, _ = O.construct_umap_graph(idx, dist, 50)
    G = umapcu.construct_umap_graph(idx, dist, n_epochs=50)
    assert (G.row_indices == r).all() and (G.col_indices == c).all()
    assert np.allclose(G.values, v, rtol=1e-6, atol=0)


# ------------------------------------------------------------- CSR

def test_csr_parity_with_from_graph():
    g = oracle_graph()
    adj = umapcu.Adjacency(g["ptr"], g["col"], g["val"])
    st = umapcu.UmapGpuState(init_embedding(3000), adj, umapcu.UmapOptimParams(n_epochs=200))
    csr = st.csr()
    stt, ref = O.csr_from_graph(3000, g["ptr"], g["col"], g["val"])
    assert csr["n_edges"] == ref["n_edges"]
    for key in ("offsets", "edge_idx", "other"):
        assert (csr[key] == ref[key]).all(), key
    assert (csr["eps"] == ref["eps"]).all() and (csr["mu"] == ref["mu"]).all()


def test_csr_triangle_kats():
    # umap_optimiser_gpu.rs:1716-1737, :1769-1785
    st = umapcu.UmapGpuState(TRI_EMBD, _tri(), _tri_params())
    c = st.csr()
    assert c["offsets"].tolist() == [0, 2, 4, 6]
    assert c["edge_idx"].tolist() == [0, 1, 0, 2, 1, 2]
    assert c["other"].tolist() == [1, 2, 0, 2, 0, 1]
    assert c["eps"].tolist() == [1.0, 2.0, 1.0]
    st = umapcu.UmapGpuState(np.zeros((2, 2), np.float32), [[(0, 1.0), (1, 1.0)], [(1, 1.0), (0, 1.0)]], _tri_params())
    assert st.n_edges == 1 and st.csr()["other"].tolist() == [1, 0]
    st = umapcu.UmapGpuState(TRI_EMBD, [[(1, 1.0), (2, 0.5)], [], []], _tri_params())
    assert st.n_edges == 2 and st.csr()["offsets"].tolist() == [0, 2, 3, 4]


def test_errors_match_reference():
    # umap_optimiser_gpu.rs:1751-1767
    with pytest.raises(umapcu.NoGraphEdges):
        umapcu.UmapGpuState(TRI_EMBD, [[], [], []], _tri_params())
    with pytest.raises(umapcu.NoData):
        umapcu.UmapGpuState(np.zeros((0, 2), np.float32), [], _tri_params())
    # a neighbour index past the last node (the reference's Vec indexing
    # panics): rejected on the device before any edge is formed
    with pytest.raises(umapcu.ManifoldsError):
        umapcu.UmapGpuState(TRI_EMBD, [[(1, 1.0), (3, 0.5)], [(0, 1.0)], [(0, 0.5)]], _tri_params())


# ------------------------------------------------------------- kernels

def test_samplers_bit_exact():
    for seed, node, epoch, el, n in [(42, 0, 5, 0, 3), (7, 123456, 199, 17, 1000000), (2 ** 40 + 5, 9, 0, 3, 97)]:
        got = umapcu.sample_negatives(umapcu.NEG_REF_HASH, seed, node, 0, epoch, el, 16, n)
        want = [O.hash_neg(seed, node, epoch, el, k, n) for k in range(16)]
        assert got.tolist() == want
        got = umapcu.sample_negatives(umapcu.NEG_PHILOX, seed, node, 1234 + el, epoch, el, 16, n)
        want = [O.philox_neg(seed, 1234 + el, epoch, k, n) for k in range(16)]
        assert got.tolist() == want


def test_adam_hook_kats_and_parity():
    # umap_optimiser_gpu.rs:2192-2295
    p = _tri_params()
    e, m, v = np.zeros((1, 1), np.float32), np.zeros((1, 1), np.float32), np.zeros((1, 1), np.float32)
    umapcu.adam_update(np.ones((1, 1), np.float32), np.ones(1, np.uint32), m, v, e, p, 0)
    assert m[0, 0] == pytest.approx(0.1, abs=1e-6) and v[0, 0] == pytest.approx(0.001, abs=1e-6)
    assert e[0, 0] == pytest.approx(1.0, abs=1e-4)
    n, d = 5, 2
    emb = (np.arange(n * d, dtype=np.float32) * 0.5 - 1.0).reshape(n, d)
    m0 = (np.arange(n * d, dtype=np.float32) * 0.01).reshape(n, d)
    v0 = (np.arange(n * d, dtype=np.float32) * 0.001 + 1e-6).reshape(n, d)
    g = np.array([((i * 7 + 3) % 5) * 0.1 for i in range(n * d)], np.float32).reshape(n, d)
    hu = np.array([1, 0, 1, 1, 0], np.uint32)
    ge, gm, gv = emb.copy(), m0.copy(), v0.copy()
    umapcu.adam_update(g, hu, gm, gv, ge, p, 4)
    oe, om, ov = emb.copy(), m0.copy(), v0.copy()
    fused, epsc = O.adam_epoch_scalars(p.lr, p.beta1, p.beta2, p.eps, 4, p.n_epochs)
    O.adam_update(g, hu, om, ov, oe, fused, epsc, p.beta1, p.beta2)
    assert (ge == oe).all() and (gm == om).all() and (gv == ov).all()
    assert (ge[1] == emb[1]).all() and (ge[4] == emb[4]).all()


def test_schedule_hook_kats():
    # umap_optimiser_gpu.rs:2342-2379
    eps = np.array([1.0, 2.0, 1.0], np.float32)
    for epoch, want in [(5, [2.0, 4.0, 2.0]), (0, [1.0, 2.0, 1.0]), (1, [2.0, 2.0, 2.0])]:
        c = eps.copy()
        umapcu.edge_schedule_update(eps, c, epoch)
        assert c.tolist() == want


def test_grad_kats_on_device():
    # umap_optimiser_gpu.rs:1995-2003 (empty epoch), :2060-2092 (hand edge)
    st = umapcu.UmapGpuState(TRI_EMBD, _tri(), _tri_params())
    g, hu = st.epoch_debug(0)
    assert (g == 0).all() and (hu == 0).all()
    p = umapcu.UmapOptimParams(a=1.0, b=1.0, lr=1.0, gamma=1.0, n_epochs=10, neg_sample_rate=0, beta1=0.9,
                               beta2=0.999, eps=1e-7)
    st = umapcu.UmapGpuState(np.array([[0, 0], [3, 0]], np.float32), [[(1, 1.0)], [(0, 1.0)]], p)
    st.run(0, 5)
    g, hu = st.epoch_debug(5)
    # after the first epochs the points moved; redo from the hand-computed
    # state at epoch 5 with fresh positions
    st.write(np.array([[0, 0], [3, 0]], np.float32))
    g, hu = st.epoch_debug(6)
    assert g.ravel().tolist() == pytest.approx([1.2, 0.0, -1.2, 0.0], abs=1e-5)


def _epoch_problem(n_dim=2):
    g = oracle_graph()
    adj = umapcu.Adjacency(g["ptr"], g["col"], g["val"])
    return g, adj


def test_pow_accuracy():
    """x^b as the kernels evaluate it vs the correctly rounded power over
    x in [1e-8, 1e6]. The MUFU form 2^(b log2 x) (lg2.approx / ex2.approx)
    carries the f32 rounding of the exponent b log2 x, so its bound grows
    with |b log2 x|: rel <= 1e-6 + 1.5e-7 |b log2 x| (<= 4e-6 at the range
    ends, about 2e-6 for squared distances below 1e4). CUDA powf within
    1e-6: the layout code is compiled without FMA contraction (the
    reference never contracts), which also applies inside CUDA's inlined
    powf and costs it a few ulp over its documented 4 ulp."""
    x = np.geomspace(1e-8, 1e6, 200001).astype(np.float32)
    for b in (0.79158, 0.9, 1.0, 0.5, 1.7):
        want = np.power(x.astype(np.float64), b)
        fast = umapcu.eval_pow(x, b, precise=False).astype(np.float64)
        prec = umapcu.eval_pow(x, b, precise=True).astype(np.float64)
        rel = np.abs(fast - want) / want
        bound = 1e-6 + 1.5e-7 * np.abs(b * np.log2(x.astype(np.float64)))
        assert (rel <= bound).all(), (b, rel.max())
        assert (np.abs(prec - want) / want).max() <= 1e-6, b


@pytest.mark.parametrize("n_dim,precise,nr", [(2, False, 5), (3, False, 5), (2, True, 5), (2, False, 7), (4, False, 2)])
def test_single_epoch_injected_negatives(n_dim, precise, nr):
    """One epoch with the reference's negatives injected,
    each epoch from the oracle's state on both sides: the gradient vs the
    oracle's mirror of umap_grad_accum; the device's Adam vs the oracle's
    applied to the same (device) gradient, bit for bit; and the device's
    update vs the reference's own (the oracle's gradient through the oracle's
    Adam), as the f64 steps the two gradients imply (update_errors): 1e-5
    relative on the elements whose step is at least a tenth of the largest
    and whose gradient sum does not cancel, and 1e-5 relative plus 64 units of
    the reference's own f32 rounding of the gradient sum on every element."""
    g, adj = _epoch_problem()
    n = 3000
    p = umapcu.UmapOptimParams(n_epochs=200, neg_sample_rate=nr)
    emb = init_embedding(n, n_dim, seed=11)
    st = umapcu.UmapGpuState(emb, adj, p, seed=42)
    st.set_precise_pow(precise)
    stt, csr = O.csr_from_graph(n, g["ptr"], g["col"], g["val"])
    cursor = csr["eps"].copy()
    epochs = 4
    m = np.zeros((n, n_dim), np.float32)
    v = np.zeros((n, n_dim), np.float32)
    y = emb.copy()
    rng = np.random.default_rng(5)
    for e in range(epochs):
        inj = rng.integers(0, n, (2 * csr["n_edges"], nr)).astype(np.uint32)
        y0, m0, v0 = y.copy(), m.copy(), v.copy()
        st.write(y0, m0, v0)
        gg, hu = st.epoch_debug(e, injected=inj)
        S = np.zeros((n, n_dim), np.float64)
        go, huo = O.grad_accum(y0, csr, cursor, e, 42, nr, p.a, p.b, p.gamma, injected=inj, abs_sum=S)
        assert (hu == huo).all()
        scale = np.abs(go).max()
        tol = 1e-6 if precise else 1e-5
        assert np.abs(gg - go).max() <= tol * max(scale, 1e-30), (e, np.abs(gg - go).max(), scale)
        fused, epsc = O.adam_epoch_scalars(p.lr, p.beta1, p.beta2, p.eps, e, p.n_epochs)
        ye, me, ve, ce = st.read()
        # the device's Adam: the oracle's, bit for bit, on the same gradient
        ya, ma, va = y0.copy(), m0.copy(), v0.copy()
        O.adam_update(gg, huo, ma, va, ya, fused, epsc, p.beta1, p.beta2)
        assert (ye == ya).all() and (me == ma).all() and (ve == va).all()
        # the reference's own update
        O.adam_update(go, huo, m, v, y, fused, epsc, p.beta1, p.beta2)
        O.schedule_update(csr["eps"], cursor, e)
        assert (ce == cursor).all()
        if not huo.any():
            continue
        act = np.repeat(huo.astype(bool)[:, None], n_dim, 1)
        r = update_errors(go, gg, S, m0, v0, fused, epsc, p.beta1, p.beta2, act)
        assert r["floor_max"] <= 1e-5 and r["bound_ok"], (e, r["floor_max"], r["worst_over_bound"])


def test_single_epoch_update_from_reference_state():
    """Embedding after one epoch from the same state, with the reference's
    own hash negatives: GPU vs oracle within 1e-5 relative (f32)."""
    g, adj = _epoch_problem()
    n = 3000
    p = umapcu.UmapOptimParams(n_epochs=200)
    emb = init_embedding(n, 2, seed=3)
    st = umapcu.UmapGpuState(emb, adj, p, seed=1234)
    stt, csr = O.csr_from_graph(n, g["ptr"], g["col"], g["val"])
    cursor = csr["eps"].copy()
    y = emb.copy()
    m = np.zeros_like(y)
    v = np.zeros_like(y)
    for e in range(6):
        # both sides start the epoch from the oracle's state
        y0 = y.copy()
        st.write(y0, m, v)
        go, huo = O.grad_accum(y0, csr, cursor, e, 1234, 5, p.a, p.b, p.gamma)
        fused, epsc = O.adam_epoch_scalars(p.lr, p.beta1, p.beta2, p.eps, e, p.n_epochs)
        O.adam_update(go, huo, m, v, y, fused, epsc, p.beta1, p.beta2)
        O.schedule_update(csr["eps"], cursor, e)
        gg, hu = st.epoch_debug(e)
        ye, me, ve, ce = st.read()
        assert (hu == huo).all() and (ce == cursor).all()
        assert np.abs(gg - go).max() <= 1e-5 * np.abs(go).max()
        d_ref = y - y0
        err = np.abs((ye - y0) - d_ref)
        assert err.max() <= 1e-5 * np.abs(d_ref).max(), (e, err.max(), np.abs(d_ref).max())
        assert np.abs(ye - y).max() <= 1e-5 * np.abs(y).max()


def test_gpu_deterministic_full_run():
    g, adj = _epoch_problem()
    p = umapcu.UmapOptimParams(n_epochs=100)
    e1 = init_embedding(3000)
    e2 = e1.copy()
    umapcu.optimise_embedding_adam_gpu(e1, adj, p, seed=42)
    umapcu.optimise_embedding_adam_gpu(e2, adj, p, seed=42)
    assert (e1 == e2).all() and np.isfinite(e1).all()


def test_gpu_driver_preserves_graph_structure():
    # umap_optimiser_gpu.rs:2383-2448
    graph = [[(1, 1.0), (2, 1.0)], [(0, 1.0), (2, 1.0)], [(0, 1.0), (1, 1.0), (3, 0.1)],
             [(2, 0.1), (4, 1.0), (5, 1.0)], [(3, 1.0), (5, 1.0)], [(3, 1.0), (4, 1.0)]]
    e = np.array([[0, 0], [10, 0], [0, 10], [10, 10], [-5, -5], [15, 15]], np.float32)
    umapcu.optimise_embedding_adam_gpu(e, graph, umapcu.UmapOptimParams(n_epochs=200), seed=42)
    d = lambda i, j: float(np.linalg.norm(e[i] - e[j]))
    intra = ((d(0, 1) + d(0, 2) + d(1, 2)) / 3 + (d(3, 4) + d(3, 5) + d(4, 5)) / 3) / 2
    inter = np.mean([d(0, 3), d(0, 4), d(0, 5), d(1, 3), d(1, 4), d(1, 5)])
    assert inter > 1.5 * intra and np.isfinite(e).all()


def test_gpu_no_nan_triangle():
    # umap_optimiser_gpu.rs:2450-2472
    e = TRI_EMBD.copy()
    umapcu.optimise_embedding_adam_gpu(e, _tri(), _tri_params(), seed=42)
    assert np.isfinite(e).all()
