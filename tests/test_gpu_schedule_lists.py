"""Schedule lists (per-epoch active-entry records built once per state) vs
the per-epoch CSR scan: the same active entries in the same CSR order and
batch boundaries, so results must agree bit for bit, for in-order runs, for
runs that skip epochs (the state falls back to the scan), after reset, and
with the densMAP term (needs a B200). The small problems run the list path
with a block per segment; the 60k-point one runs it with a warp per
segment."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")
from tests._problems import init_embedding, oracle_graph


def _state(adj, emb, p, lists, dens=None, seed=9):
    old = os.environ.pop("UMAPCU_NO_SCHEDULE_LISTS", None)
    try:
        if not lists:
            os.environ["UMAPCU_NO_SCHEDULE_LISTS"] = "1"
        return umapcu.UmapGpuState(emb, adj, p, dens, seed)
    finally:
        os.environ.pop("UMAPCU_NO_SCHEDULE_LISTS", None)
        if old is not None:
            os.environ["UMAPCU_NO_SCHEDULE_LISTS"] = old


@pytest.fixture(scope="module")
def prob():
    g = oracle_graph(n=3000, dim=50, k=15, n_epochs=80)
    return g, umapcu.Adjacency(g["ptr"], g["col"], g["val"])


@pytest.mark.parametrize("calls", [[(0, 80)], [(0, 30), (30, 50)], [(0, 10), (20, 5), (25, 40)],
                                   [(0, 40), (40, 60)]])
def test_lists_equal_scan(prob, calls):
    g, adj = prob
    p = umapcu.UmapOptimParams(n_epochs=80)
    emb = init_embedding(3000, 2, seed=4)
    a, b = _state(adj, emb, p, True), _state(adj, emb, p, False)
    for first, count in calls:  # (40, 60) runs past the lists' 80 epochs
        a.run(first, count)
        b.run(first, count)
        ya, ma, va, ca = a.read()
        yb, mb, vb, cb = b.read()
        assert np.array_equal(ya, yb) and np.array_equal(ma, mb) and np.array_equal(va, vb)
        assert np.array_equal(ca, cb)  # cursors materialised from the lists
    a.reset(emb)
    b.reset(emb)
    a.run(0, 80)
    b.run(0, 80)
    assert np.array_equal(a.read()[0], b.read()[0])
    a.close()
    b.close()


def test_lists_equal_scan_sgd_and_debug_epochs(prob):
    g, adj = prob
    p = umapcu.UmapOptimParams(n_epochs=50)
    emb = init_embedding(3000, 2, seed=6)
    a, b = _state(adj, emb, p, True), _state(adj, emb, p, False)
    a.run(0, 20, umapcu.OPT_SGD)
    b.run(0, 20, umapcu.OPT_SGD)
    ga, ha = a.epoch_debug(20)
    gb, hb = b.epoch_debug(20)
    assert np.array_equal(ga, gb) and np.array_equal(ha, hb)
    assert np.array_equal(a.read()[0], b.read()[0])


def test_lists_equal_scan_densmap():
    g = oracle_graph(n=2500, dim=30, k=15, n_epochs=60)
    coo = umapcu.CoordinateList(g["row"], g["col"], g["val"], 2500)
    dens = umapcu.DensState.new(umapcu.DensParams(), coo, g["idx"], g["dist"], True)
    adj = umapcu.Adjacency(g["ptr"], g["col"], g["val"])
    p = umapcu.UmapOptimParams(n_epochs=60)
    emb = init_embedding(2500, 2, seed=8)
    a, b = _state(adj, emb, p, True, dens), _state(adj, emb, p, False, dens)
    a.run(0, 60)
    b.run(0, 60)
    assert np.array_equal(a.read()[0], b.read()[0])


def test_lists_equal_scan_warp_per_segment():
    import umapdata.synth as S
    n = 60000  # 1875 segments: above the block-per-segment threshold
    X, _ = S.isotropic_mixture(n, 20, 10, 3)
    idx, dist = umapcu.knn_exact(X, 15)
    graph = umapcu.construct_umap_graph(idx, dist, umapcu.UmapGraphParams(), 40)
    adj = umapcu.coo_to_adjacency_list(graph)
    p = umapcu.UmapOptimParams(n_epochs=40)
    emb = init_embedding(n, 2, seed=5)
    a, b = _state(adj, emb, p, True), _state(adj, emb, p, False)
    assert a.schedule_info()["lists"] and not b.schedule_info()["lists"]
    for first, count in [(0, 25), (25, 15)]:
        a.run(first, count)
        b.run(first, count)
        ya, ma, va, ca = a.read()
        yb, mb, vb, cb = b.read()
        assert np.array_equal(ya, yb) and np.array_equal(ma, mb) and np.array_equal(va, vb)
        assert np.array_equal(ca, cb)
    a.close()
    b.close()


def _one_shot(adj, emb, p, dens=None, seed=9, precompute=True, opt=None):
    y = np.ascontiguousarray(emb.copy())
    old = os.environ.pop("UMAPCU_NO_SCHEDULE_LISTS", None)
    try:
        if not precompute:
            os.environ["UMAPCU_NO_SCHEDULE_LISTS"] = "1"
        umapcu.optimise_embedding_adam_gpu(y, adj, p, dens, seed, 0, umapcu.NEG_REF_HASH,
                                           umapcu.OPT_ADAM if opt is None else opt)
    finally:
        os.environ.pop("UMAPCU_NO_SCHEDULE_LISTS", None)
        if old is not None:
            os.environ["UMAPCU_NO_SCHEDULE_LISTS"] = old
    return y


@pytest.mark.parametrize("opt", ["adam", "sgd"])
def test_one_shot_bitmask_equals_scan(prob, opt):
    """The one-shot call runs its epochs on per-epoch bitmasks of the active
    entries; with the precomputed schedule switched off it scans the
    cursors, and a scanning state gives the same: all three bit-identical."""
    g, adj = prob
    p = umapcu.UmapOptimParams(n_epochs=70)
    o = umapcu.OPT_SGD if opt == "sgd" else umapcu.OPT_ADAM
    emb = init_embedding(3000, 2, seed=12)
    y_bits = _one_shot(adj, emb, p, opt=o)
    y_scan = _one_shot(adj, emb, p, precompute=False, opt=o)
    st = _state(adj, emb, p, False)
    st.run(0, 70, o)
    assert np.array_equal(y_bits, y_scan)
    assert np.array_equal(y_bits, st.read()[0])
    st.close()


def test_one_shot_bitmask_equals_scan_densmap_3d():
    g = oracle_graph(n=2500, dim=30, k=15, n_epochs=60)
    coo = umapcu.CoordinateList(g["row"], g["col"], g["val"], 2500)
    dens = umapcu.DensState.new(umapcu.DensParams(), coo, g["idx"], g["dist"], True)
    adj = umapcu.Adjacency(g["ptr"], g["col"], g["val"])
    p = umapcu.UmapOptimParams(n_epochs=60)
    emb = init_embedding(2500, 3, seed=13)
    assert np.array_equal(_one_shot(adj, emb, p, dens), _one_shot(adj, emb, p, dens, precompute=False))


def test_one_shot_bitmask_warp_per_segment_equals_scan():
    import umapdata.synth as S
    n = 60000  # above the block-per-segment threshold: the warp-per-segment bitmask scan
    X, _ = S.isotropic_mixture(n, 20, 10, 4)
    idx, dist = umapcu.knn_exact(X, 15)
    adj = umapcu.coo_to_adjacency_list(umapcu.construct_umap_graph(idx, dist, umapcu.UmapGraphParams(), 40))
    p = umapcu.UmapOptimParams(n_epochs=40)
    emb = init_embedding(n, 2, seed=14)
    assert np.array_equal(_one_shot(adj, emb, p), _one_shot(adj, emb, p, precompute=False))


def test_split_bitmask_build_equals_scan():
    """Bitmasks of 64 MB or more are built in two launches, epochs 8.. on a
    side stream beside the first epochs, which wait for it once before epoch
    8 (here 200k points, ~4.7 M CSR entries, 150 epochs: ~88 MB). The
    one-shot call and a resident state that switches to the bitmask form
    mid-life (its epochs on another stream) equal the cursor scan bit for
    bit."""
    import torch
    import umapdata.synth as S
    n = 200_000
    X, _ = S.isotropic_mixture(n, 16, 12, 6)
    idx, dist = umapcu.knn_exact(X, 15)
    adj = umapcu.coo_to_adjacency_list(umapcu.construct_umap_graph(idx, dist, umapcu.UmapGraphParams(), 150))
    p = umapcu.UmapOptimParams(n_epochs=150)
    assert 150 * ((int(adj.ptr[-1]) + 31) // 32) >= 16 << 20  # takes the split build
    emb = init_embedding(n, 2, seed=15)
    y_scan = _one_shot(adj, emb, p, precompute=False)
    assert np.array_equal(_one_shot(adj, emb, p), y_scan)
    st = _state(adj, emb, p, False)
    st.set_schedule(umapcu.SCHED_BITS)
    st.set_stream(torch.cuda.current_stream().cuda_stream)
    st.run(0, 150)
    assert np.array_equal(st.read()[0], y_scan)
    st.close()


def test_one_shot_bitmask_hub_segment_equals_scan():
    """A hub with 9000 neighbours puts more than 256 bitmask words into one
    segment: that segment runs the sequential scan on one warp while the
    others are shared by the block's warps; still bit-identical."""
    import scipy.sparse as sp
    g = oracle_graph(n=12000, dim=20, k=10, n_epochs=50)
    n = 12000
    A = sp.csr_matrix((g["val"].astype(np.float32), (g["row"], g["col"])), shape=(n, n))
    hub = sp.csr_matrix((np.full(9000, 0.5, np.float32), (np.zeros(9000, np.int64), np.arange(1, 9001))),
                        shape=(n, n))
    A = A.maximum(hub).maximum(hub.T).tocsr()
    A.sort_indices()
    adj = umapcu.Adjacency(A.indptr.astype(np.uint64), A.indices.astype(np.uint32), A.data.astype(np.float32))
    p = umapcu.UmapOptimParams(n_epochs=50)
    emb = init_embedding(n, 2, seed=15)
    assert np.array_equal(_one_shot(adj, emb, p), _one_shot(adj, emb, p, precompute=False))


def test_one_shot_concurrent_calls_share_the_bitmask_cache(prob):
    """Four threads run the one-shot call at once (ctypes drops the GIL): one
    takes the cached bitmask block, the others allocate their own, and every
    result equals the same call run alone."""
    import threading
    g, adj = prob
    p = umapcu.UmapOptimParams(n_epochs=40)
    embs = [init_embedding(3000, 2, seed=20 + i) for i in range(4)]
    alone = [_one_shot(adj, e, p, seed=30 + i) for i, e in enumerate(embs)]
    outs = [None] * 4

    def work(i):
        y = np.ascontiguousarray(embs[i].copy())
        umapcu.optimise_embedding_adam_gpu(y, adj, p, None, 30 + i, 0, umapcu.NEG_REF_HASH, umapcu.OPT_ADAM)
        outs[i] = y

    for _ in range(2):
        ts = [threading.Thread(target=work, args=(i,)) for i in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        for i in range(4):
            assert np.array_equal(outs[i], alone[i]), i


def test_set_schedule_forms_and_enqueue_are_bit_identical(prob):
    """umapcu_state_set_schedule rebuilds the precomputed schedule in each
    form mid-life (the bench builds the bitmasks inside every timed step);
    enqueue() is run() without the final synchronisation. All forms and
    both calls give identical results."""
    import torch
    g, adj = prob
    p = umapcu.UmapOptimParams(n_epochs=80)
    emb = init_embedding(3000, 2, seed=12)
    st = _state(adj, emb, p, True)
    assert st.schedule_form() == umapcu.SCHED_LISTS
    ref = None
    stream = torch.cuda.current_stream()
    for form in (umapcu.SCHED_SCAN, umapcu.SCHED_BITS, umapcu.SCHED_LISTS, umapcu.SCHED_BITS):
        st.set_schedule(umapcu.SCHED_SCAN)
        st.reset(emb)
        st.set_schedule(form)
        assert st.schedule_form() == form
        st.set_stream(stream.cuda_stream)
        st.enqueue(0, 30)
        st.run(30, 50)
        y = st.read()[0]
        ref = y if ref is None else ref
        assert np.array_equal(y, ref), form
    st.close()


def test_release_cached_and_pool_retention():
    """The memory-hygiene entry points run on a device with the caches in
    use and leave the library working."""
    g = oracle_graph(n=3000, dim=50, k=15, n_epochs=80)
    adj = umapcu.Adjacency(g["ptr"], g["col"], g["val"])
    p = umapcu.UmapOptimParams(n_epochs=40)
    e1 = init_embedding(3000, 2, seed=1)
    e2 = e1.copy()
    umapcu.optimise_embedding_adam_gpu(e1, adj, p, seed=5)
    umapcu.release_cached()
    umapcu.set_pool_retention(False)
    umapcu.optimise_embedding_adam_gpu(e2, adj, p, seed=5)
    umapcu.set_pool_retention(True)
    assert np.array_equal(e1, e2)
    assert umapcu.probe_l2_gather(8 << 20) > 100.0
