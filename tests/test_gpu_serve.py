"""Served form: continuous batching with device-memory admission (needs a
B200). Results must be the same alone and in the mix; admission must respect
the budget and the job limit; failures are injected on the host (cancelled
jobs, a client that never collects, an oversized job, shutdown with work
outstanding) and must leave the other jobs' results unchanged."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")


@pytest.fixture(scope="module")
def pool():
    import umapdata.synth as S
    out = []
    for i, n in enumerate([400, 2600, 1100, 5200, 700, 3300, 1800, 90]):
        X, _ = S.isotropic_mixture(n, 20, 3 + i % 5, seed=300 + i)
        idx, dist = S.exact_knn_cpu(X, 15 if n > 100 else 8)
        g = umapcu.construct_umap_graph(idx, dist, umapcu.UmapGraphParams(), 60)
        out.append((umapcu.coo_to_adjacency_list(g), umapcu.random_layout(n, 2, 400 + i)))
    return out


P60 = umapcu.UmapOptimParams(n_epochs=60) if umapcu else None


def _alone(adj, init, seed, p=None):
    y = init.copy()
    umapcu.optimise_embedding_adam_gpu(y, adj, p or P60, None, seed)
    return y


def test_served_results_equal_alone_with_staggered_arrivals(pool):
    sv = umapcu.UmapServer(budget_bytes=8 << 30, max_jobs=64, tick_epochs=7)
    tickets = []

    def client():
        for k in range(3):
            for i, (adj, init) in enumerate(pool):
                tickets.append((i, k, sv.submit(init, adj, P60, seed=1000 * k + i)))
                time.sleep(0.002 * (i % 3))

    th = threading.Thread(target=client)
    th.start()
    th.join()
    for i, k, t in tickets:
        y, lat, q = sv.wait(t)
        assert lat >= q >= 0
        assert np.array_equal(y, _alone(pool[i][0], pool[i][1], 1000 * k + i)), (i, k)
    st = sv.stats()
    assert st["completed"] == len(tickets) and st["peak_jobs"] > 1  # jobs shared launches
    sv.close()


def test_admission_respects_budget_and_job_limit(pool):
    adj, init = pool[3]
    nnz = int(adj.ptr[-1])
    one = 72 * nnz + 24 * init.shape[0] * 2 + 16 * 60 + (1 << 20)
    sv = umapcu.UmapServer(budget_bytes=2 * one + 1000, max_jobs=3, tick_epochs=10)
    ts = [sv.submit(init, adj, P60, seed=s) for s in range(6)]
    want = {s: _alone(adj, init, s) for s in range(6)}
    for s, t in enumerate(ts):
        y, _, _ = sv.wait(t)
        assert np.array_equal(y, want[s])
    st = sv.stats()
    assert st["peak_bytes"] <= 2 * one + 1000 and st["peak_jobs"] <= 2
    big = umapcu.UmapServer(budget_bytes=one // 2, max_jobs=4)
    with pytest.raises(umapcu.ManifoldsError):  # the job alone exceeds the budget
        big.submit(init, adj, P60)
    big.close()
    sv.close()


def test_host_side_failures_leave_other_jobs_unchanged(pool):
    sv = umapcu.UmapServer(budget_bytes=8 << 30, max_jobs=1, tick_epochs=5)
    t0 = sv.submit(pool[1][1], pool[1][0], P60, seed=5)
    t1 = sv.submit(pool[2][1], pool[2][0], P60, seed=6)  # queued behind t0 (one slot)
    t2 = sv.submit(pool[4][1], pool[4][0], P60, seed=7)
    sv.cancel(t1)
    with pytest.raises(umapcu.Cancelled):
        sv.wait(t1)

    # a client that submits and dies without collecting its result
    def dead_client():
        sv.submit(pool[0][1], pool[0][0], P60, seed=8)

    th = threading.Thread(target=dead_client)
    th.start()
    th.join()
    y0, _, _ = sv.wait(t0)
    y2, _, _ = sv.wait(t2)
    assert np.array_equal(y0, _alone(pool[1][0], pool[1][1], 5))
    assert np.array_equal(y2, _alone(pool[4][0], pool[4][1], 7))
    # shutdown with work outstanding returns promptly
    for s in range(4):
        sv.submit(pool[5][1], pool[5][0], P60, seed=s)
    t = time.time()
    sv.close()
    assert time.time() - t < 30


def test_edgeless_job_fails_alone_in_its_group(pool):
    """A job whose graph has no edges fails with the single build's status;
    jobs admitted in the same group are unaffected."""
    sv = umapcu.UmapServer(budget_bytes=8 << 30, max_jobs=64, tick_epochs=20)
    n = 50
    empty = umapcu.Adjacency(np.zeros(n + 1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.float32))
    ts = [sv.submit(pool[0][1], pool[0][0], P60, seed=11),
          sv.submit(umapcu.random_layout(n, 2, 3), empty, P60, seed=12),
          sv.submit(pool[6][1], pool[6][0], P60, seed=13)]
    y0, _, _ = sv.wait(ts[0])
    with pytest.raises(umapcu.NoGraphEdges):
        sv.wait(ts[1])
    y2, _, _ = sv.wait(ts[2])
    assert np.array_equal(y0, _alone(pool[0][0], pool[0][1], 11))
    assert np.array_equal(y2, _alone(pool[6][0], pool[6][1], 13))
    sv.close()


def test_submit_rejects_malformed_graphs(pool):
    sv = umapcu.UmapServer(budget_bytes=1 << 30, max_jobs=4)
    adj, init = pool[0]
    bad_col = umapcu.Adjacency(adj.ptr.copy(), adj.col.copy(), adj.w.copy())
    bad_col.col[len(bad_col.col) // 2] = init.shape[0]  # one past the last node
    with pytest.raises(umapcu.ManifoldsError):
        sv.submit(init, bad_col, P60)
    bad_ptr = umapcu.Adjacency(adj.ptr.copy(), adj.col, adj.w)
    bad_ptr.ptr[3], bad_ptr.ptr[4] = bad_ptr.ptr[4], bad_ptr.ptr[3] - 1  # not monotone
    with pytest.raises(umapcu.ManifoldsError):
        sv.submit(init, bad_ptr, P60)
    y, _, _ = sv.wait(sv.submit(init, adj, P60, seed=21))  # the server is unaffected
    assert np.array_equal(y, _alone(adj, init, 21))
    sv.close()


def test_snapshot_and_resume_equal_the_uninterrupted_job(pool):
    """A running job's snapshot (embedding, Adam moments, epochs run, read at
    a tick boundary) resumed as a new job gives the uninterrupted job's
    result bit for bit; a job not admitted yet snapshots to the state it was
    submitted with."""
    adj, init = pool[3]
    p = umapcu.UmapOptimParams(n_epochs=3000)
    sv = umapcu.UmapServer(budget_bytes=8 << 30, max_jobs=1, tick_epochs=7)
    ta = sv.submit(init, adj, p, seed=77)
    tb = sv.submit(pool[1][1], pool[1][0], P60, seed=5)  # queued behind ta (one job at a time)
    yb, mb, vb, eb = sv.snapshot(tb)
    assert eb == 0 and np.array_equal(yb, pool[1][1]) and not mb.any() and not vb.any()
    t0 = time.time()
    while sv.poll(ta) != umapcu.UmapServer.RUNNING and time.time() - t0 < 30:
        time.sleep(0.001)
    y, m, v, e = sv.snapshot(ta)
    assert 0 < e < 3000 and e % 7 == 0 and np.isfinite(y).all() and m.any()
    tc = sv.submit_resume(y, adj, p, m, v, e, seed=77)
    ya = sv.wait(ta)[0]
    sv.wait(tb)
    yc = sv.wait(tc)[0]
    assert np.array_equal(yc, ya)
    assert np.array_equal(ya, _alone(adj, init, 77, p))
    with pytest.raises(umapcu.ManifoldsError):
        sv.snapshot(ta)  # collected: unknown ticket
    sv.close()
