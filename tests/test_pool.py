"""Placement of the batched and served forms over several devices, on the
host with fake per-device backends (no GPU): the placement policy, failure
isolation (a device that refuses jobs, a cancelled job) and the identity of
every other job's result with its result alone."""
import numpy as np
import pytest

umapcu = pytest.importorskip("umapcu")
from umapcu.pool import BatchPool, ServerPool, lpt_partition  # noqa: E402


def test_lpt_partition_balanced_and_deterministic():
    rng = np.random.default_rng(3)
    w = np.exp(rng.uniform(np.log(500), np.log(50_000), 512))
    a = lpt_partition(w, 8)
    assert a == lpt_partition(w, 8)
    assert sorted(i for b in a for i in b) == list(range(512))
    loads = [w[b].sum() for b in a]
    # LPT is within 4/3 of the optimum; the optimum is at least the mean
    assert max(loads) <= 4.0 / 3.0 * max(w.sum() / 8, w.max())
    assert lpt_partition([5.0], 3) == [[0], [], []]


class FakeServer:
    """Host stand-in for one device's UmapServer: a job's 'result' is a
    deterministic function of its own arguments, so it is the same alone and
    in any mix. refuse: every submit fails like a device error; budget: jobs
    over it fail with CAPACITY."""

    def __init__(self, budget=1 << 40, refuse=False):
        self.budget, self.refuse = budget, refuse
        self.jobs, self.next, self.cancelled = {}, 1, set()

    def submit(self, embd, graph, params, seed=42, sampler=0):
        if self.refuse:
            raise umapcu.CubeclUtilsError(umapcu.CUDA_LAUNCH, "device refused")
        e = np.asarray(embd)
        need = umapcu.server_job_bytes(e.shape[0], e.shape[1], int(graph.col.size), int(params.n_epochs))
        if need > self.budget:
            raise umapcu.ManifoldsError(umapcu.CAPACITY)
        t = self.next
        self.next += 1
        self.jobs[t] = (e.astype(np.float32) * 0.5 + np.float32(seed), need)
        return t

    def poll(self, t):
        return umapcu.UmapServer.DONE

    def cancel(self, t):
        self.cancelled.add(t)

    def wait(self, t):
        y, _ = self.jobs.pop(t)
        if t in self.cancelled:
            raise umapcu.Cancelled(umapcu.CANCELLED)
        return y, 0.001, 0.0

    def stats(self):
        return dict(completed=0, ticks=0, peak_bytes=0, peak_jobs=0)

    def close(self):
        pass


def _job(n, seed):
    rng = np.random.default_rng(seed)
    adj = umapcu.Adjacency.from_lists([[((i + 1) % n, 1.0)] for i in range(n)])
    return rng.uniform(-10, 10, (n, 2)).astype(np.float32), adj


def test_server_pool_places_by_free_budget_and_isolates_failures():
    p = umapcu.UmapOptimParams(n_epochs=50)
    budget = 1 << 30
    backends = [FakeServer(budget), FakeServer(refuse=True), FakeServer(budget)]
    pool = ServerPool(budget, backends=backends)
    jobs = [_job(200 + 37 * i, i) for i in range(12)]
    tickets = [pool.submit(y, a, p, seed=i) for i, (y, a) in enumerate(jobs)]
    # the refusing device is out of the rotation after its first refusal;
    # the others share the jobs by free budget (alternating here)
    assert not pool.healthy[1] and pool.placed[1] == 0
    assert abs(pool.placed[0] - pool.placed[2]) <= 1 and pool.placed[0] + pool.placed[2] == 12
    pool.cancel(tickets[5])
    alone = ServerPool(budget, backends=[FakeServer(budget)])
    for i, t in enumerate(tickets):
        if i == 5:
            with pytest.raises(umapcu.Cancelled):
                pool.wait(t)
            continue
        y, lat, q = pool.wait(t)
        ya, _, _ = alone.wait(alone.submit(jobs[i][0], jobs[i][1], p, seed=i))
        assert np.array_equal(y, ya)
    assert pool.outstanding == [0, 0, 0]


def test_server_pool_passes_over_a_device_without_budget():
    p = umapcu.UmapOptimParams(n_epochs=50)
    y, a = _job(5000, 1)
    need = umapcu.server_job_bytes(5000, 2, int(a.col.size), 50)
    small, big = FakeServer(budget=need // 2), FakeServer(budget=need * 4)
    pool = ServerPool(need * 4, backends=[small, big])
    pool.budget = [need * 8, need * 4]  # the small device advertises more free budget than it has
    t = pool.submit(y, a, p, seed=3)
    assert pool.device_of(t) == 1 and pool.healthy == [True, True]
    pool.wait(t)
    with pytest.raises(umapcu.ManifoldsError):
        ServerPool(need, backends=[FakeServer(budget=need // 2)]).submit(y, a, p)


class FakeBatch:
    def __init__(self, embds, adjs, params, seeds):
        self.y = [np.asarray(e, np.float32) + np.float32(s) for e, s in zip(embds, seeds)]

    def autotune(self):
        return dict(mode=2, ctas_per_sm=0, ku=8)

    def run(self, mode=0):
        return 1.0

    def read(self, i):
        return self.y[i]

    def close(self):
        pass


def test_batch_pool_partition_and_read_back():
    P = 40
    embds = [_job(100 + 10 * i, i)[0] for i in range(P)]
    graphs = [_job(100 + 10 * i, i)[1] for i in range(P)]
    pool = BatchPool(embds, graphs, umapcu.UmapOptimParams(n_epochs=20), list(range(P)), devices=[0, 1, 2],
                     factory=lambda d, e, a, q, s, smp: FakeBatch(e, a, q, s))
    assert sorted(i for b in pool.shares for i in b) == list(range(P))
    assert pool.run() == [1.0, 1.0, 1.0]
    for i in range(P):
        assert np.array_equal(pool.read(i), embds[i] + np.float32(i))


def test_request_placement_least_work_first():
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    owner = bench.place_requests([10, 1, 1, 1, 1, 10, 5], 2)
    assert owner.tolist() == [0, 1, 1, 1, 1, 1, 0]
    rng = np.random.default_rng(1)
    w = rng.integers(1, 100, 2000)
    o = bench.place_requests(w, 4)
    loads = [w[o == k].sum() for k in range(4)]
    assert max(loads) - min(loads) <= w.max()
