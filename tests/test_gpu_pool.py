"""The multi-device placement front ends on the device this run has (needs
a B200): a pool over one device returns the same embeddings as the
single-device server and batch it wraps, and as the single-problem path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")
from umapcu.pool import BatchPool, ServerPool  # noqa: E402


def _problems(count=6):
    import umapdata.synth as S
    out = []
    for i in range(count):
        n = 800 + 300 * i
        X, _ = S.isotropic_mixture(n, 20, 5, seed=40 + i)
        idx, dist = umapcu.knn_exact(X, 15)
        g = umapcu.construct_umap_graph(idx, dist, umapcu.UmapGraphParams(), 100)
        out.append((umapcu.coo_to_adjacency_list(g), umapcu.random_layout(n, 2, 90 + i)))
    return out


def test_pools_on_one_device_match_single_problem_runs():
    probs = _problems()
    p = umapcu.UmapOptimParams(n_epochs=100)
    want = []
    for i, (adj, y0) in enumerate(probs):
        y = y0.copy()
        umapcu.optimise_embedding_adam_gpu(y, adj, p, seed=i)
        want.append(y)
    pool = ServerPool(8 << 30, devices=[0], tick_epochs=10)
    tickets = [pool.submit(y0, adj, p, seed=i) for i, (adj, y0) in enumerate(probs)]
    for i, t in enumerate(tickets):
        assert pool.device_of(t) == 0
        y, lat, q = pool.wait(t)
        assert np.array_equal(y, want[i]), i
    pool.close()
    bp = BatchPool([y0 for _, y0 in probs], [a for a, _ in probs], p, list(range(len(probs))), devices=[0])
    bp.run(2)
    for i in range(len(probs)):
        assert np.array_equal(bp.read(i), want[i]), i
    bp.close()
