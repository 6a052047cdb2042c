"""Batched form (many layouts in one persistent launch) vs the single-problem
path, and the persistent kernel's bounded waits (needs a B200)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")


@pytest.fixture(scope="module")
def problems():
    import umapdata.synth as S
    rng = np.random.default_rng(0)
    sizes = [300, 4700, 800, 33, 2500, 1200, 5000, 64, 900, 3100, 1500, 2000]
    out = []
    for i, n in enumerate(sizes):
        X, _ = S.isotropic_mixture(n, 20, int(rng.integers(3, 8)), seed=100 + i)
        idx, dist = S.exact_knn_cpu(X, 15 if n > 40 else 8)
        g = umapcu.construct_umap_graph(idx, dist, umapcu.UmapGraphParams(), 80)
        out.append((umapcu.coo_to_adjacency_list(g), umapcu.random_layout(n, 2, 200 + i)))
    return out


def _single(adj, init, p, seed):
    y = init.copy()
    umapcu.optimise_embedding_adam_gpu(y, adj, p, None, seed)
    return y


@pytest.mark.parametrize("mode", [1, 2, 0])
def test_batch_equals_single_problem_runs(problems, mode):
    """Each problem's result is the same alone and in the batch, bit for bit:
    the same kernel body, per-problem seeds and node indices."""
    params = [umapcu.UmapOptimParams(n_epochs=80, a=1.5 + 0.05 * (i % 3), b=0.9) for i in range(len(problems))]
    seeds = [7 + 13 * i for i in range(len(problems))]
    B = umapcu.UmapBatch([x[1] for x in problems], [x[0] for x in problems], params, seeds)
    ms = B.run(mode)
    assert ms > 0
    for i, (adj, init) in enumerate(problems):
        want = _single(adj, init, params[i], seeds[i])
        got = B.read(i)
        assert np.array_equal(got, want), i
    # a second run restarts from the initial state and reproduces it
    B.run(mode)
    assert np.array_equal(B.read(3), _single(problems[3][0], problems[3][1], params[3], seeds[3]))
    B.close()


def test_batch_autotune_picks_valid_config(problems):
    B = umapcu.UmapBatch([x[1] for x in problems], [x[0] for x in problems],
                         umapcu.UmapOptimParams(n_epochs=40), list(range(len(problems))))
    cfg = B.autotune()
    assert cfg["mode"] in (1, 2) and cfg["ku"] in (4, 8) and cfg["ctas_per_sm"] in (4, 6, 8)
    B.run(0)
    assert np.isfinite(B.read(0)).all()
    B.close()


def test_persistent_wait_is_bounded(problems):
    """Failure detection without a GPU fault: one problem's epoch barrier can
    never open; its waiting warps give up after the poll limit, the launch
    drains and the host reads UMAPCU_TIMEOUT. The batch stays usable."""
    params = umapcu.UmapOptimParams(n_epochs=30)
    B = umapcu.UmapBatch([x[1] for x in problems], [x[0] for x in problems], params, [1] * len(problems))
    assert B.wait_check(4, 20000) == umapcu.TIMEOUT
    B.run(1)
    got = B.read(2)
    assert np.array_equal(got, _single(problems[2][0], problems[2][1], params, 1))
    B.close()
