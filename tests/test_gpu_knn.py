"""Exact kNN and embedding-quality kernels vs the oracle (needs a B200).
Distances are sequential f32 FMA chains on both sides, so indices and
distances must agree bit for bit; trustworthiness and kNN preservation are
sums of integers, so they agree exactly too."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")
from oracle import oracle as O
from tests._problems import fuzzy_cross_entropy, oracle_graph


def _data(n, dim, seed, clustered=True):
    import umapdata.synth as S
    if clustered:
        X, _ = S.isotropic_mixture(n, dim, 6, seed)
        return np.ascontiguousarray(X, np.float32)
    return np.random.default_rng(seed).normal(size=(n, dim)).astype(np.float32)


@pytest.mark.parametrize("n,dim,k,metric", [(3000, 50, 15, "euclidean"), (1500, 7, 30, "euclidean"),
                                            (2049, 100, 15, "euclidean"), (1000, 33, 8, "cosine"),
                                            (129, 2, 15, "euclidean"), (40, 16, 1, "euclidean")])
def test_knn_bit_exact(n, dim, k, metric):
    X = _data(n, dim, n + dim)
    gi, gd = umapcu.knn_exact(X, k, metric)
    oi, od = O.knn_exact(X, k, metric=umapcu._metric(metric))
    assert np.array_equal(gi.astype(np.uint32), oi)
    assert np.array_equal(gd, od)


def test_knn_duplicates_tie_break_by_index():
    """Exact duplicates (distance 0 ties): ascending index, self excluded."""
    base = _data(200, 10, 5)
    X = np.concatenate([base, base, base[:50]])  # every base point 2-3 times
    gi, gd = umapcu.knn_exact(X, 12)
    oi, od = O.knn_exact(X, 12)
    assert np.array_equal(gi.astype(np.uint32), oi) and np.array_equal(gd, od)
    assert gd[0, 0] == 0.0 and gi[0, 0] == 200  # point 0's twin


def test_knn_matches_reference_convention_and_feeds_the_graph():
    """Squared distances (the ANN backends' convention), self excluded; the
    GPU kNN drives the graph stage exactly like the oracle's kNN."""
    X = _data(2000, 20, 9)
    gi, gd = umapcu.knn_exact(X, 15)
    assert not (gi == np.arange(2000)[:, None]).any()
    j = gi[7, 3]
    assert gd[7, 3] == pytest.approx(float(((X[7].astype(np.float64) - X[j]) ** 2).sum()), rel=1e-5)
    g = umapcu.construct_umap_graph(gi, gd, umapcu.UmapGraphParams(), 200)
    oi, od = O.knn_exact(X, 15)
    (r, c, v), _, _ = O.construct_umap_graph(oi.astype(np.int32), od, 200)
    assert np.array_equal(g.row_indices, r) and np.array_equal(g.col_indices, c)


def test_quality_metrics_equal_oracle_and_sklearn():
    from sklearn.manifold import trustworthiness
    X = _data(2500, 40, 11)
    Y = (X[:, :2] + 0.5 * np.random.default_rng(1).normal(size=(2500, 2))).astype(np.float32)
    ki, _ = O.knn_exact(X, 15)
    q = umapcu.embedding_quality(X, Y, ki.astype(np.int32), 15)
    assert q["trust"] == O.trustworthiness(X, Y, 15)
    assert q["knn_preservation"] == pytest.approx(O.knn_preservation(ki, Y, 15), abs=1e-12)
    unit = 2.0 / (2500 * 15 * (2.0 * 2500 - 45 - 1))
    assert abs(q["trust"] - trustworthiness(X, Y, n_neighbors=15)) <= 50 * unit
    # a query subsample (the large-run protocol): the same sums over those rows
    sub = np.random.default_rng(2).choice(2500, 600, replace=False).astype(np.uint32)
    qs = umapcu.embedding_quality(X, Y, ki.astype(np.int32), 15, queries=sub)
    assert qs["trust"] == O.trustworthiness(X, Y, 15, queries=sub)
    assert qs["knn_preservation"] == pytest.approx(O.knn_preservation(ki, Y, 15, queries=sub), abs=1e-12)


def test_quality_cosine_and_argument_errors():
    X = _data(800, 12, 4)
    Y = X[:, :2].copy()
    q = umapcu.embedding_quality(X, Y, None, 10, dist_metric="cosine")
    assert q["trust"] == O.trustworthiness(X, Y, 10, metric=1) and q["knn_preservation"] is None
    with pytest.raises(umapcu.ManifoldsError):  # sklearn requires k < n / 2
        umapcu.embedding_quality(X[:20], Y[:20], None, 10)
    with pytest.raises(umapcu.ManifoldsError):
        umapcu.knn_exact(X[:10], 10)  # n must exceed k
    with pytest.raises(umapcu.ManifoldsError):
        umapcu.knn_exact(X, 33)  # k <= 32


def test_fuzzy_cross_entropy_matches_f64_reference():
    g = oracle_graph(n=2000, dim=20)
    Y = np.random.default_rng(3).normal(size=(2000, 2)).astype(np.float32)
    coo = umapcu.CoordinateList(g["row"], g["col"], g["val"], 2000)
    a, b = float(np.float32(1.577)), float(np.float32(0.895))  # the ABI takes a, b as f32
    got = umapcu.fuzzy_cross_entropy(coo, Y, a, b)
    want = fuzzy_cross_entropy(g["row"], g["col"], g["val"], Y, a, b)
    assert got == pytest.approx(want, rel=1e-10)
