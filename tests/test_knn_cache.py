"""kNN cache file (CPU only: host I/O of the library) and the oracle's exact
kNN / trustworthiness pinned against independent f64 and sklearn
computations."""
import os

import numpy as np
import pytest

umapcu = pytest.importorskip("umapcu")
from oracle import oracle as O


def _knn(n=300, k=9, seed=0):
    rng = np.random.default_rng(seed)
    return rng.integers(0, n, (n, k)).astype(np.int32), rng.random((n, k)).astype(np.float32)


def test_round_trip_and_header(tmp_path):
    i, d = _knn()
    p = str(tmp_path / "a.knn")
    umapcu.save_knn(p, i, d, "cosine")
    raw = open(p, "rb").read()
    assert raw[:8] == b"UMAPKNN\0" and len(raw) == 48 + 8 * i.size
    i2, d2, m = umapcu.load_knn(p)
    assert np.array_equal(i, i2) and np.array_equal(d, d2) and m == umapcu.METRIC_COSINE


@pytest.mark.parametrize("corrupt", ["payload_bit", "truncate", "extra", "magic", "index_range"])
def test_damaged_files_are_rejected(tmp_path, corrupt):
    i, d = _knn()
    p = str(tmp_path / "b.knn")
    if corrupt == "index_range":
        i = i.copy()
        i[3, 2] = 300  # == n: outside the point set
    umapcu.save_knn(p, i, d)
    b = bytearray(open(p, "rb").read())
    if corrupt == "payload_bit":
        b[48 + 4 * 17] ^= 0x10
    elif corrupt == "truncate":
        b = b[:-4]
    elif corrupt == "extra":
        b += b"\0"
    elif corrupt == "magic":
        b[0] = ord("X")
    open(p, "wb").write(bytes(b))
    with pytest.raises(umapcu.ManifoldsError):
        umapcu.load_knn(p)


def test_missing_file_is_an_error(tmp_path):
    with pytest.raises(umapcu.ManifoldsError):
        umapcu.load_knn(os.path.join(str(tmp_path), "none.knn"))


@pytest.mark.parametrize("n,dim,k,seed", [(400, 20, 15, 0), (257, 7, 5, 1), (300, 50, 30, 2)])
def test_oracle_knn_matches_f64_bruteforce(n, dim, k, seed):
    """The restatement's neighbour sets equal an independent f64 brute force
    (no near ties at these sizes: the k-th and (k+1)-th f64 distances differ
    by far more than f32 rounding)."""
    X = np.random.default_rng(seed).normal(size=(n, dim)).astype(np.float32)
    idx, dist = O.knn_exact(X, k)
    D = ((X[:, None, :].astype(np.float64) - X[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(D, np.inf)
    ref = np.argsort(D, axis=1, kind="stable")[:, :k]
    assert np.array_equal(idx, ref)
    assert np.allclose(dist, np.take_along_axis(D, ref, 1), rtol=1e-5)


def test_oracle_cosine_matches_f64():
    X = np.random.default_rng(3).normal(size=(300, 12)).astype(np.float32)
    idx, dist = O.knn_exact(X, 10, metric=1)
    U = X.astype(np.float64) / np.linalg.norm(X.astype(np.float64), axis=1, keepdims=True)
    D = 1.0 - U @ U.T
    np.fill_diagonal(D, np.inf)
    ref = np.argsort(D, axis=1, kind="stable")[:, :10]
    assert np.array_equal(idx, ref)
    assert np.allclose(dist, np.take_along_axis(D, ref, 1), atol=1e-6)


def test_oracle_ties_break_by_index():
    X = np.zeros((40, 3), np.float32)  # every distance is 0
    idx, dist = O.knn_exact(X, 5)
    assert (dist == 0).all()
    for q in range(40):
        assert idx[q].tolist() == [p for p in range(40) if p != q][:5]


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_trustworthiness_matches_sklearn(seed):
    from sklearn.manifold import trustworthiness
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(500, 30)).astype(np.float32)
    Y = (X[:, :2] + 0.3 * rng.normal(size=(500, 2))).astype(np.float32)
    # sklearn ranks on f64 distances, the restatement on f32 FMA chains: a
    # near tie may swap, moving one rank by one; allow ten such swaps
    unit = 2.0 / (500 * 15 * (2.0 * 500 - 3 * 15 - 1))
    assert abs(O.trustworthiness(X, Y, 15) - trustworthiness(X, Y, n_neighbors=15)) <= 10 * unit


def test_numpy_reader_and_writer_match_the_library(tmp_path):
    """umapdata.knn_cache (NumPy, no CUDA library) reads what umapcu_knn_save
    writes and writes what umapcu_knn_load reads, byte for byte."""
    from umapdata import knn_cache
    i, d = _knn(n=257, k=7, seed=3)
    a, b = str(tmp_path / "lib.knn"), str(tmp_path / "np.knn")
    umapcu.save_knn(a, i, d)
    knn_cache.save(b, i, d)
    assert open(a, "rb").read() == open(b, "rb").read()
    i2, d2, m = knn_cache.load(a)
    assert np.array_equal(i, i2) and np.array_equal(d, d2) and m == knn_cache.METRIC_EUCLIDEAN_SQ
    i3, d3, _ = umapcu.load_knn(b)
    assert np.array_equal(i, i3) and np.array_equal(d, d3)
    assert knn_cache.header(b) == (257, 7, 0)


@pytest.mark.parametrize("corrupt", ["payload_bit", "truncate", "extra", "magic", "index_range"])
def test_numpy_reader_rejects_damaged_files(tmp_path, corrupt):
    from umapdata import knn_cache
    i, d = _knn()
    if corrupt == "index_range":
        i = i.copy()
        i[3, 2] = 300
    p = str(tmp_path / "c.knn")
    knn_cache.save(p, i, d)
    b = bytearray(open(p, "rb").read())
    if corrupt == "payload_bit":
        b[48 + 4 * 17] ^= 0x10
    elif corrupt == "truncate":
        b = b[:-4]
    elif corrupt == "extra":
        b += b"\0"
    elif corrupt == "magic":
        b[0] = ord("X")
    open(p, "wb").write(bytes(b))
    with pytest.raises(ValueError):
        knn_cache.load(p)


def test_random_layout_streams_agree():
    import umapdata.synth as S
    assert np.array_equal(S.random_layout(1000, 2, 17), umapcu.random_layout(1000, 2, 17))
