"""Spectral initialisation on the device (needs a B200): the Lanczos
eigen-solver against the reference's own known-answer tests
(src/utils/math.rs:790-868) and a dense eigen-decomposition, and the layout
against the reference's contract (src/data/init.rs:876-958, 413-524)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")
from tests._problems import oracle_graph


def _csr(dense):
    n = dense.shape[0]
    ptr, col, val = [0], [], []
    for i in range(n):
        nz = np.nonzero(dense[i])[0]
        col += nz.tolist()
        val += dense[i, nz].tolist()
        ptr.append(len(col))
    return np.array(ptr, np.uint64), np.array(col, np.uint32), np.array(val, np.float64)


def test_smallest_eigenpairs_diagonal_kat():
    # math.rs:816-838: diag(5, 4, 3, 2, 1), the three smallest ~ 1, 2, 3
    ev, vec = umapcu.compute_smallest_eigenpairs_lanczos(*_csr(np.diag([5.0, 4, 3, 2, 1])), 3, 42)
    assert ev.shape == (3,) and vec.shape == (5, 3)
    assert np.allclose(ev, [1.0, 2.0, 3.0], atol=0.1)


def test_smallest_eigenpairs_path_laplacian_kat():
    # math.rs:790-814: the path graph's Laplacian, eigenvalues positive
    L = np.array([[2.0, -1, 0], [-1, 2, -1], [0, -1, 2]])
    ev, vec = umapcu.compute_smallest_eigenpairs_lanczos(*_csr(L), 2, 42)
    assert ev.shape == (2,) and vec.shape == (3, 2) and (ev > 0).all()


def test_smallest_eigenpairs_reproducible_on_tridiagonal():
    # math.rs:840-868 (n = 5000, 2 on the diagonal, -1 off): same seed, same result
    n = 5000
    ptr, col, val = [0], [], []
    for i in range(n):
        for j, x in ((i - 1, -1.0), (i, 2.0), (i + 1, -1.0)):
            if 0 <= j < n:
                col.append(j)
                val.append(x)
        ptr.append(len(col))
    A = (np.array(ptr, np.uint64), np.array(col, np.uint32), np.array(val, np.float64))
    e1, v1 = umapcu.compute_smallest_eigenpairs_lanczos(*A, 3, 42)
    e2, v2 = umapcu.compute_smallest_eigenpairs_lanczos(*A, 3, 42)
    assert np.array_equal(e1, e2) and np.array_equal(v1, v2)
    assert np.isfinite(v1).all() and (e1 > 0).all() and (e1 < 4).all()


def _neg_norm_adjacency(g, n):
    A = np.zeros((n, n))
    np.add.at(A, (g["row"], g["col"]), g["val"].astype(np.float64))
    deg = A.sum(1)
    dis = np.where(deg > 1e-8, 1.0 / np.sqrt(deg), 0.0)
    M = -(dis[:, None] * A * dis[None, :])
    np.fill_diagonal(M, 0.0)
    return M


def test_eigenpairs_match_dense_solver():
    """The reference's step count (4 k + 30) on a 1500-point kNN graph's
    -D^-1/2 A D^-1/2: Ritz values to 1e-3, Ritz vectors of well-separated
    eigenvalues along the dense solver's (|cos| > 0.98)."""
    n = 1500
    g = oracle_graph(n=n, dim=20, k=15, clusters=1, n_epochs=200)
    M = _neg_norm_adjacency(g, n)
    w, V = np.linalg.eigh(M)
    ev, vec = umapcu.compute_smallest_eigenpairs_lanczos(*_csr(M), 3, 7)
    assert np.allclose(ev, w[:3], atol=1e-3), (ev, w[:3])
    # Ritz pairs equal the oracle's restatement of the reference's Lanczos
    # run from the same start vector (same Krylov space; rounding apart)
    from oracle import oracle as O
    ow, oV = O.lanczos_smallest(M, 3, O.splitmix_start(n, 7))
    assert np.allclose(ev, ow, rtol=1e-6, atol=1e-6), (ev, ow)
    for q in range(3):
        sg = np.sign(float(oV[:, q] @ vec[:, q]))
        assert np.abs(vec[:, q] - sg * oV[:, q]).max() < 1e-4, q


def _strip_graph(n, seed=0):
    """kNN fuzzy graph of points uniform on a 3 x 1 strip: the two lowest
    non-trivial modes of -D^-1/2 A D^-1/2 run along the long side and are
    separated from the next by a wide gap (a well-defined 2-D subspace)."""
    import umapdata.synth as S
    from oracle import oracle as O
    X = np.random.default_rng(seed).uniform([0.0, 0.0], [3.0, 1.0], (n, 2)).astype(np.float32)
    idx, dist = S.exact_knn_cpu(X, 15)
    (r, c, v), _, _ = O.construct_umap_graph(idx, dist, 200)
    return dict(row=r, col=c, val=v)


def test_spectral_layout_single_component_contract():
    n = 2000
    g = _strip_graph(n)
    coo = umapcu.CoordinateList(g["row"], g["col"], g["val"], n)
    y = umapcu.spectral_layout(coo, 2, seed=3)
    assert y.shape == (n, 2) and np.isfinite(y).all()
    assert np.abs(y.mean(0)).max() < 1e-3              # centred (noise 1e-4)
    assert abs(np.abs(y).max() - 10.0) < 1e-3          # scaled to SPECTRAL_RANGE
    assert np.array_equal(y, umapcu.spectral_layout(coo, 2, seed=3))  # deterministic
    # against the oracle's restatement of the reference's Lanczos from the
    # same start vector, then the same centring and scaling (the 1e-4 noise
    # aside); each eigenvector's sign is free
    from oracle import oracle as O
    M = _neg_norm_adjacency(g, n)
    _, V = O.lanczos_smallest(M, 3, O.splitmix_start(n, 3))
    raw = V[:, 1:3] - V[:, 1:3].mean(0)
    want = raw * (10.0 / np.abs(raw).max())
    for d in range(2):
        sg = np.sign(float(want[:, d] @ y[:, d]))
        assert np.abs(y[:, d] - sg * want[:, d]).max() < 5e-3, d


def test_spectral_layout_several_components():
    # two copies of a graph side by side: centroids on the simplex (+x, -x),
    # each component spread around its own centroid
    g = oracle_graph(n=800, dim=10, k=10, clusters=1, n_epochs=200)
    r = np.concatenate([g["row"], g["row"] + 800]).astype(np.uint32)
    c = np.concatenate([g["col"], g["col"] + 800]).astype(np.uint32)
    v = np.concatenate([g["val"], g["val"]]).astype(np.float32)
    y = umapcu.spectral_layout(umapcu.CoordinateList(r, c, v, 1600), 2, seed=5)
    assert np.isfinite(y).all() and abs(np.abs(y).max() - 10.0) < 1e-3
    a, b = y[:800].mean(0), y[800:].mean(0)
    assert np.linalg.norm(a - b) > 5.0 and abs(a[1] - b[1]) < 1.0


def test_spectral_layout_components_solved_together_match_oracle():
    """Three components of different sizes (two strips and a 5-point chain)
    go through one batched Lanczos; each strip's placed coordinates must be an
    affine image of the oracle's eigenvectors of that component alone, run
    from the component's own start vector (seed + its label)."""
    from oracle import oracle as O
    sizes = (900, 600)
    parts, off = [], 0
    for i, m in enumerate(sizes):
        g = _strip_graph(m, seed=11 + i)
        parts.append((g["row"] + off, g["col"] + off, g["val"]))
        off += m
    chain = np.arange(off, off + 4, dtype=np.uint32)           # 5 points, too small to solve
    parts.append((np.concatenate([chain, chain + 1]), np.concatenate([chain + 1, chain]), np.ones(8, np.float32)))
    n = off + 5
    r, c, v = (np.concatenate([p[k] for p in parts]) for k in range(3))
    coo = umapcu.CoordinateList(r.astype(np.uint32), c.astype(np.uint32), v.astype(np.float32), n)
    seed = 4
    y = umapcu.spectral_layout(coo, 2, seed=seed)
    assert y.shape == (n, 2) and np.isfinite(y).all() and abs(np.abs(y).max() - 10.0) < 1e-3
    off = 0
    for label, m in enumerate(sizes):
        sl = slice(off, off + m)
        sub = dict(row=parts[label][0] - off, col=parts[label][1] - off, val=parts[label][2])
        _, V = O.lanczos_smallest(_neg_norm_adjacency(sub, m), 3, O.splitmix_start(m, seed + label))
        for d in range(2):
            corr = np.corrcoef(V[:, 1 + d], y[sl, d])[0, 1]
            assert abs(corr) > 0.9999, (label, d, corr)
        off += m
