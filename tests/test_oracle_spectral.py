"""The oracle's restatement of the reference's Lanczos eigen-solver
(oracle.lanczos_smallest) pinned to the reference's own known-answer tests
(src/utils/math.rs:790-868) and to a dense solver (CPU only)."""
import numpy as np

from oracle import oracle as O


def test_diagonal_kat():
    w, V = O.lanczos_smallest(np.diag([5.0, 4, 3, 2, 1]), 3, O.splitmix_start(5, 42))
    assert np.allclose(w, [1.0, 2.0, 3.0], atol=0.1) and V.shape == (5, 3)


def test_path_laplacian_kat():
    L = np.array([[2.0, -1, 0], [-1, 2, -1], [0, -1, 2]])
    w, V = O.lanczos_smallest(L, 2, O.splitmix_start(3, 42))
    assert w.shape == (2,) and (w > 0).all()


def test_converges_to_dense_eigenpairs_when_the_space_is_full():
    rng = np.random.default_rng(0)
    A = rng.normal(size=(40, 40))
    A = A + A.T
    w, V = O.lanczos_smallest(A, 3, O.splitmix_start(40, 1))  # 42 steps >= n: exact
    dw, dV = np.linalg.eigh(A)
    assert np.allclose(w, dw[:3], atol=1e-8)
    for q in range(3):
        assert abs(abs(float(V[:, q] @ dV[:, q])) - 1.0) < 1e-8
