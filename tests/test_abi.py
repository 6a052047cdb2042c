"""CPU-only checks of the C ABI library: it loads, exports every symbol the
header declares, and its host-only entry points behave (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(umapcu_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import umapcu
    lib = C.CDLL(umapcu.LIB_PATH)
    names = _declared("umapcu.h")
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_checked_library_exports_the_same_symbols():
    import umapcu
    path = os.path.join(os.path.dirname(umapcu.LIB_PATH), "libumapcu_checked.so")
    lib = C.CDLL(path)
    missing = [n for n in _declared("umapcu.h") if not hasattr(lib, n)]
    assert not missing, missing
    lib.umapcu_version.restype = C.c_char_p
    assert b"checked" in lib.umapcu_version()


def test_status_strings_and_version():
    import umapcu
    assert umapcu.version().startswith("umapcu")
    for s in range(10):
        assert umapcu.lib().umapcu_status_string(s)


def test_fit_ab_matches_oracle_bit_exact():
    # UmapOptimParams::fit_params (umap_optimisers.rs:139-209) is host code in
    # the library too; both sides are f32 glibc arithmetic without FMA.
    import umapcu
    from oracle import oracle as O
    for md, sp in [(0.1, 1.0), (0.5, 1.0), (0.01, 2.0), (0.25, 0.5)]:
        a, b = umapcu.fit_params(md, sp)
        ao, bo = O.fit_params(md, sp)
        assert np.float32(a) == np.float32(ao) and np.float32(b) == np.float32(bo)


def test_optim_params_defaults():
    # umap_optimisers.rs:1523-1534 (default_2d) and :1536-1557
    import umapcu
    p = umapcu.UmapOptimParams.default_2d()
    assert (p.a, p.b, p.lr, p.gamma, p.n_epochs, p.neg_sample_rate) == (1.5, 0.9, 1.0, 1.0, 500, 5)
    assert p.min_dist == pytest.approx(0.1)
    q = umapcu.UmapOptimParams.from_min_dist_spread(0.1, 1.0, 1.0, 1.0, 500, 5)
    assert q.a > 0 and q.b > 0 and q.n_epochs == 500 and q.neg_sample_rate == 5


def test_parse_optimiser():
    import umapcu
    assert umapcu.parse_umap_optimiser_gpu("ADAM_GPU") == "adam_gpu"
    assert umapcu.parse_umap_optimiser_gpu("sgd") == "sgd"
    assert umapcu.parse_umap_optimiser_gpu("lbfgs") is None


def test_adjacency_helpers():
    # graph.rs:1566-1602
    import umapcu
    g = umapcu.CoordinateList(np.array([0, 0, 1, 2]), np.array([1, 2, 2, 0]), np.array([0.5, 0.3, 0.8, 0.9]), 3)
    a = umapcu.coo_to_adjacency_list(g)
    assert a.ptr.tolist() == [0, 2, 3, 4] and a.col.tolist() == [1, 2, 2, 0]
    e = umapcu.coo_to_adjacency_list(umapcu.CoordinateList(np.array([], int), np.array([], int), np.array([]), 3))
    assert e.ptr.tolist() == [0, 0, 0, 0]
    b = umapcu.Adjacency.from_lists([[(1, 1.0), (2, 0.5)], [], []])
    assert b.ptr.tolist() == [0, 2, 2, 2] and b.n == 3


def test_dens_is_active_f32():
    # density.rs:244-250, :692-718
    import umapcu
    st = umapcu.DensState(umapcu.DensParams(2.0, 0.3, 0.1), np.zeros(2), np.ones(2), 1.0)
    assert not st.is_active(69, 100) and st.is_active(70, 100) and st.is_active(99, 100)
    assert [st.is_active(e, 200) for e in range(200)].index(True) == 140


def test_bad_args_rejected_without_gpu():
    # argument validation happens before any device work
    import umapcu
    with pytest.raises(umapcu.NoData):
        umapcu.optimise_embedding_adam_gpu(np.zeros((0, 2), np.float32), [], umapcu.UmapOptimParams())
    with pytest.raises(umapcu.ManifoldsError):
        umapcu.optimise_embedding_adam_gpu(np.zeros((3, 2), np.float64), [[], [], []], umapcu.UmapOptimParams())


def test_noalloc_rejects_misaligned_pointers():
    """umapcu_optimise_csr_noalloc refuses device pointers its float2 / float4
    row accesses would fault on, before any CUDA call (so this runs without
    a GPU): the embedding must be 8-byte aligned for n_dim = 2, 16-byte
    aligned for n_dim = 4, the CSR arrays 4-byte aligned."""
    import umapcu
    fn = umapcu.lib().umapcu_optimise_csr_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                   C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]
    cp = umapcu.UmapOptimParams(n_epochs=10)._c()
    good = 1 << 20
    cases = [(good + 4, 2, good, good, good), (good + 8, 4, good, good, good), (good + 2, 3, good, good, good),
             (good, 2, good + 2, good, good), (good, 2, good, good + 1, good), (good, 2, good, good, good + 3)]
    for y, d, off, oth, per in cases:
        rc = fn(C.c_void_p(y), 100, d, C.c_void_p(off), C.c_void_p(oth), C.c_void_p(per), 600, C.byref(cp), 1, 0,
                None)
        assert rc == umapcu.BAD_ARG, (y, d, off, oth, per, rc)
