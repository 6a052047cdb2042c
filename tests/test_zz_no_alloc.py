"""The allocation-free layout entry point (umapcu_optimise_csr_noalloc).

Callers that cannot allocate device memory when they need a layout -- under
a framework that has reserved the device for its own allocator, or with a
device-memory budget fixed at start-up -- use this entry point: its scratch
lives in a fixed device array inside the library. These checks call it
through the C ABI with device buffers the test owns, and compare its
embedding with the allocating entry point's (umapcu_optimise_embedding) on
the same graph, initial embedding and seed, twice in a row (the second call
finds the first call's scratch contents).

This file is collected last so that a run which stops at the first failure
has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")


def _problem():
    import umapdata.synth as S
    X, _ = S.isotropic_mixture(2500, 20, 6, seed=3)
    idx, dist = S.exact_knn_cpu(X, 15)
    g = umapcu.construct_umap_graph(idx, dist, umapcu.UmapGraphParams(), 60)
    return umapcu.coo_to_adjacency_list(g), umapcu.random_layout(2500, 2, 9)


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    adj, init = _problem()
    p = umapcu.UmapOptimParams(n_epochs=60)
    seed = 1234
    want = init.copy()
    umapcu.optimise_embedding_adam_gpu(want, adj, p, seed=seed)

    st = umapcu.UmapGpuState(init, adj, p, None, seed)
    csr = st.csr()
    st.close()
    period = csr["eps"][csr["edge_idx"]].astype(np.float32)
    dev = torch.device("cuda")
    d_off = torch.from_numpy(csr["offsets"].view(np.int32)).to(dev)
    d_other = torch.from_numpy(csr["other"].view(np.int32)).to(dev)
    d_period = torch.from_numpy(period).to(dev)
    cp = p._c()
    fn = umapcu.lib().umapcu_optimise_csr_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                   C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]
    stream = torch.cuda.current_stream()
    for call in range(2):
        d_y = torch.from_numpy(init.copy()).to(dev)
        torch.cuda.synchronize()
        rc = fn(d_y.data_ptr(), init.shape[0], 2, d_off.data_ptr(), d_other.data_ptr(), d_period.data_ptr(),
                period.size, C.byref(cp), seed, umapcu.NEG_REF_HASH, C.c_void_p(stream.cuda_stream))
        assert rc == umapcu.OK, umapcu.lib().umapcu_status_string(rc)
        torch.cuda.synchronize()
        got = d_y.cpu().numpy()
        # same kernel, same arithmetic: agreement within the parity tolerance
        # (1e-5 relative), in practice bit for bit
        assert np.isfinite(got).all()
        assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max(), call


def test_noalloc_rejects_oversized_problem():
    cp = umapcu.UmapOptimParams(n_epochs=10)._c()
    fn = umapcu.lib().umapcu_optimise_csr_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                   C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]
    # 4M entries need 32 MiB of schedule scratch alone: refused before any
    # pointer is touched
    rc = fn(C.c_void_p(16), 1000, 2, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), 4 << 20, C.byref(cp), 1, 0,
            None)
    assert rc == umapcu.CAPACITY
