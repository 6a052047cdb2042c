"""Parity with the oracle at the benchmark workloads' full sizes (needs a
B200): C1 10k x 50 (k = 15, 500 epochs), C3 200k x 30 (k = 30, densMAP),
C2 1M x 50 (k = 15, 200 epochs), from the exact kNN of their seeded data.

Bars (the hot path's parity contract): edge index structure bit-exact;
sigma, rho and edge weights within 1e-6 relative (graph.rs:499-565,
:585-853); the optimiser CSR (UmapCsrGraph::from_graph,
umap_optimiser_gpu.rs:132-209) bit-exact; the densMAP constant state
(density.rs:181-201) at the reference's own bars (radii 1e-5, sums 1e-6).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._problems import config_oracle_graph

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")


@pytest.mark.parametrize("name", ["c1", "c3", "c2"])
def test_graph_parity_at_benchmark_size(name):
    g = config_oracle_graph(name)
    G, sig, rho = umapcu.construct_umap_graph(g["idx"], g["dist"], n_epochs=g["n_epochs"], return_sigma_rho=True)
    assert (rho == g["rho"]).all()
    srel = np.abs(sig.astype(np.float64) - g["sigma"]) / np.abs(g["sigma"].astype(np.float64))
    assert srel.max() <= 1e-6, srel.max()
    assert G.row_indices.size == g["row"].size, (G.row_indices.size, g["row"].size)
    assert (G.row_indices == g["row"]).all() and (G.col_indices == g["col"]).all()
    wrel = np.abs(G.values.astype(np.float64) - g["val"]) / g["val"].astype(np.float64)
    assert wrel.max() <= 1e-6, wrel.max()


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_optimiser_csr_parity_at_benchmark_size(name):
    g = config_oracle_graph(name)
    n = g["n"]
    adj = umapcu.Adjacency(g["ptr"], g["col"], g["val"])
    st = umapcu.UmapGpuState(np.zeros((n, 2), np.float32), adj, umapcu.UmapOptimParams(n_epochs=g["n_epochs"]))
    st.set_schedule(umapcu.SCHED_SCAN)
    csr = st.csr()
    st.close()
    stt, ref = O.csr_from_graph(n, g["ptr"], g["col"], g["val"])
    assert stt == O.OK and csr["n_edges"] == ref["n_edges"]
    for key in ("offsets", "edge_idx", "other", "eps", "mu"):
        assert np.array_equal(csr[key], ref[key]), key


def test_dens_state_parity_at_c3():
    g = config_oracle_graph("c3")
    n = g["n"]
    coo = umapcu.CoordinateList(g["row"], g["col"], g["val"], n)
    st = umapcu.DensState.new(umapcu.DensParams(), coo, g["idx"], g["dist"], True)
    ok, ref = O.dens_state_new(n, g["row"], g["col"], g["val"], g["idx"], g["dist"], True)
    assert ok == O.OK
    assert np.abs(st.r - ref["r"]).max() <= 1e-5
    rel = np.abs(st.mu_sum.astype(np.float64) - ref["mu_sum"]) / np.abs(ref["mu_sum"].astype(np.float64))
    assert rel.max() <= 1e-6, rel.max()
    assert st.mu_tot == pytest.approx(float(ref["mu_tot"]), rel=1e-6)
