"""densMAP on the device vs the oracle (needs a B200).

Tolerances follow the reference's own kernel-vs-mirror tests
(umap_optimiser_gpu.rs:1902-1993): radii and weights 1e-5, the density
gradient 1e-4 (here relative to the largest gradient component).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._problems import init_embedding

pytestmark = pytest.mark.gpu

umapcu = pytest.importorskip("umapcu")


@pytest.fixture(scope="module")
def dens_problem():
    import umapdata.synth as S
    X, lab = S.variable_density_mixture(3000, 30, 8, seed=4)
    idx, dist = S.exact_knn_cpu(X, 30)
    (r, c, v), _, _ = O.construct_umap_graph(idx, dist, 200)
    return dict(X=X, lab=lab, idx=idx, dist=dist, row=r, col=c, val=v, ptr=O.coo_to_adj_ptr(3000, r))


def test_dens_state_parity(dens_problem):
    # DensState::new (density.rs:181-201) on the device vs the oracle
    d = dens_problem
    g = umapcu.CoordinateList(d["row"], d["col"], d["val"], 3000)
    st = umapcu.DensState.new(umapcu.DensParams(), g, d["idx"], d["dist"], True)
    ok, ref = O.dens_state_new(3000, d["row"], d["col"], d["val"], d["idx"], d["dist"], True)
    assert ok == O.OK
    assert np.abs(st.r - ref["r"]).max() <= 1e-5
    assert np.abs(st.mu_sum - ref["mu_sum"]).max() <= 1e-6 * np.abs(ref["mu_sum"]).max()
    assert st.mu_tot == pytest.approx(float(ref["mu_tot"]), rel=1e-6)


def test_dens_state_degenerate(dens_problem):
    # density.rs:625-632: constant radii -> DegenerateLocalRadii
    g = umapcu.CoordinateList(np.array([0, 1], np.uint32), np.array([1, 0], np.uint32),
                              np.array([1.0, 1.0], np.float32), 2)
    with pytest.raises(umapcu.DegenerateLocalRadii):
        umapcu.DensState.new(umapcu.DensParams(), g, [[1], [0]], [[4.0], [4.0]], True)


def _dens_dict(st):
    return {"r": st.r, "lambda": st.params.lambda_, "frac": st.params.frac, "var_shift": st.params.var_shift,
            "mu_tot": st.mu_tot}


def test_dens_radii_weights_and_gradient(dens_problem):
    """umap_dens_radii + umap_dens_weights + the density gradient of
    umap_grad_accum (:769-798) vs the oracle's mirrors, one active epoch with
    the reference's negatives injected."""
    d = dens_problem
    n = 3000
    g = umapcu.CoordinateList(d["row"], d["col"], d["val"], n)
    dens = umapcu.DensState.new(umapcu.DensParams(2.0, 1.0, 0.1), g, d["idx"], d["dist"], True)
    p = umapcu.UmapOptimParams(n_epochs=200)
    adj = umapcu.Adjacency(d["ptr"], d["col"], d["val"])
    y = init_embedding(n, 2, seed=21) * 0.3
    st = umapcu.UmapGpuState(y, adj, p, dens, seed=5)
    stt, csr = O.csr_from_graph(n, d["ptr"], d["col"], d["val"])
    # radii / weights / coefficient from the current embedding
    got = st.dens_update()
    re, phi = O.dens_radii(y, csr, p.a, p.b)
    w, coeff = O.dens_weights(dens.r, re, dens.params.var_shift, dens.params.lambda_, np.float32(dens.mu_tot))
    assert np.abs(got["re"] - re).max() <= 1e-5 * max(1.0, np.abs(re).max())
    assert np.abs(got["phi_sum"] - phi).max() <= 1e-5 * np.abs(phi).max()
    assert np.abs(got["weight"] - w).max() <= 1e-5 * max(1.0, np.abs(w).max())
    assert got["coeff"] == pytest.approx(float(coeff), rel=1e-5)
    # epoch 0 fires nothing; at epoch 1 the density term is live (frac = 1)
    st.epoch_debug(0)
    cursor = csr["eps"].copy()
    O.schedule_update(csr["eps"], cursor, 0)
    inj = np.random.default_rng(2).integers(0, n, (2 * csr["n_edges"], 5)).astype(np.uint32)
    gg, hu = st.epoch_debug(1, injected=inj)
    dref = {"re": re, "phi_sum": phi, "weight": w, "coeff": coeff}
    go, huo = O.grad_accum(y, csr, cursor, 1, 5, 5, p.a, p.b, p.gamma, dens=dref, injected=inj)
    go_plain, _ = O.grad_accum(y, csr, cursor, 1, 5, 5, p.a, p.b, p.gamma, injected=inj)
    assert (hu == huo).all()
    assert np.abs(go - go_plain).max() > 1e-6  # the density term is present
    assert np.abs(gg - go).max() <= 1e-4 * np.abs(go).max()


def _log_radius_corr(X, Y, row, col, val, a, b):
    """Pearson correlation of the original and embedding log local radii."""
    n = X.shape[0]
    d2x = ((X[row].astype(np.float64) - X[col]) ** 2).sum(1)
    d2y = ((Y[row].astype(np.float64) - Y[col]) ** 2).sum(1)
    w = val.astype(np.float64)
    ro = np.log(1e-8 + np.bincount(row, w * d2x, n) / np.maximum(np.bincount(row, w, n), 1e-12))
    phi = 1.0 / (1.0 + a * d2y ** b)
    re = np.log(1e-8 + np.bincount(row, phi * d2y, n) / np.maximum(np.bincount(row, phi, n), 1e-12))
    return float(np.corrcoef(ro, re)[0, 1])


def test_densmap_full_run_raises_radius_correlation(dens_problem):
    """densmap_tests.rs:259-294, densmap_gpu_tests.rs:315-357: the density term
    raises the log-radius correlation; GPU and the oracle's restatement of
    the reference's GPU optimiser agree within 0.15."""
    d = dens_problem
    n = 3000
    g = umapcu.CoordinateList(d["row"], d["col"], d["val"], n)
    params = umapcu.UmapParamsGpu(k=30, optim_params=umapcu.UmapOptimParams(n_epochs=200))
    plain = umapcu.umap_gpu(d["idx"], d["dist"], params, seed=8).T
    dm = umapcu.densmap_gpu(d["idx"], d["dist"], params, umapcu.DensParams(), seed=8).T
    p = params.optim_params
    c_plain = _log_radius_corr(d["X"], plain, d["row"], d["col"], d["val"], p.a, p.b)
    c_dm = _log_radius_corr(d["X"], dm, d["row"], d["col"], d["val"], p.a, p.b)
    assert c_dm > c_plain + 0.05, (c_plain, c_dm)
    dens = umapcu.DensState.new(umapcu.DensParams(), g, d["idx"], d["dist"], True)
    st, yo = O.optimise_adam_gpu(umapcu.random_layout(n, 2, 8), n, d["ptr"], d["col"], d["val"], p.as_dict(), 8,
                                 _dens_dict(dens))
    c_or = _log_radius_corr(d["X"], yo, d["row"], d["col"], d["val"], p.a, p.b)
    assert c_dm > 0.5 and abs(c_dm - c_or) < 0.15, (c_dm, c_or)


def test_densmap_lambda_zero_is_umap(dens_problem):
    # densmap_tests.rs:218-256 / densmap_gpu_tests.rs:171-215: lambda = 0 is
    # plain UMAP (here bit for bit: the density kernels never run)
    d = dens_problem
    params = umapcu.UmapParamsGpu(k=30, optim_params=umapcu.UmapOptimParams(n_epochs=60))
    plain = umapcu.umap_gpu(d["idx"], d["dist"], params, seed=3)
    dm = umapcu.densmap_gpu(d["idx"], d["dist"], params, umapcu.DensParams(0.0, 0.3, 0.1), seed=3)
    assert (plain == dm).all()
