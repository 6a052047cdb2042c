"""umapcu: B200 (sm_100a) UMAP hot path behind manifolds-rs's interface.

Python mirror of the reference's UMAP / densMAP entry points and its
"adam_gpu" optimiser slot, calling the CUDA library ``libumapcu.so`` through
its C ABI (``include/umapcu.h``). Names, argument meaning and error behaviour
follow manifolds-rs (paths relative to the crate root):

* ``UmapOptimParams``        src/training/umap_optimisers.rs:24-234
* ``UmapGraphParams``        src/data/graph.rs:30-61
* ``DensParams/DensState``   src/utils/density.rs:69-251
* ``smooth_knn_dist``        src/data/graph.rs:499-565
* ``construct_umap_graph``   src/lib.rs:249-316 (graph stage :296-306)
* ``coo_to_adjacency_list``  src/data/graph.rs:709-758
* ``UmapGpuState``           src/training/umap_optimiser_gpu.rs:278-453
* ``optimise_embedding_adam_gpu``  src/training/umap_optimiser_gpu.rs:1302-1369
* ``umap_gpu / densmap_gpu`` src/lib.rs:3465-3708, :3829-3851 (precomputed kNN)

There is no CPU fallback: importing this package on a machine without the
built library raises, and every compute call runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("UMAPCU_LIB") or os.path.join(_HERE, "libumapcu.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"umapcu: CUDA library not built ({LIB_PATH} missing); run `make -C manifolds-rs_b200` "
        "or __graft_entry__.build()")

_lib = C.CDLL(LIB_PATH)

# ------------------------------------------------------------------ errors

OK, NO_DATA, NO_GRAPH_EDGES, DEGENERATE_LOCAL_RADII = 0, 1, 2, 3
CUDA_ALLOC, CUDA_LAUNCH, TIMEOUT, BAD_ARG, NO_DEVICE, CAPACITY, CANCELLED = 4, 5, 6, 7, 8, 9, 10

OPT_ADAM, OPT_SGD = 0, 1
NEG_REF_HASH, NEG_PHILOX = 0, 1
SCHED_SCAN, SCHED_BITS, SCHED_LISTS = 0, 1, 2


class ManifoldsError(RuntimeError):
    """Mirror of manifolds-rs's ManifoldsError (src/errors.rs:7-118)."""

    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = _lib.umapcu_status_string(status).decode()
        super().__init__(f"{msg}{': ' + what if what else ''} (status {status})")


class NoData(ManifoldsError):
    pass


class NoGraphEdges(ManifoldsError):
    pass


class DegenerateLocalRadii(ManifoldsError):
    pass


class CubeclUtilsError(ManifoldsError):
    """Device-side failure (allocation, launch, bounded wait); the reference's
    CubeclUtilsError variant (src/errors.rs:54)."""


class Cancelled(ManifoldsError):
    """A served job was cancelled or its server shut down."""


_ERR = {NO_DATA: NoData, NO_GRAPH_EDGES: NoGraphEdges, DEGENERATE_LOCAL_RADII: DegenerateLocalRadii,
        CUDA_ALLOC: CubeclUtilsError, CUDA_LAUNCH: CubeclUtilsError, TIMEOUT: CubeclUtilsError,
        NO_DEVICE: CubeclUtilsError, CANCELLED: Cancelled}


def _check(st: int, what: str = ""):
    if st != OK:
        raise _ERR.get(st, ManifoldsError)(st, what)


# ------------------------------------------------------------------ ABI

class _OptimParams(C.Structure):
    _fields_ = [("a", C.c_float), ("b", C.c_float), ("lr", C.c_float), ("gamma", C.c_float),
                ("n_epochs", C.c_uint32), ("neg_sample_rate", C.c_uint32), ("min_dist", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float)]


class _GraphParams(C.Structure):
    _fields_ = [("bandwidth", C.c_float), ("local_connectivity", C.c_float), ("mix_weight", C.c_float)]


class _Dens(C.Structure):
    _fields_ = [("lambda_", C.c_float), ("frac", C.c_float), ("var_shift", C.c_float),
                ("r", C.c_void_p), ("mu_sum", C.c_void_p), ("mu_tot", C.c_float)]


_vp = C.c_void_p
_u32, _u64, _f32, _i32 = C.c_uint32, C.c_uint64, C.c_float, C.c_int

_lib.umapcu_status_string.restype = C.c_char_p
_lib.umapcu_status_string.argtypes = [_i32]
_lib.umapcu_version.restype = C.c_char_p
_SIGS = {
    "umapcu_fit_ab": [_f32, _f32, _vp, _vp],
    "umapcu_smooth_knn_dist": [_vp, _u32, _u32, _f32, _f32, _u32, _vp, _vp],
    "umapcu_construct_umap_graph": [_vp, _vp, _u32, _u32, _vp, _u32, _u64, _vp, _vp, _vp, _vp, _vp, _vp],
    "umapcu_dens_state_new": [_u32, _u64, _vp, _vp, _vp, _vp, _vp, _u32, _i32, _vp, _vp, _vp],
    "umapcu_optimise_embedding": [_vp, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _u64, _u32, _u32, _i32],
    "umapcu_state_create": [_vp, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _u64, _u32, _vp],
    "umapcu_state_sizes": [_vp, _vp, _vp],
    "umapcu_state_read_csr": [_vp, _vp, _vp, _vp, _vp, _vp],
    "umapcu_state_run": [_vp, _u32, _u32, _u32],
    "umapcu_state_epoch_debug": [_vp, _u32, _u32, _vp, _vp, _vp],
    "umapcu_state_read": [_vp, _vp, _vp, _vp, _vp],
    "umapcu_state_write": [_vp, _vp, _vp, _vp],
    "umapcu_state_dens_update": [_vp, _vp, _vp, _vp, _vp, _vp],
    "umapcu_adam_update": [_vp, _vp, _vp, _vp, _vp, _u32, _u32, _vp, _u32],
    "umapcu_edge_schedule_update": [_vp, _vp, _u64, _u32],
    "umapcu_sample_negatives": [_u32, _u64, _u32, _u32, _u32, _u32, _u32, _u32, _vp],
    "umapcu_state_reset": [_vp, _vp],
    "umapcu_state_set_stream": [_vp, _vp],
    "umapcu_state_run_profiled": [_vp, _u32, _u32, _u32, _vp, _vp],
    "umapcu_state_set_precise_pow": [_vp, _i32],
    "umapcu_batch_create": [_u32, _vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _u32, _vp],
    "umapcu_batch_autotune": [_vp, _vp, _vp, _vp],
    "umapcu_batch_run": [_vp, _u32, _vp],
    "umapcu_batch_read": [_vp, _u32, _vp],
    "umapcu_batch_wait_check": [_vp, _u32, _u32],
    "umapcu_server_create": [_u64, _u32, _u32, _u32, _vp],
    "umapcu_server_submit": [_vp, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _u64, _u32, _vp],
    "umapcu_server_poll": [_vp, _u64, _vp],
    "umapcu_server_cancel": [_vp, _u64],
    "umapcu_server_wait": [_vp, _u64, _vp, _vp, _vp],
    "umapcu_server_stats": [_vp, _vp, _vp, _vp, _vp],
    "umapcu_eval_pow": [_vp, _u32, _f32, _i32, _vp],
    "umapcu_knn_exact": [_vp, _u32, _u32, _u32, _u32, _vp, _vp],
    "umapcu_state_schedule_info": [_vp, _vp, _vp, _vp],
    "umapcu_smallest_eigenpairs": [_u32, _vp, _vp, _vp, _u32, _u64, _vp, _vp, _vp],
    "umapcu_spectral_layout": [_vp, _vp, _vp, _u64, _u32, _u32, _u64, _f32, _vp],
    "umapcu_knn_exact_dev": [_vp, _u32, _u32, _vp, _u32, _u32, _u32, _vp, _vp, _vp],
    "umapcu_embedding_quality": [_vp, _u32, _u32, _vp, _u32, _vp, _u32, _u32, _vp, _u32, _u32, _vp, _vp],
    "umapcu_fuzzy_cross_entropy": [_vp, _vp, _vp, _u64, _vp, _u32, _u32, _f32, _f32, _vp],
    "umapcu_knn_save": [C.c_char_p, _u32, _u32, _u32, _vp, _vp],
    "umapcu_knn_load_header": [C.c_char_p, _vp, _vp, _vp],
    "umapcu_knn_load": [C.c_char_p, _u32, _u32, _vp, _vp],
    "umapcu_state_set_schedule": [_vp, _u32],
    "umapcu_state_enqueue": [_vp, _u32, _u32, _u32],
    "umapcu_state_schedule_form": [_vp, _vp],
    "umapcu_set_pool_retention": [_i32],
    "umapcu_release_cached": [],
    "umapcu_probe_l2_gather": [_u64, _vp],
    "umapcu_device_count": [_vp],
    "umapcu_server_job_bytes": [_u32, _u32, _u64, _u32, _vp],
    "umapcu_server_snapshot": [_vp, _u64, _vp, _vp, _vp, _vp],
    "umapcu_server_submit_resume": [_vp, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _u64, _u32, _vp, _vp, _u32, _vp],
    "umapcu_set_device": [_i32],
}
for _name, _args in _SIGS.items():
    _fn = getattr(_lib, _name)
    _fn.argtypes = _args
    _fn.restype = _i32
_lib.umapcu_state_destroy.argtypes = [_vp]
_lib.umapcu_state_destroy.restype = None
_lib.umapcu_batch_destroy.argtypes = [_vp]
_lib.umapcu_batch_destroy.restype = None
_lib.umapcu_server_destroy.argtypes = [_vp]
_lib.umapcu_server_destroy.restype = None


def lib():
    """The loaded C library (ctypes.CDLL)."""
    return _lib


def version() -> str:
    return _lib.umapcu_version().decode()


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ------------------------------------------------------------------ params

@dataclass
class UmapOptimParams:
    """UmapOptimParams<f32> (src/training/umap_optimisers.rs:24-45)."""
    a: float = 1.5
    b: float = 0.9
    lr: float = 1.0
    gamma: float = 1.0
    n_epochs: int = 500
    neg_sample_rate: int = 5
    min_dist: float = 0.1
    beta1: float = 0.5
    beta2: float = 0.9
    eps: float = 1e-7

    @classmethod
    def default_2d(cls) -> "UmapOptimParams":
        """umap_optimisers.rs:56-69 (UMAP_BETA1/2, EPS: training/mod.rs:15-24)."""
        return cls()

    @classmethod
    def from_min_dist_spread(cls, min_dist, spread, lr=None, gamma=None, n_epochs=None,
                             neg_sample_rate=None, beta1=None, beta2=None, eps=None):
        """umap_optimisers.rs:89-122: a, b fitted by fit_params (:139-209)."""
        a, b = fit_params(min_dist, spread)
        return cls(a=a, b=b, lr=1.0 if lr is None else lr, gamma=1.0 if gamma is None else gamma,
                   n_epochs=500 if n_epochs is None else n_epochs,
                   neg_sample_rate=5 if neg_sample_rate is None else neg_sample_rate,
                   min_dist=min_dist, beta1=0.5 if beta1 is None else beta1,
                   beta2=0.9 if beta2 is None else beta2, eps=1e-7 if eps is None else eps)

    def _c(self) -> _OptimParams:
        return _OptimParams(self.a, self.b, self.lr, self.gamma, int(self.n_epochs), int(self.neg_sample_rate),
                            self.min_dist, self.beta1, self.beta2, self.eps)

    def as_dict(self):
        return dict(a=self.a, b=self.b, lr=self.lr, gamma=self.gamma, n_epochs=self.n_epochs,
                    neg_sample_rate=self.neg_sample_rate, min_dist=self.min_dist, beta1=self.beta1,
                    beta2=self.beta2, eps=self.eps)


def fit_params(min_dist: float, spread: float):
    """UmapOptimParams::fit_params (umap_optimisers.rs:139-209), f32."""
    a, b = C.c_float(), C.c_float()
    _check(_lib.umapcu_fit_ab(min_dist, spread, C.byref(a), C.byref(b)))
    return a.value, b.value


@dataclass
class UmapGraphParams:
    """UmapGraphParams<f32> (src/data/graph.rs:30-61)."""
    bandwidth: float = 1e-5
    local_connectivity: float = 1.0
    mix_weight: float = 1.0


def parse_umap_optimiser_gpu(s: str) -> Optional[str]:
    """parse_umap_optimiser_gpu (umap_optimiser_gpu.rs:44-52). Only the GPU
    optimisers are served here: "adam_gpu" (default) and "sgd" (GPU SGD)."""
    s = s.lower()
    return s if s in ("adam_gpu", "sgd") else None


# ------------------------------------------------------------------ graph

@dataclass
class CoordinateList:
    """COO graph (src/data/structures.rs:22-59)."""
    row_indices: np.ndarray
    col_indices: np.ndarray
    values: np.ndarray
    n_samples: int


@dataclass
class Adjacency:
    """The reference's Vec<Vec<(usize, T)>> adjacency as row pointers:
    row i = (col[ptr[i]:ptr[i+1]], w[ptr[i]:ptr[i+1]])."""
    ptr: np.ndarray
    col: np.ndarray
    w: np.ndarray

    @property
    def n(self) -> int:
        return self.ptr.size - 1

    @classmethod
    def from_lists(cls, graph):
        ptr = np.zeros(len(graph) + 1, np.uint64)
        ptr[1:] = np.cumsum([len(r) for r in graph])
        col = np.array([j for r in graph for j, _ in r], np.uint32)
        w = np.array([w for r in graph for _, w in r], np.float32)
        return cls(ptr, col, w)


def smooth_knn_dist(dist, k=None, local_connectivity=1.0, bandwidth=1e-5, n_iter=64):
    """graph.rs:499-565 on the GPU. dist [n, k] -> (sigmas[n], rhos[n])."""
    d = _c(dist, np.float32)
    n, kk = d.shape
    if k is not None and k != kk:
        raise ManifoldsError(BAD_ARG, "k must equal the row length")
    sig = np.empty(n, np.float32)
    rho = np.empty(n, np.float32)
    _check(_lib.umapcu_smooth_knn_dist(_p(d), n, kk, local_connectivity, bandwidth, n_iter, _p(sig), _p(rho)))
    return sig, rho


def construct_umap_graph(knn_indices, knn_dists, umap_params: UmapGraphParams = None, n_epochs: int = 500,
                         return_sigma_rho=False):
    """Graph stage of construct_umap_graph (src/lib.rs:296-306) on the GPU:
    smooth_knn_dist -> knn_to_coo -> symmetrise_graph -> filter_weak_edges.
    kNN lists exclude self; distances are squared Euclidean as the
    reference's ANN backends return."""
    gp = umap_params or UmapGraphParams()
    idx = _c(knn_indices, np.int32)
    d = _c(knn_dists, np.float32)
    n, k = idx.shape
    cap = max(2 * n * k, 1)
    row = np.empty(cap, np.uint32)
    col = np.empty(cap, np.uint32)
    val = np.empty(cap, np.float32)
    nnz = C.c_uint64()
    sig = np.empty(n, np.float32)
    rho = np.empty(n, np.float32)
    cg = _GraphParams(gp.bandwidth, gp.local_connectivity, gp.mix_weight)
    _check(_lib.umapcu_construct_umap_graph(_p(idx), _p(d), n, k, C.byref(cg), n_epochs, cap, _p(row), _p(col),
                                            _p(val), C.byref(nnz), _p(sig), _p(rho)))
    m = nnz.value
    g = CoordinateList(row[:m].copy(), col[:m].copy(), val[:m].copy(), n)
    return (g, sig, rho) if return_sigma_rho else g


def coo_to_adjacency_list(graph: CoordinateList) -> Adjacency:
    """graph.rs:709-758 for a row-grouped COO (the graph stage's output)."""
    r = np.asarray(graph.row_indices)
    if r.size and np.any(r[1:] < r[:-1]):
        order = np.argsort(r, kind="stable")
        r = r[order]
        col = np.asarray(graph.col_indices)[order]
        w = np.asarray(graph.values)[order]
    else:
        col, w = graph.col_indices, graph.values
    cnt = np.bincount(r.astype(np.int64), minlength=graph.n_samples)
    ptr = np.zeros(graph.n_samples + 1, np.uint64)
    np.cumsum(cnt, out=ptr[1:])
    return Adjacency(ptr, _c(col, np.uint32), _c(w, np.float32))


# ------------------------------------------------------------------ densMAP

@dataclass
class DensParams:
    """DensParams (src/utils/density.rs:69-132); densMAP defaults."""
    lambda_: float = 2.0
    frac: float = 0.3
    var_shift: float = 0.1


@dataclass
class DensState:
    """DensState<f32> (src/utils/density.rs:140-251)."""
    params: DensParams
    r: np.ndarray
    mu_sum: np.ndarray
    mu_tot: float
    _keep: list = field(default_factory=list, repr=False)

    @classmethod
    def new(cls, params: DensParams, graph: CoordinateList, knn_indices, knn_dists, distances_squared=True):
        """DensState::new (density.rs:181-201) on the GPU."""
        n = graph.n_samples
        idx = _c(knn_indices, np.int32)
        d = _c(knn_dists, np.float32)
        row = _c(graph.row_indices, np.uint32)
        col = _c(graph.col_indices, np.uint32)
        val = _c(graph.values, np.float32)
        r = np.empty(n, np.float32)
        ms = np.empty(n, np.float32)
        mt = C.c_float()
        _check(_lib.umapcu_dens_state_new(n, row.size, _p(row), _p(col), _p(val), _p(idx), _p(d), idx.shape[1],
                                          int(distances_squared), _p(r), _p(ms), C.byref(mt)))
        return cls(params, r, ms, float(np.float32(mt.value)))

    def is_active(self, epoch: int, n_epochs: int) -> bool:
        """density.rs:244-250 in f32."""
        if self.params.lambda_ <= 0 or n_epochs == 0:
            return False
        return np.float32(epoch + 1) / np.float32(n_epochs) > np.float32(1.0) - np.float32(self.params.frac)

    def _c(self) -> _Dens:
        r = _c(self.r, np.float32)
        ms = _c(self.mu_sum, np.float32)
        self._keep = [r, ms]
        return _Dens(self.params.lambda_, self.params.frac, self.params.var_shift, _p(r), _p(ms), self.mu_tot)


# ------------------------------------------------------------------ optimiser

def _adj(graph) -> Adjacency:
    if isinstance(graph, Adjacency):
        return graph
    if isinstance(graph, CoordinateList):
        return coo_to_adjacency_list(graph)
    return Adjacency.from_lists(graph)


class UmapGpuState:
    """Device-resident optimiser state (UmapGpuState::upload,
    umap_optimiser_gpu.rs:374-452; CSR built on the device as
    UmapCsrGraph::from_graph :132-209)."""

    def __init__(self, embd, graph, params: UmapOptimParams, dens: Optional[DensState] = None, seed: int = 42,
                 sampler: int = NEG_REF_HASH):
        e = _c(embd, np.float32)
        if e.ndim != 2:
            raise ManifoldsError(BAD_ARG, "embd must be [n, n_dim]")
        a = _adj(graph)
        self.n, self.n_dim = e.shape
        self.params = params
        self._h = C.c_void_p()
        cp = params._c()
        cd = dens._c() if dens is not None else None
        _check(_lib.umapcu_state_create(_p(e), self.n, self.n_dim, _p(_c(a.ptr, np.uint64)), _p(a.col), _p(a.w),
                                        C.byref(cp), C.byref(cd) if cd is not None else None, seed & (2 ** 64 - 1),
                                        sampler, C.byref(self._h)))
        n_, ne = C.c_uint64(), C.c_uint64()
        _check(_lib.umapcu_state_sizes(self._h, C.byref(n_), C.byref(ne)))
        self.n_edges = ne.value

    def close(self):
        if self._h:
            _lib.umapcu_state_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def csr(self):
        E = self.n_edges
        off = np.empty(self.n + 1, np.uint32)
        ei = np.empty(2 * E, np.uint32)
        ot = np.empty(2 * E, np.uint32)
        eps = np.empty(E, np.float32)
        mu = np.empty(E, np.float32)
        _check(_lib.umapcu_state_read_csr(self._h, _p(off), _p(ei), _p(ot), _p(eps), _p(mu)))
        return dict(n=self.n, n_edges=E, offsets=off, edge_idx=ei, other=ot, eps=eps, mu=mu)

    def schedule_info(self):
        """-> dict(lists=bool, records=int, build_ms=float): the state's
        per-epoch active-entry lists (see umapcu_state_schedule_info)."""
        a, r, ms = C.c_int(), C.c_uint64(), C.c_float()
        _check(_lib.umapcu_state_schedule_info(self._h, C.byref(a), C.byref(r), C.byref(ms)))
        return dict(lists=bool(a.value), records=r.value, build_ms=ms.value)

    def run(self, first_epoch: int, count: int, optimiser: int = OPT_ADAM):
        _check(_lib.umapcu_state_run(self._h, first_epoch, count, optimiser))

    def enqueue(self, first_epoch: int, count: int, optimiser: int = OPT_ADAM):
        """run() without the final synchronisation (epochs enqueued on the
        state's stream)."""
        _check(_lib.umapcu_state_enqueue(self._h, first_epoch, count, optimiser))

    def set_schedule(self, form: int):
        """Rebuilds the precomputed edge schedule as SCHED_SCAN (none),
        SCHED_BITS (per-epoch bitmasks) or SCHED_LISTS (per-epoch records);
        results are bit-identical in every form."""
        _check(_lib.umapcu_state_set_schedule(self._h, form), "set_schedule")

    def schedule_form(self) -> int:
        f = C.c_uint32()
        _check(_lib.umapcu_state_schedule_form(self._h, C.byref(f)))
        return f.value

    def reset(self, embd=None):
        """Back to the initial state: embedding := embd, moments := 0, cursors := periods."""
        ce = None if embd is None else _c(embd, np.float32)
        _check(_lib.umapcu_state_reset(self._h, _p(ce)))

    def set_precise_pow(self, precise: bool = True):
        """x^b via CUDA's powf (True) or the MUFU exp2/log2 form (False, default)."""
        _check(_lib.umapcu_state_set_precise_pow(self._h, int(precise)))

    def set_stream(self, cuda_stream: int = 0):
        """Launch on the caller's cudaStream_t (an int handle, e.g.
        torch.cuda.current_stream().cuda_stream); 0 restores the own stream."""
        _check(_lib.umapcu_state_set_stream(self._h, C.c_void_p(cuda_stream or None)))

    def run_profiled(self, first_epoch: int, count: int, optimiser: int = OPT_ADAM):
        """run() with CUDA events around every launch -> (epoch-kernel ms, densMAP ms)."""
        e, d = C.c_float(), C.c_float()
        _check(_lib.umapcu_state_run_profiled(self._h, first_epoch, count, optimiser, C.byref(e), C.byref(d)))
        return e.value, d.value

    def epoch_debug(self, epoch: int, optimiser: int = OPT_ADAM, injected=None, want_grad=True):
        inj = None if injected is None else _c(injected, np.uint32)
        g = np.empty((self.n, self.n_dim), np.float32) if want_grad else None
        hu = np.empty(self.n, np.uint32) if want_grad else None
        _check(_lib.umapcu_state_epoch_debug(self._h, epoch, optimiser, _p(inj), _p(g), _p(hu)))
        return g, hu

    def read(self):
        e = np.empty((self.n, self.n_dim), np.float32)
        m = np.empty_like(e)
        v = np.empty_like(e)
        c = np.empty(self.n_edges, np.float32)
        _check(_lib.umapcu_state_read(self._h, _p(e), _p(m), _p(v), _p(c)))
        return e, m, v, c

    def write(self, embd=None, m=None, v=None):
        ce = None if embd is None else _c(embd, np.float32)
        cm = None if m is None else _c(m, np.float32)
        cv = None if v is None else _c(v, np.float32)
        _check(_lib.umapcu_state_write(self._h, _p(ce), _p(cm), _p(cv)))

    def dens_update(self):
        re = np.empty(self.n, np.float32)
        phi = np.empty(self.n, np.float32)
        w = np.empty(self.n, np.float32)
        coeff = C.c_float()
        st = np.empty(3, np.float32)
        _check(_lib.umapcu_state_dens_update(self._h, _p(re), _p(phi), _p(w), C.byref(coeff), _p(st)))
        return dict(re=re, phi_sum=phi, weight=w, coeff=np.float32(coeff.value), stats=st)


class UmapBatch:
    """Batched form: many independent layouts of uneven size advanced together
    by one persistent launch (captured in a CUDA graph), configuration picked
    by the library's autotuner. Each problem is one
    optimise_embedding_adam_gpu call's worth of arguments; the results equal
    the single-problem path's."""

    def __init__(self, embds, graphs, params, seeds, sampler: int = NEG_REF_HASH):
        P = len(embds)
        if not (len(graphs) == P and len(seeds) == P):
            raise ManifoldsError(BAD_ARG, "embds, graphs and seeds must have one entry per problem")
        plist = params if isinstance(params, (list, tuple)) else [params] * P
        self._e = [_c(e, np.float32) for e in embds]
        self._a = [_adj(g) for g in graphs]
        self.n = [e.shape[0] for e in self._e]
        self.n_dim = self._e[0].shape[1] if P else 2
        self.params = plist
        arr = lambda xs, dt: (C.c_void_p * P)(*[x.ctypes.data for x in xs])
        self._ptrs = [_c(a.ptr, np.uint64) for a in self._a]
        cp = (_OptimParams * P)(*[q._c() for q in plist])
        ns = np.array(self.n, np.uint32)
        sd = np.array([int(x) & (2 ** 64 - 1) for x in seeds], np.uint64)
        self._h = C.c_void_p()
        _check(_lib.umapcu_batch_create(P, _p(ns), self.n_dim, arr(self._e, None), arr(self._ptrs, None),
                                        arr([a.col for a in self._a], None), arr([a.w for a in self._a], None),
                                        C.cast(cp, C.c_void_p), _p(sd), sampler, C.byref(self._h)))

    def autotune(self):
        m, c, k = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(_lib.umapcu_batch_autotune(self._h, C.byref(m), C.byref(c), C.byref(k)))
        return dict(mode=m.value, ctas_per_sm=c.value, ku=k.value)

    def run(self, mode: int = 0) -> float:
        """All epochs of every problem; returns device milliseconds.
        mode 0 = autotuned, 1 = persistent launch, 2 = one launch per epoch."""
        ms = C.c_float()
        _check(_lib.umapcu_batch_run(self._h, mode, C.byref(ms)))
        return ms.value

    def read(self, p: int) -> np.ndarray:
        out = np.empty((self.n[p], self.n_dim), np.float32)
        _check(_lib.umapcu_batch_read(self._h, p, _p(out)))
        return out

    def wait_check(self, poisoned_problem: int, wait_limit: int) -> int:
        """Status of a run whose persistent-kernel barrier for one problem can
        never open (the bounded wait must report UMAPCU_TIMEOUT)."""
        return _lib.umapcu_batch_wait_check(self._h, poisoned_problem, wait_limit)

    def close(self):
        if self._h:
            _lib.umapcu_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class UmapServer:
    """Served form: continuous batching of layout jobs on one GPU. submit()
    returns at once; the library's server thread admits jobs within the
    device-memory budget and advances all admitted jobs together, each from
    its own epoch. Thread-safe."""

    PENDING, RUNNING, DONE, FAILED = 0, 1, 2, 3

    def __init__(self, budget_bytes: int, max_jobs: int = 4096, tick_epochs: int = 10, n_dim: int = 2):
        self._h = C.c_void_p()
        self.n_dim = n_dim
        self._n = {}
        _check(_lib.umapcu_server_create(int(budget_bytes), max_jobs, tick_epochs, n_dim, C.byref(self._h)))

    def submit(self, embd, graph, params: UmapOptimParams, seed: int = 42, sampler: int = NEG_REF_HASH) -> int:
        e = _c(embd, np.float32)
        a = _adj(graph)
        cp = params._c()
        t = C.c_uint64()
        _check(_lib.umapcu_server_submit(self._h, e.shape[0], e.shape[1], _p(e), _p(_c(a.ptr, np.uint64)), _p(a.col),
                                         _p(a.w), C.byref(cp), int(seed) & (2 ** 64 - 1), sampler, C.byref(t)))
        self._n[t.value] = e.shape[0]
        return t.value

    def submit_resume(self, embd, graph, params: UmapOptimParams, m, v, epochs_done: int, seed: int = 42,
                      sampler: int = NEG_REF_HASH) -> int:
        """Queues a job resuming from a snapshot (embedding, moments, epochs
        run) of a job with the same graph, parameters, seed and sampler; its
        result equals the uninterrupted job's."""
        e = _c(embd, np.float32)
        mm, vv = _c(m, np.float32), _c(v, np.float32)
        if mm.shape != e.shape or vv.shape != e.shape:
            raise ManifoldsError(BAD_ARG, "m and v must have the embedding's shape")
        a = _adj(graph)
        cp = params._c()
        t = C.c_uint64()
        _check(_lib.umapcu_server_submit_resume(self._h, e.shape[0], e.shape[1], _p(e), _p(_c(a.ptr, np.uint64)),
                                                _p(a.col), _p(a.w), C.byref(cp), int(seed) & (2 ** 64 - 1), sampler,
                                                _p(mm), _p(vv), int(epochs_done), C.byref(t)))
        self._n[t.value] = e.shape[0]
        return t.value

    def snapshot(self, ticket: int):
        """-> (embedding, m, v, epochs_done) of a pending or running job (a
        running one is read at the next tick boundary and keeps running)."""
        n = self._n.get(ticket)
        if n is None:
            raise ManifoldsError(BAD_ARG, "unknown ticket")
        y = np.empty((n, self.n_dim), np.float32)
        m = np.empty_like(y)
        v = np.empty_like(y)
        ep = C.c_uint32()
        _check(_lib.umapcu_server_snapshot(self._h, ticket, _p(y), _p(m), _p(v), C.byref(ep)), "snapshot")
        return y, m, v, ep.value

    def poll(self, ticket: int) -> int:
        st = C.c_int()
        _check(_lib.umapcu_server_poll(self._h, ticket, C.byref(st)))
        return st.value

    def cancel(self, ticket: int):
        _check(_lib.umapcu_server_cancel(self._h, ticket))

    def wait(self, ticket: int):
        """-> (embedding [n, n_dim], latency_s, queue_s); raises on failure."""
        n = self._n.pop(ticket, None)
        if n is None:
            raise ManifoldsError(BAD_ARG, "unknown ticket")
        out = np.empty((n, self.n_dim), np.float32)
        lat, q = C.c_double(), C.c_double()
        _check(_lib.umapcu_server_wait(self._h, ticket, _p(out), C.byref(lat), C.byref(q)))
        return out, lat.value, q.value

    def stats(self):
        c, t, b = C.c_uint64(), C.c_uint64(), C.c_uint64()
        j = C.c_uint32()
        _check(_lib.umapcu_server_stats(self._h, C.byref(c), C.byref(t), C.byref(b), C.byref(j)))
        return dict(completed=c.value, ticks=t.value, peak_bytes=b.value, peak_jobs=j.value)

    def close(self):
        if self._h:
            _lib.umapcu_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def optimise_embedding_adam_gpu(embd: np.ndarray, graph, params: UmapOptimParams, dens: Optional[DensState] = None,
                                seed: int = 42, verbose: int = 0, sampler: int = NEG_REF_HASH,
                                optimiser: int = OPT_ADAM) -> None:
    """optimise_embedding_adam_gpu (umap_optimiser_gpu.rs:1302-1369): embd
    [n, n_dim] float32 (C-contiguous) is optimised in place."""
    if not (isinstance(embd, np.ndarray) and embd.dtype == np.float32 and embd.flags.c_contiguous):
        raise ManifoldsError(BAD_ARG, "embd must be a C-contiguous float32 [n, n_dim] array")
    if embd.ndim != 2 or embd.shape[0] == 0:
        raise NoData(NO_DATA)
    a = _adj(graph)
    cp = params._c()
    cd = dens._c() if dens is not None else None
    _check(_lib.umapcu_optimise_embedding(_p(embd), embd.shape[0], embd.shape[1], _p(_c(a.ptr, np.uint64)),
                                          _p(a.col), _p(a.w), C.byref(cp),
                                          C.byref(cd) if cd is not None else None, seed & (2 ** 64 - 1),
                                          optimiser, sampler, verbose))


# ------------------------------------------------------------------ top level

def random_layout(n_samples: int, n_comp: int, seed: int, init_range: float = 10.0) -> np.ndarray:
    """Uniform U(-range, range) init (init.rs:1024-1041); the generator is
    numpy's PCG64 (the reference's StdRng stream is not reproduced)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-init_range, init_range, (n_samples, n_comp)).astype(np.float32)


@dataclass
class UmapParamsGpu:
    """The UMAP-relevant subset of UmapParamsGpu (src/lib.rs:3218-3346)."""
    n_dim: int = 2
    k: int = 15
    optimiser: str = "adam_gpu"
    optim_params: UmapOptimParams = field(default_factory=UmapOptimParams.default_2d)
    umap_graph_params: UmapGraphParams = field(default_factory=UmapGraphParams)
    sampler: int = NEG_REF_HASH


def _umap_gpu_inner(knn_indices, knn_dists, p: UmapParamsGpu, dens_params: Optional[DensParams], seed: int,
                    verbose: int, init=None):
    opt = parse_umap_optimiser_gpu(p.optimiser)
    if opt is None:
        opt = "adam_gpu"
    graph = construct_umap_graph(knn_indices, knn_dists, p.umap_graph_params, p.optim_params.n_epochs)
    dens = DensState.new(dens_params, graph, knn_indices, knn_dists, True) if dens_params is not None else None
    n = graph.n_samples
    embd = random_layout(n, p.n_dim, seed) if init is None else _c(init, np.float32).copy()
    optimise_embedding_adam_gpu(embd, coo_to_adjacency_list(graph), p.optim_params, dens, seed, verbose,
                                p.sampler, OPT_SGD if opt == "sgd" else OPT_ADAM)
    return embd.T.copy()  # [n_dim][n_samples] like the reference (lib.rs:3700-3707)


def umap_gpu(knn_indices, knn_dists, params: UmapParamsGpu = None, seed: int = 42, verbose: int = 0, init=None):
    """umap_gpu (src/lib.rs:3465-3487) from a precomputed kNN graph."""
    return _umap_gpu_inner(knn_indices, knn_dists, params or UmapParamsGpu(), None, seed, verbose, init)


def densmap_gpu(knn_indices, knn_dists, params: UmapParamsGpu = None, dens_params: DensParams = None, seed: int = 42,
                verbose: int = 0, init=None):
    """densmap_gpu (src/lib.rs:3829-3851) from a precomputed kNN graph."""
    return _umap_gpu_inner(knn_indices, knn_dists, params or UmapParamsGpu(), dens_params or DensParams(), seed,
                           verbose, init)


# ------------------------------------------------------------------ test hooks

def adam_update(grad, has_update, m, v, embd, params: UmapOptimParams, epoch: int):
    """umap_adam_update + launch_adam_update (umap_optimiser_gpu.rs:887-923,
    :1155-1196), in place on m, v, embd."""
    n, d = embd.shape
    cp = params._c()
    _check(_lib.umapcu_adam_update(_p(_c(grad, np.float32)), _p(_c(has_update, np.uint32)), _p(m), _p(v), _p(embd),
                                   n, d, C.byref(cp), epoch))


def edge_schedule_update(eps, cursor, epoch: int):
    """umap_edge_schedule_update (umap_optimiser_gpu.rs:940-955), in place."""
    _check(_lib.umapcu_edge_schedule_update(_p(_c(eps, np.float32)), _p(cursor), cursor.size, epoch))


def eval_pow(x, b, precise=False):
    """x^b as the layout kernels evaluate it (x > 0)."""
    xx = _c(x, np.float32)
    out = np.empty_like(xx)
    _check(_lib.umapcu_eval_pow(_p(xx), xx.size, b, int(precise), _p(out)))
    return out


def sample_negatives(sampler, seed, node, entry, epoch, edge_local, count, n):
    out = np.empty(count, np.uint32)
    _check(_lib.umapcu_sample_negatives(sampler, seed & (2 ** 64 - 1), node, entry, epoch, edge_local, count, n,
                                        _p(out)))
    return out


# ------------------------------------------------------- memory hygiene

def set_pool_retention(keep: bool = True):
    """False: restore every device pool release threshold the library raised
    and leave the pools alone from now on (see umapcu_set_pool_retention)."""
    _check(_lib.umapcu_set_pool_retention(int(bool(keep))))


def release_cached():
    """Frees the current device's cached schedule-bitmask block and trims its
    default memory pool."""
    _check(_lib.umapcu_release_cached(), "release_cached")


def server_job_bytes(n: int, n_dim: int, nnz: int, n_epochs: int) -> int:
    """Device bytes a server's admission charges for a job (its budget unit)."""
    b = C.c_uint64()
    _check(_lib.umapcu_server_job_bytes(n, n_dim, nnz, n_epochs, C.byref(b)))
    return b.value


def device_count() -> int:
    """Visible CUDA devices (0 without a driver or device)."""
    c = C.c_int()
    st = _lib.umapcu_device_count(C.byref(c))
    return c.value if st == OK else 0


def set_device(device: int):
    """Makes `device` the calling thread's current device for the library's
    entry points (states, batches and servers bind to it when created)."""
    _check(_lib.umapcu_set_device(int(device)), "set_device")


def probe_l2_gather(table_bytes: int = 8 << 20) -> float:
    """GB/s of random 8-byte gathers from an L2-resident table (the epoch
    kernel's coordinate-gather form): the L2 roofline denominator."""
    g = C.c_float()
    _check(_lib.umapcu_probe_l2_gather(int(table_bytes), C.byref(g)), "probe_l2_gather")
    return g.value


# ------------------------------------------------------- kNN and metrics

METRIC_EUCLIDEAN_SQ, METRIC_COSINE = 0, 1
_METRICS = {"euclidean": METRIC_EUCLIDEAN_SQ, "cosine": METRIC_COSINE}


def _metric(m) -> int:
    return _METRICS[m] if isinstance(m, str) else int(m)


def knn_exact(data: np.ndarray, k: int, dist_metric="euclidean"):
    """Exact kNN on the GPU, self excluded -- what run_ann_search with
    AnnSearch::Exhaustive returns (src/data/nearest_neighbours.rs:225-364):
    (indices int32 [n, k], distances f32 [n, k]), Euclidean distances
    squared as the reference's ANN backends return them."""
    X = _c(data, np.float32)
    n, dim = X.shape
    idx = np.empty((n, k), np.int32)
    dist = np.empty((n, k), np.float32)
    _check(_lib.umapcu_knn_exact(_p(X), n, dim, k, _metric(dist_metric), _p(idx), _p(dist)), "knn_exact")
    return idx, dist


def embedding_quality(data: np.ndarray, embd: np.ndarray, knn_idx=None, k: int = 15, queries=None,
                      dist_metric="euclidean", trust: bool = True):
    """trustworthiness@k (sklearn's definition) and kNN preservation@k of an
    embedding, on the GPU, over the query rows (all rows by default).
    trust=False skips trustworthiness (the ranks in the data space, the
    expensive part). -> dict(trust=... or None, knn_preservation=... or None)."""
    X = _c(data, np.float32)
    Y = _c(embd, np.float32)
    n = X.shape[0]
    q = None if queries is None else _c(queries, np.uint32)
    ki = None if knn_idx is None else _c(knn_idx, np.int32)
    t = C.c_double()
    kp = C.c_double()
    _check(_lib.umapcu_embedding_quality(_p(X), n, X.shape[1], _p(Y), Y.shape[1], _p(ki),
                                         0 if ki is None else ki.shape[1], k, _p(q), 0 if q is None else q.size,
                                         _metric(dist_metric), C.byref(t) if trust else None,
                                         None if ki is None else C.byref(kp)),
           "embedding_quality")
    return dict(trust=t.value if trust else None, knn_preservation=None if ki is None else kp.value)


def fuzzy_cross_entropy(graph: "CoordinateList", embd: np.ndarray, a: float, b: float) -> float:
    """Fuzzy cross-entropy of an embedding against its graph, f64, on the GPU."""
    Y = _c(embd, np.float32)
    r, c = _c(graph.row_indices, np.uint32), _c(graph.col_indices, np.uint32)
    w = _c(graph.values, np.float32)
    out = C.c_double()
    _check(_lib.umapcu_fuzzy_cross_entropy(_p(r), _p(c), _p(w), r.size, _p(Y), Y.shape[0], Y.shape[1], a, b,
                                           C.byref(out)), "fuzzy_cross_entropy")
    return out.value


def save_knn(path: str, knn_idx: np.ndarray, knn_dist: np.ndarray, dist_metric="euclidean"):
    """Writes a kNN cache file (format in umapcu.h)."""
    i = _c(knn_idx, np.int32)
    d = _c(knn_dist, np.float32)
    if i.shape != d.shape or i.ndim != 2:
        raise ManifoldsError(BAD_ARG, "knn_idx and knn_dist must both be [n, k]")
    _check(_lib.umapcu_knn_save(os.fsencode(path), i.shape[0], i.shape[1], _metric(dist_metric), _p(i), _p(d)),
           "knn_save")


def load_knn(path: str):
    """-> (indices int32 [n, k], distances f32 [n, k], metric) from a kNN
    cache file; checksum and indices are verified."""
    n, k, m = C.c_uint32(), C.c_uint32(), C.c_uint32()
    bp = os.fsencode(path)
    _check(_lib.umapcu_knn_load_header(bp, C.byref(n), C.byref(k), C.byref(m)), "knn_load_header")
    i = np.empty((n.value, k.value), np.int32)
    d = np.empty((n.value, k.value), np.float32)
    _check(_lib.umapcu_knn_load(bp, n.value, k.value, _p(i), _p(d)), "knn_load")
    return i, d, m.value


# ------------------------------------------------------------ spectral init

def compute_smallest_eigenpairs_lanczos(ptr, col, val, n_components: int, seed: int = 42):
    """compute_smallest_eigenpairs_lanczos (src/utils/math.rs:617) on the GPU
    for a CSR matrix: -> (evals [k] ascending, evecs [n, k])."""
    p = _c(ptr, np.uint64)
    n = p.size - 1
    c = _c(col, np.uint32)
    v = _c(val, np.float64)
    ev = np.empty(n_components, np.float32)
    vec = np.empty(n * n_components, np.float32)
    k = C.c_uint32()
    _check(_lib.umapcu_smallest_eigenpairs(n, _p(p), _p(c), _p(v), n_components, int(seed) & (2 ** 64 - 1),
                                           _p(ev), _p(vec), C.byref(k)), "smallest_eigenpairs")
    kk = k.value
    return ev[:kk].copy(), vec[: n * kk].reshape(n, kk).copy()


def spectral_layout(graph: "CoordinateList", n_comp: int = 2, seed: int = 42, range_: float = 10.0):
    """spectral_layout (src/data/init.rs:986) without a data matrix, on the
    GPU: -> embedding [n, n_comp] f32."""
    r = _c(graph.row_indices, np.uint32)
    c = _c(graph.col_indices, np.uint32)
    w = _c(graph.values, np.float32)
    n = int(graph.n_samples)
    out = np.empty((n, n_comp), np.float32)
    _check(_lib.umapcu_spectral_layout(_p(r), _p(c), _p(w), r.size, n, n_comp, int(seed) & (2 ** 64 - 1),
                                       float(range_), _p(out)), "spectral_layout")
    return out
