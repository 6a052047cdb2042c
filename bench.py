#!/usr/bin/env python
"""UMAP layout throughput on B200: edge-updates/s at 1M points.

One step = one full layout run (all epochs) of one embedding problem from its
fuzzy graph, the unit the reference's timing harness isolates
(tests/umap_gpu_bench.rs:217-252). An edge-update is one active undirected
edge in one epoch (cursor <= epoch), both endpoints' attractive and negative
terms included; the count per epoch depends only on the edge periods, so it
is the same for every implementation.

  value  : device-resident graph and embedding; each timed step starts from
           the reset state with L2 flushed (256 MiB write) and contains the
           build of the run's schedule bitmasks and every epoch (CUDA events
           on the launching stream). The other schedule forms (record lists
           built in the step, plain cursor scan) are reported beside it.
  e2e    : the reference-facing call umapcu.optimise_embedding_adam_gpu
           (C ABI umapcu_optimise_embedding) from pinned host buffers:
           H2D of graph + embedding, CSR build, bitmasks, epochs, D2H.
  roofline: the fused epoch kernel's time per epoch from the timed region,
           algorithmic HBM bytes against the measured copy bandwidth, and
           its random coordinate gathers against the measured L2 gather rate.
  cpu_baseline / --impl reference : the reference's parallel Adam
           (umap_optimisers.rs:1170-1492, restated in oracle/) on all host
           cores, whole runs from the initial embedding, epoch loop only.
           The reference arm loads no umapcu code: its inputs come from
           umapdata (NumPy) and the oracle.

Both arms share one input: the workload's brute-force kNN, cached in a kNN
cache file by whichever arm runs first (torch on the GPU, outside every timed
region).

Multi-GPU (torchrun): every rank runs its own problem (replicas, seed +
rank); value is the sum over ranks / max-over-ranks time ("weak").
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "manifolds-rs_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "UMAP layout edge-updates/s (1M pts)"
UNIT = "edge-updates/s"


def max_over_ranks(x, dist):
    """x maximised over the ranks of dist's default group, or x itself
    without one; the tensor lives where the group's backend wants it (CUDA
    for NCCL, host memory for gloo)."""
    if dist is None:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def metric_of(wl):
    """The headline metric's name for the 1M-point layout; the other layout
    workloads name their own size."""
    if wl["n"] == 1_000_000 and not wl["dens"]:
        return METRIC
    size = f"{wl['n'] // 1000}k pts" if wl["n"] < 1_000_000 else f"{wl['n'] / 1e6:g}M pts"
    return f"UMAP layout edge-updates/s ({size}{', densMAP' if wl['dens'] else ''})"

WORKLOADS = {
    "c2": dict(n=1_000_000, dim=50, clusters=30, k=15, n_epochs=200, kind="anisotropic", dens=False,
               desc="1M x 50 f32, 30-component anisotropic Gaussian mixture (eig log-U[0.1,4], Dirichlet(1) "
                    "weights), exact kNN k=15 cached, 2-D, 200 epochs, Adam, neg_rate 5, random U(-10,10) init"),
    "c1": dict(n=10_000, dim=50, clusters=10, k=15, n_epochs=500, kind="isotropic", dens=False,
               desc="10k x 50 f32, 10 isotropic Gaussians, exact kNN k=15, 2-D, 500 epochs, Adam, neg_rate 5"),
    "c4": dict(n=0, problems=512, n_lo=500, n_hi=50_000, dim=30, clusters=(5, 15), k=15, n_epochs=200,
               kind="batch", dens=False,
               desc="batched form: 512 independent problems, n log-uniform in [500, 50000], 30-D isotropic "
                    "5-15-cluster mixtures, exact kNN k=15, 2-D, 200 epochs, Adam, one persistent launch "
                    "(CUDA graph), configuration from the autotuner"),
    "c5": dict(n=0, requests=2000, pool=48, n_lo=1000, n_hi=200_000, dims=(20, 50, 100), clusters=(5, 40), k=15,
               n_epochs=200, kind="serve", dens=False, budget=120 << 30, util=0.8,
               desc="served form: 2000 requests, seeded Poisson arrivals at ~80% of the server's measured saturated throughput, sizes "
                    "log-uniform in [1000, 200000], data dims in {20, 50, 100}, 5-40 clusters, precomputed k=15 "
                    "graphs (a pool of 48, requests draw a graph and their own seed/init), 2-D, 200 epochs, Adam, "
                    "120 GB admission budget, continuous batching"),
    "spectral": dict(n=1_000_000, dim=50, clusters=30, k=15, n_epochs=200, kind="anisotropic", dens=False,
                     spectral=True,
                     desc="spectral initialisation of the 1M-point graph (the c2 data and kNN): -D^-1/2 A D^-1/2, "
                          "Lanczos with 4 k + 30 steps for the 3 smallest eigenpairs, 2-D layout"),
    "c3": dict(n=200_000, dim=30, clusters=20, k=30, n_epochs=200, kind="variable", dens=True,
               desc="densMAP 200k x 30 f32, 20 clusters sd log-U[0.2,3], k=30, 2-D, 200 epochs, last 30% "
                    "density term, lambda 2, Adam"),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------- inputs

def knn_cache_path(wl, seed):
    d = os.environ.get("UMAPCU_KNN_CACHE") or os.path.join(__import__("tempfile").gettempdir(), "umapcu_knn")
    os.makedirs(d, exist_ok=True)
    return os.path.join(d, f"{wl['kind']}_n{wl['n']}_d{wl['dim']}_c{wl['clusters']}_k{wl['k']}_s{seed}_bf.knn")


def shared_knn(X, wl, seed):
    """The workload's brute-force kNN, computed once and cached (kNN cache
    file) as the shared input of both arms: input preparation, outside every
    timed region. Read and written with the NumPy reader of the cache format
    and computed with torch (fp32 GEMM candidates, f64 distances of the
    candidates) on the GPU, or NumPy without one, so that neither arm needs
    the umapcu library to prepare it."""
    from umapdata import knn_cache
    import umapdata.synth as S
    path = knn_cache_path(wl, seed)
    if os.path.exists(path):
        try:
            idx, dist, _ = knn_cache.load(path)
            if idx.shape == (wl["n"], wl["k"]):
                log(f"[bench] kNN from cache {path}")
                return idx, dist
        except ValueError:
            pass
    import torch
    if torch.cuda.is_available():
        idx, dist = S.exact_knn_torch(X, wl["k"])
    else:
        idx, dist = S.exact_knn_cpu(X, wl["k"])
    idx, dist = idx.astype(np.int32), dist.astype(np.float32)
    tmp = f"{path}.{os.getpid()}.tmp"
    knn_cache.save(tmp, idx, dist)
    os.replace(tmp, path)
    return idx, dist


def make_data(wl, seed):
    import umapdata.synth as S
    if wl["kind"] == "anisotropic":
        return S.anisotropic_mixture(wl["n"], wl["dim"], wl["clusters"], seed)[0]
    if wl["kind"] == "variable":
        return S.variable_density_mixture(wl["n"], wl["dim"], wl["clusters"], seed)[0]
    return S.isotropic_mixture(wl["n"], wl["dim"], wl["clusters"], seed)[0]


def make_problem(wl, seed):
    """Synthetic data -> shared cached kNN -> the CUDA graph stage (umapcu
    arm)."""
    import umapcu
    import umapdata.synth as S
    t0 = time.time()
    X = make_data(wl, seed)
    idx, dist = shared_knn(X, wl, seed)
    t1 = time.time()
    graph = umapcu.construct_umap_graph(idx, dist, umapcu.UmapGraphParams(), wl["n_epochs"])
    dens = umapcu.DensState.new(umapcu.DensParams(), graph, idx, dist, True) if wl["dens"] else None
    adj = umapcu.coo_to_adjacency_list(graph)
    params = umapcu.UmapOptimParams.from_min_dist_spread(0.1, 1.0, n_epochs=wl["n_epochs"], neg_sample_rate=5)
    init = S.random_layout(wl["n"], 2, seed)
    log(f"[bench] data+kNN {t1 - t0:.1f}s, graph {time.time() - t1:.1f}s, nnz {adj.col.size}")
    return dict(X=X, idx=idx, dist=dist, graph=graph, adj=adj, dens=dens, params=params, init=init)


def make_reference_problem(wl, seed):
    """The same inputs for the reference arm, prepared without the umapcu
    library: the oracle's CPU restatement of the reference's graph stage
    (graph.rs:499-853), its densMAP state (density.rs:181-201) and its a, b
    fit (umap_optimisers.rs:139-209)."""
    import umapdata.synth as S
    from oracle import oracle as O
    t0 = time.time()
    X = make_data(wl, seed)
    idx, dist = shared_knn(X, wl, seed)
    t1 = time.time()
    (r, c, v), _, _ = O.construct_umap_graph(idx, dist, wl["n_epochs"])
    ptr = O.coo_to_adj_ptr(wl["n"], r)
    dens = None
    if wl["dens"]:
        _, d = O.dens_state_new(wl["n"], r, c, v, idx, dist, True)
        dens = {"r": d["r"], "lambda": d["lambda"], "frac": d["frac"], "var_shift": d["var_shift"],
                "mu_tot": d["mu_tot"]}
    a, b = O.fit_params(0.1, 1.0)
    params = dict(a=float(a), b=float(b), lr=1.0, gamma=1.0, n_epochs=wl["n_epochs"], neg_sample_rate=5,
                  min_dist=0.1, beta1=0.5, beta2=0.9, eps=1e-7)
    init = S.random_layout(wl["n"], 2, seed)
    log(f"[bench] data+kNN {t1 - t0:.1f}s, oracle graph {time.time() - t1:.1f}s, nnz {c.size}")
    return dict(ptr=ptr, col=c, w=v, dens=dens, params=params, init=init)


def config_of(args, wl):
    """The workload description both arms print (identical by construction)."""
    return {"workload": f"{args.workload}: {wl['desc']}", "n_points": wl["n"], "k": wl["k"],
            "epochs": wl["n_epochs"], "optimiser": args.optimiser, "neg_sample_rate": 5,
            "l2": "GPU arm: L2 flushed (256 MiB write) before every timed step; CPU arm: no device",
            "parallelism": f"replicas x{int(os.environ.get('WORLD_SIZE', '1'))}"}


def active_edges_per_epoch(eps, n_epochs):
    """A_e: edges with cursor <= e under the f32 schedule of
    umap_optimiser_gpu.rs:741/952 (cursor starts at the period)."""
    eps = np.asarray(eps, np.float32)
    cur = eps.copy()
    out = np.zeros(n_epochs, np.int64)
    for e in range(n_epochs):
        act = cur <= np.float32(e)
        out[e] = int(act.sum())
        cur[act] += eps[act]
    return out


# ----------------------------------------------------------------- clocks

class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled through NVML every
    50 ms during the timed region (reads only; no setting is changed)."""

    def __init__(self, device_index):
        self.dev = device_index
        self.samples = []
        self.stop = threading.Event()
        self.t = None

    def __enter__(self):
        try:
            import pynvml as N
            N.nvmlInit()
            self.N = N
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.dev]) if vis and vis.split(",")[self.dev].isdigit() else self.dev
            self.h = N.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM)
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        except Exception as e:  # NVML missing: record why
            self.err = str(e)
        return self

    def _run(self):
        N = self.N
        while not self.stop.is_set():
            try:
                mhz = N.nvmlDeviceGetClockInfo(self.h, N.NVML_CLOCK_SM)
                rs = N.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                util = N.nvmlDeviceGetUtilizationRates(self.h).gpu
                self.samples.append((mhz, rs, util))
            except Exception:
                pass
            self.stop.wait(0.05)

    def __exit__(self, *exc):
        self.stop.set()
        if self.t:
            self.t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled: " + getattr(self, "err", "no samples")]}
        N = self.N
        names = {"hw_slowdown": N.nvmlClocksEventReasonHwSlowdown,
                 "hw_thermal_slowdown": N.nvmlClocksEventReasonHwThermalSlowdown,
                 "sw_thermal_slowdown": N.nvmlClocksEventReasonSwThermalSlowdown,
                 "sw_power_cap": N.nvmlClocksEventReasonSwPowerCap}
        busy = [s for s in self.samples if s[2] > 0] or self.samples
        reasons = sorted({k for _, rs, _ in busy for k, bit in names.items() if rs & bit})
        return {"sm_mhz": float(np.median([s[0] for s in busy])), "sm_max_mhz": float(self.max_mhz),
                "reasons": reasons, "samples": len(busy)}


# ----------------------------------------------------------------- CPU leg

def cpu_full_runs(ptr, col, w, params, init, dens, seed, reps, threads, n_epochs):
    """Times whole runs of the oracle's adam_parallel (the reference's
    optimise_embedding_adam_parallel, umap_optimisers.rs:1170-1492) from the
    initial embedding: epoch loop only, as tests/umap_gpu_bench.rs:232-252
    times it. Returns the loop seconds of each run."""
    from oracle import oracle as O
    n = init.shape[0]
    out = []
    for _ in range(reps):
        st, _, secs = O.optimise_adam_parallel(init, n, ptr, col, w, params, seed, dens, threads, 0, 0, True)
        if st != O.OK:
            raise RuntimeError(f"oracle adam_parallel status {st}")
        out.append(secs)
    return out


# ----------------------------------------------------------------- main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="umapcu", choices=["umapcu", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--sampler", default="ref_hash", choices=["ref_hash", "philox"])
    ap.add_argument("--optimiser", default="adam", choices=["adam", "sgd"])
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile-only", action="store_true", help="a 40-epoch state, run once, for ncu captures")
    ap.add_argument("--profile-one-shot", action="store_true",
                    help="one 40-epoch one-shot call (per-epoch bitmasks), for ncu captures")
    ap.add_argument("--requests", type=int, default=0, help="served workload: number of requests")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    wl = dict(WORKLOADS[args.workload])

    import torch
    if args.impl == "reference":
        if rank != 0:
            return
        run_reference(args, wl, world)
        return
    if wl["kind"] == "batch":
        run_batched(args, wl, world, rank, local_rank)
        return
    if wl.get("spectral"):
        run_spectral(args, wl, world, rank, local_rank)
        return
    if wl["kind"] == "serve":
        run_served(args, wl, world, rank, local_rank)
        return

    torch.cuda.set_device(local_rank)
    dist = init_group(world)

    import umapcu
    seed = args.seed + rank
    prob = make_problem(wl, seed)
    sampler = umapcu.NEG_PHILOX if args.sampler == "philox" else umapcu.NEG_REF_HASH
    opt = umapcu.OPT_SGD if args.optimiser == "sgd" else umapcu.OPT_ADAM
    if args.profile_one_shot:
        # the one-shot call's epoch kernel (bitmask scan) for ncu captures
        import dataclasses
        p40 = dataclasses.replace(prob["params"], n_epochs=min(wl["n_epochs"], 40))
        y = np.ascontiguousarray(prob["init"].copy())
        umapcu.optimise_embedding_adam_gpu(y, prob["adj"], p40, prob["dens"], seed, 0, sampler, opt)
        log(f"[bench] profile-one-shot run done, finite {bool(np.isfinite(y).all())}")
        return
    if args.profile_only:
        # a short run for ncu captures: a state made for 40 epochs (schedule
        # lists of 40 epochs, ~1/5 of the full run's device memory), run once
        import dataclasses
        p40 = dataclasses.replace(prob["params"], n_epochs=min(wl["n_epochs"], 40))
        st = umapcu.UmapGpuState(prob["init"], prob["adj"], p40, prob["dens"], seed, sampler)
        st.run(0, p40.n_epochs, opt)
        torch.cuda.synchronize()
        log(f"[bench] profile-only run done, schedule {st.schedule_info()}")
        st.close()
        return
    st = umapcu.UmapGpuState(prob["init"], prob["adj"], prob["params"], prob["dens"], seed, sampler)
    E = st.n_edges
    csr = st.csr()
    ae = active_edges_per_epoch(csr["eps"], wl["n_epochs"])
    updates_per_step = int(ae.sum())
    n_ep = wl["n_epochs"]
    # a stream of our own (the legacy default stream's handle is 0, which the
    # state reads as "your own stream"): the state's launches and the events
    # share it
    stream = torch.cuda.Stream()
    st.set_stream(stream.cuda_stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2

    def time_steps(form, count):
        """count steps of the whole layout: each from the reset state (input
        embedding in HBM, moments zero, cursors at their periods) and a
        flushed L2, the schedule's precomputed form built inside the timed
        region, then every epoch. -> (step seconds, epoch-loop seconds)."""
        tot, loop = [], []
        for _ in range(count):
            st.set_schedule(umapcu.SCHED_SCAN)  # frees the previous step's form (outside the region)
            st.reset(prob["init"])
            flush.fill_(1.0)
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            e0, em, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            if form != umapcu.SCHED_SCAN:
                st.set_schedule(form)
            em.record(stream)
            st.enqueue(0, n_ep, opt)
            e1.record(stream)
            torch.cuda.synchronize()
            tot.append(e0.elapsed_time(e1) / 1e3)
            loop.append(em.elapsed_time(e1) / 1e3)
        return tot, loop

    time_steps(umapcu.SCHED_BITS, args.warmup)
    with ClockSampler(local_rank) as clk:
        times, loops = time_steps(umapcu.SCHED_BITS, args.steps)
    total = max_over_ranks(np.sum(times), dist)
    value = world * args.steps * updates_per_step / total
    ms_per_step = total / args.steps * 1e3
    # the other schedule forms, same steps (secondary figures)
    variants = {}
    for name, form in (("lists", umapcu.SCHED_LISTS), ("csr_scan", umapcu.SCHED_SCAN)):
        time_steps(form, 1)
        t = max_over_ranks(np.sum(time_steps(form, args.steps)[0]), dist)
        variants[name] = {"value": world * args.steps * updates_per_step / t,
                          "ms_per_step": round(t / args.steps * 1e3, 3)}
    variants["lists"]["note"] = "per-epoch record lists, built inside every timed step"
    variants["csr_scan"]["note"] = "no precomputed schedule: every epoch scans and advances the cursors"

    # roofline of the dominant kernel (the fused epoch kernel) from the timed
    # region: the epoch loop's device time per epoch
    avg_epoch_s = max_over_ranks(np.sum(loops), dist) / args.steps / n_ep
    dens_ms = None
    if wl["dens"]:
        st.set_schedule(umapcu.SCHED_SCAN)
        st.reset(prob["init"])
        st.set_schedule(umapcu.SCHED_BITS)
        torch.cuda.synchronize()
        k_ms, d_ms = st.run_profiled(0, n_ep, opt)
        dens_ms = d_ms
        avg_epoch_s = k_ms / 1e3 / n_ep
    n_nodes = wl["n"]
    nd = 2
    # algorithmic HBM bytes per epoch: E (tail index + period/cursor) + A_e
    # cursor writes + n * D * 4 B * 7 node-state streams
    hbm_bytes = (8.0 * E * n_ep + 4.0 * updates_per_step + 28.0 * n_nodes * nd * n_ep) / n_ep
    # algorithmic L2 gathers per epoch: 2 endpoints x (1 + neg_rate) rows of 8 B per edge-update
    l2_bytes = 2.0 * (1 + 5) * 8.0 * updates_per_step / n_ep
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    l2_peak = umapcu.probe_l2_gather(8 * n_nodes)
    traffic = None
    tf = os.path.join(ROOT, "profiles", f"k_epoch_{args.workload}_traffic.txt")
    if os.path.exists(tf):
        for ln in open(tf):
            if ln.startswith("dram_bytes_per_launch:"):
                traffic = float(ln.split(":")[1])
    achieved = hbm_bytes / avg_epoch_s / 1e9
    l2_ach = l2_bytes / avg_epoch_s / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic,
            "kernel": f"k_epoch<2,{'true' if wl['dens'] else 'false'},5,true,false,true> (bitmask scan)",
            "avg_launch_us": round(avg_epoch_s * 1e6, 2),
            "hbm_bytes_per_launch": round(hbm_bytes), "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "l2": {"achieved": round(l2_ach, 1), "peak": round(l2_peak, 1), "unit": "GB/s",
                   "frac": round(l2_ach / l2_peak, 4), "bytes_per_launch": round(l2_bytes),
                   "what": "random 8-byte coordinate gathers (2 endpoints x (1 + 5 negatives) per edge-update) "
                           "against umapcu_probe_l2_gather's measured rate of the same gather form",
                   "binding_unit": "the SMs' load pipeline (L1TEX), one random line per SM-clock "
                                   "(ncu: l1tex 85 %, lts 62 %, dram 12 % of peak)"}}

    # end to end through the reference-facing C-ABI call, pinned host buffers
    e2e = None
    if not args.no_e2e:
        adj = prob["adj"]
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        ptr_p, col_p, w_p = pin(adj.ptr), pin(adj.col), pin(adj.w)
        embd_p = pin(prob["init"])
        A = umapcu.Adjacency(ptr_p, col_p, w_p)
        init = prob["init"]
        for _ in range(max(1, args.warmup)):
            embd_p[...] = init
            umapcu.optimise_embedding_adam_gpu(embd_p, A, prob["params"], prob["dens"], seed, 0, sampler, opt)
        tt = []
        for _ in range(args.steps):
            embd_p[...] = init
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            umapcu.optimise_embedding_adam_gpu(embd_p, A, prob["params"], prob["dens"], seed, 0, sampler, opt)
            tt.append(time.perf_counter() - t0)
        et = max_over_ranks(np.sum(tt), dist)
        h2d = ptr_p.nbytes + col_p.nbytes + w_p.nbytes + embd_p.nbytes
        if prob["dens"] is not None:
            h2d += prob["dens"].r.nbytes
        e2e = {"value": world * args.steps * updates_per_step / et, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(embd_p.nbytes), "ms_per_step": round(et / args.steps * 1e3, 3)}

    quality = None
    if e2e is not None and rank == 0:
        # the finished embedding of the last end-to-end run, on a seeded
        # 10 000-query subsample against all points
        qn = min(10_000, wl["n"])
        qs = np.sort(np.random.default_rng(seed + 77).choice(wl["n"], qn, replace=False)).astype(np.uint32)
        q = umapcu.embedding_quality(prob["X"], embd_p, prob["idx"], 15, queries=qs)
        quality = {"trust15": q["trust"], "knn_preservation15": q["knn_preservation"], "queries": int(qn)}

    cpu = None
    if args.optimiser == "sgd":
        cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "not timed: the reference's SGD (umap_optimisers.rs:653-865) is sequential over all "
                         "edges; its parallel CPU path is the Adam one"}
    elif rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        adj = prob["adj"]
        dd = None
        if prob["dens"] is not None:
            d = prob["dens"]
            dd = {"r": d.r, "lambda": d.params.lambda_, "frac": d.params.frac, "var_shift": d.params.var_shift,
                  "mu_tot": d.mu_tot}
        secs = cpu_full_runs(adj.ptr, adj.col, adj.w, prob["params"].as_dict(), prob["init"], dd, seed, 3, threads,
                             n_ep)
        cpu = {"value": updates_per_step / min(secs), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"whole {n_ep}-epoch runs of the oracle's adam_parallel restatement from the same initial "
                         f"embedding, epoch loop only, best of 3 ({', '.join(f'{x:.2f}' for x in secs)} s; "
                         f"{updates_per_step} edge-updates per run)"}

    dens_launches = 0
    if wl["dens"]:
        dp = prob["dens"]
        dens_launches = sum(1 for e in range(n_ep) if dp.is_active(e, n_ep))
    if rank == 0:
        out = {
            "metric": metric_of(wl), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(args, wl),
            "n_edges": int(E), "edge_updates_per_step": updates_per_step, "sampler": args.sampler,
            "schedule": "per-epoch active-entry bitmasks (1 bit per CSR entry and epoch), built inside every "
                        "timed step, then every epoch; the graph and CSR stay resident (built once, outside)",
            "schedule_variants": variants,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            # per step: the bitmask build, one fused epoch kernel per epoch, the densMAP updates
            "gpu_launches": args.steps * (1 + n_ep + dens_launches),
            "clocks": clk.summary(),
            "densmap_ms_per_step": round(dens_ms, 3) if dens_ms is not None else None,
            "quality": quality,
        }
        print(json.dumps(out), flush=True)
    st.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def init_group(world, backend="nccl"):
    """The process group of a multi-rank run (None for one rank)."""
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return dist


def batch_problem_sizes(wl, seed):
    """The C4 problem set's sizes and cluster counts (seeded; the same in
    every rank)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(wl["n_lo"]), np.log(wl["n_hi"]), wl["problems"])).astype(int)
    clusters = rng.integers(wl["clusters"][0], wl["clusters"][1] + 1, wl["problems"])
    return sizes, clusters


def make_batch_problems(wl, seed, which):
    """Problems `which` of the C4 set: seeded data, exact kNN, CUDA graph
    stage, seeded initial layout (each problem's inputs depend only on its
    own index)."""
    import umapcu
    import umapdata.synth as S
    sizes, clusters = batch_problem_sizes(wl, seed)
    adjs, inits = [], []
    t0 = time.time()
    for i in which:
        n = int(sizes[i])
        X, _ = S.isotropic_mixture(n, wl["dim"], int(clusters[i]), seed + 1000 + i)
        idx, knn_d = umapcu.knn_exact(X, wl["k"])
        g = umapcu.construct_umap_graph(idx, knn_d, umapcu.UmapGraphParams(), wl["n_epochs"])
        adjs.append(umapcu.coo_to_adjacency_list(g))
        inits.append(S.random_layout(n, 2, seed + 5000 + i))
    log(f"[bench] {len(which)} problems, {int(sizes[which].sum())} points, prepared in {time.time() - t0:.1f}s")
    return sizes[which], adjs, inits


def run_batched(args, wl, world, rank, local_rank):
    """Batched form vs sequential single-problem runs, embeddings/s. With
    several ranks the 512 problems are placed over the GPUs by
    umapcu.pool.lpt_partition on their sizes (the same placement in every
    rank, no data exchange); each rank runs one batch of its share and the
    time is the max over ranks (strong scaling: the problem set is fixed)."""
    import torch
    import umapcu
    from umapcu.pool import lpt_partition
    torch.cuda.set_device(local_rank)
    group = init_group(world)
    seed = args.seed
    all_sizes, _ = batch_problem_sizes(wl, seed)
    shares = lpt_partition(all_sizes.astype(np.float64), world)
    mine = shares[rank]
    sizes, adjs, inits = make_batch_problems(wl, seed, mine)
    params = umapcu.UmapOptimParams.from_min_dist_spread(0.1, 1.0, n_epochs=wl["n_epochs"], neg_sample_rate=5)
    seeds = [seed + i for i in mine]
    B = umapcu.UmapBatch(inits, adjs, params, seeds)
    cfg = B.autotune()
    for _ in range(args.warmup):
        B.run(0)
    if group:
        group.barrier()
    with ClockSampler(local_rank) as clk:
        ms = [B.run(0) for _ in range(args.steps)]
    t_batch = max_over_ranks(float(np.sum(ms)) / 1e3, group)
    # edge-updates per run, from each problem's periods
    updates = 0
    states = []
    for i in range(len(sizes)):
        st = umapcu.UmapGpuState(inits[i], adjs[i], params, None, seeds[i])
        updates += int(active_edges_per_epoch(st.csr()["eps"], wl["n_epochs"]).sum())
        states.append(st)
    # sequential plain-kernel runs of the same problems (device-resident states)
    stream = torch.cuda.Stream()
    for st in states:
        st.set_stream(stream.cuda_stream)
    for i, st in enumerate(states[:8]):
        st.reset(inits[i])
        st.run(0, wl["n_epochs"])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i, st in enumerate(states):
        st.reset(inits[i])
    torch.cuda.synchronize()
    e0.record(stream)
    for st in states:
        st.enqueue(0, wl["n_epochs"])
    e1.record(stream)
    torch.cuda.synchronize()
    t_seq = max_over_ranks(e0.elapsed_time(e1) / 1e3, group)
    # identical results in the batch and alone (spot check)
    ok = True
    for i in (0, len(sizes) // 2, len(sizes) - 1):
        y_single, _, _, _ = states[i].read()
        ok &= bool(np.array_equal(B.read(i), y_single))
    for st in states:
        st.close()
    updates = max_over_ranks(updates, group) if group is None else _sum_over_ranks(updates, group)
    P = len(all_sizes)
    value = args.steps * P / t_batch
    out = {"metric": "UMAP batched embeddings/s (512 problems)", "value": value, "unit": "embeddings/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(t_batch / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"c4: {wl['desc']}", "problems": P, "points": int(all_sizes.sum()),
                      "placement": f"LPT over {world} GPU(s) by problem size; this rank {len(mine)} problems",
                      "autotuned": cfg, "l2": "not flushed (state reset kernel precedes every run)"},
           "edge_updates_per_s": args.steps * updates / t_batch,
           "sequential_plain": {"embeddings_per_s": P / t_seq, "ms": round(t_seq * 1e3, 3)},
           "speedup_vs_sequential": round((P / t_batch * args.steps) / (P / t_seq), 2) if t_seq > 0 else None,
           "same_result_alone_and_batched": ok,
           # per run: the state reset kernel, then one persistent launch or one launch per epoch
           "gpu_launches": args.steps * (1 + (1 if cfg["mode"] == 1 else wl["n_epochs"])),
           "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    B.close()
    if group:
        group.barrier()
        group.destroy_process_group()


def _sum_over_ranks(x, group):
    import torch
    dev = "cuda" if group.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    group.all_reduce(t)
    return float(t.item())


def place_requests(work, world):
    """Online placement of a request stream over ranks: each request, in
    arrival order, to the rank with the least work placed so far (ties: the
    lowest rank). Deterministic, so every rank derives the same assignment."""
    load = np.zeros(world)
    out = np.empty(len(work), np.int64)
    for r, w in enumerate(work):
        k = int(np.argmin(load))
        out[r] = k
        load[k] += w
    return out


def run_served(args, wl, world, rank, local_rank):
    """Continuous-batching server under a Poisson request stream. With
    several ranks one stream of world x requests at world x the rate is
    placed over the GPUs by place_requests (least work placed so far, the
    same assignment in every rank); each rank's server takes its share at
    the requests' arrival times; the span is the max over ranks."""
    import torch
    import umapcu
    import umapdata.synth as S
    torch.cuda.set_device(local_rank)
    group = init_group(world)
    seed = args.seed
    rng = np.random.default_rng(seed)
    t0 = time.time()
    pool = []
    for i in range(wl["pool"]):
        n = int(np.exp(rng.uniform(np.log(wl["n_lo"]), np.log(wl["n_hi"]))))
        dim = int(rng.choice(wl["dims"]))
        X, _ = S.isotropic_mixture(n, dim, int(rng.integers(wl["clusters"][0], wl["clusters"][1] + 1)), seed + 70 + i)
        idx, knn_d = umapcu.knn_exact(X, wl["k"])
        g = umapcu.construct_umap_graph(idx, knn_d, umapcu.UmapGraphParams(), wl["n_epochs"])
        pool.append(umapcu.coo_to_adjacency_list(g))
    log(f"[bench] served pool of {len(pool)} graphs prepared in {time.time() - t0:.1f}s")
    params = umapcu.UmapOptimParams.from_min_dist_spread(0.1, 1.0, n_epochs=wl["n_epochs"], neg_sample_rate=5)
    n_req = (args.requests or wl["requests"]) * world
    req_graph = rng.integers(0, len(pool), n_req)
    owner = place_requests([pool[int(g)].col.size for g in req_graph], world)

    def init_of(r):
        g = int(req_graph[r])
        return S.random_layout(pool[g].n, 2, seed + 9000 + r)

    # capacity: the server's own steady-state throughput under a saturating
    # burst (every request submitted at once; admission, graph builds and
    # ticks included), embeddings/s for this size mix, taken between the
    # 10th and 90th percentile completions (ramp-up and drain excluded); the
    # slowest rank's figure sets the stream's rate
    n_cal = 20 * len(pool)
    cal_rng = np.random.default_rng(seed + 5)
    cal = [(pool[int(g)], S.random_layout(pool[int(g)].n, 2, seed + 7000 + i))
           for i, g in enumerate(cal_rng.integers(0, len(pool), n_cal))]
    sv = umapcu.UmapServer(budget_bytes=wl["budget"], max_jobs=4096, tick_epochs=10, n_dim=2)
    for g, y0 in cal[:len(pool)]:  # warm-up
        sv.wait(sv.submit(y0, g, params, seed=1))
    subs = []
    for i, (g, y0) in enumerate(cal):
        subs.append((time.perf_counter(), sv.submit(y0, g, params, seed=i)))
    done = np.sort([ts + sv.wait(t)[1] for ts, t in subs])
    lo, hi = int(0.1 * n_cal), int(0.9 * n_cal)
    cap = (hi - lo) / (done[hi] - done[lo])
    sv.close()
    cap = -max_over_ranks(-cap, group)  # the minimum over ranks
    lam = world * wl["util"] * cap
    gaps = rng.exponential(1.0 / lam, n_req)
    arrive = np.cumsum(gaps)
    mine = [r for r in range(n_req) if owner[r] == rank]
    inits = {r: init_of(r) for r in mine}  # client-side data, made before the stream starts
    sv = umapcu.UmapServer(budget_bytes=wl["budget"], max_jobs=4096, tick_epochs=10, n_dim=2)
    tickets = []
    if group:
        group.barrier()
    t_start = time.perf_counter()
    with ClockSampler(local_rank) as clk:
        for r in mine:
            d = t_start + arrive[r] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets.append(sv.submit(inits[r], pool[int(req_graph[r])], params, seed=seed + r))
        t_sub = time.perf_counter()
        lat, queue = [], []
        for t in tickets:
            _, l, q = sv.wait(t)
            lat.append(l)
            queue.append(q)
        t_end = time.perf_counter()
    st = sv.stats()
    sv.close()
    span = max_over_ranks(t_end - t_start, group)
    if group:
        every = [None] * world
        group.all_gather_object(every, (lat, queue))
        lat = [x for a, _ in every for x in a]
        queue = [x for _, b in every for x in b]
    out = {"metric": "UMAP served embeddings/s (Poisson stream)", "value": n_req / span,
           "unit": "embeddings/s",
           "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": round(span * 1e3, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"c5: {wl['desc']}", "requests": n_req, "arrival_rate_per_s": round(lam, 2),
                      "submitted_rate_per_s_rank0": round(len(mine) / max(t_sub - t_start, 1e-9), 2),
                      "capacity_per_s_per_gpu": round(cap, 2),
                      "placement": f"least work placed so far, over {world} GPU(s)",
                      "budget_bytes": wl["budget"], "tick_epochs": 10},
           "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                         "mean": float(np.mean(lat)), "max": float(np.max(lat))},
           "queue_s": {"p50": float(np.percentile(queue, 50)), "p99": float(np.percentile(queue, 99))},
           "server": st, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if group:
        group.barrier()
        group.destroy_process_group()


def run_spectral(args, wl, world, rank, local_rank):
    """Spectral initialisation of the c2 graph through umapcu_spectral_layout
    (host COO in, layout out: the end-to-end call), against the oracle's
    numpy restatement of the reference's Lanczos (scipy sparse products) on
    the host cores for the same matrix."""
    import torch
    import umapcu
    torch.cuda.set_device(local_rank)
    seed = args.seed + rank
    prob = make_problem(wl, seed)
    g = prob["graph"]
    warm = max(3, args.warmup)
    for _ in range(warm):
        umapcu.spectral_layout(g, 2, seed=seed)
    times = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        y = umapcu.spectral_layout(g, 2, seed=seed)
        times.append(time.perf_counter() - t0)
    sec = float(np.median(times))
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import scipy.sparse as sp
        from oracle import oracle as O
        n = wl["n"]
        t0 = time.perf_counter()
        r, c, v = (np.asarray(g.row_indices), np.asarray(g.col_indices), np.asarray(g.values, np.float64))
        A = sp.csr_matrix((v, (r, c)), shape=(n, n))
        deg = np.asarray(A.sum(1)).ravel()
        dis = np.where(deg > 1e-8, 1.0 / np.sqrt(deg), 0.0)
        M = -(sp.diags(dis) @ A @ sp.diags(dis))
        M.setdiag(0.0)
        O.lanczos_smallest(M.tocsr(), 3, O.splitmix_start(n, seed))
        csec = time.perf_counter() - t0
        cpu = {"value": csec, "unit": "s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": "the whole matrix and eigen-solve, numpy/scipy restatement (layout scaling not timed)"}
    if rank == 0:
        out = {"metric": "UMAP spectral init time (1M pts)", "value": sec, "unit": "s", "n_gpus": world,
               "steps": len(times), "warmup": warm, "ms_per_step": round(sec * 1e3, 3), "higher_is_better": False,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": f"spectral: {wl['desc']}", "n_points": wl["n"],
                          "nnz": int(np.asarray(g.row_indices).size)},
               "cpu_baseline": cpu, "finite": bool(np.isfinite(y).all())}
        print(json.dumps(out), flush=True)


def run_reference(args, wl, world):
    """The reference's parallel-Adam CPU optimiser (umap_optimisers.rs:
    1170-1492, restated in oracle/) on all host cores: every step is one
    whole run of the workload's epochs from the initial embedding, epoch loop
    timed. Loads no umapcu code: inputs come from umapdata and the oracle."""
    if wl["kind"] in ("batch", "serve") or wl.get("spectral"):
        print(json.dumps({"impl": "reference", "unavailable": f"workload {args.workload} has no counterpart in "
                          "the reference (it optimises one embedding per call)"}), flush=True)
        return
    from oracle import oracle as O
    seed = args.seed
    prob = make_reference_problem(wl, seed)
    stt, csr = O.csr_from_graph(wl["n"], prob["ptr"], prob["col"], prob["w"])
    updates = int(active_edges_per_epoch(csr["eps"], wl["n_epochs"]).sum())
    threads = os.cpu_count() or 1
    run = lambda k: cpu_full_runs(prob["ptr"], prob["col"], prob["w"], prob["params"], prob["init"], prob["dens"],
                                  seed, k, threads, wl["n_epochs"])
    run(args.warmup)
    secs = run(args.steps)
    total = float(np.sum(secs))
    value = args.steps * updates / total
    sample = (f"whole {wl['n_epochs']}-epoch runs of the oracle's adam_parallel restatement from the U(-10,10) "
              f"initial embedding, epoch loop only, one run per step ({updates} edge-updates per run, "
              f"{min(secs):.2f}-{max(secs):.2f} s)")
    out = {"metric": metric_of(wl), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(total / args.steps * 1e3, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": config_of(args, wl),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
