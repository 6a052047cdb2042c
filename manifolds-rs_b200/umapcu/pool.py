"""Placement of the batched and served forms over several GPUs.

The batched form (one persistent launch over many independent layouts) and
the served form (continuous batching of layout jobs) are both sets of
independent problems, so they scale over GPUs by placing whole problems on
devices: no data moves between GPUs and no collective runs. Neither form
has a counterpart in the reference, which optimises one embedding per call
(optimise_embedding_adam_gpu, src/training/umap_optimiser_gpu.rs:1302-1369)
on one device.

* ``lpt_partition``: a static placement of weighted problems over bins
  (longest processing time first), used to split a batch -- or a bench
  rank's share of one -- by estimated work.
* ``BatchPool``: one ``UmapBatch`` per device over an LPT partition of the
  problems by edge-update work; the devices' runs proceed concurrently.
* ``ServerPool``: one ``UmapServer`` per device; every submitted job goes to
  the healthy device with the most free admission budget (the pool's own
  account of the jobs it placed there and has not collected, in the servers'
  budget unit, ``server_job_bytes``). A device whose server refuses a job
  for lack of budget is passed over for that job; one whose server fails to
  take it at all is taken out of the rotation; a job fails alone.

The per-device objects are created with the device made current
(``set_device``), as the library's entry points bind to the calling
thread's current device; tests substitute host-side fakes through the
``backends`` / ``factory`` arguments.
"""
from __future__ import annotations

import threading
from typing import Callable, Optional, Sequence

import numpy as np

from . import (CAPACITY, NEG_REF_HASH, Adjacency, ManifoldsError, UmapBatch, UmapOptimParams, UmapServer, _adj,
               device_count, server_job_bytes, set_device)


def lpt_partition(weights: Sequence[float], n_bins: int):
    """Longest-processing-time-first placement: items in decreasing weight
    (ties by index), each onto the bin with the smallest total so far (ties
    by bin index). -> list of n_bins ascending index lists. Deterministic,
    so every process of a multi-process run computes the same placement."""
    if n_bins <= 0:
        raise ValueError("n_bins must be positive")
    w = np.asarray(weights, np.float64)
    order = sorted(range(w.size), key=lambda i: (-w[i], i))
    load = np.zeros(n_bins)
    bins = [[] for _ in range(n_bins)]
    for i in order:
        b = int(np.argmin(load))
        bins[b].append(i)
        load[b] += w[i]
    return [sorted(b) for b in bins]


def _devices(devices):
    if devices is not None:
        return list(devices)
    n = device_count()
    if n == 0:
        raise ManifoldsError(8, "no CUDA device")
    return list(range(n))


class BatchPool:
    """The batched form over several devices (see the module docstring).
    Results equal a single UmapBatch's (each problem's equals its own
    single-problem run)."""

    def __init__(self, embds, graphs, params, seeds, devices=None, sampler: int = NEG_REF_HASH,
                 factory: Optional[Callable] = None):
        P = len(embds)
        if not (len(graphs) == P and len(seeds) == P):
            raise ManifoldsError(7, "embds, graphs and seeds must have one entry per problem")
        self.devices = _devices(devices)
        plist = params if isinstance(params, (list, tuple)) else [params] * P
        adjs = [_adj(g) for g in graphs]
        work = [float(a.col.size) * max(1, int(q.n_epochs)) for a, q in zip(adjs, plist)]
        self.shares = lpt_partition(work, len(self.devices))
        self.where = {}
        self.batches = []
        self._own = factory is None  # real batches: calls need their device current
        make = factory or self._make
        for d, share in zip(self.devices, self.shares):
            for k, i in enumerate(share):
                self.where[i] = (len(self.batches), k)
            self.batches.append(make(d, [embds[i] for i in share], [adjs[i] for i in share],
                                     [plist[i] for i in share], [seeds[i] for i in share], sampler)
                                if share else None)

    @staticmethod
    def _make(device, embds, adjs, params, seeds, sampler):
        set_device(device)
        return UmapBatch(embds, adjs, params, seeds, sampler)

    def _each(self, fn):
        """fn(batch) on every device's batch concurrently (the library's
        calls release the GIL); -> results in device order."""
        out = [None] * len(self.batches)
        err = []

        def work(k, b, d):
            try:
                if self._own:
                    set_device(d)
                out[k] = fn(b)
            except Exception as e:  # noqa: BLE001 - re-raised below
                err.append(e)

        ts = [threading.Thread(target=work, args=(k, b, d)) for k, (b, d) in
              enumerate(zip(self.batches, self.devices)) if b is not None]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if err:
            raise err[0]
        return out

    def autotune(self):
        return self._each(lambda b: b.autotune())

    def run(self, mode: int = 0):
        """All epochs of every problem on every device; -> per-device ms
        (None for a device without problems)."""
        return self._each(lambda b: b.run(mode))

    def read(self, p: int) -> np.ndarray:
        k, i = self.where[p]
        return self.batches[k].read(i)

    def close(self):
        for b in self.batches:
            if b is not None:
                b.close()
        self.batches = []


class ServerPool:
    """The served form over several devices (see the module docstring)."""

    def __init__(self, budget_bytes: int, max_jobs: int = 4096, tick_epochs: int = 10, n_dim: int = 2,
                 devices=None, backends=None):
        if backends is not None:
            self.devices = list(range(len(backends)))
            self.servers = list(backends)
        else:
            self.devices = _devices(devices)
            self.servers = []
            for d in self.devices:
                set_device(d)
                self.servers.append(UmapServer(budget_bytes, max_jobs, tick_epochs, n_dim))
        self.budget = [int(budget_bytes)] * len(self.servers)
        self.outstanding = [0] * len(self.servers)
        self.placed = [0] * len(self.servers)
        self.healthy = [True] * len(self.servers)
        self.n_dim = n_dim
        self._jobs = {}  # pool ticket -> (server index, server ticket, bytes)
        self._next = 1
        self._mu = threading.Lock()

    def _order(self):
        """Healthy devices by decreasing free budget (ties: fewer placed jobs,
        then device order)."""
        idx = [k for k in range(len(self.servers)) if self.healthy[k]]
        return sorted(idx, key=lambda k: (-(self.budget[k] - self.outstanding[k]), self.placed[k], k))

    def submit(self, embd, graph, params: UmapOptimParams, seed: int = 42, sampler: int = NEG_REF_HASH) -> int:
        a = graph if isinstance(graph, Adjacency) else _adj(graph)
        e = np.asarray(embd)
        need = server_job_bytes(e.shape[0], e.shape[1], int(a.col.size), int(params.n_epochs))
        last = None
        with self._mu:
            order = self._order()
        for k in order:
            try:
                t = self.servers[k].submit(embd, a, params, seed, sampler)
            except ManifoldsError as ex:
                last = ex
                if ex.status != CAPACITY:
                    with self._mu:
                        self.healthy[k] = False  # the device refused the job outright
                continue
            with self._mu:
                self.outstanding[k] += need
                self.placed[k] += 1
                ticket = self._next
                self._next += 1
                self._jobs[ticket] = (k, t, need)
            return ticket
        raise last if last is not None else ManifoldsError(8, "no healthy device")

    def device_of(self, ticket: int) -> int:
        return self.devices[self._jobs[ticket][0]]

    def poll(self, ticket: int) -> int:
        k, t, _ = self._jobs[ticket]
        return self.servers[k].poll(t)

    def cancel(self, ticket: int):
        k, t, _ = self._jobs[ticket]
        self.servers[k].cancel(t)

    def wait(self, ticket: int):
        """-> (embedding, latency_s, queue_s) like UmapServer.wait; the job's
        budget share is released whatever its outcome."""
        with self._mu:
            k, t, need = self._jobs.pop(ticket)
        try:
            return self.servers[k].wait(t)
        finally:
            with self._mu:
                self.outstanding[k] -= need

    def stats(self):
        return [dict(device=d, healthy=h, placed=p, **s.stats()) for d, h, p, s in
                zip(self.devices, self.healthy, self.placed, self.servers)]

    def close(self):
        for s in self.servers:
            s.close()
        self.servers = []
