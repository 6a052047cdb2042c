"""kNN cache file in NumPy: the format umapcu_knn_save / umapcu_knn_load use
(include/umapcu.h), readable and writable without the CUDA library.

Little-endian. A 48-byte header {char magic[8] = "UMAPKNN\\0", u32 version = 1,
u32 metric, u64 n, u32 k, u32 flags (bit 0: self excluded), u64 checksum,
u64 reserved = 0}, then idx i32 [n * k], then dist f32 [n * k]. The checksum
is FNV-1a 64 over the payload bytes (idx then dist), evaluated here by a
numba-compiled loop. Loading checks magic, version, sizes, trailing bytes,
checksum and index range, and raises ValueError on any mismatch.
"""
from __future__ import annotations

import os

import numpy as np

MAGIC = b"UMAPKNN\x00"
HEADER = np.dtype([("magic", "S8"), ("version", "<u4"), ("metric", "<u4"), ("n", "<u8"), ("k", "<u4"),
                   ("flags", "<u4"), ("checksum", "<u8"), ("reserved", "<u8")])
assert HEADER.itemsize == 48
METRIC_EUCLIDEAN_SQ, METRIC_COSINE = 0, 1
_FNV_BASIS = 0xCBF29CE484222325
_FNV_PRIME = 0x100000001B3
_fnv = None


def _fnv_kernel():
    global _fnv
    if _fnv is None:
        import numba

        @numba.njit(cache=False, nogil=True)
        def fnv(h, b):
            p = np.uint64(_FNV_PRIME)
            for i in range(b.size):
                h = (h ^ np.uint64(b[i])) * p
            return h

        _fnv = fnv
    return _fnv


def fnv1a64(*arrays) -> int:
    """FNV-1a 64 over the bytes of the arrays, in order."""
    f = _fnv_kernel()
    h = np.uint64(_FNV_BASIS)
    for a in arrays:
        h = np.uint64(int(f(h, np.ascontiguousarray(a).view(np.uint8).ravel())) & 0xFFFFFFFFFFFFFFFF)
    return int(h)


def save(path: str, knn_idx, knn_dist, metric: int = METRIC_EUCLIDEAN_SQ) -> None:
    """Writes a kNN cache file (self excluded)."""
    i = np.ascontiguousarray(knn_idx, dtype="<i4")
    d = np.ascontiguousarray(knn_dist, dtype="<f4")
    if i.shape != d.shape or i.ndim != 2 or i.shape[0] == 0 or i.shape[1] == 0:
        raise ValueError("knn_idx and knn_dist must both be non-empty [n, k] arrays")
    if metric not in (METRIC_EUCLIDEAN_SQ, METRIC_COSINE):
        raise ValueError("unknown metric")
    h = np.zeros(1, HEADER)
    h["magic"], h["version"], h["metric"] = MAGIC, 1, metric
    h["n"], h["k"], h["flags"] = i.shape[0], i.shape[1], 1
    h["checksum"] = fnv1a64(i, d)
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(i.tobytes())
        f.write(d.tobytes())


def load(path: str):
    """-> (idx int32 [n, k], dist float32 [n, k], metric)."""
    with open(path, "rb") as f:
        raw = f.read(48)
        if len(raw) != 48:
            raise ValueError("truncated header")
        h = np.frombuffer(raw, HEADER)[0]
        n, k = int(h["n"]), int(h["k"])
        if (bytes(h["magic"]).ljust(8, b"\x00") != MAGIC or int(h["version"]) != 1 or int(h["metric"]) > 1
                or n == 0 or k == 0 or n > 0xFFFFFFFF):
            raise ValueError("not a kNN cache file (magic, version, metric or sizes)")
        m = n * k
        i = np.fromfile(f, dtype="<i4", count=m)
        d = np.fromfile(f, dtype="<f4", count=m)
        if i.size != m or d.size != m or f.read(1):
            raise ValueError("payload size does not match the header")
    if fnv1a64(i, d) != int(h["checksum"]):
        raise ValueError("checksum mismatch")
    if m and (i.min() < 0 or i.max() >= n):
        raise ValueError("neighbour index out of range")
    return i.reshape(n, k), d.reshape(n, k), int(h["metric"])


def header(path: str):
    """-> (n, k, metric) after checking magic and version."""
    with open(path, "rb") as f:
        h = np.frombuffer(f.read(48), HEADER)[0]
    if bytes(h["magic"]).ljust(8, b"\x00") != MAGIC or int(h["version"]) != 1:
        raise ValueError("not a kNN cache file")
    return int(h["n"]), int(h["k"]), int(h["metric"])


def exists(path: str) -> bool:
    return os.path.exists(path)
