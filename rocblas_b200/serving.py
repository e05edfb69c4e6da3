"""Continuous-batching TRSM server on one GPU (the native loop rocblas_b200_server_*).

Requests (dtype, m, n, a resident-A key or a fresh A) arrive over time.  The server
(`csrc/server.cuh`, C++):

* owns one device arena of the HBM budget; resident A matrices and their inverted 128 x 128
  diagonal blocks (invA, the rocblas_trsm_ex format) live there and are reused for every
  request on that A;
* admits a request in arrival order once its memory (B, and a fresh A with its invA) fits the
  budget; a request that cannot fit yet waits without blocking the loop;
* collects admitted requests of one dtype until a stream is free and the window has passed,
  so while the GPU is busy the next collection grows (continuous batching); one collection is
  one variable-size batched solve (rocblas_b200_?trsm_vbatched_ex: systems up to k = 512 on
  the strip solver's size classes, larger ones on the chain solve);
* completes a collection when its event has fired, frees its memory and records each
  request's latency (completion - arrival, host steady clock).

This module builds the request list, the data the requests bring (cut from fixed device pools
by each request's seed) and hands everything to the native loop.  The kernels a request runs
depend only on that request, never on what else is in flight, so a result is bitwise the same
alone and in the mix.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch

from . import RocblasError, check, datatype_f32_r, datatype_f64_r, lib
from .workloads import condition_band_lower_torch

SMALL_K = 512  # systems above this order need invA (the chain solve of the variable-size batch)
TORCH_DT = {"d": torch.float64, "s": torch.float32}
ESIZE = {"d": 8, "s": 4}
DATATYPE = {"d": datatype_f64_r, "s": datatype_f32_r}
FRESH_MAX = 8192  # order of the pool that fresh A matrices are cut from

REQUEST_DTYPE = np.dtype([("arrival_s", np.float64), ("dtype", np.int32), ("m", np.int32),
                          ("n", np.int32), ("resident", np.int32), ("B_src", np.uint64),
                          ("A_src", np.uint64), ("lda_src", np.int32), ("reserved", np.int32),
                          ("X_dst", np.uint64)])
STATS_DTYPE = np.dtype([("wall_s", np.float64), ("peak_bytes", np.int64), ("collections", np.int64),
                        ("largest_collection", np.int64), ("kernel_launches", np.int64)])
assert REQUEST_DTYPE.itemsize == 56 and STATS_DTYPE.itemsize == 40


@dataclass
class Request:
    rid: int
    arrival: float              # seconds after the start of the run
    dtype: str                  # "d" or "s"
    m: int
    n: int
    a_key: Optional[int]        # resident A, or None for a fresh A
    seed: int
    kband: int = 0              # condition band of a resident (informational for fresh A)
    # filled in by the server when results are kept
    B: Optional[torch.Tensor] = None


@dataclass
class Resident:
    key: int
    m: int
    index: Dict[str, int] = field(default_factory=dict)           # server index per dtype
    A: Dict[str, torch.Tensor] = field(default_factory=dict)      # host-side copies (optional)


class TrsmServer:
    def __init__(self, device="cuda", hbm_budget=120_000_000_000, n_streams=2, window_us=200.0,
                 max_batch=4096, keep_resident_copies=False, payload_on_host=False):
        self.dev = torch.device(device)
        if self.dev.index is None:
            self.dev = torch.device("cuda", torch.cuda.current_device())
        torch.cuda.set_device(self.dev)
        self.budget_bytes = int(hbm_budget)
        self.keep_copies = keep_resident_copies
        self._srv = ctypes.c_void_p()
        check("server_create", lib().rocblas_b200_server_create(
            ctypes.byref(self._srv), self.budget_bytes, n_streams, float(window_us), max_batch))
        self.residents: Dict[int, Resident] = {}
        self.last_stats = None
        # request payloads are cut from fixed pools (a stand-in for data that arrives with the
        # request): B from U(-1,1) values; a fresh A is a principal submatrix of a lower
        # triangle built by the drop-in recipe (off-diagonals U(-1,1)/FRESH_MAX, diagonal
        # 1.5 + U(-1,1)/FRESH_MAX), at an offset given by the request's seed.  With
        # payload_on_host the pools are pinned host memory: the server's gather launch then
        # reads each request's B and fresh A across PCIe (mapped host memory), inside the
        # request's measured latency, as data arriving from the host would be.
        g = torch.Generator(device=self.dev)
        g.manual_seed(12345)
        self.pool = {"d": torch.rand((1 << 27) + 4096, generator=g, device=self.dev,
                                     dtype=torch.float64) * 2 - 1}
        self.pool["s"] = self.pool["d"].to(torch.float32)
        F = (torch.rand(FRESH_MAX, FRESH_MAX, generator=g, device=self.dev, dtype=torch.float64) * 2 - 1)
        F *= 1.0 / FRESH_MAX
        F.diagonal().add_(1.5)
        self.fresh = {"d": F, "s": F.to(torch.float32)}  # (col, row) storage: column-major ld FRESH_MAX
        self.payload_on_host = payload_on_host
        if payload_on_host:
            self.pool = {k: v.cpu().pin_memory() for k, v in self.pool.items()}
            self.fresh = {k: v.cpu().pin_memory() for k, v in self.fresh.items()}
        torch.cuda.synchronize(self.dev)

    # ---- resident matrices ------------------------------------------------------------
    def add_resident(self, key, m, kband, seed, dtypes=("d", "s")):
        """A resident lower-triangular A (condition-band recipe): the server copies it into its
        arena and builds its invA."""
        At, _ = condition_band_lower_torch(m, 1, kband, seed, device=self.dev)
        r = Resident(key, m)
        for dt in dtypes:
            A = At.to(TORCH_DT[dt]).contiguous()
            idx = ctypes.c_int(-1)
            check("server_add_resident", lib().rocblas_b200_server_add_resident(
                self._srv, DATATYPE[dt], m, ctypes.c_void_p(A.data_ptr()), m, ctypes.byref(idx)))
            r.index[dt] = idx.value
            if self.keep_copies:
                r.A[dt] = A
        torch.cuda.synchronize(self.dev)
        self.residents[key] = r
        return r

    # ---- request data ------------------------------------------------------------------
    def payload_B(self, q: Request):
        """The right-hand sides request q brings (a view of the pool), (n, m) column-major."""
        pool = self.pool[q.dtype]
        count = q.m * q.n
        off = (q.seed * 2654435761) % (pool.numel() - count)
        return pool[off: off + count].view(q.n, q.m)

    def fresh_offset(self, q: Request):
        return ((q.seed + 1) * 40503) % (FRESH_MAX - q.m + 1)

    def payload_A(self, q: Request):
        """The lower triangle a fresh request q brings: F[o:o+m, o:o+m], as a (m, m) view of
        the column-major pool (rows of the view are columns of A)."""
        o = self.fresh_offset(q)
        return self.fresh[q.dtype][o: o + q.m, o: o + q.m]

    @property
    def used(self):
        b = ctypes.c_size_t(0)
        check("server_used_bytes", lib().rocblas_b200_server_used_bytes(self._srv, ctypes.byref(b)))
        return b.value

    def set_budget(self, nbytes):
        check("server_set_budget", lib().rocblas_b200_server_set_budget(self._srv, int(nbytes)))
        self.budget_bytes = int(nbytes)

    def request_bytes(self, q: Request):
        """Arena bytes request q holds from admission to completion (256-byte blocks)."""
        r = lambda b: (max(b, 1) + 255) // 256 * 256  # noqa: E731
        es = ESIZE[q.dtype]
        b = r(q.m * q.n * es)
        if q.a_key is None:
            b += r(q.m * q.m * es)
            if q.m > SMALL_K:
                b += r(128 * q.m * es)
        return b

    # ---- the loop ----------------------------------------------------------------------
    def run(self, requests: List[Request], keep_results=False):
        """Serve `requests` (any order; served by arrival).  Returns per-request latencies in
        seconds, in the order of `requests`; with keep_results each request's solution is left
        in q.B."""
        order = sorted(range(len(requests)), key=lambda i: requests[i].arrival)
        rec = np.zeros(len(order), dtype=REQUEST_DTYPE)
        for j, i in enumerate(order):
            q = requests[i]
            es = ESIZE[q.dtype]
            B = self.payload_B(q)
            if q.a_key is not None:
                res, A_src, lda = self.residents[q.a_key].index[q.dtype], 0, q.m
            else:
                o = self.fresh_offset(q)
                F = self.fresh[q.dtype]
                res, A_src, lda = -1, F.data_ptr() + (o + o * FRESH_MAX) * es, FRESH_MAX
            X = 0
            if keep_results:
                q.B = torch.empty(q.n, q.m, dtype=TORCH_DT[q.dtype], device=self.dev)
                X = q.B.data_ptr()
            rec[j] = (q.arrival, DATATYPE[q.dtype], q.m, q.n, res, B.data_ptr(), A_src, lda, 0, X)
        lat = np.zeros(len(order), dtype=np.float64)
        stats = np.zeros(1, dtype=STATS_DTYPE)
        torch.cuda.synchronize(self.dev)
        st = lib().rocblas_b200_server_run(self._srv, ctypes.c_void_p(rec.ctypes.data), len(order),
                                           ctypes.c_void_p(lat.ctypes.data),
                                           ctypes.c_void_p(stats.ctypes.data))
        if st != 0:
            raise RocblasError("rocblas_b200_server_run", st)
        self.last_stats = {k: stats[0][k].item() for k in STATS_DTYPE.names}
        out = np.zeros(len(requests))
        out[np.array(order, dtype=np.int64)] = lat
        return out

    def close(self):
        if self._srv:
            lib().rocblas_b200_server_destroy(self._srv)
            self._srv = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_requests(n_requests, rate, seed, resident_sizes, reuse=0.6, fp64=0.7, m_range=(64, 8192),
                  n_range=(1, 512)):
    """Poisson arrivals at `rate` per second; m, n log-uniform; dtype 70/30; a fraction
    `reuse` of the requests use one of the resident matrices (whose size sets m)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    out = []
    keys = list(resident_sizes.keys())
    for r in range(n_requests):
        dt = "d" if rng.random() < fp64 else "s"
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        if rng.random() < reuse and keys:
            key = keys[int(rng.integers(0, len(keys)))]
            m = resident_sizes[key]
            out.append(Request(r, float(t[r]), dt, m, n, key, int(rng.integers(1 << 30))))
        else:
            m = int(round(math.exp(rng.uniform(math.log(m_range[0]), math.log(min(m_range[1], FRESH_MAX))))))
            out.append(Request(r, float(t[r]), dt, m, n, None, int(rng.integers(1 << 30)),
                               kband=int(rng.choice([0, 2, 4]))))
    return out
