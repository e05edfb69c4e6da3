"""Continuous-batching TRSM server on one GPU.

Requests (dtype, m, n, a resident-A key or a fresh A) arrive over time.  The server:

* admits a request once its device memory (B, a fresh A, workspace share) fits in the HBM
  budget, in arrival order; a request that cannot fit yet waits without blocking the loop;
* keeps resident A matrices and their inverted 128 x 128 diagonal blocks (invA, the
  rocblas_trsm_ex format) on the device and reuses them for every request on that A;
* collects admitted requests of one dtype for up to `window_us` and solves each collection
  with one variable-size batched call (rocblas_b200_?trsm_vbatched_ex): systems up to k = 512
  on the strip solver's size classes, larger ones on the chain solve with the resident (or a
  freshly built) invA, all of them in a few persistent launches;
* runs launches on a pool of streams, each with its own rocblas handle, so work admitted
  while other work is on the GPU overlaps with it;
* completes a request when its launch's event has fired, frees its budget and records its
  latency (completion - arrival, host clock).

The kernels a request runs depend only on that request (its sizes and route), never on what
else is in flight, so a result is bitwise the same alone and in the mix.
"""
from __future__ import annotations

import collections
import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch

from . import (
    DIAG, SIDE, TRANS, UPLO, Handle, check, datatype_f32_r, datatype_f64_r, lib, status_success,
)
from .workloads import condition_band_lower_torch

SMALL_K = 512  # systems above this order need invA (the chain solve of the variable-size batch)
TORCH_DT = {"d": torch.float64, "s": torch.float32}
ESIZE = {"d": 8, "s": 4}


@dataclass
class Request:
    rid: int
    arrival: float              # seconds after the start of the run
    dtype: str                  # "d" or "s"
    m: int
    n: int
    a_key: Optional[int]        # resident A, or None for a fresh A
    seed: int
    kband: int = 0              # condition band of a fresh A
    # filled in by the server
    B: Optional[torch.Tensor] = None
    A: Optional[torch.Tensor] = None
    admitted: float = -1.0
    done: float = -1.0
    bytes: int = 0


@dataclass
class Resident:
    key: int
    m: int
    A: Dict[str, torch.Tensor] = field(default_factory=dict)      # per dtype, (m, m) col-major
    invA: Dict[str, torch.Tensor] = field(default_factory=dict)   # per dtype, 128 * m elements


def _p(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


class TrsmServer:
    def __init__(self, device="cuda", hbm_budget=120 << 30, n_streams=2, window_us=200.0,
                 max_batch=4096):
        self.dev = torch.device(device)
        self.budget = int(hbm_budget)
        self.used = 0
        self.window = window_us * 1e-6
        self.max_batch = max_batch
        self.streams = [torch.cuda.Stream(self.dev) for _ in range(n_streams)]
        self.handles = []
        for s in self.streams:
            h = Handle()
            h.set_stream(ctypes.c_void_p(s.cuda_stream))
            self.handles.append(h)
        self.rr = 0
        self.residents: Dict[int, Resident] = {}
        # per stream, launches complete in order: (event, [requests], keepalive)
        self.inflight = [collections.deque() for _ in self.streams]
        # collections in flight at once: one per stream.  Each collection's persistent kernels
        # fill the GPU, so a new collection is formed only when a stream frees up; requests
        # that arrive meanwhile join the next, larger collection (continuous batching).
        self.max_inflight = n_streams
        self.one = {"d": ctypes.c_double(1.0), "s": ctypes.c_float(1.0)}
        # request payloads are cut from a fixed pool of U(-1,1) values (a stand-in for data that
        # arrives with the request): a request's B and fresh A depend only on its seed
        g = torch.Generator(device=self.dev)
        g.manual_seed(12345)
        self.pool = {"d": torch.rand((1 << 27) + 4096, generator=g, device=self.dev,
                                     dtype=torch.float64) * 2 - 1}
        self.pool["s"] = self.pool["d"].to(torch.float32)

    # ---- resident matrices ------------------------------------------------------------
    def add_resident(self, key, m, kband, seed, dtypes=("d", "s")):
        """Build a resident lower-triangular A (condition-band recipe) and its invA."""
        At, _ = condition_band_lower_torch(m, 1, kband, seed, device=self.dev)
        r = Resident(key, m)
        for dt in dtypes:
            A = At.to(TORCH_DT[dt]).contiguous()
            inv = torch.zeros(128 * m, dtype=TORCH_DT[dt], device=self.dev)
            self._build_invA(A, m, inv, dt)
            r.A[dt], r.invA[dt] = A, inv
            self.used += A.numel() * ESIZE[dt] + inv.numel() * ESIZE[dt]
        torch.cuda.synchronize(self.dev)
        self.residents[key] = r
        return r

    def _build_invA(self, A, m, inv, dt):
        L = lib()
        fn = L.rocblas_dtrtri_strided_batched if dt == "d" else L.rocblas_strtri_strided_batched
        h = self.handles[0]
        nfull, rem = divmod(m, 128)
        es = ESIZE[dt]
        if nfull:
            check("trtri", fn(h.value, UPLO["L"], DIAG["N"], 128, _p(A), m, 128 * m + 128, _p(inv), 128,
                              128 * 128, nfull))
        if rem:
            off_a = nfull * 128 * m + nfull * 128
            check("trtri", fn(h.value, UPLO["L"], DIAG["N"], rem, ctypes.c_void_p(A.data_ptr() + off_a * es),
                              m, 0, ctypes.c_void_p(inv.data_ptr() + nfull * 128 * 128 * es), 128, 0, 1))

    # ---- per-request memory ------------------------------------------------------------
    def _request_bytes(self, q: Request):
        es = ESIZE[q.dtype]
        b = q.m * q.n * es
        if q.a_key is None:
            b += q.m * q.m * es
        if q.m > SMALL_K:
            b += 128 * q.m * es  # workspace share (invA of a fresh A)
        return b

    def _cut(self, dt, count, seed):
        pool = self.pool[dt]
        span = pool.numel() - count  # > 0: the pool holds the largest A (8192^2) and more
        off = (seed * 2654435761) % span
        return pool[off: off + count]

    def _materialise(self, q: Request, stream):
        """Create B (and a fresh A) for an admitted request on `stream`: B is cut from the
        pool; a fresh lower-triangular A has off-diagonals U(-1,1)/m and diagonal 1.5 +
        U(-1,1)/m (the drop-in recipe's conditioning)."""
        with torch.cuda.stream(stream):
            q.B = self._cut(q.dtype, q.m * q.n, q.seed).clone().view(q.n, q.m)
            if q.a_key is None:
                A = self._cut(q.dtype, q.m * q.m, q.seed + 1) * (1.0 / q.m)
                A.view(q.m, q.m).diagonal().add_(1.5)
                q.A = A

    # ---- launches ----------------------------------------------------------------------
    def _next(self):
        """A stream with nothing in flight (there is one while fewer collections than streams
        are in flight), else the next one in turn."""
        i = next((j for j, d in enumerate(self.inflight) if not d), self.rr)
        self.rr = (i + 1) % len(self.streams)
        self._cur = i
        return self.streams[i], self.handles[i]

    def _n_inflight(self):
        return sum(len(d) for d in self.inflight)

    def _alpha(self, dt):
        return ctypes.cast(ctypes.byref(self.one[dt]), ctypes.c_void_p)

    def _fresh_invA(self, q: Request, h, stream):
        """invA of a fresh A (k > SMALL_K) on the collection's stream, the trsm_ex format."""
        L = lib()
        fn = L.rocblas_dtrtri_strided_batched if q.dtype == "d" else L.rocblas_strtri_strided_batched
        m, es = q.m, ESIZE[q.dtype]
        with torch.cuda.stream(stream):
            inv = torch.zeros(128 * m, dtype=TORCH_DT[q.dtype], device=self.dev)
        nfull, rem = divmod(m, 128)
        if nfull:
            check("trtri", fn(h.value, UPLO["L"], DIAG["N"], 128, _p(q.A), m, 128 * m + 128, _p(inv), 128,
                              128 * 128, nfull))
        if rem:
            off_a = nfull * 128 * m + nfull * 128
            check("trtri", fn(h.value, UPLO["L"], DIAG["N"], rem, ctypes.c_void_p(q.A.data_ptr() + off_a * es),
                              m, 0, ctypes.c_void_p(inv.data_ptr() + nfull * 128 * 128 * es), 128, 0, 1))
        return inv

    def _launch_group(self, group: List[Request], dt):
        """One variable-size batched call for a collection of admitted requests."""
        stream, h = self._next()
        keep = []
        with torch.cuda.stream(stream):
            for q in group:
                self._materialise(q, stream)
        rec = np.zeros(len(group), dtype=np.dtype([
            ("A", np.uint64), ("B", np.uint64), ("m", np.int32), ("n", np.int32), ("lda", np.int32),
            ("ldb", np.int32), ("side", np.int32), ("uplo", np.int32), ("trans", np.int32),
            ("diag", np.int32)]))
        invs = np.zeros(len(group), dtype=np.uint64)
        max_k, max_n = 1, 1
        for i, q in enumerate(group):
            if q.a_key is not None:
                r = self.residents[q.a_key]
                A, inv = r.A[dt], r.invA[dt]
            else:
                A = q.A
                inv = self._fresh_invA(q, h, stream) if q.m > SMALL_K else None
                if inv is not None:
                    keep.append(inv)
            rec[i] = (A.data_ptr(), q.B.data_ptr(), q.m, q.n, q.m, q.m, SIDE["L"], UPLO["L"], TRANS["N"],
                      DIAG["N"])
            invs[i] = inv.data_ptr() if inv is not None else 0
            max_k = max(max_k, q.m)
            max_n = max(max_n, q.n)
        host = torch.from_numpy(np.concatenate([rec.view(np.uint8), invs.view(np.uint8)])).pin_memory()
        with torch.cuda.stream(stream):
            dev = host.to(self.dev, non_blocking=True)
        nd = rec.nbytes
        fn = lib().rocblas_b200_dtrsm_vbatched_ex if dt == "d" else lib().rocblas_b200_strsm_vbatched_ex
        check("vbatched_ex (server)", fn(h.value, self._alpha(dt), _p(dev), ctypes.c_void_p(dev.data_ptr() + nd),
                                         len(group), max_k, max_n, None))
        ev = torch.cuda.Event()
        ev.record(stream)
        self.inflight[self._cur].append((ev, list(group), (host, dev, keep)))

    # ---- the loop ----------------------------------------------------------------------
    def run(self, requests: List[Request], keep_results=False):
        """Serve `requests` (sorted by arrival).  Returns per-request latencies in seconds."""
        reqs = sorted(requests, key=lambda q: q.arrival)
        for q in reqs:
            q.bytes = self._request_bytes(q)
            if q.bytes > self.budget - self.used:
                raise ValueError(f"request {q.rid} needs {q.bytes} B, more than the free budget")
        pending = collections.deque()
        window = {"d": collections.deque(), "s": collections.deque()}
        i = 0
        t0 = time.perf_counter()
        done = 0
        total = len(reqs)
        while done < total:
            now = time.perf_counter() - t0
            # arrivals
            while i < total and reqs[i].arrival <= now:
                pending.append(reqs[i])
                i += 1
            # admission in arrival order, within the HBM budget
            while pending and pending[0].bytes <= self.budget - self.used:
                q = pending.popleft()
                self.used += q.bytes
                q.admitted = now
                window[q.dtype].append(q)
            # a collection is launched when a stream is free and its window has closed (or it
            # is full, or no more requests will come); the oldest waiting dtype goes first
            while self._n_inflight() < self.max_inflight:
                ready = [dt for dt, dq in window.items()
                         if dq and (len(dq) >= self.max_batch or now - dq[0].admitted >= self.window
                                    or (i >= total and not pending))]
                if not ready:
                    break
                dt = min(ready, key=lambda d: window[d][0].admitted)
                dq = window[dt]
                group = [dq.popleft() for _ in range(min(len(dq), self.max_batch))]
                self._launch_group(group, dt)
            # completions: each stream's launches finish in order, so only heads are polled
            for dq in self.inflight:
                while dq and dq[0][0].query():
                    ev, group, _ = dq.popleft()
                    tdone = time.perf_counter() - t0
                    for q in group:
                        q.done = tdone
                        self.used -= q.bytes
                        if not keep_results:
                            q.B = None
                        q.A = None
                        done += 1
        torch.cuda.synchronize(self.dev)
        return np.array([q.done - q.arrival for q in reqs])

    def close(self):
        for h in self.handles:
            h.close()


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
            m = int(round(math.exp(rng.uniform(math.log(m_range[0]), math.log(m_range[1])))))
            out.append(Request(r, float(t[r]), dt, m, n, None, int(rng.integers(1 << 30)),
                               kband=int(rng.choice([0, 2, 4]))))
    return out
