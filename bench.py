"""TRSM benchmark: one JSON line on rank 0.

Headline workload: dtrsm side=L, uplo=L, transA=N, diag=N, m=16384, n=4096, alpha=1, lda=ldb=m,
solved by the refined precision form (rocblas_b200_dtrsm_refined: trailing updates from int8
slices on the tcgen05 tensor cores, FP64 diagonal blocks, then the test against the plain FP64
solve of sampled right-hand sides and, when it fails, FP64-residual corrections) and, beside it,
by the plain FP64 form (rocblas_dtrsm).  A is the condition-band recipe at k=0 (off-diagonal
N(0,1)/sqrt(m), diagonal 1 + U(0, 0.1)) with a NaN upper triangle; B ~ U(-1,1).  One step =
restore the right-hand side (a device copy of 512 MiB, inside the timed region) + one solve
through the C ABI.  A (2 GiB) and B (512 MiB) are larger than the 126 MB L2, so no flush is
needed between steps.  Errors are reported for that matrix and for matrices with singular values
graded from 1 to 10^-k, k in {0,2,4,6}, against the oracle's extended-precision X* and the host
FP64 CBLAS, with the refinement's iteration counts.  The end-to-end figure (`e2e`) calls
rocblas_b200_dtrsm_mixed_host on pinned host buffers (transfers inside the timed region).
Extras: the drop-in sweep (16 combinations, FP32 and FP64, 8192-sized), the variable-size and
strided batches, the serving loop, complex z/ctrsm.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: a single solve does not shard (replicas only), so N ranks each run their
own independent solve; `value` is the sum over ranks of m*n*k flops / the max-over-ranks time.
`--impl reference` times the host CBLAS trsm (OpenBLAS bundled with scipy, the library the
reference's ref_trsm wraps) on all host cores on the whole problem, every step.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M, N = 16384, 4096
FLOPS = float(M) * M * N  # m*n*k, k = m (clients/include/flops.hpp:722-725)

# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per launch, from one ncu capture
# of this command's own launches at the default size:
# the sliced GEMM averaged over the 7 launches of a precision-form solve, and the chain kernel
# of the plain solve (one launch per solve)
SLICED_TRAFFIC_PER_LAUNCH = 1.0795e9
SLICED_TRAFFIC_SOURCE = ("ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum of "
                         "`bench.py --no-extras --steps 2 --warmup 3`: 77 launches, mean per launch "
                         "(0.248 / 1.035 / 4.496 GB for the 4 / 2 / 1 launches of each solve)")
CRT_TRAFFIC_PER_LAUNCH = 1.91e9
CRT_TRAFFIC_SOURCE = ("ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum of `bench.py --case crt "
                      "--moduli 16` (CTA-pair form) at the solve's three update shapes (8192x4096x8192: "
                      "6.74 GB, 4096^3: 2.03 GB, 2048x4096x2048: 0.64 GB per launch), weighted by their "
                      "1 / 2 / 4 launches per solve (16384-deep exponent chunks)")
CHAIN_TRAFFIC_PER_LAUNCH = 35.57e9
CHAIN_TRAFFIC_SOURCE = ("same capture: the 8 plain-solve launches of trsm_chain_kernel (45.5 ms each); "
                        "A (1.07 GB) is streamed once per 64-column strip group")


METRIC = "dtrsm TFLOP/s (refined precision form, FP64 accuracy)"


def workload_name():
    return f"dtrsm L/L/N/N m={M} n={N} lda=ldb={M} alpha=1 (condition band k=0)"


def max_over_ranks(dist, value, device):
    """The largest of every rank's `value` (all ranks call it in the same order)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(units_per_rank, world, max_ms):
    """Whole-job rate of N independent replicas: all ranks' units over the slowest rank's time."""
    return units_per_rank * world / (max_ms * 1e-3)


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.dev)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    """The pool's measured peaks (HBM copy GB/s, bf16 dense TF/s burst and sustained)."""
    out = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
           "source": "fallback (earlier measurement on this pool)"}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        for k in ("hbm_gbs", "bf16_tflops", "bf16_tflops_sustained"):
            out[k] = float(d[k])
        out["source"] = "MEASURED_PEAKS.json"
    except (OSError, KeyError, ValueError):
        pass
    return out


def headline_slices(L, S):
    """The slice count a call with `S` uses (0: the tuning table's mixed_slices)."""
    if S:
        return S
    v = ctypes.c_int(0)
    assert L.rocblas_b200_get_tuning(b"mixed_slices", ctypes.byref(v)) == 0
    return v.value


def headline_engine(L, S):
    """The integer GEMM engine of the precision form's updates for a call with `S` (0: the
    tuning table's engine, the residue GEMM with mixed_moduli moduli unless that is 0; 1..8: the
    slice GEMM with S slices): {"engine", "moduli" | "slices", "kernel", "label"}."""
    nm = ctypes.c_int(0)
    assert L.rocblas_b200_get_tuning(b"mixed_moduli", ctypes.byref(nm)) == 0
    if S == 0 and nm.value > 0:
        return {"engine": "residue", "moduli": nm.value,
                "kernel": f"crt_gemm_kernel<{nm.value}> (tcgen05 kind::i8, {nm.value} residue products)",
                "label": f"int8 residue (CRT) tensor-core updates, {nm.value} moduli"}
    S_used = headline_slices(L, S)
    return {"engine": "slices", "slices": S_used,
            "kernel": f"ozaki_gemm_kernel<64,64,{S_used}> (tcgen05 kind::i8, {S_used} slices)",
            "label": f"int8-slice tensor-core updates, {S_used} slices"}


def kernel_timing(L, cls):
    """(total ms, total work, launches) of one kernel class since timing was enabled."""
    ms, work, n = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_int(0)
    assert L.rocblas_b200_kernel_timing_query(cls.encode(), ctypes.byref(ms), ctypes.byref(work),
                                              ctypes.byref(n)) == 0
    return ms.value, work.value, n.value


def fp64_peak_tflops(torch, dev):
    """Measured FP64 dense peak on this GPU: cuBLAS DGEMM 8192^3 (torch.matmul), best of 5."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12


def cpu_cblas_sample(A_host, B_host, ncols, threads):
    """Time host cblas_dtrsm on the first `ncols` right-hand sides; returns (TFLOP/s, s, X)."""
    import oracle

    oracle.cblas_set_threads(threads)
    Bs = np.array(B_host[:, :ncols], order="F", copy=True)  # the solve overwrites it
    # the host BLAS may read the unused triangle in blocked kernels: give it zeros there
    t0 = time.perf_counter()
    oracle.cblas_trsm_inplace("L", "L", "N", "N", 1.0, A_host, Bs)
    dt = time.perf_counter() - t0
    return float(M) * M * ncols / dt / 1e12, dt, Bs


def run_reference(args):
    """The reference arm: host CBLAS cblas_dtrsm (OpenBLAS, the library rocblas-test's
    ref_trsm wraps) on all host cores, on the whole headline problem (all N right-hand sides)
    per step; the reference's own GPU path is HIP and does not run here."""
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    import oracle

    threads = os.cpu_count() or 1
    m = M
    # host copy of the same recipe (numpy stream): lower triangle, zeros above for the CBLAS
    A, B = oracle.condition_band_problem(0, m, N, 0)
    A = np.asfortranarray(np.tril(np.nan_to_num(A, nan=0.0)))
    for _ in range(args.warmup):
        cpu_cblas_sample(A, B, N, threads)
    times = []
    for _ in range(args.steps):
        _, dt, _ = cpu_cblas_sample(A, B, N, threads)
        times.append(dt)
    tot = sum(times)
    val = float(m) * m * N * args.steps / tot / 1e12
    line = {
        "metric": METRIC, "value": val, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": workload_name(), "m": M, "n": N},
        "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": threads, "kind": "reference",
                         "sample": f"host cblas_dtrsm (OpenBLAS {oracle.cblas_config().split()[1]}) on "
                                   f"the whole problem per step (all {N} right-hand sides, m={M})"},
        "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def vbatched_workload(torch, dev, count, seed, dt):
    """The variable-size batch's systems: m log-uniform [16, 512], n uniform [1, 64], side and uplo uniform,
    transA N, diag N, A and B by the drop-in recipe, all in two device arrays; returns the
    device descriptor array (rocblas_b200_trsm_problem records) and the arrays behind it."""
    tdt, es = (torch.float64, 8) if dt == "d" else (torch.float32, 4)
    rng = np.random.default_rng(seed)
    ms = np.exp(rng.uniform(np.log(16), np.log(512), size=count)).astype(np.int64)
    ns = rng.integers(1, 65, size=count)
    sides = rng.choice([141, 142], size=count)
    uplos = rng.choice([121, 122], size=count)
    ks = np.where(sides == 141, ms, ns)
    order = np.argsort(ks, kind="stable")  # group equal k so that A is generated per k
    a_off = np.zeros(count, dtype=np.int64)
    b_off = np.zeros(count, dtype=np.int64)
    a_tot = b_tot = 0
    for i in order:
        a_off[i] = a_tot
        a_tot += int(ks[i]) ** 2
    for i in range(count):
        b_off[i] = b_tot
        b_tot += int(ms[i] * ns[i])
    Aar = torch.empty(a_tot, dtype=tdt, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    # per distinct k: off-diagonal U(-1,1)/k, diagonal 1 + U(0,1) (the drop-in recipe)
    uk, first = np.unique(ks[order], return_index=True)
    for j, k in enumerate(uk):
        lo = first[j]
        hi = first[j + 1] if j + 1 < len(uk) else count
        cnt = hi - lo
        base = int(a_off[order[lo]])
        blk = (torch.rand(cnt, int(k), int(k), generator=g, device=dev, dtype=torch.float64) * 2 - 1) / k
        idx = torch.arange(int(k), device=dev)
        blk[:, idx, idx] = 1.0 + torch.rand(cnt, int(k), generator=g, device=dev, dtype=torch.float64)
        Aar[base: base + cnt * int(k) * int(k)] = blk.reshape(-1).to(tdt)
    B0 = (torch.rand(b_tot, generator=g, device=dev, dtype=torch.float64) * 2 - 1).to(tdt)
    Bar = B0.clone()
    rec = np.zeros(count, dtype=np.dtype([
        ("A", np.uint64), ("B", np.uint64), ("m", np.int32), ("n", np.int32), ("lda", np.int32),
        ("ldb", np.int32), ("side", np.int32), ("uplo", np.int32), ("trans", np.int32),
        ("diag", np.int32)]))
    rec["A"] = Aar.data_ptr() + a_off * es
    rec["B"] = Bar.data_ptr() + b_off * es
    rec["m"], rec["n"], rec["lda"], rec["ldb"] = ms, ns, ks, ms
    rec["side"], rec["uplo"], rec["trans"], rec["diag"] = sides, uplos, 111, 131
    desc = torch.from_numpy(rec.view(np.uint8).copy()).to(dev)
    return {"desc": desc, "A": Aar, "B": Bar, "B0": B0, "m": ms, "n": ns, "k": ks, "es": es, "g": g}


def bench_batched(torch, rb, L, h, dev, hbm_gbs, count=20000, seed=2024):
    """The variable-size batch: `count` uneven systems (m log-uniform [16, 512], n uniform [1, 64], side and
    uplo uniform, transA N, diag N) through rocblas_b200_?trsm_vbatched, FP64 and FP32; plus
    the uniform strided batch (4096 x m=128, n=32) through rocblas_?trsm_strided_batched.
    Solves/s and algorithmic GB/s against the HBM roofline."""
    out = {}
    for dt, tdt in (("d", torch.float64), ("s", torch.float32)):
        w = vbatched_workload(torch, dev, count, seed, dt)
        desc, Aar, Bar, B0, ms, ns, ks, es, g = (w[k] for k in ("desc", "A", "B", "B0", "m", "n", "k", "es", "g"))
        alpha = ctypes.c_double(1.0) if dt == "d" else ctypes.c_float(1.0)
        ap = ctypes.cast(ctypes.byref(alpha), ctypes.c_void_p)
        fn = L.rocblas_b200_dtrsm_vbatched if dt == "d" else L.rocblas_b200_strsm_vbatched

        def run():
            st = fn(h.value, ap, ctypes.c_void_p(desc.data_ptr()), count, 512, None)
            assert st == 0, st

        for _ in range(3):
            Bar.copy_(B0)
            run()
        torch.cuda.synchronize(dev)
        times = []
        for _ in range(10):
            Bar.copy_(B0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run()
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        t = statistics.median(times) * 1e-3
        # the same call captured once into a CUDA graph and replayed (prepass and class
        # launches in one graph launch)
        cap = torch.cuda.Stream(dev)
        h.set_stream(ctypes.c_void_p(cap.cuda_stream))
        graph = torch.cuda.CUDAGraph()
        torch.cuda.synchronize(dev)
        with torch.cuda.graph(graph, stream=cap):
            run()
        h.set_stream(ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
        gtimes = []
        for r in range(11):
            Bar.copy_(B0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            graph.replay()
            e1.record()
            e1.synchronize()
            if r:
                gtimes.append(e0.elapsed_time(e1))
        del graph
        tg = statistics.median(gtimes) * 1e-3
        flops = float(np.sum(ms * ns * ks))
        nbytes = float(np.sum(es * (ks * (ks + 1) / 2 + 2 * ms * ns)))
        out[f"vbatched_{dt}"] = {"systems": count, "solves_per_s": count / t, "ms": t * 1e3,
                                 "graph_replay_ms": tg * 1e3, "graph_solves_per_s": count / tg,
                                 "tflops": flops / t / 1e12, "algorithmic_GBps": nbytes / t / 1e9,
                                 "hbm_frac": nbytes / t / 1e9 / hbm_gbs}
        del Aar, Bar, B0, desc, w
        # uniform strided batch: 4096 x (m=128, n=32), side L lower
        bc, m, n = 4096, 128, 32
        As = torch.rand(bc, m, m, generator=g, device=dev, dtype=torch.float64) * 2 - 1
        As /= m
        idx = torch.arange(m, device=dev)
        As[:, idx, idx] = 1.0 + torch.rand(bc, m, generator=g, device=dev, dtype=torch.float64)
        As = As.to(tdt).contiguous()
        Bs0 = (torch.rand(bc, n, m, generator=g, device=dev, dtype=torch.float64) * 2 - 1).to(tdt)
        Bs = Bs0.clone()
        sfn = L.rocblas_dtrsm_strided_batched if dt == "d" else L.rocblas_strsm_strided_batched

        def run_sb():
            st = sfn(h.value, 141, 122, 111, 131, m, n, ap, ctypes.c_void_p(As.data_ptr()), m, m * m,
                     ctypes.c_void_p(Bs.data_ptr()), m, m * n, bc)
            assert st == 0, st

        for _ in range(3):
            Bs.copy_(Bs0)
            run_sb()
        torch.cuda.synchronize(dev)
        times = []
        for _ in range(10):
            Bs.copy_(Bs0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run_sb()
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        t = statistics.median(times) * 1e-3
        nbytes = bc * es * (m * (m + 1) / 2 + 2 * m * n)
        out[f"strided_batched_{dt}"] = {"batch": bc, "m": m, "n": n, "solves_per_s": bc / t, "ms": t * 1e3,
                                        "tflops": bc * m * m * n / t / 1e12,
                                        "algorithmic_GBps": nbytes / t / 1e9,
                                        "hbm_frac": nbytes / t / 1e9 / hbm_gbs}
        del As, Bs, Bs0
    return out


SWEEP_SHAPES = ((8192, 8192), (8192, 512), (512, 8192))


def sweep_matrix(torch, dev, k, uplo, diag, tdt, g):
    """The drop-in recipe on the device: strictly-triangular entries U(-1,1)/k, diagonal
    1 + U(0,1), the other triangle NaN, and for diag U a NaN diagonal (it must not be read);
    returned as the (ncols, ld) view of column-major storage."""
    At = (torch.rand(k, k, generator=g, device=dev, dtype=torch.float64) * 2 - 1) / k
    At.diagonal().copy_(1.0 + torch.rand(k, generator=g, device=dev, dtype=torch.float64))
    # At[j, i] = A(i, j): A lower <=> At upper, so A's upper triangle is At's strict lower one
    mask = torch.ones(k, k, dtype=torch.bool, device=dev)
    mask = mask.tril_(-1) if uplo == "L" else mask.triu_(1)
    At.masked_fill_(mask, float("nan"))
    if diag == "U":
        At.diagonal().fill_(float("nan"))
    return At.to(tdt).contiguous()


def _timed_median(torch, fn, reset, reps):
    """Median of `reps` event-timed calls of fn after one untimed call; reset() before each
    call, outside the timing."""
    times = []
    for r in range(reps + 1):
        reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        if r:
            times.append(e0.elapsed_time(e1))
    return statistics.median(times) * 1e-3


def bench_sweep(torch, rb, L, h, dev, reps=3):
    """The drop-in sweep: rocblas_{d,s}trsm for all 16 side/uplo/trans/diag combinations at
    m = n = 8192 and the rectangular 8192 x 512 and 512 x 8192, alpha = 1, lda = k, ldb = m,
    plus rocblas_trsm_ex with a caller-supplied invA (NB = 128, built by
    rocblas_?trtri_strided_batched the way testing_trsm_ex.hpp:329-336 builds it) at 8192^2.
    Each entry: TFLOP/s (m n k flops) of the median of `reps` event-timed solves after one
    warm-up, B restored from a copy before each solve (outside the timing)."""
    import itertools

    g = torch.Generator(device=dev)
    g.manual_seed(8192)
    out = {}
    for dt, tdt in (("d", torch.float64), ("s", torch.float32)):
        alpha = ctypes.c_double(1.0) if dt == "d" else ctypes.c_float(1.0)
        ap = ctypes.cast(ctypes.byref(alpha), ctypes.c_void_p)
        fn = getattr(L, f"rocblas_{dt}trsm")
        res = {}
        mats = {}
        for m, n in SWEEP_SHAPES:
            B0 = (torch.rand(n, m, generator=g, device=dev, dtype=torch.float64) * 2 - 1).to(tdt)
            Bt = torch.empty_like(B0)
            shape = {}
            for side, uplo, trans, diag in itertools.product("LR", "UL", "NT", "NU"):
                k = m if side == "L" else n
                key = (k, uplo, diag)
                if key not in mats:
                    mats = {kk: v for kk, v in mats.items() if kk[0] == k}  # keep memory bounded
                    mats[key] = sweep_matrix(torch, dev, k, uplo, diag, tdt, g)
                At = mats[key]

                def solve():
                    st = fn(h.value, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag], m, n, ap,
                            ctypes.c_void_p(At.data_ptr()), k, ctypes.c_void_p(Bt.data_ptr()), m)
                    assert st == 0, (side, uplo, trans, diag, m, n, st)

                t = _timed_median(torch, solve, lambda: Bt.copy_(B0), reps)
                shape[side + uplo + trans + diag] = float(m) * n * k / t / 1e12
            vals = sorted(shape.values())
            res[f"{m}x{n}"] = {"tflops": shape, "min": vals[0], "median": statistics.median(vals),
                               "max": vals[-1]}
            del B0, Bt
        mats.clear()
        # _ex with the caller's invA at 8192^2, L/L/N/N and R/U/T/N
        m = n = 8192
        ex = {}
        for side, uplo, trans, diag in (("L", "L", "N", "N"), ("R", "U", "T", "N")):
            At = sweep_matrix(torch, dev, m, uplo, diag, tdt, g)
            inv = torch.zeros(128 * m, dtype=tdt, device=dev)
            tri = getattr(L, f"rocblas_{dt}trtri_strided_batched")
            st = tri(h.value, rb.UPLO[uplo], rb.DIAG[diag], 128, ctypes.c_void_p(At.data_ptr()), m, 128 * m + 128,
                     ctypes.c_void_p(inv.data_ptr()), 128, 128 * 128, m // 128)
            assert st == 0, st
            B0 = (torch.rand(n, m, generator=g, device=dev, dtype=torch.float64) * 2 - 1).to(tdt)
            Bt = torch.empty_like(B0)

            def solve_ex():
                st = L.rocblas_trsm_ex(h.value, rb.SIDE[side], rb.UPLO[uplo], rb.TRANS[trans], rb.DIAG[diag], m,
                                       n, ap, ctypes.c_void_p(At.data_ptr()), m, ctypes.c_void_p(Bt.data_ptr()), m,
                                       ctypes.c_void_p(inv.data_ptr()), 128 * m,
                                       rb.datatype_f64_r if dt == "d" else rb.datatype_f32_r)
                assert st == 0, st

            t = _timed_median(torch, solve_ex, lambda: Bt.copy_(B0), reps)
            ex[side + uplo + trans + diag] = float(m) * n * m / t / 1e12
            del At, inv, B0, Bt
        res["ex_invA_8192x8192"] = ex
        out[dt + "trsm"] = res
        torch.cuda.empty_cache()
    out["unit"] = "TFLOP/s"
    return out


def bench_complex(torch, L, h, dev, fp64_peak, m=8192, n=2048, steps=5):
    """Complex trsm (rocblas_ztrsm / rocblas_ctrsm, L/L/N/N) at m = 8192, n = 2048: A as the
    drop-in recipe with imaginary parts (off-diagonal (U + iU)/m, diagonal 1 + U(0,1) + iU/2),
    B ~ U + iU.  TFLOP/s uses the reference's complex flop count, 4 m^2 n
    (clients/include/flops.hpp:727-737); the complex DMMA update kernel is timed with CUDA events
    and set against the cuBLAS DGEMM rate measured in the same run (its work counted as 8 real
    flops per complex multiply-add)."""
    out = {}
    g = torch.Generator(device=dev)
    g.manual_seed(99)
    for dt, tdt, rdt in (("z", torch.complex128, torch.float64), ("c", torch.complex64, torch.float32)):
        At = torch.complex(torch.rand(m, m, generator=g, device=dev, dtype=rdt) * 2 - 1,
                           torch.rand(m, m, generator=g, device=dev, dtype=rdt) * 2 - 1) / m
        At.diagonal().copy_(torch.complex(1 + torch.rand(m, generator=g, device=dev, dtype=rdt),
                                          torch.rand(m, generator=g, device=dev, dtype=rdt) - 0.5))
        At = At.triu().contiguous()  # (col, row) storage: upper in At is A lower
        B0 = torch.complex(torch.rand(n, m, generator=g, device=dev, dtype=rdt) * 2 - 1,
                           torch.rand(n, m, generator=g, device=dev, dtype=rdt) * 2 - 1)
        Bt = torch.empty_like(B0)
        alpha = torch.tensor([1.0 + 0.0j], dtype=tdt)
        fn = getattr(L, f"rocblas_{dt}trsm")

        def solve():
            st = fn(h.value, 141, 122, 111, 131, m, n, ctypes.c_void_p(alpha.data_ptr()),
                    ctypes.c_void_p(At.data_ptr()), m, ctypes.c_void_p(Bt.data_ptr()), m)
            assert st == 0, st

        for _ in range(2):
            Bt.copy_(B0)
            solve()
        torch.cuda.synchronize(dev)
        L.rocblas_b200_kernel_timing_enable(1)
        tot = 0.0
        for _ in range(steps):
            Bt.copy_(B0)
            s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record()
            solve()
            e0.record()
            e0.synchronize()
            tot += s0.elapsed_time(e0)
        g_ms, g_work, g_n = kernel_timing(L, "dmma")
        L.rocblas_b200_kernel_timing_enable(0)
        ms = tot / steps
        gemm_tf = g_work / (g_ms * 1e-3) / 1e12 if g_ms > 0 else None
        out[dt + "trsm"] = {
            "value": 4.0 * m * m * n / (ms * 1e-3) / 1e12, "unit": "TFLOP/s", "ms": ms,
            "m": m, "n": n, "flop_count": "4 m^2 n (complex)",
            "update_kernel": {"name": "gemm_cdmma_kernel", "achieved_tflops_fp64": gemm_tf,
                              "frac_of_measured_dgemm": gemm_tf / fp64_peak if gemm_tf else None,
                              "share_of_solve": g_ms / tot if tot > 0 else None, "launches": g_n},
        }
        del At, B0, Bt
        torch.cuda.empty_cache()
    out["dgemm_tflops_measured"] = fp64_peak
    return out


def bench_trsv(torch, L, h, dev, hbm_gbs):
    """rocblas_?trsv of one vector (the memory-bound flag-synchronised solve) at n = 4096 ..
    32768, lower, no-trans: median of 7 event-timed calls, reported as GB/s of A's triangle
    (n (n + 1) / 2 elements, the solve's algorithmic bytes) and as a fraction of the measured
    HBM copy bandwidth."""
    import rocblas_b200 as rb
    from rocblas_b200 import workloads

    rb_fill_lower, rb_op_none, rb_diag_non_unit = rb.fill_lower, rb.operation_none, rb.diagonal_non_unit
    out = {}
    for dt, tdt, es, fn in (("d", torch.float64, 8, L.rocblas_dtrsv), ("s", torch.float32, 4, L.rocblas_strsv)):
        for n in (4096, 16384, 32768):
            At, x0 = workloads.condition_band_lower_torch(n, 1, 0, seed=3, device=dev, dtype=tdt)
            x = x0.clone()
            args = (h.value, rb_fill_lower, rb_op_none, rb_diag_non_unit, n, ctypes.c_void_p(At.data_ptr()), n,
                    ctypes.c_void_p(x.data_ptr()), 1)
            ts = []
            for it in range(9):
                x.copy_(x0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                st = fn(*args)
                e1.record()
                e1.synchronize()
                assert st == 0, st
                if it >= 2:
                    ts.append(e0.elapsed_time(e1))
            ms = statistics.median(ts)
            gbs = n * (n + 1) / 2 * es / (ms * 1e-3) / 1e9
            out[f"{dt}trsv_{n}"] = {"us": ms * 1e3, "GBps": gbs, "hbm_frac": gbs / hbm_gbs}
            del At, x0, x
    return out


def bench_serving(torch, dev, n_requests, rate, seed=7, payload_on_host=False):
    """The serving workload: Poisson arrivals, m log-uniform [64, 8192], n log-uniform [1, 512], 70% FP64,
    60% of requests on one of 256 resident A (condition-band recipe, k in {0, 2, 4}), 120 GB
    (120e9 bytes) budget.  The native server loop (rocblas_b200_server_run) serves the list;
    returns p50 / p99 latency, solves/s over the server's own wall time, and its batching
    statistics.  payload_on_host: each request's B and fresh A are read from pinned host memory
    across PCIe by the server's gather launch, inside the measured latency."""
    from rocblas_b200 import serving

    rng = np.random.default_rng(seed)
    srv = serving.TrsmServer(device=dev, hbm_budget=120_000_000_000, n_streams=2, window_us=200.0,
                             payload_on_host=payload_on_host)
    sizes = {}
    for key in range(256):
        m = int(round(np.exp(rng.uniform(np.log(64), np.log(8192)))))
        srv.add_resident(key, m, kband=int(rng.choice([0, 2, 4])), seed=1000 + key)
        sizes[key] = m
    reqs = serving.make_requests(n_requests, rate, seed, sizes)
    flops = float(sum(q.m * q.m * q.n for q in reqs))
    lat = srv.run(reqs)
    st = srv.last_stats
    wall = st["wall_s"]
    srv.close()
    return {"requests": n_requests, "arrival_rate_per_s": rate,
            "arrival_span_s": float(reqs[-1].arrival),
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "solves_per_s": n_requests / wall,
            "tflops": flops / wall / 1e12, "wall_s": wall, "resident_matrices": 256,
            "collections": st["collections"], "largest_collection": st["largest_collection"],
            "peak_arena_gb": st["peak_bytes"] / 1e9, "gpu_launches": st["kernel_launches"],
            "fp64_fraction": float(np.mean([q.dtype == "d" for q in reqs])),
            "reuse_fraction": float(np.mean([q.a_key is not None for q in reqs])),
            "budget_bytes": 120_000_000_000,
            "payload": ("pinned host memory, read across PCIe by the gather launch inside each request's "
                        "latency" if payload_on_host else "device pools (copied device to device)"),
            "payload_bytes": int(sum(q.m * q.n * (8 if q.dtype == "d" else 4)
                                     + (0 if q.a_key is not None else q.m * (q.m + 1) // 2 * (8 if q.dtype == "d" else 4))
                                     for q in reqs))}


ERROR_COLUMNS = 64  # right-hand sides per band checked against the extended-precision X*


def band_errors(torch, dev, Ab, Bb, solve_plain, solve_refined, threads):
    """One condition band at the headline size: the plain FP64 form and the refined precision
    form solved on the GPU (one event-timed call each), and their normwise forward errors on
    ERROR_COLUMNS right-hand sides spread over B, against the oracle's extended-precision X*
    (host CBLAS solve + two double-double refinement steps) and against the host FP64 CBLAS
    solution itself."""
    import oracle

    def once(fn):
        X = Bb.clone()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn(X, Ab)
        e1.record()
        e1.synchronize()
        return X, e0.elapsed_time(e1), r

    Xp, p_ms, _ = once(solve_plain)
    Xr, r_ms, info = once(solve_refined)
    cols = np.linspace(0, Bb.shape[0] - 1, ERROR_COLUMNS).round().astype(np.int64)
    A_host = np.asfortranarray(np.nan_to_num(Ab.cpu().numpy().T, nan=0.0))
    B_s = np.asfortranarray(Bb[cols].cpu().numpy().T)
    oracle.cblas_set_threads(threads)
    Xh, Xl = oracle.refined_solution("L", "L", "N", "N", 1.0, A_host, B_s)
    Xc = oracle.cblas_trsm("L", "L", "N", "N", 1.0, A_host, B_s)
    Xr_s = Xr[cols].cpu().numpy().T
    Xp_s = Xp[cols].cpu().numpy().T
    del A_host
    return {
        "refined_vs_xstar": oracle.forward_error_dd(Xr_s, Xh, Xl),
        "plain_fp64_vs_xstar": oracle.forward_error_dd(Xp_s, Xh, Xl),
        "fp64_cblas_vs_xstar": oracle.forward_error_dd(Xc, Xh, Xl),
        "refined_vs_fp64_cblas": oracle.normwise_forward_error(Xr_s, Xc),
        "refinement_iterations": info["iterations"],
        "converged": info["converged"], "fell_back": info["fell_back"],
        "error_estimate_first_solve": info["error_estimate_first"],
        "error_estimate_final": info["error_estimate"], "test_tolerance": info["tolerance"],
        "refined_ms": r_ms, "plain_ms": p_ms,
    }


def apply_tuning(L, args):
    """The --tuning key=value entries, set in the library's tuning table before any call."""
    for kv in args.tuning:
        key, val = kv.split("=")
        assert L.rocblas_b200_set_tuning(key.encode(), int(val)) == 0, kv


def run_ours(args):
    import torch

    import rocblas_b200 as rb
    from rocblas_b200 import workloads

    rank, world, local = _env_rank()
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    rb.build()
    L = rb.lib()
    apply_tuning(L, args)
    S = args.slices

    At, B0 = workloads.condition_band_lower_torch(M, N, 0, seed=1234 + rank, device=dev)
    Bt = B0.clone()
    stream = torch.cuda.current_stream(dev)
    h = rb.Handle()
    h.set_stream(ctypes.c_void_p(stream.cuda_stream))
    one = ctypes.c_double(1.0)
    one_p = ctypes.cast(ctypes.byref(one), ctypes.c_void_p)
    args_common = (rb.side_left, rb.fill_lower, rb.operation_none, rb.diagonal_non_unit, M, N, one_p)

    def solve_plain(Bbuf, Abuf):
        st = L.rocblas_dtrsm(h.value, *args_common, ctypes.c_void_p(Abuf.data_ptr()), M,
                             ctypes.c_void_p(Bbuf.data_ptr()), M)
        if st != 0:
            raise rb.RocblasError("rocblas_dtrsm", st)

    opts = rb.RefineOptions(S, -1, args.check_columns, 1, 0.0)
    opts_p = ctypes.cast(ctypes.byref(opts), ctypes.c_void_p)
    last_info = rb.RefineInfo()
    info_p = ctypes.cast(ctypes.byref(last_info), ctypes.c_void_p)

    def solve_refined(Bbuf, Abuf):
        # the headline: precision-form solve, the test against the plain FP64 solve of sampled
        # right-hand sides and, if it fails, FP64-residual corrections (the call returns once
        # the test has been read)
        st = L.rocblas_b200_dtrsm_refined(h.value, *args_common, ctypes.c_void_p(Abuf.data_ptr()), M,
                                          ctypes.c_void_p(Bbuf.data_ptr()), M, opts_p, info_p)
        if st != 0:
            raise rb.RocblasError("rocblas_b200_dtrsm_refined", st)
        return last_info.as_dict()

    # workspace by the size-query protocol, reserved before timing (no allocation inside)
    assert L.rocblas_start_device_memory_size_query(h.value) == 0
    L.rocblas_dtrsm(h.value, *args_common, None, M, None, M)
    L.rocblas_b200_dtrsm_refined(h.value, *args_common, None, M, None, M, opts_p, None)
    ws = ctypes.c_size_t(0)
    assert L.rocblas_stop_device_memory_size_query(h.value, ctypes.byref(ws)) == 0
    assert L.rocblas_set_device_memory_size(h.value, ws.value) == 0

    def timed(solve, steps, warmup):
        for _ in range(max(warmup, 0)):
            Bt.copy_(B0)
            solve(Bt, At)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        l0 = L.rocblas_b200_kernel_launch_count()
        ev_m = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ev_e = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for i in range(steps):
            Bt.copy_(B0)
            ev_m[i].record(stream)
            solve(Bt, At)
            ev_e[i].record(stream)
        t1.record(stream)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        launches = L.rocblas_b200_kernel_launch_count() - l0
        total = max_over_ranks(dist, t0.elapsed_time(t1), dev)
        return total, [ev_m[i].elapsed_time(ev_e[i]) for i in range(steps)], launches

    # ---- timed region: the refined precision form (headline), then the plain FP64 form -------
    # Every launch of the dominant kernels is bracketed by CUDA events on its stream inside the
    # timed region (rocblas_b200_kernel_timing_*), for the roofline of the kernel itself.
    sampler = ClockSampler(dev.index if dev.index is not None else 0)
    sampler.start()
    for _ in range(max(args.warmup, 0)):
        Bt.copy_(B0)
        solve_refined(Bt, At)
    L.rocblas_b200_kernel_timing_enable(1)
    total_ms, solve_ms, launches = timed(solve_refined, args.steps, 0)
    headline_info = last_info.as_dict()
    sliced_t = kernel_timing(L, "sliced")
    mixed_chain_t = kernel_timing(L, "chain")
    L.rocblas_b200_kernel_timing_enable(0)
    clocks = sampler.stop()
    ms_per_step = total_ms / args.steps
    value = replicas_value(FLOPS, world, ms_per_step) / 1e12
    for _ in range(max(args.warmup, 0)):
        Bt.copy_(B0)
        solve_plain(Bt, At)
    L.rocblas_b200_kernel_timing_enable(1)
    p_total, p_solve, p_launches = timed(solve_plain, args.steps, 0)
    chain_t = kernel_timing(L, "chain")
    L.rocblas_b200_kernel_timing_enable(0)
    plain_value = replicas_value(FLOPS, world, p_total / args.steps) / 1e12

    # ---- e2e: host buffers through the C ABI, copies inside the timed region -----------
    e2e = None
    if rank == 0:
        A_host = torch.empty_like(At, device="cpu").pin_memory()
        B_host = torch.empty_like(B0, device="cpu").pin_memory()
        A_host.copy_(At)
        B_host.copy_(B0)

        one_h = ctypes.c_double(1.0)

        def e2e_step():
            # the host-buffer entry point: A's block rows and B's rows, the solve and the rows of X
            # coming back overlap inside the call
            st = L.rocblas_b200_dtrsm_mixed_host(h.value, rb.side_left, rb.fill_lower, rb.operation_none,
                                                 rb.diagonal_non_unit, M, N, ctypes.byref(one_h),
                                                 ctypes.c_void_p(A_host.data_ptr()), M,
                                                 ctypes.c_void_p(B_host.data_ptr()), M, S)
            assert st == 0, st

        e2e_step()
        torch.cuda.synchronize(dev)
        B_host.copy_(B0)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ksteps = max(2, min(args.steps, 5))
        s0.record(stream)
        for _ in range(ksteps):
            e2e_step()
        s1.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms = s0.elapsed_time(s1) / ksteps
        # bytes the call moves: B, and A's lower triangle in block rows of host_step_blocks x 128
        # rows (each block row: its rows, the columns from 0 to the end of its diagonal block)
        step_blocks = ctypes.c_int()
        assert L.rocblas_b200_get_tuning(b"host_step_blocks", ctypes.byref(step_blocks)) == 0
        pw = 128 * step_blocks.value
        a_h2d = sum((min(M, r0 + pw) - r0) * min(M, r0 + pw) for r0 in range(0, M, pw)) * 8
        e2e = {"value": FLOPS / (e2e_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(a_h2d + B0.numel() * 8),
               "d2h_bytes_per_step": int(B0.numel() * 8), "ms_per_step": e2e_ms,
               "form": f"precision form ({headline_engine(L, S)['label']}), rocblas_b200_dtrsm_mixed_host on pinned host "
                       "buffers (transfers of A's block rows, of B and of X overlap the left-looking solve)"}
        del A_host, B_host

    # ---- errors per condition band against the extended-precision oracle, CPU baseline --------
    extra = {}
    peak = None
    if rank == 0:
        import oracle

        peak = fp64_peak_tflops(torch, dev)
        med_ref = statistics.median(solve_ms)
        med_plain = statistics.median(p_solve)
        threads = os.cpu_count() or 1
        bands = {"c2_recipe_k0": band_errors(torch, dev, At, B0, solve_plain, solve_refined, threads)}
        if not args.no_bands:
            for kb, Ab, Bb in workloads.graded_condition_bands_torch(M, N, (0, 2, 4, 6), seed=99, device=dev):
                bands[f"graded_k{kb}"] = band_errors(torch, dev, Ab, Bb, solve_plain, solve_refined, threads)
                del Ab, Bb
            torch.cuda.empty_cache()
        # host CBLAS on the whole headline problem (all N right-hand sides), all host cores
        A_host = np.asfortranarray(np.nan_to_num(At.cpu().numpy().T, nan=0.0))
        B_host = np.asfortranarray(B0.cpu().numpy().T)
        cpu_tflops, cpu_s, _ = cpu_cblas_sample(A_host, B_host, N, threads)
        del A_host, B_host
        pk = measured_peaks()
        # dominant kernel of the headline: the integer tensor-core GEMM of the updates (the
        # residue GEMM crt_gemm_kernel, work = int8 tensor operations of its NM residue products,
        # 2 * NM * M * N * K per launch; or the slice GEMM ozaki_gemm_kernel, 2 * pairs * M * N * K),
        # timed per launch with CUDA events on the solve's stream inside the timed region.  The
        # peak is the burst figure: the kernel is timed in short launches and the clocks stay at
        # their maximum (the `clocks` record), not under the power cap the sustained figure saw.
        s_ms, s_ops, s_n = sliced_t
        achieved = s_ops / (s_ms * 1e-3) / 1e12 if s_ms > 0 else 0.0
        i8_peak = 2.0 * pk["bf16_tflops"]
        eng = headline_engine(L, S)
        traffic, traffic_src = ((CRT_TRAFFIC_PER_LAUNCH, CRT_TRAFFIC_SOURCE) if eng["engine"] == "residue"
                                else (SLICED_TRAFFIC_PER_LAUNCH, SLICED_TRAFFIC_SOURCE))
        roofline = {"bound": "tensor", "achieved": achieved, "peak": i8_peak, "unit": "TOP/s (int8)",
                    "frac": achieved / i8_peak, "traffic": traffic,
                    "kernel": eng["kernel"],
                    "launches": s_n, "kernel_ms_per_step": s_ms / args.steps,
                    "kernel_share_of_step": s_ms / total_ms,
                    "peak_source": "int8 dense = 2 x bf16_tflops (burst) of " + pk["source"]
                                   + " (B200's dense int8 rate is twice bf16)",
                    "frac_of_sustained": achieved / (2.0 * pk["bf16_tflops_sustained"]),
                    "sm_mhz_median": clocks.get("sm_mhz"),
                    "traffic_source": traffic_src,
                    "fp64_equivalent": {"achieved": FLOPS / (med_ref * 1e-3) / 1e12, "peak": peak,
                                        "unit": "TFLOP/s", "what": "whole refined solve, m*n*k flops, "
                                        "against cuBLAS DGEMM 8192^3 measured in this run"}}
        c_ms, c_fl, c_n = chain_t
        plain_roofline = {"bound": "tensor", "kernel": "trsm_chain_kernel (mma.sync f64 DMMA)",
                          "achieved": c_fl / (c_ms * 1e-3) / 1e12 if c_ms > 0 else 0.0, "peak": peak,
                          "unit": "TFLOP/s", "launches": c_n,
                          "frac": (c_fl / (c_ms * 1e-3) / 1e12) / peak if c_ms > 0 else 0.0,
                          "traffic": CHAIN_TRAFFIC_PER_LAUNCH, "traffic_source": CHAIN_TRAFFIC_SOURCE,
                          "peak_source": "cuBLAS DGEMM 8192^3 (torch.matmul fp64) measured in this run; "
                                         "MEASURED_PEAKS.json has no FP64 figure"}
        worst = max(b["refined_vs_xstar"] for b in bands.values())
        extra = {
            # the two targets and the accuracy evidence first, where a truncated record keeps them
            "plain_fp64_tflops": plain_value,
            "refined_vs_plain": value / plain_value,
            "plain_frac_of_measured_dgemm": plain_value / peak,
            "max_refined_error_vs_xstar": worst,
            "refinement_iterations": {k: b["refinement_iterations"] for k, b in bands.items()},
            "headline_refine_info": headline_info,
            "roofline": roofline,
            "plain_fp64": {"value": plain_value, "unit": "TFLOP/s", "ms_per_step": p_total / args.steps,
                           "solve_ms_median": med_plain,
                           "solve_ms_p99": float(np.percentile(p_solve, 99)),
                           "frac_of_fp64_peak": plain_value / peak,
                           "gpu_launches": int(p_launches), "roofline": plain_roofline},
            "cpu_baseline": {"value": cpu_tflops, "unit": "TFLOP/s", "cores": threads, "kind": "reference",
                             "sample": f"host cblas_dtrsm (OpenBLAS {oracle.cblas_config().split()[1]}) "
                                       f"on the whole problem (all {N} right-hand sides, m={M}), one solve, "
                                       f"{cpu_s:.2f} s"},
            "error_bands": bands,
            "error_sample": f"normwise ||X - X*||_F / ||X*||_F on {ERROR_COLUMNS} right-hand sides spread "
                            "over B (linspace); X* = host CBLAS solve + 2 double-double refinement steps "
                            "(oracle.refined_solution); bands: c2_recipe_k0 = the headline matrix, "
                            "graded_kK = singular values graded 1..10^-K (kappa_2 = 10^K, dlatms-style)",
            "solve_ms_median": med_ref,
            "solve_ms_p99": float(np.percentile(solve_ms, 99)),
            "solve_ms_samples": len(solve_ms),
        }

    if rank == 0 and not args.no_extras:
        hbm = measured_peaks()["hbm_gbs"]
        extra["sweep"] = bench_sweep(torch, rb, L, h, dev)
        extra["batched"] = bench_batched(torch, rb, L, h, dev, hbm)
        extra["complex"] = bench_complex(torch, L, h, dev, peak)
        extra["trsv"] = bench_trsv(torch, L, h, dev, hbm)
        extra["serving"] = bench_serving(torch, dev, args.serving_requests, 50000.0)
        # the same stream with its payloads arriving from pinned host memory, on a bounded
        # sample of the requests (the fresh A matrices make the payload several MB per request
        # on average; the total is in payload_bytes)
        extra["serving_host_payload"] = bench_serving(torch, dev, max(1000, args.serving_requests // 10),
                                                      50000.0, payload_on_host=True)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value,
            "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": workload_name(), "m": M, "n": N,
                       "form": f"refined precision form: {headline_engine(L, S)['label']}, "
                               f"FP64 diagonal blocks; test: agreement to "
                               f"1e-12 with the plain FP64 form on {args.check_columns or 8} right-hand sides "
                               "(solved on a second stream), FP64-residual corrections if it fails",
                       "l2": "inputs larger than L2 (A 2 GiB, B 512 MiB); no flush",
                       "step": "device copy of B (512 MiB) + one solve",
                       "parallelism": f"replicas x{world}"},
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
        }
        early = ("plain_fp64_tflops", "refined_vs_plain", "plain_frac_of_measured_dgemm",
                 "max_refined_error_vs_xstar", "refinement_iterations")
        head = {k: line[k] for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup",
                                     "ms_per_step", "higher_is_better", "scaling", "vs_baseline",
                                     "dtype", "data")}
        head.update({k: extra[k] for k in early if k in extra})
        head.update({k: v for k, v in line.items() if k not in head})
        head.update({k: v for k, v in extra.items() if k not in head})
        # the targets again as the last key, so that either end of a cut record shows them
        head["targets"] = {k: extra.get(k) for k in early}
        line = head
        print(json.dumps(line), flush=True)
    h.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_case(args):
    """One kernel on one small shape, a few launches, for ncu captures (no JSON line):
    sliced: rocblas_b200_dgemm_sliced m x n x k, S slices; crt: rocblas_b200_dgemm_crt m x n x k
    with --moduli moduli; dmma: rocblas_b200_dgemm m x n x k;
    zgemm: rocblas_b200_zgemm m x n x k (the complex DMMA tiles); chain: rocblas_dtrsm L/L/N/N
    m x n (the chain solve); strsm: rocblas_strsm L/L/N/N m x n (FP32: the recursive solve with
    FFMA tile updates above 512 columns); trsv: rocblas_dtrsv lower, no-trans, order m (the flag
    solve); serving: the serving loop over --count requests (m up to 2048, 16 resident A; its
    gather launch, variable-size batched solves and their chain solves); vbatched: rocblas_b200_dtrsm_vbatched over --count systems of the
    variable-size batch recipe; strided: rocblas_dtrsm_strided_batched, --count systems of m x n (L/L/N/N);
    trtri: rocblas_dtrtri_strided_batched, --count lower m x m blocks."""
    import torch

    import rocblas_b200 as rb
    from rocblas_b200 import workloads

    rb.build()
    L = rb.lib()
    apply_tuning(L, args)
    h = rb.Handle()
    dev = torch.device("cuda", 0)
    m, n, k = args.m, args.n, args.k
    minus = ctypes.c_double(-1.0)
    one = ctypes.c_double(1.0)
    pm = ctypes.cast(ctypes.byref(minus), ctypes.c_void_p)
    po = ctypes.cast(ctypes.byref(one), ctypes.c_void_p)
    g = torch.Generator(device=dev).manual_seed(5)
    if args.case == "chain":
        At, Bt = workloads.condition_band_lower_torch(m, n, 0, seed=5, device=dev)

        def run():
            st = L.rocblas_dtrsm(h.value, rb.side_left, rb.fill_lower, rb.operation_none,
                                 rb.diagonal_non_unit, m, n, po, ctypes.c_void_p(At.data_ptr()), m,
                                 ctypes.c_void_p(Bt.data_ptr()), m)
            assert st == 0, st
    elif args.case == "strsm":
        At, Bt = workloads.condition_band_lower_torch(m, n, 0, seed=5, device=dev, dtype=torch.float32)
        one_f = ctypes.c_float(1.0)

        def run():
            st = L.rocblas_strsm(h.value, rb.side_left, rb.fill_lower, rb.operation_none,
                                 rb.diagonal_non_unit, m, n, ctypes.cast(ctypes.byref(one_f), ctypes.c_void_p),
                                 ctypes.c_void_p(At.data_ptr()), m, ctypes.c_void_p(Bt.data_ptr()), m)
            assert st == 0, st
    elif args.case == "trsv":
        At, xt = workloads.condition_band_lower_torch(m, 1, 0, seed=5, device=dev)

        def run():
            st = L.rocblas_dtrsv(h.value, rb.fill_lower, rb.operation_none, rb.diagonal_non_unit, m,
                                 ctypes.c_void_p(At.data_ptr()), m, ctypes.c_void_p(xt.data_ptr()), 1)
            assert st == 0, st
    elif args.case == "serving":
        from rocblas_b200 import serving

        rng = np.random.default_rng(7)
        srv = serving.TrsmServer(device=dev, hbm_budget=8 << 30, n_streams=2, window_us=200.0)
        sizes = {}
        for key in range(16):
            sizes[key] = int(round(np.exp(rng.uniform(np.log(64), np.log(2048)))))
            srv.add_resident(key, sizes[key], kband=0, seed=1000 + key)
        reqs = serving.make_requests(args.count, 50000.0, 7, sizes, m_range=(64, 2048))

        def run():
            srv.run(reqs)
    elif args.case == "vbatched":
        w = vbatched_workload(torch, dev, args.count, 2024, "d")
        one_d = ctypes.c_double(1.0)

        def run():
            st = L.rocblas_b200_dtrsm_vbatched(h.value, ctypes.cast(ctypes.byref(one_d), ctypes.c_void_p),
                                               ctypes.c_void_p(w["desc"].data_ptr()), args.count, 512, None)
            assert st == 0, st
    elif args.case == "strided":
        bc = args.count
        As = torch.rand(bc, m, m, generator=g, device=dev, dtype=torch.float64) / m
        idx = torch.arange(m, device=dev)
        As[:, idx, idx] = 1.0 + torch.rand(bc, m, generator=g, device=dev, dtype=torch.float64)
        Bs = torch.rand(bc, n, m, generator=g, device=dev, dtype=torch.float64) * 2 - 1

        def run():
            st = L.rocblas_dtrsm_strided_batched(h.value, 141, 122, 111, 131, m, n, po,
                                                 ctypes.c_void_p(As.data_ptr()), m, m * m,
                                                 ctypes.c_void_p(Bs.data_ptr()), m, m * n, bc)
            assert st == 0, st
    elif args.case == "trtri":
        bc = args.count
        At = torch.rand(bc, m, m, generator=g, device=dev, dtype=torch.float64) / m
        At.diagonal(dim1=1, dim2=2).add_(1.0)
        Inv = torch.zeros_like(At)

        def run():
            st = L.rocblas_dtrtri_strided_batched(h.value, rb.fill_lower, rb.diagonal_non_unit, m,
                                                  ctypes.c_void_p(At.data_ptr()), m, m * m,
                                                  ctypes.c_void_p(Inv.data_ptr()), m, m * m, bc)
            assert st == 0, st
    elif args.case == "zgemm":
        A = torch.randn(k, m, dtype=torch.complex128, device=dev, generator=g)
        B = torch.randn(n, k, dtype=torch.complex128, device=dev, generator=g)
        C = torch.randn(n, m, dtype=torch.complex128, device=dev, generator=g)
        za = torch.tensor([-1.0 + 0.5j], dtype=torch.complex128)
        zb = torch.tensor([1.0 + 0.0j], dtype=torch.complex128)

        def run():
            st = L.rocblas_b200_zgemm(h.value, rb.operation_none, rb.operation_none, m, n, k,
                                      ctypes.c_void_p(za.data_ptr()), ctypes.c_void_p(A.data_ptr()), m,
                                      ctypes.c_void_p(B.data_ptr()), k, ctypes.c_void_p(zb.data_ptr()),
                                      ctypes.c_void_p(C.data_ptr()), m)
            assert st == 0, st
    else:
        A = torch.randn(k, m, dtype=torch.float64, device=dev, generator=g)
        B = torch.randn(n, k, dtype=torch.float64, device=dev, generator=g)
        C = torch.randn(n, m, dtype=torch.float64, device=dev, generator=g)
        gemm_args = (h.value, rb.operation_none, rb.operation_none, m, n, k, pm,
                     ctypes.c_void_p(A.data_ptr()), m, ctypes.c_void_p(B.data_ptr()), k, po,
                     ctypes.c_void_p(C.data_ptr()), m)

        def run():
            if args.case == "sliced":
                st = L.rocblas_b200_dgemm_sliced(*gemm_args, headline_slices(L, args.slices))
            elif args.case == "crt":
                st = L.rocblas_b200_dgemm_crt(*gemm_args, args.moduli)
            else:
                st = L.rocblas_b200_dgemm(*gemm_args)
            assert st == 0, st
    if args.case in ("sliced", "crt"):
        # one untimed call, then the steps with the library's kernel timer (the integer GEMM
        # kernel alone) and CUDA events around the whole calls
        run()
        torch.cuda.synchronize()
        L.rocblas_b200_kernel_timing_enable(1)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
    for _ in range(max(args.steps, 1)):
        run()
    torch.cuda.synchronize()
    timing = ""
    if args.case in ("sliced", "crt"):
        ev1.record()
        ev1.synchronize()
        k_ms, _, k_n = kernel_timing(L, "sliced")
        L.rocblas_b200_kernel_timing_enable(0)
        timing = (f"; GEMM kernel {1000 * k_ms / max(k_n, 1):.0f} us per launch, whole call "
                  f"{1000 * ev0.elapsed_time(ev1) / max(args.steps, 1):.0f} us")
    code = ctypes.c_int(-1)
    assert L.rocblas_b200_get_device_error(h.value, ctypes.byref(code)) == 0 and code.value == 0
    print(f"case {args.case} m={m} n={n} k={k}: {args.steps} launches ok{timing}", flush=True)
    h.close()


def main():
    global M, N, FLOPS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--m", type=int, default=M, help="problem size (profiling runs use smaller)")
    ap.add_argument("--n", type=int, default=N)
    ap.add_argument("--slices", type=int, default=0,
                    help="slices of the precision form (0: the tuning table's mixed_slices)")
    ap.add_argument("--serving-requests", type=int, default=200000)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the sweep, batched, complex and serving sections (profiling runs)")
    ap.add_argument("--no-bands", action="store_true",
                    help="skip the graded condition bands (errors of the headline matrix only)")
    ap.add_argument("--check-columns", type=int, default=0,
                    help="right-hand sides the refined form's test uses (0: its default, 8)")
    ap.add_argument("--moduli", type=int, default=16, help="moduli of a --case crt GEMM")
    ap.add_argument("--tuning", action="append", default=[],
                    help="key=value tuning-table entry set before the run (repeatable)")
    ap.add_argument("--case", choices=["sliced", "crt", "dmma", "zgemm", "chain", "strsm", "trsv", "serving",
                                       "vbatched", "strided", "trtri"],
                    help="run one kernel on one shape (--m --n --k), --steps times, for ncu captures")
    ap.add_argument("--k", type=int, default=4096, help="inner dimension of a --case GEMM")
    ap.add_argument("--count", type=int, default=4000,
                    help="systems of a --case vbatched (variable-size batch recipe) or strided (m x n each) run")
    args = ap.parse_args()
    if args.case:
        run_case(args)
        return
    M, N = args.m, args.n
    FLOPS = float(M) * M * N
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
