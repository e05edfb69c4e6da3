"""Layer logging (ROCBLAS_LAYER) of the TRSM entry points, on CPU.

The reference logs every call before its argument check (library/src/blas3/rocblas_trsm_imp.hpp:
74-143, rocblas_trsm_batched_imp.hpp:84-131, rocblas_trsm_strided_batched_imp.hpp), so calls
with an invalid size are logged and return without touching a device: the whole protocol runs
here. The mode and the log files are taken when the handle is created, so each case runs in a
child process with its own environment.
"""
import os
import subprocess
import sys
import textwrap

import pytest

import rocblas_b200 as rb

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent(r"""
    import ctypes, sys
    sys.path.insert(0, {repo!r})
    import rocblas_b200 as rb
    L = rb.lib()
    h = ctypes.c_void_p()
    assert L.rocblas_create_handle(ctypes.byref(h)) == 0
    a = ctypes.c_double(0.5)
    pa = ctypes.cast(ctypes.byref(a), ctypes.c_void_p)
    A = ctypes.c_void_p(0x1000)
    B = ctypes.c_void_p(0x2000)
    # m = -1: invalid size, returned after the log lines
    for _ in range(2):
        assert L.rocblas_dtrsm(h, 141, 122, 111, 131, -1, 8, pa, A, 8, B, 8) == rb.status_invalid_size
    assert L.rocblas_dtrsm_strided_batched(h, 142, 121, 112, 132, -1, 4, pa, A, 4, 16, B, 4, 64,
                                           3) == rb.status_invalid_size
    af = ctypes.c_float(2.0)
    pf = ctypes.cast(ctypes.byref(af), ctypes.c_void_p)
    assert L.rocblas_strsm_batched(h, 141, 121, 113, 131, -1, 4, pf, A, 4, B, 4, 5) == rb.status_invalid_size
    z = (ctypes.c_double * 2)(1.5, -2.0)
    assert L.rocblas_ztrsm_64(h, 141, 122, 113, 131, -1, 4, ctypes.cast(z, ctypes.c_void_p), A, 4, B, 4) \
        == rb.status_invalid_size
    assert L.rocblas_trsm_ex(h, 141, 122, 111, 131, -1, 8, pa, A, 8, B, 8, None, 0,
                             rb.datatype_f64_r) == rb.status_invalid_size
    assert L.rocblas_set_atomics_mode(h, rb.atomics_not_allowed) == 0
    assert L.rocblas_dtrsm(h, 141, 122, 111, 131, -1, 8, pa, A, 8, B, 8) == rb.status_invalid_size
    assert L.rocblas_destroy_handle(h) == 0
""")


def _run(tmp_path, layer):
    env = dict(os.environ)
    env["ROCBLAS_LAYER"] = str(layer)
    paths = {k: str(tmp_path / f"{k}.log") for k in ("trace", "bench", "profile")}
    env["ROCBLAS_LOG_TRACE_PATH"] = paths["trace"]
    env["ROCBLAS_LOG_BENCH_PATH"] = paths["bench"]
    env["ROCBLAS_LOG_PROFILE_PATH"] = paths["profile"]
    r = subprocess.run([sys.executable, "-c", CHILD.format(repo=REPO)], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = {}
    for k, p in paths.items():
        out[k] = open(p).read().splitlines() if os.path.exists(p) else None
    return out


@pytest.fixture(scope="module", autouse=True)
def _built():
    rb.build()


def test_trace_and_bench_lines(tmp_path):
    out = _run(tmp_path, 3)
    assert out["profile"] is None  # bit 4 off: no profile file
    trace = out["trace"]
    assert trace[0] == "rocblas_dtrsm,L,L,N,N,-1,8,0.5,0x1000,8,0x2000,8,atomics_allowed"
    assert trace[1] == trace[0]
    assert trace[2] == ("rocblas_strided_batched_dtrsm,R,U,T,U,-1,4,0.5,0x1000,4,16,0x2000,4,64,3,"
                        "atomics_allowed")
    assert trace[3] == "rocblas_batched_strsm,L,U,C,N,-1,4,2,0x1000,4,0x2000,4,5,atomics_allowed"
    assert trace[4] == "rocblas_ztrsm_64,L,L,C,N,-1,4,(1.5,-2),0x1000,4,0x2000,4,atomics_allowed"
    # rocblas_trsm_ex logs under the typed name, as the reference's shared implementation does
    assert trace[5] == trace[0]
    # the atomics mode: the set call's trace line (new mode, then the handle's old one), then
    # the mode on the next call's line
    assert trace[6] == "rocblas_set_atomics_mode,atomics_not_allowed,atomics_allowed"
    assert trace[7] == trace[0].replace("atomics_allowed", "atomics_not_allowed")
    assert len(trace) == 8
    bench = out["bench"]
    assert bench[0] == ("./rocblas-bench -f trsm -r f64_r --side L --uplo L --transposeA N --diag N "
                        "-m -1 -n 8 --alpha 0.5 --lda 8 --ldb 8")
    assert bench[2] == ("./rocblas-bench -f trsm_strided_batched -r f64_r --side R --uplo U "
                        "--transposeA T --diag U -m -1 -n 4 --alpha 0.5 --lda 4 --stride_a 16 --ldb 4 "
                        "--stride_b 64 --batch_count 3")
    assert bench[3] == ("./rocblas-bench -f trsm_batched -r f32_r --side L --uplo U --transposeA C "
                        "--diag N -m -1 -n 4 --alpha 2 --lda 4 --ldb 4 --batch_count 5")
    assert bench[4] == ("./rocblas-bench --api 1 -f trsm -r f64_c --side L --uplo L --transposeA C "
                        "--diag N -m -1 -n 4 --alpha 1.5 --alphai -2 --lda 4 --ldb 4")
    assert bench[6] == bench[0] + " --atomics_not_allowed"
    assert len(bench) == 7


def test_profile_counts_at_exit(tmp_path):
    out = _run(tmp_path, 4)
    assert out["trace"] is None and out["bench"] is None
    prof = out["profile"]
    # one line per distinct argument set, in first-seen order, written at process exit
    assert prof[0] == ('- { rocblas_function: "rocblas_dtrsm", atomics_mode: atomics_allowed, side: L, '
                       'uplo: L, transA: N, diag: N, m: -1, n: 8, lda: 8, ldb: 8, call_count: 3 }')
    assert prof[1].startswith('- { rocblas_function: "rocblas_strided_batched_dtrsm"')
    assert prof[1].endswith("stride_A: 16, ldb: 4, stride_B: 64, batch_count: 3, call_count: 1 }")
    # the call with atomics not allowed is a distinct argument set
    assert prof[4] == prof[0].replace("atomics_allowed", "atomics_not_allowed").replace("call_count: 3",
                                                                                      "call_count: 1")
    assert len(prof) == 5


def test_no_layer_no_files(tmp_path):
    out = _run(tmp_path, 0)
    assert out == {"trace": None, "bench": None, "profile": None}
