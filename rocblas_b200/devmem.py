"""Device-memory helpers for callers that hold column-major matrices as numpy arrays.

A column-major ``ld x ncols`` matrix is kept on the GPU as a C-contiguous torch tensor of
shape ``(ncols, ld)``: element (i, j) sits at ``j * ld + i``, exactly the layout the C ABI
expects.  PyTorch only provides device memory and streams here; every computation goes
through librocblas_b200.so.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import (
    DIAG, SIDE, TRANS, UPLO, check, datatype_f32_c, datatype_f32_r, datatype_f64_c, datatype_f64_r,
    lib, pointer_mode_device,
    pointer_mode_host, status_perf_degraded, status_success,
)


def to_device(a: np.ndarray, device="cuda") -> torch.Tensor:
    """Fortran-ordered (ld x ncols) numpy array -> (ncols x ld) device tensor, same bytes."""
    a = np.asfortranarray(a)
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(device)


def to_host(t: torch.Tensor) -> np.ndarray:
    """(ncols x ld) device tensor -> Fortran-ordered (ld x ncols) numpy array."""
    return np.asfortranarray(t.detach().cpu().numpy().T)


def empty(ld, ncols, dtype, device="cuda", fill=float("nan")) -> torch.Tensor:
    return torch.full((ncols, ld), fill, dtype=dtype, device=device)


def _code(table, v):
    return v if isinstance(v, int) else table[v]


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def _is_double(t):
    return t.dtype == torch.float64


_PREFIX = {torch.float32: "s", torch.float64: "d", torch.complex64: "c", torch.complex128: "z"}
_DATATYPE = {torch.float32: datatype_f32_r, torch.float64: datatype_f64_r,
             torch.complex64: datatype_f32_c, torch.complex128: datatype_f64_c}


def _fn(name, t):
    """rocblas_<s|d|c|z><name> for the element type of device tensor t."""
    return getattr(lib(), f"rocblas_{_PREFIX[t.dtype]}{name}")


def trsm(handle, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb, alpha_on_device=False,
         allow=(status_success,)):
    """rocblas_?trsm on device tensors; alpha is a Python float (host pointer mode) or, with
    alpha_on_device, placed in device memory and passed in device pointer mode."""
    fn = _fn("trsm", B)
    keep, aptr = _alpha(handle, alpha, B.dtype, alpha_on_device, B.device)
    st = fn(handle.value, _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans),
            _code(DIAG, diag), m, n, aptr, _ptr(A), lda, _ptr(B), ldb)
    _restore(handle, alpha_on_device)
    return check("rocblas_trsm", st, allow)


def trsm_refined(handle, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb, slices=0,
                 max_iterations=-1, check_columns=0, fallback=1, tolerance=0.0,
                 allow=(status_success,)):
    """rocblas_b200_dtrsm_refined on FP64 device tensors (host alpha); returns the
    rocblas_b200_refine_info fields as a dict."""
    from . import RefineInfo, RefineOptions

    a = ctypes.c_double(alpha)
    opts = RefineOptions(slices, max_iterations, check_columns, fallback, tolerance)
    info = RefineInfo()
    st = lib().rocblas_b200_dtrsm_refined(
        handle.value, _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans), _code(DIAG, diag), m, n,
        ctypes.cast(ctypes.byref(a), ctypes.c_void_p), _ptr(A), lda, _ptr(B), ldb,
        ctypes.cast(ctypes.byref(opts), ctypes.c_void_p), ctypes.cast(ctypes.byref(info), ctypes.c_void_p))
    check("rocblas_b200_dtrsm_refined", st, allow)
    return info.as_dict()


def trsm_ex(handle, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb, invA, invA_size,
            alpha_on_device=False, allow=(status_success,)):
    keep, aptr = _alpha(handle, alpha, B.dtype, alpha_on_device, B.device)
    st = lib().rocblas_trsm_ex(handle.value, _code(SIDE, side), _code(UPLO, uplo),
                               _code(TRANS, trans), _code(DIAG, diag), m, n, aptr, _ptr(A), lda,
                               _ptr(B), ldb, _ptr(invA), invA_size, _DATATYPE[B.dtype])
    _restore(handle, alpha_on_device)
    return check("rocblas_trsm_ex", st, allow)


def trsm_strided_batched(handle, side, uplo, trans, diag, m, n, alpha, A, lda, stride_a, B, ldb,
                         stride_b, batch, alpha_on_device=False, allow=(status_success,)):
    fn = _fn("trsm_strided_batched", B)
    keep, aptr = _alpha(handle, alpha, B.dtype, alpha_on_device, B.device)
    st = fn(handle.value, _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans),
            _code(DIAG, diag), m, n, aptr, _ptr(A), lda, stride_a, _ptr(B), ldb, stride_b, batch)
    _restore(handle, alpha_on_device)
    return check("rocblas_trsm_strided_batched", st, allow)


def trmm(handle, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb, C, ldc, alpha_on_device=False,
         allow=(status_success,)):
    """rocblas_?trmm on device tensors: C := alpha op(A) B (side L) or alpha B op(A) (side R);
    C may be B (in place, ldc == ldb)."""
    fn = _fn("trmm", C)
    keep, aptr = _alpha(handle, alpha, C.dtype, alpha_on_device, C.device)
    st = fn(handle.value, _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans), _code(DIAG, diag),
            m, n, aptr, _ptr(A), lda, _ptr(B), ldb, _ptr(C), ldc)
    _restore(handle, alpha_on_device)
    return check("rocblas_trmm", st, allow)


def trmm_strided_batched(handle, side, uplo, trans, diag, m, n, alpha, A, lda, stride_a, B, ldb,
                         stride_b, C, ldc, stride_c, batch, allow=(status_success,)):
    fn = _fn("trmm_strided_batched", C)
    keep, aptr = _alpha(handle, alpha, C.dtype, False, C.device)
    st = fn(handle.value, _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans), _code(DIAG, diag),
            m, n, aptr, _ptr(A), lda, stride_a, _ptr(B), ldb, stride_b, _ptr(C), ldc, stride_c, batch)
    return check("rocblas_trmm_strided_batched", st, allow)


def trsm_batched(handle, side, uplo, trans, diag, m, n, alpha, A_list, lda, B_list, ldb,
                 alpha_on_device=False, allow=(status_success,)):
    """A_list / B_list: lists of device tensors; their addresses are gathered into device
    arrays of device pointers, as the _batched API takes them."""
    fn = _fn("trsm_batched", B_list[0])
    dev = B_list[0].device
    Ap = torch.tensor([a.data_ptr() for a in A_list], dtype=torch.int64, device=dev)
    Bp = torch.tensor([b.data_ptr() for b in B_list], dtype=torch.int64, device=dev)
    keep, aptr = _alpha(handle, alpha, B_list[0].dtype, alpha_on_device, dev)
    st = fn(handle.value, _code(SIDE, side), _code(UPLO, uplo), _code(TRANS, trans),
            _code(DIAG, diag), m, n, aptr, _ptr(Ap), lda, _ptr(Bp), ldb, len(B_list))
    _restore(handle, alpha_on_device)
    torch.cuda.synchronize(dev)
    return check("rocblas_trsm_batched", st, allow)


def trtri(handle, uplo, diag, n, A, lda, invA, ldinv, allow=(status_success,)):
    dbl = _is_double(A)
    fn = lib().rocblas_dtrtri if dbl else lib().rocblas_strtri
    st = fn(handle.value, _code(UPLO, uplo), _code(DIAG, diag), n, _ptr(A), lda, _ptr(invA), ldinv)
    return check("rocblas_trtri", st, allow)


def trtri_strided_batched(handle, uplo, diag, n, A, lda, stride_a, invA, ldinv, stride_inv, batch,
                          a_offset=0, inv_offset=0, allow=(status_success,)):
    dbl = _is_double(A)
    fn = lib().rocblas_dtrtri_strided_batched if dbl else lib().rocblas_strtri_strided_batched
    es = A.element_size()
    st = fn(handle.value, _code(UPLO, uplo), _code(DIAG, diag), n,
            ctypes.c_void_p(A.data_ptr() + a_offset * es), lda, stride_a,
            ctypes.c_void_p(invA.data_ptr() + inv_offset * es), ldinv, stride_inv, batch)
    return check("rocblas_trtri_strided_batched", st, allow)


def _alpha(handle, alpha, dtype, on_device, device):
    """alpha of the call's element type, in host memory or (on_device) in device memory."""
    if on_device:
        t = torch.tensor([alpha], dtype=dtype, device=device)
        lib().rocblas_set_pointer_mode(handle.value, pointer_mode_device)
        return t, ctypes.c_void_p(t.data_ptr())
    t = torch.tensor([alpha], dtype=dtype)
    return t, ctypes.c_void_p(t.data_ptr())


def _restore(handle, on_device):
    if on_device:
        # the kernels read alpha asynchronously: keep its storage alive until they ran
        torch.cuda.synchronize()
        lib().rocblas_set_pointer_mode(handle.value, pointer_mode_host)


def build_invA(handle, uplo, diag, A, lda, k, nb=128):
    """invA for rocblas_trsm_ex, built the way rocblas-test builds it
    (clients/include/blas_ex/testing_trsm_ex.hpp:329-336, 408-436): trtri_strided_batched
    over the k // nb full blocks (stride nb*lda + nb in A, nb*nb in invA), then the
    remainder block with batch 1."""
    invA = torch.zeros(nb * k, dtype=A.dtype, device=A.device)
    nfull, rem = divmod(k, nb)
    if nfull:
        trtri_strided_batched(handle, uplo, diag, nb, A, lda, nb * lda + nb, invA, nb, nb * nb, nfull)
    if rem:
        trtri_strided_batched(handle, uplo, diag, rem, A, lda, 0, invA, nb, 0, 1,
                              a_offset=nfull * nb * lda + nfull * nb, inv_offset=nfull * nb * nb)
    return invA


__all__ = ["to_device", "to_host", "empty", "trsm", "trsm_ex", "trsm_strided_batched", "trmm",
           "trmm_strided_batched",
           "trsm_batched", "trtri", "trtri_strided_batched", "build_invA", "status_perf_degraded",
           "pointer_mode_host", "pointer_mode_device"]
