// The C ABI of librocblas_b200.so: handle functions, trsm / trsm_ex / trtri in their plain,
// _batched and _strided_batched forms.  Every entry point is `extern "C"`, catches every
// exception (as the reference's IMPL wrappers do, library/src/blas3/rocblas_trsm_imp.hpp:
// 285-314) and validates its arguments in the reference's order before touching the GPU.
#include <cuda.h> // CUcontext and CUresult for the driver entry points (no libcuda link)

#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <mutex>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/rocblas_b200_ext.h"
#include "check_numerics.cuh"
#include "layer_log.hpp"
#include "refine.cuh"
#include "sliced_driver.cuh"
#include "trsv_flag.cuh"
#include "trsm_driver.cuh"
#include "server.cuh"
#include "vbatched.cuh"
#include "vbatched_chain.cuh"

using namespace rb200;

// =========================================================================================
// handle
// =========================================================================================
void* _rocblas_handle::borrow(size_t bytes)
{
    bytes = roundup(bytes);
    if(bytes == 0)
        return mem; // may be nullptr; callers that need 0 bytes never dereference it
    if(owner != MemOwner::managed)
        return bytes <= mem_size ? mem : nullptr;
    if(bytes <= mem_size && mem)
        return mem;
    // grow: wait for work that may still use the old buffer, then reallocate
    if(mem)
    {
        cudaStreamSynchronize(stream);
        cudaFree(mem);
        mem      = nullptr;
        mem_size = 0;
    }
    if(cudaMalloc(&mem, bytes) != cudaSuccess)
    {
        cudaGetLastError();
        mem = nullptr;
        return nullptr;
    }
    mem_size = bytes;
    return mem;
}

rocblas_status _rocblas_handle::free_mem()
{
    if(mem && owner != MemOwner::user_owned)
    {
        cudaStreamSynchronize(stream);
        cudaFree(mem);
    }
    mem      = nullptr;
    mem_size = 0;
    owner    = MemOwner::managed;
    return rocblas_status_success;
}

namespace
{
// Device capability of the handle's device: 0 ok, otherwise a rocblas_status to return.
// Set by the complex trtri while it solves A X = I: complex solves then read a zero non-unit
// diagonal entry of A as 1 (the trtri rule), and no other call sees it.
thread_local bool t_zero_diag_is_one = false;

// Restores the device that was current when the scope began, if a call switched it: the
// handle's device is made current for the call only, as the reference's
// _rocblas_saved_device_id does (library/src/include/handle.hpp:134-170).
class DeviceScope
{
    int saved_ = -1;

public:
    DeviceScope() { cudaGetDevice(&saved_); }
    ~DeviceScope()
    {
        int cur = -1;
        if(saved_ >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != saved_)
            cudaSetDevice(saved_);
    }
    DeviceScope(const DeviceScope&)            = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
};

// Makes the handle's device current; the enclosing entry point holds a DeviceScope.
rocblas_status device_ready(rocblas_handle h)
{
    if(h->device < 0)
        return rocblas_status_internal_error; // no CUDA device was visible at create time
    int cur = -1;
    cudaGetDevice(&cur);
    if(cur != h->device)
        cudaSetDevice(h->device);
    return rocblas_status_success;
}

rocblas_status launch_status()
{
    cudaError_t e = cudaGetLastError();
    if(e == cudaSuccess)
        return rocblas_status_success;
    if(e == cudaErrorMemoryAllocation)
        return rocblas_status_memory_error;
    if(e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDeviceFunction)
        return rocblas_status_arch_mismatch;
    return rocblas_status_internal_error;
}

rocblas_status exception_status()
{
    try
    {
        throw;
    }
    catch(const std::bad_alloc&)
    {
        return rocblas_status_memory_error;
    }
    catch(...)
    {
        return rocblas_status_internal_error;
    }
}

template <typename T>
__global__ void zero_fill_kernel(BatchPtr<T> B, int64_t ldb, int m, int n, int batch_base)
{
    T*        b = B.get(batch_base + blockIdx.z);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if(i < m)
        b[i + (int64_t)j * ldb] = T(0);
}

// set_block_unit with val 0 (library/src/blas3/rocblas_trsm_kernels.hpp:213-265)
template <typename T>
void zero_fill(BatchPtr<T> B, int64_t ldb, int m, int n, int batch, cudaStream_t s)
{
    for(int b0 = 0; b0 < batch; b0 += kMaxGridYZ)
        for(int j0 = 0; j0 < n; j0 += kMaxGridYZ)
        {
            dim3 grid((unsigned)ceil_div(m, 256), (unsigned)std::min(kMaxGridYZ, n - j0),
                      (unsigned)std::min(kMaxGridYZ, batch - b0));
            zero_fill_kernel<T><<<grid, 256, 0, s>>>(B.shifted((int64_t)j0 * ldb), ldb, m,
                                                     std::min(kMaxGridYZ, n - j0), b0);
            count_launch();
        }
}

// rocblas_trsm_arg_check (library/src/blas3/rocblas_trsm.hpp:30-82)
template <typename T>
rocblas_status trsm_arg_check(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                              rocblas_operation trans, rocblas_diagonal diag, int64_t m,
                              int64_t n, const T* alpha, const void* A, int64_t lda,
                              const void* B, int64_t ldb, int64_t batch)
{
    if(side != rocblas_side_left && side != rocblas_side_right)
        return rocblas_status_invalid_value;
    if(uplo != rocblas_fill_lower && uplo != rocblas_fill_upper)
        return rocblas_status_invalid_value;
    if(trans != rocblas_operation_none && trans != rocblas_operation_transpose
       && trans != rocblas_operation_conjugate_transpose)
        return rocblas_status_invalid_value;
    if(diag != rocblas_diagonal_non_unit && diag != rocblas_diagonal_unit)
        return rocblas_status_invalid_value;
    const int64_t k = side == rocblas_side_left ? m : n;
    if(batch < 0 || m < 0 || n < 0 || lda < k || ldb < m)
        return rocblas_status_invalid_size;
    if(!m || !n || !batch)
        return h->size_query ? rocblas_status_size_unchanged : rocblas_status_success;
    if(!h->size_query)
    {
        if(!B || !alpha || (h->pointer_mode == rocblas_pointer_mode_host && *alpha != T(0) && !A))
            return rocblas_status_invalid_pointer;
    }
    return rocblas_status_continue;
}

int* ensure_err(rocblas_handle h);

// The body shared by all trsm entry points (rocblas_trsm_ex_impl,
// library/src/blas3/rocblas_trsm_imp.hpp:55-272 and its batched / strided twins).
template <typename T>
rocblas_status trsm_impl(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                         rocblas_operation trans, rocblas_diagonal diag, int m, int n,
                         const T* alpha, const void* Aptr, BatchPtr<T> A, int64_t lda,
                         const void* Bptr, BatchPtr<T> B, int64_t ldb, int batch,
                         const void* invA_ptr, BatchPtr<T> invA, int64_t invA_size,
                         int conj = -1)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    rocblas_status st
        = trsm_arg_check<T>(h, side, uplo, trans, diag, m, n, alpha, Aptr, lda, Bptr, ldb, batch);
    if(st != rocblas_status_continue)
        return st;

    if(h->pointer_mode == rocblas_pointer_mode_host && alpha && *alpha == T(0))
    {
        if(h->size_query)
            return rocblas_status_size_unchanged;
        if((st = device_ready(h)) != rocblas_status_success)
            return st;
        zero_fill<T>(B, ldb, m, n, batch, h->stream);
        return launch_status();
    }

    TrsmProblem<T> pr{};
    pr.side_left = side == rocblas_side_left;
    pr.upper     = uplo == rocblas_fill_upper;
    pr.trans     = trans != rocblas_operation_none;
    pr.unit      = diag == rocblas_diagonal_unit ? 1 : (is_cplx<T>::value && t_zero_diag_is_one ? 2 : 0);
    // complex trans C reads conj(A); trsv's side-right form of trans C asks for conj(A)
    // without the transpose through `conj`
    pr.conj = is_cplx<T>::value && (conj >= 0 ? conj != 0 : trans == rocblas_operation_conjugate_transpose);
    pr.m = m;
    pr.n = n;
    pr.batch = batch;
    pr.A = A;
    pr.lda = lda;
    pr.B = B;
    pr.ldb = ldb;
    pr.stream   = h->stream;
    pr.sm_count = h->sm_count;

    const int64_t k = pr.k();
    // a supplied invA smaller than 128 * k elements is ignored (rocblas_trsm_kernels.hpp:3832-3836)
    rocblas_status perf = rocblas_status_success;
    // complex solves use block-solver leaves and do not read a supplied invA
    bool           have_invA = invA_ptr != nullptr && !is_cplx<T>::value;
    if(have_invA && invA_size / kInvNB < k)
    {
        have_invA = false;
        perf      = rocblas_status_perf_degraded;
        static bool warned = false;
        if(!warned)
        {
            warned = true;
            fprintf(stderr, "WARNING: TRSM invA_size argument is too small; invA argument is being "
                            "ignored; TRSM performance is degraded\n");
        }
    }

    const size_t ws_bytes = trsm_workspace_bytes<T>(pr, have_invA);
    if(h->size_query)
        return ws_bytes ? h->set_optimal_size(ws_bytes) : rocblas_status_size_unchanged;

    if((st = device_ready(h)) != rocblas_status_success)
        return st;

    if(h->pointer_mode == rocblas_pointer_mode_host)
        pr.alpha.val = *alpha;
    else
        pr.alpha.ptr = alpha;

    void* ws = nullptr;
    if(ws_bytes)
    {
        ws = h->borrow(ws_bytes);
        if(!ws && !have_invA)
        {
            // backup: recursive solve with block-solver leaves needs no workspace
            perf = rocblas_status_perf_degraded;
            static bool warned = false;
            if(!warned)
            {
                warned = true;
                fprintf(stderr, "WARNING: Device memory allocation size is too small for TRSM; TRSM "
                                "performance is degraded\n");
            }
        }
    }
    if(have_invA)
        pr.invA = invA;
    pr.err_dev = h->err_dev;
    if(!pr.err_dev && ws && strsm_slice_bytes(pr))
        pr.err_dev = ensure_err(h); // the sliced FP32 updates' bounded waits report here
    trsm_run<T>(pr, ws, have_invA);
    st = launch_status();
    return st != rocblas_status_success ? st : perf;
}

template <typename T>
BatchPtr<T> strided(const T* p, int64_t stride)
{
    BatchPtr<T> b;
    b.base   = const_cast<T*>(p);
    b.stride = stride;
    return b;
}

template <typename T>
BatchPtr<T> arrayed(const void* arr)
{
    BatchPtr<T> b;
    b.arr = arr;
    return b;
}

// TA: the ABI's element type; T: the library's (same layout; cplx<R> for the complex structs)
template <typename T, typename TA>
const T* as_impl(const TA* p)
{
    return reinterpret_cast<const T*>(p);
}
template <typename T, typename TA>
T* as_impl(TA* p)
{
    return reinterpret_cast<T*>(p);
}

// ---- trmm ----------------------------------------------------------------------------------
// C := alpha op(A) B (side L) or alpha B op(A) (side R), A triangular; the reference's
// out-of-place API (rocblas-functions.h:18300-18393), with C == B allowed when ldc == ldb.
// One GEMM on the tiles of the solve with A's unused triangle masked at load time; a unit
// diagonal is the strict triangle plus B itself (C := alpha op(A_strict) B + alpha B).  In
// place, B is first copied to the workspace.

template <typename T>
__global__ void copy_matrix_kernel(BatchPtr<T> src, int64_t lds, BatchPtr<T> dst, int64_t ldd, int m,
                                   int n, int batch_base)
{
    const T*  s = src.get(batch_base + blockIdx.z);
    T*        d = dst.get(batch_base + blockIdx.z);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if(i < m)
        d[i + (int64_t)j * ldd] = s[i + (int64_t)j * lds];
}

template <typename T>
void copy_matrix(BatchPtr<T> src, int64_t lds, BatchPtr<T> dst, int64_t ldd, int m, int n, int batch,
                 cudaStream_t s)
{
    for(int b0 = 0; b0 < batch; b0 += kMaxGridYZ)
        for(int j0 = 0; j0 < n; j0 += kMaxGridYZ)
        {
            dim3 grid((unsigned)ceil_div(m, 256), (unsigned)std::min(kMaxGridYZ, n - j0),
                      (unsigned)std::min(kMaxGridYZ, batch - b0));
            copy_matrix_kernel<T><<<grid, 256, 0, s>>>(src.shifted((int64_t)j0 * lds), lds,
                                                       dst.shifted((int64_t)j0 * ldd), ldd, m,
                                                       std::min(kMaxGridYZ, n - j0), b0);
            count_launch();
        }
}

// rocblas_trmm_arg_check (library/src/blas3/rocblas_trmm.hpp:51-105)
template <typename T>
rocblas_status trmm_arg_check(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                              rocblas_operation trans, rocblas_diagonal diag, int64_t m, int64_t n,
                              const T* alpha, const void* A, int64_t lda, const void* B, int64_t ldb,
                              const void* C, int64_t ldc, int64_t batch)
{
    if(side != rocblas_side_left && side != rocblas_side_right)
        return rocblas_status_invalid_value;
    if(uplo != rocblas_fill_lower && uplo != rocblas_fill_upper)
        return rocblas_status_invalid_value;
    if(trans != rocblas_operation_none && trans != rocblas_operation_transpose
       && trans != rocblas_operation_conjugate_transpose)
        return rocblas_status_invalid_value;
    if(diag != rocblas_diagonal_non_unit && diag != rocblas_diagonal_unit)
        return rocblas_status_invalid_value;
    if(batch < 0 || m < 0 || n < 0 || ldc < m || ldb < m
       || (side == rocblas_side_left ? lda < m : lda < n))
        return rocblas_status_invalid_size;
    if(!m || !n || !batch)
        return h->size_query ? rocblas_status_size_unchanged : rocblas_status_success;
    if(!h->size_query)
    {
        if(!C || !alpha
           || (h->pointer_mode == rocblas_pointer_mode_host && *alpha != T(0) && (!A || !B)))
            return rocblas_status_invalid_pointer;
    }
    if(B == C && ldb != ldc)
        return rocblas_status_invalid_value;
    return rocblas_status_continue;
}

template <typename T>
rocblas_status trmm_impl(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                         rocblas_operation trans, rocblas_diagonal diag, int m, int n,
                         const T* alpha, const void* Aptr, BatchPtr<T> A, int64_t lda,
                         const void* Bptr, BatchPtr<T> B, int64_t ldb, const void* Cptr,
                         BatchPtr<T> C, int64_t ldc, int batch)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    rocblas_status st = trmm_arg_check<T>(h, side, uplo, trans, diag, m, n, alpha, Aptr, lda, Bptr,
                                          ldb, Cptr, ldc, batch);
    if(st != rocblas_status_continue)
        return st;
    const bool   in_place = Bptr == Cptr;
    const size_t ws_bytes = in_place ? sizeof(T) * (size_t)m * n * batch : 0;
    if(h->size_query)
        return ws_bytes ? h->set_optimal_size(ws_bytes) : rocblas_status_size_unchanged;
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    if(h->pointer_mode == rocblas_pointer_mode_host && *alpha == T(0))
    {
        zero_fill<T>(C, ldc, m, n, batch, h->stream);
        return launch_status();
    }
    BatchPtr<T> src = B;
    int64_t     lds = ldb;
    if(in_place)
    {
        void* ws = h->borrow(ws_bytes);
        if(!ws)
            return rocblas_status_memory_error;
        src.base   = reinterpret_cast<T*>(ws);
        src.arr    = nullptr;
        src.stride = (int64_t)m * n;
        src.offset = 0;
        lds        = m;
        copy_matrix<T>(B, ldb, src, lds, m, n, batch, h->stream);
    }
    const bool unit = diag == rocblas_diagonal_unit;
    if(unit && !in_place)
        copy_matrix<T>(B, ldb, C, ldc, m, n, batch, h->stream); // C := B, the diagonal's part
    const bool lower = uplo == rocblas_fill_lower;
    const int  tri   = unit ? (lower ? kTriLowerStrict : kTriUpperStrict) : (lower ? kTriLower : kTriUpper);
    GemmParams<T> g{};
    g.M = m;
    g.N = n;
    if(side == rocblas_side_left)
    {
        g.K = m;
        g.P = A; g.ldp = lda; g.transP = trans != rocblas_operation_none; g.triP = tri;
        g.conjP = trans == rocblas_operation_conjugate_transpose;
        g.Q = src; g.ldq = lds; g.transQ = 0; g.triQ = kTriNone;
    }
    else
    {
        g.K = n;
        g.P = src; g.ldp = lds; g.transP = 0; g.triP = kTriNone;
        g.Q = A; g.ldq = lda; g.transQ = trans != rocblas_operation_none; g.triQ = tri;
        g.conjQ = trans == rocblas_operation_conjugate_transpose;
    }
    g.C = C;
    g.ldc = ldc;
    g.a_imm = T(1); g.a_user = 1;              // a = alpha
    g.b_imm = T(0); g.b_user = unit ? 1 : 0;   // b = alpha (unit: C holds B) or 0
    g.ualpha.val = h->pointer_mode == rocblas_pointer_mode_host ? *alpha : T(1);
    g.ualpha.ptr = h->pointer_mode == rocblas_pointer_mode_host ? nullptr : alpha;
    g.zero_guard = 1;
    launch_gemm<T>(g, batch, h->stream, h->sm_count);
    return launch_status();
}

// ---- trsv ----------------------------------------------------------------------------------
// x := op(A)^-1 x (rocblas-functions.h:9900-9908, batched :10041-10050, strided :10198-10209).
// The vector x with increment incx > 0 is a 1 x n row matrix with leading dimension incx, and
// op(A) x = b is x^T op(A)^T = b^T: a trsm with side right, m = 1 and the transpose flipped.
// A negative increment (x traversed backwards) goes through a reversed contiguous copy.

template <typename T>
__global__ void trsv_reverse_kernel(BatchPtr<T> x, int64_t incx, T* tmp, int n, int to_tmp, int batch_base)
{
    const int b = batch_base + blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    // element i of the vector lives at x + (n - 1 - i) * |incx| when incx < 0
    T* xp = x.get(b) + (int64_t)(n - 1 - i) * (-incx);
    T* tp = tmp + (int64_t)b * n + i;
    if(to_tmp)
        *tp = *xp;
    else
        *xp = *tp;
}

// rocblas_trsv_arg_check (library/src/blas2/rocblas_trsv.hpp:31-80)
inline rocblas_status trsv_arg_check(rocblas_handle h, rocblas_fill uplo, rocblas_operation trans,
                                     rocblas_diagonal diag, int64_t n, const void* A, int64_t lda,
                                     const void* x, int64_t incx, int64_t batch)
{
    if(uplo != rocblas_fill_lower && uplo != rocblas_fill_upper)
        return rocblas_status_invalid_value;
    if(trans != rocblas_operation_none && trans != rocblas_operation_transpose
       && trans != rocblas_operation_conjugate_transpose)
        return rocblas_status_invalid_value;
    if(diag != rocblas_diagonal_unit && diag != rocblas_diagonal_non_unit)
        return rocblas_status_invalid_value;
    if(n < 0 || lda < n || lda < 1 || !incx || batch < 0)
        return rocblas_status_invalid_size;
    if(!n || !batch)
        return h->size_query ? rocblas_status_size_unchanged : rocblas_status_success;
    if(!h->size_query && (!A || !x))
        return rocblas_status_invalid_pointer;
    return rocblas_status_continue;
}

// The flag-synchronised solve (trsv_flag.cuh) with NR right-hand sides: a persistent grid of at
// most `sms` SMs' worth of CTAs, each taking its row blocks in increasing order, so that a block
// only waits on blocks that are done or in progress.
template <typename T, int NB, int NR, int TR = -1>
void launch_trsv_flag_nr(const TrsvParams<T>& p, int nblk, int sms, cudaStream_t s)
{
    constexpr size_t smem = trsv_flag_smem_bytes<T, NB, NR>();
    static int per_sm = 0;
    if(!per_sm)
    {
        cudaFuncSetAttribute((const void*)trsv_flag_kernel<T, NB, NR, TR>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsv_flag_kernel<T, NB, NR, TR>, kTvThreads, smem)
               != cudaSuccess
           || per_sm < 1)
        {
            cudaGetLastError();
            per_sm = 1;
        }
    }
    const int grid = std::min(nblk, sms * per_sm);
    trsv_flag_kernel<T, NB, NR, TR><<<grid, kTvThreads, smem, s>>>(p);
}

// one vector (rocblas_?trsv)
template <typename T, int NB>
void launch_trsv_flag(const TrsvParams<T>& p, int nblk, int sms, cudaStream_t s)
{
    launch_trsv_flag_nr<T, NB, 1>(p, nblk, sms, s);
}

template <typename T>
rocblas_status trsv_impl(rocblas_handle h, rocblas_fill uplo, rocblas_operation trans,
                         rocblas_diagonal diag, int n, const void* Aptr, BatchPtr<T> A, int64_t lda,
                         const void* xptr, BatchPtr<T> x, int64_t incx, int batch)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    rocblas_status ast = trsv_arg_check(h, uplo, trans, diag, n, Aptr, lda, xptr, incx, batch);
    if(ast != rocblas_status_continue)
        return ast;
    // one real vector with a positive increment: the memory-bound flag-synchronised solve
    if constexpr(!is_cplx<T>::value)
    {
        if(batch == 1 && incx > 0 && n >= tuning().trsv_flag_min_n)
        {
            const int    NB    = tuning().trsv_flag_nb == 128 ? 128 : 64;
            const int    nblk  = (int)ceil_div(n, NB);
            const size_t bytes = (size_t)nblk * sizeof(int);
            if(h->size_query)
                return h->set_optimal_size(bytes);
            rocblas_status st;
            if((st = device_ready(h)) != rocblas_status_success)
                return st;
            int*  err = ensure_err(h);
            void* ws  = h->borrow(bytes);
            if(err && ws)
            {
                cudaMemsetAsync(ws, 0, bytes, h->stream);
                TrsvParams<T> p{};
                p.A     = A.base + A.offset;
                p.lda   = lda;
                p.x     = x.base + x.offset;
                p.incx  = incx;
                p.nrhs  = 1;
                p.alpha = T(1);
                p.n     = n;
                const bool lower = uplo == rocblas_fill_lower;
                p.trans = trans != rocblas_operation_none;
                p.rev   = lower == p.trans; // op(A) upper: the solve starts at the last row
                p.unit  = diag == rocblas_diagonal_unit;
                p.flags = reinterpret_cast<int*>(ws);
                p.error = err;
                p.wait_cycles = 1ll << tuning().wait_cycles_log2;
                if(NB == 128)
                    launch_trsv_flag<T, 128>(p, nblk, h->sm_count, h->stream);
                else
                    launch_trsv_flag<T, 64>(p, nblk, h->sm_count, h->stream);
                count_launch();
                return launch_status();
            }
            // no workspace: the blocked path below needs none
        }
    }
    // op(A) x = b is x^T op(A)^T = b^T: op(A)^T is A^T for N, A for T, conj(A) for C
    const rocblas_operation flip
        = trans == rocblas_operation_none ? rocblas_operation_transpose : rocblas_operation_none;
    const int conj = trans == rocblas_operation_conjugate_transpose ? 1 : 0;
    static const T one = T(1);
    // the solve's alpha is 1 whatever the pointer mode
    const rocblas_pointer_mode mode = h->pointer_mode;
    h->pointer_mode                 = rocblas_pointer_mode_host;
    rocblas_status st;
    if(incx > 0)
    {
        st = trsm_impl<T>(h, rocblas_side_right, uplo, flip, diag, 1, n, &one, Aptr, A, lda, xptr, x,
                          incx, batch, nullptr, BatchPtr<T>{}, 0, conj);
    }
    else if(h->size_query)
    {
        st = trsm_impl<T>(h, rocblas_side_right, uplo, flip, diag, 1, n, &one, Aptr, A, lda, xptr, x,
                          1, batch, nullptr, BatchPtr<T>{}, 0, conj);
    }
    else
    {
        st = device_ready(h);
        T* tmp = nullptr;
        if(st == rocblas_status_success
           && cudaMallocAsync(reinterpret_cast<void**>(&tmp), sizeof(T) * (size_t)n * batch, h->stream)
                  != cudaSuccess)
        {
            cudaGetLastError();
            st = rocblas_status_memory_error;
        }
        if(st == rocblas_status_success)
        {
            for(int b0 = 0; b0 < batch; b0 += kMaxGridYZ)
            {
                dim3 grid((unsigned)ceil_div(n, 256), (unsigned)std::min(kMaxGridYZ, batch - b0));
                trsv_reverse_kernel<T><<<grid, 256, 0, h->stream>>>(x, incx, tmp, n, 1, b0);
                count_launch();
            }
            st = trsm_impl<T>(h, rocblas_side_right, uplo, flip, diag, 1, n, &one, Aptr, A, lda, tmp,
                              strided<T>(tmp, n), 1, batch, nullptr, BatchPtr<T>{}, 0, conj);
            if(st == rocblas_status_success || st == rocblas_status_perf_degraded)
                for(int b0 = 0; b0 < batch; b0 += kMaxGridYZ)
                {
                    dim3 grid((unsigned)ceil_div(n, 256), (unsigned)std::min(kMaxGridYZ, batch - b0));
                    trsv_reverse_kernel<T><<<grid, 256, 0, h->stream>>>(x, incx, tmp, n, 0, b0);
                    count_launch();
                }
            cudaFreeAsync(tmp, h->stream);
        }
    }
    h->pointer_mode = mode;
    return st;
}

// ---- ILP64 bodies ---------------------------------------------------------------------------
// The _64 entry points (rocblas_internal_trsm_launcher_64,
// library/src/src64/blas3/rocblas_trsm_kernels_64.cpp:31-225, and the trsv / trmm twins in
// library/src/src64/blas2/rocblas_trsv_kernels_64.cpp:28-86 and src64/blas3) take 64-bit sizes,
// leading dimensions, increments and batch counts.  Leading dimensions are 64-bit in every
// kernel of this library, so only sizes need splitting:
// * the order k of A stays a 32-bit size: A is k x k, so a larger k cannot be in memory, and the
//   reference returns invalid_size for it as this does;
// * the dimension of B that the solve (or product) treats independently - its columns for side
//   left, its rows for side right - is cut into chunks.  Columns of B are the GEMM tiles' grid
//   y dimension (at most 65535 tiles of at least 32 columns), so side left takes 2^20 columns
//   per chunk; rows are the grid x dimension, so side right takes 2^28 rows;
// * the batch is cut into chunks of 2^30.
// The 32-bit entry points run through the same bodies, so a 32-bit size beyond a chunk is
// split as well.
constexpr int64_t kIlpColChunk   = int64_t(1) << 20;
constexpr int64_t kIlpRowChunk   = int64_t(1) << 28;
constexpr int64_t kIlpBatchChunk = int64_t(1) << 30;

template <typename T>
BatchPtr<T> batch_advance(BatchPtr<T> p, int64_t b0)
{
    if(p.arr)
        p.arr = reinterpret_cast<T* const*>(p.arr) + b0;
    else if(p.base)
        p.base += b0 * p.stride;
    return p;
}

// Folds the statuses of chunked calls: an error ends the loop and is returned; otherwise
// perf_degraded (or, in a size query, size_increased) outranks success (size_unchanged).
struct ChunkStatus
{
    rocblas_status st = rocblas_status_continue;

    bool add(rocblas_status s)
    {
        const bool ok = s == rocblas_status_success || s == rocblas_status_perf_degraded
                        || s == rocblas_status_size_unchanged || s == rocblas_status_size_increased;
        if(!ok || st == rocblas_status_continue)
        {
            st = s;
            return ok;
        }
        if(s == rocblas_status_perf_degraded || s == rocblas_status_size_increased)
            st = s;
        return true;
    }
};

template <typename T>
constexpr char prec_letter()
{
    return std::is_same<T, float>::value ? 's' : std::is_same<T, double>::value ? 'd'
         : std::is_same<T, cplx<float>>::value ? 'c' : 'z';
}

// alpha's value for the log lines (read from the device in device pointer mode; NaN if null)
template <typename T>
void log_alpha(rocblas_handle h, const T* alpha, double* re, double* im)
{
    *re = *im = std::numeric_limits<double>::quiet_NaN();
    if(!alpha)
        return;
    T v;
    if(h->pointer_mode == rocblas_pointer_mode_device)
    {
        if(cudaMemcpyAsync(&v, alpha, sizeof(T), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess
           || cudaStreamSynchronize(h->stream) != cudaSuccess)
        {
            cudaGetLastError();
            return;
        }
    }
    else
        v = *alpha;
    if constexpr(is_cplx<T>::value)
    {
        *re = (double)v.x;
        *im = (double)v.y;
    }
    else
    {
        *re = (double)v;
        *im = 0.0;
    }
}

// Host <-> device copies of the auxiliary API (rocblas_auxiliary.cpp:305-790): the argument
// rules of the reference, one contiguous copy when both sides are dense, else one 2D copy (a
// vector with increments is a 2D copy of elem_size-byte rows). Copy errors are printed and the
// call still returns success, as the reference's PRINT_IF_HIP_ERROR does.
rocblas_status aux_copy_vector(int64_t n, int64_t es, const void* src, int64_t incs, void* dst,
                               int64_t incd, cudaMemcpyKind kind, cudaStream_t s, bool async)
{
    if(n == 0)
        return rocblas_status_success;
    if(n < 0 || incs <= 0 || incd <= 0 || es <= 0)
        return rocblas_status_invalid_size;
    if(!src || !dst)
        return rocblas_status_invalid_pointer;
    const size_t e = (size_t)es;
    cudaError_t  err;
    if(incs == 1 && incd == 1)
        err = async ? cudaMemcpyAsync(dst, src, e * n, kind, s) : cudaMemcpy(dst, src, e * n, kind);
    else
        err = async ? cudaMemcpy2DAsync(dst, e * incd, src, e * incs, e, n, kind, s)
                    : cudaMemcpy2D(dst, e * incd, src, e * incs, e, n, kind);
    if(err != cudaSuccess)
    {
        fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err));
        cudaGetLastError();
    }
    return rocblas_status_success;
}

rocblas_status aux_copy_matrix(int64_t rows, int64_t cols, int64_t es, const void* src, int64_t lds,
                               void* dst, int64_t ldd, cudaMemcpyKind kind, cudaStream_t s, bool async)
{
    if(rows == 0 || cols == 0)
        return rocblas_status_success;
    if(rows < 0 || cols < 0 || lds <= 0 || ldd <= 0 || rows > lds || rows > ldd || es <= 0)
        return rocblas_status_invalid_size;
    if(!src || !dst)
        return rocblas_status_invalid_pointer;
    const size_t e = (size_t)es;
    cudaError_t  err;
    if(lds == rows && ldd == rows)
        err = async ? cudaMemcpyAsync(dst, src, e * rows * cols, kind, s)
                    : cudaMemcpy(dst, src, e * rows * cols, kind);
    else
        err = async ? cudaMemcpy2DAsync(dst, e * ldd, src, e * lds, e * rows, cols, kind, s)
                    : cudaMemcpy2D(dst, e * ldd, src, e * lds, e * rows, cols, kind);
    if(err != cudaSuccess)
    {
        fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err));
        cudaGetLastError();
    }
    return rocblas_status_success;
}

int* ensure_err(rocblas_handle h);

// Check-numerics of A's referenced triangle (inputs only) and of B; the name is the entry
// point's, as in the log lines.
template <typename T>
rocblas_status trsm_check_numerics(rocblas_handle h, const TrsmLogInfo& li, rocblas_side side,
                                   rocblas_fill uplo, int64_t m, int64_t n, BatchPtr<T> A,
                                   int64_t lda, BatchPtr<T> B, int64_t ldb, int64_t batch,
                                   bool is_input)
{
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if(cudaStreamIsCapturing(h->stream, &cap) != cudaSuccess)
    {
        cudaGetLastError();
        return rocblas_status_internal_error;
    }
    if(cap != cudaStreamCaptureStatusNone)
        return rocblas_status_success;
    int* err = ensure_err(h);
    if(!err)
        return rocblas_status_memory_error;
    // the flags word sits beside the bounded-wait error word, in the same 256-byte allocation
    unsigned* flags_dev = reinterpret_cast<unsigned*>(err) + 32;
    const char* kinds[3] = {"", "batched_", "strided_batched_"};
    std::string name = std::string("rocblas_") + kinds[li.kind] + prec_letter<T>() + "trsm";
    if(li.ilp64)
        name += "_64";
    const int64_t k = side == rocblas_side_left ? m : n;
    unsigned      fa = 0, fb = 0;
    for(int64_t b0 = 0; b0 < batch; b0 += kIlpBatchChunk)
    {
        const int64_t nb = std::min(kIlpBatchChunk, batch - b0);
        unsigned      f  = 0;
        if(is_input)
        {
            if(!check_numerics_scan<T>(batch_advance(A, b0), lda, k, k, uplo == rocblas_fill_upper ? 2 : 1,
                                       nb, flags_dev, h->stream, &f))
                return launch_status();
            fa |= f;
        }
        if(!check_numerics_scan<T>(batch_advance(B, b0), ldb, m, n, 0, nb, flags_dev, h->stream, &f))
            return launch_status();
        fb |= f;
    }
    if(is_input)
    {
        const rocblas_status st = check_numerics_report(name.c_str(), h->check_numerics, true, fa);
        if(st != rocblas_status_success)
            return st;
    }
    return check_numerics_report(name.c_str(), h->check_numerics, is_input, fb);
}

// li: the calling entry point (log lines and check-numerics); nullptr for the library's own
// uses of the solve, which neither log nor check.
template <typename T>
rocblas_status trsm_impl_64(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                            rocblas_operation trans, rocblas_diagonal diag, int64_t m, int64_t n,
                            const T* alpha, const void* Aptr, BatchPtr<T> A, int64_t lda,
                            const void* Bptr, BatchPtr<T> B, int64_t ldb, int64_t batch,
                            const void* invA_ptr = nullptr, BatchPtr<T> invA = BatchPtr<T>{},
                            int64_t invA_size = 0, const TrsmLogInfo* li = nullptr)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    // layer logging comes before the argument check (rocblas_trsm_imp.hpp:74-143)
    if(li && h->layer_mode && !h->size_query)
    {
        TrsmLogCall c{};
        c.info = *li;
        c.prec = prec_letter<T>();
        c.side = side;
        c.uplo = uplo;
        c.trans = trans;
        c.diag = diag;
        c.m = m;
        c.n = n;
        log_alpha<T>(h, alpha, &c.alpha_re, &c.alpha_im);
        c.A = Aptr;
        c.B = Bptr;
        c.lda = lda;
        c.ldb = ldb;
        c.batch = batch;
        c.atomics = h->atomics_mode != 0;
        write_trsm_log(h->layer_mode, h->log_trace_os, h->log_bench_os, h->log_profile_os, c);
    }
    rocblas_status st
        = trsm_arg_check<T>(h, side, uplo, trans, diag, m, n, alpha, Aptr, lda, Bptr, ldb, batch);
    if(st != rocblas_status_continue)
        return st;
    const bool left = side == rocblas_side_left;
    if((left ? m : n) > INT32_MAX)
        return rocblas_status_invalid_size;
    // check-numerics of the inputs, after the host alpha == 0 quick return (which checks nothing)
    const bool check = li && h->check_numerics && !h->size_query
                       && !(h->pointer_mode == rocblas_pointer_mode_host && *alpha == T(0));
    if(check)
    {
        if((st = device_ready(h)) != rocblas_status_success)
            return st;
        if((st = trsm_check_numerics<T>(h, *li, side, uplo, m, n, A, lda, B, ldb, batch, true))
           != rocblas_status_success)
            return st;
    }
    const int64_t dim   = left ? n : m;
    const int64_t chunk = left ? kIlpColChunk : kIlpRowChunk;
    ChunkStatus   cs;
    for(int64_t b0 = 0; b0 < batch; b0 += kIlpBatchChunk)
    {
        const int nb = (int)std::min(kIlpBatchChunk, batch - b0);
        for(int64_t d0 = 0; d0 < dim; d0 += chunk)
        {
            const int nd = (int)std::min(chunk, dim - d0);
            st = trsm_impl<T>(h, side, uplo, trans, diag, left ? (int)m : nd, left ? nd : (int)n,
                              alpha, Aptr, batch_advance(A, b0), lda, Bptr,
                              batch_advance(B, b0).shifted(left ? d0 * ldb : d0), ldb, nb, invA_ptr,
                              batch_advance(invA, b0), invA_size);
            if(!cs.add(st))
                return cs.st;
        }
    }
    if(check && (cs.st == rocblas_status_success || cs.st == rocblas_status_perf_degraded))
    {
        // the result (rocblas_trsm_imp.hpp:248-270)
        st = trsm_check_numerics<T>(h, *li, side, uplo, m, n, A, lda, B, ldb, batch, false);
        if(st != rocblas_status_success)
            return st;
    }
    return cs.st;
}

template <typename T>
rocblas_status trsv_impl_64(rocblas_handle h, rocblas_fill uplo, rocblas_operation trans,
                            rocblas_diagonal diag, int64_t n, const void* Aptr, BatchPtr<T> A,
                            int64_t lda, const void* xptr, BatchPtr<T> x, int64_t incx,
                            int64_t batch)
{
    if(!h)
        return rocblas_status_invalid_handle;
    rocblas_status st = trsv_arg_check(h, uplo, trans, diag, n, Aptr, lda, xptr, incx, batch);
    if(st != rocblas_status_continue)
        return st;
    if(n > INT32_MAX)
        return rocblas_status_invalid_size;
    ChunkStatus cs;
    for(int64_t b0 = 0; b0 < batch; b0 += kIlpBatchChunk)
    {
        st = trsv_impl<T>(h, uplo, trans, diag, (int)n, Aptr, batch_advance(A, b0), lda, xptr,
                          batch_advance(x, b0), incx, (int)std::min(kIlpBatchChunk, batch - b0));
        if(!cs.add(st))
            return cs.st;
    }
    return cs.st;
}

template <typename T>
rocblas_status trmm_impl_64(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                            rocblas_operation trans, rocblas_diagonal diag, int64_t m, int64_t n,
                            const T* alpha, const void* Aptr, BatchPtr<T> A, int64_t lda,
                            const void* Bptr, BatchPtr<T> B, int64_t ldb, const void* Cptr,
                            BatchPtr<T> C, int64_t ldc, int64_t batch)
{
    if(!h)
        return rocblas_status_invalid_handle;
    rocblas_status st = trmm_arg_check<T>(h, side, uplo, trans, diag, m, n, alpha, Aptr, lda, Bptr,
                                          ldb, Cptr, ldc, batch);
    if(st != rocblas_status_continue)
        return st;
    const bool left = side == rocblas_side_left;
    if((left ? m : n) > INT32_MAX)
        return rocblas_status_invalid_size;
    const int64_t dim   = left ? n : m;
    const int64_t chunk = left ? kIlpColChunk : kIlpRowChunk;
    ChunkStatus   cs;
    for(int64_t b0 = 0; b0 < batch; b0 += kIlpBatchChunk)
    {
        const int nb = (int)std::min(kIlpBatchChunk, batch - b0);
        for(int64_t d0 = 0; d0 < dim; d0 += chunk)
        {
            const int nd = (int)std::min(chunk, dim - d0);
            st = trmm_impl<T>(h, side, uplo, trans, diag, left ? (int)m : nd, left ? nd : (int)n,
                              alpha, Aptr, batch_advance(A, b0), lda, Bptr,
                              batch_advance(B, b0).shifted(left ? d0 * ldb : d0), ldb, Cptr,
                              batch_advance(C, b0).shifted(left ? d0 * ldc : d0), ldc, nb);
            if(!cs.add(st))
                return cs.st;
        }
    }
    return cs.st;
}

// ---- trtri ---------------------------------------------------------------------------------
// rocblas_trtri_arg_check (library/src/blas3/rocblas_trtri.hpp:30-64)
rocblas_status trtri_arg_check(rocblas_fill uplo, rocblas_diagonal diag, int64_t n,
                               const void* A, int64_t lda, const void* invA, int64_t ldinvA,
                               int64_t batch)
{
    if(uplo != rocblas_fill_lower && uplo != rocblas_fill_upper)
        return rocblas_status_invalid_value;
    if(diag != rocblas_diagonal_non_unit && diag != rocblas_diagonal_unit)
        return rocblas_status_invalid_value;
    if(batch < 0 || n < 0 || lda < n || ldinvA < n)
        return rocblas_status_invalid_size;
    if(!n || !batch)
        return rocblas_status_success;
    if(!A || !invA)
        return rocblas_status_invalid_pointer;
    return rocblas_status_continue;
}

template <typename T>
size_t trtri_workspace_bytes(int n, int batch)
{
    if(n <= kInvNB)
        return 0;
    const int64_t half = ceil_div(ceil_div(n, kInvNB), 2) * kInvNB;
    return sizeof(T) * (size_t)half * (size_t)half * (size_t)batch;
}

// inv(A) for n > 128: diagonal blocks by the fused kernel, then recursive merges
//   lower: X21 = -X22 (A21 X11),   upper: X12 = -X11 (A12 X22)
// (the role of rocblas_trtri_large, library/src/blas3/rocblas_trtri.hpp:732-1100).
template <typename T>
struct TrtriRec
{
    int          n, upper;
    BatchPtr<T>  A, X, Tmp;
    int64_t      lda, ldx, ldt;
    int          batch;
    cudaStream_t s;

    int row_of(int b) const { return std::min(b * kInvNB, n); }

    void gemm(int M, int N, int K, BatchPtr<T> P, int64_t ldp, int triP, BatchPtr<T> Q,
              int64_t ldq, int triQ, BatchPtr<T> C, int64_t ldc, T a) const
    {
        GemmParams<T> g{};
        g.M = M; g.N = N; g.K = K;
        g.P = P; g.ldp = ldp; g.transP = 0; g.triP = triP;
        g.Q = Q; g.ldq = ldq; g.transQ = 0; g.triQ = triQ;
        g.C = C; g.ldc = ldc;
        g.a_imm = a; g.a_user = 0; g.b_imm = T(0); g.b_user = 0;
        g.zero_guard = 0;
        launch_gemm<T>(g, batch, s);
    }

    void run(int b0, int b1) const
    {
        if(b1 - b0 <= 1)
            return;
        const int bm = (b0 + b1) / 2;
        run(b0, bm);
        run(bm, b1);
        const int r0 = row_of(b0), rm = row_of(bm), r1 = row_of(b1);
        const int tri = upper ? kTriUpper : kTriLower;
        auto at = [](BatchPtr<T> p, int64_t ld, int i, int j) { return p.shifted(i + (int64_t)j * ld); };
        if(!upper)
        {
            const int M = r1 - rm, N = rm - r0;
            gemm(M, N, N, at(A, lda, rm, r0), lda, kTriNone, at(X, ldx, r0, r0), ldx, tri, Tmp, M, T(1));
            gemm(M, N, M, at(X, ldx, rm, rm), ldx, tri, Tmp, M, kTriNone, at(X, ldx, rm, r0), ldx, T(-1));
        }
        else
        {
            const int M = rm - r0, N = r1 - rm;
            gemm(M, N, N, at(A, lda, r0, rm), lda, kTriNone, at(X, ldx, rm, rm), ldx, tri, Tmp, M, T(1));
            gemm(M, N, M, at(X, ldx, r0, r0), ldx, tri, Tmp, M, kTriNone, at(X, ldx, r0, rm), ldx, T(-1));
        }
    }
};

template <typename T>
__global__ void set_unit_diagonal_kernel(BatchPtr<T> X, int64_t ld, int n, int batch_base)
{
    T*        x = X.get(batch_base + blockIdx.y);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n)
        x[i + (int64_t)i * ld] = T(1);
}

template <typename T>
rocblas_status trtri_impl(rocblas_handle h, rocblas_fill uplo, rocblas_diagonal diag, int n,
                          const void* Aptr, BatchPtr<T> A, int lda, const void* Xptr,
                          BatchPtr<T> X, int ldinv, int batch)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    if constexpr(is_cplx<T>::value)
    {
        // complex: inv(A) is the solution of A X = I, by the complex solve on invA itself (the
        // opposite triangle of the solution is exactly zero, as rocblas_trtri_fill leaves it).
        // A zero non-unit diagonal entry is read as 1, as the reference's trtri does
        // (library/src/blas3/rocblas_trtri.hpp:128-141): the solve's diagonal tiles apply that
        // rule while t_zero_diag_is_one is set.
        rocblas_status st = trtri_arg_check(uplo, diag, n, Aptr, lda, Xptr, ldinv, batch);
        if(h->size_query)
            return rocblas_status_size_unchanged;
        if(st != rocblas_status_continue)
            return st;
        if((st = device_ready(h)) != rocblas_status_success)
            return st;
        zero_fill<T>(X, ldinv, n, n, batch, h->stream);
        for(int b0 = 0; b0 < batch; b0 += kMaxGridYZ)
        {
            dim3 grid((unsigned)ceil_div(n, 256), (unsigned)std::min(kMaxGridYZ, batch - b0));
            set_unit_diagonal_kernel<T><<<grid, 256, 0, h->stream>>>(X, ldinv, n, b0);
            count_launch();
        }
        static const T             one = T(1);
        const rocblas_pointer_mode mode = h->pointer_mode;
        h->pointer_mode                 = rocblas_pointer_mode_host;
        t_zero_diag_is_one = true;
        st = trsm_impl_64<T>(h, rocblas_side_left, uplo, rocblas_operation_none, diag, n, n, &one, Aptr, A,
                             lda, Xptr, X, ldinv, batch, nullptr, BatchPtr<T>{}, 0);
        t_zero_diag_is_one = false;
        h->pointer_mode = mode;
        return st;
    }
    const size_t ws_bytes = trtri_workspace_bytes<T>(n, std::max(batch, 0));
    if(h->size_query)
    {
        if(!n || !ws_bytes)
            return rocblas_status_size_unchanged;
        return h->set_optimal_size(ws_bytes);
    }
    rocblas_status st = trtri_arg_check(uplo, diag, n, Aptr, lda, Xptr, ldinv, batch);
    if(st != rocblas_status_continue)
        return st;
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    void* ws = nullptr;
    if(ws_bytes && !(ws = h->borrow(ws_bytes)))
        return rocblas_status_memory_error;

    TrtriParams<T> t{};
    t.k = n;
    t.nb = kInvNB;
    t.A = A;
    t.lda = lda;
    t.inv = X;
    t.ldinv = ldinv;
    t.inv_block_stride = (int64_t)kInvNB * ldinv + kInvNB;
    t.upper = uplo == rocblas_fill_upper;
    t.unit = diag == rocblas_diagonal_unit;
    launch_trtri<T>(t, (int)ceil_div(n, kInvNB), batch, h->stream);
    if(n > kInvNB)
    {
        TrtriRec<T> r;
        r.n = n;
        r.upper = t.upper;
        r.A = A;
        r.X = X;
        r.lda = lda;
        r.ldx = ldinv;
        const int64_t half = ceil_div(ceil_div(n, kInvNB), 2) * kInvNB;
        r.Tmp = strided<T>(reinterpret_cast<T*>(ws), half * half);
        r.ldt = 0;
        r.batch = batch;
        r.s = h->stream;
        r.run(0, (int)ceil_div(n, kInvNB));
    }
    return launch_status();
}

__global__ void vb_copy_invalid_kernel(const int* invalid, rocblas_int* out)
{
    *out = *invalid;
}

static_assert(sizeof(VbProblem) == sizeof(rocblas_b200_trsm_problem), "descriptor layout");

// Persistent strip-solver launch over one queue; shared memory sized for systems up to kmax.
template <typename T>
void launch_vb_queue(rocblas_handle h, const VbParams<T>& p, int kmax)
{
    if(kmax <= kVbWarpMaxK)
    {
        // the smallest class: one strip per warp (vb_warp_kernel)
        const size_t smem   = vb_warp_smem_bytes<T>();
        int          per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vb_warp_kernel<T>, 32 * kVbWarpsPerCta, smem);
        per_sm = std::max(per_sm, 1);
        TimedLaunch tl(KernelClass::strip, h->stream, 0.0);
        vb_warp_kernel<T><<<h->sm_count * per_sm, 32 * kVbWarpsPerCta, smem, h->stream>>>(p);
        count_launch();
        return;
    }
    const size_t smem = block_solve_smem_bytes<T>(std::max(kmax, 1));
    cudaFuncSetAttribute((const void*)vb_persistent_kernel<T>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vb_persistent_kernel<T>, kBsThreads, smem);
    per_sm = std::max(per_sm, 1);
    TimedLaunch tl(KernelClass::strip, h->stream, 0.0);
    vb_persistent_kernel<T><<<h->sm_count * per_sm, kBsThreads, smem, h->stream>>>(p);
    count_launch();
}

template <typename T>
rocblas_status trsm_vbatched_impl(rocblas_handle h, const T* alpha,
                                  const rocblas_b200_trsm_problem* problems, int count,
                                  int max_k, rocblas_int* invalid_count)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    if(count < 0 || max_k < 0 || max_k > kBlockSolveMaxK)
        return rocblas_status_invalid_size;
    const size_t ws_bytes
        = sizeof(VbClassState) + sizeof(int) * (size_t)kVbClasses * ((size_t)count + 1);
    if(h->size_query)
        return count ? h->set_optimal_size(ws_bytes) : rocblas_status_size_unchanged;
    if(!count)
        return rocblas_status_success;
    if(!alpha || !problems)
        return rocblas_status_invalid_pointer;
    rocblas_status st;
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    void* ws = h->borrow(ws_bytes);
    if(!ws)
        return rocblas_status_memory_error;
    VbClassState* state   = reinterpret_cast<VbClassState*>(ws);
    int*          offsets = reinterpret_cast<int*>(state + 1);
    cudaMemsetAsync(state, 0, sizeof(VbClassState), h->stream);
    const VbProblem* probs = reinterpret_cast<const VbProblem*>(problems);
    vb_prepass_classes_kernel<<<1, kVbPrepThreads, 0, h->stream>>>(probs, count, max_k, INT_MAX,
                                                                    offsets, state);
    count_launch();

    VbParams<T> p;
    p.probs = probs;
    p.count = count;
    if(h->pointer_mode == rocblas_pointer_mode_host)
        p.alpha.val = *alpha;
    else
        p.alpha.ptr = alpha;
    // largest class first, so its long strips start while the small classes fill in behind
    for(int c = kVbClasses - 1; c >= 0; --c)
    {
        if(c > 0 && vb_class_kmax(c - 1) >= max_k)
            continue; // no valid system reaches this class
        p.offsets = offsets + (size_t)c * ((size_t)count + 1);
        p.counter = &state->counter[c];
        launch_vb_queue<T>(h, p, std::min(vb_class_kmax(c), std::max(max_k, 1)));
    }
    if(invalid_count)
    {
        vb_copy_invalid_kernel<<<1, 1, 0, h->stream>>>(&state->invalid, invalid_count);
        count_launch();
    }
    return launch_status();
}

// ---- variable-size batch of any order: strip solver for k <= 512, chain above -------------
__global__ void vb_sum_invalid_kernel(const int* a, const int* b, rocblas_int* out)
{
    *out = *a + *b;
}

template <typename T>
rocblas_status trsm_vbatched_ex_impl(rocblas_handle h, const T* alpha,
                                     const rocblas_b200_trsm_problem* problems,
                                     const T* const* invA, int count, int max_k, int max_n,
                                     rocblas_int* invalid_count)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    if(count < 0 || max_k < 0 || max_n < 0 || max_k > kChainVbMaxNB * kChainNB)
        return rocblas_status_invalid_size;
    const size_t        cls_bytes = sizeof(VbClassState) + sizeof(int) * (size_t)kVbClasses * ((size_t)count + 1);
    const bool          chain     = max_k > kChainVbMinK;
    const ChainVbLayout cl        = chain_vb_layout<T>(count, max_k, max_n);
    const size_t        cls_off   = chain ? cl.total : 0;
    const size_t        ws_bytes  = cls_off + cls_bytes;
    if(h->size_query)
        return count ? h->set_optimal_size(ws_bytes) : rocblas_status_size_unchanged;
    if(!count)
        return rocblas_status_success;
    if(!alpha || !problems || (chain && !invA))
        return rocblas_status_invalid_pointer;
    rocblas_status st;
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    char* ws = reinterpret_cast<char*>(h->borrow(ws_bytes));
    if(!ws)
        return rocblas_status_memory_error;
    const VbProblem* probs = reinterpret_cast<const VbProblem*>(problems);
    Scalar<T>        a;
    if(h->pointer_mode == rocblas_pointer_mode_host)
        a.val = *alpha;
    else
        a.ptr = alpha;

    // chain part: systems with k > 512
    ChainVbWork<T> w{};
    if(chain)
    {
        w.hdr      = reinterpret_cast<ChainVbHeader<T>*>(ws + cl.hdr);
        w.sys      = reinterpret_cast<ChainSys<T>*>(ws + cl.sys);
        w.P        = reinterpret_cast<int*>(ws + cl.P);
        w.G        = reinterpret_cast<int*>(ws + cl.G);
        w.cnt      = reinterpret_cast<int*>(ws + cl.cnt);
        w.L        = reinterpret_cast<int64_t*>(ws + cl.L);
        w.flags    = reinterpret_cast<int*>(ws + cl.flags);
        w.flag_cap = cl.flag_cap;
        w.counters = reinterpret_cast<unsigned long long*>(ws + cl.counters);
        w.invalid  = reinterpret_cast<int*>(ws + cl.invalid);
        // counters, invalid and every flag start at zero
        cudaMemsetAsync(ws + cl.counters, 0, cl.total - cl.counters, h->stream);
        chain_vb_prepass_kernel<T><<<1, kVbPrepThreads, 0, h->stream>>>(probs, invA, count, max_k,
                                                                        max_n, w);
        count_launch();
        for(int c = 0; c < kChainVbCombos; ++c)
        {
            ChainParams<T> p{};
            p.vhdr    = w.hdr + c;
            p.alpha   = a;
            p.first   = 1;
            p.counter = reinterpret_cast<int*>(w.counters + c);
            p.error   = h->err_dev ? h->err_dev : w.invalid + 1;
            p.wait_cycles = 1ll << tuning().wait_cycles_log2;
            const bool kcp = ((c >> 1) & 1) != 0, kcq = (c & 1) != 0;
            if(chain_vb_width(c) == kChainVbWideW)
                launch_chain_w<T, kChainVbWideW, true>(p, kcp, kcq, h->sm_count, INT64_MAX, h->stream);
            else
                launch_chain_w<T, kChainVbW, true>(p, kcp, kcq, h->sm_count, INT64_MAX, h->stream);
            count_launch();
        }
    }

    // strip-solver part: systems with k <= 512
    VbClassState* state   = reinterpret_cast<VbClassState*>(ws + cls_off);
    int*          offsets = reinterpret_cast<int*>(state + 1);
    cudaMemsetAsync(state, 0, sizeof(VbClassState), h->stream);
    const int kb = std::min(max_k, kChainVbMinK);
    vb_prepass_classes_kernel<<<1, kVbPrepThreads, 0, h->stream>>>(probs, count, kb, kChainVbMinK,
                                                                    offsets, state);
    count_launch();
    VbParams<T> p;
    p.probs = probs;
    p.count = count;
    p.alpha = a;
    for(int c = kVbClasses - 1; c >= 0; --c)
    {
        if(c > 0 && vb_class_kmax(c - 1) >= kb)
            continue;
        p.offsets = offsets + (size_t)c * ((size_t)count + 1);
        p.counter = &state->counter[c];
        launch_vb_queue<T>(h, p, std::min(vb_class_kmax(c), std::max(kb, 1)));
    }
    if(invalid_count)
    {
        if(chain)
            vb_sum_invalid_kernel<<<1, 1, 0, h->stream>>>(&state->invalid, w.invalid, invalid_count);
        else
            vb_copy_invalid_kernel<<<1, 1, 0, h->stream>>>(&state->invalid, invalid_count);
        count_launch();
    }
    return launch_status();
}

// collection solve of the server: the variable-size batch of any order with alpha 1
rocblas_status server_solve(_rocblas_handle* h, int dtype, const rocblas_b200_trsm_problem* probs,
                            const void* invs, int count, int max_k, int max_n)
{
    if(dtype == TrsmServerCore::kF64)
    {
        static const double one = 1.0;
        return trsm_vbatched_ex_impl<double>(h, &one, probs, reinterpret_cast<const double* const*>(invs),
                                             count, max_k, max_n, nullptr);
    }
    static const float one = 1.0f;
    return trsm_vbatched_ex_impl<float>(h, &one, probs, reinterpret_cast<const float* const*>(invs),
                                        count, max_k, max_n, nullptr);
}

static_assert(sizeof(ServerRequestC) == sizeof(rocblas_b200_request), "request layout");
static_assert(sizeof(ServerStatsC) == sizeof(rocblas_b200_server_stats), "stats layout");

// ---- variable-size batch without any allocation ------------------------------------------
// Scratch of rocblas_b200_dtrsm_vbatched_noalloc: the queue state and the prefix sums of work
// items for at most kVbNoAllocMaxCount descriptors, in a fixed device array that every GPU
// loading the library holds until exit (256 KiB + 16 B).  Host code reaches it only through
// the address cudaGetSymbolAddress returns for the current device.
constexpr int kVbNoAllocMaxCount = 65536;
static __device__ __align__(256) unsigned char
    g_vb_noalloc_scratch[sizeof(VbState) + sizeof(int) * (kVbNoAllocMaxCount + 1)];

constexpr int kVbNoAllocMaxDevices = 64;
std::mutex    g_vb_noalloc_mutex;
// per device: the address found at set-up and the unique id of the context it belongs to (a
// symbol's address is only valid in the context that loaded the module; after a device reset
// or primary-context teardown the next context gets a new id and the lookup is made again)
void*              g_vb_noalloc_addr[kVbNoAllocMaxDevices] = {};
unsigned long long g_vb_noalloc_ctx[kVbNoAllocMaxDevices]  = {};

// Unique id of the current context (cuCtxGetId, reached through the runtime's driver entry
// points so the library does not link libcuda).  0 if there is none or it cannot be read.
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId      = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId      get_id      = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if(cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) ==
               cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if(cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) ==
               cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    CUcontext          ctx = nullptr;
    unsigned long long id  = 0;
    if(!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx ||
       get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of the scratch array on `device`, which must be current (the runtime has made
// its primary context current by then).  Set-up looks it up once per device and context;
// without a readable context id it is looked up on every call.  nullptr if the lookup fails.
void* vb_noalloc_scratch(int device)
{
    if(device < 0 || device >= kVbNoAllocMaxDevices)
        return nullptr;
    std::lock_guard<std::mutex> lock(g_vb_noalloc_mutex);
    const unsigned long long ctx = current_context_id();
    if(!g_vb_noalloc_addr[device] || ctx == 0 || ctx != g_vb_noalloc_ctx[device])
    {
        void* ptr = nullptr;
        if(cudaGetSymbolAddress(&ptr, g_vb_noalloc_scratch) != cudaSuccess)
        {
            cudaGetLastError();
            g_vb_noalloc_addr[device] = nullptr;
            return nullptr;
        }
        g_vb_noalloc_addr[device] = ptr;
        g_vb_noalloc_ctx[device]  = ctx;
    }
    return g_vb_noalloc_addr[device];
}

rocblas_status trsm_vbatched_noalloc_impl(rocblas_handle h, const double* alpha,
                                          const rocblas_b200_trsm_problem* problems, int count,
                                          int max_k, rocblas_int* invalid_count)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    if(count < 0 || max_k < 0 || max_k > kBlockSolveMaxK)
        return rocblas_status_invalid_size;
    if(count > kVbNoAllocMaxCount)
    {
        fprintf(stderr,
                "rocblas_b200_dtrsm_vbatched_noalloc: count %d exceeds the fixed scratch limit of "
                "%d systems; use rocblas_b200_dtrsm_vbatched\n",
                count, kVbNoAllocMaxCount);
        return rocblas_status_invalid_size;
    }
    if(h->size_query)
        return rocblas_status_size_unchanged; // needs no workspace
    if(!count)
        return rocblas_status_success;
    if(!alpha || !problems)
        return rocblas_status_invalid_pointer;
    rocblas_status st;
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    void* scratch = vb_noalloc_scratch(h->device);
    if(!scratch)
        return rocblas_status_internal_error;
    VbState* state   = reinterpret_cast<VbState*>(scratch);
    int*     offsets = reinterpret_cast<int*>(state + 1);
    // the queue head and the invalid count must start at zero; the previous call left its values
    cudaMemsetAsync(state, 0, sizeof(VbState), h->stream);
    const VbProblem* probs = reinterpret_cast<const VbProblem*>(problems);
    vb_prepass_kernel<<<1, kVbPrepThreads, 0, h->stream>>>(probs, count, max_k, offsets, state);
    count_launch();
    VbParams<double> p;
    p.probs   = probs;
    p.count   = count;
    p.offsets = offsets;
    p.counter = &state->counter;
    if(h->pointer_mode == rocblas_pointer_mode_host)
        p.alpha.val = *alpha;
    else
        p.alpha.ptr = alpha;
    launch_vb_queue<double>(h, p, max_k);
    if(invalid_count)
    {
        vb_copy_invalid_kernel<<<1, 1, 0, h->stream>>>(&state->invalid, invalid_count);
        count_launch();
    }
    return launch_status();
}

int* ensure_err(rocblas_handle h)
{
    if(!h->err_dev)
    {
        if(cudaMalloc(&h->err_dev, 256) != cudaSuccess)
        {
            cudaGetLastError();
            h->err_dev = nullptr;
            return nullptr;
        }
        cudaMemset(h->err_dev, 0, 256);
    }
    return h->err_dev;
}

rocblas_status gemm_sliced_impl(rocblas_handle h, rocblas_operation ta, rocblas_operation tb, int m,
                                int n, int k, const double* alpha, const double* A, int lda,
                                const double* B, int ldb, const double* beta, double* C, int ldc,
                                int slices, int moduli = 0)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    auto okop = [](rocblas_operation t) {
        return t == rocblas_operation_none || t == rocblas_operation_transpose
               || t == rocblas_operation_conjugate_transpose;
    };
    if(!okop(ta) || !okop(tb) || slices < 1 || slices > kOzMaxS)
        return rocblas_status_invalid_value;
    if(moduli && !crt_moduli_supported(moduli))
        return rocblas_status_invalid_value;
    const bool nA = ta == rocblas_operation_none, nB = tb == rocblas_operation_none;
    if(m < 0 || n < 0 || k < 0 || lda < (nA ? m : k) || ldb < (nB ? k : n) || ldc < m)
        return rocblas_status_invalid_size;
    if(!m || !n)
        return h->size_query ? rocblas_status_size_unchanged : rocblas_status_success;
    const size_t ws_bytes = update_workspace_bytes(m, n, k, slices, moduli, h->sm_count);
    if(h->size_query)
        return h->set_optimal_size(ws_bytes);
    if(!alpha || !beta || !C || (k && (!A || !B)))
        return rocblas_status_invalid_pointer;
    if(h->pointer_mode != rocblas_pointer_mode_host)
        return rocblas_status_not_implemented;
    rocblas_status st;
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    int* err = ensure_err(h);
    void* ws = h->borrow(ws_bytes);
    if(!ws || !err)
        return rocblas_status_memory_error;
    SlicedGemm g{};
    g.sms = h->sm_count;
    g.M = m;
    g.N = n;
    g.K = k;
    g.S = slices;
    g.moduli = moduli;
    g.P = nA ? SliceOperand{A, 1, lda} : SliceOperand{A, lda, 1};
    g.Q = nB ? SliceOperand{B, ldb, 1} : SliceOperand{B, 1, ldb};
    g.C = C;
    g.ldc = ldc;
    g.a = *alpha;
    g.b_imm = *beta;
    if(!run_sliced_gemm(g, ws, err, h->stream))
        return rocblas_status_arch_mismatch;
    return launch_status();
}

// C := alpha op(A) op(B) + beta C on the FP64 DMMA tiles (host pointer mode).
// C := alpha op(A) op(B) + beta C on the tiles of the trsm updates (FP64: DMMA; complex: the
// complex DMMA tiles, trans C conjugating), with rocblas_?gemm's argument meaning.
template <typename T>
rocblas_status gemm_tiles_impl(rocblas_handle h, rocblas_operation ta, rocblas_operation tb, int m,
                               int n, int k, const T* alpha, const T* A, int lda, const T* B,
                               int ldb, const T* beta, T* C, int ldc)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    auto okop = [](rocblas_operation t) {
        return t == rocblas_operation_none || t == rocblas_operation_transpose
               || t == rocblas_operation_conjugate_transpose;
    };
    if(!okop(ta) || !okop(tb))
        return rocblas_status_invalid_value;
    const bool nA = ta == rocblas_operation_none, nB = tb == rocblas_operation_none;
    if(m < 0 || n < 0 || k < 0 || lda < (nA ? m : k) || ldb < (nB ? k : n) || ldc < m)
        return rocblas_status_invalid_size;
    if(!m || !n)
        return h->size_query ? rocblas_status_size_unchanged : rocblas_status_success;
    if(h->size_query)
        return rocblas_status_size_unchanged;
    if(!alpha || !beta || !C || (k && (!A || !B)))
        return rocblas_status_invalid_pointer;
    if(h->pointer_mode != rocblas_pointer_mode_host)
        return rocblas_status_not_implemented;
    rocblas_status st;
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    GemmParams<T> g{};
    g.M = m;
    g.N = n;
    g.K = k;
    g.P = strided<T>(A, 0);
    g.ldp = lda;
    g.transP = nA ? 0 : 1;
    g.conjP  = ta == rocblas_operation_conjugate_transpose;
    g.Q = strided<T>(B, 0);
    g.ldq = ldb;
    g.transQ = nB ? 0 : 1;
    g.conjQ  = tb == rocblas_operation_conjugate_transpose;
    g.C = strided<T>(C, 0);
    g.ldc = ldc;
    g.a_imm = *alpha;
    g.b_imm = *beta;
    g.zero_guard = 0;
    launch_gemm<T>(g, 1, h->stream, h->sm_count);
    return launch_status();
}

// Workspace of one precision-form solve: invA blocks, the largest sliced update's slice
// panels, the chain sub-solves' flags (all zero when the problem is small enough for the plain
// path, which needs none).
struct MixedPlan
{
    bool   recursive = false;
    size_t inv_bytes = 0, sl_bytes = 0, ch_bytes = 0, total = 0;
};

MixedPlan mixed_plan(const TrsmProblem<double>& pr, int slices, int moduli)
{
    MixedPlan p;
    p.recursive = choose_algo(pr) == Algo::recursive;
    if(!p.recursive)
        return p;
    p.inv_bytes = align256((size_t)kInvNB * pr.k() * sizeof(double));
    p.sl_bytes  = mixed_slice_workspace_bytes(pr, slices, moduli);
    p.ch_bytes  = mixed_chain_workspace_bytes(pr);
    p.total     = p.inv_bytes + align256(p.sl_bytes) + align256(p.ch_bytes);
    return p;
}

// The precision-form solve of pr (alpha, A, B as set there) on the workspace laid out by
// mixed_plan.  invA is built into the workspace when build_inv, else the blocks already there
// (from an earlier solve with the same A) are used.  false if the GPU lacks the tensor path.
bool mixed_run(TrsmProblem<double> pr, int slices, int moduli, const MixedPlan& plan, void* ws, int* err,
               bool build_inv)
{
    if(!plan.recursive)
    {
        trsm_run<double>(pr, nullptr, false);
        return true;
    }
    pr.err_dev = err;
    BatchPtr<double> inv;
    inv.base   = reinterpret_cast<double*>(ws);
    inv.stride = (int64_t)kInvNB * pr.k();
    if(build_inv)
        build_invA<double>(pr, inv);
    pr.invA = inv;
    MixedRecursive rec{{pr, (int)pr.k(), (int)ceil_div(pr.k(), kInvNB)}};
    rec.S        = slices;
    rec.moduli   = moduli;
    rec.slice_ws = reinterpret_cast<unsigned char*>(ws) + plan.inv_bytes;
    rec.err_dev  = err;
    if(plan.ch_bytes)
        rec.chain_ws = reinterpret_cast<unsigned char*>(ws) + plan.inv_bytes + align256(plan.sl_bytes);
    rec.solve_mixed(0, rec.nblk, 1);
    return rec.ok;
}

rocblas_status trsm_mixed_impl(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                               rocblas_operation trans, rocblas_diagonal diag, int m, int n,
                               const double* alpha, const double* A, int lda, double* B, int ldb,
                               int slices)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    rocblas_status st
        = trsm_arg_check<double>(h, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb, 1);
    if(st != rocblas_status_continue)
        return st;
    // slices 0: the tuning table's engine (the residue engine with mixed_moduli moduli, or
    // mixed_slices slices); 1..8: the slice engine with that many slices
    const int moduli = slices == 0 ? tuning().mixed_moduli : 0;
    if(slices == 0)
        slices = tuning().mixed_slices;
    if(slices < 1 || slices > kOzMaxS)
        return rocblas_status_invalid_value;
    if(h->pointer_mode == rocblas_pointer_mode_host && alpha && *alpha == 0.0)
    {
        if(h->size_query)
            return rocblas_status_size_unchanged;
        if((st = device_ready(h)) != rocblas_status_success)
            return st;
        zero_fill<double>(strided<double>(B, 0), ldb, m, n, 1, h->stream);
        return launch_status();
    }
    TrsmProblem<double> pr{};
    pr.side_left = side == rocblas_side_left;
    pr.upper     = uplo == rocblas_fill_upper;
    pr.trans     = trans != rocblas_operation_none;
    pr.unit      = diag == rocblas_diagonal_unit;
    pr.m = m;
    pr.n = n;
    pr.batch = 1;
    pr.A = strided<double>(A, 0);
    pr.lda = lda;
    pr.B = strided<double>(B, 0);
    pr.ldb = ldb;
    pr.stream   = h->stream;
    pr.sm_count = h->sm_count;
    const MixedPlan plan = mixed_plan(pr, slices, moduli);
    if(h->size_query)
        return plan.total ? h->set_optimal_size(plan.total) : rocblas_status_size_unchanged;
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    if(h->pointer_mode == rocblas_pointer_mode_host)
        pr.alpha.val = *alpha;
    else
        pr.alpha.ptr = alpha;
    int*  err = plan.recursive ? ensure_err(h) : nullptr;
    void* ws  = plan.total ? h->borrow(plan.total) : nullptr;
    if(plan.recursive && (!ws || !err))
        return rocblas_status_memory_error;
    if(!mixed_run(pr, slices, moduli, plan, ws, err, true))
        return rocblas_status_arch_mismatch;
    return launch_status();
}

// ---- host-buffer precision form (rocblas_b200_dtrsm_mixed_host) -----------------------------
} // namespace

// Streams, events and the device buffers of the host-buffer entry points, per handle.
struct HostPathRes
{
    cudaStream_t             in = nullptr, out = nullptr, tri = nullptr;
    std::vector<cudaEvent_t> ev;
    void*                    dbuf   = nullptr;
    size_t                   dbytes = 0;

    bool init()
    {
        if(in)
            return true;
        if(cudaStreamCreateWithFlags(&in, cudaStreamNonBlocking) != cudaSuccess
           || cudaStreamCreateWithFlags(&out, cudaStreamNonBlocking) != cudaSuccess
           || cudaStreamCreateWithFlags(&tri, cudaStreamNonBlocking) != cudaSuccess)
        {
            cudaGetLastError();
            return false;
        }
        return true;
    }
    cudaEvent_t event(size_t i)
    {
        while(ev.size() <= i)
        {
            cudaEvent_t e = nullptr;
            if(cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            {
                cudaGetLastError();
                return nullptr;
            }
            ev.push_back(e);
        }
        return ev[i];
    }
    void* buffer(size_t bytes)
    {
        if(bytes <= dbytes)
            return dbuf;
        if(dbuf)
            cudaFree(dbuf);
        dbuf   = nullptr;
        dbytes = 0;
        if(cudaMalloc(&dbuf, bytes) != cudaSuccess)
        {
            cudaGetLastError();
            return nullptr;
        }
        dbytes = bytes;
        return dbuf;
    }
    void release()
    {
        if(in)
            cudaStreamSynchronize(in);
        if(out)
            cudaStreamSynchronize(out);
        if(tri)
            cudaStreamSynchronize(tri);
        for(auto e : ev)
            cudaEventDestroy(e);
        ev.clear();
        if(dbuf)
            cudaFree(dbuf);
        if(in)
            cudaStreamDestroy(in);
        if(out)
            cudaStreamDestroy(out);
        if(tri)
            cudaStreamDestroy(tri);
        in = out = tri = nullptr;
        dbuf      = nullptr;
        dbytes    = 0;
    }
};

namespace
{

// ---- precision form with iterative refinement (rocblas_b200_dtrsm_refined) -------------------
// Mixed-precision iterative refinement (Wilkinson's; Buttari, Dongarra et al. 2007 for the
// form of LAPACK's dsgesv) around the sliced solve: the test compares the result on a sample
// of right-hand sides with the plain FP64 form's solution of the same right-hand sides, solved
// on a second stream while the sliced solve runs; corrections use FP64 residuals on the DMMA
// tiles and the sliced solve with the first solve's invA.

// C := C - op(A) X (side left, C rows x cols, K = m) or C - X op(A) (side right, K = n) in FP64
// on the DMMA tiles; A's triangle is masked at load time (the strict triangle for a unit
// diagonal, whose part the caller has already put into C), and K blocks outside it are skipped.
void refine_product(const TrsmProblem<double>& pr, const double* X, int64_t ldx, double* C, int64_t ldc,
                    int rows, int cols)
{
    GemmParams<double> g{};
    const int tri = pr.unit ? (pr.upper ? kTriUpperStrict : kTriLowerStrict) : (pr.upper ? kTriUpper : kTriLower);
    g.M = rows;
    g.N = cols;
    if(pr.side_left)
    {
        g.K = pr.m;
        g.P = pr.A; g.ldp = pr.lda; g.transP = pr.trans; g.triP = tri;
        g.Q = strided<double>(X, 0); g.ldq = ldx; g.transQ = 0; g.triQ = kTriNone;
    }
    else
    {
        g.K = pr.n;
        g.P = strided<double>(X, 0); g.ldp = ldx; g.transP = 0; g.triP = kTriNone;
        g.Q = pr.A; g.ldq = pr.lda; g.transQ = pr.trans; g.triQ = tri;
    }
    g.C = strided<double>(C, 0);
    g.ldc = ldc;
    g.a_imm = -1.0; g.a_user = 0;
    g.b_imm = 1.0;  g.b_user = 0;
    g.ualpha.val = 1.0;
    g.zero_guard = 0;
    launch_gemm<double>(g, 1, pr.stream, pr.sm_count);
}

// O := alpha B0(src) - (unit ? X(src) : 0) and, when Xs is given, Xs := X(src), for the rows x
// cols output O (ld ldo); X is pr's B.  sampled: src picks the tested right-hand sides.
void refine_prep(const TrsmProblem<double>& pr, const double* B0, int64_t ldb0, int rows, int cols, int sampled,
                 int64_t nrhs, double alpha, int unit, double* O, int64_t ldo, double* Xs)
{
    const dim3 grid((unsigned)ceil_div(rows, 256), (unsigned)std::min(cols, 65535));
    refine_prep_kernel<<<grid, 256, 0, pr.stream>>>(pr.B.base, pr.ldb, B0, ldb0, rows, cols, sampled,
                                                    pr.side_left, nrhs, alpha, unit, O, ldo, Xs, ldo);
    count_launch();
}

rocblas_status trsm_refined_impl(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                                 rocblas_operation trans, rocblas_diagonal diag, int m, int n,
                                 const double* alpha, const double* A, int lda, double* B, int ldb,
                                 const rocblas_b200_refine_options* opt, rocblas_b200_refine_info* info)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    rocblas_b200_refine_info out{};
    rocblas_status st
        = trsm_arg_check<double>(h, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb, 1);
    if(st != rocblas_status_continue)
    {
        if(st == rocblas_status_success && info)
        {
            out.converged = 1;
            *info         = out;
        }
        return st;
    }
    if(h->pointer_mode != rocblas_pointer_mode_host)
        return rocblas_status_not_implemented;
    const int S      = opt && opt->slices ? opt->slices : tuning().mixed_slices;
    const int moduli = opt && opt->slices ? 0 : tuning().mixed_moduli; // an explicit slice count: slices
    if(S < 1 || S > kOzMaxS || (opt && (opt->check_columns < 0 || opt->tolerance < 0.0)))
        return rocblas_status_invalid_value;
    const bool   left     = side == rocblas_side_left;
    const int    nrhs     = left ? n : m;
    const int    max_it   = opt ? (opt->max_iterations < 0 ? 10 : opt->max_iterations) : 10;
    const int    c        = std::min(nrhs, opt && opt->check_columns > 0 ? opt->check_columns : 8);
    const bool   fallback = opt ? opt->fallback != 0 : true;
    const double tol      = opt && opt->tolerance > 0.0 ? opt->tolerance : 1e-12;
    out.checked_columns   = c;
    out.tolerance         = tol;
    if(*alpha == 0.0)
    {
        if(h->size_query)
            return rocblas_status_size_unchanged;
        if((st = device_ready(h)) != rocblas_status_success)
            return st;
        zero_fill<double>(strided<double>(B, 0), ldb, m, n, 1, h->stream);
        out.converged = 1;
        if(info)
            *info = out;
        return launch_status();
    }
    TrsmProblem<double> pr{};
    pr.side_left = left;
    pr.upper     = uplo == rocblas_fill_upper;
    pr.trans     = trans != rocblas_operation_none;
    pr.unit      = diag == rocblas_diagonal_unit;
    pr.m = m;
    pr.n = n;
    pr.batch = 1;
    pr.A = strided<double>(A, 0);
    pr.lda = lda;
    pr.B = strided<double>(B, 0);
    pr.ldb = ldb;
    pr.stream    = h->stream;
    pr.sm_count  = h->sm_count;
    pr.alpha.val = *alpha;
    // the tested right-hand sides, solved by the plain FP64 form: side left m x c, side right
    // c x n (the same rows of B), ld = their row count.  That solve is a chain of dependent
    // steps whose CTAs hold their SMs while they wait, so it gets a few SMs of its own
    // (refine_check_sms, chain strips of 32) and the sliced solve's persistent kernels size
    // their grids for the others.
    TrsmProblem<double> ps = pr;
    const int           srows = left ? m : c, scols = left ? c : n;
    ps.m   = srows;
    ps.n   = scols;
    ps.ldb = srows;
    const bool ps_chain = use_chain(ps);
    ps.sm_count         = std::max(1, std::min(tuning().refine_check_sms, h->sm_count / 4));
    // the test solve's chain in clusters of two CTAs (refine_check_pairs, an even SM count):
    // it then holds whole SM pairs and the precision-form solve may use the CTA-pair GEMM
    const bool ps_pairs = tuning().refine_check_pairs != 0 && ps.sm_count % 2 == 0
                          && tuning().refine_check_flag == 0 && (h->sm_count - ps.sm_count) % 2 == 0;
    // up to 8 tested right-hand sides: the memory-bound flag-synchronised solve (one pass over
    // A's triangle for all of them), else the chain
    const bool ps_flag = c <= 8 && tuning().refine_check_flag != 0;
    const int  nb_flag = (int)ceil_div(left ? m : n, 128);
    // workspace: the precision form's | B0 (m x n) | R (m x n) | the tested right-hand sides |
    // their chain flags | the test's maxima
    const MixedPlan plan  = mixed_plan(pr, S, moduli);
    const size_t    mn    = (size_t)m * n * sizeof(double);
    const size_t    smp   = (size_t)srows * scols * sizeof(double);
    // the chain's strip width: 16 wastes half as much DMMA work on up to 8 tested columns
    const int       ps_w  = tuning().refine_check_w == 16 && c <= 16 ? 16 : 32;
    const size_t    fl    = ps_flag    ? (size_t)nb_flag * 2 * sizeof(int)
                            : ps_chain ? chain_workspace_bytes(chain_shape(ps.k(), c, 1, ps_w))
                                       : 0;
    const size_t    o_b0  = align256(plan.total), o_r = o_b0 + align256(mn);
    const size_t    o_xs  = o_r + (max_it > 0 ? align256(mn) : 0), o_fl = o_xs + align256(smp);
    const size_t    o_mx  = o_fl + align256(fl);
    const size_t    total = o_mx + align256(sizeof(double) * 2 * (size_t)c);
    if(h->size_query)
        return h->set_optimal_size(total);
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    if(!h->host_res)
        h->host_res = new HostPathRes();
    HostPathRes& res = *h->host_res;
    cudaEvent_t  ev_ready = nullptr, ev_ref = nullptr, ev_copied = nullptr, ev_inv = nullptr;
    if(!res.init() || !(ev_ready = res.event(0)) || !(ev_ref = res.event(1)) || !(ev_copied = res.event(2))
       || !(ev_inv = res.event(3)))
        return rocblas_status_internal_error;
    int*           err = ensure_err(h);
    unsigned char* ws  = reinterpret_cast<unsigned char*>(h->borrow(total));
    if(!ws || !err)
        return rocblas_status_memory_error;
    pr.err_dev = ps.err_dev = err;
    double*      B0 = reinterpret_cast<double*>(ws + o_b0);
    double*      R  = reinterpret_cast<double*>(ws + o_r);
    double*      Xs = reinterpret_cast<double*>(ws + o_xs);
    double*      mx = reinterpret_cast<double*>(ws + o_mx);
    cudaStream_t s  = h->stream;

    // On the side stream, once the caller's earlier work on B is done: B0 := B and the tested
    // right-hand sides gathered, while the main stream builds invA (once, for every solve below).
    TrsmProblem<double> pside = pr;
    pside.stream              = res.tri;
    cudaEventRecord(ev_ready, s);
    cudaStreamWaitEvent(res.tri, ev_ready, 0);
    cudaMemcpy2DAsync(B0, (size_t)m * sizeof(double), B, (size_t)ldb * sizeof(double),
                      (size_t)m * sizeof(double), n, cudaMemcpyDeviceToDevice, res.tri);
    refine_prep(pside, B0, m, srows, scols, 1, nrhs, 1.0, 0, Xs, srows, nullptr);
    cudaEventRecord(ev_copied, res.tri);
    if(plan.recursive)
    {
        BatchPtr<double> inv;
        inv.base   = reinterpret_cast<double*>(ws);
        inv.stride = (int64_t)kInvNB * pr.k();
        build_invA<double>(pr, inv);
        ps.invA = inv;
    }
    // the solve overwrites B: it waits for the copies; the reference solve of the tested
    // right-hand sides waits for invA and then runs beside the precision-form solve
    cudaStreamWaitEvent(s, ev_copied, 0);
    cudaEventRecord(ev_inv, s);
    cudaStreamWaitEvent(res.tri, ev_inv, 0);
    ps.B      = strided<double>(Xs, 0);
    ps.stream = res.tri;
    bool check_in_pairs = false;
    if(ps_flag)
    {
        // side L: op(A) x_v = alpha b_v, x_v a column of Xs (m x c); side R: x_v op(A) = alpha b_v
        // is op(A)^T x_v^T = alpha b_v^T, x_v a row of Xs (c x n)
        TrsvParams<double> tp{};
        const bool tr = left ? pr.trans : !pr.trans;
        tp.A           = A;
        tp.lda         = lda;
        tp.x           = Xs;
        tp.incx        = left ? 1 : srows;
        tp.ldx         = left ? srows : 1;
        tp.nrhs        = c;
        tp.alpha       = *alpha;
        tp.n           = left ? m : n;
        tp.trans       = tr ? 1 : 0;
        tp.rev         = pr.upper != tr ? 1 : 0; // op(A) (side R: its transpose) upper
        tp.unit        = pr.unit ? 1 : 0;
        tp.flags       = reinterpret_cast<int*>(ws + o_fl);
        tp.error       = err;
        tp.wait_cycles = 1ll << tuning().wait_cycles_log2;
        cudaMemsetAsync(tp.flags, 0, (size_t)nb_flag * 2 * sizeof(int), res.tri);
        if(tr)
            launch_trsv_flag_nr<double, 64, 8, 1>(tp, (int)ceil_div(tp.n, 64), ps.sm_count, res.tri);
        else
            launch_trsv_flag_nr<double, 128, 8, 0>(tp, nb_flag, ps.sm_count, res.tri);
        count_launch();
    }
    else if(ps_chain && plan.recursive)
    {
        launch_chain_sub<double>(ps, 0, (int)ceil_div(ps.k(), kInvNB), 1, ps_w, ws + o_fl, ps_pairs);
        check_in_pairs = ps_pairs;
    }
    else
        trsm_run<double>(ps, nullptr, false);
    cudaEventRecord(ev_ref, res.tri);

    TrsmProblem<double> pr1 = pr; // the first solve shares the GPU with the reference solve
    pr1.sm_count            = std::max(1, h->sm_count - ps.sm_count);
    pr1.crt_pair_ok         = check_in_pairs ? 1 : 0; // the test solve holds whole SM pairs
    if(!mixed_run(pr1, S, moduli, plan, ws, err, false))
        return rocblas_status_arch_mismatch;
    cudaStreamWaitEvent(s, ev_ref, 0);

    // the test: max over the tested right-hand sides v of ||x_v - xref_v||_inf / ||xref_v||_inf
    std::vector<double> hmx(2 * (size_t)c);
    auto test = [&](double* err_est) -> rocblas_status {
        refine_compare_kernel<<<(unsigned)c, 256, 0, s>>>(B, ldb, Xs, srows, scols, left, nrhs, mx);
        count_launch();
        if(cudaMemcpyAsync(hmx.data(), mx, hmx.size() * sizeof(double), cudaMemcpyDeviceToHost, s)
               != cudaSuccess
           || cudaStreamSynchronize(s) != cudaSuccess)
        {
            cudaGetLastError();
            return rocblas_status_internal_error;
        }
        double e = 0.0;
        for(int v = 0; v < c; ++v)
        {
            const double d = hmx[2 * (size_t)v], x = hmx[2 * (size_t)v + 1];
            const double ev = d == 0.0 ? 0.0 : d / x; // x == 0 with d != 0: inf
            if(!(ev <= e))                            // NaN propagates
                e = ev;
        }
        *err_est = e;
        return rocblas_status_success;
    };

    double e = 0.0;
    if((st = test(&e)) != rocblas_status_success)
        return st;
    out.error_estimate_first = e;
    TrsmProblem<double> prc = pr; // the correction solve: op(A) D = R
    prc.B         = strided<double>(R, 0);
    prc.ldb       = m;
    prc.alpha.val = 1.0;
    while(!(e <= tol) && out.iterations < max_it)
    {
        // R := alpha B0 - op(A) X in FP64, D := the precision-form solve of op(A) D = R, X += D
        refine_prep(pr, B0, m, m, n, 0, nrhs, *alpha, pr.unit, R, m, nullptr);
        refine_product(pr, B, ldb, R, m, m, n);
        if(!mixed_run(prc, S, moduli, plan, ws, err, false))
            return rocblas_status_arch_mismatch;
        const dim3 grid((unsigned)ceil_div(m, 256), (unsigned)std::min(n, 65535));
        refine_update_kernel<<<grid, 256, 0, s>>>(B, ldb, R, m, m, n);
        count_launch();
        ++out.iterations;
        if((st = test(&e)) != rocblas_status_success)
            return st;
    }
    out.error_estimate = e;
    out.converged      = e <= tol;
    if(!out.converged && fallback)
    {
        // the plain FP64 form from the original right-hand sides
        cudaMemcpy2DAsync(B, (size_t)ldb * sizeof(double), B0, (size_t)m * sizeof(double),
                          (size_t)m * sizeof(double), n, cudaMemcpyDeviceToDevice, s);
        st = trsm_impl<double>(h, side, uplo, trans, diag, m, n, alpha, A, strided<double>(A, 0), lda, B,
                               strided<double>(B, 0), ldb, 1, nullptr, BatchPtr<double>{}, 0);
        if(st != rocblas_status_success && st != rocblas_status_perf_degraded)
            return st;
        out.fell_back = 1;
    }
    if(info)
        *info = out;
    return launch_status();
}


// The precision form with A and B in host memory: the call copies A's triangle and B to the
// device, solves, and copies X back into B, returning when B holds X.  For side left the
// three overlap: the solve runs left-looking over steps of rows, and each step's rows of B and
// block row of op(A) go over in solve order on a copy stream (its 128-blocks inverted on a
// third stream as soon as they land), so a step waits only for its own data; each step's rows
// of X go back as soon as they are final.  Side right copies everything first and then solves.
rocblas_status trsm_mixed_host_impl(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                                    rocblas_operation trans, rocblas_diagonal diag, int m, int n,
                                    const double* alpha, const double* hA, int lda, double* hB,
                                    int ldb, int slices)
{
    DeviceScope device_scope; // the caller's current device is restored on return
    if(!h)
        return rocblas_status_invalid_handle;
    if(h->size_query)
        return rocblas_status_size_unchanged; // the device memory is the call's own
    const rocblas_pointer_mode mode = h->pointer_mode;
    h->pointer_mode                 = rocblas_pointer_mode_host; // alpha is a host value here
    rocblas_status st = trsm_arg_check<double>(h, side, uplo, trans, diag, m, n, alpha, hA, lda, hB, ldb, 1);
    h->pointer_mode = mode;
    if(st != rocblas_status_continue)
        return st;
    const int moduli = slices == 0 ? tuning().mixed_moduli : 0; // 0: the tuned engine
    if(slices == 0)
        slices = tuning().mixed_slices;
    if(slices < 1 || slices > kOzMaxS)
        return rocblas_status_invalid_value;
    if(*alpha == 0.0)
    {
        for(int j = 0; j < n; ++j)
            std::memset(hB + (size_t)j * ldb, 0, sizeof(double) * (size_t)m);
        return rocblas_status_success;
    }
    if((st = device_ready(h)) != rocblas_status_success)
        return st;
    if(!h->host_res)
        h->host_res = new HostPathRes();
    HostPathRes& R = *h->host_res;
    if(!R.init())
        return rocblas_status_internal_error;
    const bool    left = side == rocblas_side_left;
    const int     k    = left ? m : n;
    const size_t  a_bytes = align256((size_t)k * k * sizeof(double));
    const size_t  b_bytes = align256((size_t)m * n * sizeof(double));
    char*         buf     = reinterpret_cast<char*>(R.buffer(a_bytes + b_bytes));
    if(!buf)
        return rocblas_status_memory_error;
    double* dA = reinterpret_cast<double*>(buf);
    double* dB = reinterpret_cast<double*>(buf + a_bytes);
    const size_t es = sizeof(double);

    TrsmProblem<double> pr{};
    pr.side_left = left;
    pr.upper     = uplo == rocblas_fill_upper;
    pr.trans     = trans != rocblas_operation_none;
    pr.unit      = diag == rocblas_diagonal_unit;
    pr.m = m;
    pr.n = n;
    pr.batch = 1;
    pr.A = strided<double>(dA, 0);
    pr.lda = k;
    pr.B = strided<double>(dB, 0);
    pr.ldb = m;
    pr.stream   = h->stream;
    pr.sm_count = h->sm_count;
    pr.alpha.val = *alpha;
    const bool recursive = choose_algo(pr) == Algo::recursive;

    if(!left || !recursive)
    {
        cudaEvent_t eB = R.event(0);
        if(!eB)
            return rocblas_status_internal_error;
        cudaMemcpy2DAsync(dB, (size_t)m * es, hB, (size_t)ldb * es, (size_t)m * es, n, cudaMemcpyHostToDevice, R.in);
        cudaMemcpy2DAsync(dA, (size_t)k * es, hA, (size_t)lda * es, (size_t)k * es, k, cudaMemcpyHostToDevice,
                          R.in);
        cudaEventRecord(eB, R.in);
        cudaStreamWaitEvent(h->stream, eB, 0);
        const rocblas_pointer_mode saved = h->pointer_mode;
        h->pointer_mode                  = rocblas_pointer_mode_host;
        st = trsm_mixed_impl(h, side, uplo, trans, diag, m, n, alpha, dA, k, dB, m, slices);
        h->pointer_mode = saved;
        if(st != rocblas_status_success)
            return st;
        cudaMemcpy2DAsync(hB, (size_t)ldb * es, dB, (size_t)m * es, (size_t)m * es, n, cudaMemcpyDeviceToHost,
                          h->stream);
        cudaStreamSynchronize(h->stream);
        return launch_status();
    }

    // Left-looking over steps of DB = host_step_blocks 128-blocks of rows, in solve order.
    // Every step needs only its own data: its rows of B and its block row of M = op(A) (the
    // diagonal block and the solved side), so the solve starts as soon as the first block row
    // has landed and then follows the transfer. B_q := alpha B_q - M_q X_solved is the one
    // update of those rows (one sliced product of depth = the rows solved so far), so alpha
    // goes to it (to the diagonal solve in the first step, which has no update).
    const int    nblk      = (int)ceil_div(k, kInvNB);
    const int    DB        = std::max(1, tuning().host_step_blocks);
    const int    nstep     = (int)ceil_div(nblk, DB);
    const bool   forward   = pr.oplower();
    const size_t inv_bytes = align256((size_t)kInvNB * k * sizeof(double));
    const size_t sl_bytes  = update_workspace_bytes(std::min(k, DB * kInvNB), n, k, slices, moduli,
                                                    pr.sm_count);
    const size_t ch_bytes  = mixed_chain_workspace_bytes(pr);
    const size_t ws_bytes  = inv_bytes + (sl_bytes + 255) / 256 * 256 + (ch_bytes + 255) / 256 * 256;
    int*         err       = ensure_err(h);
    void*        ws        = h->borrow(ws_bytes);
    if(!ws || !err)
        return rocblas_status_memory_error;
    pr.err_dev = err;
    BatchPtr<double> inv;
    inv.base   = reinterpret_cast<double*>(ws);
    inv.stride = (int64_t)kInvNB * k;
    pr.invA    = inv;

    MixedRecursive rec{{pr, k, nblk}};
    rec.S        = slices;
    rec.moduli   = moduli;
    rec.slice_ws = reinterpret_cast<unsigned char*>(ws) + inv_bytes;
    rec.err_dev  = err;
    if(ch_bytes)
        rec.chain_ws = reinterpret_cast<unsigned char*>(ws) + inv_bytes + (sl_bytes + 255) / 256 * 256;
    for(int q = 0; q < nstep && rec.ok; ++q)
    {
        const int d  = forward ? q : nstep - 1 - q;
        const int b0 = d * DB, b1 = std::min(nblk, b0 + DB);
        const int r0 = rec.row_of(b0), r1 = rec.row_of(b1);
        // the block row of M: columns [0, r1) (forward) or [r0, k) (backward); rows of A for
        // trans N, columns of A for trans T
        const int c0 = forward ? 0 : r0, c1 = forward ? r1 : k;
        cudaEvent_t ea = R.event(3 * (size_t)q), et = R.event(3 * (size_t)q + 1), ex = R.event(3 * (size_t)q + 2);
        if(!ea || !et || !ex)
            return rocblas_status_internal_error;
        cudaMemcpy2DAsync(dB + r0, (size_t)m * es, hB + r0, (size_t)ldb * es, (size_t)(r1 - r0) * es, n,
                          cudaMemcpyHostToDevice, R.in);
        if(!pr.trans)
            cudaMemcpy2DAsync(dA + r0 + (int64_t)c0 * k, (size_t)k * es, hA + r0 + (int64_t)c0 * lda,
                              (size_t)lda * es, (size_t)(r1 - r0) * es, c1 - c0, cudaMemcpyHostToDevice, R.in);
        else
            cudaMemcpy2DAsync(dA + c0 + (int64_t)r0 * k, (size_t)k * es, hA + c0 + (int64_t)r0 * lda,
                              (size_t)lda * es, (size_t)(c1 - c0) * es, r1 - r0, cudaMemcpyHostToDevice, R.in);
        cudaEventRecord(ea, R.in);

        // the step's diagonal 128-blocks, inverted on their own stream while the update runs
        cudaStreamWaitEvent(R.tri, ea, 0);
        TrtriParams<double> t{};
        t.k                = r1 - r0;
        t.nb               = kInvNB;
        t.A                = pr.A.shifted(r0 + (int64_t)r0 * k);
        t.lda              = k;
        t.inv              = inv.shifted((int64_t)b0 * kInvNB * kInvNB);
        t.ldinv            = kInvNB;
        t.inv_block_stride = (int64_t)kInvNB * kInvNB;
        t.upper            = pr.upper;
        t.unit             = pr.unit;
        launch_trtri<double>(t, b1 - b0, 1, R.tri);
        count_launch();
        cudaEventRecord(et, R.tri);

        cudaStreamWaitEvent(h->stream, ea, 0);
        int first = 1;
        if(forward && r0 > 0)
            rec.update_sliced(r0, r1, 0, r0, 1), first = 0;
        else if(!forward && r1 < k)
            rec.update_sliced(r0, r1, r1, k, 1), first = 0;
        cudaStreamWaitEvent(h->stream, et, 0);
        rec.solve_mixed(b0, b1, first);
        // rows [r0, r1) of X are final: send them home on the out stream
        cudaEventRecord(ex, h->stream);
        cudaStreamWaitEvent(R.out, ex, 0);
        cudaMemcpy2DAsync(hB + r0, (size_t)ldb * es, dB + r0, (size_t)m * es, (size_t)(r1 - r0) * es, n,
                          cudaMemcpyDeviceToHost, R.out);
    }
    cudaStreamSynchronize(R.out);
    cudaStreamSynchronize(h->stream);
    if(!rec.ok)
        return rocblas_status_arch_mismatch;
    return launch_status();
}

} // namespace

// =========================================================================================
// exported functions
// =========================================================================================
extern "C" {

uint64_t rocblas_b200_kernel_launch_count(void)
{
    return g_kernel_launches.load(std::memory_order_relaxed);
}

rocblas_status rocblas_create_handle(rocblas_handle* handle)
try
{
    if(!handle)
        return rocblas_status_invalid_pointer;
    auto* h = new _rocblas_handle();
    int   dev = -1;
    if(cudaGetDevice(&dev) == cudaSuccess)
    {
        cudaDeviceProp prop;
        if(cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
        {
            h->device   = dev;
            h->sm_count = prop.multiProcessorCount;
        }
        // the device error word of the bounded waits exists from the start, so no call made
        // under stream capture has to allocate it
        ensure_err(h);
    }
    cudaGetLastError();
    // the layer-logging and check-numerics modes of the handle (handle.cpp:856-877, 921-931)
    if(const char* v = std::getenv("ROCBLAS_LAYER"))
    {
        h->layer_mode = (int)std::strtol(v, nullptr, 0);
        if(h->layer_mode & kLayerTrace)
            h->log_trace_os = layer_log_stream("ROCBLAS_LOG_TRACE_PATH");
        if(h->layer_mode & kLayerBench)
            h->log_bench_os = layer_log_stream("ROCBLAS_LOG_BENCH_PATH");
        if(h->layer_mode & kLayerProfile)
            h->log_profile_os = layer_log_stream("ROCBLAS_LOG_PROFILE_PATH");
    }
    if(const char* v = std::getenv("ROCBLAS_CHECK_NUMERICS"))
        h->check_numerics = (int)std::strtol(v, nullptr, 0);
    *handle = h;
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_destroy_handle(rocblas_handle handle)
try
{
    if(!handle)
        return rocblas_status_invalid_handle;
    handle->free_mem();
    if(handle->err_dev)
        cudaFree(handle->err_dev);
    if(handle->host_res)
    {
        handle->host_res->release();
        delete handle->host_res;
    }
    delete handle;
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_set_stream(rocblas_handle handle, cudaStream_t stream)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    handle->stream = stream;
    return rocblas_status_success;
}

rocblas_status rocblas_get_stream(rocblas_handle handle, cudaStream_t* stream)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!stream)
        return rocblas_status_invalid_pointer;
    *stream = handle->stream;
    return rocblas_status_success;
}

rocblas_status rocblas_set_pointer_mode(rocblas_handle handle, rocblas_pointer_mode mode)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(mode != rocblas_pointer_mode_host && mode != rocblas_pointer_mode_device)
        return rocblas_status_invalid_value;
    handle->pointer_mode = mode;
    return rocblas_status_success;
}

rocblas_status rocblas_get_pointer_mode(rocblas_handle handle, rocblas_pointer_mode* mode)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!mode)
        return rocblas_status_invalid_pointer;
    *mode = handle->pointer_mode;
    return rocblas_status_success;
}

rocblas_status rocblas_set_math_mode(rocblas_handle handle, rocblas_math_mode mode)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    // only the default math mode exists here (rocblas_auxiliary.cpp:145-178: an unsupported mode
    // is logged and ignored, and the call succeeds)
    const bool supported = mode == rocblas_default_math;
    if(handle->layer_mode & kLayerTrace)
        layer_log_line(handle->log_trace_os, "rocblas_set_math_mode," + std::to_string((int)mode)
                                                 + (supported ? "," : ",is not supported,")
                                                 + atomics_mode_string(handle->atomics_mode));
    if(supported)
        handle->math_mode = mode;
    return rocblas_status_success;
}

rocblas_status rocblas_get_math_mode(rocblas_handle handle, rocblas_math_mode* mode)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!mode)
        return rocblas_status_invalid_pointer;
    *mode = (rocblas_math_mode)handle->math_mode;
    if(handle->layer_mode & kLayerTrace)
        layer_log_line(handle->log_trace_os, "rocblas_get_math_mode," + std::to_string((int)*mode) + ","
                                                 + atomics_mode_string(handle->atomics_mode));
    return rocblas_status_success;
}

rocblas_status rocblas_set_performance_metric(rocblas_handle handle, rocblas_performance_metric metric)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    handle->performance_metric = metric;
    return rocblas_status_success;
}

rocblas_status rocblas_get_performance_metric(rocblas_handle handle, rocblas_performance_metric* metric)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!metric)
        return rocblas_status_invalid_pointer;
    *metric = (rocblas_performance_metric)handle->performance_metric;
    return rocblas_status_success;
}

rocblas_status rocblas_set_solution_fitness_query(rocblas_handle handle, double* fitness)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    handle->fitness_query = fitness;
    if(fitness)
        *fitness = std::numeric_limits<double>::lowest();
    return rocblas_status_success;
}

rocblas_status rocblas_set_atomics_mode(rocblas_handle handle, rocblas_atomics_mode mode)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(handle->layer_mode & kLayerTrace)
        layer_log_line(handle->log_trace_os, std::string("rocblas_set_atomics_mode,")
                                                 + atomics_mode_string(mode) + ","
                                                 + atomics_mode_string(handle->atomics_mode));
    handle->atomics_mode = mode;
    return rocblas_status_success;
}

rocblas_status rocblas_get_atomics_mode(rocblas_handle handle, rocblas_atomics_mode* mode)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!mode)
        return rocblas_status_invalid_pointer;
    *mode = (rocblas_atomics_mode)handle->atomics_mode;
    if(handle->layer_mode & kLayerTrace)
        layer_log_line(handle->log_trace_os, std::string("rocblas_get_atomics_mode,")
                                                 + atomics_mode_string(*mode) + ","
                                                 + atomics_mode_string(handle->atomics_mode));
    return rocblas_status_success;
}

rocblas_status rocblas_set_vector(rocblas_int n, rocblas_int elem_size, const void* x_h, rocblas_int incx, void* y_d,
                                  rocblas_int incy)
try
{
    return aux_copy_vector(n, elem_size, x_h, incx, y_d, incy, cudaMemcpyHostToDevice, nullptr, false);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_get_vector(rocblas_int n, rocblas_int elem_size, const void* x_d, rocblas_int incx, void* y_h,
                                  rocblas_int incy)
try
{
    return aux_copy_vector(n, elem_size, x_d, incx, y_h, incy, cudaMemcpyDeviceToHost, nullptr, false);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_set_vector_async(rocblas_int n, rocblas_int elem_size, const void* x_h, rocblas_int incx,
                                        void* y_d, rocblas_int incy, cudaStream_t stream)
try
{
    return aux_copy_vector(n, elem_size, x_h, incx, y_d, incy, cudaMemcpyHostToDevice, stream, true);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_get_vector_async(rocblas_int n, rocblas_int elem_size, const void* x_d, rocblas_int incx,
                                        void* y_h, rocblas_int incy, cudaStream_t stream)
try
{
    return aux_copy_vector(n, elem_size, x_d, incx, y_h, incy, cudaMemcpyDeviceToHost, stream, true);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_set_matrix(rocblas_int rows, rocblas_int cols, rocblas_int elem_size, const void* a_h, rocblas_int lda,
                                  void* b_d, rocblas_int ldb)
try
{
    return aux_copy_matrix(rows, cols, elem_size, a_h, lda, b_d, ldb, cudaMemcpyHostToDevice, nullptr, false);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_get_matrix(rocblas_int rows, rocblas_int cols, rocblas_int elem_size, const void* a_d, rocblas_int lda,
                                  void* b_h, rocblas_int ldb)
try
{
    return aux_copy_matrix(rows, cols, elem_size, a_d, lda, b_h, ldb, cudaMemcpyDeviceToHost, nullptr, false);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_set_matrix_async(rocblas_int rows, rocblas_int cols, rocblas_int elem_size, const void* a_h,
                                        rocblas_int lda, void* b_d, rocblas_int ldb, cudaStream_t stream)
try
{
    return aux_copy_matrix(rows, cols, elem_size, a_h, lda, b_d, ldb, cudaMemcpyHostToDevice, stream, true);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_get_matrix_async(rocblas_int rows, rocblas_int cols, rocblas_int elem_size, const void* a_d,
                                        rocblas_int lda, void* b_h, rocblas_int ldb, cudaStream_t stream)
try
{
    return aux_copy_matrix(rows, cols, elem_size, a_d, lda, b_h, ldb, cudaMemcpyDeviceToHost, stream, true);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_set_vector_64(int64_t n, int64_t elem_size, const void* x_h, int64_t incx, void* y_d,
                                  int64_t incy)
try
{
    return aux_copy_vector(n, elem_size, x_h, incx, y_d, incy, cudaMemcpyHostToDevice, nullptr, false);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_get_vector_64(int64_t n, int64_t elem_size, const void* x_d, int64_t incx, void* y_h,
                                  int64_t incy)
try
{
    return aux_copy_vector(n, elem_size, x_d, incx, y_h, incy, cudaMemcpyDeviceToHost, nullptr, false);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_set_vector_async_64(int64_t n, int64_t elem_size, const void* x_h, int64_t incx,
                                        void* y_d, int64_t incy, cudaStream_t stream)
try
{
    return aux_copy_vector(n, elem_size, x_h, incx, y_d, incy, cudaMemcpyHostToDevice, stream, true);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_get_vector_async_64(int64_t n, int64_t elem_size, const void* x_d, int64_t incx,
                                        void* y_h, int64_t incy, cudaStream_t stream)
try
{
    return aux_copy_vector(n, elem_size, x_d, incx, y_h, incy, cudaMemcpyDeviceToHost, stream, true);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_set_matrix_64(int64_t rows, int64_t cols, int64_t elem_size, const void* a_h, int64_t lda,
                                  void* b_d, int64_t ldb)
try
{
    return aux_copy_matrix(rows, cols, elem_size, a_h, lda, b_d, ldb, cudaMemcpyHostToDevice, nullptr, false);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_get_matrix_64(int64_t rows, int64_t cols, int64_t elem_size, const void* a_d, int64_t lda,
                                  void* b_h, int64_t ldb)
try
{
    return aux_copy_matrix(rows, cols, elem_size, a_d, lda, b_h, ldb, cudaMemcpyDeviceToHost, nullptr, false);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_set_matrix_async_64(int64_t rows, int64_t cols, int64_t elem_size, const void* a_h,
                                        int64_t lda, void* b_d, int64_t ldb, cudaStream_t stream)
try
{
    return aux_copy_matrix(rows, cols, elem_size, a_h, lda, b_d, ldb, cudaMemcpyHostToDevice, stream, true);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_get_matrix_async_64(int64_t rows, int64_t cols, int64_t elem_size, const void* a_d,
                                        int64_t lda, void* b_h, int64_t ldb, cudaStream_t stream)
try
{
    return aux_copy_matrix(rows, cols, elem_size, a_d, lda, b_h, ldb, cudaMemcpyDeviceToHost, stream, true);
}
catch(...)
{
    return exception_status();
}

rocblas_pointer_mode rocblas_pointer_to_mode(void* ptr)
{
    cudaPointerAttributes attr;
    if(cudaPointerGetAttributes(&attr, ptr) == cudaSuccess && attr.type == cudaMemoryTypeDevice)
        return rocblas_pointer_mode_device;
    cudaGetLastError();
    return rocblas_pointer_mode_host;
}

rocblas_status rocblas_start_device_memory_size_query(rocblas_handle handle)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(handle->size_query)
        return rocblas_status_size_query_mismatch;
    handle->size_query = true;
    handle->query_size = 0;
    return rocblas_status_success;
}

rocblas_status rocblas_stop_device_memory_size_query(rocblas_handle handle, size_t* size)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!handle->size_query)
        return rocblas_status_size_query_mismatch;
    if(!size)
        return rocblas_status_invalid_pointer;
    *size              = handle->query_size;
    handle->size_query = false;
    return rocblas_status_success;
}

bool rocblas_is_device_memory_size_query(rocblas_handle handle)
{
    return handle && handle->size_query;
}

rocblas_status rocblas_get_device_memory_size(rocblas_handle handle, size_t* size)
{
    if(!handle)
        return rocblas_status_invalid_handle;
    if(!size)
        return rocblas_status_invalid_pointer;
    *size = handle->mem_size;
    return rocblas_status_success;
}

rocblas_status rocblas_set_device_memory_size(rocblas_handle handle, size_t size)
try
{
    if(!handle)
        return rocblas_status_invalid_handle;
    handle->free_mem();
    if(!size)
        return rocblas_status_success;
    if(handle->device < 0)
        return rocblas_status_memory_error;
    size = _rocblas_handle::roundup(size);
    if(cudaMalloc(&handle->mem, size) != cudaSuccess)
    {
        cudaGetLastError();
        handle->mem = nullptr;
        return rocblas_status_memory_error;
    }
    handle->mem_size = size;
    handle->owner    = MemOwner::user_managed;
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_set_workspace(rocblas_handle handle, void* addr, size_t size)
try
{
    if(!handle)
        return rocblas_status_invalid_handle;
    handle->free_mem();
    if(size && addr)
    {
        handle->owner    = MemOwner::user_owned;
        handle->mem      = addr;
        handle->mem_size = size;
    }
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

bool rocblas_is_managing_device_memory(rocblas_handle handle)
{
    return handle && handle->owner == MemOwner::managed;
}

bool rocblas_is_user_managing_device_memory(rocblas_handle handle)
{
    return handle && handle->owner == MemOwner::user_managed;
}

// ---- trsm ------------------------------------------------------------------------------------
#define TRSM_PLAIN(NAME, TA, T, I)                                                                \
    rocblas_status NAME(rocblas_handle h, rocblas_side side, rocblas_fill uplo,                  \
                        rocblas_operation trans, rocblas_diagonal diag, I m, I n,                \
                        const TA* alpha, const TA* A, I lda, TA* B, I ldb)                        \
    try                                                                                          \
    {                                                                                            \
        const TrsmLogInfo li{0, sizeof(I) == 8, 0, 0};                                           \
        return trsm_impl_64<T>(h, side, uplo, trans, diag, m, n, as_impl<T>(alpha), A,           \
                               strided<T>(as_impl<T>(A), 0), lda, B,                             \
                               strided<T>(as_impl<T>(B), 0), ldb, 1, nullptr, BatchPtr<T>{}, 0,  \
                               &li);                                                             \
    }                                                                                            \
    catch(...)                                                                                   \
    {                                                                                            \
        return exception_status();                                                               \
    }

#define TRSM_BATCHED(NAME, TA, T, I)                                                              \
    rocblas_status NAME(rocblas_handle h, rocblas_side side, rocblas_fill uplo,                  \
                        rocblas_operation trans, rocblas_diagonal diag, I m, I n,                \
                        const TA* alpha, const TA* const A[], I lda, TA* const B[], I ldb,       \
                        I batch_count)                                                           \
    try                                                                                          \
    {                                                                                            \
        const TrsmLogInfo li{1, sizeof(I) == 8, 0, 0};                                           \
        return trsm_impl_64<T>(h, side, uplo, trans, diag, m, n, as_impl<T>(alpha), A,           \
                               arrayed<T>(A), lda, B, arrayed<T>(B), ldb, batch_count, nullptr,  \
                               BatchPtr<T>{}, 0, &li);                                           \
    }                                                                                            \
    catch(...)                                                                                   \
    {                                                                                            \
        return exception_status();                                                               \
    }

#define TRSM_STRIDED(NAME, TA, T, I)                                                              \
    rocblas_status NAME(rocblas_handle h, rocblas_side side, rocblas_fill uplo,                  \
                        rocblas_operation trans, rocblas_diagonal diag, I m, I n,                \
                        const TA* alpha, const TA* A, I lda, rocblas_stride stride_a, TA* B,     \
                        I ldb, rocblas_stride stride_b, I batch_count)                           \
    try                                                                                          \
    {                                                                                            \
        const TrsmLogInfo li{2, sizeof(I) == 8, stride_a, stride_b};                             \
        return trsm_impl_64<T>(h, side, uplo, trans, diag, m, n, as_impl<T>(alpha), A,           \
                               strided<T>(as_impl<T>(A), stride_a), lda, B,                      \
                               strided<T>(as_impl<T>(B), stride_b), ldb, batch_count, nullptr,   \
                               BatchPtr<T>{}, 0, &li);                                           \
    }                                                                                            \
    catch(...)                                                                                   \
    {                                                                                            \
        return exception_status();                                                               \
    }

#define TRSM_ALL(S, TA, T)                                                 \
    TRSM_PLAIN(rocblas_##S##trsm, TA, T, rocblas_int)                      \
    TRSM_PLAIN(rocblas_##S##trsm_64, TA, T, int64_t)                       \
    TRSM_BATCHED(rocblas_##S##trsm_batched, TA, T, rocblas_int)            \
    TRSM_BATCHED(rocblas_##S##trsm_batched_64, TA, T, int64_t)             \
    TRSM_STRIDED(rocblas_##S##trsm_strided_batched, TA, T, rocblas_int)    \
    TRSM_STRIDED(rocblas_##S##trsm_strided_batched_64, TA, T, int64_t)

TRSM_ALL(s, float, float)
TRSM_ALL(d, double, double)
TRSM_ALL(c, rocblas_float_complex, cplx<float>)
TRSM_ALL(z, rocblas_double_complex, cplx<double>)

// rocblas_trsm_ex type switch (library/src/blas3/rocblas_trsm.cpp:28-73)
rocblas_status rocblas_trsm_ex(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                               rocblas_operation trans, rocblas_diagonal diag, rocblas_int m,
                               rocblas_int n, const void* alpha, const void* A, rocblas_int lda,
                               void* B, rocblas_int ldb, const void* invA, rocblas_int invA_size,
                               rocblas_datatype compute_type)
try
{
    const TrsmLogInfo li{0, false, 0, 0};
    switch(compute_type)
    {
    case rocblas_datatype_f32_r:
        return trsm_impl_64<float>(h, side, uplo, trans, diag, m, n, (const float*)alpha, A,
                                strided<float>((const float*)A, 0), lda, B,
                                strided<float>((float*)B, 0), ldb, 1, invA,
                                strided<float>((const float*)invA, 0), invA_size, &li);
    case rocblas_datatype_f64_r:
        return trsm_impl_64<double>(h, side, uplo, trans, diag, m, n, (const double*)alpha, A,
                                 strided<double>((const double*)A, 0), lda, B,
                                 strided<double>((double*)B, 0), ldb, 1, invA,
                                 strided<double>((const double*)invA, 0), invA_size, &li);
    case rocblas_datatype_f32_c:
        return trsm_impl_64<cplx<float>>(h, side, uplo, trans, diag, m, n,
                                         (const cplx<float>*)alpha, A,
                                         strided<cplx<float>>((const cplx<float>*)A, 0), lda, B,
                                         strided<cplx<float>>((cplx<float>*)B, 0), ldb, 1, invA,
                                         strided<cplx<float>>((const cplx<float>*)invA, 0),
                                         invA_size, &li);
    case rocblas_datatype_f64_c:
        return trsm_impl_64<cplx<double>>(h, side, uplo, trans, diag, m, n,
                                          (const cplx<double>*)alpha, A,
                                          strided<cplx<double>>((const cplx<double>*)A, 0), lda, B,
                                          strided<cplx<double>>((cplx<double>*)B, 0), ldb, 1, invA,
                                          strided<cplx<double>>((const cplx<double>*)invA, 0),
                                          invA_size, &li);
    default:
        return rocblas_status_not_implemented;
    }
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_trsm_batched_ex(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                                       rocblas_operation trans, rocblas_diagonal diag,
                                       rocblas_int m, rocblas_int n, const void* alpha,
                                       const void* A, rocblas_int lda, void* B, rocblas_int ldb,
                                       rocblas_int batch_count, const void* invA,
                                       rocblas_int invA_size, rocblas_datatype compute_type)
try
{
    const TrsmLogInfo li{1, false, 0, 0};
    switch(compute_type)
    {
    case rocblas_datatype_f32_r:
        return trsm_impl_64<float>(h, side, uplo, trans, diag, m, n, (const float*)alpha, A,
                                arrayed<float>(A), lda, B, arrayed<float>(B), ldb, batch_count,
                                invA, arrayed<float>(invA), invA_size, &li);
    case rocblas_datatype_f64_r:
        return trsm_impl_64<double>(h, side, uplo, trans, diag, m, n, (const double*)alpha, A,
                                 arrayed<double>(A), lda, B, arrayed<double>(B), ldb, batch_count,
                                 invA, arrayed<double>(invA), invA_size, &li);
    case rocblas_datatype_f32_c:
        return trsm_impl_64<cplx<float>>(h, side, uplo, trans, diag, m, n,
                                         (const cplx<float>*)alpha, A, arrayed<cplx<float>>(A), lda,
                                         B, arrayed<cplx<float>>(B), ldb, batch_count, invA,
                                         arrayed<cplx<float>>(invA), invA_size, &li);
    case rocblas_datatype_f64_c:
        return trsm_impl_64<cplx<double>>(h, side, uplo, trans, diag, m, n,
                                          (const cplx<double>*)alpha, A, arrayed<cplx<double>>(A),
                                          lda, B, arrayed<cplx<double>>(B), ldb, batch_count, invA,
                                          arrayed<cplx<double>>(invA), invA_size, &li);
    default:
        return rocblas_status_not_implemented;
    }
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_trsm_strided_batched_ex(rocblas_handle h, rocblas_side side,
                                               rocblas_fill uplo, rocblas_operation trans,
                                               rocblas_diagonal diag, rocblas_int m,
                                               rocblas_int n, const void* alpha, const void* A,
                                               rocblas_int lda, rocblas_stride stride_A, void* B,
                                               rocblas_int ldb, rocblas_stride stride_B,
                                               rocblas_int batch_count, const void* invA,
                                               rocblas_int invA_size, rocblas_stride stride_invA,
                                               rocblas_datatype compute_type)
try
{
    const TrsmLogInfo li{2, false, stride_A, stride_B};
    switch(compute_type)
    {
    case rocblas_datatype_f32_r:
        return trsm_impl_64<float>(h, side, uplo, trans, diag, m, n, (const float*)alpha, A,
                                strided<float>((const float*)A, stride_A), lda, B,
                                strided<float>((float*)B, stride_B), ldb, batch_count, invA,
                                strided<float>((const float*)invA, stride_invA), invA_size, &li);
    case rocblas_datatype_f64_r:
        return trsm_impl_64<double>(h, side, uplo, trans, diag, m, n, (const double*)alpha, A,
                                 strided<double>((const double*)A, stride_A), lda, B,
                                 strided<double>((double*)B, stride_B), ldb, batch_count, invA,
                                 strided<double>((const double*)invA, stride_invA), invA_size, &li);
    case rocblas_datatype_f32_c:
        return trsm_impl_64<cplx<float>>(
            h, side, uplo, trans, diag, m, n, (const cplx<float>*)alpha, A,
            strided<cplx<float>>((const cplx<float>*)A, stride_A), lda, B,
            strided<cplx<float>>((cplx<float>*)B, stride_B), ldb, batch_count, invA,
            strided<cplx<float>>((const cplx<float>*)invA, stride_invA), invA_size, &li);
    case rocblas_datatype_f64_c:
        return trsm_impl_64<cplx<double>>(
            h, side, uplo, trans, diag, m, n, (const cplx<double>*)alpha, A,
            strided<cplx<double>>((const cplx<double>*)A, stride_A), lda, B,
            strided<cplx<double>>((cplx<double>*)B, stride_B), ldb, batch_count, invA,
            strided<cplx<double>>((const cplx<double>*)invA, stride_invA), invA_size, &li);
    default:
        return rocblas_status_not_implemented;
    }
}
catch(...)
{
    return exception_status();
}

// ---- variable-size batched (rocblas_b200_ext.h) --------------------------------------------
rocblas_status rocblas_b200_dtrsm_vbatched(rocblas_handle h, const double* alpha,
                                           const rocblas_b200_trsm_problem* problems,
                                           rocblas_int count, rocblas_int max_k,
                                           rocblas_int* invalid_count)
try
{
    return trsm_vbatched_impl<double>(h, alpha, problems, count, max_k, invalid_count);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_dtrsm_vbatched_noalloc(rocblas_handle h, const double* alpha,
                                                   const rocblas_b200_trsm_problem* problems,
                                                   rocblas_int count, rocblas_int max_k,
                                                   rocblas_int* invalid_count)
try
{
    return trsm_vbatched_noalloc_impl(h, alpha, problems, count, max_k, invalid_count);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_strsm_vbatched(rocblas_handle h, const float* alpha,
                                           const rocblas_b200_trsm_problem* problems,
                                           rocblas_int count, rocblas_int max_k,
                                           rocblas_int* invalid_count)
try
{
    return trsm_vbatched_impl<float>(h, alpha, problems, count, max_k, invalid_count);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_dtrsm_vbatched_ex(rocblas_handle h, const double* alpha,
                                              const rocblas_b200_trsm_problem* problems,
                                              const double* const* invA, rocblas_int count,
                                              rocblas_int max_k, rocblas_int max_n,
                                              rocblas_int* invalid_count)
try
{
    return trsm_vbatched_ex_impl<double>(h, alpha, problems, invA, count, max_k, max_n, invalid_count);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_strsm_vbatched_ex(rocblas_handle h, const float* alpha,
                                              const rocblas_b200_trsm_problem* problems,
                                              const float* const* invA, rocblas_int count,
                                              rocblas_int max_k, rocblas_int max_n,
                                              rocblas_int* invalid_count)
try
{
    return trsm_vbatched_ex_impl<float>(h, alpha, problems, invA, count, max_k, max_n, invalid_count);
}
catch(...)
{
    return exception_status();
}

// ---- trsv (rocblas-functions.h:9900-9908, 10041-10050, 10198-10209) ------------------------
#define TRSV_ALL(TA, T, S, I, SUF)                                                                 \
    rocblas_status rocblas_##S##trsv##SUF(rocblas_handle h, rocblas_fill uplo,                      \
                                          rocblas_operation transA, rocblas_diagonal diag, I n,     \
                                          const TA* A, I lda, TA* x, I incx)                        \
    try                                                                                             \
    {                                                                                               \
        return trsv_impl_64<T>(h, uplo, transA, diag, n, A, strided<T>(as_impl<T>(A), 0), lda, x,  \
                               strided<T>(as_impl<T>(x), 0), incx, 1);                              \
    }                                                                                               \
    catch(...)                                                                                      \
    {                                                                                               \
        return exception_status();                                                                  \
    }                                                                                               \
    rocblas_status rocblas_##S##trsv_batched##SUF(rocblas_handle h, rocblas_fill uplo,              \
                                                  rocblas_operation transA, rocblas_diagonal diag,  \
                                                  I n, const TA* const A[], I lda, TA* const x[],   \
                                                  I incx, I batch_count)                            \
    try                                                                                             \
    {                                                                                               \
        return trsv_impl_64<T>(h, uplo, transA, diag, n, A, arrayed<T>(A), lda, x, arrayed<T>(x),   \
                               incx, batch_count);                                                  \
    }                                                                                               \
    catch(...)                                                                                      \
    {                                                                                               \
        return exception_status();                                                                  \
    }                                                                                               \
    rocblas_status rocblas_##S##trsv_strided_batched##SUF(                                          \
        rocblas_handle h, rocblas_fill uplo, rocblas_operation transA, rocblas_diagonal diag, I n,  \
        const TA* A, I lda, rocblas_stride stride_A, TA* x, I incx, rocblas_stride stride_x,        \
        I batch_count)                                                                              \
    try                                                                                             \
    {                                                                                               \
        return trsv_impl_64<T>(h, uplo, transA, diag, n, A, strided<T>(as_impl<T>(A), stride_A),    \
                               lda, x, strided<T>(as_impl<T>(x), stride_x), incx, batch_count);     \
    }                                                                                               \
    catch(...)                                                                                      \
    {                                                                                               \
        return exception_status();                                                                  \
    }
TRSV_ALL(float, float, s, rocblas_int, )
TRSV_ALL(double, double, d, rocblas_int, )
TRSV_ALL(rocblas_float_complex, cplx<float>, c, rocblas_int, )
TRSV_ALL(rocblas_double_complex, cplx<double>, z, rocblas_int, )
TRSV_ALL(float, float, s, int64_t, _64)
TRSV_ALL(double, double, d, int64_t, _64)
TRSV_ALL(rocblas_float_complex, cplx<float>, c, int64_t, _64)
TRSV_ALL(rocblas_double_complex, cplx<double>, z, int64_t, _64)

// ---- trmm (rocblas-functions.h:18300-18393, 18630-18644, 18904-18921) -----------------------
#define TRMM_ALL(TA, T, S, I, SUF)                                                                  \
    rocblas_status rocblas_##S##trmm##SUF(rocblas_handle h, rocblas_side side, rocblas_fill uplo,   \
                                          rocblas_operation transA, rocblas_diagonal diag, I m,     \
                                          I n, const TA* alpha, const TA* A, I lda, const TA* B,    \
                                          I ldb, TA* C, I ldc)                                      \
    try                                                                                             \
    {                                                                                               \
        return trmm_impl_64<T>(h, side, uplo, transA, diag, m, n, as_impl<T>(alpha), A,             \
                               strided<T>(as_impl<T>(A), 0), lda, B, strided<T>(as_impl<T>(B), 0),  \
                               ldb, C, strided<T>(as_impl<T>(C), 0), ldc, 1);                       \
    }                                                                                               \
    catch(...)                                                                                      \
    {                                                                                               \
        return exception_status();                                                                  \
    }                                                                                               \
    rocblas_status rocblas_##S##trmm_batched##SUF(                                                  \
        rocblas_handle h, rocblas_side side, rocblas_fill uplo, rocblas_operation transA,           \
        rocblas_diagonal diag, I m, I n, const TA* alpha, const TA* const A[], I lda,               \
        const TA* const B[], I ldb, TA* const C[], I ldc, I batch_count)                            \
    try                                                                                             \
    {                                                                                               \
        return trmm_impl_64<T>(h, side, uplo, transA, diag, m, n, as_impl<T>(alpha), A,             \
                               arrayed<T>(A), lda, B, arrayed<T>(B), ldb, C, arrayed<T>(C), ldc,    \
                               batch_count);                                                        \
    }                                                                                               \
    catch(...)                                                                                      \
    {                                                                                               \
        return exception_status();                                                                  \
    }                                                                                               \
    rocblas_status rocblas_##S##trmm_strided_batched##SUF(                                          \
        rocblas_handle h, rocblas_side side, rocblas_fill uplo, rocblas_operation transA,           \
        rocblas_diagonal diag, I m, I n, const TA* alpha, const TA* A, I lda,                       \
        rocblas_stride stride_A, const TA* B, I ldb, rocblas_stride stride_B, TA* C, I ldc,         \
        rocblas_stride stride_C, I batch_count)                                                     \
    try                                                                                             \
    {                                                                                               \
        return trmm_impl_64<T>(h, side, uplo, transA, diag, m, n, as_impl<T>(alpha), A,             \
                               strided<T>(as_impl<T>(A), stride_A), lda, B,                         \
                               strided<T>(as_impl<T>(B), stride_B), ldb, C,                         \
                               strided<T>(as_impl<T>(C), stride_C), ldc, batch_count);              \
    }                                                                                               \
    catch(...)                                                                                      \
    {                                                                                               \
        return exception_status();                                                                  \
    }
TRMM_ALL(float, float, s, rocblas_int, )
TRMM_ALL(double, double, d, rocblas_int, )
TRMM_ALL(rocblas_float_complex, cplx<float>, c, rocblas_int, )
TRMM_ALL(rocblas_double_complex, cplx<double>, z, rocblas_int, )
TRMM_ALL(float, float, s, int64_t, _64)
TRMM_ALL(double, double, d, int64_t, _64)
TRMM_ALL(rocblas_float_complex, cplx<float>, c, int64_t, _64)
TRMM_ALL(rocblas_double_complex, cplx<double>, z, int64_t, _64)

// ---- server (rocblas_b200_ext.h) --------------------------------------------------------------
struct rocblas_b200_server_
{
    TrsmServerCore core{server_solve};
};

rocblas_status rocblas_b200_server_create(rocblas_b200_server* server, size_t hbm_budget,
                                          rocblas_int n_streams, double window_us,
                                          rocblas_int max_batch)
try
{
    if(!server)
        return rocblas_status_invalid_pointer;
    *server = nullptr;
    int dev = 0, sms = 148;
    if(cudaGetDevice(&dev) != cudaSuccess)
    {
        cudaGetLastError();
        return rocblas_status_internal_error;
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto*          s  = new rocblas_b200_server_();
    rocblas_status st = s->core.create(hbm_budget, n_streams, window_us, max_batch, dev, sms);
    if(st != rocblas_status_success)
    {
        delete s;
        return st;
    }
    *server = s;
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_server_destroy(rocblas_b200_server server)
try
{
    if(!server)
        return rocblas_status_invalid_handle;
    delete server;
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_server_add_resident(rocblas_b200_server server, rocblas_datatype dtype,
                                                rocblas_int m, const void* A, rocblas_int lda,
                                                rocblas_int* index)
try
{
    if(!server)
        return rocblas_status_invalid_handle;
    return server->core.add_resident((int)dtype, m, A, lda, index);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_server_set_budget(rocblas_b200_server server, size_t hbm_budget)
try
{
    if(!server)
        return rocblas_status_invalid_handle;
    server->core.set_budget(hbm_budget);
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_server_used_bytes(rocblas_b200_server server, size_t* bytes)
try
{
    if(!server)
        return rocblas_status_invalid_handle;
    if(!bytes)
        return rocblas_status_invalid_pointer;
    *bytes = server->core.used();
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_server_run(rocblas_b200_server server, const rocblas_b200_request* requests,
                                       rocblas_int count, double* latency_s,
                                       rocblas_b200_server_stats* stats)
try
{
    if(!server)
        return rocblas_status_invalid_handle;
    return server->core.run(reinterpret_cast<const ServerRequestC*>(requests), count, latency_s,
                            reinterpret_cast<ServerStatsC*>(stats));
}
catch(...)
{
    return exception_status();
}

// ---- kernel timing (rocblas_b200_ext.h) ------------------------------------------------------
rocblas_status rocblas_b200_kernel_timing_enable(rocblas_int enable)
try
{
    KernelTiming&               t = kernel_timing();
    std::lock_guard<std::mutex> lock(t.mu);
    for(auto& r : t.recs)
        cudaEventSynchronize(r.e1);
    t.recycle();
    t.on = enable != 0;
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_kernel_timing_query(const char* kernel_class, double* total_ms,
                                                double* total_work, rocblas_int* launches)
try
{
    const int cls = kernel_class_of(kernel_class);
    if(cls < 0)
        return rocblas_status_invalid_value;
    if(!total_ms || !total_work || !launches)
        return rocblas_status_invalid_pointer;
    KernelTiming&               t = kernel_timing();
    std::lock_guard<std::mutex> lock(t.mu);
    double ms = 0.0, work = 0.0;
    int    n  = 0;
    for(auto& r : t.recs)
    {
        if(r.cls != cls)
            continue;
        float e = 0.0f;
        if(cudaEventSynchronize(r.e1) != cudaSuccess || cudaEventElapsedTime(&e, r.e0, r.e1) != cudaSuccess)
            return rocblas_status_internal_error;
        ms += e;
        work += r.work;
        ++n;
    }
    *total_ms   = ms;
    *total_work = work;
    *launches   = n;
    return rocblas_status_success;
}
catch(...)
{
    return exception_status();
}

// ---- sliced GEMM / precision form (rocblas_b200_ext.h) -----------------------------------------
rocblas_status rocblas_b200_dgemm_sliced(rocblas_handle h, rocblas_operation transA,
                                         rocblas_operation transB, rocblas_int m, rocblas_int n,
                                         rocblas_int k, const double* alpha, const double* A,
                                         rocblas_int lda, const double* B, rocblas_int ldb,
                                         const double* beta, double* C, rocblas_int ldc,
                                         rocblas_int slices)
try
{
    return gemm_sliced_impl(h, transA, transB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, slices);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_dgemm_crt(rocblas_handle h, rocblas_operation transA,
                                      rocblas_operation transB, rocblas_int m, rocblas_int n,
                                      rocblas_int k, const double* alpha, const double* A,
                                      rocblas_int lda, const double* B, rocblas_int ldb,
                                      const double* beta, double* C, rocblas_int ldc,
                                      rocblas_int moduli)
try
{
    if(!moduli)
        moduli = kCrtMaxModuli;
    return gemm_sliced_impl(h, transA, transB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 1,
                            moduli);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_dgemm(rocblas_handle h, rocblas_operation transA,
                                  rocblas_operation transB, rocblas_int m, rocblas_int n,
                                  rocblas_int k, const double* alpha, const double* A,
                                  rocblas_int lda, const double* B, rocblas_int ldb,
                                  const double* beta, double* C, rocblas_int ldc)
try
{
    return gemm_tiles_impl<double>(h, transA, transB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}
catch(...)
{
    return exception_status();
}

#define GEMM_CPLX(NAME, TA, T)                                                                    \
    rocblas_status NAME(rocblas_handle h, rocblas_operation transA, rocblas_operation transB,     \
                        rocblas_int m, rocblas_int n, rocblas_int k, const TA* alpha, const TA* A, \
                        rocblas_int lda, const TA* B, rocblas_int ldb, const TA* beta, TA* C,     \
                        rocblas_int ldc)                                                          \
    try                                                                                           \
    {                                                                                             \
        return gemm_tiles_impl<T>(h, transA, transB, m, n, k, as_impl<T>(alpha), as_impl<T>(A),   \
                                  lda, as_impl<T>(B), ldb, as_impl<T>(beta), as_impl<T>(C), ldc); \
    }                                                                                             \
    catch(...)                                                                                    \
    {                                                                                             \
        return exception_status();                                                                \
    }
GEMM_CPLX(rocblas_b200_zgemm, rocblas_double_complex, cplx<double>)
GEMM_CPLX(rocblas_b200_cgemm, rocblas_float_complex, cplx<float>)

rocblas_status rocblas_b200_dtrsm_mixed(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                                        rocblas_operation transA, rocblas_diagonal diag,
                                        rocblas_int m, rocblas_int n, const double* alpha,
                                        const double* A, rocblas_int lda, double* B,
                                        rocblas_int ldb, rocblas_int slices)
try
{
    return trsm_mixed_impl(h, side, uplo, transA, diag, m, n, alpha, A, lda, B, ldb, slices);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_dtrsm_refined(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                                          rocblas_operation transA, rocblas_diagonal diag,
                                          rocblas_int m, rocblas_int n, const double* alpha,
                                          const double* A, rocblas_int lda, double* B, rocblas_int ldb,
                                          const rocblas_b200_refine_options* options,
                                          rocblas_b200_refine_info*          info)
try
{
    return trsm_refined_impl(h, side, uplo, transA, diag, m, n, alpha, A, lda, B, ldb, options, info);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_dtrsm_mixed_host(rocblas_handle h, rocblas_side side, rocblas_fill uplo,
                                             rocblas_operation transA, rocblas_diagonal diag,
                                             rocblas_int m, rocblas_int n, const double* alpha,
                                             const double* A, rocblas_int lda, double* B,
                                             rocblas_int ldb, rocblas_int slices)
try
{
    return trsm_mixed_host_impl(h, side, uplo, transA, diag, m, n, alpha, A, lda, B, ldb, slices);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_b200_set_tuning(const char* key, rocblas_int value)
{
    if(!key)
        return rocblas_status_invalid_pointer;
    return tuning_set(tuning(), key, value) ? rocblas_status_success : rocblas_status_invalid_value;
}

rocblas_status rocblas_b200_get_tuning(const char* key, rocblas_int* value)
{
    if(!key || !value)
        return rocblas_status_invalid_pointer;
    return tuning_get(tuning(), key, value) ? rocblas_status_success : rocblas_status_invalid_value;
}

rocblas_status rocblas_b200_get_device_error(rocblas_handle h, rocblas_int* code)
try
{
    if(!h)
        return rocblas_status_invalid_handle;
    if(!code)
        return rocblas_status_invalid_pointer;
    *code = 0;
    if(!h->err_dev)
        return rocblas_status_success;
    if(cudaStreamSynchronize(h->stream) != cudaSuccess)
        return rocblas_status_internal_error;
    int v = 0;
    cudaMemcpy(&v, h->err_dev, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemset(h->err_dev, 0, sizeof(int));
    *code = v;
    return launch_status();
}
catch(...)
{
    return exception_status();
}

// ---- trtri ------------------------------------------------------------------------------------
rocblas_status rocblas_strtri(rocblas_handle h, rocblas_fill uplo, rocblas_diagonal diag,
                              rocblas_int n, const float* A, rocblas_int lda, float* invA,
                              rocblas_int ldinvA)
try
{
    return trtri_impl<float>(h, uplo, diag, n, A, strided<float>(A, 0), lda, invA,
                             strided<float>(invA, 0), ldinvA, 1);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_dtrtri(rocblas_handle h, rocblas_fill uplo, rocblas_diagonal diag,
                              rocblas_int n, const double* A, rocblas_int lda, double* invA,
                              rocblas_int ldinvA)
try
{
    return trtri_impl<double>(h, uplo, diag, n, A, strided<double>(A, 0), lda, invA,
                              strided<double>(invA, 0), ldinvA, 1);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_strtri_batched(rocblas_handle h, rocblas_fill uplo, rocblas_diagonal diag,
                                      rocblas_int n, const float* const A[], rocblas_int lda,
                                      float* const invA[], rocblas_int ldinvA,
                                      rocblas_int batch_count)
try
{
    return trtri_impl<float>(h, uplo, diag, n, A, arrayed<float>(A), lda, invA,
                             arrayed<float>(invA), ldinvA, batch_count);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_dtrtri_batched(rocblas_handle h, rocblas_fill uplo, rocblas_diagonal diag,
                                      rocblas_int n, const double* const A[], rocblas_int lda,
                                      double* const invA[], rocblas_int ldinvA,
                                      rocblas_int batch_count)
try
{
    return trtri_impl<double>(h, uplo, diag, n, A, arrayed<double>(A), lda, invA,
                              arrayed<double>(invA), ldinvA, batch_count);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_strtri_strided_batched(rocblas_handle h, rocblas_fill uplo,
                                              rocblas_diagonal diag, rocblas_int n,
                                              const float* A, rocblas_int lda,
                                              rocblas_stride stride_a, float* invA,
                                              rocblas_int ldinvA, rocblas_stride stride_invA,
                                              rocblas_int batch_count)
try
{
    return trtri_impl<float>(h, uplo, diag, n, A, strided<float>(A, stride_a), lda, invA,
                             strided<float>(invA, stride_invA), ldinvA, batch_count);
}
catch(...)
{
    return exception_status();
}

rocblas_status rocblas_dtrtri_strided_batched(rocblas_handle h, rocblas_fill uplo,
                                              rocblas_diagonal diag, rocblas_int n,
                                              const double* A, rocblas_int lda,
                                              rocblas_stride stride_a, double* invA,
                                              rocblas_int ldinvA, rocblas_stride stride_invA,
                                              rocblas_int batch_count)
try
{
    return trtri_impl<double>(h, uplo, diag, n, A, strided<double>(A, stride_a), lda, invA,
                              strided<double>(invA, stride_invA), ldinvA, batch_count);
}
catch(...)
{
    return exception_status();
}

#define TRTRI_CPLX(S, TA, T)                                                                       \
    rocblas_status rocblas_##S##trtri(rocblas_handle h, rocblas_fill uplo, rocblas_diagonal diag,   \
                                      rocblas_int n, const TA* A, rocblas_int lda, TA* invA,        \
                                      rocblas_int ldinvA)                                           \
    try                                                                                             \
    {                                                                                               \
        return trtri_impl<T>(h, uplo, diag, n, A, strided<T>(as_impl<T>(A), 0), lda, invA,          \
                             strided<T>(as_impl<T>(invA), 0), ldinvA, 1);                          \
    }                                                                                               \
    catch(...)                                                                                      \
    {                                                                                               \
        return exception_status();                                                                  \
    }                                                                                               \
    rocblas_status rocblas_##S##trtri_batched(rocblas_handle h, rocblas_fill uplo,                  \
                                              rocblas_diagonal diag, rocblas_int n,                 \
                                              const TA* const A[], rocblas_int lda,                 \
                                              TA* const invA[], rocblas_int ldinvA,                 \
                                              rocblas_int batch_count)                              \
    try                                                                                             \
    {                                                                                               \
        return trtri_impl<T>(h, uplo, diag, n, A, arrayed<T>(A), lda, invA, arrayed<T>(invA),       \
                             ldinvA, batch_count);                                                  \
    }                                                                                               \
    catch(...)                                                                                      \
    {                                                                                               \
        return exception_status();                                                                  \
    }                                                                                               \
    rocblas_status rocblas_##S##trtri_strided_batched(                                              \
        rocblas_handle h, rocblas_fill uplo, rocblas_diagonal diag, rocblas_int n, const TA* A,     \
        rocblas_int lda, rocblas_stride stride_a, TA* invA, rocblas_int ldinvA,                     \
        rocblas_stride stride_invA, rocblas_int batch_count)                                        \
    try                                                                                             \
    {                                                                                               \
        return trtri_impl<T>(h, uplo, diag, n, A, strided<T>(as_impl<T>(A), stride_a), lda, invA,   \
                             strided<T>(as_impl<T>(invA), stride_invA), ldinvA, batch_count);      \
    }                                                                                               \
    catch(...)                                                                                      \
    {                                                                                               \
        return exception_status();                                                                  \
    }
TRTRI_CPLX(c, rocblas_float_complex, cplx<float>)
TRTRI_CPLX(z, rocblas_double_complex, cplx<double>)

} // extern "C"
