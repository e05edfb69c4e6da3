// Check-numerics of the TRSM operands: the reference's ROCBLAS_CHECK_NUMERICS protocol.
//
//   * the mode is read from ROCBLAS_CHECK_NUMERICS when a handle is created (bits: 1 info,
//     2 warn, 4 fail, 8 NaN and Inf only; library/src/handle.cpp:921-931);
//   * before the solve the referenced triangle of A (diagonal included) and all of B are
//     scanned, after it all of B (library/src/blas3/rocblas_trmm_kernels.cpp:2306-2362, called
//     from rocblas_trsm_imp.hpp:159-181 and :248-270); a host alpha == 0 call returns before
//     any check;
//   * one flag each for NaN, zero, Inf and denormal values (library/src/check_numerics_matrix.cpp;
//     the predicates of library/src/include/utility.hpp:484-672: a complex value is NaN, Inf or
//     denormal if either part is, zero if both parts are);
//   * info prints the flags of every check, warn prints them when a NaN, Inf or denormal value
//     was found (denormals not counted with bit 8), fail returns
//     rocblas_status_check_numerics_fail for such a value (check_numerics_vector.cpp:95-136).
// The scan reads every element once (HBM-bound) and synchronizes the handle's stream to read
// its flags; under stream capture the check is skipped, as the reference does.
#pragma once
#include <algorithm>
#include <cfloat>
#include <cstdio>

#include "common.cuh"

namespace rb200
{

enum : unsigned
{
    kNumNaN    = 1,
    kNumZero   = 2,
    kNumInf    = 4,
    kNumDenorm = 8,
};

enum : int
{
    kCheckInfo       = 1,
    kCheckWarn       = 2,
    kCheckFail       = 4,
    kCheckOnlyNanInf = 8,
};

template <typename R>
__device__ __forceinline__ unsigned num_flags_part(R v)
{
    const R  a     = v < R(0) ? -v : v;
    const R  tiny  = sizeof(R) == 4 ? R(FLT_MIN) : R(DBL_MIN);
    unsigned flags = 0;
    if(isnan(v))
        flags |= kNumNaN;
    if(isinf(v))
        flags |= kNumInf;
    if(a > R(0) && a < tiny)
        flags |= kNumDenorm;
    return flags;
}

template <typename T>
__device__ __forceinline__ unsigned num_flags(T v)
{
    return num_flags_part(v) | (v == T(0) ? kNumZero : 0u);
}

template <typename R>
__device__ __forceinline__ unsigned num_flags(cplx<R> v)
{
    return num_flags_part(v.x) | num_flags_part(v.y) | (v.x == R(0) && v.y == R(0) ? kNumZero : 0u);
}

// rows x cols of every batch entry (blockIdx.z + batch_base), the launch covering the rows from
// row0; tri: 0 every element, 1 the lower triangle (row >= col), 2 the upper one (row <= col).
// Column loop over gridDim.y.
template <typename T>
__global__ void __launch_bounds__(256)
    check_numerics_kernel(BatchPtr<T> A, int64_t lda, int64_t row0, int64_t rows, int64_t cols,
                          int tri, int batch_base, unsigned* flags)
{
    const int64_t row   = row0 + (int64_t)blockIdx.x * 256 + threadIdx.x;
    unsigned      local = 0;
    if(row < rows)
    {
        const T* a = A.get(batch_base + (int)blockIdx.z);
        for(int64_t col = blockIdx.y; col < cols; col += gridDim.y)
        {
            if((tri == 1 && row < col) || (tri == 2 && row > col))
                continue;
            local |= num_flags(a[row + col * lda]);
        }
    }
    local = __reduce_or_sync(0xffffffffu, local);
    if((threadIdx.x & 31) == 0 && local)
        atomicOr(flags, local);
}

// Prints and decides as the reference's rocblas_check_numerics_abnormal_struct.
inline rocblas_status check_numerics_report(const char* name, int mode, bool is_input, unsigned f)
{
    const bool nan = f & kNumNaN, inf = f & kNumInf, zero = f & kNumZero, den = f & kNumDenorm;
    const bool abnormal = nan || inf || (den && !(mode & kCheckOnlyNanInf));
    if((mode & kCheckInfo) || ((mode & kCheckWarn) && abnormal))
        std::fprintf(stderr, "Function name:\t%s :- %s :\t has_NaN %d has_zero %d has_Inf %d has_denorm %d\n",
                     name, is_input ? "Input" : "Output", (int)nan, (int)zero, (int)inf, (int)den);
    if(abnormal && (mode & kCheckFail))
        return rocblas_status_check_numerics_fail;
    return rocblas_status_success;
}

// Scans rows x cols (tri as in the kernel) of `batch` matrices into *flags_dev on `s` and
// returns the flags (synchronizes s). flags_dev: one device word.
template <typename T>
bool check_numerics_scan(BatchPtr<T> A, int64_t lda, int64_t rows, int64_t cols, int tri, int64_t batch,
                         unsigned* flags_dev, cudaStream_t s, unsigned* flags)
{
    *flags = 0;
    if(rows <= 0 || cols <= 0 || batch <= 0 || !A.valid())
        return true;
    if(cudaMemsetAsync(flags_dev, 0, sizeof(unsigned), s) != cudaSuccess)
        return false;
    // rows in launches of at most 2^30 (grid x stays far below its limit); batch entries in
    // launches of at most 65535 (grid z)
    constexpr int64_t kRowChunk = int64_t(1) << 30;
    const unsigned    gy        = (unsigned)std::min<int64_t>(cols, 1024);
    for(int64_t r0 = 0; r0 < rows; r0 += kRowChunk)
    {
        const unsigned gx = (unsigned)((std::min(kRowChunk, rows - r0) + 255) / 256);
        for(int64_t b0 = 0; b0 < batch; b0 += 65535)
        {
            const unsigned gz = (unsigned)std::min<int64_t>(65535, batch - b0);
            check_numerics_kernel<T><<<dim3(gx, gy, gz), 256, 0, s>>>(A, lda, r0, rows, cols, tri,
                                                                       (int)b0, flags_dev);
        }
    }
    if(cudaMemcpyAsync(flags, flags_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return false;
    return cudaStreamSynchronize(s) == cudaSuccess;
}

} // namespace rb200
