// Kernels of the iteratively refined precision-form solve (rocblas_b200_dtrsm_refined): the
// FP64 residual's elementwise part (and the gather of the tested right-hand sides), the
// comparison of the test, and the correction X += D.  All of them are HBM-bound passes; the
// residual's product itself runs on the FP64 DMMA tiles (gemm_dmma.cuh).
//
// Right-hand sides are the columns of B for side left and its rows for side right.  A test on
// c of nrhs right-hand sides uses the evenly spaced ones idx(j) = floor((2j + 1) nrhs / (2c)).
#pragma once
#include "common.cuh"

namespace rb200
{

__device__ __forceinline__ int64_t refine_sample_index(int64_t j, int64_t nrhs, int64_t c)
{
    return ((2 * j + 1) * nrhs) / (2 * c);
}

// O := alpha B0(src) - (unit ? X(src) : 0), and Xs := X(src) when Xs != nullptr, for the
// rows x cols output O (ld ldo).  sampled == 0: src = (i, j) (the full residual's start);
// sampled, side left: src = (i, idx(j)) with idx over the n columns; sampled, side right:
// src = (idx(i), j) over the m rows.  The product - op(A) X (strict triangle when unit) is
// added to O afterwards by one GEMM.
__global__ void __launch_bounds__(256)
    refine_prep_kernel(const double* X, int64_t ldx, const double* B0, int64_t ldb0, int rows, int cols,
                       int sampled, int side_left, int64_t nrhs, double alpha, int unit, double* O,
                       int64_t ldo, double* Xs, int64_t ldxs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= rows)
        return;
    for(int j = blockIdx.y; j < cols; j += gridDim.y)
    {
        int64_t si = i, sj = j;
        if(sampled)
        {
            if(side_left)
                sj = refine_sample_index(j, nrhs, cols);
            else
                si = refine_sample_index(i, nrhs, rows);
        }
        const double x = X[si + sj * ldx];
        const double b = B0[si + sj * ldb0];
        O[i + (int64_t)j * ldo] = alpha * b - (unit ? x : 0.0);
        if(Xs)
            Xs[i + (int64_t)j * ldxs] = x;
    }
}

// The larger of a and b, NaN if either is NaN (fmax would drop it).
__device__ __forceinline__ double max_nan(double a, double b)
{
    if(a != a)
        return a;
    if(b != b)
        return b;
    return a > b ? a : b;
}

// The test of the refined solve, for each tested right-hand side v (block v):
// out[2v] = max |X(v) - Xref(v)|, out[2v + 1] = max |Xref(v)| (NaN if any entry is NaN).
// X is the solution in place in B (ld ldx); Xref holds the tested right-hand sides solved by
// the plain FP64 form: side left the columns idx(v) of X in an srows x c buffer, side right the
// rows idx(v) in a c x scols buffer (ld srows = c).
__global__ void __launch_bounds__(256)
    refine_compare_kernel(const double* X, int64_t ldx, const double* Xref, int srows, int scols,
                          int side_left, int64_t nrhs, double* out)
{
    __shared__ double dd[256], xx[256];
    const int     v   = blockIdx.x;
    const int     c   = side_left ? scols : srows;
    const int64_t src = refine_sample_index(v, nrhs, c);
    const int     len = side_left ? srows : scols;
    double        md = 0.0, mx = 0.0;
    for(int q = threadIdx.x; q < len; q += blockDim.x)
    {
        const double x = side_left ? X[q + src * ldx] : X[src + (int64_t)q * ldx];
        const double r = side_left ? Xref[q + (int64_t)v * srows] : Xref[v + (int64_t)q * srows];
        md = max_nan(md, fabs(x - r));
        mx = max_nan(mx, fabs(r));
    }
    dd[threadIdx.x] = md;
    xx[threadIdx.x] = mx;
    __syncthreads();
    for(int w = 128; w > 0; w >>= 1)
    {
        if(threadIdx.x < w)
        {
            dd[threadIdx.x] = max_nan(dd[threadIdx.x], dd[threadIdx.x + w]);
            xx[threadIdx.x] = max_nan(xx[threadIdx.x], xx[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if(threadIdx.x == 0)
    {
        out[2 * v]     = dd[0];
        out[2 * v + 1] = xx[0];
    }
}

// X := X + D over m x n (ld ldx, ldd).
__global__ void __launch_bounds__(256)
    refine_update_kernel(double* X, int64_t ldx, const double* D, int64_t ldd, int m, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m)
        return;
    for(int j = blockIdx.y; j < n; j += gridDim.y)
        X[i + (int64_t)j * ldx] += D[i + (int64_t)j * ldd];
}

} // namespace rb200
