// Variable-size batched TRSM: thousands of independent systems of different (m, n),
// side, uplo, transA and diag in one call.
//
// The reference has no variable-size batch API (rocblas_trsm_batched requires one m, n for
// every entry, library/src/blas3/rocblas_trsm_batched_imp.hpp:57-300), so a caller with
// uneven systems makes one call per system.  Here one prepass and one persistent launch per
// size class cover the whole batch:
//   1. a single-CTA prepass validates every problem descriptor, sorts it into a size class by
//      its triangle order k (k <= 32, 64, 128, 256, 512), counts its work items (strips of 32
//      right-hand sides) and writes, per class, the exclusive prefix sum of those counts
//      (problems of other classes count 0);
//   2. per class, a persistent kernel (grid = SMs x resident CTAs, shared memory sized for
//      that class's largest k, so small systems run many CTAs per SM) pulls work-item indices
//      from the class's device-side queue head (one atomicAdd per item), maps an item to its
//      (problem, strip) by binary search over the class's prefix sum, and runs the one-CTA
//      strip solver (block_solve.cuh) on it; the k <= 32 class runs one strip per warp
//      instead (vb_warp_kernel).  There is no inter-CTA waiting, so no wait can hang.
// All launches are stream-ordered and capturable in a CUDA graph.
#pragma once
#include "block_solve.cuh"

namespace rb200
{

// Problem descriptor, same layout as rocblas_b200_trsm_problem in rocblas_b200_ext.h.
struct VbProblem
{
    const void* A;
    void*       B;
    int         m, n, lda, ldb;
    int         side, uplo, trans, diag;
};

struct VbState
{
    int counter; // queue head
    int invalid; // number of rejected descriptors
    int pad[2];
};

// Size classes of the batch: class c holds the systems with k <= vb_class_kmax(c).
constexpr int kVbClasses = 5;
__host__ __device__ constexpr int vb_class_kmax(int c)
{
    return 32 << c;
}
static_assert(vb_class_kmax(kVbClasses - 1) == kBlockSolveMaxK, "classes cover the strip solver");

__device__ __forceinline__ int vb_class(int k)
{
    int c = 0;
    while(c < kVbClasses - 1 && k > vb_class_kmax(c))
        ++c;
    return c;
}

struct VbClassState
{
    int counter[kVbClasses]; // queue head per class
    int invalid;             // number of rejected descriptors
    int pad[3];
};

constexpr int kVbPrepThreads = 1024;

__device__ __forceinline__ bool vb_valid(const VbProblem& p, int max_k)
{
    if(p.side != kLeft && p.side != kRight)
        return false;
    if(p.uplo != kLower && p.uplo != kUpper)
        return false;
    if(p.trans != kOpN && p.trans != kOpT && p.trans != kOpC)
        return false;
    if(p.diag != kNonUnit && p.diag != kUnit)
        return false;
    const int k = p.side == kLeft ? p.m : p.n;
    if(p.m < 0 || p.n < 0 || p.lda < k || p.ldb < p.m || k > max_k)
        return false;
    if((p.m > 0 && p.n > 0) && (!p.A || !p.B))
        return false;
    return true;
}

__device__ __forceinline__ int vb_items(const VbProblem& p)
{
    const int ncols = p.side == kLeft ? p.n : p.m;
    const int k     = p.side == kLeft ? p.m : p.n;
    if(k == 0 || ncols == 0)
        return 0;
    return (ncols + kBsW - 1) / kBsW;
}

// offsets[i] = number of work items of problems 0..i-1; offsets[count] = total.
__global__ void __launch_bounds__(kVbPrepThreads)
    vb_prepass_kernel(const VbProblem* probs, int count, int max_k, int* offsets, VbState* st)
{
    __shared__ int part[kVbPrepThreads];
    const int tid   = threadIdx.x;
    const int chunk = (count + kVbPrepThreads - 1) / kVbPrepThreads;
    const int lo = min(count, tid * chunk), hi = min(count, lo + chunk);
    int       sum = 0, bad = 0;
    for(int i = lo; i < hi; ++i)
    {
        const VbProblem p = probs[i];
        if(vb_valid(p, max_k))
            sum += vb_items(p);
        else
            ++bad;
    }
    part[tid] = sum;
    __syncthreads();
    // inclusive scan of the per-thread sums (Hillis-Steele)
    for(int off = 1; off < kVbPrepThreads; off <<= 1)
    {
        const int v = tid >= off ? part[tid - off] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = part[tid] - sum; // exclusive prefix of this thread's chunk
    for(int i = lo; i < hi; ++i)
    {
        offsets[i]        = run;
        const VbProblem p = probs[i];
        if(vb_valid(p, max_k))
            run += vb_items(p);
    }
    if(tid == kVbPrepThreads - 1)
    {
        offsets[count] = part[tid];
        st->counter    = 0;
    }
    if(bad)
        atomicAdd(&st->invalid, bad);
}

// Per class c: offsets[c * (count + 1) + i] = work items of the class-c problems among
// 0..i-1; offsets[c * (count + 1) + count] = the class total.  Problems with k > skip_above
// belong to another path of the call: they count neither as work nor as invalid.
__global__ void __launch_bounds__(kVbPrepThreads)
    vb_prepass_classes_kernel(const VbProblem* probs, int count, int max_k, int skip_above,
                              int* offsets, VbClassState* st)
{
    __shared__ int part[kVbClasses][kVbPrepThreads];
    const int tid   = threadIdx.x;
    const int chunk = (count + kVbPrepThreads - 1) / kVbPrepThreads;
    const int lo = min(count, tid * chunk), hi = min(count, lo + chunk);
    int       sum[kVbClasses] = {};
    int       bad             = 0;
    for(int i = lo; i < hi; ++i)
    {
        const VbProblem p = probs[i];
        if((p.side == kLeft ? p.m : p.n) > skip_above)
            continue; // another path of the call solves it (or rejects it)
        if(vb_valid(p, max_k))
            sum[vb_class(p.side == kLeft ? p.m : p.n)] += vb_items(p);
        else
            ++bad;
    }
#pragma unroll
    for(int c = 0; c < kVbClasses; ++c)
        part[c][tid] = sum[c];
    __syncthreads();
    // inclusive scan of the per-thread sums, all classes at once (Hillis-Steele)
    for(int off = 1; off < kVbPrepThreads; off <<= 1)
    {
        int v[kVbClasses];
#pragma unroll
        for(int c = 0; c < kVbClasses; ++c)
            v[c] = tid >= off ? part[c][tid - off] : 0;
        __syncthreads();
#pragma unroll
        for(int c = 0; c < kVbClasses; ++c)
            part[c][tid] += v[c];
        __syncthreads();
    }
    int run[kVbClasses];
#pragma unroll
    for(int c = 0; c < kVbClasses; ++c)
        run[c] = part[c][tid] - sum[c];
    const int64_t cstride = (int64_t)count + 1;
    for(int i = lo; i < hi; ++i)
    {
#pragma unroll
        for(int c = 0; c < kVbClasses; ++c)
            offsets[c * cstride + i] = run[c];
        const VbProblem p = probs[i];
        if((p.side == kLeft ? p.m : p.n) <= skip_above && vb_valid(p, max_k))
            run[vb_class(p.side == kLeft ? p.m : p.n)] += vb_items(p);
    }
    if(tid == kVbPrepThreads - 1)
    {
#pragma unroll
        for(int c = 0; c < kVbClasses; ++c)
        {
            offsets[c * cstride + count] = part[c][tid];
            st->counter[c]               = 0;
        }
    }
    if(bad)
        atomicAdd(&st->invalid, bad);
}

template <typename T>
struct VbParams
{
    const VbProblem* probs;
    int              count;
    const int*       offsets; // count + 1 prefix sums of the work items this launch serves
    int*             counter; // queue head of this launch
    Scalar<T>        alpha;
};

template <typename T>
__global__ void __launch_bounds__(kBsThreads, 2) vb_persistent_kernel(VbParams<T> p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    const int total = p.offsets[p.count];
    const T   alpha = p.alpha.get();
    for(;;)
    {
        if(threadIdx.x == 0)
            s_item = atomicAdd(p.counter, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if(item >= total)
            break;
        // problem index: last i with offsets[i] <= item (empty problems share offsets)
        int lo = 0, hi = p.count - 1;
        while(lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if(p.offsets[mid] <= item)
                lo = mid;
            else
                hi = mid - 1;
        }
        const VbProblem q = p.probs[lo];
        const int strip = item - p.offsets[lo];
        const int left  = q.side == kLeft;
        const int k     = left ? q.m : q.n;
        const int ncols = left ? q.n : q.m;
        const int trans = q.trans != kOpN;
        const int tM    = trans != (left ? 0 : 1);
        const int oplow = (q.uplo == kLower) != (trans != 0);
        const int mlow  = left ? oplow : !oplow;
        block_solve_strip<T>(reinterpret_cast<const T*>(q.A), q.lda, reinterpret_cast<T*>(q.B),
                             q.ldb, k, left, tM, !mlow, q.diag == kUnit, 0, alpha, strip * kBsW,
                             ncols, smem_raw);
        __syncthreads();
    }
}

// ---- warp-level strips for the smallest class (k <= 32) ------------------------------------
// A CTA-wide strip solve spends most of its time on loads and barriers when k is small, and
// the batch has tens of thousands of such strips (every side-right system with few columns in
// A).  Here a warp solves a whole strip on its own: lane = column of the strip, the column in
// 32 registers, the diagonal tile of M through a warp-private 32 x 33 buffer, no CTA barrier.
// (A second panel would double the unrolled code, and the warps' instruction fetch is then
// what bounds the kernel; k in (32, 64] stays on the CTA solver.)
constexpr int kVbWarpMaxK   = 32;
constexpr int kVbWarpsPerCta = 4;

template <typename T>
__host__ __device__ constexpr size_t vb_warp_smem_bytes()
{
    return sizeof(T) * (size_t)kVbWarpsPerCta * (32 * 33 + 32);
}

template <typename T>
__device__ void warp_strip_solve(const T* A, int64_t lda, T* B, int64_t ldb, int k, int side_left,
                                 int tM, int rev, int unit, T alpha, int s0, int ncols, T* Ws, T* rd)
{
    const int lane = threadIdx.x & 31;
    const int W    = min(kBsW, ncols - s0);
    T* const      B0  = B + (side_left ? (int64_t)s0 * ldb : (int64_t)s0);
    const int64_t bdr = side_left ? 1 : ldb, bdc = side_left ? ldb : 1;
    // C'(i, col): row i of the reversed orientation (rev: C row k-1-i)
    auto caddr = [&](int i, int col) -> T* { return B0 + (rev ? k - 1 - i : i) * bdr + col * bdc; };
    if(alpha == T(0))
    {
        if(lane < W)
            for(int i = 0; i < k; ++i)
                *caddr(i, lane) = T(0);
        return;
    }
    const int64_t  sgn = rev ? -1 : 1;
    const int64_t  dI = (tM ? lda : 1) * sgn, dJ = (tM ? 1 : lda) * sgn;
    const T* const M0 = A + (rev ? (int64_t)(k - 1) * (1 + lda) : 0);
    const bool     icontig = !tM; // A's contiguous direction runs along i of M'
    // tile (i0, j0) of M' into Ws (zero outside k); a diagonal tile keeps its strict lower part
    // and the reciprocal diagonal in rd (unit: 1; padding rows: 1)
    auto load_tile = [&](int i0, int j0, bool diagonal) {
        // 8 independent loads in flight per lane before their stores
#pragma unroll 1
        for(int t0 = 0; t0 < 32; t0 += 8)
        {
            T v[8];
#pragma unroll
            for(int u = 0; u < 8; ++u)
            {
                const int t = t0 + u;
                const int i = icontig ? lane : t, j = icontig ? t : lane;
                const int gi = i0 + i, gj = j0 + j;
                v[u]         = T(0);
                if(gi < k && gj < k && (!diagonal || j <= i) && !(diagonal && i == j && unit))
                    v[u] = M0[gi * dI + gj * dJ];
            }
#pragma unroll
            for(int u = 0; u < 8; ++u)
            {
                const int t = t0 + u;
                const int i = icontig ? lane : t, j = icontig ? t : lane;
                if(diagonal && i == j)
                {
                    // unit, padding rows and (as in the strip solver) nothing else: 1 / M_ii
                    rd[i] = (i0 + i < k && !unit) ? T(1) / v[u] : T(1);
                    v[u]  = T(0);
                }
                Ws[i * 33 + j] = v[u];
            }
        }
        __syncwarp();
    };
    auto substitute = [&](T (&y)[32]) {
#pragma unroll
        for(int j = 0; j < 32; ++j)
        {
            y[j] *= rd[j];
#pragma unroll
            for(int i = j + 1; i < 32; ++i)
                y[i] -= Ws[i * 33 + j] * y[j];
        }
    };
    const bool col_ok = lane < W;
    T          y[32];
#pragma unroll
    for(int i = 0; i < 32; ++i)
        y[i] = (col_ok && i < k) ? alpha * *caddr(i, lane) : T(0);
    load_tile(0, 0, true);
    substitute(y);
    if(col_ok)
    {
#pragma unroll
        for(int i = 0; i < 32; ++i)
            if(i < k)
                *caddr(i, lane) = y[i];
    }
    __syncwarp();
}

// The class queue of vb_persistent_kernel, one item per warp.
template <typename T>
__global__ void __launch_bounds__(32 * kVbWarpsPerCta) vb_warp_kernel(VbParams<T> p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp  = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T*        Ws    = reinterpret_cast<T*>(smem_raw) + (size_t)warp * (32 * 33 + 32);
    T*        rd    = Ws + 32 * 33;
    const int total = p.offsets[p.count];
    const T   alpha = p.alpha.get();
    for(;;)
    {
        int item = 0;
        if(lane == 0)
            item = atomicAdd(p.counter, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if(item >= total)
            break;
        // problem index: last i with offsets[i] <= item (empty problems share offsets)
        int lo = 0, hi = p.count - 1;
        while(lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if(p.offsets[mid] <= item)
                lo = mid;
            else
                hi = mid - 1;
        }
        const VbProblem q     = p.probs[lo];
        const int       strip = item - p.offsets[lo];
        const int       left  = q.side == kLeft;
        const int       k     = left ? q.m : q.n;
        const int       ncols = left ? q.n : q.m;
        const int       trans = q.trans != kOpN;
        const int       tM    = trans != (left ? 0 : 1);
        const int       oplow = (q.uplo == kLower) != (trans != 0);
        const int       mlow  = left ? oplow : !oplow;
        warp_strip_solve<T>(reinterpret_cast<const T*>(q.A), q.lda, reinterpret_cast<T*>(q.B), q.ldb,
                            k, left, tM, !mlow, q.diag == kUnit, alpha, strip * kBsW, ncols, Ws, rd);
    }
}

} // namespace rb200
