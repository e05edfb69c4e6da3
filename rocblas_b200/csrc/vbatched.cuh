// Variable-size batched TRSM: thousands of independent systems of different (m, n),
// side, uplo, transA and diag in one call.
//
// The reference has no variable-size batch API (rocblas_trsm_batched requires one m, n for
// every entry, library/src/blas3/rocblas_trsm_batched_imp.hpp:57-300), so a caller with
// uneven systems makes one call per system.  Here one prepass and one persistent launch per
// size class cover the whole batch:
//   1. a single-CTA prepass validates every problem descriptor, sorts it into a size class by
//      its triangle order k (k <= 64, 128, 256, 512), counts its work items (strips of 32
//      right-hand sides) and writes, per class, the exclusive prefix sum of those counts
//      (problems of other classes count 0);
//   2. per class, a persistent kernel (grid = SMs x resident CTAs, shared memory sized for
//      that class's largest k, so small systems run many CTAs per SM) pulls work-item indices
//      from the class's device-side queue head (one atomicAdd per item), maps an item to its
//      (problem, strip) by binary search over the class's prefix sum, and runs the one-CTA
//      strip solver (block_solve.cuh) on it.  There is no inter-CTA waiting, so no wait can
//      hang.
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
constexpr int kVbClasses = 4;
__host__ __device__ constexpr int vb_class_kmax(int c)
{
    return 64 << c;
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
    __shared__ int4 part[kVbPrepThreads];
    const int tid   = threadIdx.x;
    const int chunk = (count + kVbPrepThreads - 1) / kVbPrepThreads;
    const int lo = min(count, tid * chunk), hi = min(count, lo + chunk);
    int       sum[kVbClasses] = {0, 0, 0, 0};
    int       bad             = 0;
    static_assert(kVbClasses == 4, "one int4 of partial sums per thread");
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
    part[tid] = make_int4(sum[0], sum[1], sum[2], sum[3]);
    __syncthreads();
    // inclusive scan of the per-thread sums, four classes at once (Hillis-Steele)
    for(int off = 1; off < kVbPrepThreads; off <<= 1)
    {
        const int4 v = tid >= off ? part[tid - off] : make_int4(0, 0, 0, 0);
        __syncthreads();
        int4 w = part[tid];
        w.x += v.x;
        w.y += v.y;
        w.z += v.z;
        w.w += v.w;
        part[tid] = w;
        __syncthreads();
    }
    const int4 incl = part[tid];
    int run[kVbClasses] = {incl.x - sum[0], incl.y - sum[1], incl.z - sum[2], incl.w - sum[3]};
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
        offsets[0 * cstride + count] = incl.x;
        offsets[1 * cstride + count] = incl.y;
        offsets[2 * cstride + count] = incl.z;
        offsets[3 * cstride + count] = incl.w;
#pragma unroll
        for(int c = 0; c < kVbClasses; ++c)
            st->counter[c] = 0;
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

} // namespace rb200
