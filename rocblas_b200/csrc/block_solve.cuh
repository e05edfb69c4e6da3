// One-CTA triangular solve of a strip of right-hand sides, for small and batched systems.
//
// Replaces the reference's small and substitution kernels
// (library/src/blas3/rocblas_trsm_kernels.hpp: rocblas_trsm_small_right_device :1962-2227,
// rocblas_trsm_small_left_device :2359-2560, ..._sharedB :2562-2780, the blocked
// forward/backward substitution :3059-3261 and its host loop :3263-3515) with one kernel
// that handles all 16 side/uplo/trans/diag combinations through an index map:
//
//   side L:  op(A) X = alpha B          ->  M Y = alpha C with M = op(A),   C = B,   Y = X
//   side R:  X op(A) = alpha B          ->  M Y = alpha C with M = op(A)^T, C = B^T, Y = X^T
//
// M(i,j) is A(i,j) or A(j,i).  If M is upper the rows are reversed (i -> k-1-i), which turns
// every case into a forward (lower) solve.  A CTA owns one strip of W = 32 columns of C
// (32 columns of B for side L, 32 rows of B for side R), keeps the whole k x 32 strip in
// shared memory, and walks the diagonal in 32-row panels:
//   1. stage the 32 x 32 diagonal tile of M (reciprocal diagonal precomputed, as the
//      reference does at :3204-3219);
//   2. forward substitution with warp shuffles: warp w owns columns w, w+8, w+16, w+24,
//      lane l owns row l; each solved row value is broadcast with __shfl_sync (the
//      reference broadcasts through LDS with two __syncthreads per row, :3225-3248);
//   3. rank-32 update of the remaining rows from panels of M streamed through shared
//      memory in 64-row chunks.
// k is at most kBlockSolveMaxK; larger systems use the blocked recursive path.
#pragma once
#include "common.cuh"

namespace rb200
{

constexpr int kBsW       = 32;  // right-hand sides per CTA
constexpr int kBsPitch   = kBsW + 1;
constexpr int kBsThreads = 256;
constexpr int kBsChunk   = 64;  // panel rows per update chunk
constexpr int kBlockSolveMaxK = 512;

// The largest order one CTA solves: the k x 32 strip of C lives in shared memory, so complex
// double (16-byte elements) stops at 256 to stay within 227 KB.
template <typename T>
constexpr int block_solve_max_k()
{
    return sizeof(T) > 8 ? 256 : kBlockSolveMaxK;
}

// One system (or a uniform batch of systems).
template <typename T>
struct BlockSolveParams
{
    int         m, n, k;        // B is m x n; A is k x k
    int         side_left;
    int         tM;             // M(i,j) = tM ? A(j,i) : A(i,j)
    int         rev;            // M upper: rows reversed
    int         unit;
    int         conj;           // M's entries are conjugated (complex trans C)
    BatchPtr<T> A;
    int64_t     lda;
    BatchPtr<T> B;
    int64_t     ldb;
    Scalar<T>   ualpha;         // the caller's alpha
    int         first;          // 1: this solve applies ualpha; 0: it applies 1
    int         batch_base;
};

template <typename T>
constexpr size_t block_solve_smem_bytes(int k)
{
    const int kpad = (int)ceil_div(k, 32) * 32;
    return sizeof(T) * (size_t)(kpad * kBsPitch + 32 * 33 + 32 + kBsChunk * 33);
}

// The core: solve M Y = alpha C for one strip.  The caller resolves pointers / sizes.
template <typename T>
__device__ void block_solve_strip(const T* A, int64_t lda, T* B, int64_t ldb, int k,
                                  int side_left, int tM, int rev, int unit, int conj, T alpha,
                                  int s0, int ncols, unsigned char* smem_raw)
{
    T* Cs    = reinterpret_cast<T*>(smem_raw);
    const int kpad = ((k + 31) / 32) * 32;
    T* Ds    = Cs + kpad * kBsPitch;
    T* rdiag = Ds + 32 * 33;
    T* Ps    = rdiag + 32;

    const int tid  = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int W    = min(kBsW, ncols - s0); // valid columns of this strip

    // C(r, col) address in B: side L -> B[r + (s0+col) ldb]; side R -> B[(s0+col) + r ldb]
    auto baddr = [&](int r, int col) -> T* {
        return side_left ? B + r + (int64_t)(s0 + col) * ldb : B + (s0 + col) + (int64_t)r * ldb;
    };
    // M'(i, j) (reversed, lower orientation) -> A element
    auto mval = [&](int i, int j) -> T {
        const int a = rev ? k - 1 - i : i, b = rev ? k - 1 - j : j;
        const int r = tM ? b : a, c = tM ? a : b;
        return conj_if(A[r + (int64_t)c * lda], conj);
    };

    if(alpha == T(0))
    {
        // B := 0 without reading A or B (rocblas_trsm_imp.hpp:154-157 semantics)
        for(int idx = tid; idx < k * kBsW; idx += kBsThreads)
        {
            int r, col;
            if(side_left) { r = idx % k; col = idx / k; }
            else          { col = idx % kBsW; r = idx / kBsW; }
            if(col < W)
                *baddr(r, col) = T(0);
        }
        return;
    }

    // ---- load alpha * C' (rows reversed when rev), zero-pad rows k..kpad-1 ----------------
    for(int idx = tid; idx < kpad * kBsW; idx += kBsThreads)
    {
        int r, col;
        if(side_left) { r = idx % kpad; col = idx / kpad; }
        else          { col = idx % kBsW; r = idx / kBsW; }
        T v = T(0);
        if(r < k && col < W)
            v = alpha * (*baddr(r, col));
        const int i = (r < k && rev) ? k - 1 - r : r;
        Cs[i * kBsPitch + col] = v;
    }
    __syncthreads();

    // A is read-only, so the loads of the next diagonal tile or update chunk are issued into
    // registers before the current step computes, and land in shared memory after it.
    constexpr int kDiagPer  = 32 * 32 / kBsThreads;       // 4 values per thread
    constexpr int kChunkPer = kBsChunk * 32 / kBsThreads; // 8 values per thread
    static_assert(kDiagPer <= kChunkPer, "one prefetch buffer serves both steps");
    T pre[kChunkPer];
    auto fetch_diag = [&](int p) {
#pragma unroll
        for(int u = 0; u < kDiagPer; ++u)
        {
            const int idx = tid + u * kBsThreads;
            int       i, j;
            if(!tM) { i = idx % 32; j = idx / 32; }
            else    { j = idx % 32; i = idx / 32; }
            T v = T(0);
            if(p + i < k)
            {
                if(j < i)
                    v = mval(p + i, p + j);
                else if(i == j)
                    v = unit ? T(1) : mval(p + i, p + i);
            }
            else if(i == j)
                v = T(1); // padding rows solve 0 = 0
            pre[u] = v;
        }
    };
    auto store_diag = [&]() {
#pragma unroll
        for(int u = 0; u < kDiagPer; ++u)
        {
            const int idx = tid + u * kBsThreads;
            int       i, j;
            if(!tM) { i = idx % 32; j = idx / 32; }
            else    { j = idx % 32; i = idx / 32; }
            if(i == j)
                rdiag[i] = T(1) / pre[u];
            Ds[i * 33 + j] = j < i ? pre[u] : T(0);
        }
    };
    auto fetch_chunk = [&](int p, int i0) {
#pragma unroll
        for(int u = 0; u < kChunkPer; ++u)
        {
            const int idx = tid + u * kBsThreads;
            int       r, t;
            if(!tM) { r = idx % kBsChunk; t = idx / kBsChunk; }
            else    { t = idx % 32; r = idx / 32; }
            T v = T(0);
            if(i0 + r < k && p + t < k)
                v = mval(i0 + r, p + t);
            pre[u] = v;
        }
    };
    auto store_chunk = [&]() {
#pragma unroll
        for(int u = 0; u < kChunkPer; ++u)
        {
            const int idx = tid + u * kBsThreads;
            int       r, t;
            if(!tM) { r = idx % kBsChunk; t = idx / kBsChunk; }
            else    { t = idx % 32; r = idx / 32; }
            Ps[r * 33 + t] = pre[u];
        }
    };

    fetch_diag(0);
    for(int p = 0; p < k; p += 32)
    {
        // ---- 1. diagonal tile of M' (prefetched) -------------------------------------------
        store_diag();
        __syncthreads();
        if(p + 32 < k)
            fetch_chunk(p, p + 32);

        // ---- 2. substitution with shuffle broadcast -----------------------------------------
        {
            T y[4];
#pragma unroll
            for(int q = 0; q < 4; ++q)
                y[q] = Cs[(p + lane) * kBsPitch + warp + 8 * q];
            const T dl = rdiag[lane];
#pragma unroll 4
            for(int t = 0; t < 32; ++t)
            {
                const T lt = Ds[lane * 33 + t];
#pragma unroll
                for(int q = 0; q < 4; ++q)
                {
                    if(lane == t)
                        y[q] *= dl;
                    const T v = shfl_idx(y[q], t);
                    if(lane > t)
                        y[q] -= lt * v;
                }
            }
#pragma unroll
            for(int q = 0; q < 4; ++q)
                Cs[(p + lane) * kBsPitch + warp + 8 * q] = y[q];
        }
        __syncthreads();

        // ---- 3. update rows p+32 .. k-1 (chunks prefetched one step ahead) ----------------
        for(int i0 = p + 32; i0 < k; i0 += kBsChunk)
        {
            store_chunk();
            __syncthreads();
            if(i0 + kBsChunk < k)
                fetch_chunk(p, i0 + kBsChunk);
            else
                fetch_diag(p + 32); // p + 32 < k here
            const int col = lane;
#pragma unroll
            for(int q = 0; q < kBsChunk / 8; ++q)
            {
                const int r = warp + 8 * q;
                T         acc = T(0);
#pragma unroll 8
                for(int t = 0; t < 32; ++t)
                    acc += Ps[r * 33 + t] * Cs[(p + t) * kBsPitch + col];
                if(i0 + r < kpad)
                    Cs[(i0 + r) * kBsPitch + col] -= acc;
            }
            __syncthreads();
        }
    }

    // ---- store Y (undo the row reversal) ---------------------------------------------------
    for(int idx = tid; idx < k * kBsW; idx += kBsThreads)
    {
        int r, col;
        if(side_left) { r = idx % k; col = idx / k; }
        else          { col = idx % kBsW; r = idx / kBsW; }
        if(col < W)
        {
            const int i = rev ? k - 1 - r : r;
            *baddr(r, col) = Cs[i * kBsPitch + col];
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kBsThreads) block_solve_kernel(BlockSolveParams<T> p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int batch = p.batch_base + blockIdx.y;
    const int ncols = p.side_left ? p.n : p.m; // columns of C
    const int s0    = blockIdx.x * kBsW;
    // alpha == 0 anywhere in the call means B := 0 with A unreferenced, also for the
    // sub-solves of the blocked path that would otherwise apply 1
    const T ua    = p.ualpha.get();
    const T alpha = ua == T(0) ? T(0) : (p.first ? ua : T(1));
    block_solve_strip<T>(p.A.get(batch), p.lda, p.B.get(batch), p.ldb, p.k, p.side_left, p.tM,
                         p.rev, p.unit, p.conj, alpha, s0, ncols, smem_raw);
}

} // namespace rb200
