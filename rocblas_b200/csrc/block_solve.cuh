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
//   2. forward substitution of the diagonal tile: for real types one warp solves it, one
//      column per lane held in registers, with the tile's entries broadcast from shared
//      memory; complex types, whose column would need too many registers, spread the columns
//      over the warps and broadcast each solved row value with __shfl_sync (the reference
//      broadcasts through LDS with two __syncthreads per row, :3225-3248);
//   3. rank-32 update of the remaining rows from panels of M streamed through shared
//      memory in 64-row chunks.
// k is at most kBlockSolveMaxK; larger systems use the blocked recursive path.
#pragma once
#include <type_traits>

#include "common.cuh"
#include "mma_f64.cuh"

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
__host__ __device__ constexpr int block_solve_max_k()
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

// Row pitches (elements) of the strip C and of the streamed panel chunk in shared memory.  FP64
// runs the update on DMMA, whose fragment reads (lanes (g, t) reading element (g, t) of the
// chunk and (t, g) of the solved rows) fall on distinct bank pairs of each half-warp with a
// pitch of 36; FP32 reads the chunk as float4, which a pitch of 36 keeps 16-byte aligned.
// Other types keep 33, which makes the column reads of the substitution conflict-free.
template <typename T>
__host__ __device__ constexpr int bs_cpitch()
{
    return std::is_same<T, double>::value ? 36 : kBsPitch;
}
template <typename T>
__host__ __device__ constexpr int bs_ppitch()
{
    return std::is_same<T, double>::value || std::is_same<T, float>::value ? 36 : kBsPitch;
}

template <typename T>
__host__ __device__ constexpr size_t block_solve_smem_bytes(int k)
{
    const int kpad = (int)ceil_div(k, 32) * 32;
    return sizeof(T) * (size_t)(kpad * bs_cpitch<T>() + 32 * 33 + 32 + kBsChunk * bs_ppitch<T>());
}

// FP64 update of one chunk on the tensor path: C[0:rows, 0:32] -= P[0:64, 0:32] X[0:32, 0:32]
// (P: the chunk of M, pitch 36; X: the solved panel rows and C: the rows below, pitch 36; rows
// >= `rows` do not exist and are not written).  Warp w owns rows 16 (w % 4) .. + 16 and columns
// 16 (w / 4) .. + 16: two mma.sync m16n8k8 tiles per 8-deep k step, 8 MMAs per warp.
__device__ __forceinline__ void bs_update_dmma(const double* Ps, const double* Xs, double* Cc,
                                               int rows, int warp, int lane)
{
    constexpr int P = 36;
    const int     wr = (warp & 3) * 16, wc = (warp >> 2) * 16;
    const int     g = lane >> 2, t = lane & 3;
    double        acc[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
#pragma unroll
    for(int ks = 0; ks < 32; ks += 8)
    {
        const double a[4] = {Ps[(wr + g) * P + ks + t], Ps[(wr + g + 8) * P + ks + t],
                             Ps[(wr + g) * P + ks + t + 4], Ps[(wr + g + 8) * P + ks + t + 4]};
#pragma unroll
        for(int j = 0; j < 2; ++j)
        {
            const double b[2] = {Xs[(ks + t) * P + wc + 8 * j + g], Xs[(ks + t + 4) * P + wc + 8 * j + g]};
            dmma_16x8x8(acc[j], a, b);
        }
    }
#pragma unroll
    for(int j = 0; j < 2; ++j)
#pragma unroll
        for(int e = 0; e < 4; ++e)
        {
            const int r = wr + g + (e >> 1) * 8, c = wc + 8 * j + 2 * t + (e & 1);
            if(r < rows)
                Cc[r * P + c] -= acc[j][e];
        }
}

// The core: solve M Y = alpha C for one strip.  The caller resolves pointers / sizes.
template <typename T>
__device__ void block_solve_strip(const T* A, int64_t lda, T* B, int64_t ldb, int k,
                                  int side_left, int tM, int rev, int unit, int conj, T alpha,
                                  int s0, int ncols, unsigned char* smem_raw)
{
    constexpr int PC = bs_cpitch<T>(), PP = bs_ppitch<T>();
    constexpr int NW = kBsThreads / 32; // warps
    T* Cs    = reinterpret_cast<T*>(smem_raw);
    const int kpad = ((k + 31) / 32) * 32;
    T* Ds    = Cs + kpad * PC;
    T* rdiag = Ds + 32 * 33;
    T* Ps    = rdiag + 32;

    const int tid  = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int W    = min(kBsW, ncols - s0); // valid columns of this strip

    // C(r, col) address in B: side L -> B[r + (s0+col) ldb]; side R -> B[(s0+col) + r ldb]
    T* const      B0  = B + (side_left ? (int64_t)s0 * ldb : (int64_t)s0);
    const int64_t bdr = side_left ? 1 : ldb, bdc = side_left ? ldb : 1;
    auto baddr = [&](int r, int col) -> T* { return B0 + r * bdr + col * bdc; };
    // M'(i, j), the reversed lower orientation of M (= A or A^T): with a = i, b = j (or k-1-i,
    // k-1-j when rev) it is A[a + b lda] (or A[b + a lda] when tM), i.e. M0[i dI + j dJ]
    const int64_t sgn = rev ? -1 : 1;
    const int64_t dI = (tM ? lda : 1) * sgn, dJ = (tM ? 1 : lda) * sgn;
    const T* const M0 = A + (rev ? (int64_t)(k - 1) * (1 + lda) : 0);
    auto mval = [&](int i, int j) -> T { return conj_if(M0[i * dI + j * dJ], conj); };

    // B is walked with lanes along its contiguous direction: rows of C for side L, columns of C
    // (rows of B) for side R
    if(alpha == T(0))
    {
        // B := 0 without reading A or B (rocblas_trsm_imp.hpp:154-157 semantics)
        if(side_left)
        {
            for(int col = warp; col < W; col += NW)
                for(int r = lane; r < k; r += 32)
                    *baddr(r, col) = T(0);
        }
        else
        {
            for(int r = warp; r < k; r += NW)
                if(lane < W)
                    *baddr(r, lane) = T(0);
        }
        return;
    }

    // ---- load alpha * C' (rows reversed when rev), zero-pad rows k..kpad-1 ----------------
    auto load_c = [&](int r, int col) {
        T v = T(0);
        if(r < k && col < W)
            v = alpha * (*baddr(r, col));
        const int i = (r < k && rev) ? k - 1 - r : r;
        Cs[i * PC + col] = v;
    };
    if(side_left)
    {
        for(int col = warp; col < kBsW; col += NW)
            for(int r = lane; r < kpad; r += 32)
                load_c(r, col);
    }
    else
    {
        for(int r = warp; r < kpad; r += NW)
            load_c(r, lane);
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
                {
                    // unit 1: a unit diagonal, not read; unit 2: read, and a zero entry
                    // counts as 1 (the trtri rule for singular matrices)
                    v = unit == 1 ? T(1) : mval(p + i, p + i);
                    if(unit == 2 && v == T(0))
                        v = T(1);
                }
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
            Ps[r * PP + t] = pre[u];
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

        // ---- 2. substitution of the 32 x 32 diagonal tile ------------------------------------
        // One warp, one column per lane held in registers: y_j *= 1/M_jj, then
        // y_i -= M_ij y_j for i > j (the reference's column order); M_ij is a shared-memory
        // broadcast.  Complex types (64 / 128 registers for the column) broadcast solved rows by
        // shuffle across all warps instead: warp w owns columns w, w+8, w+16, w+24, lane = row.
        if constexpr(!is_cplx<T>::value)
        {
            if(warp == 0)
            {
                T y[32];
#pragma unroll
                for(int i = 0; i < 32; ++i)
                    y[i] = Cs[(p + i) * PC + lane];
#pragma unroll
                for(int j = 0; j < 32; ++j)
                {
                    y[j] *= rdiag[j];
#pragma unroll
                    for(int i = j + 1; i < 32; ++i)
                        y[i] -= Ds[i * 33 + j] * y[j];
                }
#pragma unroll
                for(int i = 0; i < 32; ++i)
                    Cs[(p + i) * PC + lane] = y[i];
            }
        }
        else
        {
            T y[4];
#pragma unroll
            for(int q = 0; q < 4; ++q)
                y[q] = Cs[(p + lane) * PC + warp + 8 * q];
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
                Cs[(p + lane) * PC + warp + 8 * q] = y[q];
        }
        __syncthreads();

        // ---- 3. update rows p+32 .. k-1 (chunks prefetched one step ahead) ----------------
        // FP32 keeps this thread's column of the solved panel in registers for all chunks
        float xr[std::is_same<T, float>::value ? 32 : 1];
        if constexpr(std::is_same<T, float>::value)
        {
            if(p + 32 < k)
#pragma unroll
                for(int t = 0; t < 32; ++t)
                    xr[t] = Cs[(p + t) * PC + lane];
        }
        for(int i0 = p + 32; i0 < k; i0 += kBsChunk)
        {
            store_chunk();
            __syncthreads();
            if(i0 + kBsChunk < k)
                fetch_chunk(p, i0 + kBsChunk);
            else
                fetch_diag(p + 32); // p + 32 < k here
            if constexpr(std::is_same<T, double>::value)
            {
                bs_update_dmma(Ps, Cs + (size_t)p * PC, Cs + (size_t)i0 * PC, kpad - i0, warp, lane);
            }
            else if constexpr(std::is_same<T, float>::value)
            {
#pragma unroll
                for(int q = 0; q < kBsChunk / NW; ++q)
                {
                    const int r   = warp + NW * q;
                    float     acc = 0.0f;
#pragma unroll
                    for(int t = 0; t < 32; t += 4)
                    {
                        const float4 m4 = *reinterpret_cast<const float4*>(&Ps[r * PP + t]);
                        acc += m4.x * xr[t] + m4.y * xr[t + 1] + m4.z * xr[t + 2] + m4.w * xr[t + 3];
                    }
                    if(i0 + r < kpad)
                        Cs[(i0 + r) * PC + lane] -= acc;
                }
            }
            else
            {
                const int col = lane;
#pragma unroll
                for(int q = 0; q < kBsChunk / NW; ++q)
                {
                    const int r = warp + NW * q;
                    T         acc = T(0);
#pragma unroll 8
                    for(int t = 0; t < 32; ++t)
                        acc += Ps[r * PP + t] * Cs[(p + t) * PC + col];
                    if(i0 + r < kpad)
                        Cs[(i0 + r) * PC + col] -= acc;
                }
            }
            __syncthreads();
        }
    }

    // ---- store Y (undo the row reversal) ---------------------------------------------------
    auto store_y = [&](int r, int col) {
        if(col < W)
            *baddr(r, col) = Cs[(rev ? k - 1 - r : r) * PC + col];
    };
    if(side_left)
    {
        for(int col = warp; col < W; col += NW)
            for(int r = lane; r < k; r += 32)
                store_y(r, col);
    }
    else
    {
        for(int r = warp; r < k; r += NW)
            store_y(r, lane);
    }
}

template <typename T>
__global__ void __launch_bounds__(kBsThreads, 2) block_solve_kernel(BlockSolveParams<T> p)
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
