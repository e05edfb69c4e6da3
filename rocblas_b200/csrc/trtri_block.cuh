// Inversion of the diagonal blocks of a triangular matrix, one CTA per block of up to 128.
//
// Replaces the reference's invA construction for TRSM (rocblas_trtri_trsm_template,
// library/src/blas3/trtri_trsm.hpp:110-381: 16x16 trtri kernels, three rounds of
// strided-batched GEMM merges 32->64->128, a separate fill kernel for the unused
// triangle and a remainder trtri) with a single fused kernel: the block (at most 128 x 128)
// is staged in shared memory as 4 x 4 tiles of 32 x 32 (lower orientation; an upper block U
// is handled as the lower block J U J, J the exchange matrix), the four diagonal tiles are
// inverted by four warps (lane = column, substitution in registers, A entries broadcast
// from shared memory), and the off-diagonal tiles follow by diagonal distance d = 1, 2, 3:
//     X(i,j) = -X(i,i) * sum_{t=j}^{i-1} L(i,t) X(t,j).
// The result, with zeros in the opposite triangle (what rocblas_trtri_fill does,
// rocblas_trtri.hpp:393-426), is written to invA.
//
// Diagonal semantics follow rocblas_custom_trtri_device (rocblas_trtri.hpp:128-141):
// diag == unit reads no diagonal and uses 1; a zero non-unit diagonal entry is treated as 1.
#pragma once
#include <type_traits>

#include "common.cuh"
#include "mma_f64.cuh"

namespace rb200
{

template <typename T>
struct TrtriParams
{
    int         k;            // order of A (the blocks tile A's diagonal)
    int         nb;           // block order (<= 128)
    BatchPtr<T> A;            // A(0,0) of every batch entry
    int64_t     lda;
    BatchPtr<T> inv;          // block b of batch entry e goes to inv.get(e) + b * inv_block_stride
    int64_t     ldinv;
    int64_t     inv_block_stride;
    int         upper, unit;
    int         batch_base;
    // variable batch: order and leading dimension per entry (A and inv then come from
    // pointer arrays); blocks beyond an entry's order exit at once
    const int*     vk   = nullptr;
    const int64_t* vlda = nullptr;
};

constexpr int kTrtriNB      = 128;
constexpr int kTrtriSB      = 32;  // tile order
constexpr int kTrtriNT      = 4;   // tiles per side
constexpr int kTrtriNTiles  = kTrtriNT * (kTrtriNT + 1) / 2; // 10 lower tiles
constexpr int kTrtriThreads = 256;

// Tile row pitch in shared memory: 33 keeps the column reads of the FMA products
// conflict-free; FP64 runs the products on DMMA, whose fragment reads (lanes (g, t) reading
// (g, t) of the left tile and (t, g) of the right one) need a pitch of 4 mod 16.
template <typename T>
__host__ __device__ constexpr int trtri_pitch()
{
    return std::is_same<T, double>::value ? 36 : 33;
}
template <typename T>
__host__ __device__ constexpr int trtri_tile()
{
    return kTrtriSB * trtri_pitch<T>();
}

template <typename T>
constexpr size_t trtri_smem_bytes()
{
    // L tiles, X tiles, 3 temporaries, reciprocal diagonal
    return sizeof(T) * (size_t)(2 * kTrtriNTiles * trtri_tile<T>() + 3 * trtri_tile<T>() + kTrtriNB);
}

// acc (the 16 x 8 block of warp (wr, wc) of a 32 x 32 tile product) += Lt Rt, FP64 DMMA.
__device__ __forceinline__ void trtri_tile_mma(double (&acc)[4], const double* Lt, const double* Rt,
                                               int wr, int wc, int g, int t)
{
    constexpr int P = 36;
#pragma unroll
    for(int ks = 0; ks < kTrtriSB; ks += 8)
    {
        const double a[4] = {Lt[(wr + g) * P + ks + t], Lt[(wr + g + 8) * P + ks + t],
                             Lt[(wr + g) * P + ks + t + 4], Lt[(wr + g + 8) * P + ks + t + 4]};
        const double b[2] = {Rt[(ks + t) * P + wc + g], Rt[(ks + t + 4) * P + wc + g]};
        dmma_16x8x8(acc, a, b);
    }
}

__device__ __forceinline__ int trtri_tile_index(int bi, int bj)
{
    return bi * (bi + 1) / 2 + bj;
}

template <typename T>
__global__ void __launch_bounds__(kTrtriThreads) trtri_block_kernel(TrtriParams<T> p)
{
    constexpr int kTrtriPitch = trtri_pitch<T>(), kTrtriTile = trtri_tile<T>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* Ls    = reinterpret_cast<T*>(smem_raw);
    T* Xs    = Ls + kTrtriNTiles * kTrtriTile;
    T* Ts    = Xs + kTrtriNTiles * kTrtriTile;
    T* rdiag = Ts + 3 * kTrtriTile;

    const int     tid   = threadIdx.x;
    const int     blk   = blockIdx.x;
    const int     batch = p.batch_base + blockIdx.y;
    const int     k     = p.vk ? p.vk[batch] : p.k;
    const int64_t lda   = p.vk ? p.vlda[batch] : p.lda;
    const int     r0    = blk * p.nb;
    if(r0 >= k)
        return; // (variable batch) this entry has fewer blocks
    const int bs = min(p.nb, k - r0);

    const T* A   = p.A.get(batch) + r0 + (int64_t)r0 * lda;
    T*       out = p.inv.get(batch) + (int64_t)blk * p.inv_block_stride;

    // ---- stage the block in lower orientation, identity-padded to 128 ----------------
    // The 10 lower 32 x 32 tiles, 40 elements per thread, row index fastest so that a lower
    // block is read down its columns; loads are issued 8 at a time before their stores.
    {
        constexpr int kPer = kTrtriNTiles * kTrtriSB * kTrtriSB / kTrtriThreads; // 40
        constexpr int kBatch = 8;
        static_assert(kPer % kBatch == 0, "staging batches");
        auto coords = [&](int e, int& tl, int& i, int& j) {
            tl = e >> 10; // tile in trtri_tile_index order
            int bi = 0;
            while(trtri_tile_index(bi + 1, 0) <= tl)
                ++bi;
            const int bj = tl - trtri_tile_index(bi, 0);
            i = bi * kTrtriSB + (e & 31);
            j = bj * kTrtriSB + ((e >> 5) & 31);
        };
#pragma unroll 1
        for(int u0 = 0; u0 < kPer; u0 += kBatch)
        {
            T v[kBatch];
#pragma unroll
            for(int u = 0; u < kBatch; ++u)
            {
                int tl, i, j;
                coords(tid + (u0 + u) * kTrtriThreads, tl, i, j);
                v[u] = T(0);
                if(j <= i && i < bs && j < bs && !(i == j && p.unit))
                {
                    const int r = p.upper ? bs - 1 - i : i;
                    const int c = p.upper ? bs - 1 - j : j;
                    v[u] = A[r + (int64_t)c * lda];
                }
            }
#pragma unroll
            for(int u = 0; u < kBatch; ++u)
            {
                int tl, i, j;
                coords(tid + (u0 + u) * kTrtriThreads, tl, i, j);
                T x = v[u];
                if(i == j)
                {
                    // unit diagonal, identity padding, and a zero diagonal entry read as 1
                    if(p.unit || i >= bs || x == T(0))
                        x = T(1);
                    rdiag[i] = T(1) / x;
                }
                Ls[tl * kTrtriTile + (i % kTrtriSB) * kTrtriPitch + (j % kTrtriSB)] = x;
            }
        }
    }
    __syncthreads();

    // ---- invert the four diagonal tiles: warp w < 4 takes tile w, lane = column -------
    {
        const int w = tid >> 5, lane = tid & 31;
        if(w < kTrtriNT)
        {
            const T* L = Ls + trtri_tile_index(w, w) * kTrtriTile;
            T        x[kTrtriSB];
#pragma unroll
            for(int i = 0; i < kTrtriSB; ++i)
                x[i] = (i == lane) ? T(1) : T(0);
#pragma unroll
            for(int t = 0; t < kTrtriSB; ++t)
            {
                x[t] *= rdiag[w * kTrtriSB + t];
#pragma unroll
                for(int i = t + 1; i < kTrtriSB; ++i)
                    x[i] -= L[i * kTrtriPitch + t] * x[t];
            }
            T* X = Xs + trtri_tile_index(w, w) * kTrtriTile;
#pragma unroll
            for(int i = 0; i < kTrtriSB; ++i)
                X[i * kTrtriPitch + lane] = x[i];
        }
    }
    __syncthreads();

    // ---- off-diagonal tiles by distance d ------------------------------------------------
    const int c  = tid & 31;   // tile column handled by this thread
    const int rb = tid >> 5;   // rows rb, rb+8, rb+16, rb+24
    if constexpr(std::is_same<T, double>::value)
    {
        // FP64: both products on DMMA, warp w owns the 16 x 8 block at rows 16 (w % 2),
        // columns 8 (w / 2) of each 32 x 32 tile
        const int lane = tid & 31, w = tid >> 5, g = lane >> 2, t = lane & 3;
        const int wr = (w & 1) * 16, wc = (w >> 1) * 8;
        for(int d = 1; d < kTrtriNT; ++d)
        {
            const int npairs = kTrtriNT - d;
            for(int pr = 0; pr < npairs; ++pr)
            {
                const int bj = pr, bi = pr + d;
                double    acc[4] = {0.0, 0.0, 0.0, 0.0};
                for(int bt = bj; bt < bi; ++bt)
                    trtri_tile_mma(acc, Ls + trtri_tile_index(bi, bt) * kTrtriTile,
                                   Xs + trtri_tile_index(bt, bj) * kTrtriTile, wr, wc, g, t);
#pragma unroll
                for(int e = 0; e < 4; ++e)
                    Ts[pr * kTrtriTile + (wr + g + (e >> 1) * 8) * kTrtriPitch + wc + 2 * t + (e & 1)]
                        = acc[e];
            }
            __syncthreads();
            for(int pr = 0; pr < npairs; ++pr)
            {
                const int bj = pr, bi = pr + d;
                double    acc[4] = {0.0, 0.0, 0.0, 0.0};
                trtri_tile_mma(acc, Xs + trtri_tile_index(bi, bi) * kTrtriTile, Ts + pr * kTrtriTile,
                               wr, wc, g, t);
                T* Xo = Xs + trtri_tile_index(bi, bj) * kTrtriTile;
#pragma unroll
                for(int e = 0; e < 4; ++e)
                    Xo[(wr + g + (e >> 1) * 8) * kTrtriPitch + wc + 2 * t + (e & 1)] = -acc[e];
            }
            __syncthreads();
        }
    }
    else
    for(int d = 1; d < kTrtriNT; ++d)
    {
        const int npairs = kTrtriNT - d;
        // T_p = sum_{t=j}^{i-1} L(i,t) X(t,j),   (i, j) = (j + d, j), j = p
        for(int pr = 0; pr < npairs; ++pr)
        {
            const int bj = pr, bi = pr + d;
            T         acc[4] = {T(0), T(0), T(0), T(0)};
            for(int bt = bj; bt < bi; ++bt)
            {
                const T* L = Ls + trtri_tile_index(bi, bt) * kTrtriTile;
                const T* X = Xs + trtri_tile_index(bt, bj) * kTrtriTile;
#pragma unroll 8
                for(int kk = 0; kk < kTrtriSB; ++kk)
                {
                    const T xv = X[kk * kTrtriPitch + c];
#pragma unroll
                    for(int q = 0; q < 4; ++q)
                        acc[q] += L[(rb + 8 * q) * kTrtriPitch + kk] * xv;
                }
            }
#pragma unroll
            for(int q = 0; q < 4; ++q)
                Ts[pr * kTrtriTile + (rb + 8 * q) * kTrtriPitch + c] = acc[q];
        }
        __syncthreads();
        // X(i,j) = -X(i,i) T_p
        for(int pr = 0; pr < npairs; ++pr)
        {
            const int bj = pr, bi = pr + d;
            const T*  Xd = Xs + trtri_tile_index(bi, bi) * kTrtriTile;
            const T*  Tp = Ts + pr * kTrtriTile;
            T         acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll 8
            for(int kk = 0; kk < kTrtriSB; ++kk)
            {
                const T tv = Tp[kk * kTrtriPitch + c];
#pragma unroll
                for(int q = 0; q < 4; ++q)
                    acc[q] += Xd[(rb + 8 * q) * kTrtriPitch + kk] * tv;
            }
            T* Xo = Xs + trtri_tile_index(bi, bj) * kTrtriTile;
#pragma unroll
            for(int q = 0; q < 4; ++q)
                Xo[(rb + 8 * q) * kTrtriPitch + c] = -acc[q];
        }
        __syncthreads();
    }

    // ---- write inv(A_block) (bs x bs, ld = ldinv), zeros in the opposite triangle ----
    for(int idx = tid; idx < bs * bs; idx += kTrtriThreads)
    {
        const int i = idx % bs, j = idx / bs;
        // lower-orientation coordinates
        const int li = p.upper ? bs - 1 - i : i;
        const int lj = p.upper ? bs - 1 - j : j;
        T         v  = T(0);
        if(li >= lj)
            v = Xs[trtri_tile_index(li / kTrtriSB, lj / kTrtriSB) * kTrtriTile
                   + (li % kTrtriSB) * kTrtriPitch + (lj % kTrtriSB)];
        out[i + (int64_t)j * p.ldinv] = v;
    }
}

} // namespace rb200
