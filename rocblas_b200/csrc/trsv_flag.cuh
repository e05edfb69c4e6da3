// Triangular solve of one or a few right-hand sides, op(A) x_v = alpha b_v (rocblas_?trsv with
// one vector; up to 8 vectors for the refined form's test solve), as a memory-bound kernel: the
// work is one read of A's triangle (n^2 / 2 elements) for all of them and the bound is HBM
// bandwidth, not arithmetic.
//
// The reference solves it with its own flag-synchronised substitution
// (library/src/blas2/rocblas_trsv_kernels.cpp:461-775).  Here:
//   * logical indices turn every uplo / trans into a forward solve of a lower triangle:
//     logical row r' is physical row r = rev ? n - 1 - r' : r' (rev when op(A) is upper), and
//     M(r', c') = op(A)(r, c), so that M is lower triangular in logical indices;
//   * rows are cut into blocks of kTvNB; a persistent grid (every CTA resident) gives block b
//     to CTA b % gridDim.x, and a CTA takes its blocks in increasing order, so every block only
//     waits on blocks that are done or in progress, and the solve cannot deadlock;
//   * for block b a CTA streams the tiles M(b, j), j < b: it issues a tile's loads of A, then
//     waits (bounded) for block j's flag, then reads x_j (bypassing L1) and accumulates; the
//     tiles of finished blocks stream at full speed and only the last ones wait;
//   * before any wait the CTA stages its diagonal block in shared memory and inverts it (64
//     threads per 64-row half, one column each); after the tiles, the partial sums of the 8
//     warps meet in shared memory and x_b = inv(M_bb) (alpha b_b - sum) is one product with the
//     inverse per right-hand side, so that the critical path from one block's flag to the next
//     is a tile product, a reduction and that product; the CTA writes x_b, fences, and sets
//     block b's flag.
// A wait that runs out records error 5 in the handle's error word and the CTA stops; the
// blocks after it then stop too (their waits run out), and the call reports the error through
// rocblas_b200_get_device_error.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace rb200
{

constexpr int kTvNB      = 64;  // rows per 64-row block (the inverse is built from blocks of this)
constexpr int kTvThreads = 256; // 8 warps
constexpr int kTvWarps   = kTvThreads / 32;

template <typename T>
struct TrsvParams
{
    const T*  A;
    int64_t   lda;
    T*        x;
    int64_t   incx; // > 0
    int64_t   ldx;  // distance between the right-hand sides (nrhs > 1)
    int       nrhs; // right-hand sides, 1 .. the kernel's NR
    T         alpha; // op(A) x_v = alpha b_v (1 for trsv)
    int       n;
    int       rev;   // op(A) is upper: the solve runs from the last row
    int       trans; // op(A) = A^T (A^H reads the same for real types)
    int       unit;
    int*      flags; // one per block, zero on entry
    int*      error;
    long long wait_cycles;
};

template <typename T>
__device__ __forceinline__ T tv_load(const TrsvParams<T>& p, int rl, int cl)
{
    const int r = p.rev ? p.n - 1 - rl : rl, c = p.rev ? p.n - 1 - cl : cl;
    return p.trans ? p.A[c + (int64_t)r * p.lda] : p.A[r + (int64_t)c * p.lda];
}

template <typename T>
__device__ __forceinline__ T* tv_x(const TrsvParams<T>& p, int rl, int v = 0)
{
    const int r = p.rev ? p.n - 1 - rl : rl;
    return p.x + (int64_t)v * p.ldx + (int64_t)r * p.incx;
}

// bounded wait for block j's flag (acquire); false when it ran out
__device__ __forceinline__ bool tv_wait_flag(const int* flag, long long limit)
{
    const long long t0 = clock64();
    int             v;
    while(true)
    {
        asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if(v)
            return true;
        if(clock64() - t0 > limit)
            return false;
        __nanosleep(64);
    }
}

// Dynamic shared memory of the NB-row kernel with NR right-hand sides: the diagonal block
// (NB x NB + 1; for NB = 128 its inverse in place), 64 x 65 scratch blocks for the inverses of its
// 64-row halves (one for NB = 64, where it holds the inverse, two for NB = 128) and the 8 warps'
// partial sums (8 x NR x NB; for NB = 128 over the two scratch blocks, free by then).
template <typename T, int NB, int NR = 1>
constexpr size_t trsv_flag_smem_bytes()
{
    return sizeof(T) * ((size_t)NB * (NB + 1) + (NB / kTvNB) * kTvNB * (kTvNB + 1)
                        + (NB == 64 ? (size_t)kTvWarps * NR * NB : 0));
}

// inverse of the lower-triangular 64 x 64 block S (stride ls) into D (stride ld), zero above the
// diagonal: thread c < 64 of the calling group solves S z = e_c by forward substitution
template <typename T>
__device__ __forceinline__ void tv_invert64(const T* S, int ls, T* D, int ld, int c)
{
    for(int r = 0; r < c; ++r)
        D[r * ld + c] = T(0);
    D[c * ld + c] = T(1) / S[c * ls + c];
    for(int r = c + 1; r < kTvNB; ++r)
    {
        T acc = T(0);
        for(int k = c; k < r; ++k)
            acc += S[r * ls + k] * D[k * ld + c];
        D[r * ld + c] = -acc / S[r * ls + r];
    }
}

// TR: -1 takes op(A)'s transposition from p.trans; 0 / 1 fix it at compile time (fewer
// registers: the accumulators of one layout only).
template <typename T, int NB, int NR = 1, int TR = -1>
__global__ void __launch_bounds__(kTvThreads) trsv_flag_kernel(const TrsvParams<T> p)
{
    static_assert(NB == 64 || NB == 128, "block rows");
    static_assert(NR >= 1 && NR <= 8, "right-hand sides");
    static_assert(NB == 64 || kTvWarps * NR * NB <= 2 * kTvNB * (kTvNB + 1), "partial sums fit the scratch");
    constexpr int RPL = NB / 32;          // no-trans: rows per lane
    constexpr int CPW = kTvNB / kTvWarps; // columns per warp in a 64-column half tile
    constexpr int RPW = NB / kTvWarps;    // trans: rows per warp
    constexpr int LD  = NB + 1;
    constexpr int NACC = TR == 0 ? RPL : TR == 1 ? RPW : (RPL > RPW ? RPL : RPW);
    const bool    trans = TR < 0 ? p.trans != 0 : TR == 1;
    constexpr int G    = kTvThreads / NB;   // right-hand-side groups of the final product
    constexpr int VPT  = (NR + G - 1) / G;  // right-hand sides per thread in it
    extern __shared__ __align__(16) unsigned char tv_smem[];
    T* dg = reinterpret_cast<T*>(tv_smem); // diagonal block, then its inverse in place
    T* s1 = dg + NB * LD;                  // NB = 128: inverses of the two 64-row halves
    T* s2 = s1 + kTvNB * (kTvNB + 1);
    // partial sums [warp][v][row]: NB = 128 over s1 / s2 (dead once the inverse is assembled),
    // NB = 64 after s1
    T* part = NB == 128 ? s1 : s1 + kTvNB * (kTvNB + 1);
    __shared__ T   ysh[NR][NB];
    __shared__ int stop;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nblk = (p.n + NB - 1) / NB;
    const int fr = threadIdx.x % NB, fg = threadIdx.x / NB; // final product: row, group
    if(threadIdx.x == 0)
        stop = 0;
    __syncthreads();
    for(int b = blockIdx.x; b < nblk; b += gridDim.x)
    {
        const int r0 = b * NB, rows = min(NB, p.n - r0);
        // the diagonal block, staged before any wait (zero outside the triangle; rows past the
        // matrix get a unit diagonal so that the inverse stays finite)
        for(int e = threadIdx.x; e < NB * NB; e += kTvThreads)
        {
            const int rr = e % NB, cc = e / NB;
            T v = (rr < rows && cc <= rr) ? tv_load(p, r0 + rr, r0 + cc) : T(0);
            if(rr == cc && (p.unit || rr >= rows))
                v = T(1);
            dg[rr * LD + cc] = v;
        }
        // this block's right-hand sides, read before any wait (no other block writes them)
        T xb[VPT];
#pragma unroll
        for(int i = 0; i < VPT; ++i)
        {
            const int v = fg + G * i;
            xb[i] = (fr < rows && v < NR && v < p.nrhs) ? *tv_x(p, r0 + fr, v) : T(0);
        }
        __syncthreads();
        // its inverse, also before any wait: after the wait on the block before (the critical
        // path) only a product with it remains
        if constexpr(NB == 64)
        {
            if(threadIdx.x < kTvNB)
                tv_invert64(dg, LD, s1, kTvNB + 1, threadIdx.x);
        }
        else
        {
            // [[L11, 0], [L21, L22]]^-1 = [[I11, 0], [-I22 L21 I11, I22]] with I = inverses of the
            // 64-row halves: threads 0..63 invert L11 into s1, threads 64..127 L22 into s2
            if(threadIdx.x < kTvNB)
                tv_invert64(dg, LD, s1, kTvNB + 1, threadIdx.x);
            else if(threadIdx.x < 2 * kTvNB)
                tv_invert64(dg + kTvNB * LD + kTvNB, LD, s2, kTvNB + 1, threadIdx.x - kTvNB);
            __syncthreads();
            // W = L21 I11 (64 x 64, 16 entries per thread), written over L21
            T w[16];
#pragma unroll
            for(int q = 0; q < 16; ++q)
            {
                const int e = threadIdx.x + q * kTvThreads, rr = e % kTvNB, cc = e / kTvNB;
                T         acc = T(0);
                for(int k = cc; k < kTvNB; ++k)
                    acc += dg[(kTvNB + rr) * LD + k] * s1[k * (kTvNB + 1) + cc];
                w[q] = acc;
            }
            __syncthreads();
#pragma unroll
            for(int q = 0; q < 16; ++q)
            {
                const int e = threadIdx.x + q * kTvThreads, rr = e % kTvNB, cc = e / kTvNB;
                dg[(kTvNB + rr) * LD + cc] = w[q];
            }
            __syncthreads();
            // -I22 W over the lower-left block, then the half inverses on the diagonal
#pragma unroll
            for(int q = 0; q < 16; ++q)
            {
                const int e = threadIdx.x + q * kTvThreads, rr = e % kTvNB, cc = e / kTvNB;
                T         acc = T(0);
                for(int k = 0; k <= rr; ++k)
                    acc += s2[rr * (kTvNB + 1) + k] * dg[(kTvNB + k) * LD + cc];
                w[q] = -acc;
            }
            __syncthreads();
#pragma unroll
            for(int q = 0; q < 16; ++q)
            {
                const int e = threadIdx.x + q * kTvThreads, rr = e % kTvNB, cc = e / kTvNB;
                dg[(kTvNB + rr) * LD + cc] = w[q];
                dg[rr * LD + cc]                   = s1[rr * (kTvNB + 1) + cc];
                dg[(kTvNB + rr) * LD + kTvNB + cc] = s2[rr * (kTvNB + 1) + cc];
                dg[rr * LD + kTvNB + cc]           = T(0);
            }
        }
        // the tiles j < b, in 64-column halves: no-trans maps lanes to rows (RPL each) and warps
        // to columns (8 of each half), trans maps lanes to columns (2 of each half) and warps to
        // rows (RPW each)
        T acc[NR][NACC];
#pragma unroll
        for(int v = 0; v < NR; ++v)
#pragma unroll
            for(int q = 0; q < NACC; ++q)
                acc[v][q] = T(0);
        bool ok = true;
        for(int j = 0; j < b && ok; ++j)
        {
            for(int hf = 0; hf < NB / kTvNB; ++hf)
            {
                const int c0 = j * NB + hf * kTvNB; // a full block: j < b
                constexpr int kAv = TR == 0 ? RPL * CPW : TR == 1 ? 2 * RPW : (RPL * CPW > 2 * RPW ? RPL * CPW : 2 * RPW);
                T             av[kAv];
                if(!trans)
                {
                    if constexpr(TR != 1)
                    {
#pragma unroll
                        for(int q = 0; q < CPW; ++q)
#pragma unroll
                            for(int t = 0; t < RPL; ++t)
                            {
                                const int rr = lane + 32 * t;
                                av[q * RPL + t] = rr < rows ? tv_load(p, r0 + rr, c0 + warp + q * kTvWarps) : T(0);
                            }
                    }
                }
                else
                {
                    if constexpr(TR != 0)
                    {
#pragma unroll
                        for(int q = 0; q < RPW; ++q)
                        {
                            const int rr = warp + q * kTvWarps;
                            av[2 * q]     = rr < rows ? tv_load(p, r0 + rr, c0 + lane) : T(0);
                            av[2 * q + 1] = rr < rows ? tv_load(p, r0 + rr, c0 + lane + 32) : T(0);
                        }
                    }
                }
                if(hf == 0)
                {
                    // x_j is final once block j's flag is set
                    int bad = 0;
                    if(lane == 0)
                        bad = (*(volatile int*)&stop) || !tv_wait_flag(p.flags + j, p.wait_cycles);
                    bad = __shfl_sync(0xffffffffu, bad, 0);
                    __syncwarp(); // lane 0's acquire orders the whole warp's reads of x_j below
                    if(bad)
                    {
                        ok = false;
                        break;
                    }
                }
                if(!trans)
                {
                    if constexpr(TR != 1)
                    {
#pragma unroll
                        for(int q = 0; q < CPW; ++q)
#pragma unroll
                            for(int v = 0; v < NR; ++v)
                            {
                                const T xv = v < p.nrhs ? __ldcg(tv_x(p, c0 + warp + q * kTvWarps, v)) : T(0);
#pragma unroll
                                for(int t = 0; t < RPL; ++t)
                                    acc[v][t] += av[q * RPL + t] * xv;
                            }
                    }
                }
                else
                {
                    if constexpr(TR != 0)
                    {
#pragma unroll
                        for(int v = 0; v < NR; ++v)
                        {
                            const bool live = v < p.nrhs;
                            const T    x0   = live ? __ldcg(tv_x(p, c0 + lane, v)) : T(0);
                            const T    x1   = live ? __ldcg(tv_x(p, c0 + lane + 32, v)) : T(0);
#pragma unroll
                            for(int q = 0; q < RPW; ++q)
                                acc[v][q] += av[2 * q] * x0 + av[2 * q + 1] * x1;
                        }
                    }
                }
            }
        }
        if(!ok && lane == 0)
        {
            atomicCAS(p.error, 0, 5);
            atomicExch(&stop, 1);
        }
        __syncthreads(); // NB = 128: the partial sums reuse the inverse's scratch
        // partial sums into part[warp][v][row] (trans: only warp 0's slots, one warp owns a row)
        if(!trans)
        {
            if constexpr(TR != 1)
            {
#pragma unroll
                for(int v = 0; v < NR; ++v)
#pragma unroll
                    for(int t = 0; t < RPL; ++t)
                        part[(warp * NR + v) * NB + lane + 32 * t] = acc[v][t];
            }
        }
        else
        {
            if constexpr(TR != 0)
            {
#pragma unroll
                for(int v = 0; v < NR; ++v)
#pragma unroll
                    for(int q = 0; q < RPW; ++q)
                    {
                        T s = acc[v][q];
#pragma unroll
                        for(int off = 16; off; off >>= 1)
                            s += __shfl_xor_sync(0xffffffffu, s, off);
                        if(lane == 0)
                            part[v * NB + warp + q * kTvWarps] = s;
                    }
            }
        }
        __syncthreads();
        if(*(volatile int*)&stop)
            break;
        // y = alpha b - sum, then x_b = inv y: thread (row fr, group fg) takes the right-hand
        // sides fg, fg + G, ...
        const int nw = trans ? 1 : kTvWarps;
#pragma unroll
        for(int i = 0; i < VPT; ++i)
        {
            const int v = fg + G * i;
            if(v < NR)
            {
                T sum = T(0);
                for(int w = 0; w < nw; ++w)
                    sum += part[(w * NR + v) * NB + fr];
                ysh[v][fr] = p.alpha * xb[i] - sum;
            }
        }
        __syncthreads();
        {
            // the inverse: s1 (stride 65) for NB = 64, the block itself for NB = 128
            const T*  inv = NB == 64 ? s1 : dg;
            const int li  = NB == 64 ? kTvNB + 1 : LD;
            T         out[VPT];
#pragma unroll
            for(int i = 0; i < VPT; ++i)
                out[i] = T(0);
            if(fg < NR)
                for(int cc = 0; cc <= fr; ++cc)
                {
                    const T a = inv[fr * li + cc];
#pragma unroll
                    for(int i = 0; i < VPT; ++i)
                        if(fg + G * i < NR)
                            out[i] += a * ysh[fg + G * i][cc];
                }
#pragma unroll
            for(int i = 0; i < VPT; ++i)
            {
                const int v = fg + G * i;
                if(fr < rows && v < NR && v < p.nrhs)
                    *tv_x(p, r0 + fr, v) = out[i];
            }
        }
        __threadfence();
        __syncthreads();
        if(threadIdx.x == 0)
            asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p.flags + b), "r"(1) : "memory");
        __syncthreads(); // the buffers are reused by the CTA's next block
    }
}

} // namespace rb200
