// Single right-hand side triangular solve, op(A) x = b (rocblas_?trsv with one vector), as a
// memory-bound kernel: the work is one read of A's triangle (n^2 / 2 elements) and the bound is
// HBM bandwidth, not arithmetic.
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
//     threads, one column each); after the tiles, the partial sums of the 8 warps meet in shared
//     memory and x_b = inv(M_bb) (b_b - sum) is one 64 x 64 product, so that the critical path
//     from one block's flag to the next is a tile product, a reduction and that product; the
//     CTA writes x_b, fences, and sets block b's flag.
// A wait that runs out records error 5 in the handle's error word and the CTA stops; the
// blocks after it then stop too (their waits run out), and the call reports the error through
// rocblas_b200_get_device_error.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace rb200
{

constexpr int kTvNB      = 64;  // rows per block
constexpr int kTvThreads = 256; // 8 warps
constexpr int kTvWarps   = kTvThreads / 32;

template <typename T>
struct TrsvParams
{
    const T*  A;
    int64_t   lda;
    T*        x;
    int64_t   incx; // > 0
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
__device__ __forceinline__ T* tv_x(const TrsvParams<T>& p, int rl)
{
    const int r = p.rev ? p.n - 1 - rl : rl;
    return p.x + (int64_t)r * p.incx;
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

template <typename T>
constexpr size_t trsv_flag_smem_bytes()
{
    return 2 * sizeof(T) * kTvNB * (kTvNB + 1);
}

template <typename T>
__global__ void __launch_bounds__(kTvThreads) trsv_flag_kernel(const TrsvParams<T> p)
{
    // the diagonal block and its inverse in dynamic shared memory (trsv_flag_smem_bytes)
    extern __shared__ __align__(16) unsigned char tv_smem[];
    T(*diag)[kTvNB + 1] = reinterpret_cast<T(*)[kTvNB + 1]>(tv_smem);
    T(*inv)[kTvNB + 1]  = reinterpret_cast<T(*)[kTvNB + 1]>(tv_smem + sizeof(T) * kTvNB * (kTvNB + 1));
    __shared__ T   part[kTvWarps][kTvNB];
    __shared__ T   ysh[kTvNB];
    __shared__ int stop;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nblk = (p.n + kTvNB - 1) / kTvNB;
    if(threadIdx.x == 0)
        stop = 0;
    __syncthreads();
    for(int b = blockIdx.x; b < nblk; b += gridDim.x)
    {
        const int r0 = b * kTvNB, rows = min(kTvNB, p.n - r0);
        // the diagonal block, staged before any wait (zero outside the triangle; rows past the
        // matrix get a unit diagonal so that the inverse below stays finite)
        for(int e = threadIdx.x; e < kTvNB * kTvNB; e += kTvThreads)
        {
            const int rr = e % kTvNB, cc = e / kTvNB;
            T v = (rr < rows && cc <= rr) ? tv_load(p, r0 + rr, r0 + cc) : T(0);
            if(rr == cc && (p.unit || rr >= rows))
                v = T(1);
            diag[rr][cc] = v;
        }
        __syncthreads();
        // its inverse, also before any wait (the wait on the block before is the critical path,
        // and after it only a product with the inverse remains): thread c < 64 solves
        // diag z = e_c by forward substitution (column c of the inverse; zero above the diagonal)
        if(threadIdx.x < kTvNB)
        {
            const int c = threadIdx.x;
            for(int r = 0; r < c; ++r)
                inv[r][c] = T(0);
            const T zc = T(1) / diag[c][c];
            inv[c][c]  = zc;
            for(int r = c + 1; r < kTvNB; ++r)
            {
                T s = T(0);
                for(int k = c; k < r; ++k)
                    s += diag[r][k] * inv[k][c];
                inv[r][c] = -s / diag[r][r];
            }
        }
        // this block's right-hand side, read before any wait (no other block writes it)
        const T xb = threadIdx.x < rows ? *tv_x(p, r0 + threadIdx.x) : T(0);
        // the tiles j < b: no-trans maps lanes to rows (2 each, columns warp, warp + 8, ..),
        // trans maps lanes to columns (2 each) and warps to rows (8 each)
        T    acc[8];
#pragma unroll
        for(int q = 0; q < 8; ++q)
            acc[q] = T(0);
        bool ok = true;
        for(int j = 0; j < b && ok; ++j)
        {
            const int c0 = j * kTvNB; // a full block: j < b
            T         a[16];
            if(!p.trans)
            {
#pragma unroll
                for(int q = 0; q < 8; ++q)
                {
                    const int cc = c0 + warp + q * kTvWarps;
                    a[2 * q]     = lane < rows ? tv_load(p, r0 + lane, cc) : T(0);
                    a[2 * q + 1] = lane + 32 < rows ? tv_load(p, r0 + lane + 32, cc) : T(0);
                }
            }
            else
            {
#pragma unroll
                for(int q = 0; q < 8; ++q)
                {
                    const int rr = warp + q * kTvWarps;
                    a[2 * q]     = rr < rows ? tv_load(p, r0 + rr, c0 + lane) : T(0);
                    a[2 * q + 1] = rr < rows ? tv_load(p, r0 + rr, c0 + lane + 32) : T(0);
                }
            }
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
            if(!p.trans)
            {
#pragma unroll
                for(int q = 0; q < 8; ++q)
                {
                    const T xv = __ldcg(tv_x(p, c0 + warp + q * kTvWarps));
                    acc[0] += a[2 * q] * xv;
                    acc[1] += a[2 * q + 1] * xv;
                }
            }
            else
            {
                const T x0 = __ldcg(tv_x(p, c0 + lane)), x1 = __ldcg(tv_x(p, c0 + lane + 32));
#pragma unroll
                for(int q = 0; q < 8; ++q)
                    acc[q] += a[2 * q] * x0 + a[2 * q + 1] * x1;
            }
        }
        if(!ok)
        {
            if(lane == 0)
            {
                atomicCAS(p.error, 0, 5);
                atomicExch(&stop, 1);
            }
        }
        // partial sums of the 8 warps into part[warp][row]
        if(!p.trans)
        {
            part[warp][lane]      = acc[0];
            part[warp][lane + 32] = acc[1];
        }
        else
        {
#pragma unroll
            for(int q = 0; q < 8; ++q)
            {
                T v = acc[q];
#pragma unroll
                for(int off = 16; off; off >>= 1)
                    v += __shfl_xor_sync(0xffffffffu, v, off);
                if(lane == 0)
                {
                    // row warp + 8 q: one warp owns each row, the others contribute zero
                    const int rr = warp + q * kTvWarps;
                    for(int w = 0; w < kTvWarps; ++w)
                        part[w][rr] = w == warp ? v : T(0);
                }
            }
        }
        __syncthreads();
        if(*(volatile int*)&stop)
            break;
        // y = b - sum, then x_b = inv y, by the first 64 threads (named barrier 1 between them:
        // the other warps go on to stage the CTA's next block once the barrier below lets them)
        if(threadIdx.x < kTvNB)
        {
            const int rr = threadIdx.x;
            T         s  = T(0);
#pragma unroll
            for(int w = 0; w < kTvWarps; ++w)
                s += part[w][rr];
            ysh[rr] = xb - s;
            asm volatile("bar.sync 1, %0;" ::"n"(kTvNB) : "memory");
            T v = T(0);
            for(int cc = 0; cc <= rr; ++cc)
                v += inv[rr][cc] * ysh[cc];
            if(rr < rows)
                *tv_x(p, r0 + rr) = v;
            __threadfence();
            asm volatile("bar.sync 1, %0;" ::"n"(kTvNB) : "memory");
            if(rr == 0)
                asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p.flags + b), "r"(1) : "memory");
        }
        __syncthreads(); // diag and part are reused by the CTA's next block
    }
}

} // namespace rb200
