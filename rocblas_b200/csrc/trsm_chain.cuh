// Left-looking blocked TRSM in one persistent launch (a dependency chain over the 128-row
// blocks of the triangle), for few right-hand sides per system.
//
// The reference's left-looking path (special_trsm_template,
// library/src/blas3/rocblas_trsm_kernels.hpp:1164-1456) walks the diagonal blocks on the
// host: per 128-row block j one GEMM tmp = alpha B_j - A_{j,<j} X_{<j} and one GEMM
// X_j = invA_jj tmp, two launches per block.  With few right-hand sides every launch is
// small, so the solve is bound by launch latency.  Here one launch does the whole solve:
//
//   * work items are (system, block j in solve order, strip of W right-hand sides); a CTA
//     claims items from a device-side counter in increasing id order, id = (system * nb + j)
//     * ns + strip, so every item an item depends on (same system and strip, earlier block)
//     was claimed before it by a CTA that is running.  The earliest unfinished claimed item
//     therefore never waits on an unfinished one: no deadlock, whatever the residency;
//   * an item accumulates M_{b,i} X_i over the finished blocks i in solve order through a
//     cp.async pipeline of 16-deep K chunks on DMMA (mma.sync m16n8k8 f64), waiting on a
//     block's flag (ld.acquire.gpu by one thread, then a CTA barrier) before its first chunk;
//   * then T = alpha C_b - acc goes to shared memory, X_b = inv(M_bb) T (the caller's or the
//     fused trtri's invA block, its triangle masked) is written over C_b, and the block's
//     flag is released (CTA barrier, then st.release.gpu by one thread);
//   * every wait is bounded (about a second); on timeout the kernel records an error code
//     and the item gives up, so a wrong flag cannot hang the GPU.
//
// The 16 side/uplo/trans/diag cases use the index map of block_solve.cuh: side L solves
// M Y = alpha C with M = op(A), C = B; side R solves M Y = alpha C with M = op(A)^T, C = B^T;
// M(r, c) = tM ? A(c, r) : A(r, c).  Blocks are solved in increasing order when M is lower
// and in decreasing order when M is upper; the K chunks of an item follow the same order.
// Unit diagonals need nothing here: invA already holds the inverse of the unit triangle.
#pragma once
#include "gemm_dmma.cuh"

namespace rb200
{

constexpr int kChainThreads = 256;
constexpr int kChainBK      = 16;
constexpr int kChainStages  = 4;
constexpr int kChainNB      = 128;

struct ChainParams
{
    BatchPtr<double> A;
    int64_t          lda;
    BatchPtr<double> invA;    // blocks of 128 x 128, ld 128
    BatchPtr<double> B;
    int64_t          ldb;
    int           k;          // triangle order
    int           ncols;      // right-hand sides (n for side L, m for side R)
    int           nb, ns;     // blocks, strips
    int           forward;    // 1: blocks in increasing order (M lower)
    int64_t       items;      // systems * nb * ns
    Scalar<double> alpha;
    int*          flags;      // systems * nb * ns, zero at launch
    int*          counter;    // zero at launch
    int*          error;      // set to 4 if a wait timed out
};

__device__ __forceinline__ int chain_ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.global.acquire.gpu.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void chain_st_release(int* p, int v)
{
    asm volatile("st.global.release.gpu.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// smem layouts: P (M rows o x K) [k][o] pitch 132 (KCP = false) or [o][k] pitch BK+4 (KCP);
// Q (K x W) [k][n] pitch W+4 (KCQ = false) or [n][k] pitch BK+4 (KCQ).
template <int W, bool KCP, bool KCQ>
struct ChainCfg
{
    static constexpr int kPitchP  = KCP ? kChainBK + 4 : kChainNB + 4;
    static constexpr int kPitchQ  = KCQ ? kChainBK + 4 : W + 4;
    static constexpr int kStageP  = KCP ? kChainNB * kPitchP : kChainBK * kPitchP;
    static constexpr int kStageQ  = KCQ ? W * kPitchQ : kChainBK * kPitchQ;
    static constexpr int kStage   = kStageP + kStageQ;
    static constexpr int kPitchT  = W + 4;             // T tile [k = row o][n]
    static constexpr size_t kSmem = sizeof(double) * ((size_t)kChainStages * kStage + kChainNB * kPitchT);
};

// W right-hand sides per item (32 or 64); 8 warps as 4 (rows) x 2 (columns), each warp
// 32 x W/2 of the 128 x W block.  KCP: M's K index is contiguous in memory (tM); KCQ: C's
// row index is contiguous (side L).
template <int W, bool KCP, bool KCQ>
__global__ void __launch_bounds__(kChainThreads, 1) trsm_chain_kernel(ChainParams p)
{
    using Cfg = ChainCfg<W, KCP, KCQ>;
    constexpr int TM = 2, TN = W / 16; // per warp: 32 rows x W/2 columns
    constexpr int WN = W / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double*    smem = reinterpret_cast<double*>(smem_raw);
    double*    Ts   = smem + kChainStages * Cfg::kStage;
    __shared__ int64_t s_item;
    __shared__ int     s_abort;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int g = lane >> 2, t = lane & 3;
    const double alpha = p.alpha.get();

    if(tid == 0)
        s_abort = 0;

    for(;;)
    {
        __syncthreads();
        if(tid == 0)
            s_item = atomicAdd(reinterpret_cast<unsigned long long*>(p.counter), 1ull);
        __syncthreads();
        const int64_t item = s_item;
        if(item >= p.items || s_abort)
            break;
        const int     strip = (int)(item % p.ns);
        const int64_t sj    = item / p.ns;
        const int     j     = (int)(sj % p.nb);
        const int64_t sys   = sj / p.nb;
        const int     b     = p.forward ? j : p.nb - 1 - j;
        const int     r0    = b * kChainNB;
        const int     bs    = min(kChainNB, p.k - r0);
        const int     c0    = strip * W;
        const int     wv    = min(W, p.ncols - c0);
        const double* A     = p.A.get((int)sys);
        const double* inv   = p.invA.get((int)sys) + (int64_t)b * kChainNB * kChainNB;
        double*       B     = p.B.get((int)sys);
        int*          flags = p.flags + sys * (int64_t)p.nb * p.ns;

        // M(r, c) and C(r, col) addresses
        auto maddr = [&](int r, int c) -> const double* {
            return KCP ? A + c + (int64_t)r * p.lda : A + r + (int64_t)c * p.lda;
        };
        auto caddr = [&](int r, int col) -> double* {
            return KCQ ? B + r + (int64_t)col * p.ldb : B + col + (int64_t)r * p.ldb;
        };

        double acc[TM][TN][4];
#pragma unroll
        for(int i = 0; i < TM; ++i)
#pragma unroll
            for(int jn = 0; jn < TN; ++jn)
#pragma unroll
                for(int e = 0; e < 4; ++e)
                    acc[i][jn][e] = 0.0;

        // ---- 1. acc = M[rows of b, finished rows] * X[finished rows, strip] ---------------
        // K rows of the finished blocks: forward [0, r0) ascending; backward [r0 + bs, k)
        // descending, in 16-row chunks aligned to multiples of 16 (never across a block).
        const int klo = p.forward ? 0 : r0 + bs;
        const int khi = p.forward ? r0 : p.k;
        const int ktop = (int)ceil_div(khi, kChainBK) * kChainBK;
        const int nk = p.forward ? (int)ceil_div(khi, kChainBK) : (ktop - klo) / kChainBK;
        bool      zero = alpha == 0.0;
        int       waited = p.forward ? 0 : p.nb; // blocks known finished: [0, waited) or [waited, nb)

        auto chunk_row0 = [&](int c) { return p.forward ? c * kChainBK : ktop - (c + 1) * kChainBK; };
        // wait until the block holding chunk c is finished (uniform across the CTA)
        auto wait_chunk = [&](int c) -> bool {
            const int blk  = max(chunk_row0(c), klo) / kChainNB;
            const bool need = p.forward ? blk >= waited : blk < waited;
            if(!need)
                return true;
            if(tid == 0)
            {
                const int       jb = blk * p.ns + strip;
                const long long t0 = clock64();
                while(chain_ld_acquire(&flags[jb]) == 0)
                {
                    if(clock64() - t0 > (1ll << 31))
                    {
                        atomicExch(p.error, 4);
                        s_abort = 1;
                        break;
                    }
                }
            }
            __syncthreads();
            if(s_abort)
                return false;
            waited = p.forward ? blk + 1 : blk;
            return true;
        };
        auto load_chunk = [&](int stage, int c) {
            double*   sP = smem + stage * Cfg::kStage;
            double*   sQ = sP + Cfg::kStageP;
            const int k0 = chunk_row0(c);
            // P: M(r0 + o, k0 + kk), o < 128, kk < 16
#pragma unroll
            for(int i = 0; i < kChainNB * kChainBK / kChainThreads; ++i)
            {
                const int e = tid + i * kChainThreads;
                int       o, kk;
                if(KCP) { kk = e % kChainBK; o = e / kChainBK; }
                else    { o = e % kChainNB; kk = e / kChainNB; }
                const int  kr    = k0 + kk;
                const bool valid = o < bs && kr >= klo && kr < khi;
                const double* src = valid ? maddr(r0 + o, kr) : A;
                double* dst = KCP ? sP + o * Cfg::kPitchP + kk : sP + kk * Cfg::kPitchP + o;
                cp_async_8(dst, src, valid);
            }
            // Q: C(k0 + kk, c0 + n), kk < 16, n < W
#pragma unroll
            for(int i = 0; i < W * kChainBK / kChainThreads; ++i)
            {
                const int e = tid + i * kChainThreads;
                int       n, kk;
                if(KCQ) { kk = e % kChainBK; n = e / kChainBK; }
                else    { n = e % W; kk = e / W; }
                const int  kr    = k0 + kk;
                const bool valid = n < wv && kr >= klo && kr < khi;
                const double* src = valid ? caddr(kr, c0 + n) : B;
                double* dst = KCQ ? sQ + n * Cfg::kPitchQ + kk : sQ + kk * Cfg::kPitchQ + n;
                cp_async_8(dst, src, valid);
            }
        };
        auto ldP = [&](const double* sP, int o, int kk) {
            return KCP ? sP[o * Cfg::kPitchP + kk] : sP[kk * Cfg::kPitchP + o];
        };
        auto ldQ = [&](const double* sQ, int n, int kk) {
            return KCQ ? sQ[n * Cfg::kPitchQ + kk] : sQ[kk * Cfg::kPitchQ + n];
        };

        if(!zero && nk > 0)
        {
            bool ok = true;
#pragma unroll 1
            for(int s = 0; s < kChainStages - 1; ++s)
            {
                if(s < nk && ok)
                {
                    ok = wait_chunk(s);
                    if(ok)
                        load_chunk(s, s);
                }
                cp_async_commit();
            }
#pragma unroll 1
            for(int kt = 0; kt < nk && ok; ++kt)
            {
                cp_async_wait<kChainStages - 2>();
                __syncthreads();
                const double* sP = smem + (kt % kChainStages) * Cfg::kStage;
                const double* sQ = sP + Cfg::kStageP;
#pragma unroll
                for(int ks = 0; ks < kChainBK / 8; ++ks)
                {
                    const int kk = ks * 8 + t;
                    double    fa[TM][4], fb[TN][2];
#pragma unroll
                    for(int i = 0; i < TM; ++i)
                    {
                        const int o = wm * 32 + i * 16 + g;
                        fa[i][0] = ldP(sP, o, kk);
                        fa[i][1] = ldP(sP, o + 8, kk);
                        fa[i][2] = ldP(sP, o, kk + 4);
                        fa[i][3] = ldP(sP, o + 8, kk + 4);
                    }
#pragma unroll
                    for(int jn = 0; jn < TN; ++jn)
                    {
                        const int n = wn * WN + jn * 8 + g;
                        fb[jn][0] = ldQ(sQ, n, kk);
                        fb[jn][1] = ldQ(sQ, n, kk + 4);
                    }
#pragma unroll
                    for(int i = 0; i < TM; ++i)
#pragma unroll
                        for(int jn = 0; jn < TN; ++jn)
                            dmma_16x8x8(acc[i][jn], fa[i], fb[jn]);
                }
                const int nxt = kt + kChainStages - 1;
                if(nxt < nk)
                {
                    ok = wait_chunk(nxt);
                    if(ok)
                        load_chunk(nxt % kChainStages, nxt);
                }
                cp_async_commit();
            }
            cp_async_wait<0>();
            __syncthreads();
            if(!ok)
                break;
        }

        // ---- 2. T = alpha C_b - acc into shared memory ([row o][col n]) --------------------
#pragma unroll
        for(int i = 0; i < TM; ++i)
#pragma unroll
            for(int jn = 0; jn < TN; ++jn)
#pragma unroll
                for(int e = 0; e < 4; ++e)
                {
                    const int o = wm * 32 + i * 16 + g + (e >> 1) * 8;
                    const int n = wn * WN + jn * 8 + 2 * t + (e & 1);
                    double    v = 0.0;
                    if(!zero && o < bs && n < wv)
                        v = alpha * __ldcg(caddr(r0 + o, c0 + n)) - acc[i][jn][e];
                    Ts[o * Cfg::kPitchT + n] = v;
                }

        // ---- 3. X_b = inv(M_bb) T: invA chunks through the pipeline, T resident ---------
        // inv(M_bb)(o, kk) = tM ? invA(kk, o) : invA(o, kk); its triangle: lower when M is
        // lower (forward), upper otherwise; rows / columns >= bs are zero.
#pragma unroll
        for(int i = 0; i < TM; ++i)
#pragma unroll
            for(int jn = 0; jn < TN; ++jn)
#pragma unroll
                for(int e = 0; e < 4; ++e)
                    acc[i][jn][e] = 0.0;
        const int nki = (int)ceil_div(bs, kChainBK);
        auto load_inv = [&](int stage, int c) {
            double*   sP = smem + stage * Cfg::kStage;
            const int k0 = c * kChainBK;
#pragma unroll
            for(int i = 0; i < kChainNB * kChainBK / kChainThreads; ++i)
            {
                const int e = tid + i * kChainThreads;
                int       o, kk;
                if(KCP) { kk = e % kChainBK; o = e / kChainBK; }
                else    { o = e % kChainNB; kk = e / kChainNB; }
                const int  kr    = k0 + kk;
                const bool tri   = p.forward ? kr <= o : kr >= o;
                const bool valid = !zero && o < bs && kr < bs && tri;
                const double* src = valid ? (KCP ? inv + kr + (int64_t)o * kChainNB
                                                 : inv + o + (int64_t)kr * kChainNB)
                                          : inv;
                double* dst = KCP ? sP + o * Cfg::kPitchP + kk : sP + kk * Cfg::kPitchP + o;
                cp_async_8(dst, src, valid);
            }
        };
#pragma unroll 1
        for(int s = 0; s < kChainStages - 1; ++s)
        {
            if(s < nki)
                load_inv(s, s);
            cp_async_commit();
        }
#pragma unroll 1
        for(int kt = 0; kt < nki; ++kt)
        {
            cp_async_wait<kChainStages - 2>();
            __syncthreads();
            const double* sP = smem + (kt % kChainStages) * Cfg::kStage;
#pragma unroll
            for(int ks = 0; ks < kChainBK / 8; ++ks)
            {
                const int kk = ks * 8 + t;
                const int kg = kt * kChainBK + kk; // row of T
                double    fa[TM][4], fb[TN][2];
#pragma unroll
                for(int i = 0; i < TM; ++i)
                {
                    const int o = wm * 32 + i * 16 + g;
                    fa[i][0] = ldP(sP, o, kk);
                    fa[i][1] = ldP(sP, o + 8, kk);
                    fa[i][2] = ldP(sP, o, kk + 4);
                    fa[i][3] = ldP(sP, o + 8, kk + 4);
                }
#pragma unroll
                for(int jn = 0; jn < TN; ++jn)
                {
                    const int n = wn * WN + jn * 8 + g;
                    fb[jn][0] = Ts[kg * Cfg::kPitchT + n];
                    fb[jn][1] = Ts[(kg + 4) * Cfg::kPitchT + n];
                }
#pragma unroll
                for(int i = 0; i < TM; ++i)
#pragma unroll
                    for(int jn = 0; jn < TN; ++jn)
                        dmma_16x8x8(acc[i][jn], fa[i], fb[jn]);
            }
            const int nxt = kt + kChainStages - 1;
            if(nxt < nki)
                load_inv(nxt % kChainStages, nxt);
            cp_async_commit();
        }
        cp_async_wait<0>();

        // ---- 4. X_b over C_b, then release the block's flag --------------------------------
#pragma unroll
        for(int i = 0; i < TM; ++i)
#pragma unroll
            for(int jn = 0; jn < TN; ++jn)
#pragma unroll
                for(int e = 0; e < 4; ++e)
                {
                    const int o = wm * 32 + i * 16 + g + (e >> 1) * 8;
                    const int n = wn * WN + jn * 8 + 2 * t + (e & 1);
                    if(o < bs && n < wv)
                        *caddr(r0 + o, c0 + n) = acc[i][jn][e];
                }
        __syncthreads();
        if(tid == 0)
            chain_st_release(&flags[b * p.ns + strip], 1);
    }
}

// Blocks, strips and the workspace of one chain solve: flags (systems * nb * ns ints), then
// (8-byte aligned) the 8-byte claim counter and a spare error word.
struct ChainShape
{
    int     nb, ns, w;
    int64_t items;
};

inline ChainShape chain_shape(int k, int ncols, int batch, int w)
{
    ChainShape c;
    c.w     = w;
    c.nb    = (int)ceil_div(k, kChainNB);
    c.ns    = (int)ceil_div(ncols, w);
    c.items = (int64_t)batch * c.nb * c.ns;
    return c;
}

inline size_t chain_workspace_bytes(const ChainShape& c)
{
    return ((size_t)c.items * sizeof(int) + 7) / 8 * 8 + 16;
}

template <int W, bool KCP, bool KCQ>
static void launch_chain_cfg(const ChainParams& p, int sms, cudaStream_t s)
{
    using Cfg = ChainCfg<W, KCP, KCQ>;
    auto kern = trsm_chain_kernel<W, KCP, KCQ>;
    cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::kSmem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kChainThreads, Cfg::kSmem);
    const int64_t grid = std::min<int64_t>(p.items, (int64_t)sms * std::max(per_sm, 1));
    kern<<<(unsigned)grid, kChainThreads, Cfg::kSmem, s>>>(p);
}

template <int W>
static void launch_chain_w(const ChainParams& p, bool kcp, bool kcq, int sms, cudaStream_t s)
{
    if(kcp && kcq)
        launch_chain_cfg<W, true, true>(p, sms, s);
    else if(kcp)
        launch_chain_cfg<W, true, false>(p, sms, s);
    else if(kcq)
        launch_chain_cfg<W, false, true>(p, sms, s);
    else
        launch_chain_cfg<W, false, false>(p, sms, s);
}

} // namespace rb200
