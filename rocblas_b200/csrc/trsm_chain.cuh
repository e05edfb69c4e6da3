// Left-looking blocked TRSM in one persistent launch (a dependency chain over the 128-row
// blocks of the triangle), for few right-hand sides per system and for batches of systems of
// different sizes.
//
// The reference's left-looking path (special_trsm_template,
// library/src/blas3/rocblas_trsm_kernels.hpp:1164-1456) walks the diagonal blocks on the
// host: per 128-row block j one GEMM tmp = alpha B_j - A_{j,<j} X_{<j} and one GEMM
// X_j = invA_jj tmp, two launches per block.  With few right-hand sides every launch is
// small, so the solve is bound by launch latency.  Here one launch does the whole solve:
//
//   * work items are (block position j in solve order, system, strip of W right-hand sides),
//     enumerated level by level: all systems' items of position 0, then of position 1, ...
//     A CTA claims item ids from a device-side counter in increasing order, so every item an
//     item depends on (same system and strip, earlier position) was claimed before it by a
//     CTA that is running; the earliest unfinished claimed item therefore never waits on an
//     unfinished one: no deadlock, whatever the residency.  With many systems in one launch
//     (the variable-size batch) a CTA rarely waits at all: the items claimed before it are
//     mostly other systems' work of the same level;
//   * an item accumulates M_{b,i} X_i over the finished blocks i in solve order through a
//     cp.async pipeline of 32- or 16-deep K chunks (ChainCfg) on DMMA (mma.sync m16n8k8 f64),
//     waiting on a block's flag (ld.acquire.gpu by one thread, then a CTA barrier) before its
//     first chunk;
//   * then T = alpha C_b - acc goes to shared memory, X_b = inv(M_bb) T (the caller's or the
//     fused trtri's invA block, its triangle masked) is written over C_b, and the item's
//     flag is released (CTA barrier, then st.release.gpu by one thread);
//   * every wait is bounded (about a second); on timeout the kernel records an error code
//     and the CTA stops, so a wrong flag cannot hang the GPU.
// FP32 systems are staged as FP32 and computed in FP64 (the chain is latency-bound, and the
// DMMA path is the one this kernel has); the result is rounded to FP32 once.
//
// The 16 side/uplo/trans/diag cases use the index map of block_solve.cuh: side L solves
// M Y = alpha C with M = op(A), C = B; side R solves M Y = alpha C with M = op(A)^T, C = B^T;
// M(r, c) = tM ? A(c, r) : A(r, c).  Blocks are solved in increasing order when M is lower
// and in decreasing order when M is upper; the K chunks of an item follow the same order.
// Unit diagonals need nothing here: invA already holds the inverse of the unit triangle.
#pragma once
#include "gemm_dmma.cuh"
#include "timing.hpp"

namespace rb200
{

constexpr int kChainThreads = 256;
constexpr int kChainBK      = 16;
constexpr int kChainStages  = 4;
constexpr int kChainNB      = 128;

// One system of a variable-size chain launch (sorted by block count, largest first).
template <typename T>
struct ChainSys
{
    const T* A;
    const T* invA; // blocks of 128 x 128, ld 128
    T*       B;
    int64_t  lda, ldb;
    int      k, ncols, nb, ns;
    int      forward, pad;
};

// Tables of a variable-size chain launch for one (tM, side) combination.
template <typename T>
struct ChainVbHeader
{
    const ChainSys<T>* vsys;  // its systems, sorted by nb descending
    const int*         vP;    // vP[i]: prefix sum of ns over vsys[0..i)
    const int*         vcnt;  // vcnt[j]: systems with nb > j
    const int64_t*     vL;    // vL[j]: first item id of level j; vL[maxnb] = its items
    int*               flags; // one per item id
    int                maxnb;
    int                pad;
};

template <typename T>
struct ChainParams
{
    // uniform batch (VB = false): every system has these sizes
    BatchPtr<T>    A;
    int64_t        lda;
    BatchPtr<T>    invA;
    BatchPtr<T>    B;
    int64_t        ldb;
    int            k;       // triangle order
    int            ncols;   // right-hand sides (n for side L, m for side R)
    int            nb, ns;  // blocks, strips
    int            forward; // 1: blocks in increasing order (M lower)
    int64_t        items;   // nb * systems * ns
    int            systems;
    // variable batch (VB = true): the tables of one (tM, side) combination, built on the
    // device by chain_vb_prepass_kernel
    const ChainVbHeader<T>* vhdr;
    Scalar<T>      alpha;   // the caller's alpha
    int            first;   // 1: this solve applies alpha; 0: it applies 1 (a sub-solve after an update)
    int*           flags;   // one per item id, zero at launch
    int*           counter; // 8-byte claim counter, zero at launch
    int*           error;   // set to 4 if a wait timed out
    long long      wait_cycles = 1ll << 31; // a flag wait gives up after this many clock cycles
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

template <typename T>
__device__ __forceinline__ void chain_cp_async(T* smem, const T* gmem, bool valid)
{
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    const int      n = valid ? (int)sizeof(T) : 0;
    if constexpr(sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}

// smem layouts: P (M rows o x K) [k][o] pitch 132 (KCP = false) or [o][k] pitch BK+4 (KCP);
// Q (K x W) [k][n] pitch W+4 (KCQ = false) or [n][k] pitch BK+4 (KCQ); elements of type T.
// K chunks are 32 deep in 3 stages where that fits in shared memory (fewer CTA barriers per
// MMA; measured faster for one large system), else 16 deep in 4 stages (measured faster for
// the variable-size batch, VB); either depth divides the 128-row blocks, so a chunk never
// spans two blocks.
template <typename T, int W, bool KCP, bool KCQ, bool VB = false>
struct ChainCfg
{
    static constexpr size_t bytes(int bk, int stages)
    {
        const int pp = KCP ? bk + 4 : kChainNB + 4, pq = KCQ ? bk + 4 : W + 4;
        const int sp = KCP ? kChainNB * pp : bk * pp, sq = KCQ ? W * pq : bk * pq;
        return sizeof(T) * (size_t)stages * (sp + sq) + sizeof(double) * (size_t)kChainNB * (W + 4);
    }
    static constexpr bool kDeep   = !VB && bytes(32, 3) <= 227 * 1024 - 64; // room for the static words
    static constexpr int kBK      = kDeep ? 32 : kChainBK;
    static constexpr int kStages  = kDeep ? 3 : kChainStages;
    static constexpr int kPitchP  = KCP ? kBK + 4 : kChainNB + 4;
    static constexpr int kPitchQ  = KCQ ? kBK + 4 : W + 4;
    static constexpr int kStageP  = KCP ? kChainNB * kPitchP : kBK * kPitchP;
    static constexpr int kStageQ  = KCQ ? W * kPitchQ : kBK * kPitchQ;
    static constexpr int kStage   = kStageP + kStageQ; // elements of T
    static constexpr int kPitchT  = W + 4;             // T tile [k = row o][n], doubles
    static constexpr size_t kSmem = bytes(kBK, kStages);
};

// W right-hand sides per item (32 or 64); 8 warps as 4 (rows) x 2 (columns), each warp
// 32 x W/2 of the 128 x W block.  KCP: M's K index is contiguous in memory (tM); KCQ: C's
// row index is contiguous (side L).  VB: the variable-size tables of p describe the items.
template <typename T, int W, bool KCP, bool KCQ, bool VB>
__global__ void __launch_bounds__(kChainThreads, 1) trsm_chain_kernel(ChainParams<T> p)
{
    using Cfg = ChainCfg<T, W, KCP, KCQ, VB>;
    constexpr int TM = 2, TN = W / 16; // per warp: 32 rows x W/2 columns
    constexpr int WN = W / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T*         smem = reinterpret_cast<T*>(smem_raw);
    double*    Ts   = reinterpret_cast<double*>(smem_raw + sizeof(T) * (size_t)Cfg::kStages * Cfg::kStage);
    __shared__ int64_t s_item;
    __shared__ int     s_abort;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int g = lane >> 2, t = lane & 3;
    // alpha == 0 anywhere in the call means B := 0 with A unreferenced, also for sub-solves
    // that would otherwise apply 1
    const double ua    = (double)p.alpha.get();
    const double alpha = ua == 0.0 ? 0.0 : (p.first ? ua : 1.0);
    ChainVbHeader<T> H{};
    if constexpr(VB)
        H = *p.vhdr;
    int* const    flags = VB ? H.flags : p.flags;
    const int64_t total = VB ? (H.maxnb > 0 ? H.vL[H.maxnb] : 0) : p.items;

    if(tid == 0)
        s_abort = 0;

    for(;;)
    {
        __syncthreads();
        if(tid == 0)
            s_item = atomicAdd(reinterpret_cast<unsigned long long*>(p.counter), 1ull);
        __syncthreads();
        const int64_t item = s_item;
        if(item >= total || s_abort)
            break;

        // ---- resolve the item: (level j, system, strip) ------------------------------------
        const T* A;
        const T* invA;
        T*       B;
        int64_t  lda, ldb, sysi;
        int      k, ncols, nb, ns, forward, j, strip;
        if constexpr(VB)
        {
            // level: last j with vL[j] <= item; system: last i < vcnt[j] with vP[i] <= r
            int lo = 0, hi = H.maxnb - 1;
            while(lo < hi)
            {
                const int mid = (lo + hi + 1) >> 1;
                if(H.vL[mid] <= item)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            j = lo;
            const int r = (int)(item - H.vL[j]);
            int       a = 0, z = H.vcnt[j] - 1;
            while(a < z)
            {
                const int mid = (a + z + 1) >> 1;
                if(H.vP[mid] <= r)
                    a = mid;
                else
                    z = mid - 1;
            }
            sysi  = a;
            strip = r - H.vP[a];
            const ChainSys<T> q = H.vsys[a];
            A = q.A; invA = q.invA; B = q.B; lda = q.lda; ldb = q.ldb;
            k = q.k; ncols = q.ncols; nb = q.nb; ns = q.ns; forward = q.forward;
        }
        else
        {
            strip = (int)(item % p.ns);
            const int64_t js = item / p.ns;
            sysi  = js % p.systems;
            j     = (int)(js / p.systems);
            A = p.A.get((int)sysi); invA = p.invA.get((int)sysi); B = p.B.get((int)sysi);
            lda = p.lda; ldb = p.ldb; k = p.k; ncols = p.ncols; nb = p.nb; ns = p.ns;
            forward = p.forward;
        }
        // flag of this system's strip at solve position jj (= that item's id)
        auto flag_of = [&](int jj) -> int* {
            if constexpr(VB)
                return flags + H.vL[jj] + H.vP[sysi] + strip;
            else
                return flags + ((int64_t)jj * p.systems + sysi) * ns + strip;
        };
        const int b  = forward ? j : nb - 1 - j;
        const int r0 = b * kChainNB;
        const int bs = min(kChainNB, k - r0);
        const int c0 = strip * W;
        const int wv = min(W, ncols - c0);
        const T*  inv = invA + (int64_t)b * kChainNB * kChainNB;

        // M(r, c) and C(r, col) addresses
        auto maddr = [&](int rr, int cc) -> const T* {
            return KCP ? A + cc + (int64_t)rr * lda : A + rr + (int64_t)cc * lda;
        };
        auto caddr = [&](int rr, int col) -> T* {
            return KCQ ? B + rr + (int64_t)col * ldb : B + col + (int64_t)rr * ldb;
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
        // descending, in chunks of Cfg::kBK rows aligned to multiples of kBK (never across a
        // block).
        const int klo  = forward ? 0 : r0 + bs;
        const int khi  = forward ? r0 : k;
        const int ktop = (int)ceil_div(khi, Cfg::kBK) * Cfg::kBK;
        const int nk   = forward ? (int)ceil_div(khi, Cfg::kBK) : (ktop - klo) / Cfg::kBK;
        const bool zero = alpha == 0.0;
        int waited = forward ? 0 : nb; // blocks known finished: [0, waited) or [waited, nb)

        auto chunk_row0 = [&](int c) { return forward ? c * Cfg::kBK : ktop - (c + 1) * Cfg::kBK; };
        // wait until the block holding chunk c is finished (uniform across the CTA)
        auto wait_chunk = [&](int c) -> bool {
            const int  blk  = max(chunk_row0(c), klo) / kChainNB;
            const bool need = forward ? blk >= waited : blk < waited;
            if(!need)
                return true;
            if(tid == 0)
            {
                const int*      f  = flag_of(forward ? blk : nb - 1 - blk);
                const long long t0 = clock64();
                while(chain_ld_acquire(f) == 0)
                {
                    if(clock64() - t0 > p.wait_cycles)
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
            waited = forward ? blk + 1 : blk;
            return true;
        };
        auto load_chunk = [&](int stage, int c) {
            T*        sP = smem + stage * Cfg::kStage;
            T*        sQ = sP + Cfg::kStageP;
            const int k0 = chunk_row0(c);
            // P: M(r0 + o, k0 + kk), o < 128, kk < 16
#pragma unroll
            for(int i = 0; i < kChainNB * Cfg::kBK / kChainThreads; ++i)
            {
                const int e = tid + i * kChainThreads;
                int       o, kk;
                if(KCP) { kk = e % Cfg::kBK; o = e / Cfg::kBK; }
                else    { o = e % kChainNB; kk = e / kChainNB; }
                const int  kr    = k0 + kk;
                const bool valid = o < bs && kr >= klo && kr < khi;
                const T*   src   = valid ? maddr(r0 + o, kr) : A;
                T*         dst   = KCP ? sP + o * Cfg::kPitchP + kk : sP + kk * Cfg::kPitchP + o;
                chain_cp_async<T>(dst, src, valid);
            }
            // Q: C(k0 + kk, c0 + n), kk < 16, n < W
#pragma unroll
            for(int i = 0; i < W * Cfg::kBK / kChainThreads; ++i)
            {
                const int e = tid + i * kChainThreads;
                int       n, kk;
                if(KCQ) { kk = e % Cfg::kBK; n = e / Cfg::kBK; }
                else    { n = e % W; kk = e / W; }
                const int  kr    = k0 + kk;
                const bool valid = n < wv && kr >= klo && kr < khi;
                const T*   src   = valid ? caddr(kr, c0 + n) : B;
                T*         dst   = KCQ ? sQ + n * Cfg::kPitchQ + kk : sQ + kk * Cfg::kPitchQ + n;
                chain_cp_async<T>(dst, src, valid);
            }
        };
        auto ldP = [&](const T* sP, int o, int kk) -> double {
            return (double)(KCP ? sP[o * Cfg::kPitchP + kk] : sP[kk * Cfg::kPitchP + o]);
        };
        auto ldQ = [&](const T* sQ, int n, int kk) -> double {
            return (double)(KCQ ? sQ[n * Cfg::kPitchQ + kk] : sQ[kk * Cfg::kPitchQ + n]);
        };

        if(!zero && nk > 0)
        {
            bool ok = true;
#pragma unroll 1
            for(int s = 0; s < Cfg::kStages - 1; ++s)
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
                cp_async_wait<Cfg::kStages - 2>();
                __syncthreads();
                const T* sP = smem + (kt % Cfg::kStages) * Cfg::kStage;
                const T* sQ = sP + Cfg::kStageP;
#pragma unroll
                for(int ks = 0; ks < Cfg::kBK / 8; ++ks)
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
                const int nxt = kt + Cfg::kStages - 1;
                if(nxt < nk)
                {
                    ok = wait_chunk(nxt);
                    if(ok)
                        load_chunk(nxt % Cfg::kStages, nxt);
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
                        v = alpha * (double)__ldcg(caddr(r0 + o, c0 + n)) - acc[i][jn][e];
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
        const int nki = (int)ceil_div(bs, Cfg::kBK);
        auto load_inv = [&](int stage, int c) {
            T*        sP = smem + stage * Cfg::kStage;
            const int k0 = c * Cfg::kBK;
#pragma unroll
            for(int i = 0; i < kChainNB * Cfg::kBK / kChainThreads; ++i)
            {
                const int e = tid + i * kChainThreads;
                int       o, kk;
                if(KCP) { kk = e % Cfg::kBK; o = e / Cfg::kBK; }
                else    { o = e % kChainNB; kk = e / kChainNB; }
                const int  kr    = k0 + kk;
                const bool tri   = forward ? kr <= o : kr >= o;
                const bool valid = !zero && o < bs && kr < bs && tri;
                const T*   src   = valid ? (KCP ? inv + kr + (int64_t)o * kChainNB
                                                : inv + o + (int64_t)kr * kChainNB)
                                         : inv;
                T* dst = KCP ? sP + o * Cfg::kPitchP + kk : sP + kk * Cfg::kPitchP + o;
                chain_cp_async<T>(dst, src, valid);
            }
        };
#pragma unroll 1
        for(int s = 0; s < Cfg::kStages - 1; ++s)
        {
            if(s < nki)
                load_inv(s, s);
            cp_async_commit();
        }
#pragma unroll 1
        for(int kt = 0; kt < nki; ++kt)
        {
            cp_async_wait<Cfg::kStages - 2>();
            __syncthreads();
            const T* sP = smem + (kt % Cfg::kStages) * Cfg::kStage;
#pragma unroll
            for(int ks = 0; ks < Cfg::kBK / 8; ++ks)
            {
                const int kk = ks * 8 + t;
                const int kg = kt * Cfg::kBK + kk; // row of T
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
            const int nxt = kt + Cfg::kStages - 1;
            if(nxt < nki)
                load_inv(nxt % Cfg::kStages, nxt);
            cp_async_commit();
        }
        cp_async_wait<0>();

        // ---- 4. X_b over C_b, then release the item's flag ---------------------------------
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
                        *caddr(r0 + o, c0 + n) = (T)acc[i][jn][e];
                }
        __syncthreads();
        if(tid == 0)
            chain_st_release(flags + item, 1);
    }
}

// Blocks, strips and the workspace of one uniform chain solve: flags (one per item), then
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

inline size_t chain_flags_bytes(int64_t items)
{
    return ((size_t)items * sizeof(int) + 7) / 8 * 8 + 16;
}

inline size_t chain_workspace_bytes(const ChainShape& c)
{
    return chain_flags_bytes(c.items);
}

// cluster2: the grid as clusters of two CTAs (placement only; the kernel uses no cluster
// feature), for an even grid
template <typename T, int W, bool KCP, bool KCQ, bool VB>
static void launch_chain_cfg(const ChainParams<T>& p, int sms, int64_t max_items, cudaStream_t s,
                             bool cluster2 = false)
{
    using Cfg = ChainCfg<T, W, KCP, KCQ, VB>;
    auto kern = trsm_chain_kernel<T, W, KCP, KCQ, VB>;
    cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::kSmem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kChainThreads, Cfg::kSmem);
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(max_items, (int64_t)sms * std::max(per_sm, 1)));
    // algorithmic work (uniform batch): k * k * ncols per system, the trsm flop count
    const double work = VB ? 0.0 : (double)p.systems * p.k * (double)p.k * p.ncols;
    TimedLaunch tl(KernelClass::chain, s, work);
    if(cluster2 && grid % 2 == 0)
    {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim          = dim3((unsigned)grid);
        cfg.blockDim         = dim3(kChainThreads);
        cfg.dynamicSmemBytes = Cfg::kSmem;
        cfg.stream           = s;
        cudaLaunchAttribute at[1];
        at[0].id               = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 2;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs    = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, kern, p);
    }
    else
        kern<<<(unsigned)grid, kChainThreads, Cfg::kSmem, s>>>(p);
}

template <typename T, int W, bool VB>
static void launch_chain_w(const ChainParams<T>& p, bool kcp, bool kcq, int sms, int64_t max_items,
                           cudaStream_t s, bool cluster2 = false)
{
    if(kcp && kcq)
        launch_chain_cfg<T, W, true, true, VB>(p, sms, max_items, s, cluster2);
    else if(kcp)
        launch_chain_cfg<T, W, true, false, VB>(p, sms, max_items, s, cluster2);
    else if(kcq)
        launch_chain_cfg<T, W, false, true, VB>(p, sms, max_items, s, cluster2);
    else
        launch_chain_cfg<T, W, false, false, VB>(p, sms, max_items, s, cluster2);
}

} // namespace rb200
