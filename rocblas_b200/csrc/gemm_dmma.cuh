// FP64 GEMM tiles on the DMMA tensor path with a cp.async multistage pipeline.
//
//     C := a * op(P) * op(Q) + b * C        (same contract as gemm_tile.cuh, GemmParams<double>)
//
// B200's FP64 tensor instruction is mma.sync m8n8k4 (the tcgen05 tensor cores have no f64
// kind), so these tiles feed DMMA from shared memory filled by 8-byte cp.async copies
// (any leading dimension, zero-fill for out-of-range and masked-triangle elements) in a
// 3..4-stage ring.  Each operand is staged in the orientation that keeps both the copies and
// the fragment reads free of bank conflicts:
//   operand rows contiguous in memory (kc = false): smem [k][o], pitch O + 4 doubles;
//   operand k contiguous in memory   (kc = true) : smem [o][k], pitch 16 + 4 doubles.
// Every warp owns a 32 x 32 block of C computed with mma.sync m16n8k8 .f64 (2 x 4 MMAs per
// 8-deep k step).  Tile shapes range from 128 x 128 (16 warps) over 64 x 128 / 128 x 64
// (8 warps, two CTAs per SM) down to 128 x 32 / 32 x 128 (4 warps), so that small trailing
// updates and the invA leaves still fill the 148 SMs.
#pragma once
#include "gemm_tile.cuh"
#include "mma_f64.cuh"
#include "timing.hpp"
#include "tuning.hpp"

namespace rb200
{

constexpr int kDBK = 16;

__device__ __forceinline__ void cp_async_8(void* smem, const void* gmem, bool valid)
{
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    const int      n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int BM, int BN, int WM, int WN, int STAGES, bool KCP, bool KCQ, int BK = kDBK>
struct DmmaCfg
{
    static constexpr int kBK      = BK;
    static constexpr int kWarpsM  = BM / WM;
    static constexpr int kWarpsN  = BN / WN;
    static constexpr int kThreads = kWarpsM * kWarpsN * 32;
    static constexpr int kPitchA  = KCP ? (BK + 4) : (BM + 4);
    static constexpr int kPitchB  = KCQ ? (BK + 4) : (BN + 4);
    static constexpr int kStageA  = KCP ? BM * kPitchA : BK * kPitchA; // doubles
    static constexpr int kStageB  = KCQ ? BN * kPitchB : BK * kPitchB;
    static constexpr int kStage   = kStageA + kStageB;
    static constexpr size_t kSmem = (size_t)STAGES * kStage * sizeof(double);
};

// Loads one BK-deep stage of an operand tile of `O` rows (o0..o0+O-1 of the logical operand)
// with cp.async.  Logical (o, k) is stored at ptr[r + c*ld], (r, c) = kc ? (k, o) : (o, k).
template <int O, int NT, bool KC, int BK>
__device__ __forceinline__ void dmma_load_stage(double* s, const double* ptr, int64_t ld, int tri,
                                                int o0, int k0, int Olim, int Klim, int tid)
{
    constexpr int PER = O * BK / NT;
    static_assert(PER * NT == O * BK, "tile / thread mismatch");
#pragma unroll
    for(int i = 0; i < PER; ++i)
    {
        const int e = tid + i * NT;
        int       o, kk;
        if(KC)
        {
            kk = e % BK;
            o  = e / BK;
        }
        else
        {
            o  = e % O;
            kk = e / O;
        }
        const int     go = o0 + o, gk = k0 + kk;
        const int64_t r = KC ? gk : go, c = KC ? go : gk;
        const bool    valid = go < Olim && gk < Klim && tri_keep(tri, r, c);
        const double* src   = valid ? ptr + r + c * ld : ptr;
        double*       dst   = KC ? s + o * (BK + 4) + kk : s + kk * (O + 4) + o;
        cp_async_8(dst, src, valid);
    }
}

// Narrows the K-block range [kt0, kt1) of a tile whose rows (P) or columns (Q) start at o0
// and span O to the blocks inside the operand's triangle mask.  The mask is in stored
// coordinates, as dmma_load_stage applies it: for P, stored (r, c) = transP ? (k, o) : (o, k);
// for Q, transQ ? (o, k) : (k, o).  A lower mask keeps r >= c, an upper one r <= c; the strict
// masks keep a subset of the same range.
__device__ __forceinline__ void dmma_tri_k_range(int tri, bool trans, bool is_p, int o0, int O, int BK,
                                                 int& kt0, int& kt1)
{
    if(tri == kTriNone)
        return;
    const bool lower    = tri == kTriLower || tri == kTriLowerStrict;
    const bool o_is_row = is_p ? !trans : trans; // o is the stored row index
    const bool k_le_o   = o_is_row ? lower : !lower; // the kept region has k <= o (else k >= o)
    if(k_le_o)
        kt1 = min(kt1, (o0 + O + BK - 1) / BK);
    else
        kt0 = max(kt0, o0 / BK);
}

template <int BM, int BN, int WM, int WN, int STAGES, bool KCP, bool KCQ, int BK, int MK>
__global__ void __launch_bounds__(DmmaCfg<BM, BN, WM, WN, STAGES, KCP, KCQ, BK>::kThreads,
                                  DmmaCfg<BM, BN, WM, WN, STAGES, KCP, KCQ, BK>::kThreads <= 256 ? 2 : 1)
    gemm_dmma_kernel(GemmParams<double> p)
{
    using Cfg = DmmaCfg<BM, BN, WM, WN, STAGES, KCP, KCQ, BK>;
    constexpr int NT = Cfg::kThreads;
    constexpr int TM = WM / 16, TN = WN / 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* smem = reinterpret_cast<double*>(smem_raw);

    const int tid   = threadIdx.x;
    const int lane  = tid & 31, warp = tid >> 5;
    const int wm    = warp % Cfg::kWarpsM, wn = warp / Cfg::kWarpsM;
    const int m0    = blockIdx.x * BM;
    const int n0    = blockIdx.y * BN;
    const int batch = p.batch_base + blockIdx.z;

    double*      C  = p.C.get(batch);
    const double ua = (p.zero_guard || p.a_user || p.b_user) ? p.ualpha.get() : 1.0;
    const bool   zero_out = p.zero_guard && ua == 0.0;
    const double a  = p.a_user ? ua : p.a_imm;
    const double b  = p.b_user ? ua : p.b_imm;

    double acc[TM][TN][4];
#pragma unroll
    for(int i = 0; i < TM; ++i)
#pragma unroll
        for(int j = 0; j < TN; ++j)
#pragma unroll
            for(int e = 0; e < 4; ++e)
                acc[i][j][e] = 0.0;

    const int g = lane >> 2, t = lane & 3;
    if(!zero_out)
    {
        const double* P  = p.P.get(batch);
        const double* Q  = p.Q.get(batch);
        // K blocks that can meet a masked triangle of this tile: the rest are all zeros, so
        // a triangular operand costs half of a dense one
        int kt0 = 0, kt1 = (p.K + BK - 1) / BK;
        dmma_tri_k_range(p.triP, p.transP != 0, true, m0, BM, BK, kt0, kt1);
        dmma_tri_k_range(p.triQ, p.transQ != 0, false, n0, BN, BK, kt0, kt1);
        const int nk = kt1 > kt0 ? kt1 - kt0 : 0;
        auto load = [&](int stage, int kt) {
            kt += kt0;
            double* sA = smem + stage * Cfg::kStage;
            double* sB = sA + Cfg::kStageA;
            dmma_load_stage<BM, NT, KCP, BK>(sA, P, p.ldp, p.triP, m0, kt * BK, p.M, p.K, tid);
            dmma_load_stage<BN, NT, KCQ, BK>(sB, Q, p.ldq, p.triQ, n0, kt * BK, p.N, p.K, tid);
        };
        auto ldA = [&](const double* sA, int m, int k) {
            return KCP ? sA[m * Cfg::kPitchA + k] : sA[k * Cfg::kPitchA + m];
        };
        auto ldB = [&](const double* sB, int n, int k) {
            return KCQ ? sB[n * Cfg::kPitchB + k] : sB[k * Cfg::kPitchB + n];
        };
#pragma unroll
        for(int s = 0; s < STAGES - 1; ++s)
        {
            if(s < nk)
                load(s, s);
            cp_async_commit();
        }
        for(int kt = 0; kt < nk; ++kt)
        {
            cp_async_wait<STAGES - 2>();
            __syncthreads();
            const double* sA = smem + (kt % STAGES) * Cfg::kStage;
            const double* sB = sA + Cfg::kStageA;
            if constexpr(MK == 16)
            {
#pragma unroll
                for(int ks = 0; ks < BK / 16; ++ks)
                {
                    const int k = ks * 16 + t;
                    double    fa[TM][8], fb[TN][4];
#pragma unroll
                    for(int i = 0; i < TM; ++i)
                    {
                        const int m = wm * WM + i * 16 + g;
#pragma unroll
                        for(int q = 0; q < 4; ++q)
                        {
                            fa[i][2 * q]     = ldA(sA, m, k + 4 * q);
                            fa[i][2 * q + 1] = ldA(sA, m + 8, k + 4 * q);
                        }
                    }
#pragma unroll
                    for(int j = 0; j < TN; ++j)
                    {
                        const int n = wn * WN + j * 8 + g;
#pragma unroll
                        for(int q = 0; q < 4; ++q)
                            fb[j][q] = ldB(sB, n, k + 4 * q);
                    }
#pragma unroll
                    for(int i = 0; i < TM; ++i)
#pragma unroll
                        for(int j = 0; j < TN; ++j)
                            dmma_16x8x16(acc[i][j], fa[i], fb[j]);
                }
            }
            else
#pragma unroll
            for(int ks = 0; ks < BK / 8; ++ks)
            {
                const int k = ks * 8 + t;
                double    fa[TM][4], fb[TN][2];
#pragma unroll
                for(int i = 0; i < TM; ++i)
                {
                    const int m = wm * WM + i * 16 + g;
                    fa[i][0] = ldA(sA, m, k);
                    fa[i][1] = ldA(sA, m + 8, k);
                    fa[i][2] = ldA(sA, m, k + 4);
                    fa[i][3] = ldA(sA, m + 8, k + 4);
                }
#pragma unroll
                for(int j = 0; j < TN; ++j)
                {
                    const int n = wn * WN + j * 8 + g;
                    fb[j][0] = ldB(sB, n, k);
                    fb[j][1] = ldB(sB, n, k + 4);
                }
#pragma unroll
                for(int i = 0; i < TM; ++i)
#pragma unroll
                    for(int j = 0; j < TN; ++j)
                        dmma_16x8x8(acc[i][j], fa[i], fb[j]);
            }
            const int nxt = kt + STAGES - 1;
            if(nxt < nk)
                load(nxt % STAGES, nxt);
            cp_async_commit();
        }
        cp_async_wait<0>();
    }

    const int64_t ldc = p.ldc;
#pragma unroll
    for(int i = 0; i < TM; ++i)
#pragma unroll
        for(int j = 0; j < TN; ++j)
#pragma unroll
            for(int e = 0; e < 4; ++e)
            {
                const int gr = m0 + wm * WM + i * 16 + g + (e >> 1) * 8;
                const int gc = n0 + wn * WN + j * 8 + 2 * t + (e & 1);
                if(gr < p.M && gc < p.N)
                {
                    double* cp = C + gr + (int64_t)gc * ldc;
                    double  out;
                    if(zero_out)
                        out = 0.0;
                    else if(b == 0.0)
                        out = a * acc[i][j][e];
                    else
                        out = fma(a, acc[i][j][e], b * (*cp));
                    *cp = out;
                }
            }
}

// ---- launch --------------------------------------------------------------------------------
template <int BM, int BN, int WM, int WN, int STAGES, bool KCP, bool KCQ, int BK = kDBK, int MK = 8>
static void launch_dmma_cfg(const GemmParams<double>& p0, int batch, cudaStream_t s)
{
    using Cfg = DmmaCfg<BM, BN, WM, WN, STAGES, KCP, KCQ, BK>;
    auto kern = gemm_dmma_kernel<BM, BN, WM, WN, STAGES, KCP, KCQ, BK, MK>;
    cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::kSmem);
    for(int b0 = 0; b0 < batch; b0 += 65535)
    {
        GemmParams<double> p = p0;
        p.batch_base = b0;
        dim3 grid((unsigned)ceil_div(p.M, BM), (unsigned)ceil_div(p.N, BN),
                  (unsigned)std::min(65535, batch - b0));
        TimedLaunch tl(KernelClass::dmma, s, 2.0 * p.M * p.N * p.K * grid.z);
        kern<<<grid, Cfg::kThreads, Cfg::kSmem, s>>>(p);
    }
}

enum class DmmaTile
{
    t128x128 = 1,
    t128x64,
    t64x128,
    t64x64,
    t128x32,
    t32x128,
    t128x128k32,
    t128x64w64, // 4 warps of 64 x 32
    t64x128w64, // 4 warps of 32 x 64
    t64x64w64,  // 2 warps of 64 x 32
    t64x64k16   // as t64x64 with mma.sync m16n8k16
};
constexpr int kDmmaTiles = 11;

template <bool KCP, bool KCQ>
static void launch_dmma_tile(DmmaTile t, const GemmParams<double>& p, int batch, cudaStream_t s)
{
    switch(t)
    {
    case DmmaTile::t128x128: launch_dmma_cfg<128, 128, 32, 32, 3, KCP, KCQ>(p, batch, s); break;
    case DmmaTile::t128x64:  launch_dmma_cfg<128, 64, 32, 32, 3, KCP, KCQ>(p, batch, s); break;
    case DmmaTile::t64x128:  launch_dmma_cfg<64, 128, 32, 32, 3, KCP, KCQ>(p, batch, s); break;
    case DmmaTile::t64x64:   launch_dmma_cfg<64, 64, 32, 32, 4, KCP, KCQ>(p, batch, s); break;
    case DmmaTile::t128x32:  launch_dmma_cfg<128, 32, 32, 32, 4, KCP, KCQ>(p, batch, s); break;
    case DmmaTile::t32x128:  launch_dmma_cfg<32, 128, 32, 32, 4, KCP, KCQ>(p, batch, s); break;
    case DmmaTile::t128x128k32: launch_dmma_cfg<128, 128, 32, 32, 3, KCP, KCQ, 32>(p, batch, s); break;
    case DmmaTile::t128x64w64: launch_dmma_cfg<128, 64, 64, 32, 4, KCP, KCQ>(p, batch, s); break;
    case DmmaTile::t64x128w64: launch_dmma_cfg<64, 128, 32, 64, 4, KCP, KCQ>(p, batch, s); break;
    case DmmaTile::t64x64w64:  launch_dmma_cfg<64, 64, 64, 32, 4, KCP, KCQ>(p, batch, s); break;
    case DmmaTile::t64x64k16:  launch_dmma_cfg<64, 64, 32, 32, 4, KCP, KCQ, 16, 16>(p, batch, s); break;
    }
}

// Tile choice: the largest tile that still gives every SM work.  `full_m` / `full_n` force a
// tile that spans all M rows (N columns), which the in-place invA application needs.
static DmmaTile choose_dmma_tile(int64_t M, int64_t N, int64_t batch, int sms, bool full_m, bool full_n)
{
    auto tiles = [&](int bm, int bn) { return ceil_div(M, bm) * ceil_div(N, bn) * batch; };
    const int forced = tuning().dmma_force_tile;
    if(forced >= 1 && forced <= kDmmaTiles)
    {
        const DmmaTile f = (DmmaTile)forced;
        // a forced tile must still respect the in-place constraint of the invA leaves
        const bool spans_m = f == DmmaTile::t128x128 || f == DmmaTile::t128x64 || f == DmmaTile::t128x32
                             || f == DmmaTile::t128x128k32 || f == DmmaTile::t128x64w64;
        const bool spans_n = f == DmmaTile::t128x128 || f == DmmaTile::t64x128 || f == DmmaTile::t32x128
                             || f == DmmaTile::t128x128k32 || f == DmmaTile::t64x128w64;
        if((!full_m || spans_m) && (!full_n || spans_n))
            return f;
    }
    if(full_m)
    {
        if(tiles(128, 128) >= sms)
            return DmmaTile::t128x128;
        if(tiles(128, 64) >= sms)
            return DmmaTile::t128x64;
        return DmmaTile::t128x32;
    }
    if(full_n)
    {
        if(tiles(128, 128) >= sms)
            return DmmaTile::t128x128;
        if(tiles(64, 128) >= sms)
            return DmmaTile::t64x128;
        return DmmaTile::t32x128;
    }
    // 64 x 64 tiles (three CTAs per SM) measured fastest at every size with enough tiles;
    // the wider tiles remain reachable through dmma_big_tile_pct
    if(tiles(128, 128) * 100 >= (int64_t)sms * tuning().dmma_big_tile_pct)
        return tuning().dmma_big_bk == 32 ? DmmaTile::t128x128k32 : DmmaTile::t128x128;
    return DmmaTile::t64x64;
}

static void launch_gemm_dmma(const GemmParams<double>& p, int batch, cudaStream_t s, int sms,
                             bool full_m, bool full_n)
{
    if(p.M <= 0 || p.N <= 0)
        return;
    const DmmaTile t   = choose_dmma_tile(p.M, p.N, batch, sms, full_m, full_n);
    const bool     kcP = p.transP != 0, kcQ = p.transQ == 0;
    if(kcP && kcQ)
        launch_dmma_tile<true, true>(t, p, batch, s);
    else if(kcP)
        launch_dmma_tile<true, false>(t, p, batch, s);
    else if(kcQ)
        launch_dmma_tile<false, true>(t, p, batch, s);
    else
        launch_dmma_tile<false, false>(t, p, batch, s);
}

} // namespace rb200
