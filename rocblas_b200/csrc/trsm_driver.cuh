// Host side of the TRSM path: algorithm choice, workspace, and the launch sequence.
//
// Replaces rocblas_internal_trsm_launcher (library/src/blas3/rocblas_trsm_kernels.hpp:
// 3594-3987) and the host loops it drives (rocblas_trsm_left/right :269-1162,
// special_trsm_template :1164-1456, small substitution :3263-3589).  The reference picks
// among five algorithms and, for large k, runs a host loop of two GEMMs per 128-row block;
// for m=16384, n=4096 that is 256 GEMMs whose outputs are only 128 rows tall.  Here:
//
//   * k <= 512 and enough strips (or k <= 128): the one-CTA block solver (block_solve.cuh).
//   * otherwise: a recursive blocked solve on the 128-block grid of A.  A node of
//     blocks [b0, b1) splits at the middle block bm and runs
//         solve(first half, alpha); B2 := alpha_or_1 * B2 - op(A)21 * X1; solve(second half, 1)
//     so that half of all flops land in one large GEMM at the top level and the chain of
//     dependent launches is short.  Leaves apply the inverted 128x128 diagonal block (invA,
//     built by the fused trtri kernel or supplied through the _ex API) as an in-place GEMM.
//     Without workspace for invA the leaves use the block solver instead and the call
//     reports rocblas_status_perf_degraded, as the reference's backup path does
//     (rocblas_trsm_kernels.hpp:1926-1944).
//   * complex types: the same recursion with block-solver leaves (no invA) and the complex
//     DMMA tiles (gemm_cdmma.cuh) for the updates; trans C conjugates A in both.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <type_traits>

#include "block_solve.cuh"
#include "gemm_cdmma.cuh"
#include "gemm_dmma.cuh"
#include "gemm_tile.cuh"
#include "handle.hpp"
#include "trsm_chain.cuh"
#include "trtri_block.cuh"
#include "tuning.hpp"

namespace rb200
{

constexpr int kInvNB     = 128;   // invA block order (rocblas-functions.h:23112-23135)
constexpr int kMaxGridYZ = 65535;

// every kernel launch of the library bumps this (rocblas_b200_kernel_launch_count)
inline std::atomic<uint64_t> g_kernel_launches{0};
inline void count_launch()
{
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

// A full problem description (all entries of a batch share sizes and flags).
template <typename T>
struct TrsmProblem
{
    int         side_left, upper, trans, unit; // trans: op(A) is a transpose of A
    int         conj;                          // complex: op(A)'s entries conjugated
    int         m, n, batch;
    BatchPtr<T> A;
    int64_t     lda;
    BatchPtr<T> B;
    int64_t     ldb;
    Scalar<T>   alpha;
    BatchPtr<T> invA; // valid() when blocks are available (workspace or supplied)
    cudaStream_t stream;
    int         sm_count;
    int*        err_dev;  // device error word of the bounded waits (or nullptr)
    int         crt_pair_ok = 0; // the residue GEMM may run as CTA pairs on sm_count SMs that
                                 // are whole SM pairs (set beside a kernel placed in pairs)
    int         k() const { return side_left ? m : n; }
    // op(A) lower?
    int oplower() const { return (!upper) != (trans != 0); }
};

template <typename T>
static void ensure_smem_attr(const void* fn, size_t bytes)
{
    // cudaFuncSetAttribute is per device; calling it again is cheap and idempotent
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// ----------------------------------------------------------------------------------------
// GEMM dispatch: FP64 on the DMMA multistage tiles, FP32 on the FFMA tiles.  full_m / full_n:
// the tile must span all M rows / N columns (in-place application of an inverted block).
template <typename T>
static void launch_gemm(const GemmParams<T>& p0, int batch, cudaStream_t s, int sms = 148,
                        bool full_m = false, bool full_n = false)
{
    if(p0.M <= 0 || p0.N <= 0)
        return;
    if constexpr(std::is_same<T, double>::value)
    {
        launch_gemm_dmma(p0, batch, s, sms, full_m, full_n);
        for(int b0 = 0; b0 < batch; b0 += kMaxGridYZ)
            count_launch();
        return;
    }
    else if constexpr(is_cplx<T>::value)
    {
        launch_gemm_cdmma(p0, batch, s, sms);
        for(int b0 = 0; b0 < batch; b0 += kMaxGridYZ)
            count_launch();
        return;
    }
    else
    {
        const size_t smem = gemm_smem_bytes<T>();
        ensure_smem_attr<T>((const void*)gemm_tile_kernel<T>, smem);
        for(int b0 = 0; b0 < batch; b0 += kMaxGridYZ)
        {
            GemmParams<T> p = p0;
            p.batch_base    = b0;
            dim3 grid((unsigned)ceil_div(p.M, kGemmBM), (unsigned)ceil_div(p.N, kGemmBN),
                      (unsigned)std::min(kMaxGridYZ, batch - b0));
            gemm_tile_kernel<T><<<grid, kGemmThreads, smem, s>>>(p);
            count_launch();
        }
    }
}

template <typename T>
static void launch_trtri(const TrtriParams<T>& p0, int nblocks, int batch, cudaStream_t s)
{
    const size_t smem = trtri_smem_bytes<T>();
    ensure_smem_attr<T>((const void*)trtri_block_kernel<T>, smem);
    for(int b0 = 0; b0 < batch; b0 += kMaxGridYZ)
    {
        TrtriParams<T> p = p0;
        p.batch_base     = b0;
        dim3 grid((unsigned)nblocks, (unsigned)std::min(kMaxGridYZ, batch - b0));
        TimedLaunch tl(KernelClass::trtri, s, (double)grid.x * grid.y * kInvNB * kInvNB * kInvNB / 3.0);
        trtri_block_kernel<T><<<grid, kTrtriThreads, smem, s>>>(p);
        count_launch();
    }
}

// Block solver over a (sub)problem: A, B already offset to the sub-block.
template <typename T>
static void launch_block_solve(const TrsmProblem<T>& pr, int m, int n, BatchPtr<T> A,
                               BatchPtr<T> B, int first)
{
    BlockSolveParams<T> p;
    p.m = m;
    p.n = n;
    p.k = pr.side_left ? m : n;
    p.side_left = pr.side_left;
    // M = op(A) (side L) or op(A)^T (side R): M(i,j) = A(j,i) iff exactly one transpose
    p.tM   = (pr.trans != 0) != (pr.side_left == 0);
    // M lower <=> op(A) lower (side L) or op(A) upper (side R)
    const int mlower = pr.side_left ? pr.oplower() : !pr.oplower();
    p.rev  = !mlower;
    p.unit = pr.unit;
    p.conj = pr.conj;
    p.A = A;
    p.lda = pr.lda;
    p.B = B;
    p.ldb = pr.ldb;
    p.ualpha = pr.alpha;
    p.first  = first;
    const int    ncols   = pr.side_left ? n : m;
    const int    nstrips = (int)ceil_div(ncols, kBsW);
    const size_t smem    = block_solve_smem_bytes<T>(p.k);
    ensure_smem_attr<T>((const void*)block_solve_kernel<T>, block_solve_smem_bytes<T>(block_solve_max_k<T>()));
    for(int b0 = 0; b0 < pr.batch; b0 += kMaxGridYZ)
    {
        p.batch_base = b0;
        dim3 grid((unsigned)nstrips, (unsigned)std::min(kMaxGridYZ, pr.batch - b0));
        block_solve_kernel<T><<<grid, kBsThreads, smem, pr.stream>>>(p);
        count_launch();
    }
}

// ---- recursive blocked solve --------------------------------------------------------------
// The FP32 solve's trailing updates on the int8 slice engine (sliced_driver.cuh, later in this
// translation unit): C := beta C - op(A) X (side L) or C - X op(A) (side R); false if not run.
template <typename T>
static bool sliced_trsm_update(const TrsmProblem<T>& q, int c_lo, int c_hi, int x_lo, int x_hi,
                               int first, int S, int moduli, void* ws, int* err);
static size_t sliced_gemm_workspace_bytes(int64_t M, int64_t N, int64_t K, int S);

template <typename T>
struct Recursive
{
    const TrsmProblem<T>& pr;
    int                   k, nblk;
    // FP32: workspace of the trailing updates on the int8 slice engine (nullptr: FFMA tiles)
    void*                 slice_ws = nullptr;
    int                   slice_S  = 0;

    int row_of(int b) const { return std::min(b * kInvNB, k); }

    // op(A)[i0:i0+mi, j0:j0+nj] as a GEMM operand: pointer shift and transpose flag
    void opA_block(int i0, int j0, BatchPtr<T>& ptr, int& trans) const
    {
        if(!pr.trans)
        {
            ptr   = pr.A.shifted(i0 + (int64_t)j0 * pr.lda);
            trans = 0;
        }
        else
        {
            ptr   = pr.A.shifted(j0 + (int64_t)i0 * pr.lda);
            trans = 1;
        }
    }

    void leaf(int b, int first) const
    {
        const int r0 = row_of(b), bs = row_of(b + 1) - r0;
        if(!pr.invA.valid())
        {
            // no invA: solve the diagonal block with the block solver
            BatchPtr<T> Ab = pr.A.shifted(r0 + (int64_t)r0 * pr.lda);
            if(pr.side_left)
                launch_block_solve<T>(pr, bs, pr.n, Ab, pr.B.shifted(r0), first);
            else
                launch_block_solve<T>(pr, pr.m, bs, Ab, pr.B.shifted((int64_t)r0 * pr.ldb), first);
            return;
        }
        GemmParams<T> g{};
        BatchPtr<T>   inv = pr.invA.shifted((int64_t)b * kInvNB * kInvNB);
        const int     tri = pr.upper ? kTriUpper : kTriLower;
        if(pr.side_left)
        {
            // B_b := s * op(inv_b) * B_b, in place (tile spans all bs <= 128 rows)
            g.M = bs; g.N = pr.n; g.K = bs;
            g.P = inv; g.ldp = kInvNB; g.transP = pr.trans; g.triP = tri;
            g.Q = pr.B.shifted(r0); g.ldq = pr.ldb; g.transQ = 0; g.triQ = kTriNone;
            g.C = g.Q; g.ldc = pr.ldb;
        }
        else
        {
            // B_b := s * B_b * op(inv_b), in place (tile spans all bs <= 128 columns)
            g.M = pr.m; g.N = bs; g.K = bs;
            g.P = pr.B.shifted((int64_t)r0 * pr.ldb); g.ldp = pr.ldb; g.transP = 0; g.triP = kTriNone;
            g.Q = inv; g.ldq = kInvNB; g.transQ = pr.trans; g.triQ = tri;
            g.C = g.P; g.ldc = pr.ldb;
        }
        g.a_imm = T(1); g.a_user = first;
        g.b_imm = T(0); g.b_user = 0;
        g.ualpha = pr.alpha; g.zero_guard = 1;
        launch_gemm<T>(g, pr.batch, pr.stream, pr.sm_count, pr.side_left != 0, pr.side_left == 0);
    }

    // C := beta * C - opA(rows i0.., cols j0..) * X  (side L)   or
    // C := beta * C - X * opA(rows i0.., cols j0..)  (side R)
    void update(int c_lo, int c_hi, int x_lo, int x_hi, int first) const
    {
        if constexpr(std::is_same<T, float>::value)
        {
            if(slice_ws && x_hi - x_lo >= tuning().strsm_sliced_min_k
               && sliced_trsm_update<T>(pr, c_lo, c_hi, x_lo, x_hi, first, slice_S, 0, slice_ws, pr.err_dev))
                return;
        }
        GemmParams<T> g{};
        if(pr.side_left)
        {
            g.M = c_hi - c_lo; g.N = pr.n; g.K = x_hi - x_lo;
            opA_block(c_lo, x_lo, g.P, g.transP); g.ldp = pr.lda; g.triP = kTriNone;
            g.conjP = pr.conj;
            g.Q = pr.B.shifted(x_lo); g.ldq = pr.ldb; g.transQ = 0; g.triQ = kTriNone;
            g.C = pr.B.shifted(c_lo); g.ldc = pr.ldb;
        }
        else
        {
            g.M = pr.m; g.N = c_hi - c_lo; g.K = x_hi - x_lo;
            g.P = pr.B.shifted((int64_t)x_lo * pr.ldb); g.ldp = pr.ldb; g.transP = 0; g.triP = kTriNone;
            opA_block(x_lo, c_lo, g.Q, g.transQ); g.ldq = pr.lda; g.triQ = kTriNone;
            g.conjQ = pr.conj;
            g.C = pr.B.shifted((int64_t)c_lo * pr.ldb); g.ldc = pr.ldb;
        }
        g.a_imm = T(-1); g.a_user = 0;
        g.b_imm = T(1); g.b_user = first;
        g.ualpha = pr.alpha; g.zero_guard = 1;
        launch_gemm<T>(g, pr.batch, pr.stream, pr.sm_count);
    }

    void solve(int b0, int b1, int first) const
    {
        if(b1 - b0 == 1)
        {
            leaf(b0, first);
            return;
        }
        const int bm = (b0 + b1) / 2;
        const int r0 = row_of(b0), rm = row_of(bm), r1 = row_of(b1);
        // blocks are solved in increasing order when op(A) is lower (side L) or upper (side R)
        const bool forward = pr.side_left ? pr.oplower() : !pr.oplower();
        if(forward)
        {
            solve(b0, bm, first);
            update(rm, r1, r0, rm, first);
            solve(bm, b1, 0);
        }
        else
        {
            solve(bm, b1, first);
            update(r0, rm, rm, r1, first);
            solve(b0, bm, 0);
        }
    }
};

// Build invA for all diagonal blocks of A (k x k) into `inv` (ld 128, stride 128*128).
template <typename T>
static void build_invA(const TrsmProblem<T>& pr, BatchPtr<T> inv)
{
    const int      k = pr.k();
    TrtriParams<T> t{};
    t.k = k;
    t.nb = kInvNB;
    t.A = pr.A;
    t.lda = pr.lda;
    t.inv = inv;
    t.ldinv = kInvNB;
    t.inv_block_stride = (int64_t)kInvNB * kInvNB;
    t.upper = pr.upper;
    t.unit = pr.unit;
    launch_trtri<T>(t, (int)ceil_div(k, kInvNB), pr.batch, pr.stream);
}

enum class Algo
{
    block,
    recursive
};

template <typename T>
static Algo choose_algo(const TrsmProblem<T>& pr)
{
    const Tuning& t = tuning();
    const int     k = pr.k();
    if(k > std::min(t.block_max_k, block_solve_max_k<T>()))
        return Algo::recursive;
    if(k <= t.block_always_k)
        return Algo::block;
    const int64_t ncols   = pr.side_left ? pr.n : pr.m;
    const int64_t nstrips = ceil_div(ncols, kBsW) * (int64_t)pr.batch;
    return nstrips * 100 >= (int64_t)pr.sm_count * t.block_min_strips_pct ? Algo::block
                                                                         : Algo::recursive;
}

// The recursive solve with few right-hand sides runs as one chain launch (trsm_chain.cuh)
// when invA is available: FP64, more than one 128-row block, at most chain_max_cols columns.
template <typename T>
static bool use_chain(const TrsmProblem<T>& pr)
{
    if(is_cplx<T>::value || choose_algo(pr) != Algo::recursive)
        return false;
    const int64_t ncols = pr.side_left ? pr.n : pr.m;
    const int64_t limit = std::is_same<T, double>::value ? tuning().chain_max_cols
                                                         : tuning().chain_max_cols_f32;
    return pr.k() > kInvNB && ncols <= limit;
}

template <typename T>
static ChainShape chain_shape_of(const TrsmProblem<T>& pr)
{
    const int ncols = pr.side_left ? pr.n : pr.m;
    const int t     = tuning().chain_w;
    const int w     = t == 32 || t == 64 ? t : (ncols <= 32 ? 32 : 64);
    return chain_shape(pr.k(), ncols, pr.batch, w);
}

__global__ void chain_set_counter_kernel(int* counter, int v)
{
    counter[0] = v; // low word of the 8-byte claim counter; the launch's memset zeroed both
}

// Chain solve of the diagonal blocks [b0, b1) of pr (all of it: 0, nblk) with invA available:
// `first` as in Recursive::solve; `ws` holds chain_workspace_bytes of the sub-problem.
template <typename T>
// cluster2: launch the CTAs as clusters of two (placement only: each pair takes both SMs of an SM
// pair, so that a CTA-pair kernel beside it finds the other SMs in whole pairs)
static void launch_chain_sub(const TrsmProblem<T>& pr, int b0, int b1, int first, int w, void* ws,
                             bool cluster2 = false)
{
    const int        r0    = b0 * kInvNB;
    const int        kk    = std::min(b1 * kInvNB, pr.k()) - r0;
    const int        ncols = pr.side_left ? pr.n : pr.m;
    const ChainShape cs    = chain_shape(kk, ncols, pr.batch, w);
    int*             flags = reinterpret_cast<int*>(ws);
    cudaMemsetAsync(flags, 0, chain_workspace_bytes(cs), pr.stream);
    ChainParams<T> c{};
    c.A       = pr.A.shifted(r0 + (int64_t)r0 * pr.lda);
    c.lda     = pr.lda;
    c.invA    = pr.invA.shifted((int64_t)b0 * kInvNB * kInvNB);
    c.B       = pr.B.shifted(pr.side_left ? (int64_t)r0 : (int64_t)r0 * pr.ldb);
    c.ldb     = pr.ldb;
    c.k       = kk;
    c.ncols   = ncols;
    c.nb      = cs.nb;
    c.ns      = cs.ns;
    c.forward = pr.side_left ? pr.oplower() : !pr.oplower();
    c.items   = cs.items;
    c.systems = pr.batch;
    c.alpha   = pr.alpha;
    c.first   = first;
    c.flags   = flags;
    // the 8-byte claim counter and the error word follow the flags
    const size_t tail = ((size_t)cs.items * sizeof(int) + 7) / 8 * 8;
    c.counter = reinterpret_cast<int*>(reinterpret_cast<char*>(flags) + tail);
    // the error word: the handle's, else a slot after the counter
    c.error       = pr.err_dev ? pr.err_dev : c.counter + 2;
    c.wait_cycles = 1ll << tuning().wait_cycles_log2;
    if(tuning().chain_first_item > 0)
    {
        // failure injection (tests): the items before it are never claimed, so their flags
        // stay 0 and every wait on them runs out
        chain_set_counter_kernel<<<1, 1, 0, pr.stream>>>(c.counter, tuning().chain_first_item);
        count_launch();
    }
    // KCP: M's column index (K) is contiguous in memory when M(r, c) = A(c, r)
    const bool tM  = pr.trans != (pr.side_left ? 0 : 1);
    const bool kcq = pr.side_left != 0;
    if(w == 16)
        launch_chain_w<T, 16, false>(c, tM, kcq, pr.sm_count, cs.items, pr.stream, cluster2);
    else if(w == 32)
        launch_chain_w<T, 32, false>(c, tM, kcq, pr.sm_count, cs.items, pr.stream, cluster2);
    else
        launch_chain_w<T, 64, false>(c, tM, kcq, pr.sm_count, cs.items, pr.stream, cluster2);
    count_launch();
}

// Workspace bytes the call wants: invA for the recursive path unless supplied, then the
// chain's flags when the chain runs.
template <typename T>
static size_t trsm_invA_bytes(const TrsmProblem<T>& pr, bool have_supplied_invA)
{
    // complex solves use block-solver leaves and need no invA
    if(is_cplx<T>::value || choose_algo(pr) != Algo::recursive || have_supplied_invA)
        return 0;
    return (size_t)kInvNB * (size_t)pr.k() * sizeof(T) * (size_t)pr.batch;
}

// The FP32 recursive solve's slice workspace: the largest trailing update (the top node's)
// when its updates run on the int8 slice engine (strsm_slices > 0, one system, no chain).
template <typename T>
static size_t strsm_slice_bytes(const TrsmProblem<T>& pr)
{
    if constexpr(!std::is_same<T, float>::value)
        return 0;
    else
    {
        const Tuning& t = tuning();
        if(t.strsm_slices <= 0 || pr.batch != 1 || choose_algo(pr) != Algo::recursive || use_chain(pr))
            return 0;
        const int64_t k    = pr.k();
        const int64_t nblk = ceil_div(k, kInvNB);
        const int64_t rm   = std::min<int64_t>(nblk / 2 * kInvNB, k);
        const int64_t big  = std::max(rm, k - rm);
        if(big < t.strsm_sliced_min_k)
            return 0;
        return pr.side_left ? sliced_gemm_workspace_bytes(big, pr.n, big, t.strsm_slices)
                            : sliced_gemm_workspace_bytes(pr.m, big, big, t.strsm_slices);
    }
}

template <typename T>
static size_t trsm_workspace_bytes(const TrsmProblem<T>& pr, bool have_supplied_invA)
{
    size_t b = trsm_invA_bytes(pr, have_supplied_invA);
    if(use_chain(pr))
        b = (b + 255) / 256 * 256 + chain_workspace_bytes(chain_shape_of(pr));
    else if(const size_t sl = strsm_slice_bytes(pr))
        b = (b + 255) / 256 * 256 + sl;
    return b;
}

// Run the solve.  `ws` is the workspace of trsm_workspace_bytes (nullptr => without it: the
// supplied invA if any, else the degraded path).
template <typename T>
static void trsm_run(TrsmProblem<T> pr, void* ws, bool supplied_invA)
{
    if(choose_algo(pr) == Algo::block)
    {
        launch_block_solve<T>(pr, pr.m, pr.n, pr.A, pr.B, 1);
        return;
    }
    const int k = pr.k();
    if constexpr(is_cplx<T>::value)
    {
        pr.invA = BatchPtr<T>{};
    }
    else
    {
        if(!supplied_invA)
        {
            if(ws)
            {
                BatchPtr<T> inv;
                inv.base   = reinterpret_cast<T*>(ws);
                inv.stride = (int64_t)kInvNB * k;
                build_invA<T>(pr, inv);
                pr.invA = inv;
            }
            else
                pr.invA = BatchPtr<T>{};
        }
        if(ws && pr.invA.valid() && use_chain(pr))
        {
            const size_t off = (trsm_invA_bytes(pr, supplied_invA) + 255) / 256 * 256;
            launch_chain_sub<T>(pr, 0, (int)ceil_div(k, kInvNB), 1, chain_shape_of(pr).w,
                                reinterpret_cast<char*>(ws) + off);
            return;
        }
    }
    Recursive<T> rec{pr, k, (int)ceil_div(k, kInvNB)};
    if(ws && pr.err_dev && strsm_slice_bytes(pr))
    {
        rec.slice_ws = reinterpret_cast<char*>(ws) + (trsm_invA_bytes(pr, supplied_invA) + 255) / 256 * 256;
        rec.slice_S  = tuning().strsm_slices;
    }
    rec.solve(0, rec.nblk, 1);
}

} // namespace rb200
