// Variable-size batch with systems of any order: the systems with k > 512 go through the
// chain solve (trsm_chain.cuh) in one persistent launch per combination of (tM, side) and strip
// width (32 columns for systems with at most 32 right-hand sides, else 64), using an
// inverted-diagonal-block array (invA, the rocblas_trsm_ex format) the caller supplies per
// system; the systems with k <= 512 take the size classes of the strip solver (vbatched.cuh).
//
// A single-CTA prepass builds the chain's tables on the device from the descriptors, so the
// call needs no host synchronisation and can be captured in a CUDA graph:
//   1. classify every k > 512 descriptor (valid, invA present, right-hand sides within the
//      caller's bound) into its combination c = 2 tM + side_left + 4 wide (wide: more than 32
//      right-hand sides, strips of 64) and its block count nb;
//   2. counting-sort the systems by (c ascending, nb descending) into ChainSys records;
//   3. per combination: vP = prefix sums of the strips ns over its sorted systems,
//      vcnt[j] = systems with nb > j (a prefix of the sorted order, since nb descends),
//      vL[j] = first item id of level j = sum over j' < j of vP[vcnt[j']];
//   4. per combination a header with its table pointers and its slice of the flag array.
#pragma once
#include "trsm_chain.cuh"
#include "vbatched.cuh"

namespace rb200
{

constexpr int kChainVbMaxNB   = 256; // chain systems up to k = 32768
constexpr int kChainVbCombos  = 8;   // (tM, side) x strip width
constexpr int kChainVbW       = 32;  // the narrow strip width (the flag bound assumes it)
constexpr int kChainVbWideW   = 64;  // the strip width of systems with more than 32 columns
constexpr int kChainVbMinK    = kBlockSolveMaxK; // k above this goes to the chain

__host__ __device__ constexpr int chain_vb_width(int combo)
{
    return combo >= 4 ? kChainVbWideW : kChainVbW;
}

template <typename T>
struct ChainVbWork
{
    ChainVbHeader<T>*   hdr;      // [kChainVbCombos]
    ChainSys<T>*        sys;      // [count]
    int*                P;        // [count + kChainVbCombos]: combination c's array starts at start_c + c
    int*                G;        // [count + 1]: global prefix (scratch)
    int*                cnt;      // [kChainVbCombos][kChainVbMaxNB]
    int64_t*            L;        // [kChainVbCombos][kChainVbMaxNB + 1]
    int*                flags;    // [flag_cap]
    int64_t             flag_cap;
    unsigned long long* counters; // [kChainVbCombos]
    int*                invalid;  // [1]
};

__device__ __forceinline__ int chain_vb_combo(const VbProblem& p)
{
    const int left  = p.side == kLeft;
    const int tM    = (p.trans != kOpN) != (left ? 0 : 1);
    const int ncols = left ? p.n : p.m;
    return 2 * tM + left + (ncols > kChainVbW ? 4 : 0);
}

template <typename T>
__global__ void __launch_bounds__(kVbPrepThreads)
    chain_vb_prepass_kernel(const VbProblem* probs, const T* const* invs, int count, int max_k,
                            int max_n, ChainVbWork<T> ws)
{
    __shared__ int hist[kChainVbCombos][kChainVbMaxNB + 1];
    __shared__ int cursor[kChainVbCombos][kChainVbMaxNB + 1];
    __shared__ int start[kChainVbCombos + 1];
    __shared__ int part[kVbPrepThreads];
    __shared__ int64_t items[kChainVbCombos];
    const int tid = threadIdx.x;

    for(int i = tid; i < kChainVbCombos * (kChainVbMaxNB + 1); i += kVbPrepThreads)
        (&hist[0][0])[i] = 0;
    __syncthreads();

    // classification: -1 not for the chain (k <= 512 or nothing to do), -2 invalid, else
    // combination * 1024 + nb
    auto classify = [&](int i, VbProblem& p) -> int {
        p = probs[i];
        const int k = p.side == kLeft ? p.m : p.n;
        if(k <= kChainVbMinK)
            return -1;
        const int ncols = p.side == kLeft ? p.n : p.m;
        if(!vb_valid(p, max_k) || k > kChainVbMaxNB * kChainNB || ncols > max_n)
            return -2;
        if(p.m == 0 || p.n == 0)
            return -1;
        if(!invs[i])
            return -2;
        return chain_vb_combo(p) * 1024 + (int)ceil_div(k, kChainNB);
    };

    int bad = 0;
    for(int i = tid; i < count; i += kVbPrepThreads)
    {
        VbProblem p;
        const int c = classify(i, p);
        if(c == -2)
            ++bad;
        else if(c >= 0)
            atomicAdd(&hist[c >> 10][c & 1023], 1);
    }
    if(bad)
        atomicAdd(ws.invalid, bad);
    __syncthreads();

    // bucket order: combination ascending, nb descending
    if(tid == 0)
    {
        int run = 0;
        for(int c = 0; c < kChainVbCombos; ++c)
        {
            start[c] = run;
            for(int nb = kChainVbMaxNB; nb >= 1; --nb)
            {
                cursor[c][nb] = run;
                run += hist[c][nb];
            }
        }
        start[kChainVbCombos] = run;
    }
    __syncthreads();

    for(int i = tid; i < count; i += kVbPrepThreads)
    {
        VbProblem p;
        const int c = classify(i, p);
        if(c < 0)
            continue;
        const int   pos  = atomicAdd(&cursor[c >> 10][c & 1023], 1);
        const int   left = p.side == kLeft;
        const int   k    = left ? p.m : p.n;
        ChainSys<T> q;
        q.A       = reinterpret_cast<const T*>(p.A);
        q.invA    = invs[i];
        q.B       = reinterpret_cast<T*>(p.B);
        q.lda     = p.lda;
        q.ldb     = p.ldb;
        q.k       = k;
        q.ncols   = left ? p.n : p.m;
        q.nb      = c & 1023;
        q.ns      = (int)ceil_div(q.ncols, chain_vb_width(c >> 10));
        const int oplower = (p.uplo == kLower) != (p.trans != kOpN);
        q.forward = left ? oplower : !oplower;
        q.pad     = 0;
        ws.sys[pos] = q;
    }
    __syncthreads();

    // global exclusive prefix G of ns over the sorted systems (chunked Hillis-Steele scan)
    const int E     = start[kChainVbCombos];
    const int chunk = (E + kVbPrepThreads - 1) / kVbPrepThreads;
    const int lo = min(E, tid * chunk), hi = min(E, lo + chunk);
    int       sum = 0;
    for(int i = lo; i < hi; ++i)
        sum += ws.sys[i].ns;
    part[tid] = sum;
    __syncthreads();
    for(int off = 1; off < kVbPrepThreads; off <<= 1)
    {
        const int v = tid >= off ? part[tid - off] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = part[tid] - sum;
    for(int i = lo; i < hi; ++i)
    {
        ws.G[i] = run;
        run += ws.sys[i].ns;
    }
    if(tid == kVbPrepThreads - 1)
        ws.G[E] = part[tid];
    __syncthreads();

    // per combination: relative prefix vP (n_c + 1 entries at start_c + c)
    for(int i = tid; i < E + kChainVbCombos; i += kVbPrepThreads)
    {
        // entry i of P belongs to combination c with start_c + c <= i <= start_{c+1} + c
        int c = 0;
        while(c < kChainVbCombos - 1 && i > start[c + 1] + c)
            ++c;
        const int gi = i - c; // index into G
        ws.P[i] = ws.G[gi] - ws.G[start[c]];
    }
    __syncthreads();

    // per combination: vcnt, vL, header
    if(tid < kChainVbCombos)
    {
        const int c     = tid;
        int       maxnb = 0;
        for(int nb = kChainVbMaxNB; nb >= 1 && !maxnb; --nb)
            if(hist[c][nb])
                maxnb = nb;
        int*       cnt = ws.cnt + c * kChainVbMaxNB;
        int64_t*   L   = ws.L + c * (kChainVbMaxNB + 1);
        const int* P   = ws.P + start[c] + c;
        int        cum = 0;
        for(int j = maxnb - 1; j >= 0; --j)
        {
            cum += hist[c][j + 1]; // systems with nb >= j + 1
            cnt[j] = cum;
        }
        int64_t lr = 0;
        for(int j = 0; j < maxnb; ++j)
        {
            L[j] = lr;
            lr += P[cnt[j]];
        }
        L[maxnb]   = lr;
        items[c]   = lr;
        ChainVbHeader<T> h;
        h.vsys  = ws.sys + start[c];
        h.vP    = P;
        h.vcnt  = cnt;
        h.vL    = L;
        h.flags = nullptr;
        h.maxnb = maxnb;
        h.pad   = 0;
        ws.hdr[c] = h;
    }
    __syncthreads();
    if(tid == 0)
    {
        int64_t fb = 0;
        for(int c = 0; c < kChainVbCombos; ++c)
        {
            ws.hdr[c].flags = ws.flags + fb;
            fb += items[c];
        }
        if(fb > ws.flag_cap)
        {
            // more items than the caller's bounds allow for: solve nothing, report them all
            for(int c = 0; c < kChainVbCombos; ++c)
                ws.hdr[c].maxnb = 0;
            atomicAdd(ws.invalid, E);
        }
    }
}

// Workspace of the chain part of a variable batch of `count` systems with k <= max_k and at
// most max_n right-hand sides: the flag array is sized by that bound.
struct ChainVbLayout
{
    size_t hdr, sys, P, G, cnt, L, counters, invalid, flags, total;
    int64_t flag_cap;
};

template <typename T>
inline ChainVbLayout chain_vb_layout(int count, int max_k, int max_n)
{
    auto a256 = [](size_t b) { return (b + 255) & ~size_t(255); };
    ChainVbLayout l{};
    size_t off = 0;
    l.hdr = off;      off += a256(sizeof(ChainVbHeader<T>) * kChainVbCombos);
    l.sys = off;      off += a256(sizeof(ChainSys<T>) * (size_t)std::max(count, 1));
    l.P = off;        off += a256(sizeof(int) * ((size_t)count + kChainVbCombos));
    l.G = off;        off += a256(sizeof(int) * ((size_t)count + 1));
    l.cnt = off;      off += a256(sizeof(int) * kChainVbCombos * kChainVbMaxNB);
    l.L = off;        off += a256(sizeof(int64_t) * kChainVbCombos * (kChainVbMaxNB + 1));
    l.counters = off; off += a256(sizeof(unsigned long long) * kChainVbCombos + 2 * sizeof(int));
    l.invalid = l.counters + sizeof(unsigned long long) * kChainVbCombos;
    l.flag_cap = (int64_t)count * ceil_div(std::max(max_k, 1), kChainNB)
                 * ceil_div(std::max(max_n, 1), kChainVbW);
    l.flags = off;    off += a256(sizeof(int) * (size_t)l.flag_cap);
    l.total = off;
    return l;
}

} // namespace rb200
