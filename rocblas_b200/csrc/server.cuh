// Continuous-batching TRSM server (rocblas_b200_server_* in rocblas_b200_ext.h).
//
// The host loop of the serving form, in C++ so that the per-request host work is a few
// microseconds (copies of the request's data into the server's memory, its descriptor, and
// for a request that brings its own large A, the inversion of its diagonal blocks):
//
//   * memory: one device arena of the HBM budget (first-fit, coalescing free list, 256-byte
//     blocks). Resident matrices and their invA live in it for the server's life; a request
//     holds its B (and its own A and invA) from admission to completion. Admission is in
//     arrival order while the request's blocks fit under the budget;
//   * continuous batching: admitted requests of one dtype collect in a window; a collection
//     is formed when a stream is free and the oldest request has waited `window` (or the
//     collection is full, or no more requests will come), so while the GPU is busy the next
//     collection grows. A collection is one variable-size batched solve
//     (rocblas_b200_?trsm_vbatched_ex: strip solver for k <= 512, chain solve above, with each
//     system's resident or fresh invA) on its stream, after the copies of its requests' data;
//   * completion: one event per collection, polled in stream order; the latency of a request
//     is completion - arrival on the host's steady clock.
// What a request computes depends only on that request (its sizes, data and route), never on
// the collection it lands in, so results are bitwise the same alone and in the mix.
#pragma once
#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <vector>

#include "../../include/rocblas_b200_ext.h"
#include "handle.hpp"
#include "trsm_driver.cuh"
#include "vbatched_chain.cuh"

namespace rb200
{

// First-fit arena over one device allocation.
class DeviceArena
{
public:
    bool init(size_t bytes)
    {
        bytes = (bytes + 255) & ~size_t(255);
        if(cudaMalloc(&base_, bytes) != cudaSuccess)
        {
            cudaGetLastError();
            base_ = nullptr;
            return false;
        }
        size_ = bytes;
        free_.clear();
        free_[0] = bytes;
        return true;
    }
    void release()
    {
        if(base_)
            cudaFree(base_);
        base_ = nullptr;
        size_ = 0;
        free_.clear();
    }
    static size_t round(size_t b) { return (std::max<size_t>(b, 1) + 255) & ~size_t(255); }
    // nullptr if no free block is large enough
    void* alloc(size_t bytes)
    {
        bytes = round(bytes);
        for(auto it = free_.begin(); it != free_.end(); ++it)
        {
            if(it->second < bytes)
                continue;
            const size_t off = it->first, sz = it->second;
            free_.erase(it);
            if(sz > bytes)
                free_[off + bytes] = sz - bytes;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return base_ + off;
        }
        return nullptr;
    }
    void free(void* p, size_t bytes)
    {
        if(!p)
            return;
        bytes      = round(bytes);
        size_t off = (size_t)(reinterpret_cast<char*>(p) - base_);
        used_ -= bytes;
        auto next = free_.lower_bound(off);
        if(next != free_.end() && off + bytes == next->first)
        {
            bytes += next->second;
            next = free_.erase(next);
        }
        if(next != free_.begin())
        {
            auto prev = std::prev(next);
            if(prev->first + prev->second == off)
            {
                prev->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }
    void   reset_peak() { peak_ = used_; }

private:
    char*                    base_ = nullptr;
    size_t                   size_ = 0;
    size_t                   used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;
};

struct ServerRequestC // layout of rocblas_b200_request
{
    double      arrival_s;
    int         dtype; // rocblas_datatype: f32_r 151, f64_r 152
    int         m, n;
    int         resident;
    const void* B_src;
    const void* A_src;
    int         lda_src;
    int         pad;
    void*       X_dst;
};

struct ServerStatsC // layout of rocblas_b200_server_stats
{
    double  wall_s;
    int64_t peak_bytes;
    int64_t collections;
    int64_t largest_collection;
    int64_t kernel_launches;
};

// One collection's arriving data in one launch (instead of a copy call per request): for each
// request its B (m x n, contiguous from B_src) and, for a fresh A, the lower triangle of A
// (m x m from A_src with leading dimension lda_src; the solve and the inversion read nothing
// else) into the request's arena blocks.  Work items are blocks of kGatherCols columns, B's
// first and then A's; item ranges per request come from the exclusive prefix array.
constexpr int kGatherCols = 32;

struct GatherReq
{
    const void* srcB;
    void*       dstB;
    const void* srcA; // nullptr: no A to copy
    void*       dstA;
    int64_t     lda_src;
    int         m, n;
    int         itemsB, pad;
};

template <typename T>
__global__ void __launch_bounds__(256) server_gather_kernel(const GatherReq* reqs, const int* prefix,
                                                            int cnt)
{
    const int bid = blockIdx.x;
    // the request of this item: the last r with prefix[r] <= bid
    int lo = 0, hi = cnt - 1;
    while(lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if(prefix[mid] <= bid)
            lo = mid;
        else
            hi = mid - 1;
    }
    const GatherReq q    = reqs[lo];
    const int       item = bid - prefix[lo];
    const bool      isB  = item < q.itemsB;
    const int       c0   = (isB ? item : item - q.itemsB) * kGatherCols;
    const int       c1   = min(isB ? q.n : q.m, c0 + kGatherCols);
    const T*        src  = reinterpret_cast<const T*>(isB ? q.srcB : q.srcA);
    T*              dst  = reinterpret_cast<T*>(isB ? q.dstB : q.dstA);
    const int64_t   lds  = isB ? q.m : q.lda_src;
    for(int c = c0; c < c1; ++c)
    {
        const T* s = src + (int64_t)c * lds;
        T*       d = dst + (int64_t)c * q.m;
        for(int r = (isB ? 0 : c) + (int)threadIdx.x; r < q.m; r += blockDim.x)
            d[r] = s[r];
    }
}

// The collection solve: rocblas_b200_?trsm_vbatched_ex on the lane's handle with alpha 1
// (dtype kF64 or kF32; invs is a device array of per-system invA pointers).
typedef rocblas_status (*ServerSolveFn)(_rocblas_handle* h, int dtype,
                                        const rocblas_b200_trsm_problem* probs, const void* invs,
                                        int count, int max_k, int max_n);

class TrsmServerCore
{
public:
    static constexpr int kF32 = 151, kF64 = 152;
    // staging per request: its descriptor and invA pointer, for a fresh A the batched trtri's A
    // pointer, invA pointer, order and leading dimension, then (8-byte aligned) its gather
    // record and its item offset
    static constexpr size_t kStagePerRequest = sizeof(VbProblem) + sizeof(void*) + 2 * sizeof(void*)
                                               + sizeof(int64_t) + sizeof(int) + sizeof(GatherReq)
                                               + sizeof(int);
    static constexpr size_t kStageSlack = 64; // alignment of the gather records, prefix[cnt]
    static size_t gather_offset(int cnt)
    {
        const size_t o = (size_t)cnt * (sizeof(VbProblem) + 3 * sizeof(void*) + sizeof(int64_t)
                                        + sizeof(int));
        return (o + 15) & ~size_t(15);
    }

    explicit TrsmServerCore(ServerSolveFn solve) : solve_(solve) {}

    ~TrsmServerCore() { destroy(); }

    rocblas_status create(size_t budget, int n_streams, double window_us, int max_batch, int device,
                          int sms)
    {
        if(n_streams < 1 || n_streams > 16 || max_batch < 1 || budget == 0)
            return rocblas_status_invalid_size;
        if(!arena_.init(budget))
            return rocblas_status_memory_error;
        budget_     = budget;
        arena_size_ = budget;
        window_s_  = std::max(0.0, window_us) * 1e-6;
        max_batch_ = max_batch;
        for(int i = 0; i < n_streams; ++i)
        {
            Lane l;
            if(cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking) != cudaSuccess)
                return rocblas_status_internal_error;
            l.h           = new _rocblas_handle();
            l.h->device   = device;
            l.h->sm_count = sms;
            l.h->stream   = l.stream;
            if(cudaMalloc(&l.h->err_dev, 256) != cudaSuccess)
                return rocblas_status_memory_error;
            cudaMemset(l.h->err_dev, 0, 256);
            const size_t stage = (size_t)max_batch * kStagePerRequest + kStageSlack;
            if(cudaMallocHost(&l.host_stage, stage) != cudaSuccess
               || cudaMalloc(&l.dev_stage, stage) != cudaSuccess)
                return rocblas_status_memory_error;
            if(cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) != cudaSuccess)
                return rocblas_status_internal_error;
            lanes_.push_back(l);
        }
        return rocblas_status_success;
    }

    void destroy()
    {
        for(auto& l : lanes_)
        {
            if(l.stream)
                cudaStreamSynchronize(l.stream);
            if(l.h)
            {
                l.h->free_mem();
                if(l.h->err_dev)
                    cudaFree(l.h->err_dev);
                delete l.h;
            }
            if(l.host_stage)
                cudaFreeHost(l.host_stage);
            if(l.dev_stage)
                cudaFree(l.dev_stage);
            if(l.done)
                cudaEventDestroy(l.done);
            if(l.stream)
                cudaStreamDestroy(l.stream);
        }
        lanes_.clear();
        residents_.clear();
        arena_.release();
    }

    // resident matrix: a copy of A (m x m, lower, ld lda) and its invA, in the arena
    rocblas_status add_resident(int dtype, int m, const void* A, int lda, int* index)
    {
        if((dtype != kF32 && dtype != kF64) || m < 1 || lda < m)
            return rocblas_status_invalid_size;
        if(!A || !index)
            return rocblas_status_invalid_pointer;
        const size_t es = dtype == kF64 ? 8 : 4;
        Resident     r{dtype, m, nullptr, nullptr, (size_t)m * m * es, (size_t)kInvNB * m * es};
        if(arena_.used() + DeviceArena::round(r.a_bytes) + DeviceArena::round(r.inv_bytes) > budget_)
            return rocblas_status_memory_error;
        r.A   = arena_.alloc(r.a_bytes);
        r.inv = arena_.alloc(r.inv_bytes);
        if(!r.A || !r.inv)
            return rocblas_status_memory_error;
        Lane& l = lanes_[0];
        cudaMemcpy2DAsync(r.A, m * es, A, (size_t)lda * es, m * es, m, cudaMemcpyDeviceToDevice, l.stream);
        build_inv(dtype, m, r.A, r.inv, l.stream);
        cudaStreamSynchronize(l.stream);
        residents_.push_back(r);
        *index = (int)residents_.size() - 1;
        return launch_status_now();
    }

    void set_budget(size_t b) { budget_ = std::min(b, arena_size_); }
    size_t used() const { return arena_.used(); }

    rocblas_status run(const ServerRequestC* reqs, int count, double* latency, ServerStatsC* stats)
    {
        using clock = std::chrono::steady_clock;
        if(count < 0)
            return rocblas_status_invalid_size;
        if(count && (!reqs || !latency))
            return rocblas_status_invalid_pointer;
        for(int i = 0; i < count; ++i)
        {
            const auto& q = reqs[i];
            if((q.dtype != kF32 && q.dtype != kF64) || q.m < 1 || q.n < 1 || !q.B_src
               || (q.resident >= 0 && (q.resident >= (int)residents_.size()
                                       || residents_[q.resident].dtype != q.dtype
                                       || residents_[q.resident].m != q.m))
               || (q.resident < 0 && (!q.A_src || q.lda_src < q.m)))
                return rocblas_status_invalid_value;
            if(i && q.arrival_s < reqs[i - 1].arrival_s)
                return rocblas_status_invalid_value; // requests must come in arrival order
            if(request_bytes(q) > budget_ - std::min(budget_, resident_bytes()))
                return rocblas_status_memory_error; // could never be admitted
        }
        arena_.reset_peak();
        const uint64_t launches0 = g_kernel_launches.load();
        std::vector<Held> held(count);
        std::deque<int>   pending, window[2];
        int64_t           collections = 0, largest = 0;
        int               next = 0, done = 0;
        const auto        t0 = clock::now();
        auto now_s = [&]() { return std::chrono::duration<double>(clock::now() - t0).count(); };

        while(done < count)
        {
            const double now = now_s();
            while(next < count && reqs[next].arrival_s <= now)
                pending.push_back(next++);
            // admission in arrival order under the budget
            while(!pending.empty())
            {
                const int i = pending.front();
                if(!admit(reqs[i], held[i]))
                    break;
                held[i].admitted = now;
                window[reqs[i].dtype == kF64 ? 1 : 0].push_back(i);
                pending.pop_front();
            }
            // collections: one per free lane, oldest window first
            for(;;)
            {
                int lane = -1;
                for(int j = 0; j < (int)lanes_.size(); ++j)
                    if(lanes_[j].inflight.empty())
                    {
                        lane = j;
                        break;
                    }
                if(lane < 0)
                    break;
                int pick = -1;
                for(int w = 0; w < 2; ++w)
                {
                    if(window[w].empty())
                        continue;
                    const int    oldest = window[w].front();
                    const bool   ready  = (int)window[w].size() >= max_batch_
                                     || now - held[oldest].admitted >= window_s_
                                     || (next >= count && pending.empty());
                    if(ready && (pick < 0 || held[oldest].admitted < held[window[pick].front()].admitted))
                        pick = w;
                }
                if(pick < 0)
                    break;
                std::vector<int> group;
                while(!window[pick].empty() && (int)group.size() < max_batch_)
                {
                    group.push_back(window[pick].front());
                    window[pick].pop_front();
                }
                rocblas_status st = launch(lanes_[lane], group, reqs, held);
                if(st != rocblas_status_success)
                    return st;
                ++collections;
                largest = std::max<int64_t>(largest, (int64_t)group.size());
            }
            // completions
            for(auto& l : lanes_)
            {
                if(l.inflight.empty())
                    continue;
                const cudaError_t e = cudaEventQuery(l.done);
                if(e == cudaErrorNotReady)
                    continue;
                if(e != cudaSuccess)
                    return rocblas_status_internal_error;
                const double t = now_s();
                for(int i : l.inflight)
                {
                    latency[i] = t - reqs[i].arrival_s;
                    release(held[i]);
                    ++done;
                }
                l.inflight.clear();
            }
        }
        for(auto& l : lanes_)
            cudaStreamSynchronize(l.stream);
        if(stats)
        {
            stats->wall_s             = now_s();
            stats->peak_bytes         = (int64_t)arena_.peak();
            stats->collections        = collections;
            stats->largest_collection = largest;
            stats->kernel_launches    = (int64_t)(g_kernel_launches.load() - launches0);
        }
        return launch_status_now();
    }

private:
    struct Resident
    {
        int    dtype, m;
        void*  A;
        void*  inv;
        size_t a_bytes, inv_bytes;
    };
    struct Held
    {
        void*  B = nullptr;
        void*  A = nullptr;
        void*  inv = nullptr;
        size_t b_bytes = 0, a_bytes = 0, inv_bytes = 0;
        double admitted = 0.0;
    };
    struct Lane
    {
        cudaStream_t     stream     = nullptr;
        _rocblas_handle* h          = nullptr;
        void*            host_stage = nullptr;
        void*            dev_stage  = nullptr;
        cudaEvent_t      done       = nullptr;
        std::vector<int> inflight;
    };

    static rocblas_status launch_status_now()
    {
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? rocblas_status_success : rocblas_status_internal_error;
    }

    size_t resident_bytes() const
    {
        size_t b = 0;
        for(const auto& r : residents_)
            b += DeviceArena::round(r.a_bytes) + DeviceArena::round(r.inv_bytes);
        return b;
    }

    static size_t request_bytes(const ServerRequestC& q)
    {
        const size_t es = q.dtype == kF64 ? 8 : 4;
        size_t       b  = DeviceArena::round((size_t)q.m * q.n * es);
        if(q.resident < 0)
        {
            b += DeviceArena::round((size_t)q.m * q.m * es);
            if(q.m > kChainVbMinK)
                b += DeviceArena::round((size_t)kInvNB * q.m * es);
        }
        return b;
    }

    bool admit(const ServerRequestC& q, Held& h)
    {
        if(arena_.used() + request_bytes(q) > budget_)
            return false;
        const size_t es = q.dtype == kF64 ? 8 : 4;
        h.b_bytes       = (size_t)q.m * q.n * es;
        h.B             = arena_.alloc(h.b_bytes);
        if(!h.B)
            return false;
        if(q.resident < 0)
        {
            h.a_bytes = (size_t)q.m * q.m * es;
            h.A       = arena_.alloc(h.a_bytes);
            if(q.m > kChainVbMinK)
            {
                h.inv_bytes = (size_t)kInvNB * q.m * es;
                h.inv       = arena_.alloc(h.inv_bytes);
            }
            if(!h.A || (q.m > kChainVbMinK && !h.inv))
            {
                release(h);
                return false;
            }
        }
        return true;
    }

    void release(Held& h)
    {
        arena_.free(h.B, h.b_bytes);
        arena_.free(h.A, h.a_bytes);
        arena_.free(h.inv, h.inv_bytes);
        h.B = h.A = h.inv = nullptr;
    }

    static void build_inv(int dtype, int m, void* A, void* inv, cudaStream_t s)
    {
        if(dtype == kF64)
            build_inv_t<double>(m, A, inv, s);
        else
            build_inv_t<float>(m, A, inv, s);
    }
    template <typename T>
    static void build_inv_t(int m, void* A, void* inv, cudaStream_t s)
    {
        TrtriParams<T> t{};
        t.k                = m;
        t.nb               = kInvNB;
        t.A.base           = reinterpret_cast<T*>(A);
        t.lda              = m;
        t.inv.base         = reinterpret_cast<T*>(inv);
        t.ldinv            = kInvNB;
        t.inv_block_stride = (int64_t)kInvNB * kInvNB;
        t.upper            = 0;
        t.unit             = 0;
        launch_trtri<T>(t, (int)ceil_div(m, kInvNB), 1, s);
    }

    rocblas_status launch(Lane& l, const std::vector<int>& group, const ServerRequestC* reqs,
                          std::vector<Held>& held)
    {
        const int    cnt = (int)group.size();
        const int    dt  = reqs[group[0]].dtype;
        // host staging: [descriptors][invA pointers][fresh A ptrs][fresh inv ptrs][lda][k]
        char*  hs     = reinterpret_cast<char*>(l.host_stage);
        auto*  probs  = reinterpret_cast<VbProblem*>(hs);
        auto*  invs   = reinterpret_cast<const void**>(hs + (size_t)cnt * sizeof(VbProblem));
        auto*  fA     = invs + cnt;
        auto*  fInv   = reinterpret_cast<void**>(hs + (size_t)cnt * (sizeof(VbProblem) + 2 * sizeof(void*)));
        auto*  fLda   = reinterpret_cast<int64_t*>(fInv + cnt);
        auto*  fK     = reinterpret_cast<int*>(fLda + cnt);
        const size_t o_g    = gather_offset(cnt);
        auto*        gat    = reinterpret_cast<GatherReq*>(hs + o_g);
        auto*        prefix = reinterpret_cast<int*>(gat + cnt);
        int    nfresh = 0, fresh_nb = 0, items = 0;
        int    max_k = 1, max_n = 1;
        for(int j = 0; j < cnt; ++j)
        {
            const ServerRequestC& q = reqs[group[j]];
            Held&                 h = held[group[j]];
            // the request's data arrives: B, and its own A (copied by the gather launch)
            GatherReq& g = gat[j];
            g.srcB    = q.B_src;
            g.dstB    = h.B;
            g.srcA    = nullptr;
            g.dstA    = nullptr;
            g.lda_src = q.lda_src;
            g.m       = q.m;
            g.n       = q.n;
            g.itemsB  = (int)ceil_div(q.n, kGatherCols);
            g.pad     = 0;
            prefix[j] = items;
            items += g.itemsB;
            const void* A;
            const void* inv = nullptr;
            if(q.resident >= 0)
            {
                A   = residents_[q.resident].A;
                inv = residents_[q.resident].inv;
            }
            else
            {
                g.srcA = q.A_src;
                g.dstA = h.A;
                items += (int)ceil_div(q.m, kGatherCols);
                A = h.A;
                if(h.inv)
                {
                    inv          = h.inv;
                    fA[nfresh]   = h.A;
                    fInv[nfresh] = h.inv;
                    fLda[nfresh] = q.m;
                    fK[nfresh]   = q.m;
                    fresh_nb     = std::max(fresh_nb, (int)ceil_div(q.m, kInvNB));
                    ++nfresh;
                }
            }
            VbProblem p;
            p.A     = A;
            p.B     = h.B;
            p.m     = q.m;
            p.n     = q.n;
            p.lda   = q.m;
            p.ldb   = q.m;
            p.side  = kLeft;
            p.uplo  = kLower;
            p.trans = kOpN;
            p.diag  = kNonUnit;
            probs[j] = p;
            invs[j]  = inv;
            max_k    = std::max(max_k, q.m);
            max_n    = std::max(max_n, q.n);
        }
        prefix[cnt] = items;
        const size_t bytes = o_g + (size_t)cnt * sizeof(GatherReq) + ((size_t)cnt + 1) * sizeof(int);
        cudaMemcpyAsync(l.dev_stage, l.host_stage, bytes, cudaMemcpyHostToDevice, l.stream);
        const char* ds = reinterpret_cast<const char*>(l.dev_stage);
        if(items)
        {
            auto* dg = reinterpret_cast<const GatherReq*>(ds + o_g);
            auto* dp = reinterpret_cast<const int*>(dg + cnt);
            if(dt == kF64)
                server_gather_kernel<double><<<items, 256, 0, l.stream>>>(dg, dp, cnt);
            else
                server_gather_kernel<float><<<items, 256, 0, l.stream>>>(dg, dp, cnt);
            count_launch();
        }
        // the fresh A's diagonal blocks, all of them in one variable-size trtri launch
        if(nfresh)
        {
            const size_t o_fA = (size_t)cnt * (sizeof(VbProblem) + sizeof(void*));
            if(dt == kF64)
                build_inv_batch<double>(ds, o_fA, cnt, nfresh, fresh_nb, l.stream);
            else
                build_inv_batch<float>(ds, o_fA, cnt, nfresh, fresh_nb, l.stream);
        }
        auto* dprobs = reinterpret_cast<const rocblas_b200_trsm_problem*>(ds);
        auto* dinvs  = ds + (size_t)cnt * sizeof(VbProblem);
        const rocblas_status st = solve_(l.h, dt, dprobs, dinvs, cnt, max_k, max_n);
        if(st != rocblas_status_success)
            return st;
        for(int j = 0; j < cnt; ++j)
        {
            const ServerRequestC& q = reqs[group[j]];
            if(q.X_dst)
                cudaMemcpyAsync(q.X_dst, held[group[j]].B, held[group[j]].b_bytes,
                                cudaMemcpyDeviceToDevice, l.stream);
        }
        cudaEventRecord(l.done, l.stream);
        l.inflight = group;
        return rocblas_status_success;
    }

    // trtri of `nfresh` fresh A's whose pointer / order arrays start at device offset o_fA of
    // the staging buffer (layout of launch()): grid (largest block count, nfresh)
    template <typename T>
    static void build_inv_batch(const char* ds, size_t o_fA, int cnt, int nfresh, int max_nb,
                                cudaStream_t s)
    {
        TrtriParams<T> t{};
        t.nb               = kInvNB;
        t.k                = max_nb * kInvNB;
        t.A.arr            = ds + o_fA;
        t.inv.arr          = ds + o_fA + (size_t)cnt * sizeof(void*);
        t.vlda             = reinterpret_cast<const int64_t*>(ds + o_fA + 2 * (size_t)cnt * sizeof(void*));
        t.vk               = reinterpret_cast<const int*>(ds + o_fA + 2 * (size_t)cnt * sizeof(void*)
                                                          + (size_t)cnt * sizeof(int64_t));
        t.ldinv            = kInvNB;
        t.inv_block_stride = (int64_t)kInvNB * kInvNB;
        t.upper            = 0;
        t.unit             = 0;
        launch_trtri<T>(t, max_nb, nfresh, s);
    }

    ServerSolveFn         solve_;
    DeviceArena           arena_;
    size_t                budget_ = 0, arena_size_ = 0;
    double                window_s_ = 0.0;
    int                   max_batch_ = 1;
    std::vector<Lane>     lanes_;
    std::vector<Resident> residents_;
};

} // namespace rb200
