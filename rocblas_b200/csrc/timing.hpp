// Optional per-launch timing of the library's main kernels with CUDA events on the launching
// stream (rocblas_b200_kernel_timing_* in rocblas_b200_ext.h).  Off by default; when on, every
// launch of a timed kernel class is bracketed by two events from a pool and its algorithmic
// work is recorded, so a caller can compute achieved rates of one kernel inside a larger call.
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <vector>

namespace rb200
{

enum class KernelClass : int
{
    sliced = 0, // ozaki_gemm_kernel (work: int8 tensor operations)
    dmma   = 1, // gemm_dmma_kernel (work: FP64 flops)
    chain  = 2, // trsm_chain_kernel (work: FP64 flops of the solve)
    trtri  = 3, // trtri_block_kernel (work: nb^3 / 3 flops per 128-block)
    strip  = 4, // the variable-size batch's strip-solver queues (work: 0)
    count  = 5
};

struct KernelTiming
{
    struct Rec
    {
        int         cls;
        cudaEvent_t e0, e1;
        double      work;
    };
    std::mutex               mu;
    bool                     on = false;
    std::vector<Rec>         recs;
    std::vector<cudaEvent_t> pool;

    cudaEvent_t take()
    {
        if(!pool.empty())
        {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void recycle()
    {
        for(auto& r : recs)
        {
            pool.push_back(r.e0);
            pool.push_back(r.e1);
        }
        recs.clear();
    }
};

inline KernelTiming& kernel_timing()
{
    static KernelTiming t;
    return t;
}

// Brackets one launch: construct before the launch, destroy after it.
class TimedLaunch
{
public:
    TimedLaunch(KernelClass c, cudaStream_t s, double work) : s_(s)
    {
        KernelTiming& t = kernel_timing();
        std::lock_guard<std::mutex> lock(t.mu);
        if(!t.on)
            return;
        rec_.cls  = (int)c;
        rec_.work = work;
        rec_.e0   = t.take();
        rec_.e1   = t.take();
        cudaEventRecord(rec_.e0, s_);
        active_ = true;
    }
    ~TimedLaunch()
    {
        if(!active_)
            return;
        KernelTiming& t = kernel_timing();
        std::lock_guard<std::mutex> lock(t.mu);
        cudaEventRecord(rec_.e1, s_);
        t.recs.push_back(rec_);
    }
    TimedLaunch(const TimedLaunch&) = delete;
    TimedLaunch& operator=(const TimedLaunch&) = delete;

private:
    cudaStream_t     s_;
    KernelTiming::Rec rec_{};
    bool             active_ = false;
};

inline int kernel_class_of(const char* name)
{
    if(!name)
        return -1;
    if(!std::strcmp(name, "sliced"))
        return (int)KernelClass::sliced;
    if(!std::strcmp(name, "dmma"))
        return (int)KernelClass::dmma;
    if(!std::strcmp(name, "chain"))
        return (int)KernelClass::chain;
    if(!std::strcmp(name, "trtri"))
        return (int)KernelClass::trtri;
    if(!std::strcmp(name, "strip"))
        return (int)KernelClass::strip;
    return -1;
}

} // namespace rb200
