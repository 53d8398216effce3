// Process-wide launch counter and optional CUDA-event timing of the FP64
// tensor-core GEMM launches (C ABI: gprat_cu_stats_*).
#include "common.cuh"
#include "gprat_cu.h"

#include <atomic>
#include <vector>

namespace gprat_cu
{
namespace
{

std::atomic<int64_t> g_launches{ 0 };
std::atomic<bool> g_timing{ false };

struct Pending
{
    cudaEvent_t start, stop;
    double flops;
};

std::mutex g_mtx;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_free_events;
int64_t g_gemm_launches = 0;
double g_gemm_ms = 0.0;
double g_gemm_flops = 0.0;
thread_local cudaEvent_t t_open = nullptr;

cudaEvent_t take_event()
{
    std::lock_guard<std::mutex> lk(g_mtx);
    if (!g_free_events.empty())
    {
        cudaEvent_t e = g_free_events.back();
        g_free_events.pop_back();
        return e;
    }
    cudaEvent_t e;
    GPRAT_CUDA_CHECK(cudaEventCreate(&e));
    return e;
}

void drain()
{
    std::lock_guard<std::mutex> lk(g_mtx);
    for (auto &p : g_pending)
    {
        GPRAT_CUDA_CHECK(cudaEventSynchronize(p.stop));
        float ms = 0.f;
        GPRAT_CUDA_CHECK(cudaEventElapsedTime(&ms, p.start, p.stop));
        g_gemm_ms += ms;
        g_gemm_flops += p.flops;
        g_gemm_launches += 1;
        g_free_events.push_back(p.start);
        g_free_events.push_back(p.stop);
    }
    g_pending.clear();
}

}  // namespace

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

bool gemm_timing_enabled() { return g_timing.load(std::memory_order_relaxed); }

void gemm_timing_begin(cudaStream_t s)
{
    t_open = take_event();
    GPRAT_CUDA_CHECK(cudaEventRecord(t_open, s));
}

void gemm_timing_end(cudaStream_t s, double flops)
{
    cudaEvent_t stop = take_event();
    GPRAT_CUDA_CHECK(cudaEventRecord(stop, s));
    std::lock_guard<std::mutex> lk(g_mtx);
    g_pending.push_back({ t_open, stop, flops });
    t_open = nullptr;
}

}  // namespace gprat_cu

extern "C" {

int gprat_cu_stats_reset(void)
{
    try
    {
        gprat_cu::drain();
        std::lock_guard<std::mutex> lk(gprat_cu::g_mtx);
        gprat_cu::g_launches = 0;
        gprat_cu::g_gemm_launches = 0;
        gprat_cu::g_gemm_ms = 0.0;
        gprat_cu::g_gemm_flops = 0.0;
        return GPRAT_CU_OK;
    }
    catch (const gprat_cu::Error &e)
    {
        return e.code;
    }
}

int gprat_cu_stats_enable_timing(int enable)
{
    gprat_cu::g_timing = enable != 0;
    return GPRAT_CU_OK;
}

int gprat_cu_stats_read(int64_t *launches, int64_t *gemm_launches, double *gemm_ms, double *gemm_flops)
{
    try
    {
        gprat_cu::drain();
        std::lock_guard<std::mutex> lk(gprat_cu::g_mtx);
        if (launches != nullptr)
        {
            *launches = gprat_cu::g_launches.load();
        }
        if (gemm_launches != nullptr)
        {
            *gemm_launches = gprat_cu::g_gemm_launches;
        }
        if (gemm_ms != nullptr)
        {
            *gemm_ms = gprat_cu::g_gemm_ms;
        }
        if (gemm_flops != nullptr)
        {
            *gemm_flops = gprat_cu::g_gemm_flops;
        }
        return GPRAT_CU_OK;
    }
    catch (const gprat_cu::Error &e)
    {
        return e.code;
    }
}

}  // extern "C"
