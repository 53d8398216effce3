// Process-wide launch counter, optional CUDA-event timing of the tensor-core
// GEMM launches (C ABI: gprat_cu_stats_*), and per-phase step timers with the
// reference's APEX step labels (C ABI: gprat_cu_steps_*).
#include "common.cuh"
#include "gprat_cu.h"

#include <atomic>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
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

// ---------------------------------------------------------------------------
// Step timers: the reference samples APEX timers around the phases of each
// pipeline ("predict_step cholesky", ... core/src/cpu/gp_functions.cpp:29-678,
// core/include/apex_utils.hpp:19-54).  Here each phase is bracketed by CUDA
// events on the stream that runs it; reading synchronises them.
namespace
{
struct StepPending
{
    std::string label;
    cudaEvent_t start, stop;
};
std::atomic<bool> g_steps{ false };
std::vector<StepPending> g_step_open;  // index = slot
std::vector<int> g_step_done;          // slots whose stop was recorded
int g_step_running = 0;                 // slots opened and not yet closed
std::map<std::string, std::pair<int64_t, double>> g_step_totals;
thread_local std::string t_step_prefix;

void drain_steps()
{
    std::lock_guard<std::mutex> lk(g_mtx);
    for (int slot : g_step_done)
    {
        StepPending &p = g_step_open[slot];
        float ms = 0.f;
        if (cudaEventSynchronize(p.stop) == cudaSuccess && cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess)
        {
            auto &t = g_step_totals[p.label];
            t.first += 1;
            t.second += ms;
        }
        cudaGetLastError();
        g_free_events.push_back(p.start);
        g_free_events.push_back(p.stop);
        p.label.clear();
    }
    g_step_done.clear();
    if (g_step_running == 0)
    {
        g_step_open.clear();
    }
}
}  // namespace

bool steps_enabled() { return g_steps.load(std::memory_order_relaxed); }

StepPrefix::StepPrefix(const char *prefix) : saved(t_step_prefix) { t_step_prefix = prefix; }
StepPrefix::~StepPrefix() { t_step_prefix = saved; }

StepScope::StepScope(const char *phase, cudaStream_t s) : slot(-1), stream(s)
{
    if (!steps_enabled())
    {
        return;
    }
    cudaEvent_t a = take_event(), b = take_event();
    if (cudaEventRecord(a, s) != cudaSuccess)
    {
        return;
    }
    std::lock_guard<std::mutex> lk(g_mtx);
    std::string label = t_step_prefix.empty() ? std::string(phase) : t_step_prefix + " " + phase;
    g_step_open.push_back({ std::move(label), a, b });
    slot = static_cast<int>(g_step_open.size()) - 1;
    ++g_step_running;
}

StepScope::~StepScope()
{
    if (slot < 0)
    {
        return;
    }
    std::lock_guard<std::mutex> lk(g_mtx);
    --g_step_running;
    if (cudaEventRecord(g_step_open[slot].stop, stream) == cudaSuccess)
    {
        g_step_done.push_back(slot);
    }
    cudaGetLastError();
}

}  // namespace gprat_cu

extern "C" {

int gprat_cu_steps_enable(int enable)
{
    gprat_cu::g_steps = enable != 0;
    return GPRAT_CU_OK;
}

int gprat_cu_steps_reset(void)
{
    try
    {
        gprat_cu::drain_steps();
        std::lock_guard<std::mutex> lk(gprat_cu::g_mtx);
        gprat_cu::g_step_totals.clear();
        return GPRAT_CU_OK;
    }
    catch (const gprat_cu::Error &e)
    {
        return e.code;
    }
}

int gprat_cu_steps_csv(char *buf, int64_t cap, int64_t *needed)
{
    try
    {
        gprat_cu::drain_steps();
        std::ostringstream os;
        os << "label,calls,total_ms,mean_ms\n";
        {
            std::lock_guard<std::mutex> lk(gprat_cu::g_mtx);
            for (const auto &kv : gprat_cu::g_step_totals)
            {
                os << kv.first << "," << kv.second.first << "," << kv.second.second << ","
                   << kv.second.second / static_cast<double>(kv.second.first) << "\n";
            }
        }
        const std::string text = os.str();
        if (needed != nullptr)
        {
            *needed = static_cast<int64_t>(text.size()) + 1;
        }
        if (buf != nullptr && cap > 0)
        {
            const size_t n = std::min<size_t>(text.size(), static_cast<size_t>(cap - 1));
            std::memcpy(buf, text.data(), n);
            buf[n] = '\0';
        }
        return GPRAT_CU_OK;
    }
    catch (const gprat_cu::Error &e)
    {
        return e.code;
    }
}

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
