// Kernel launch counting and optional CUDA-event timing per kernel kind.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "rg_internal.cuh"

namespace rg {

namespace {

struct Pending {
    int kind;
    cudaEvent_t a, b;
};

std::mutex g_mu;
bool g_on = false;
long long g_launches[T_COUNT] = {};
double g_ms[T_COUNT] = {};
long long g_timed[T_COUNT] = {};
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;
cudaEvent_t g_open[T_COUNT] = {};

const char* kNames[T_COUNT] = {"pattern", "assemble", "assemble_boundary", "insert_constraint",
                               "spmv", "balance", "norms", "residual", "paso_spmv",
                               "paso_update1", "paso_update2", "std_spmv", "std_update",
                               "f32_spmv", "f32_update", "vector", "batch_spmv", "batch_update",
                               "batch_outer", "ws_conv", "ws_wgrad", "ws_ops"};

cudaEvent_t get_event()
{
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

}  // namespace

void timer_begin(int kind)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_launches[kind]++;
    if (!g_on) return;
    cudaEvent_t e = get_event();
    cudaEventRecord(e, stream());
    g_open[kind] = e;
}

void timer_end(int kind)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_on || !g_open[kind]) return;
    cudaEvent_t e = get_event();
    cudaEventRecord(e, stream());
    g_pending.push_back({kind, g_open[kind], e});
    g_open[kind] = nullptr;
    if (g_pending.size() > 8192) {
        // keep the pool bounded during long solves
        for (Pending& p : g_pending) {
            float ms = 0.f;
            cudaEventSynchronize(p.b);
            cudaEventElapsedTime(&ms, p.a, p.b);
            g_ms[p.kind] += ms;
            g_timed[p.kind]++;
            g_pool.push_back(p.a);
            g_pool.push_back(p.b);
        }
        g_pending.clear();
    }
}

void timers_collect()
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (Pending& p : g_pending) {
        float ms = 0.f;
        cudaEventSynchronize(p.b);
        cudaEventElapsedTime(&ms, p.a, p.b);
        g_ms[p.kind] += ms;
        g_timed[p.kind]++;
        g_pool.push_back(p.a);
        g_pool.push_back(p.b);
    }
    g_pending.clear();
}

bool timers_on()
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_on;
}

void timers_snapshot(long long out[T_COUNT])
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (int k = 0; k < T_COUNT; ++k) out[k] = g_launches[k];
}

void timers_add(const long long delta[T_COUNT], long long times)
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (int k = 0; k < T_COUNT; ++k) g_launches[k] += delta[k] * times;
}

}  // namespace rg

extern "C" {

int rg_timers_enable(int on)
{
    rg::timers_collect();
    std::lock_guard<std::mutex> lk(rg::g_mu);
    rg::g_on = on != 0;
    return RG_OK;
}

int rg_timers_reset(void)
{
    rg::timers_collect();
    std::lock_guard<std::mutex> lk(rg::g_mu);
    for (int k = 0; k < rg::T_COUNT; ++k) {
        rg::g_launches[k] = 0;
        rg::g_ms[k] = 0.0;
        rg::g_timed[k] = 0;
    }
    return RG_OK;
}

int rg_timers_count(void) { return rg::T_COUNT; }

const char* rg_timer_name(int kind) { return (kind >= 0 && kind < rg::T_COUNT) ? rg::kNames[kind] : ""; }

int rg_timers_read(int kind, int64_t* launches, int64_t* timed, double* total_ms)
{
    if (kind < 0 || kind >= rg::T_COUNT) return RG_INVALID_ARG;
    rg::timers_collect();
    std::lock_guard<std::mutex> lk(rg::g_mu);
    if (launches) *launches = rg::g_launches[kind];
    if (timed) *timed = rg::g_timed[kind];
    if (total_ms) *total_ms = rg::g_ms[kind];
    return RG_OK;
}

}  // extern "C"
