#include "stats.h"
#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>
#include "../../include/regb200.h"

namespace regb {

std::atomic<long long> g_launches{0};

namespace {
struct Pending {
    cudaEvent_t a, b;
    int kind;
    long long tasks;
    double voxels, bytes;
};
std::mutex g_m;
std::atomic<int> g_timing{0};
std::vector<Pending> g_pending;
regb_stats g_acc{};
cudaEvent_t g_origin = nullptr;                     // recorded when timing starts
std::vector<std::pair<float, float>> g_mi_spans;  // MI launches: [start, end] ms after it

// Length of the union of the spans (launches on two streams may overlap).
double union_ms(std::vector<std::pair<float, float>> v)
{
    std::sort(v.begin(), v.end());
    double total = 0.0, lo = 0.0, hi = -1.0;
    bool open = false;
    for (const auto& s : v) {
        if (!open || s.first > hi) {
            if (open)
                total += hi - lo;
            lo = s.first;
            hi = s.second;
            open = true;
        } else if (s.second > hi)
            hi = s.second;
    }
    if (open)
        total += hi - lo;
    return total;
}

void drain_locked()
{
    for (auto& p : g_pending) {
        float ms = 0.0f;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            float t0 = 0.0f, t1 = 0.0f;
            if (p.kind == 0 && g_origin && cudaEventElapsedTime(&t0, g_origin, p.a) == cudaSuccess &&
                cudaEventElapsedTime(&t1, g_origin, p.b) == cudaSuccess)
                g_mi_spans.push_back({t0, t1});
            if (p.kind == 0) {
                g_acc.mi_launches += 1;
                g_acc.mi_tasks += p.tasks;
                g_acc.mi_voxels += p.voxels;
                g_acc.mi_bytes += p.bytes;
                g_acc.mi_ms += ms;
            } else {
                g_acc.corr_launches += 1;
                g_acc.corr_tasks += p.tasks;
                g_acc.corr_voxels += p.voxels;
                g_acc.corr_bytes += p.bytes;
                g_acc.corr_ms += ms;
            }
        }
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    g_pending.clear();
    (void)cudaGetLastError();
}
}  // namespace

void KernelTimer::begin(cudaStream_t st, int k)
{
    on = g_timing.load() != 0;
    kind = k;
    if (!on)
        return;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
        on = false;
        (void)cudaGetLastError();
        return;
    }
    cudaEventRecord(a, st);
}

void count_cdm_level(long long iterations, long long voxels, int pixel_bytes)
{
    std::lock_guard<std::mutex> g(g_m);
    g_acc.cdm_iterations += iterations;
    g_acc.cdm_voxel_iterations += (double)iterations * (double)voxels;
    g_acc.cdm_model_bytes += (double)iterations * (double)voxels * (596.0 + 4.0 * pixel_bytes);
}

void KernelTimer::end(cudaStream_t st, long long tasks, double voxels, double bytes)
{
    if (!on)
        return;
    cudaEventRecord(b, st);
    std::lock_guard<std::mutex> g(g_m);
    g_pending.push_back({a, b, kind, tasks, voxels, bytes});
}

}  // namespace regb

using namespace regb;

extern "C" {

regb_status regb_stats_reset(int timing)
{
    std::lock_guard<std::mutex> g(g_m);
    drain_locked();
    g_acc = regb_stats{};
    g_mi_spans.clear();
    g_launches.store(0);
    if (g_origin) {
        cudaEventDestroy(g_origin);
        g_origin = nullptr;
    }
    if (timing && cudaEventCreate(&g_origin) == cudaSuccess) {
        // the device timestamp all MI launch spans are measured from
        if (cudaEventRecord(g_origin, 0) != cudaSuccess) {
            cudaEventDestroy(g_origin);
            g_origin = nullptr;
        }
    }
    (void)cudaGetLastError();
    g_timing.store(timing ? 1 : 0);
    return REGB_OK;
}

regb_status regb_stats_get(regb_stats* out)
{
    if (!out)
        return REGB_ERR_ARG;
    std::lock_guard<std::mutex> g(g_m);
    drain_locked();
    *out = g_acc;
    out->launches = g_launches.load();
    out->mi_busy_ms = union_ms(g_mi_spans);
    return REGB_OK;
}

}  // extern "C"
