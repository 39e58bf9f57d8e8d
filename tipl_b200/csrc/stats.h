// Launch accounting and optional CUDA-event timing of the affine cost kernels.
#pragma once
#include <atomic>
#include <cuda_runtime.h>

namespace regb {

extern std::atomic<long long> g_launches;  // kernels launched by this library
inline void count_launch(long long k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// Adds one finished CDM level to the statistics: its iterations, voxels and the pass
// model's bytes (596 + 4 x bytes per pixel per voxel and iteration).
void count_cdm_level(long long iterations, long long voxels, int pixel_bytes);

// Records an event pair around one affine cost launch when timing is on.
struct KernelTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    bool on = false;
    int kind = 0;  // 0 MI, 1 correlation
    void begin(cudaStream_t st, int k);
    void end(cudaStream_t st, long long tasks, double voxels, double bytes);
};

}  // namespace regb
