// Storage conversions at the boundary: uint16 / BF16 / float volumes to the uint8 the
// affine search takes (normalize_upper_lower2, numerical/numerical.hpp:909-927), and
// uint16 / BF16 to float for the FP32 nonlinear path (exact widening).
//
// BF16 voxels are the upper 16 bits of an IEEE float, so widening is a shift; uint16
// values are exact in float.  The quantisation is the reference's float arithmetic
// ((v - min) * (upper / (max - min)), truncated), with min/max found exactly.
#include <algorithm>
#include "kernels.h"

namespace regb {

namespace {

constexpr int kThreads = 256;

template <int DT>
__device__ __forceinline__ float load_as_float(const void* p, long long i);
template <>
__device__ __forceinline__ float load_as_float<0>(const void* p, long long i)
{
    return (float)((const uint8_t*)p)[i];
}
template <>
__device__ __forceinline__ float load_as_float<1>(const void* p, long long i)
{
    return ((const float*)p)[i];
}
template <>
__device__ __forceinline__ float load_as_float<2>(const void* p, long long i)
{
    return (float)((const uint16_t*)p)[i];
}
template <>
__device__ __forceinline__ float load_as_float<3>(const void* p, long long i)
{
    return __uint_as_float((unsigned)((const uint16_t*)p)[i] << 16);
}

// Order-preserving integer key of a float (for atomicMin/atomicMax).
__device__ __forceinline__ unsigned key_of(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// mm[0] = min key, mm[1] = max key; mm must hold {0xffffffff, 0} on entry.
template <int DT>
__global__ void __launch_bounds__(kThreads) minmax_kernel(const void* __restrict__ v, long long n,
                                                           unsigned* __restrict__ mm)
{
    unsigned lo = 0xffffffffu, hi = 0u;
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads) {
        const unsigned k = key_of(load_as_float<DT>(v, i));
        lo = min(lo, k);
        hi = max(hi, k);
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    __shared__ unsigned slo[kThreads / 32], shi[kThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        slo[threadIdx.x >> 5] = lo;
        shi[threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kThreads / 32; ++k) {
            lo = min(lo, slo[k]);
            hi = max(hi, shi[k]);
        }
        atomicMin(&mm[0], lo);
        atomicMax(&mm[1], hi);
    }
}

__device__ __forceinline__ float float_of(unsigned k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// out[i] = uint8((v[i] - min) * (upper / (max - min))); leaves out untouched when max == min.
template <int DT>
__global__ void __launch_bounds__(kThreads) normalize_kernel(const void* __restrict__ v, long long n,
                                                              const unsigned* __restrict__ mm, float upper,
                                                              uint8_t* __restrict__ out)
{
    const float mn = float_of(mm[0]), mx = float_of(mm[1]);
    const float range = __fsub_rn(mx, mn);
    if (range == 0.0f)
        return;
    const float scale = __fdiv_rn(upper, range);
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads)
        out[i] = (uint8_t)(unsigned)__fmul_rn(__fsub_rn(load_as_float<DT>(v, i), mn), scale);
}

template <int DT>
__global__ void __launch_bounds__(kThreads) widen_kernel(const void* __restrict__ v, long long n,
                                                          float* __restrict__ out)
{
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads)
        out[i] = load_as_float<DT>(v, i);
}

int grid_for(long long n)
{
    long long b = (n + kThreads - 1) / kThreads;
    return (int)std::min<long long>(std::max<long long>(b, 1), 148LL * 16);
}

}  // namespace

cudaError_t launch_normalize_to_u8(const void* in, int dtype, long long n, float upper, uint8_t* out, unsigned* mm,
                                   cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(mm, 0xff, sizeof(unsigned), st);  // min key
    if (e == cudaSuccess)
        e = cudaMemsetAsync(mm + 1, 0, sizeof(unsigned), st);         // max key
    if (e != cudaSuccess)
        return e;
    const int g = grid_for(n), gm = std::min(g, 148 * 4);
    switch (dtype) {
    case 0: minmax_kernel<0><<<gm, kThreads, 0, st>>>(in, n, mm); normalize_kernel<0><<<g, kThreads, 0, st>>>(in, n, mm, upper, out); break;
    case 1: minmax_kernel<1><<<gm, kThreads, 0, st>>>(in, n, mm); normalize_kernel<1><<<g, kThreads, 0, st>>>(in, n, mm, upper, out); break;
    case 2: minmax_kernel<2><<<gm, kThreads, 0, st>>>(in, n, mm); normalize_kernel<2><<<g, kThreads, 0, st>>>(in, n, mm, upper, out); break;
    case 3: minmax_kernel<3><<<gm, kThreads, 0, st>>>(in, n, mm); normalize_kernel<3><<<g, kThreads, 0, st>>>(in, n, mm, upper, out); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_minmax(const void* in, int dtype, long long n, unsigned* mm, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(mm, 0xff, sizeof(unsigned), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(mm + 1, 0, sizeof(unsigned), st);
    if (e != cudaSuccess)
        return e;
    const int g = std::min(grid_for(n), 148 * 4);  // one atomic pair per block
    switch (dtype) {
    case 0: minmax_kernel<0><<<g, kThreads, 0, st>>>(in, n, mm); break;
    case 1: minmax_kernel<1><<<g, kThreads, 0, st>>>(in, n, mm); break;
    case 2: minmax_kernel<2><<<g, kThreads, 0, st>>>(in, n, mm); break;
    case 3: minmax_kernel<3><<<g, kThreads, 0, st>>>(in, n, mm); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_widen_to_f32(const void* in, int dtype, long long n, float* out, cudaStream_t st)
{
    const int g = grid_for(n);
    switch (dtype) {
    case 0: widen_kernel<0><<<g, kThreads, 0, st>>>(in, n, out); break;
    case 1: widen_kernel<1><<<g, kThreads, 0, st>>>(in, n, out); break;
    case 2: widen_kernel<2><<<g, kThreads, 0, st>>>(in, n, out); break;
    case 3: widen_kernel<3><<<g, kThreads, 0, st>>>(in, n, out); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace regb
