// Shared device helpers for the registration kernels.
//
// Arithmetic rule: every kernel file is compiled with -fmad=false and the float
// expressions below are written in the reference's evaluation order, so products
// and sums round exactly as the reference's CPU build (-ffp-contract=off) does.
// That is what makes uint8 outputs and histogram counts bit-identical.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "kernels.h"

namespace regb {

// p' = sr * p + shift with the reference's left-to-right sums
// (numerical/transformation.hpp:58-73): ((x*r0 + y*r1) + z*r2) + s0.
struct Xform {
    float m[12];  // sr[9] row-major, shift[3]
};

__device__ __forceinline__ void apply_xform(const float* __restrict__ T, float x, float y, float z, float& ox,
                                            float& oy, float& oz)
{
    ox = x * T[0] + y * T[1] + z * T[2] + T[9];
    oy = x * T[3] + y * T[4] + z * T[5] + T[10];
    oz = x * T[6] + y * T[7] + z * T[8] + T[11];
}

// Cell test of interpolator::linear<3>::get_location
// (numerical/interpolation.hpp:337-350): reject negative coordinates and any
// cell whose +1 neighbour leaves the volume.  For x >= 0, trunc(x)+1 >= w is the
// same as x >= w-1, and w-1 is exact in float for every accepted extent.
struct Cell {
    int base;      // flat index of the (ix, iy, iz) corner
    float r[8];    // weights in the reference's order
};

__device__ __forceinline__ bool trilinear_cell(const Dim3& D, float x, float y, float z, Cell& c)
{
    if (x < 0.0f || y < 0.0f || z < 0.0f)
        return false;
    if (!(x < (float)(D.w - 1)) || !(y < (float)(D.h - 1)) || !(z < (float)(D.d - 1)))
        return false;
    int ix = (int)x, iy = (int)y, iz = (int)z;
    float p0 = x - (float)ix, p1 = y - (float)iy, p2 = z - (float)iz;
    float n0 = 1.0f - p0, n1 = 1.0f - p1, n2 = 1.0f - p2;
    float n0n1 = n0 * n1, p0n1 = p0 * n1, n0p1 = n0 * p1, p0p1 = p0 * p1;
    c.r[0] = n0n1 * n2;
    c.r[1] = p0n1 * n2;
    c.r[2] = n0p1 * n2;
    c.r[3] = p0p1 * n2;
    c.r[4] = n0n1 * p2;
    c.r[5] = p0n1 * p2;
    c.r[6] = n0p1 * p2;
    c.r[7] = p0p1 * p2;
    c.base = (iz * D.h + iy) * D.w + ix;
    return true;
}

template <typename T>
__device__ __forceinline__ float ld_pix(const T* __restrict__ p, int i)
{
    return (float)__ldg(p + i);
}

// weighted_sum (numerical/interpolation.hpp:61-73): r = I0*w0; r += I1*w1; ...
template <typename T>
__device__ __forceinline__ float cell_sum(const T* __restrict__ I, const Dim3& D, const Cell& c)
{
    const int w = D.w, wh = D.wh(), b = c.base;
    float acc = ld_pix(I, b) * c.r[0];
    acc += ld_pix(I, b + 1) * c.r[1];
    acc += ld_pix(I, b + w) * c.r[2];
    acc += ld_pix(I, b + w + 1) * c.r[3];
    acc += ld_pix(I, b + wh) * c.r[4];
    acc += ld_pix(I, b + wh + 1) * c.r[5];
    acc += ld_pix(I, b + wh + w) * c.r[6];
    acc += ld_pix(I, b + wh + w + 1) * c.r[7];
    return acc;
}

// interp_type<T>::assign (numerical/interpolation.hpp:28-34).
template <typename T>
__device__ __forceinline__ T assign_pix(float v);
template <>
__device__ __forceinline__ uint8_t assign_pix<uint8_t>(float v)
{
    return v <= 0.0f ? (uint8_t)0 : (uint8_t)v;
}
template <>
__device__ __forceinline__ float assign_pix<float>(float v)
{
    return v;
}

// Vector-field cell sum: each component accumulated as the scalar case.
__device__ __forceinline__ float3 cell_sum_vec(const float* __restrict__ F, const Dim3& D, const Cell& c)
{
    const int w = D.w, wh = D.wh(), b = c.base;
    const int off[8] = {0, 1, w, w + 1, wh, wh + 1, wh + w, wh + w + 1};
    const float* p = F + 3LL * b;
    float3 acc;
    acc.x = __ldg(p) * c.r[0];
    acc.y = __ldg(p + 1) * c.r[0];
    acc.z = __ldg(p + 2) * c.r[0];
#pragma unroll
    for (int k = 1; k < 8; ++k) {
        const float* q = F + 3LL * (b + off[k]);
        acc.x += __ldg(q) * c.r[k];
        acc.y += __ldg(q + 1) * c.r[k];
        acc.z += __ldg(q + 2) * c.r[k];
    }
    return acc;
}

__device__ __forceinline__ void unflat(int i, const Dim3& D, int& x, int& y, int& z)
{
    x = i % D.w;
    int t = i / D.w;
    y = t % D.h;
    z = t / D.h;
}

// Block-wide reductions over a power-of-two block (<= 1024 threads).
template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ T block_sum(T v, T* scratch /* >= 32 */)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0)
        scratch[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? scratch[threadIdx.x] : T(0);
    if (wid == 0)
        v = warp_sum(v);
    return v;  // valid in thread 0
}

}  // namespace regb
