// Mapping steps of the mm_reg pipeline on the device (reg/mm_reg.hpp:271-345):
// displacement_to_mapping with an affine (numerical/dif.hpp:42-51),
// inv_displacement_to_mapping (:53-66), compose_mapping of a uint8 image (:70-80),
// and exact integer moments for the correlation of two uint8 images
// (numerical/statistics.hpp:569-598).  One thread per output voxel; float
// expressions in the reference's order (the build does not contract them).
#include <algorithm>
#include "common.cuh"
#include "kernels.h"

namespace regb {

namespace {

constexpr int kMThreads = 256;

int mgrid(long long n)
{
    return (int)std::min<long long>(std::max<long long>((n + kMThreads - 1) / kMThreads, 1), 148LL * 16);
}

// mapping[i] = T(dis[i] + index)
__global__ void __launch_bounds__(kMThreads) d2m_kernel(const float* __restrict__ dis, Dim3 D, Xform T,
                                                         float* __restrict__ mapping)
{
    const long long n = D.n();
    for (long long i = (long long)blockIdx.x * kMThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kMThreads) {
        int x, y, z;
        unflat((int)i, D, x, y, z);
        const float v0 = dis[3 * i] + (float)x, v1 = dis[3 * i + 1] + (float)y, v2 = dis[3 * i + 2] + (float)z;
        float o0, o1, o2;
        apply_xform(T.m, v0, v1, v2, o0, o1, o2);
        mapping[3 * i] = o0;
        mapping[3 * i + 1] = o1;
        mapping[3 * i + 2] = o2;
    }
}

// inv_mapping[i] = p + estimate(inv_dis, p), p = iT(index); zero estimate off the field
__global__ void __launch_bounds__(kMThreads) inv_d2m_kernel(const float* __restrict__ inv_dis, Dim3 DD, Xform iT,
                                                             Dim3 MD, float* __restrict__ out)
{
    const long long n = MD.n();
    for (long long i = (long long)blockIdx.x * kMThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kMThreads) {
        int x, y, z;
        unflat((int)i, MD, x, y, z);
        float p0, p1, p2;
        apply_xform(iT.m, (float)x, (float)y, (float)z, p0, p1, p2);
        Cell c;
        float3 d = make_float3(0.0f, 0.0f, 0.0f);
        if (trilinear_cell(DD, p0, p1, p2, c))
            d = cell_sum_vec(inv_dis, DD, c);
        out[3 * i] = p0 + d.x;
        out[3 * i + 1] = p1 + d.y;
        out[3 * i + 2] = p2 + d.z;
    }
}

// to[i] = uint8 trilinear(from, mapping[i]), 0 where the cell leaves from
__global__ void __launch_bounds__(kMThreads) compose_mapping_kernel(const uint8_t* __restrict__ from, Dim3 FD,
                                                                     const float* __restrict__ mapping, Dim3 MD,
                                                                     uint8_t* __restrict__ to)
{
    const long long n = MD.n();
    for (long long i = (long long)blockIdx.x * kMThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kMThreads) {
        Cell c;
        uint8_t v = 0;
        if (trilinear_cell(FD, mapping[3 * i], mapping[3 * i + 1], mapping[3 * i + 2], c))
            v = assign_pix<uint8_t>(cell_sum(from, FD, c));
        to[i] = v;
    }
}

// m[0..5] += sum x, sum y, sum x^2, sum y^2, sum x*y, count (exact, 64-bit), over all
// voxels or, when masked, over the voxels with y > 0 (correlation_ygz)
__global__ void __launch_bounds__(kMThreads) moments_u8_kernel(const uint8_t* __restrict__ x,
                                                                const uint8_t* __restrict__ y, long long n,
                                                                int masked, unsigned long long* __restrict__ m)
{
    unsigned long long sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0, cnt = 0;
    for (long long i = (long long)blockIdx.x * kMThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kMThreads) {
        const unsigned a = x[i], b = y[i];
        if (masked && !b)
            continue;
        sx += a;
        sy += b;
        sxx += a * a;
        syy += b * b;
        sxy += a * b;
        ++cnt;
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    sxx = warp_sum(sxx);
    syy = warp_sum(syy);
    sxy = warp_sum(sxy);
    cnt = warp_sum(cnt);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(m, sx);
        atomicAdd(m + 1, sy);
        atomicAdd(m + 2, sxx);
        atomicAdd(m + 3, syy);
        atomicAdd(m + 4, sxy);
        atomicAdd(m + 5, cnt);
    }
}

// It_match_fov (reg/mm_reg.hpp:313-329): template voxels whose transformed position is
// outside the subject's volume (shape::is_valid, utility/shape.hpp:116-122) become 0
__global__ void __launch_bounds__(kMThreads) match_fov_kernel(const uint8_t* __restrict__ It, Dim3 FD, Xform T,
                                                               Dim3 MD, uint8_t* __restrict__ out)
{
    const long long n = FD.n();
    for (long long i = (long long)blockIdx.x * kMThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kMThreads) {
        int x, y, z;
        unflat((int)i, FD, x, y, z);
        float p0, p1, p2;
        apply_xform(T.m, (float)x, (float)y, (float)z, p0, p1, p2);
        const bool ok = !(p0 < 0.0f || p0 >= (float)MD.w || p1 < 0.0f || p1 >= (float)MD.h || p2 < 0.0f ||
                          p2 >= (float)MD.d);
        out[i] = ok ? It[i] : (uint8_t)0;
    }
}

}  // namespace

cudaError_t launch_match_fov_u8(const uint8_t* It, Dim3 FD, const float* T, Dim3 MD, uint8_t* out, cudaStream_t st)
{
    Xform X;
    for (int k = 0; k < 12; ++k)
        X.m[k] = T[k];
    match_fov_kernel<<<mgrid(FD.n()), kMThreads, 0, st>>>(It, FD, X, MD, out);
    return cudaGetLastError();
}

cudaError_t launch_displacement_to_mapping(const float* dis, Dim3 D, const float* T, float* mapping, cudaStream_t st)
{
    Xform X;
    for (int k = 0; k < 12; ++k)
        X.m[k] = T[k];
    d2m_kernel<<<mgrid(D.n()), kMThreads, 0, st>>>(dis, D, X, mapping);
    return cudaGetLastError();
}

cudaError_t launch_inv_displacement_to_mapping(const float* inv_dis, Dim3 DD, const float* iT, Dim3 MD, float* out,
                                               cudaStream_t st)
{
    Xform X;
    for (int k = 0; k < 12; ++k)
        X.m[k] = iT[k];
    inv_d2m_kernel<<<mgrid(MD.n()), kMThreads, 0, st>>>(inv_dis, DD, X, MD, out);
    return cudaGetLastError();
}

cudaError_t launch_compose_mapping_u8(const uint8_t* from, Dim3 FD, const float* mapping, Dim3 MD, uint8_t* to,
                                      cudaStream_t st)
{
    compose_mapping_kernel<<<mgrid(MD.n()), kMThreads, 0, st>>>(from, FD, mapping, MD, to);
    return cudaGetLastError();
}

cudaError_t launch_moments_u8(const uint8_t* x, const uint8_t* y, long long n, int masked, unsigned long long* m,
                              cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(m, 0, 6 * sizeof(unsigned long long), st);
    if (e != cudaSuccess)
        return e;
    moments_u8_kernel<<<mgrid(n), kMThreads, 0, st>>>(x, y, n, masked, m);
    return cudaGetLastError();
}

}  // namespace regb
