// Mask counts for the mask-moment initialisation of an affine registration
// (has_mask, numerical/basic_op.hpp:811-830; estimate_affine_param's moments,
// numerical/transformation.hpp:943-982).
//
// One pass over a uint8 volume makes the exact number of voxels > 0 on every
// (x, y) column, (x, z) row-plane line and (y, z) row: xy[y*w + x] (summed over z),
// xz[z*w + x] (over y), yz[z*h + y] (over x).  Every first and second coordinate
// moment, the voxel count and the bounding box follow from these three tables on
// the host, so nothing here depends on summation order.
#include "kernels.h"

namespace regb {

namespace {

constexpr int kTX = 32, kTY = 32, kZS = 16;

// grid (ceil(w/32), ceil(h/32), ceil(d/16)), block (32, 32): a 32x32 (x, y) tile
// over 16 planes.  The three tables must be zero on entry.
__global__ void __launch_bounds__(kTX * kTY) mask_count_kernel(const uint8_t* __restrict__ v, int w, int h, int d,
                                                                 uint32_t* __restrict__ xy, uint32_t* __restrict__ xz,
                                                                 uint32_t* __restrict__ yz)
{
    __shared__ uint32_t s_xz[kZS][kTX];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = blockIdx.x * kTX + tx, y = blockIdx.y * kTY + ty;
    const int z0 = blockIdx.z * kZS;
    const int tid = ty * kTX + tx;
    if (tid < kZS * kTX)
        s_xz[tid / kTX][tid % kTX] = 0;
    __syncthreads();
    const bool in = x < w && y < h;
    uint32_t col = 0;
    for (int k = 0; k < kZS; ++k) {
        const int z = z0 + k;
        if (z >= d)
            break;
        const bool m = in && v[((long long)z * h + y) * w + x] != 0;
        col += m ? 1u : 0u;
        // the warp is one row (y, z) across 32 x
        const uint32_t r = __popc(__ballot_sync(0xffffffffu, m));
        if (tx == 0 && r && y < h)
            atomicAdd(&yz[(long long)z * h + y], r);
        if (m)
            atomicAdd(&s_xz[k][tx], 1u);
    }
    if (in && col)
        atomicAdd(&xy[(long long)y * w + x], col);
    __syncthreads();
    if (tid < kZS * kTX) {
        const int k = tid / kTX, xx = blockIdx.x * kTX + tid % kTX, z = z0 + k;
        const uint32_t c = s_xz[k][tid % kTX];
        if (c && xx < w && z < d)
            atomicAdd(&xz[(long long)z * w + xx], c);
    }
}

}  // namespace

cudaError_t launch_mask_counts(const uint8_t* v, Dim3 dim, uint32_t* xy, uint32_t* xz, uint32_t* yz, cudaStream_t st)
{
    cudaError_t e;
    if ((e = cudaMemsetAsync(xy, 0, sizeof(uint32_t) * (size_t)dim.w * dim.h, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(xz, 0, sizeof(uint32_t) * (size_t)dim.w * dim.d, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(yz, 0, sizeof(uint32_t) * (size_t)dim.h * dim.d, st)) != cudaSuccess)
        return e;
    const dim3 grid((dim.w + kTX - 1) / kTX, (dim.h + kTY - 1) / kTY, (dim.d + kZS - 1) / kZS);
    mask_count_kernel<<<grid, dim3(kTX, kTY), 0, st>>>(v, dim.w, dim.h, dim.d, xy, xz, yz);
    return cudaGetLastError();
}

}  // namespace regb
