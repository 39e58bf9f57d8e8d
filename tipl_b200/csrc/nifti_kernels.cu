// Device side of the NIfTI reader: the voxel bytes of one volume, as stored in the
// file, become the float32 LPS volume in one pass.  Per output voxel: its file voxel
// through the reorientation map, the stored element (byte order swapped for a
// big-endian file), its conversion to float the way the reference's reader converts
// it (io/nifti.hpp:1033-1131: a C++ value conversion, round to nearest), then
// scl_slope / scl_inter (io/nifti.hpp:1152-1158).
#include <algorithm>
#include "common.cuh"
#include "kernels.h"
#include "stats.h"

namespace regb {

namespace {

constexpr int kNThreads = 256;

__device__ __forceinline__ uint16_t bswap16(uint16_t v) { return (uint16_t)((v >> 8) | (v << 8)); }
__device__ __forceinline__ uint32_t bswap32(uint32_t v) { return __byte_perm(v, 0u, 0x0123); }
__device__ __forceinline__ unsigned long long bswap64(unsigned long long v)
{
    const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
    return ((unsigned long long)bswap32(lo) << 32) | bswap32(hi);
}

__device__ __forceinline__ float element(const uint8_t* __restrict__ raw, long long i, int dt, bool be)
{
    switch (dt) {
    case 2: return (float)raw[i];
    case 256: return (float)(signed char)raw[i];
    case 4: {
        uint16_t v = reinterpret_cast<const uint16_t*>(raw)[i];
        return (float)(int16_t)(be ? bswap16(v) : v);
    }
    case 512: {
        uint16_t v = reinterpret_cast<const uint16_t*>(raw)[i];
        return (float)(be ? bswap16(v) : v);
    }
    case 8: {
        uint32_t v = reinterpret_cast<const uint32_t*>(raw)[i];
        return __int2float_rn((int)(be ? bswap32(v) : v));
    }
    case 768: {
        uint32_t v = reinterpret_cast<const uint32_t*>(raw)[i];
        return __uint2float_rn(be ? bswap32(v) : v);
    }
    case 16: {
        uint32_t v = reinterpret_cast<const uint32_t*>(raw)[i];
        return __uint_as_float(be ? bswap32(v) : v);
    }
    case 64: {
        unsigned long long v = reinterpret_cast<const unsigned long long*>(raw)[i];
        return __double2float_rn(__longlong_as_double((long long)(be ? bswap64(v) : v)));
    }
    case 1024: {
        unsigned long long v = reinterpret_cast<const unsigned long long*>(raw)[i];
        return __ll2float_rn((long long)(be ? bswap64(v) : v));
    }
    case 1280: {
        unsigned long long v = reinterpret_cast<const unsigned long long*>(raw)[i];
        return __ull2float_rn(be ? bswap64(v) : v);
    }
    case 128: {
        // tipl::rgb(r, g, b) as uint32 (b in the low byte, alpha 0), then to float: exact
        // below 2^24 (io/nifti.hpp:1113-1115)
        const uint8_t* p = raw + 3 * i;
        return (float)(((uint32_t)p[0] << 16) | ((uint32_t)p[1] << 8) | (uint32_t)p[2]);
    }
    default: return 0.0f;  // no conversion in the reference's read: the voxel stays 0
    }
}

__global__ void __launch_bounds__(kNThreads) nifti_convert_kernel(const uint8_t* __restrict__ raw, NiftiMap m,
                                                                    float* __restrict__ out)
{
    const long long n = (long long)m.out.w * m.out.h * m.out.d;
    for (long long i = blockIdx.x * (long long)kNThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kNThreads) {
        const long long x = i % m.out.w, t = i / m.out.w, y = t % m.out.h, z = t / m.out.h;
        const long long sx = m.M[0] * x + m.M[1] * y + m.M[2] * z + m.o[0];
        const long long sy = m.M[3] * x + m.M[4] * y + m.M[5] * z + m.o[1];
        const long long sz = m.M[6] * x + m.M[7] * y + m.M[8] * z + m.o[2];
        float v = element(raw, (sz * m.file.h + sy) * m.file.w + sx, m.datatype, m.big_endian != 0);
        if (m.scl_slope != 0.0f) {
            if (m.scl_slope != 1.0f)
                v = v * m.scl_slope;
            if (m.scl_inter != 0.0f)
                v = v + m.scl_inter;
        }
        out[i] = v;
    }
}

}  // namespace

cudaError_t launch_nifti_convert(const uint8_t* raw, const NiftiMap& m, float* out, cudaStream_t st)
{
    const long long n = (long long)m.out.w * m.out.h * m.out.d;
    if (n <= 0)
        return cudaSuccess;
    const int blocks = (int)std::min<long long>((n + kNThreads - 1) / kNThreads, 148LL * 16);
    nifti_convert_kernel<<<blocks, kNThreads, 0, st>>>(raw, m, out);
    count_launch();
    return cudaGetLastError();
}

}  // namespace regb
