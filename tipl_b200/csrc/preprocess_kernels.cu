// Subject preprocessing of the mm_reg pipeline on the device (reg/mm_reg.hpp:14-20,
// subject_image_pre): the separable [1 2 1] Gaussian (filter/gaussian.hpp:18-88), the
// Otsu threshold histogram, the order-preserving selection of the voxels above it,
// chunked median selection (numerical/statistics.hpp:343-363) and the final
// normalisation to uint8 (numerical/otsu.hpp:110-136).
//
// Every float expression keeps the reference's evaluation order; the device build
// does not contract multiply-adds, so results are bit-identical.
#include <algorithm>
#include "kernels.h"

namespace regb {

namespace {

// ------------------------------------------------------------------ Gaussian
// One round of the reference's x, y, z passes fused in one kernel.  A block owns a
// 32 x 8 x 8 tile of outputs: it stages the tile and a one-voxel halo (34 x 10 x 10) in
// shared memory, then runs the x pass over every staged row, the y pass over the rows
// the z pass needs, and the z pass into the output -- three barriers a block, 13
// independent loads in flight per thread.  Halo and edge samples come from clamped
// coordinates, which is exactly the reference's "repeat the edge sample" rule for every
// pass (the x pass of a clamped row is the x pass of the edge row).
constexpr int kGx = 32, kGy = 8, kGz = 8, kGThreads = 256;

struct GaussSmem {
    float in[kGz + 2][kGy + 2][kGx + 2];
    float xp[kGz + 2][kGy + 2][kGx];
    float yp[kGz + 2][kGy][kGx];
};

__device__ __forceinline__ float tap3(float l, float c, float r)
{
    // (a[left] + (a[i] + a[i])) + a[right], filter/gaussian.hpp:45-48
    return __fadd_rn(__fadd_rn(l, __fadd_rn(c, c)), r);
}

__global__ void __launch_bounds__(kGThreads) gaussian_round_kernel(const float* __restrict__ in,
                                                                    float* __restrict__ out, int w, int h, int d,
                                                                    float scale, int apply_scale)
{
    extern __shared__ float4 gsm4[];
    GaussSmem& s = *reinterpret_cast<GaussSmem*>(gsm4);
    // thread (tx, ty) of a 32 x 8 block owns staged column tx + 1 of rows ty and ty + 8
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int x0 = blockIdx.x * kGx, y0 = blockIdx.y * kGy, z0 = blockIdx.z * kGz;
    const int gxc = min(x0 + tx, w - 1);
    // the two halo columns: lanes 0 and 1 also load x0 - 1 and x0 + 32 (clamped)
    const int gxh = (tx == 0) ? max(x0 - 1, 0) : min(x0 + kGx, w - 1);
    const bool row2 = ty < 2;  // rows 8 and 9 of the staged tile
    const int gy0 = min(max(y0 + ty - 1, 0), h - 1), gy1 = min(max(y0 + ty + 7, 0), h - 1);
    float c0[kGz + 2], c1[kGz + 2], h0[kGz + 2], h1[kGz + 2];
#pragma unroll
    for (int lz = 0; lz < kGz + 2; ++lz) {
        const int gz = min(max(z0 + lz - 1, 0), d - 1);
        const float* plane = in + (long long)gz * w * h;
        c0[lz] = __ldg(plane + (long long)gy0 * w + gxc);
        if (row2)
            c1[lz] = __ldg(plane + (long long)gy1 * w + gxc);
        if (tx < 2) {
            h0[lz] = __ldg(plane + (long long)gy0 * w + gxh);
            if (row2)
                h1[lz] = __ldg(plane + (long long)gy1 * w + gxh);
        }
    }
    const int hx = (tx == 0) ? 0 : kGx + 1;
#pragma unroll
    for (int lz = 0; lz < kGz + 2; ++lz) {
        s.in[lz][ty][tx + 1] = c0[lz];
        if (row2)
            s.in[lz][ty + 8][tx + 1] = c1[lz];
        if (tx < 2) {
            s.in[lz][ty][hx] = h0[lz];
            if (row2)
                s.in[lz][ty + 8][hx] = h1[lz];
        }
    }
    __syncthreads();
#pragma unroll
    for (int lz = 0; lz < kGz + 2; ++lz) {
        s.xp[lz][ty][tx] = tap3(s.in[lz][ty][tx], s.in[lz][ty][tx + 1], s.in[lz][ty][tx + 2]);
        if (row2)
            s.xp[lz][ty + 8][tx] = tap3(s.in[lz][ty + 8][tx], s.in[lz][ty + 8][tx + 1], s.in[lz][ty + 8][tx + 2]);
    }
    __syncthreads();
#pragma unroll
    for (int lz = 0; lz < kGz + 2; ++lz)
        s.yp[lz][ty][tx] = tap3(s.xp[lz][ty][tx], s.xp[lz][ty + 1][tx], s.xp[lz][ty + 2][tx]);
    __syncthreads();
    const int gx = x0 + tx, gy = y0 + ty;
    if (gx < w && gy < h) {
        float* o = out + (long long)gy * w + gx;
#pragma unroll
        for (int lz = 0; lz < kGz; ++lz) {
            const int gz = z0 + lz;
            if (gz < d) {
                float v = tap3(s.yp[lz][ty][tx], s.yp[lz + 1][ty][tx], s.yp[lz + 2][ty][tx]);
                if (apply_scale)
                    v = __fmul_rn(v, scale);
                o[(long long)gz * w * h] = v;
            }
        }
    }
}

// ------------------------------------------------------------------ Otsu histogram
// hist[clamp(floor((v - mn) * range), 0, 255)]++ over the image (numerical/basic_op.hpp:
// 1293-1311); exact integer counts, per-block shared histograms.
constexpr int kPThreads = 256;

__global__ void __launch_bounds__(kPThreads) otsu_hist_kernel(const float* __restrict__ v, long long n, float mn,
                                                               float range, unsigned* __restrict__ hist)
{
    __shared__ unsigned sh[256];
    sh[threadIdx.x] = 0u;
    __syncthreads();
    for (long long i = (long long)blockIdx.x * kPThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kPThreads) {
        const float val = __fmul_rn(__fsub_rn(v[i], mn), range);
        int b = (int)floorf(val);
        b = b < 0 ? 0 : (b > 255 ? 255 : b);
        atomicAdd(&sh[b], 1u);
    }
    __syncthreads();
    if (sh[threadIdx.x])
        atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

// ------------------------------------------------------------------ compaction
// The voxels above the threshold, in voxel order (otsu.hpp:91-95), in three steps:
// per-tile counts, an exclusive scan of the counts, and an ordered scatter.
constexpr int kTile = 4096;

__global__ void __launch_bounds__(kPThreads) above_count_kernel(const float* __restrict__ v, long long n, float ot,
                                                                 unsigned* __restrict__ counts)
{
    const long long b = (long long)blockIdx.x * kTile;
    unsigned c = 0;
    for (int k = threadIdx.x; k < kTile; k += kPThreads) {
        const long long i = b + k;
        c += (i < n && v[i] > ot) ? 1u : 0u;
    }
    __shared__ unsigned red[kPThreads / 32];
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned s = 0;
        for (int k = 0; k < kPThreads / 32; ++k)
            s += red[k];
        counts[blockIdx.x] = s;
    }
}

// One block: counts[i] -> exclusive prefix (in place); total in counts[nt].
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(unsigned* __restrict__ counts, int nt)
{
    __shared__ unsigned carry;
    __shared__ unsigned wsum[32];
    if (threadIdx.x == 0)
        carry = 0u;
    __syncthreads();
    for (int base = 0; base < nt; base += 1024) {
        const int i = base + threadIdx.x;
        const unsigned v = i < nt ? counts[i] : 0u;
        unsigned x = v;  // inclusive warp scan
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31) >= o)
                x += y;
        }
        if ((threadIdx.x & 31) == 31)
            wsum[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            unsigned ws = wsum[threadIdx.x];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, ws, o);
                if (threadIdx.x >= o)
                    ws += y;
            }
            wsum[threadIdx.x] = ws;
        }
        __syncthreads();
        const unsigned before = carry + ((threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0u) + x - v;
        if (i < nt)
            counts[i] = before;
        __syncthreads();
        if (threadIdx.x == 1023)
            carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        counts[nt] = carry;
}

// Ordered scatter: tile b writes its values above ot from offset[b] on, in order.
__global__ void __launch_bounds__(kPThreads) above_scatter_kernel(const float* __restrict__ v, long long n, float ot,
                                                                   const unsigned* __restrict__ offset,
                                                                   float* __restrict__ out)
{
    __shared__ unsigned wbase[kPThreads / 32];
    __shared__ unsigned run;
    const long long b = (long long)blockIdx.x * kTile;
    if (threadIdx.x == 0)
        run = offset[blockIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k0 = 0; k0 < kTile; k0 += kPThreads) {
        const long long i = b + k0 + threadIdx.x;
        const float x = i < n ? v[i] : 0.0f;
        const bool keep = i < n && x > ot;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0)
            wbase[wid] = __popc(m);
        __syncthreads();
        unsigned before = run;
        for (int k = 0; k < wid; ++k)
            before += wbase[k];
        if (keep)
            out[before + __popc(m & ((1u << lane) - 1u))] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned t = 0;
            for (int k = 0; k < kPThreads / 32; ++k)
                t += wbase[k];
            run += t;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ chunk medians
// median(container) (numerical/statistics.hpp:343-363) over m >= 2048 values: chunk c
// of 256 is [c*cs + min(c, rem), +cs + (c < rem)); its middle is the (len/2)-th
// smallest.  One block per chunk selects it exactly by radix selection on
// order-preserving keys, 11 + 11 + 10 bits.
__device__ __forceinline__ unsigned fkey(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void __launch_bounds__(512) chunk_median_kernel(const float* __restrict__ v, long long m,
                                                            float* __restrict__ med)
{
    __shared__ unsigned hist[2048];
    __shared__ unsigned part[512];
    __shared__ unsigned sel_bin, sel_rank;
    const long long cs = m / 256, rem = m % 256, c = blockIdx.x;
    const long long s0 = c * cs + (c < rem ? c : rem);
    const long long len = cs + (c < rem ? 1 : 0);
    const int t = threadIdx.x;
    unsigned rank = (unsigned)(len / 2);  // 0-based rank sought
    unsigned prefix = 0u, pmask = 0u;
    const int shifts[3] = {21, 10, 0}, widths[3] = {11, 11, 10};
    for (int pass = 0; pass < 3; ++pass) {
        const int sh = shifts[pass], nb = 1 << widths[pass];
        for (int i = t; i < 2048; i += blockDim.x)
            hist[i] = 0u;
        __syncthreads();
        // values of one chunk crowd into few bins: one atomic per distinct bin per warp
        for (long long i0 = 0; i0 < len; i0 += blockDim.x) {
            const long long i = i0 + t;
            bool in = i < len;
            unsigned k = in ? fkey(v[s0 + i]) : 0u;
            in = in && (k & pmask) == prefix;
            const unsigned bin = in ? (k >> sh) & (nb - 1) : 0xffffffffu;
            const unsigned peers = __match_any_sync(0xffffffffu, bin);
            if (in && (threadIdx.x & 31) == (__ffs(peers) - 1))
                atomicAdd(&hist[bin], (unsigned)__popc(peers));
        }
        __syncthreads();
        // block prefix over the bins: thread t owns bins 4t..4t+3
        unsigned own = 0u;
        for (int k = 0; k < 4; ++k)
            own += (4 * t + k < nb) ? hist[4 * t + k] : 0u;
        part[t] = own;
        __syncthreads();
        for (int o = 1; o < 512; o <<= 1) {
            const unsigned add = t >= o ? part[t - o] : 0u;
            __syncthreads();
            part[t] += add;
            __syncthreads();
        }
        const unsigned before = t ? part[t - 1] : 0u;
        if (before <= rank && rank < part[t]) {
            unsigned acc = before;
            for (int k = 0; k < 4; ++k) {
                const unsigned hk = hist[4 * t + k];
                if (rank < acc + hk) {
                    sel_bin = (unsigned)(4 * t + k);
                    sel_rank = rank - acc;
                    break;
                }
                acc += hk;
            }
        }
        __syncthreads();
        prefix |= sel_bin << sh;
        pmask |= (unsigned)(nb - 1) << sh;
        rank = sel_rank;
        __syncthreads();
    }
    if (t == 0)
        med[c] = __uint_as_float((prefix & 0x80000000u) ? (prefix & 0x7fffffffu) : ~prefix);
}

// ------------------------------------------------------------------ normalisation
// count of voxels with v * s > 0 (normalize_otsu_median's majority test)
__global__ void __launch_bounds__(kPThreads) positive_count_kernel(const float* __restrict__ v, long long n, float s,
                                                                    unsigned long long* __restrict__ cnt)
{
    unsigned c = 0;
    for (long long i = (long long)blockIdx.x * kPThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kPThreads)
        c += __fmul_rn(v[i], s) > 0.0f ? 1u : 0u;
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c)
        atomicAdd(cnt, (unsigned long long)c);
}

// out = uint8(clamp(v * s - (shift ? c : 0), 0, upper)) (otsu.hpp:126-135, then the
// float -> uint8 conversion of subject_image_pre)
__global__ void __launch_bounds__(kPThreads) otsu_normalize_kernel(const float* __restrict__ v, long long n, float s,
                                                                    int shift, float c, float upper,
                                                                    uint8_t* __restrict__ out)
{
    for (long long i = (long long)blockIdx.x * kPThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kPThreads) {
        float x = __fmul_rn(v[i], s);
        if (shift)
            x = __fsub_rn(x, c);
        x = x > upper ? upper : (x < 0.0f ? 0.0f : x);
        out[i] = (uint8_t)(unsigned)x;
    }
}

int pgrid(long long n)
{
    return (int)std::min<long long>(std::max<long long>((n + kPThreads - 1) / kPThreads, 1), 148LL * 8);
}

}  // namespace

cudaError_t launch_gaussian_round(const float* in, float* out, int w, int h, int d, float scale, int apply_scale,
                                  cudaStream_t st)
{
    static bool attr_done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 64 && !attr_done[dev]) {
        e = cudaFuncSetAttribute(gaussian_round_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(GaussSmem));
        if (e != cudaSuccess)
            return e;
        attr_done[dev] = true;
    }
    const dim3 grid((w + kGx - 1) / kGx, (h + kGy - 1) / kGy, (d + kGz - 1) / kGz);
    gaussian_round_kernel<<<grid, kGThreads, sizeof(GaussSmem), st>>>(in, out, w, h, d, scale, apply_scale);
    return cudaGetLastError();
}

cudaError_t launch_otsu_hist(const float* v, long long n, float mn, float range, unsigned* hist, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned), st);
    if (e != cudaSuccess)
        return e;
    otsu_hist_kernel<<<pgrid(n), kPThreads, 0, st>>>(v, n, mn, range, hist);
    return cudaGetLastError();
}

long long compact_tiles(long long n) { return (n + kTile - 1) / kTile; }

cudaError_t launch_compact_above(const float* v, long long n, float ot, unsigned* counts, float* out, cudaStream_t st)
{
    const long long nt = compact_tiles(n);
    if (nt > 0x7fffffffLL)
        return cudaErrorInvalidValue;
    above_count_kernel<<<(unsigned)nt, kPThreads, 0, st>>>(v, n, ot, counts);
    exclusive_scan_kernel<<<1, 1024, 0, st>>>(counts, (int)nt);
    above_scatter_kernel<<<(unsigned)nt, kPThreads, 0, st>>>(v, n, ot, counts, out);
    return cudaGetLastError();
}

cudaError_t launch_chunk_medians(const float* v, long long m, float* med, cudaStream_t st)
{
    chunk_median_kernel<<<256, 512, 0, st>>>(v, m, med);
    return cudaGetLastError();
}

cudaError_t launch_positive_count(const float* v, long long n, float s, unsigned long long* cnt, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess)
        return e;
    positive_count_kernel<<<pgrid(n), kPThreads, 0, st>>>(v, n, s, cnt);
    return cudaGetLastError();
}

cudaError_t launch_otsu_normalize(const float* v, long long n, float s, int shift, float c, float upper, uint8_t* out,
                                  cudaStream_t st)
{
    otsu_normalize_kernel<<<pgrid(n), kPThreads, 0, st>>>(v, n, s, shift, c, upper, out);
    return cudaGetLastError();
}

}  // namespace regb
