// Affine hot path: trilinear resample, the MI joint histogram with its MI
// reduction, and the correlation moments with the correlation cost.
//
// Reference behaviour followed:
//   resample                      numerical/resampling.hpp:1239-1298
//   get_mutual_info               reg/linear.hpp:138-169
//   get_mutual_info_mean          reg/linear.hpp:87-134
//   correlation cost              reg/linear.hpp:23-78, numerical/statistics.hpp:569-625
//
// Batching: one launch evaluates many (job, candidate transform) tasks.  Each
// task is split into voxel chunks; gridDim.y indexes tasks and gridDim.x chunks.
// The last block of a task (ticket counter) reduces that task's counts to its
// cost and clears the task's scratch, so the next launch finds it zeroed.
#include <atomic>
#include <mutex>
#include <cuda_fp16.h>
#include "common.cuh"
#include "stats.h"
#include "kernels.h"

namespace regb {

// ---------------------------------------------------------------- resample
template <typename T>
__global__ void __launch_bounds__(256) resample_kernel(const T* __restrict__ from, Dim3 fd, T* __restrict__ to,
                                                       Dim3 td, Xform X)
{
    const long long n = td.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        unflat((int)i, td, x, y, z);
        float px, py, pz;
        apply_xform(X.m, (float)x, (float)y, (float)z, px, py, pz);
        Cell c;
        T v = T(0);
        if (trilinear_cell(fd, px, py, pz, c))
            v = assign_pix<T>(cell_sum(from, fd, c));
        to[i] = v;
    }
}

// The CPU resample's integer-shift fast path (numerical/resampling.hpp:1243-1262):
// a copy of the overlap, zero elsewhere.
template <typename T>
__global__ void __launch_bounds__(256) shift_copy_kernel(const T* __restrict__ from, Dim3 fd, T* __restrict__ to,
                                                         Dim3 td, int sx, int sy, int sz)
{
    const long long n = td.n();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        unflat((int)i, td, x, y, z);
        int fx = x + sx, fy = y + sy, fz = z + sz;
        T v = T(0);
        if (fx >= 0 && fy >= 0 && fz >= 0 && fx < fd.w && fy < fd.h && fz < fd.d)
            v = from[(fz * fd.h + fy) * fd.w + fx];
        to[i] = v;
    }
}

template <typename T>
cudaError_t launch_resample(const T* from, Dim3 fd, T* to, Dim3 td, const float* Tm, const int* shift,
                            cudaStream_t st)
{
    const long long n = td.n();
    if (n == 0)
        return cudaSuccess;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    if (shift)
        shift_copy_kernel<T><<<blocks, 256, 0, st>>>(from, fd, to, td, shift[0], shift[1], shift[2]);
    else {
        Xform X;
        for (int k = 0; k < 12; ++k)
            X.m[k] = Tm[k];
        resample_kernel<T><<<blocks, 256, 0, st>>>(from, fd, to, td, X);
    }
    count_launch();
    return cudaGetLastError();
}
template cudaError_t launch_resample<uint8_t>(const uint8_t*, Dim3, uint8_t*, Dim3, const float*, const int*,
                                              cudaStream_t);
template cudaError_t launch_resample<float>(const float*, Dim3, float*, Dim3, const float*, const int*,
                                            cudaStream_t);

// ---------------------------------------------------------------- MI
// Per-block private histogram: 65536 bins packed two per 32-bit word as 16-bit
// counters (128 KB of shared memory).  A block never counts more than
// kMiChunkMax voxels, so no 16-bit counter can overflow.  Bin 0 (template 0,
// moving sample 0 -- the background) is not counted at all: its count is the
// voxel total minus every other bin, recovered in the reduction.
constexpr int kMiThreads = 768;  // 80 registers a thread at one block per SM
constexpr int kMiSmemWords = 32768;
static_assert(kMiThreads % 128 == 0 && kMiThreads >= 256, "the flush maps threads to 128 word columns");

__device__ __forceinline__ void mi_count(uint32_t* sh, uint32_t bin)
{
    if (bin != 0u)
        atomicAdd(sh + (bin >> 1), 1u << ((bin & 1u) << 4));
}

// Reduction of the complete 256x256 histograms to the reference's MI cost
// (reg/linear.hpp:87-104): with the column sums already formed by the histogram
// blocks, each of kMiReduceBlocks blocks per task sums n*ln(n/row/col) in double
// over 2048 bins (8 rows; thread t takes column t) and clears them; the last block
// of the task adds the partial sums in block order, writes -sum/65536, and clears
// the column sums and the ticket.  The order of every sum is fixed, so a task's cost
// does not depend on what it is batched with.
//
// Each term is formed as n*ln(n) - n*(ln(row) + ln(col)): n*ln(n) from a table for
// n < 65536 (g_nlogn, filled once per device), ln(row) and ln(col) once per block.
// Against n*ln(n/row/col) with its two divisions and a logarithm per bin, that is a
// few FP64 operations a bin (the reduction was FP64-throughput bound); each term
// moves by rounding only, ~1e-16 of its size, against the ~1e-16 * sqrt(bins) the
// block-parallel summation order already allows.
constexpr int kMiReduceThreads = 256;
constexpr int kMiReduceRows = 256 / kMiReduceBlocks;
constexpr int kNlognTable = 65536;
__device__ double g_nlogn[kNlognTable];  // n * ln(n); 0 for n = 0

__global__ void nlogn_table_kernel()
{
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < kNlognTable; n += gridDim.x * blockDim.x)
        g_nlogn[n] = n ? (double)n * log((double)n) : 0.0;
}

__device__ __forceinline__ double nlogn(uint32_t n)
{
    return n < (uint32_t)kNlognTable ? g_nlogn[n] : (double)n * log((double)n);
}

__global__ void __launch_bounds__(kMiReduceThreads) mi_reduce_kernel(const AffineTask* __restrict__ tasks)
{
    const AffineTask& tk = tasks[blockIdx.y];
    if (tk.keep)
        return;
    __shared__ uint32_t col[256];
    __shared__ unsigned long long red64[32];
    __shared__ double red[32];
    __shared__ unsigned int last;
    const int t = threadIdx.x;
    const uint32_t c = __ldcg(tk.col + t);
    col[t] = c;
    // every voxel is in one bin: the uncounted background bin is the remainder
    const unsigned long long tot = block_sum((unsigned long long)c, red64);
    __shared__ uint32_t n00_s;
    __shared__ double lrow[kMiReduceRows];
    if (t == 0) {
        n00_s = (uint32_t)(tk.fd.n() - (long long)tot);
        col[0] += n00_s;
    }
    if (t < kMiReduceRows) {
        const int32_t rh = tk.row_hist[blockIdx.x * kMiReduceRows + t];
        lrow[t] = rh > 0 ? log((double)rh) : 0.0;  // a row with no template voxels has no counts
    }
    __syncthreads();
    const uint32_t n00 = n00_s;
    uint32_t* __restrict__ hist = tk.hist;
    const double lcol = col[t] ? log((double)col[t]) : 0.0;
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < kMiReduceRows; ++k) {
        const int row = blockIdx.x * kMiReduceRows + k;
        const int b = row * 256 + t;
        const uint32_t n = (b == 0) ? n00 : __ldcg(hist + b);
        if (n) {
            acc += nlogn(n) - (double)n * (lrow[k] + lcol);
            hist[b] = 0u;
        }
    }
    acc = block_sum(acc, red);
    if (t == 0)
        tk.part[blockIdx.x] = acc;
    __threadfence();
    __syncthreads();
    if (t == 0)
        last = (atomicAdd(tk.ticket, 1u) == (unsigned)kMiReduceBlocks - 1u);
    __syncthreads();
    if (!last)
        return;
    __threadfence();
    if (t == 0) {
        double sum = 0.0;
        for (int i = 0; i < kMiReduceBlocks; ++i)
            sum += __ldcg(tk.part + i);
        *tk.cost = -(sum / 65536.0);
        *tk.ticket = 0u;
    }
    tk.col[t] = 0u;  // every block of the task has read the column sums
}

template <bool TEX>
__global__ void __launch_bounds__(kMiThreads, 1) mi_kernel(const AffineTask* __restrict__ tasks)
{
    extern __shared__ uint32_t sh[];
    const AffineTask& tk = tasks[blockIdx.y];
    const int chunk = blockIdx.x;
    if (chunk >= tk.nchunk)
        return;
    for (int i = threadIdx.x * 4; i < kMiSmemWords; i += blockDim.x * 4)
        *reinterpret_cast<uint4*>(sh + i) = make_uint4(0, 0, 0, 0);
    __syncthreads();
    const Dim3 fd = tk.fd;
    const SampleGeo g = sample_geo(tk.md);
    // a chunk is a run of whole rows (y, z); warps take rows, lanes take x
    const int rows = fd.h * fd.d;
    const int r0 = chunk * tk.chunk, r1 = min(rows, r0 + tk.chunk);
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const uint8_t* __restrict__ moving = tk.moving;
    const float hf = (float)tk.md.h;
    const float* __restrict__ T = tk.T;
    ColXform cx;
    cx.set(T);
    // two adjacent rows per warp at a time: their loads overlap, and the second
    // row's trilinear corners mostly fall on lines the first row just cached
    // (neighbouring warps work on neighbouring pairs at the same time)
    for (int r = r0 + 2 * (threadIdx.x >> 5); r < r1; r += 2 * nw) {
        const int rb = r + 1;
        const bool two = rb < r1;
        RowXform xa, xb;
        xa.set(T, r % fd.h, r / fd.h);
        xb.set(T, (two ? rb : r) % fd.h, (two ? rb : r) / fd.h);
        const uint8_t* __restrict__ fa = tk.fixed + (long long)r * fd.w;
        const uint8_t* __restrict__ fb = tk.fixed + (long long)(two ? rb : r) * fd.w;
        // rows r and rb share every FP instruction (packed pairs)
        const float2 yt0 = make_float2(xa.yt[0], xb.yt[0]), yt1 = make_float2(xa.yt[1], xb.yt[1]),
                     yt2 = make_float2(xa.yt[2], xb.yt[2]);
        const float2 zt0 = make_float2(xa.zt[0], xb.zt[0]), zt1 = make_float2(xa.zt[1], xb.zt[1]),
                     zt2 = make_float2(xa.zt[2], xb.zt[2]);
        const float2 s0 = bc2(cx.s[0]), s1 = bc2(cx.s[1]), s2 = bc2(cx.s[2]);
        float fx = (float)lane;
        for (int x = lane; x < fd.w; x += 32, fx += 32.0f) {
            // x*T[3a] is the same in both rows: one scalar product (never contracted) per axis
            const float2 px = add2(add2(add2(bc2(__fmul_rn(fx, cx.t0[0])), yt0), zt0), s0);
            const float2 py = add2(add2(add2(bc2(__fmul_rn(fx, cx.t0[1])), yt1), zt1), s1);
            const float2 pz = add2(add2(add2(bc2(__fmul_rn(fx, cx.t0[2])), yt2), zt2), s2);
            const uint32_t fva = __ldg(fa + x);
            const uint32_t fvb = two ? (uint32_t)__ldg(fb + x) : 0u;
            uint32_t ta, tb;
            if constexpr (TEX)
                sample_tex_pair((cudaTextureObject_t)tk.tex, g, hf, px, py, pz, true, two, ta, tb);
            else
                sample_u8_pair(moving, g, px, py, pz, true, two, ta, tb);
            mi_count(sh, (fva << 8) | ta);
            if (two)
                mi_count(sh, (fvb << 8) | tb);
        }
    }
    __syncthreads();
    // flush the non-zero counters to the task's global histogram.  Thread t walks
    // word column c = t % 128 (bins 2c, 2c+1 of every row) over rows t / 128 + 6k,
    // summing the two columns as it goes; the six partial column sums meet in
    // shared memory and go to the task's column sums.
    uint32_t* __restrict__ gh = tk.hist;
    const int wc = threadIdx.x & 127;
    uint32_t clo = 0u, chi = 0u;
    for (int r = threadIdx.x >> 7; r < 256; r += kMiThreads / 128) {
        const int wi = r * 128 + wc;
        const uint32_t w = sh[wi];
        if (w) {
            const uint32_t lo = w & 0xffffu, hi = w >> 16;
            clo += lo;
            chi += hi;
            // bins 2wi and 2wi+1 are adjacent 32-bit counters: one 64-bit add updates both
            // (a bin never exceeds the voxel count < 2^32, so no carry crosses between them)
            atomicAdd(reinterpret_cast<unsigned long long*>(gh + 2 * wi),
                      ((unsigned long long)hi << 32) | (unsigned long long)lo);
        }
    }
    __shared__ uint32_t colp[256];
    if (threadIdx.x < 256)
        colp[threadIdx.x] = 0u;
    __syncthreads();
    if (clo)
        atomicAdd(colp + 2 * wc, clo);
    if (chi)
        atomicAdd(colp + 2 * wc + 1, chi);
    __syncthreads();
    if (threadIdx.x < 256 && colp[threadIdx.x])
        atomicAdd(tk.col + threadIdx.x, colp[threadIdx.x]);
}

// g_nlogn of the current device, filled before its first reduction launch on any stream
// (the fill is synchronised before the device counts as ready, so a launch on another
// stream never reads the table half written).
static cudaError_t ensure_nlogn_table(int dev, cudaStream_t st)
{
    static std::atomic<unsigned long long> ready{0};  // one bit per device
    static std::mutex m;
    const unsigned long long bit = 1ull << (dev & 63);
    if (ready.load() & bit)
        return cudaSuccess;
    std::lock_guard<std::mutex> g(m);
    if (ready.load() & bit)
        return cudaSuccess;
    nlogn_table_kernel<<<64, 256, 0, st>>>();
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e == cudaSuccess)
        ready.fetch_or(bit);
    return e;
}

template <bool TEX>
static cudaError_t launch_mi_impl(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st)
{
    static std::atomic<unsigned long long> attr_set{0};  // one bit per device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_set.load() & bit)) {
        e = cudaFuncSetAttribute(mi_kernel<TEX>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMiSmemWords * 4);
        if (e != cudaSuccess)
            return e;
        attr_set.fetch_or(bit);
    }
    e = ensure_nlogn_table(dev, st);
    if (e != cudaSuccess)
        return e;
    dim3 grid(max_chunks, ntask);
    mi_kernel<TEX><<<grid, kMiThreads, kMiSmemWords * 4, st>>>(d_tasks);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    mi_reduce_kernel<<<dim3(kMiReduceBlocks, ntask), kMiReduceThreads, 0, st>>>(d_tasks);
    return cudaGetLastError();
}

cudaError_t launch_mi(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st)
{
    return launch_mi_impl<false>(d_tasks, ntask, max_chunks, st);
}

cudaError_t launch_mi_tex(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st)
{
    return launch_mi_impl<true>(d_tasks, ntask, max_chunks, st);
}

__global__ void __launch_bounds__(256) u8_to_half_kernel(const uint8_t* __restrict__ in, int w, long long rows,
                                                         __half* __restrict__ out, size_t pitch)
{
    const long long n = (long long)w * rows;
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
        const long long r = i / w;
        out[r * (long long)pitch + (i - r * w)] = __uint2half_rn((unsigned)in[i]);  // exact below 2048
    }
}

cudaError_t launch_u8_to_half_pitched(const uint8_t* in, int w, long long rows, void* out, size_t pitch,
                                      cudaStream_t st)
{
    const long long n = (long long)w * rows;
    if (n == 0)
        return cudaSuccess;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    u8_to_half_kernel<<<blocks, 256, 0, st>>>(in, w, rows, (__half*)out, pitch);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------- MI, 32 x 32 bins
// The same joint histogram with 5-bit bins (the reference fixes mi_band_width at 8,
// reg/linear.hpp:84-85): both volumes hold values 0..31 (quantised per pyramid level
// by normalize_upper_lower2(v, 31.99), the reference mutual_information's step for
// non-uint8 images, reg/linear.hpp:190-197), bin = (template << 5) + sample.  The
// 1024-bin per-block histogram is 4 KB of shared memory, so blocks are small and many;
// bin 0 is again recovered as the remainder.  Cost = -sum n ln(n / (row col)) / 1024.
constexpr int kMi32Threads = 768;
constexpr int kMi32Copies = 8;  // shared histogram copies; warp w counts into copy w % 8

template <bool TEX>
__global__ void __launch_bounds__(kMi32Threads, 1) mi32_kernel(const AffineTask* __restrict__ tasks)
{
    extern __shared__ uint32_t sh[];  // kMi32Copies x 1024 counters
    __shared__ uint32_t col[32];
    __shared__ double red[32];
    __shared__ unsigned long long tot;
    __shared__ unsigned int last;
    const AffineTask& tk = tasks[blockIdx.y];
    const int chunk = blockIdx.x;
    if (chunk >= tk.nchunk)
        return;
    for (int i = threadIdx.x; i < kMi32Copies * 1024; i += blockDim.x)
        sh[i] = 0u;
    __syncthreads();
    const Dim3 fd = tk.fd;
    const SampleGeo g = sample_geo(tk.md);
    const int rows = fd.h * fd.d;
    const int r0 = chunk * tk.chunk, r1 = min(rows, r0 + tk.chunk);
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    uint32_t* __restrict__ mine = sh + ((threadIdx.x >> 5) % kMi32Copies) * 1024;
    const uint8_t* __restrict__ moving = tk.moving;
    const float hf = (float)tk.md.h;
    const float* __restrict__ T = tk.T;
    ColXform cx;
    cx.set(T);
    auto count = [&](uint32_t bin, bool on) {
        if (on && bin != 0u)
            atomicAdd(mine + bin, 1u);
    };
    // the sampling loop of mi_kernel: two adjacent rows per warp, packed pair arithmetic
    for (int r = r0 + 2 * (threadIdx.x >> 5); r < r1; r += 2 * nw) {
        const int rb = r + 1;
        const bool two = rb < r1;
        RowXform xa, xb;
        xa.set(T, r % fd.h, r / fd.h);
        xb.set(T, (two ? rb : r) % fd.h, (two ? rb : r) / fd.h);
        const uint8_t* __restrict__ fa = tk.fixed + (long long)r * fd.w;
        const uint8_t* __restrict__ fb = tk.fixed + (long long)(two ? rb : r) * fd.w;
        const float2 yt0 = make_float2(xa.yt[0], xb.yt[0]), yt1 = make_float2(xa.yt[1], xb.yt[1]),
                     yt2 = make_float2(xa.yt[2], xb.yt[2]);
        const float2 zt0 = make_float2(xa.zt[0], xb.zt[0]), zt1 = make_float2(xa.zt[1], xb.zt[1]),
                     zt2 = make_float2(xa.zt[2], xb.zt[2]);
        const float2 s0 = bc2(cx.s[0]), s1 = bc2(cx.s[1]), s2 = bc2(cx.s[2]);
        // lanes past the row's end sample nothing and count nothing
        for (int x0 = 0; x0 < fd.w; x0 += 32) {
            const int x = x0 + lane;
            const bool in = x < fd.w;
            const float fx = (float)x;
            const float2 px = add2(add2(add2(bc2(__fmul_rn(fx, cx.t0[0])), yt0), zt0), s0);
            const float2 py = add2(add2(add2(bc2(__fmul_rn(fx, cx.t0[1])), yt1), zt1), s1);
            const float2 pz = add2(add2(add2(bc2(__fmul_rn(fx, cx.t0[2])), yt2), zt2), s2);
            const uint32_t fva = in ? (uint32_t)__ldg(fa + x) : 0u;
            const uint32_t fvb = (in && two) ? (uint32_t)__ldg(fb + x) : 0u;
            uint32_t ta, tb;
            if constexpr (TEX)
                sample_tex_pair((cudaTextureObject_t)tk.tex, g, hf, px, py, pz, in, in && two, ta, tb);
            else
                sample_u8_pair(moving, g, px, py, pz, in, in && two, ta, tb);
            count((fva << 5) | ta, in);
            count((fvb << 5) | tb, in && two);
        }
    }
    __syncthreads();
    uint32_t* __restrict__ gh = tk.hist;
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) {
        uint32_t v = 0u;
#pragma unroll
        for (int c = 0; c < kMi32Copies; ++c)
            v += sh[c * 1024 + i];
        if (v)
            atomicAdd(gh + i, v);
    }
    if (tk.keep)
        return;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        last = (atomicAdd(tk.ticket, 1u) == (unsigned)tk.nchunk - 1u);
    __syncthreads();
    if (!last)
        return;
    __threadfence();
    // reduction (reg/linear.hpp:87-104 with 32 x 32 bins); the block is the last one
    const int t = threadIdx.x;
    if (t < 32)
        col[t] = 0u;
    if (t == 0)
        tot = 0ull;
    __syncthreads();
    for (int b = t; b < 1024; b += blockDim.x) {
        const uint32_t v = __ldcg(gh + b);
        sh[b] = v;
        if (v) {
            atomicAdd(col + (b & 31), v);
            atomicAdd(&tot, (unsigned long long)v);
        }
    }
    __syncthreads();
    const uint32_t n00 = (uint32_t)(fd.n() - (long long)tot);
    if (t == 0) {
        sh[0] = n00;
        col[0] += n00;
    }
    __syncthreads();
    double acc = 0.0;
    for (int b = t; b < 1024; b += blockDim.x) {
        const uint32_t nb = sh[b];
        if (nb) {
            const double mu = (double)nb;
            acc += mu * log(mu / (double)tk.row_hist[b >> 5] / (double)col[b & 31]);
        }
    }
    acc = block_sum(acc, red);
    if (t == 0) {
        *tk.cost = -(acc / 1024.0);
        *tk.ticket = 0u;
    }
    for (int b = t; b < 1024; b += blockDim.x)
        gh[b] = 0u;
}

template <bool TEX>
static cudaError_t launch_mi32_impl(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st)
{
    constexpr int smem = kMi32Copies * 1024 * 4;
    static std::atomic<unsigned long long> attr_set{0};  // one bit per device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_set.load() & bit)) {
        e = cudaFuncSetAttribute(mi32_kernel<TEX>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
        attr_set.fetch_or(bit);
    }
    mi32_kernel<TEX><<<dim3(max_chunks, ntask), kMi32Threads, smem, st>>>(d_tasks);
    return cudaGetLastError();
}

cudaError_t launch_mi32(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st)
{
    return launch_mi32_impl<false>(d_tasks, ntask, max_chunks, st);
}

cudaError_t launch_mi32_tex(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st)
{
    return launch_mi32_impl<true>(d_tasks, ntask, max_chunks, st);
}

// ---------------------------------------------------------------- correlation
// Exact integer moments of the resampled moving volume y against the fixed grid
// x: sum y, sum y^2, sum x*y (the template's sum x and sum x^2 are per job).  A
// thread sums at most kCorrPerThread voxels in 32 bits (255^2 * 64 < 2^32).
constexpr int kCorrThreads = 256;

template <bool TEX>
__global__ void __launch_bounds__(kCorrThreads) corr_kernel(const AffineTask* __restrict__ tasks)
{
    const AffineTask& tk = tasks[blockIdx.y];
    const int chunk = blockIdx.x;
    if (chunk >= tk.nchunk)
        return;
    const Dim3 fd = tk.fd, md = tk.md;
    const SampleGeo g = sample_geo(md);
    const long long n = fd.n();
    const int rows = fd.h * fd.d;
    const int r0 = chunk * tk.chunk, r1 = min(rows, r0 + tk.chunk);
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const uint8_t* __restrict__ moving = tk.moving;
    const float* __restrict__ T = tk.T;
    ColXform cx;
    cx.set(T);
    uint32_t sy = 0, syy = 0, sxy = 0;
    auto acc = [&](uint32_t f, uint32_t v) {
        sy += v;
        syy += v * v;
        sxy += f * v;
    };
    if (tk.mode == 1) {
        // the CPU resample's integer-shift copy (numerical/resampling.hpp:1243-1262)
        for (int r = r0 + (threadIdx.x >> 5); r < r1; r += nw) {
            const int yy = r % fd.h, zz = r / fd.h;
            const uint8_t* __restrict__ frow = tk.fixed + (long long)r * fd.w;
            const int ay = yy + tk.shift[1], az = zz + tk.shift[2];
            const bool rowin = ay >= 0 && az >= 0 && ay < md.h && az < md.d;
            for (int x = lane; x < fd.w; x += 32) {
                const int ax = x + tk.shift[0];
                uint32_t v = 0;
                if (rowin && ax >= 0 && ax < md.w)
                    v = __ldg(moving + (az * md.h + ay) * md.w + ax);
                acc(__ldg(frow + x), v);
            }
        }
    } else {
        for (int r = r0 + 2 * (threadIdx.x >> 5); r < r1; r += 2 * nw) {
            const int rb = r + 1;
            const bool two = rb < r1;
            RowXform xa, xb;
            xa.set(T, r % fd.h, r / fd.h);
            xb.set(T, (two ? rb : r) % fd.h, (two ? rb : r) / fd.h);
            const uint8_t* __restrict__ fa = tk.fixed + (long long)r * fd.w;
            const uint8_t* __restrict__ fb = tk.fixed + (long long)(two ? rb : r) * fd.w;
            const float2 yt0 = make_float2(xa.yt[0], xb.yt[0]), yt1 = make_float2(xa.yt[1], xb.yt[1]),
                         yt2 = make_float2(xa.yt[2], xb.yt[2]);
            const float2 zt0 = make_float2(xa.zt[0], xb.zt[0]), zt1 = make_float2(xa.zt[1], xb.zt[1]),
                         zt2 = make_float2(xa.zt[2], xb.zt[2]);
            const float2 s0 = bc2(cx.s[0]), s1 = bc2(cx.s[1]), s2 = bc2(cx.s[2]);
            float fx = (float)lane;
            for (int x = lane; x < fd.w; x += 32, fx += 32.0f) {
                // x*T[3a] is the same in both rows: one scalar product (never contracted) per axis
                const float2 px = add2(add2(add2(bc2(__fmul_rn(fx, cx.t0[0])), yt0), zt0), s0);
                const float2 py = add2(add2(add2(bc2(__fmul_rn(fx, cx.t0[1])), yt1), zt1), s1);
                const float2 pz = add2(add2(add2(bc2(__fmul_rn(fx, cx.t0[2])), yt2), zt2), s2);
                uint32_t va, vb;
                if constexpr (TEX)
                    sample_tex_pair((cudaTextureObject_t)tk.tex, g, (float)md.h, px, py, pz, true, two, va, vb);
                else
                    sample_u8_pair(moving, g, px, py, pz, true, two, va, vb);
                acc(__ldg(fa + x), va);
                if (two)
                    acc(__ldg(fb + x), vb);
            }
        }
    }
    __shared__ unsigned long long red[32];
    unsigned long long a = block_sum<unsigned long long>(sy, red);
    unsigned long long b = block_sum<unsigned long long>(syy, red);
    unsigned long long c = block_sum<unsigned long long>(sxy, red);
    if (threadIdx.x == 0) {
        atomicAdd(tk.moments + 0, a);
        atomicAdd(tk.moments + 1, b);
        atomicAdd(tk.moments + 2, c);
    }
    __threadfence();
    __syncthreads();
    __shared__ unsigned int last;
    if (threadIdx.x == 0)
        last = (atomicAdd(tk.ticket, 1u) == (unsigned)tk.nchunk - 1u);
    __syncthreads();
    if (!last || threadIdx.x != 0)
        return;
    __threadfence();
    // tipl::correlation with exact integer moments (numerical/statistics.hpp:569-580),
    // then 1 - r^2 in float (reg/linear.hpp:34-35).
    const unsigned long long Sy = __ldcg(tk.moments + 0), Syy = __ldcg(tk.moments + 1), Sxy = __ldcg(tk.moments + 2);
    const double dn = (double)n;
    const double mx = (double)tk.sx / dn, my = (double)Sy / dn;
    const double vx = (double)tk.sxx / dn - mx * mx, vy = (double)Syy / dn - my * my;
    const double sd1 = vx > 0.0 ? sqrt(vx) : 0.0, sd2 = vy > 0.0 ? sqrt(vy) : 0.0;
    double r = 0.0;
    if (!(sd1 == 0.0 || sd2 == 0.0))
        r = ((double)Sxy / dn - mx * my) / sd1 / sd2;
    const float cf = (float)r;
    *tk.cost = (double)(1.0f - cf * cf);
    tk.moments[0] = tk.moments[1] = tk.moments[2] = 0ull;
    *tk.ticket = 0u;
}

cudaError_t launch_corr(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st)
{
    dim3 grid(max_chunks, ntask);
    corr_kernel<false><<<grid, kCorrThreads, 0, st>>>(d_tasks);
    return cudaGetLastError();
}

cudaError_t launch_corr_tex(const AffineTask* d_tasks, int ntask, int max_chunks, cudaStream_t st)
{
    dim3 grid(max_chunks, ntask);
    corr_kernel<true><<<grid, kCorrThreads, 0, st>>>(d_tasks);
    return cudaGetLastError();
}

int cost_blocks_per_sm(bool is_corr)
{
    if (!is_corr)
        return 1;  // __launch_bounds__(768, 1)
    static std::atomic<int> occ{0};
    int v = occ.load();
    if (!v) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, corr_kernel<true>, kCorrThreads, 0) != cudaSuccess ||
            v < 1) {
            (void)cudaGetLastError();
            v = 1;
        }
        occ.store(v);
    }
    return v;
}

// ---------------------------------------------------------------- template statistics
// Row histogram of the fixed volume (histogram(from, 0, 255, 256), which for uint8
// is the value count) and its exact sums for the correlation cost.
__global__ void fixed_stats_kernel(const uint8_t* __restrict__ f, long long n, int32_t* __restrict__ hist,
                                   unsigned long long* __restrict__ sums)
{
    __shared__ uint32_t h[256];
    __shared__ unsigned long long red[32];
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        h[i] = 0;
    __syncthreads();
    unsigned long long s = 0, ss = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        uint32_t v = __ldg(f + i);
        atomicAdd(h + v, 1u);
        s += v;
        ss += v * v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i])
            atomicAdd((unsigned int*)hist + i, h[i]);
    unsigned long long a = block_sum(s, red);
    unsigned long long b = block_sum(ss, red);
    if (threadIdx.x == 0) {
        atomicAdd(sums, a);
        atomicAdd(sums + 1, b);
    }
}

cudaError_t launch_fixed_stats(const uint8_t* f, long long n, int32_t* hist, unsigned long long* sums,
                               cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(hist, 0, 256 * sizeof(int32_t), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(sums, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess)
        return e;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 4);
    if (blocks < 1)
        blocks = 1;
    fixed_stats_kernel<<<blocks, 256, 0, st>>>(f, n, hist, sums);
    count_launch();
    return cudaGetLastError();
}

}  // namespace regb
