// regb_mi_cost_noalloc: the MI cost batch (the kernels of affine_kernels.cu) with
// every piece of scratch in one file-scope device array instead of allocations.
//
// Who needs it: code that runs where no device allocation is allowed -- a
// processing callback of a host application that owns all device memory through
// its own pool (a cudaMalloc from inside the callback may fail or stall the whole
// device), or a latency-critical loop that must not pay the implicit device-wide
// synchronisation that cudaMalloc/cudaFree can cause.  Such a caller allocates its
// inputs and outputs up front and passes them in; this entry point allocates
// nothing at all.
//
// Limits and sharing:
//   - at most kNoAllocMaxK = 16 transforms per call; scratch is 4 MiB of
//     histograms plus about 25 KiB of column sums, partial sums, counters, descriptors and the template's row
//     histogram, held by every device that loads the library until the process
//     exits;
//   - every call uses the same array; it keeps the last call's contents, so each
//     call first clears the counters it relies on.  Calls that overlap on the GPU
//     (issued on different streams, or from different host threads, without
//     ordering between them) race on the array and give wrong costs;
//   - the first call on a device looks up the array's address and, because the CUDA
//     runtime loads device code lazily, is the call on which this library's kernels
//     and the array itself are loaded into device memory: make it at initialisation;
//   - each call synchronises its stream before returning (the transform descriptors
//     are copied from a host stack array).
#include <cstring>
#include <mutex>
#include <string>
#include "affine_eval.h"
#include "host.h"
#include "stats.h"

namespace regb {

namespace {

constexpr int kNoAllocMaxK = 16;

struct NoAllocScratch {
    uint32_t hist[kNoAllocMaxK][65536];   // joint histograms, one per transform
    uint32_t col[kNoAllocMaxK][256];      // their column sums
    double part[kNoAllocMaxK][kMiReduceBlocks];  // partial sums of the MI reduction
    unsigned int ticket[kNoAllocMaxK];    // completed blocks per transform
    unsigned long long moments[kNoAllocMaxK * 3];
    int32_t row_hist[256];                // the fixed volume's value histogram
    unsigned long long sums[2];           // fixed sum x, sum x^2 (unused by MI)
    AffineTask tasks[kNoAllocMaxK];
};

static __device__ __align__(256) NoAllocScratch g_scratch;

// Device address of g_scratch per device.  The symbol name is only a host-side
// stand-in, so the address is looked up once per device with that device current.
std::mutex g_m;
NoAllocScratch* g_addr[64] = {nullptr};

NoAllocScratch* scratch_on_current_device()
{
    int dev = 0;
    REGB_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64)
        throw Failure(REGB_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> g(g_m);
    if (!g_addr[dev]) {
        void* p = nullptr;
        REGB_CK(cudaGetSymbolAddress(&p, g_scratch));
        g_addr[dev] = (NoAllocScratch*)p;
    }
    return g_addr[dev];
}

}  // namespace

}  // namespace regb

using namespace regb;

extern "C" regb_status regb_mi_cost_noalloc(const uint8_t* fixed, const int fixed_dim[3], const uint8_t* moving,
                                            const int moving_dim[3], const float* T, int K, double* cost,
                                            void* stream)
{
    try {
        if (!fixed || !moving || !fixed_dim || !moving_dim || !T || !cost)
            throw Failure(REGB_ERR_ARG, "regb_mi_cost_noalloc: null argument");
        if (K < 0 || K > kNoAllocMaxK)
            throw Failure(REGB_ERR_ARG, "regb_mi_cost_noalloc: K must be in [0, 16] (the static scratch holds "
                                        "16 joint histograms)");
        for (int i = 0; i < 3; ++i)
            if (fixed_dim[i] <= 0 || moving_dim[i] <= 0)
                throw Failure(REGB_ERR_ARG, "regb_mi_cost_noalloc: non-positive dimension");
        check_mi_width(fixed_dim[0], "regb_mi_cost_noalloc");
        const long long nf = (long long)fixed_dim[0] * fixed_dim[1] * fixed_dim[2];
        const long long nm = (long long)moving_dim[0] * moving_dim[1] * moving_dim[2];
        if (nf > (1LL << 31) - 1 || nm > (1LL << 31) - 1)
            throw Failure(REGB_ERR_ARG, "regb_mi_cost_noalloc: more than 2^31-1 voxels");
        if (K == 0)
            return REGB_OK;
        cudaStream_t st = (cudaStream_t)stream;
        // the call ends with a stream synchronisation, which a capture cannot hold
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        REGB_CK(cudaStreamIsCapturing(st, &cap));
        if (cap != cudaStreamCaptureStatusNone)
            throw Failure(REGB_ERR_ARG, "regb_mi_cost_noalloc: the call is synchronous and cannot be made while "
                                        "its stream is being captured");
        NoAllocScratch* s = scratch_on_current_device();
        // counters the kernels expect at zero; the array keeps whatever the last call left
        REGB_CK(cudaMemsetAsync(s->hist, 0, sizeof(uint32_t) * 65536 * K, st));
        REGB_CK(cudaMemsetAsync(s->col, 0, sizeof(uint32_t) * 256 * K, st));
        REGB_CK(cudaMemsetAsync(s->ticket, 0, sizeof(unsigned int) * K, st));
        REGB_CK(launch_fixed_stats(fixed, nf, s->row_hist, s->sums, st));
        AffineTask h[kNoAllocMaxK];
        const Dim3 fd{fixed_dim[0], fixed_dim[1], fixed_dim[2]}, md{moving_dim[0], moving_dim[1], moving_dim[2]};
        int max_chunks = 1;
        for (int k = 0; k < K; ++k) {
            AffineTask& t = h[k];
            std::memset(&t, 0, sizeof(t));
            t.fixed = fixed;
            t.moving = moving;
            t.fd = fd;
            t.md = md;
            std::memcpy(t.T, T + 12 * k, sizeof(t.T));
            t.row_hist = s->row_hist;
            t.hist = s->hist[k];
            t.col = s->col[k];
            t.part = s->part[k];
            t.ticket = s->ticket + k;
            t.moments = s->moments + 3 * k;
            t.cost = cost + k;
            set_task_chunks(t, REGB_COST_MI);
        }
        fill_wave(h, K, REGB_COST_MI);
        for (int k = 0; k < K; ++k)
            max_chunks = h[k].nchunk > max_chunks ? h[k].nchunk : max_chunks;
        REGB_CK(cudaMemcpyAsync(s->tasks, h, sizeof(AffineTask) * K, cudaMemcpyHostToDevice, st));
        REGB_CK(launch_mi(s->tasks, K, max_chunks, st));
        count_launch(2);  // the histogram and the reduction (launch_fixed_stats counts its own)
        // h is a stack array: the copy must have read it before returning
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    } catch (const Failure& e) {
        set_last_error(e.what());
        return e.code;
    }
}
