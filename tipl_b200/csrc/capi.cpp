// extern "C" entry points of libregb200.so (declared in include/regb200.h).
// Every entry validates its views, stages host memory through device buffers when
// a view lives on the host, and turns failures into regb_status codes.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include "affine_eval.h"
#include "cdm_level.h"
#include "host.h"
#include "nifti.h"
#include "mask_init.h"
#include "preprocess.h"
#include "stats.h"

namespace regb {
const std::string& last_error();
}

using namespace regb;

namespace {

const long long kMaxVoxels = (1LL << 31) - 1;

void check_dims(const int* d, const char* what)
{
    if (d[0] <= 0 || d[1] <= 0 || d[2] <= 0)
        throw Failure(REGB_ERR_ARG, std::string(what) + ": non-positive dimension");
    if ((long long)d[0] * d[1] * d[2] > kMaxVoxels)
        throw Failure(REGB_ERR_ARG, std::string(what) + ": more than 2^31-1 voxels");
}

void check_vol(const regb_volume* v, const char* what, bool u8_or_f32 = true)
{
    if (!v || !v->ptr)
        throw Failure(REGB_ERR_ARG, std::string(what) + ": null volume");
    check_dims(v->dim, what);
    if (u8_or_f32 && v->dtype != REGB_U8 && v->dtype != REGB_F32)
        throw Failure(REGB_ERR_ARG, std::string(what) + ": dtype must be U8 or F32");
    if (v->location != REGB_HOST && v->location != REGB_DEVICE)
        throw Failure(REGB_ERR_ARG, std::string(what) + ": bad location");
}

void check_field(const regb_field* f, const char* what)
{
    if (!f || !f->ptr)
        throw Failure(REGB_ERR_ARG, std::string(what) + ": null field");
    check_dims(f->dim, what);
    if (f->location != REGB_HOST && f->location != REGB_DEVICE)
        throw Failure(REGB_ERR_ARG, std::string(what) + ": bad location");
}

bool same_dims(const int* a, const int* b) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; }
size_t nvox(const int* d) { return (size_t)d[0] * d[1] * d[2]; }

// Device view of a volume or field; host data is staged through an owned buffer.
// Image pairs one affine search takes (the reference's mm_reg holds at most 12 modalities).
constexpr int kMaxLinearPairs = 12;

struct Staged {
    DevBuf<uint8_t> own;
    void* d = nullptr;
    size_t bytes = 0;
    bool host = false;
    void in(void* ptr, size_t b, int location, cudaStream_t st, bool copy)
    {
        bytes = b;
        host = (location == REGB_HOST);
        if (!host) {
            d = ptr;
            return;
        }
        own.alloc(b, st);
        d = own.p;
        if (copy)
            REGB_CK(cudaMemcpyAsync(d, ptr, b, cudaMemcpyHostToDevice, st));
    }
    void out(void* ptr, cudaStream_t st)
    {
        if (host)
            REGB_CK(cudaMemcpyAsync(ptr, d, bytes, cudaMemcpyDeviceToHost, st));
    }
};

template <typename F>
regb_status guarded(F&& f)
{
    try {
        return f();
    } catch (const Failure& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return REGB_ERR_NOMEM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return REGB_ERR_ARG;
    }
}

// A single-segment CDM view for the standalone passes.
struct OneSeg {
    DevBuf<CdmSeg> seg;
    DevBuf<CdmCtl> ctl;
    DevBuf<double> part;
    CdmSeg h{};
    CdmCtl c{};
    OneSeg(const int* dim, cudaStream_t st)
    {
        h.w = dim[0];
        h.h = dim[1];
        h.d = dim[2];
        h.nblk = cdm_blocks_for((long long)dim[0] * dim[1] * dim[2]);
        part.alloc(h.nblk, st);
        ctl.alloc(1, st);
        seg.alloc(1, st);
        h.cost_part = part.p;
        h.ctl = ctl.p;
        std::memset(&c, 0, sizeof(c));
        c.max_iter = 200;
    }
    void upload(cudaStream_t st)
    {
        REGB_CK(cudaMemcpyAsync(ctl.p, &c, sizeof(c), cudaMemcpyHostToDevice, st));
        REGB_CK(cudaMemcpyAsync(seg.p, &h, sizeof(h), cudaMemcpyHostToDevice, st));
        REGB_CK(cudaStreamSynchronize(st));
    }
};

int pix_of(int dtype) { return dtype == REGB_F32 ? 1 : 0; }

}  // namespace

namespace regb {
namespace {
std::atomic<size_t> g_fail_bytes{0};
std::atomic<int> g_fail_count{0};
}  // namespace

bool alloc_fault_injected(size_t bytes)
{
    if (g_fail_count.load(std::memory_order_relaxed) <= 0 || g_fail_bytes.load(std::memory_order_relaxed) != bytes)
        return false;
    return g_fail_count.fetch_sub(1) > 0;
}
}  // namespace regb

extern "C" {

void regb_linear_param_default(regb_linear_param* p)
{
    if (!p)
        return;
    p->reg_type = REGB_REG_AFFINE;
    p->cost_type = REGB_COST_MI;
    p->bound = REGB_BOUND_REG;
    p->search_count = 16;
    p->absolute_bound = 1;
}

void regb_cdm_param_default(regb_cdm_param* p)
{
    if (!p)
        return;
    p->resolution = 2.0f;
    p->speed = 0.3f;
    p->smoothing = 0.05f;
    p->min_dimension = 16;
    p->gradient_type = 'r';
}

const char* regb_version(void) { return "regb200 1.0 (sm_100a)"; }
const char* regb_last_error(void) { return last_error().c_str(); }

regb_status regb_device_info(int* device, int* sm_count, size_t* free_bytes, size_t* total_bytes)
{
    return guarded([&] {
        int dev = 0;
        REGB_CK(cudaGetDevice(&dev));
        int sms = 0;
        REGB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        size_t fr = 0, tot = 0;
        REGB_CK(cudaMemGetInfo(&fr, &tot));
        if (device) *device = dev;
        if (sm_count) *sm_count = sms;
        if (free_bytes) *free_bytes = fr;
        if (total_bytes) *total_bytes = tot;
        return REGB_OK;
    });
}

regb_status regb_debug_fail_allocations(size_t bytes, int count)
{
    if (count < 0)
        return REGB_ERR_ARG;
    g_fail_count.store(0);
    g_fail_bytes.store(bytes);
    g_fail_count.store(count);
    return REGB_OK;
}

regb_status regb_release(void)
{
    return guarded([&] {
        int dev = 0;
        REGB_CK(cudaGetDevice(&dev));
        cudaMemPool_t pool;
        REGB_CK(cudaDeviceGetDefaultMemPool(&pool, dev));
        REGB_CK(cudaDeviceSynchronize());
        REGB_CK(cudaMemPoolTrimTo(pool, 0));
        pinned_trim();
        return REGB_OK;
    });
}

regb_status regb_autotune_buckets(const char* cache_path, int tuned[12], double* seconds, int* from_cache)
{
    return guarded([&] {
        Stream s;
        int chosen[kTuneBuckets * 3] = {0};
        const double dt = autotune_cost_kernels(s.s, chosen, cache_path, from_cache);
        s.sync();
        if (tuned)
            std::memcpy(tuned, chosen, sizeof(chosen));
        if (seconds)
            *seconds = dt;
        return REGB_OK;
    });
}

regb_status regb_autotune(int tuned[3], double* seconds)
{
    int table[kTuneBuckets * 3];
    const regb_status st = regb_autotune_buckets(nullptr, table, seconds, nullptr);
    if (st == REGB_OK && tuned)
        std::memcpy(tuned, table + 3 * tune_bucket(182LL * 218 * 182), 3 * sizeof(int));
    return st;
}

regb_status regb_tuning_get_buckets(int tuned[12])
{
    if (!tuned)
        return REGB_ERR_ARG;
    for (int b = 0; b < kTuneBuckets; ++b)
        for (int c = 0; c < 3; ++c)
            tuned[b * 3 + c] = min_block_voxels(b, c);
    return REGB_OK;
}

regb_status regb_tuning_get(int tuned[3])
{
    if (!tuned)
        return REGB_ERR_ARG;
    for (int c = 0; c < 3; ++c)
        tuned[c] = min_block_voxels(tune_bucket(182LL * 218 * 182), c);
    return REGB_OK;
}

regb_status regb_affine_to_matrix(const float param[12], const int from_dim[3], const float from_vs[3],
                                  const int to_dim[3], const float to_vs[3], float T[12])
{
    if (!param || !from_dim || !from_vs || !to_dim || !to_vs || !T)
        return REGB_ERR_ARG;
    affine_to_matrix(param, from_dim, from_vs, to_dim, to_vs, T);
    return REGB_OK;
}

regb_status regb_affine_to_matrix_f64(const double param[12], const int from_dim[3], const double from_vs[3],
                                      const int to_dim[3], const double to_vs[3], double T[12])
{
    if (!param || !from_dim || !from_vs || !to_dim || !to_vs || !T)
        return REGB_ERR_ARG;
    affine_to_matrix_f64(param, from_dim, from_vs, to_dim, to_vs, T);
    return REGB_OK;
}

regb_status regb_matrix_inverse(float T[12])
{
    if (!T)
        return REGB_ERR_ARG;
    return matrix_inverse(T) ? REGB_OK : REGB_FALSE;
}

regb_status regb_matrix_to_affine_param(const float T[12], const int from_dim[3], const float from_vs[3],
                                        const int to_dim[3], const float to_vs[3], float param[12])
{
    return guarded([&] {
        if (!T || !from_dim || !from_vs || !to_dim || !to_vs || !param)
            throw Failure(REGB_ERR_ARG, "null argument");
        matrix_to_affine_param(T, from_dim, from_vs, to_dim, to_vs, param);
        return REGB_OK;
    });
}

regb_status regb_normalize_to_u8(const regb_volume* in, regb_volume* out, float upper, void* stream)
{
    return guarded([&] {
        check_vol(in, "in", false);
        check_vol(out, "out");
        if (!pix_size(in->dtype) || out->dtype != REGB_U8 || !same_dims(in->dim, out->dim))
            throw Failure(REGB_ERR_ARG, "normalize: in U8/F32/U16/BF16, out U8 of the same shape");
        const bool dev = in->location == REGB_DEVICE && out->location == REGB_DEVICE;
        std::unique_ptr<Stream> own;  // only when the caller's stream is not used
        cudaStream_t st = (dev && stream) ? (cudaStream_t)stream : (own = std::make_unique<Stream>())->s;
        const size_t n = nvox(in->dim);
        Staged a, b;
        a.in(in->ptr, n * pix_size(in->dtype), in->location, st, true);
        b.in(out->ptr, n, out->location, st, true);
        DevBuf<unsigned> mm(2, st);
        REGB_CK(launch_normalize_to_u8(a.d, in->dtype, (long long)n, upper, (uint8_t*)b.d, mm.p, st));
        count_launch(2);
        b.out(out->ptr, st);
        unsigned h[2];
        REGB_CK(cudaMemcpyAsync(h, mm.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        REGB_CK(cudaStreamSynchronize(st));
        return h[0] == h[1] ? REGB_FALSE : REGB_OK;
    });
}

regb_status regb_widen_to_f32(const regb_volume* in, regb_volume* out, void* stream)
{
    return guarded([&] {
        check_vol(in, "in", false);
        check_vol(out, "out");
        if (!pix_size(in->dtype) || in->dtype == REGB_F32 || out->dtype != REGB_F32 ||
            !same_dims(in->dim, out->dim))
            throw Failure(REGB_ERR_ARG, "widen: in U8/U16/BF16, out F32 of the same shape");
        const bool dev = in->location == REGB_DEVICE && out->location == REGB_DEVICE;
        std::unique_ptr<Stream> own;  // only when the caller's stream is not used
        cudaStream_t st = (dev && stream) ? (cudaStream_t)stream : (own = std::make_unique<Stream>())->s;
        const size_t n = nvox(in->dim);
        Staged a, b;
        a.in(in->ptr, n * pix_size(in->dtype), in->location, st, true);
        b.in(out->ptr, n * 4, out->location, st, false);
        REGB_CK(launch_widen_to_f32(a.d, in->dtype, (long long)n, (float*)b.d, st));
        count_launch();
        b.out(out->ptr, st);
        if (!dev || !stream)
            REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_gaussian(const regb_volume* in, regb_volume* out, int bandwidth, void* stream)
{
    return guarded([&] {
        check_vol(in, "in");
        check_vol(out, "out");
        if (in->dtype != REGB_F32 || out->dtype != REGB_F32 || !same_dims(in->dim, out->dim) || bandwidth < 0 ||
            bandwidth > 64)
            throw Failure(REGB_ERR_ARG, "gaussian: F32 in and out of one shape, bandwidth 0..64");
        if (in->ptr == out->ptr)
            throw Failure(REGB_ERR_ARG, "gaussian: in and out must be distinct");
        const bool dev = in->location == REGB_DEVICE && out->location == REGB_DEVICE;
        std::unique_ptr<Stream> own;  // only when the caller's stream is not used
        cudaStream_t st = (dev && stream) ? (cudaStream_t)stream : (own = std::make_unique<Stream>())->s;
        const size_t n = nvox(in->dim);
        Staged a, b;
        a.in(in->ptr, n * 4, in->location, st, true);
        b.in(out->ptr, n * 4, out->location, st, false);
        gaussian((const float*)a.d, in->dim, bandwidth, (float*)b.d, st);
        b.out(out->ptr, st);
        if (!dev || !stream)
            REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_subject_image_pre(const regb_volume* in, regb_volume* out, void* stream)
{
    return guarded([&] {
        check_vol(in, "in", false);
        check_vol(out, "out");
        if (!pix_size(in->dtype) || out->dtype != REGB_U8 || !same_dims(in->dim, out->dim))
            throw Failure(REGB_ERR_ARG, "subject_image_pre: in U8/F32/U16/BF16, out U8 of the same shape");
        const bool dev = in->location == REGB_DEVICE && out->location == REGB_DEVICE;
        std::unique_ptr<Stream> own;  // only when the caller's stream is not used
        cudaStream_t st = (dev && stream) ? (cudaStream_t)stream : (own = std::make_unique<Stream>())->s;
        const size_t n = nvox(in->dim);
        Staged a, b;
        a.in(in->ptr, n * pix_size(in->dtype), in->location, st, true);
        b.in(out->ptr, n, out->location, st, false);
        DevBuf<float> wide;
        const float* f = (const float*)a.d;
        if (in->dtype != REGB_F32) {
            wide.alloc(n, st);
            REGB_CK(launch_widen_to_f32(a.d, in->dtype, (long long)n, wide.p, st));
            count_launch();
            f = wide.p;
        }
        subject_image_pre(f, in->dim, (uint8_t*)b.d, st);
        b.out(out->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_has_mask(const regb_volume* img, int* out)
{
    return guarded([&] {
        check_vol(img, "img");
        if (img->dtype != REGB_U8 || !out)
            throw Failure(REGB_ERR_ARG, "has_mask takes a uint8 volume and an output");
        Stream s;
        Staged a;
        a.in(img->ptr, nvox(img->dim), img->location, s.s, true);
        MaskCounts c;
        mask_counts((const uint8_t*)a.d, img->dim, c, s.s);
        *out = has_mask(c) ? 1 : 0;
        return REGB_OK;
    });
}

regb_status regb_estimate_affine_param(const regb_volume* source, const float source_vs[3],
                                       const regb_volume* target, const float target_vs[3], float param[12])
{
    return guarded([&] {
        check_vol(source, "source");
        check_vol(target, "target");
        if (source->dtype != REGB_U8 || target->dtype != REGB_U8)
            throw Failure(REGB_ERR_ARG, "estimate_affine_param takes uint8 volumes");
        if (!source_vs || !target_vs || !param)
            throw Failure(REGB_ERR_ARG, "null voxel size / param");
        Stream s;
        Staged a, b;
        a.in(source->ptr, nvox(source->dim), source->location, s.s, true);
        b.in(target->ptr, nvox(target->dim), target->location, s.s, true);
        MaskCounts cs, ct;
        mask_counts((const uint8_t*)a.d, source->dim, cs, s.s);
        mask_counts((const uint8_t*)b.d, target->dim, ct, s.s);
        return estimate_affine_param(cs, source_vs, ct, target_vs, param) ? REGB_OK : REGB_FALSE;
    });
}

regb_status regb_resample(const regb_volume* from, regb_volume* to, const float T[12], int allow_shift_copy,
                          void* stream)
{
    return guarded([&] {
        check_vol(from, "from");
        check_vol(to, "to");
        if (!T)
            throw Failure(REGB_ERR_ARG, "null transform");
        if (from->dtype != to->dtype)
            throw Failure(REGB_ERR_ARG, "from/to dtype differ");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t ps = pix_size(from->dtype);
        Staged a, b;
        a.in(from->ptr, nvox(from->dim) * ps, from->location, st, true);
        b.in(to->ptr, nvox(to->dim) * ps, to->location, st, false);
        int shift[3];
        const int* sh = (allow_shift_copy && integer_shift(T, shift)) ? shift : nullptr;
        Dim3 fd{from->dim[0], from->dim[1], from->dim[2]}, td{to->dim[0], to->dim[1], to->dim[2]};
        if (from->dtype == REGB_U8)
            REGB_CK(launch_resample<uint8_t>((const uint8_t*)a.d, fd, (uint8_t*)b.d, td, T, sh, st));
        else
            REGB_CK(launch_resample<float>((const float*)a.d, fd, (float*)b.d, td, T, sh, st));
        b.out(to->ptr, st);
        if (a.host || b.host)
            REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

static regb_status affine_cost(const regb_volume* fixed, const regb_volume* moving, const float* T, int K,
                               double* cost, int32_t* hist_out, int cost_type, void* stream)
{
    return guarded([&] {
        check_vol(fixed, "fixed");
        check_vol(moving, "moving");
        if (fixed->dtype != REGB_U8 || moving->dtype != REGB_U8)
            throw Failure(REGB_ERR_ARG, "affine costs take uint8 volumes (reg/linear.hpp:622-629)");
        if (!T || !cost || K < 0)
            throw Failure(REGB_ERR_ARG, "bad transform/cost arguments");
        if (cost_type == REGB_COST_MI)
            check_mi_width(fixed->dim[0], "regb_mi_cost");
        if (K == 0)
            return REGB_OK;
        cudaStream_t st = (cudaStream_t)stream;
        Staged a, b;
        a.in(fixed->ptr, nvox(fixed->dim), fixed->location, st, true);
        b.in(moving->ptr, nvox(moving->dim), moving->location, st, true);
        AffineEvaluator::Pair pr{(const uint8_t*)a.d, Dim3{fixed->dim[0], fixed->dim[1], fixed->dim[2]},
                                 (const uint8_t*)b.d, Dim3{moving->dim[0], moving->dim[1], moving->dim[2]}};
        AffineEvaluator ev({pr}, cost_type, st);
        if (hist_out && cost_type != REGB_COST_CORR) {
            // histograms requested: evaluate one task at a time and read its counts
            // before the kernel's last block clears them.
            const int nb = cost_type == REGB_COST_MI ? 65536 : 1024;
            TaskScratch s;
            s.ensure(1, true, st);
            PinBuf<uint32_t> h(65536);
            for (int k = 0; k < K; ++k) {
                ev.make_task(0, T + 12 * k, s.h_tasks.p[0]);
                AffineTask& t = s.h_tasks.p[0];
                t.ticket = s.ticket.p;
                t.cost = s.cost.p;
                t.moments = s.moments.p;
                t.hist = s.hist.p;
                t.col = s.col.p;
                t.part = s.part.p;
                t.keep = 1;  // leave the counts in place for the read-back
                REGB_CK(cudaMemcpyAsync(s.tasks.p, s.h_tasks.p, sizeof(AffineTask), cudaMemcpyHostToDevice, st));
                if (cost_type == REGB_COST_MI)
                    REGB_CK(launch_mi(s.tasks.p, 1, t.nchunk, st));
                else
                    REGB_CK(launch_mi32(s.tasks.p, 1, t.nchunk, st));
                count_launch(cost_type == REGB_COST_MI ? 2 : 1);
                REGB_CK(cudaMemcpyAsync(h.p, s.hist.p, (size_t)nb * 4, cudaMemcpyDeviceToHost, st));
                REGB_CK(cudaStreamSynchronize(st));
                // bin 0 is not counted on the device; it is the remainder
                long long tot = 0;
                for (int i = 1; i < nb; ++i)
                    tot += h.p[i];
                h.p[0] = (uint32_t)((long long)nvox(fixed->dim) - tot);
                std::memcpy(hist_out + (size_t)k * nb, h.p, (size_t)nb * 4);
                REGB_CK(cudaMemsetAsync(s.hist.p, 0, (size_t)nb * 4, st));
                REGB_CK(cudaMemsetAsync(s.col.p, 0, 256 * 4, st));
            }
        }
        std::vector<double> c = ev.eval(0, T, K);
        std::memcpy(cost, c.data(), sizeof(double) * K);
        return REGB_OK;
    });
}

regb_status regb_mi_cost(const regb_volume* fixed, const regb_volume* moving, const float* T, int K, double* cost,
                         int32_t* hist_out, void* stream)
{
    return affine_cost(fixed, moving, T, K, cost, hist_out, REGB_COST_MI, stream);
}

regb_status regb_mi32_cost(const regb_volume* fixed, const regb_volume* moving, const float* T, int K, double* cost,
                           int32_t* hist_out, void* stream)
{
    return affine_cost(fixed, moving, T, K, cost, hist_out, REGB_COST_MI32, stream);
}

regb_status regb_corr_cost(const regb_volume* fixed, const regb_volume* moving, const float* T, int K, double* cost,
                           void* stream)
{
    return affine_cost(fixed, moving, T, K, cost, nullptr, REGB_COST_CORR, stream);
}

static void fill_nifti_info(const NiftiFile& f, regb_nifti_info* info)
{
    std::memset(info, 0, sizeof(*info));
    const NiftiHeader& h = f.h;
    for (int i = 0; i < 3; ++i) {
        info->dim[i] = h.dim[i + 1];
        info->vs[i] = h.pixdim[i + 1];
    }
    std::memcpy(info->srow, h.srow, sizeof(info->srow));
    for (int i = 0; i < 8; ++i)
        info->file_dim[i] = f.file_dim[i];
    info->datatype = h.datatype;
    info->bitpix = h.bitpix;
    long long nvol = 1;
    for (int i = 4; i <= 7 && i <= f.file_dim[0]; ++i)
        nvol *= std::max<int>(f.file_dim[i], 1);
    info->nvolumes = (int)nvol;
    info->scl_slope = h.scl_slope;
    info->scl_inter = h.scl_inter;
    info->sform_code = h.sform_code;
    const float* R = h.srow;
    // gz_nifti::is_mni (io/nifti.hpp:856-864)
    info->is_mni = h.sform_code >= 4 && R[3] != 0.0f && R[7] != 0.0f && R[11] != 0.0f && R[1] == 0.0f &&
                   R[2] == 0.0f && R[4] == 0.0f && R[6] == 0.0f && R[8] == 0.0f && R[9] == 0.0f;
    info->big_endian = h.big_endian ? 1 : 0;
    info->nifti2 = h.nifti2 ? 1 : 0;
    info->n_steps = (int)f.seq.size();
    for (size_t i = 0; i < f.seq.size() && i < 8; ++i)
        info->steps[i] = f.seq[i];
    std::memcpy(info->descrip, h.descrip, 80);
    info->descrip[80] = 0;
}

regb_status regb_nifti_info_read(const char* path, regb_nifti_info* info)
{
    return guarded([&] {
        if (!path || !info)
            throw Failure(REGB_ERR_ARG, "null argument");
        fill_nifti_info(nifti_open(path), info);
        return REGB_OK;
    });
}

regb_status regb_nifti_load(const char* path, int volume, regb_volume* out, regb_nifti_info* info, void* stream)
{
    return guarded([&] {
        if (!path)
            throw Failure(REGB_ERR_ARG, "null path");
        check_vol(out, "out");
        if (out->dtype != REGB_F32)
            throw Failure(REGB_ERR_ARG, "regb_nifti_load writes float32 volumes");
        const NiftiFile f = nifti_open(path);
        if (info)
            fill_nifti_info(f, info);
        for (int i = 0; i < 3; ++i)
            if (out->dim[i] != f.h.dim[i + 1])
                throw Failure(REGB_ERR_ARG, "out dims differ from the file's (LPS) dims");
        const std::vector<uint8_t> bytes = nifti_read_voxels(path, f, volume);
        cudaStream_t st = (cudaStream_t)stream;
        DevBuf<uint8_t> raw(bytes.size(), st);
        REGB_CK(cudaMemcpyAsync(raw.p, bytes.data(), bytes.size(), cudaMemcpyHostToDevice, st));
        Staged o;
        o.in(out->ptr, nvox(out->dim) * sizeof(float), out->location, st, false);
        NiftiMap m;
        m.file = Dim3{f.file_dim[1], f.file_dim[2], f.file_dim[3]};
        m.out = Dim3{out->dim[0], out->dim[1], out->dim[2]};
        std::memcpy(m.M, f.M, sizeof(m.M));
        for (int i = 0; i < 3; ++i)
            m.o[i] = f.o[i];
        m.datatype = f.h.datatype;
        m.big_endian = f.h.big_endian ? 1 : 0;
        m.scl_slope = f.h.scl_slope;
        m.scl_inter = f.h.scl_inter;
        REGB_CK(launch_nifti_convert(raw.p, m, (float*)o.d, st));
        o.out(out->ptr, st);
        if (o.host)
            REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_nifti_save(const char* path, const regb_volume* vol, const float vs[3], const float srow[12],
                            int is_mni, const char* descrip)
{
    return guarded([&] {
        if (!path || !vs || !srow)
            throw Failure(REGB_ERR_ARG, "null argument");
        check_vol(vol, "vol", false);
        // the reference's type table (io/nifti.hpp:264-330): uint16 is written with the
        // int16 code
        int dt = 0, bp = 0;
        switch (vol->dtype) {
        case REGB_U8: dt = 2; bp = 8; break;
        case REGB_U16: dt = 4; bp = 16; break;
        case REGB_F32: dt = 16; bp = 32; break;
        default: throw Failure(REGB_ERR_ARG, "regb_nifti_save takes U8, U16 or F32 volumes");
        }
        for (int i = 0; i < 3; ++i)
            if (vol->dim[i] > 32767)
                throw Failure(REGB_ERR_ARG, "NIfTI-1 dims are at most 32767");
        const size_t bytes = nvox(vol->dim) * (size_t)(bp / 8);
        std::vector<uint8_t> h;
        const void* data = vol->ptr;
        if (vol->location == REGB_DEVICE) {
            h.resize(bytes);
            REGB_CK(cudaMemcpy(h.data(), vol->ptr, bytes, cudaMemcpyDeviceToHost));
            data = h.data();
        }
        nifti_write(path, data, dt, bp, vol->dim, vs, srow, is_mni ? 4 : 1, descrip);
        return REGB_OK;
    });
}

regb_status regb_mm_reg_export_fields(const char* path, const regb_field* f2t, const regb_field* t2f, const float vs[3],
                                      const float srow[12])
{
    return guarded([&] {
        if (!path || !vs || !srow)
            throw Failure(REGB_ERR_ARG, "null argument");
        check_field(f2t, "f2t");
        check_field(t2f, "t2f");
        if (!same_dims(f2t->dim, t2f->dim))
            throw Failure(REGB_ERR_ARG, "export: f2t and t2f shapes differ");
        for (int i = 0; i < 3; ++i)
            if (f2t->dim[i] > 32767)
                throw Failure(REGB_ERR_ARG, "NIfTI-1 dims are at most 32767");
        const size_t n = nvox(f2t->dim);
        std::vector<float> a(3 * n), b(3 * n), buf(6 * n);
        const regb_field* src[2] = {f2t, t2f};
        std::vector<float>* dst[2] = {&a, &b};
        for (int k = 0; k < 2; ++k) {
            if (src[k]->location == REGB_DEVICE)
                REGB_CK(cudaMemcpy(dst[k]->data(), src[k]->ptr, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost));
            else
                std::memcpy(dst[k]->data(), src[k]->ptr, sizeof(float) * 3 * n);
        }
        // volume c < 3 is f2t's component c, volume 3 + c is t2f's (reg/mm_reg.hpp:421-438)
        for (int c = 0; c < 3; ++c)
            for (size_t i = 0; i < n; ++i) {
                buf[c * n + i] = a[3 * i + c];
                buf[(3 + c) * n + i] = b[3 * i + c];
            }
        nifti_write(path, buf.data(), 16, 32, f2t->dim, vs, srow, 1, nullptr, 6);
        return REGB_OK;
    });
}

regb_status regb_compose_displacement(const regb_volume* from, const regb_field* dis, regb_volume* to, void* stream)
{
    return guarded([&] {
        check_vol(from, "from");
        check_field(dis, "dis");
        check_vol(to, "to");
        if (!same_dims(from->dim, dis->dim) || !same_dims(from->dim, to->dim) || from->dtype != to->dtype)
            throw Failure(REGB_ERR_ARG, "compose: shapes/dtypes differ");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t n = nvox(from->dim), ps = pix_size(from->dtype);
        Staged a, f, o;
        a.in(from->ptr, n * ps, from->location, st, true);
        f.in(dis->ptr, n * 12, dis->location, st, true);
        o.in(to->ptr, n * ps, to->location, st, false);
        OneSeg s(from->dim, st);
        s.h.Is[0] = a.d;
        s.h.cur_d = (float*)f.d;
        s.h.Js = o.d;
        s.upload(st);
        REGB_CK(launch_cdm_compose(s.seg.p, 1, s.h.nblk, pix_of(from->dtype), st));
        o.out(to->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_displacement_to_mapping(const regb_field* dis, const float T[12], regb_field* mapping, void* stream)
{
    return guarded([&] {
        check_field(dis, "dis");
        check_field(mapping, "mapping");
        if (!T || !same_dims(dis->dim, mapping->dim))
            throw Failure(REGB_ERR_ARG, "displacement_to_mapping: null T or shapes differ");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t n = nvox(dis->dim);
        Staged a, o;
        a.in(dis->ptr, n * 12, dis->location, st, true);
        o.in(mapping->ptr, n * 12, mapping->location, st, false);
        REGB_CK(launch_displacement_to_mapping((const float*)a.d, Dim3{dis->dim[0], dis->dim[1], dis->dim[2]}, T,
                                               (float*)o.d, st));
        count_launch();
        o.out(mapping->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_inv_displacement_to_mapping(const regb_field* inv_dis, const float T[12], regb_field* inv_mapping,
                                             void* stream)
{
    return guarded([&] {
        check_field(inv_dis, "inv_dis");
        check_field(inv_mapping, "inv_mapping");
        if (!T)
            throw Failure(REGB_ERR_ARG, "inv_displacement_to_mapping: null T");
        float iT[12];
        std::memcpy(iT, T, sizeof(iT));
        if (!matrix_inverse(iT))
            return REGB_FALSE;
        cudaStream_t st = (cudaStream_t)stream;
        const size_t nd = nvox(inv_dis->dim), nm = nvox(inv_mapping->dim);
        Staged a, o;
        a.in(inv_dis->ptr, nd * 12, inv_dis->location, st, true);
        o.in(inv_mapping->ptr, nm * 12, inv_mapping->location, st, false);
        REGB_CK(launch_inv_displacement_to_mapping(
            (const float*)a.d, Dim3{inv_dis->dim[0], inv_dis->dim[1], inv_dis->dim[2]}, iT,
            Dim3{inv_mapping->dim[0], inv_mapping->dim[1], inv_mapping->dim[2]}, (float*)o.d, st));
        count_launch();
        o.out(inv_mapping->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_compose_mapping(const regb_volume* from, const regb_field* mapping, regb_volume* to, void* stream)
{
    return guarded([&] {
        check_vol(from, "from");
        check_field(mapping, "mapping");
        check_vol(to, "to");
        if (from->dtype != REGB_U8 || to->dtype != REGB_U8 || !same_dims(mapping->dim, to->dim))
            throw Failure(REGB_ERR_ARG, "compose_mapping: uint8 from/to, to shaped like the mapping");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t nf = nvox(from->dim), nm = nvox(mapping->dim);
        Staged a, m, o;
        a.in(from->ptr, nf, from->location, st, true);
        m.in(mapping->ptr, nm * 12, mapping->location, st, true);
        o.in(to->ptr, nm, to->location, st, false);
        REGB_CK(launch_compose_mapping_u8((const uint8_t*)a.d, Dim3{from->dim[0], from->dim[1], from->dim[2]},
                                          (const float*)m.d, Dim3{mapping->dim[0], mapping->dim[1], mapping->dim[2]},
                                          (uint8_t*)o.d, st));
        count_launch();
        o.out(to->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_match_fov(const regb_volume* It, const float T[12], const int moving_dim[3], regb_volume* out,
                           void* stream)
{
    return guarded([&] {
        check_vol(It, "It");
        check_vol(out, "out");
        if (!T || !moving_dim || It->dtype != REGB_U8 || out->dtype != REGB_U8 || !same_dims(It->dim, out->dim))
            throw Failure(REGB_ERR_ARG, "match_fov: uint8 It and out of one shape, T, moving_dim");
        check_dims(moving_dim, "moving_dim");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t n = nvox(It->dim);
        Staged a, o;
        a.in(It->ptr, n, It->location, st, true);
        o.in(out->ptr, n, out->location, st, false);
        REGB_CK(launch_match_fov_u8((const uint8_t*)a.d, Dim3{It->dim[0], It->dim[1], It->dim[2]}, T,
                                    Dim3{moving_dim[0], moving_dim[1], moving_dim[2]}, (uint8_t*)o.d, st));
        count_launch();
        o.out(out->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_correlation(const regb_volume* x, const regb_volume* y, int masked, double* r)
{
    return guarded([&] {
        check_vol(x, "x");
        check_vol(y, "y");
        if (!r || x->dtype != REGB_U8 || y->dtype != REGB_U8 || !same_dims(x->dim, y->dim))
            throw Failure(REGB_ERR_ARG, "correlation: two uint8 volumes of one shape");
        Stream s;
        const size_t n = nvox(x->dim);
        Staged a, b;
        a.in(x->ptr, n, x->location, s.s, true);
        b.in(y->ptr, n, y->location, s.s, true);
        *r = correlation_u8((const uint8_t*)a.d, (const uint8_t*)b.d, (long long)n, masked != 0, s.s);
        return REGB_OK;
    });
}

regb_status regb_accumulate_displacement(const regb_field* dis, regb_field* new_dis, void* stream)
{
    return guarded([&] {
        check_field(dis, "dis");
        check_field(new_dis, "new_dis");
        if (!same_dims(dis->dim, new_dis->dim))
            throw Failure(REGB_ERR_ARG, "accumulate: shapes differ");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t n = nvox(dis->dim);
        Staged a, b;
        a.in(dis->ptr, n * 12, dis->location, st, true);
        b.in(new_dis->ptr, n * 12, new_dis->location, st, true);
        DevBuf<float> out(3 * n, st);
        OneSeg s(dis->dim, st);
        s.h.cur_d = (float*)a.d;
        s.h.aux_d = (float*)b.d;
        s.h.tmp_d = out.p;
        s.c.scale = 1.0f;
        s.upload(st);
        REGB_CK(launch_cdm_accumulate(s.seg.p, 1, s.h.nblk, st));
        REGB_CK(cudaMemcpyAsync(b.d, out.p, n * 12, cudaMemcpyDeviceToDevice, st));
        b.out(new_dis->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_downsample(const regb_volume* in, regb_volume* out, void* stream)
{
    return guarded([&] {
        check_vol(in, "in");
        check_vol(out, "out");
        const int od[3] = {(in->dim[0] + 1) / 2, (in->dim[1] + 1) / 2, (in->dim[2] + 1) / 2};
        if (!same_dims(od, out->dim) || in->dtype != out->dtype)
            throw Failure(REGB_ERR_ARG, "downsample: out must be (d+1)/2 with the same dtype");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t ps = pix_size(in->dtype);
        Staged a, b;
        a.in(in->ptr, nvox(in->dim) * ps, in->location, st, true);
        b.in(out->ptr, nvox(out->dim) * ps, out->location, st, false);
        REGB_CK(launch_downsample(a.d, b.d, in->dim[0], in->dim[1], in->dim[2], pix_of(in->dtype), st));
        b.out(out->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_upsample_field_x2(const regb_field* in, regb_field* out, void* stream)
{
    return guarded([&] {
        check_field(in, "in");
        check_field(out, "out");
        cudaStream_t st = (cudaStream_t)stream;
        Staged a, b;
        a.in(in->ptr, nvox(in->dim) * 12, in->location, st, true);
        b.in(out->ptr, nvox(out->dim) * 12, out->location, st, false);
        REGB_CK(launch_upsample_field_x2((const float*)a.d, in->dim[0], in->dim[1], in->dim[2], (float*)b.d,
                                         out->dim[0], out->dim[1], out->dim[2], st));
        b.out(out->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_cdm_gradient(const regb_volume* Js, const regb_volume* It, regb_field* new_d, int gradient_type,
                              float* cost, void* stream)
{
    return guarded([&] {
        check_vol(Js, "Js");
        check_vol(It, "It");
        check_field(new_d, "new_d");
        if (!same_dims(Js->dim, It->dim) || !same_dims(Js->dim, new_d->dim) || Js->dtype != It->dtype)
            throw Failure(REGB_ERR_ARG, "gradient: shapes/dtypes differ");
        if (gradient_type != 'r' && gradient_type != 'd')
            throw Failure(REGB_ERR_ARG, "gradient_type must be 'r' or 'd'");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t n = nvox(Js->dim), ps = pix_size(Js->dtype);
        Staged a, b, o;
        a.in(Js->ptr, n * ps, Js->location, st, true);
        b.in(It->ptr, n * ps, It->location, st, true);
        o.in(new_d->ptr, n * 12, new_d->location, st, false);
        OneSeg s(Js->dim, st);
        s.h.Js = a.d;
        s.h.It[0] = b.d;
        s.h.new_d = (float*)o.d;
        s.upload(st);
        REGB_CK(launch_cdm_gradient(s.seg.p, 1, s.h.nblk, pix_of(Js->dtype), gradient_type, st));
        DevBuf<float> c(1, st);
        REGB_CK(launch_cost_mean(s.seg.p, 1, c.p, st));
        float hc = 0.0f;
        REGB_CK(cudaMemcpyAsync(&hc, c.p, 4, cudaMemcpyDeviceToHost, st));
        o.out(new_d->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        if (cost)
            *cost = hc;
        return REGB_OK;
    });
}

regb_status regb_cdm_poisson(regb_field* new_d, void* stream)
{
    return guarded([&] {
        check_field(new_d, "new_d");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t n = nvox(new_d->dim);
        Staged a;
        a.in(new_d->ptr, n * 12, new_d->location, st, true);
        DevBuf<float> A(3 * n, st), B(3 * n, st);
        OneSeg s(new_d->dim, st);
        s.h.new_d = (float*)a.d;
        s.h.aux_d = A.p;
        s.h.tmp_d = B.p;
        s.upload(st);
        REGB_CK(launch_cdm_poisson(s.seg.p, 1, s.h.nblk, 12, st));
        REGB_CK(cudaMemcpyAsync(a.d, A.p, n * 12, cudaMemcpyDeviceToDevice, st));
        a.out(new_d->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_cdm_max_length(const regb_field* d, float* out, void* stream)
{
    return guarded([&] {
        check_field(d, "d");
        if (!out)
            throw Failure(REGB_ERR_ARG, "null output");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t n = nvox(d->dim);
        Staged a;
        a.in(d->ptr, n * 12, d->location, st, true);
        OneSeg s(d->dim, st);
        s.h.aux_d = (float*)a.d;
        s.c.speed = 1.0f;
        s.upload(st);
        REGB_CK(launch_cdm_theta(s.seg.p, 1, s.h.nblk, st));
        CdmCtl c;
        REGB_CK(cudaMemcpyAsync(&c, s.ctl.p, sizeof(c), cudaMemcpyDeviceToHost, st));
        REGB_CK(cudaStreamSynchronize(st));
        *out = c.theta;
        return REGB_OK;
    });
}

regb_status regb_cdm_smooth(const regb_field* d, regb_field* dd, float smoothing, void* stream)
{
    return guarded([&] {
        check_field(d, "d");
        check_field(dd, "dd");
        if (!same_dims(d->dim, dd->dim))
            throw Failure(REGB_ERR_ARG, "smooth: shapes differ");
        cudaStream_t st = (cudaStream_t)stream;
        const size_t n = nvox(d->dim);
        Staged a, b;
        a.in(d->ptr, n * 12, d->location, st, true);
        b.in(dd->ptr, n * 12, dd->location, st, true);
        OneSeg s(d->dim, st);
        s.h.tmp_d = (float*)a.d;
        s.h.cur_d = (float*)b.d;
        s.c.cur_smoothing = smoothing;
        s.upload(st);
        REGB_CK(launch_cdm_smooth(s.seg.p, 1, s.h.nblk, st));
        b.out(dd->ptr, st);
        REGB_CK(cudaStreamSynchronize(st));
        return REGB_OK;
    });
}

regb_status regb_cdm_multi(const regb_volume* It, const regb_volume* Is, int nmod, regb_field* dis_out,
                           const regb_cdm_param* param, const char* gradient_types, volatile const int* terminated)
{
    return guarded([&] {
        if (!It || !Is || nmod < 1 || nmod > kCdmMaxModalities)
            throw Failure(REGB_ERR_ARG, "cdm: 1 to 12 modality pairs");
        check_field(dis_out, "dis_out");
        for (int m = 0; m < nmod; ++m) {
            check_vol(&It[m], "It");
            check_vol(&Is[m], "Is");
            if (!same_dims(It[m].dim, dis_out->dim) || !same_dims(Is[m].dim, dis_out->dim) ||
                It[m].dtype != It[0].dtype || Is[m].dtype != It[0].dtype)
                throw Failure(REGB_ERR_ARG, "cdm: It/Is/dis shapes or dtypes differ");
        }
        regb_cdm_param p;
        regb_cdm_param_default(&p);
        if (param)
            p = *param;
        const char one[2] = {(char)p.gradient_type, 0};
        const char* gtypes = gradient_types ? gradient_types : one;
        Stream s;
        const size_t n = nvox(It[0].dim), ps = pix_size(It[0].dtype);
        Staged a[kCdmMaxModalities], b[kCdmMaxModalities], f;
        const void* dt[kCdmMaxModalities];
        const void* ds[kCdmMaxModalities];
        for (int m = 0; m < nmod; ++m) {
            a[m].in(It[m].ptr, n * ps, It[m].location, s.s, true);
            b[m].in(Is[m].ptr, n * ps, Is[m].location, s.s, true);
            dt[m] = a[m].d;
            ds[m] = b[m].d;
        }
        f.in(dis_out->ptr, n * 12, dis_out->location, s.s, false);
        regb_status r = cdm_register_multi(dt, ds, nmod, gtypes, It[0].dim, pix_of(It[0].dtype), (float*)f.d, p,
                                           terminated, s.s);
        if (r == REGB_OK || r == REGB_CANCELLED)
            f.out(dis_out->ptr, s.s);
        s.sync();
        return r;
    });
}

regb_status regb_cdm2d_multi(const regb_volume* It, const regb_volume* Is, int nmod, regb_field* dis_out,
                             const regb_cdm_param* param, const char* gradient_types, volatile const int* terminated)
{
    return guarded([&] {
        if (!It || !Is || nmod < 1 || nmod > kCdmMaxModalities)
            throw Failure(REGB_ERR_ARG, "cdm2d: 1 to 12 modality pairs");
        check_field(dis_out, "dis_out");
        if (dis_out->dim[2] != 1)
            throw Failure(REGB_ERR_ARG, "cdm2d: 2-D images have dims (w, h, 1)");
        for (int m = 0; m < nmod; ++m) {
            check_vol(&It[m], "It");
            check_vol(&Is[m], "Is");
            if (!same_dims(It[m].dim, dis_out->dim) || !same_dims(Is[m].dim, dis_out->dim))
                throw Failure(REGB_ERR_ARG, "cdm2d: It/Is/dis shapes differ");
            if (It[m].dtype != REGB_U8 || Is[m].dtype != REGB_U8)
                throw Failure(REGB_ERR_ARG, "cdm2d takes uint8 images (cdm_cuda<out, unsigned char, 2>)");
        }
        regb_cdm_param p;
        regb_cdm_param_default(&p);
        if (param)
            p = *param;
        const char one[2] = {(char)p.gradient_type, 0};
        const char* gtypes = gradient_types ? gradient_types : one;
        Stream s;
        const size_t n = nvox(It[0].dim);
        Staged a[kCdmMaxModalities], b[kCdmMaxModalities], f;
        const void* dt[kCdmMaxModalities];
        const void* ds[kCdmMaxModalities];
        for (int m = 0; m < nmod; ++m) {
            a[m].in(It[m].ptr, n, It[m].location, s.s, true);
            b[m].in(Is[m].ptr, n, Is[m].location, s.s, true);
            dt[m] = a[m].d;
            ds[m] = b[m].d;
        }
        // the levels hold xyz fields whose z stays 0; the caller's field is x, y pairs
        DevBuf<float> xyz(3 * n, s.s);
        f.in(dis_out->ptr, n * 8, dis_out->location, s.s, false);
        regb_status r = cdm_register_multi(dt, ds, nmod, gtypes, It[0].dim, 0, xyz.p, p, terminated, s.s, nullptr,
                                           nullptr, 2);
        if (r == REGB_OK || r == REGB_CANCELLED) {
            REGB_CK(launch_field_xy(xyz.p, (long long)n, (float*)f.d, s.s));
            f.out(dis_out->ptr, s.s);
        }
        s.sync();
        return r;
    });
}

regb_status regb_cdm(const regb_volume* It, const regb_volume* Is, regb_field* dis_out, const regb_cdm_param* param,
                     volatile const int* terminated)
{
    return regb_cdm_multi(It, Is, 1, dis_out, param, nullptr, terminated);
}

regb_status regb_linear_multi(const regb_volume* from, const float from_vs[3], const regb_volume* to,
                              const float to_vs[3], int npairs, float arg[12], const regb_linear_param* param,
                              volatile const int* terminated, float* cost_out, long long* cost_evals)
{
    return guarded([&] {
        if (!from || !to || npairs < 1 || npairs > kMaxLinearPairs)
            throw Failure(REGB_ERR_ARG, "linear: 1 to 12 image pairs");
        for (int k = 0; k < npairs; ++k) {
            check_vol(&from[k], "from");
            check_vol(&to[k], "to");
            if (from[k].dtype != REGB_U8 || to[k].dtype != REGB_U8)
                throw Failure(REGB_ERR_ARG, "linear takes uint8 volumes (reg/linear.hpp:622-629)");
            if (!same_dims(from[k].dim, from[0].dim) || !same_dims(to[k].dim, to[0].dim))
                throw Failure(REGB_ERR_ARG, "linear: the pairs' from (to) volumes must share dims");
        }
        if (!from_vs || !to_vs || !arg)
            throw Failure(REGB_ERR_ARG, "null voxel size / arg");
        regb_linear_param p;
        regb_linear_param_default(&p);
        if (param)
            p = *param;
        if (p.cost_type != REGB_COST_MI && p.cost_type != REGB_COST_CORR && p.cost_type != REGB_COST_MI32)
            throw Failure(REGB_ERR_ARG, "cost_type must be MI, MI32 or CORR");
        Stream s;
        Staged a[kMaxLinearPairs], b[kMaxLinearPairs];
        const uint8_t* df[kMaxLinearPairs];
        const uint8_t* dt[kMaxLinearPairs];
        for (int k = 0; k < npairs; ++k) {
            a[k].in(from[k].ptr, nvox(from[k].dim), from[k].location, s.s, true);
            b[k].in(to[k].ptr, nvox(to[k].dim), to[k].location, s.s, true);
            df[k] = (const uint8_t*)a[k].d;
            dt[k] = (const uint8_t*)b[k].d;
        }
        LinearResult r = linear_register_multi(df, dt, npairs, from[0].dim, from_vs, to[0].dim, to_vs, arg, p,
                                               terminated, s.s);
        s.sync();
        if (cost_out)
            *cost_out = r.cost;
        if (cost_evals)
            *cost_evals = r.evals;
        return (terminated && *terminated) ? REGB_CANCELLED : REGB_OK;
    });
}

regb_status regb_linear(const regb_volume* from, const float from_vs[3], const regb_volume* to, const float to_vs[3],
                        float arg[12], const regb_linear_param* param, volatile const int* terminated,
                        float* cost_out, long long* cost_evals)
{
    return regb_linear_multi(from, from_vs, to, to_vs, 1, arg, param, terminated, cost_out, cost_evals);
}

regb_status regb_runner_state_from_param(const int from_dim[3], const float from_vs[3], const int to_dim[3],
                                         const float to_vs[3], const float arg[12], const regb_linear_param* param,
                                         regb_runner_state* out)
{
    return guarded([&] {
        if (!from_dim || !from_vs || !to_dim || !to_vs || !arg || !out)
            throw Failure(REGB_ERR_ARG, "null argument");
        regb_linear_param p;
        regb_linear_param_default(&p);
        if (param)
            p = *param;
        runner_state_from_param(from_dim, from_vs, to_dim, to_vs, arg, p, *out);
        return REGB_OK;
    });
}

regb_status regb_linear_run_multi(const regb_volume* from, const float from_vs[3], const regb_volume* to,
                                  const float to_vs[3], int npairs, float arg[12], const regb_runner_state* state,
                                  volatile const int* terminated, float* cost_out, long long* cost_evals)
{
    return guarded([&] {
        if (!from || !to || npairs < 1 || npairs > kMaxLinearPairs)
            throw Failure(REGB_ERR_ARG, "linear: 1 to 12 image pairs");
        for (int k = 0; k < npairs; ++k) {
            check_vol(&from[k], "from");
            check_vol(&to[k], "to");
            if (from[k].dtype != REGB_U8 || to[k].dtype != REGB_U8)
                throw Failure(REGB_ERR_ARG, "linear takes uint8 volumes (reg/linear.hpp:622-629)");
            if (!same_dims(from[k].dim, from[0].dim) || !same_dims(to[k].dim, to[0].dim))
                throw Failure(REGB_ERR_ARG, "linear: the pairs' from (to) volumes must share dims");
        }
        if (!from_vs || !to_vs || !arg || !state)
            throw Failure(REGB_ERR_ARG, "null voxel size / arg / state");
        if (state->cost_type != REGB_COST_MI && state->cost_type != REGB_COST_CORR && state->cost_type != REGB_COST_MI32)
            throw Failure(REGB_ERR_ARG, "cost_type must be MI, MI32 or CORR");
        Stream s;
        Staged a[kMaxLinearPairs], b[kMaxLinearPairs];
        const uint8_t* df[kMaxLinearPairs];
        const uint8_t* dt[kMaxLinearPairs];
        for (int k = 0; k < npairs; ++k) {
            a[k].in(from[k].ptr, nvox(from[k].dim), from[k].location, s.s, true);
            b[k].in(to[k].ptr, nvox(to[k].dim), to[k].location, s.s, true);
            df[k] = (const uint8_t*)a[k].d;
            dt[k] = (const uint8_t*)b[k].d;
        }
        LinearResult r = linear_register_state_multi(df, dt, npairs, from[0].dim, from_vs, to[0].dim, to_vs, arg,
                                                     *state, terminated, s.s);
        s.sync();
        if (cost_out)
            *cost_out = r.cost;
        if (cost_evals)
            *cost_evals = r.evals;
        return (terminated && *terminated) ? REGB_CANCELLED : REGB_OK;
    });
}

regb_status regb_linear_run(const regb_volume* from, const float from_vs[3], const regb_volume* to,
                            const float to_vs[3], float arg[12], const regb_runner_state* state,
                            volatile const int* terminated, float* cost_out, long long* cost_evals)
{
    return regb_linear_run_multi(from, from_vs, to, to_vs, 1, arg, state, terminated, cost_out, cost_evals);
}

}  // extern "C"
