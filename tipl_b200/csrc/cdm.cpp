// CDM nonlinear registration driver (reg/cdm.hpp:373-474, cdm_common 534-558) on
// device-resident images of one job.
//
// Pyramid: levels are built by downsample_with_padding while min(shape) >
// min_dimension (reg/cdm.hpp:382-392).  The coarsest level always iterates; a
// finer level starts from the doubled, upsampled field of the level below and
// iterates only when its resolution (param.resolution halved per level) is at
// most 1 (reg/cdm.hpp:400-405).
//
// Each iteration is the kernel sequence of cdm_kernels.cu; the loop decisions run
// on the device (CdmCtl).  This single-job driver replays the iterations through
// a CUDA graph and reads the done flag back once per graph launch.
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <string>
#include <vector>
#include "cdm_level.h"
#include "host.h"
#include "scheduler.h"
#include "stats.h"

namespace regb {

void GraphExec::capture(const std::function<void(cudaStream_t)>& body)
{
    reset();
    cudaStream_t cs;
    REGB_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    const long long before = g_launches.load();
    if (e == cudaSuccess) {
        try {
            body(cs);
        } catch (...) {
            cudaStreamEndCapture(cs, &graph);
            if (graph)
                cudaGraphDestroy(graph);
            cudaStreamDestroy(cs);
            throw;
        }
        e = cudaStreamEndCapture(cs, &graph);
    }
    // captured launches are counted when the graph runs, once per replay
    nodes = g_launches.load() - before;
    g_launches.fetch_sub(nodes);
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph)
        cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess)
        throw_cuda(e, "graph capture");
}

void GraphExec::launch(cudaStream_t st)
{
    REGB_CK(cudaGraphLaunch(exec, st));
    count_launch(nodes);
}

void GraphExec::reset()
{
    if (exec)
        cudaGraphExecDestroy(exec);
    exec = nullptr;
}

void CdmLevel::init(const void* const* It_, const void* const* Is_, const std::string& gtypes_, int w, int h, int d,
                    int pix_, const regb_cdm_param& p, float* best, cudaStream_t st, int ndim)
{
    pix = pix_;
    gtypes = gtypes_;
    seg = CdmSeg{};
    seg.w = w;
    seg.h = h;
    seg.d = d;
    const long long n = (long long)w * h * d;
    seg.nblk = cdm_blocks_for(n);
    seg.nmod = (int)gtypes.size();
    seg.ndim = ndim;
    for (int m = 0; m < seg.nmod; ++m) {
        seg.It[m] = It_[m];
        seg.Is[m] = Is_[m];
    }
    js.alloc((size_t)n * (pix ? 4 : 1), st);
    cur.alloc(3 * n, st);
    nd.alloc(3 * n, st);
    aux.alloc(3 * n, st);
    tmp.alloc(3 * n, st);
    part.alloc(seg.nblk, st);
    ctl.alloc(1, st);
    seg.Js = js.p;
    seg.cur_d = cur.p;
    seg.best_d = best;
    seg.new_d = nd.p;
    seg.aux_d = aux.p;
    seg.tmp_d = tmp.p;
    seg.cost_part = part.p;
    seg.ctl = ctl.p;
    CdmCtl c;
    std::memset(&c, 0, sizeof(c));
    c.best_cost = FLT_MAX;
    c.cur_smoothing = 0.8f;
    c.speed = p.speed;
    c.smoothing = p.smoothing;
    c.max_iter = 200;
    h_ctl = c;
    REGB_CK(cudaMemcpyAsync(ctl.p, &h_ctl, sizeof(CdmCtl), cudaMemcpyHostToDevice, st));
    REGB_CK(cudaMemcpyAsync(cur.p, best, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, st));  // cur_d(best_d)
    d_seg.alloc(1, st);
    REGB_CK(cudaMemcpyAsync(d_seg.p, &seg, sizeof(CdmSeg), cudaMemcpyHostToDevice, st));
    REGB_CK(cudaStreamSynchronize(st));  // h_ctl / seg are stack-staged: keep the copies ordered before reuse
}

void launch_iteration(const CdmSeg* d_segs, int nseg, int blocks, int pix, const std::string& gtypes,
                      cudaStream_t st)
{
    // compose and differentiate each modality in turn (reg/cdm.hpp:422-434); the
    // last gradient launch also makes the loop decisions
    for (int m = 0; m < (int)gtypes.size(); ++m) {
        REGB_CK(launch_cdm_compose(d_segs, nseg, blocks, pix, st, m));
        REGB_CK(launch_cdm_gradient(d_segs, nseg, blocks, pix, gtypes[m], st, m));
    }
    REGB_CK(launch_cdm_poisson(d_segs, nseg, blocks, 12, st));                    // + best_d copy, theta
    REGB_CK(launch_cdm_accumulate(d_segs, nseg, blocks, st));
    REGB_CK(launch_cdm_smooth(d_segs, nseg, blocks, st));
}

void accumulate_displacement_device(const float* dis, float* new_dis, const int* dim, cudaStream_t st)
{
    // the accumulate pass of a CDM iteration with speed / theta = 1 (an exact scaling)
    const long long n = (long long)dim[0] * dim[1] * dim[2];
    CdmSeg seg{};
    seg.w = dim[0];
    seg.h = dim[1];
    seg.d = dim[2];
    seg.nblk = cdm_blocks_for(n);
    CdmCtl c;
    std::memset(&c, 0, sizeof(c));
    c.scale = 1.0f;
    c.max_iter = 200;
    DevBuf<float> out(3 * n, st);
    DevBuf<CdmCtl> ctl(1, st);
    DevBuf<CdmSeg> d_seg(1, st);
    seg.cur_d = const_cast<float*>(dis);
    seg.aux_d = new_dis;
    seg.tmp_d = out.p;
    seg.ctl = ctl.p;
    REGB_CK(cudaMemcpyAsync(ctl.p, &c, sizeof(c), cudaMemcpyHostToDevice, st));
    REGB_CK(cudaMemcpyAsync(d_seg.p, &seg, sizeof(seg), cudaMemcpyHostToDevice, st));
    REGB_CK(launch_cdm_accumulate(d_seg.p, 1, seg.nblk, st));
    REGB_CK(cudaMemcpyAsync(new_dis, out.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, st));
    REGB_CK(cudaStreamSynchronize(st));  // c and seg are stack-staged
}

regb_status cdm_register(const void* d_It, const void* d_Is, const int* dim, int pix, float* d_field,
                         const regb_cdm_param& p, volatile const int* terminated, cudaStream_t st, int* iterations,
                         CdmScheduler* sched)
{
    const char gt[2] = {(char)p.gradient_type, 0};
    return cdm_register_multi(&d_It, &d_Is, 1, gt, dim, pix, d_field, p, terminated, st, iterations, sched);
}

regb_status cdm_register_multi(const void* const* d_It, const void* const* d_Is, int nmod, const char* gtypes_in,
                               const int* dim, int pix, float* d_field, const regb_cdm_param& p,
                               volatile const int* terminated, cudaStream_t st, int* iterations, CdmScheduler* sched,
                               int ndim)
{
    if (nmod < 1 || nmod > kCdmMaxModalities)
        throw Failure(REGB_ERR_ARG, "cdm: 1 to 12 modality pairs");
    if (ndim == 2 && dim[2] != 1)
        throw Failure(REGB_ERR_ARG, "cdm: a 2-D registration takes images of depth 1");
    // cdm_param::gradient_type: modality i takes its i-th char, 'r' past the end
    std::string gtypes(nmod, 'r');
    const size_t ntype = gtypes_in ? std::strlen(gtypes_in) : 0;
    for (int m = 0; m < nmod && (size_t)m < ntype; ++m)
        gtypes[m] = gtypes_in[m];
    for (char c : gtypes)
        if (c != 'r' && c != 'd')
            throw Failure(REGB_ERR_ARG, "gradient types must be 'r' or 'd'");
    const size_t psz = pix ? 4 : 1;
    struct Lv {
        int w, h, d;
        const void* It[kCdmMaxModalities];
        const void* Is[kCdmMaxModalities];
        DevBuf<uint8_t> bt[kCdmMaxModalities], bs[kCdmMaxModalities];
        DevBuf<float> best;
        float resolution;
    };
    std::vector<Lv> lv;
    lv.emplace_back();
    lv[0].w = dim[0];
    lv[0].h = dim[1];
    lv[0].d = dim[2];
    for (int m = 0; m < nmod; ++m) {
        lv[0].It[m] = d_It[m];
        lv[0].Is[m] = d_Is[m];
    }
    lv[0].resolution = p.resolution;
    for (;;) {
        Lv& c = lv.back();
        // min_value(It[0].shape()) over the image's own dimensions (reg/cdm.hpp:382)
        const int mn = ndim == 2 ? std::min(c.w, c.h) : std::min(c.w, std::min(c.h, c.d));
        if (!((unsigned int)mn > p.min_dimension))
            break;
        Lv n;
        n.w = (c.w + 1) / 2;
        n.h = (c.h + 1) / 2;
        n.d = (c.d + 1) / 2;
        if (n.w == c.w && n.h == c.h && n.d == c.d)
            // only min_dimension 0 gets here (an axis of 1 voxel passes "min > 0" forever);
            // the reference recurses without end and overflows its stack
            throw Failure(REGB_ERR_ARG, "cdm: min_dimension 0 with a one-voxel axis never stops downsampling");
        n.resolution = c.resolution / 2.0f;
        const size_t nn = (size_t)n.w * n.h * n.d;
        for (int m = 0; m < nmod; ++m) {
            n.bt[m].alloc(nn * psz, st);
            n.bs[m].alloc(nn * psz, st);
            REGB_CK(launch_downsample(c.It[m], n.bt[m].p, c.w, c.h, c.d, pix, st));
            REGB_CK(launch_downsample(c.Is[m], n.bs[m].p, c.w, c.h, c.d, pix, st));
            n.It[m] = n.bt[m].p;
            n.Is[m] = n.bs[m].p;
        }
        lv.push_back(std::move(n));
    }
    const int top = (int)lv.size() - 1;
    int iters = 0;
    regb_status status = REGB_OK;
    for (int k = top; k >= 0; --k) {
        Lv& L = lv[k];
        const size_t n = (size_t)L.w * L.h * L.d;
        float* best = d_field;
        if (k > 0) {
            L.best.alloc(3 * n, st);
            best = L.best.p;
        }
        if (k == top)
            REGB_CK(cudaMemsetAsync(best, 0, sizeof(float) * 3 * n, st));
        else {
            const Lv& C = lv[k + 1];
            const float* cb = C.best.p;
            REGB_CK(launch_upsample_field_x2(cb, C.w, C.h, C.d, best, L.w, L.h, L.d, st, ndim));
            if (L.resolution > 1.0f)
                continue;  // reg/cdm.hpp:404-405
        }
        if (status != REGB_OK)
            continue;
        CdmLevel run;
        run.init(L.It, L.Is, gtypes, L.w, L.h, L.d, pix, p, best, st, ndim);
        if (sched) {
            // batched with the other jobs' levels; the scheduler returns once this
            // level's loop has ended
            sched->run(run, terminated);
            REGB_CK(cudaMemcpyAsync(&run.h_ctl, run.ctl.p, sizeof(CdmCtl), cudaMemcpyDeviceToHost, st));
            REGB_CK(cudaStreamSynchronize(st));
            if (terminated && *terminated && !run.h_ctl.done)
                status = REGB_CANCELLED;
        }
        if (!sched) {
            // kIters iterations per graph launch; the loop decisions live on the
            // device, so iterations launched after the loop has ended are no-ops
            constexpr int kIters = 4;
            GraphExec g;
            g.capture([&](cudaStream_t cs) {
                for (int k = 0; k < kIters; ++k)
                    launch_iteration(run.d_seg.p, 1, run.seg.nblk, pix, gtypes, cs);
            });
            for (int it = 0; it < 201; it += kIters) {
                if (terminated && *terminated) {
                    status = REGB_CANCELLED;
                    break;
                }
                g.launch(st);
                REGB_CK(cudaMemcpyAsync(&run.h_ctl, run.ctl.p, sizeof(CdmCtl), cudaMemcpyDeviceToHost, st));
                REGB_CK(cudaStreamSynchronize(st));
                if (run.h_ctl.done)
                    break;
            }
        }
        iters += run.h_ctl.iters_run;
        count_cdm_level(run.h_ctl.iters_run, (long long)n, pix ? 4 : 1);
        if (run.h_ctl.done == 2)
            return REGB_FALSE;  // reg/cdm.hpp:428-429: a zero cost sum fails the whole call
    }
    REGB_CK(cudaStreamSynchronize(st));
    if (iterations)
        *iterations = iters;
    return status;
}

}  // namespace regb
