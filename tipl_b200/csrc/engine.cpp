// Serving engine: registration jobs submitted as they arrive run concurrently on
// one GPU with continuous batching.
//
//   admission  -- a job starts when a slot is free and its estimated device memory
//                 fits the engine's HBM budget; others wait in arrival order;
//   affine     -- each running job drives its own optimiser (host threads); its
//                 probe sets go to the shared AffineBatcher, which evaluates the
//                 pending sets of all jobs in one launch;
//   nonlinear  -- each job's CDM levels are segments of the shared CdmScheduler,
//                 which iterates all of them in the same launches;
//   state      -- volumes, pyramids, fields and optimiser state stay on the device
//                 for the whole job; templates can be made resident once and shared.
// A job's result does not depend on what it ran alongside: every cost and every
// CDM decision is computed from that job's data alone (the tests check alone vs
// in the mix).
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include "batcher.h"
#include "host.h"
#include "kernels.h"
#include "preprocess.h"
#include "stats.h"
#include "scheduler.h"

using Clock = std::chrono::steady_clock;

namespace regb {

struct EngineTemplate {
    DevBuf<uint8_t> data;  // as given (U8, F32, U16 or BF16)
    DevBuf<uint8_t> u8;    // normalize_upper_lower2(data, 255.999) when data is not U8
    DevBuf<float> f32;     // data widened to float when it is U16 or BF16
    int dim[3];
    int dtype;
    float vs[3];
    const uint8_t* as_u8() const { return dtype == REGB_U8 ? data.p : u8.p; }
    const float* as_f32() const { return dtype == REGB_F32 ? (const float*)data.p : f32.p; }
};

// The affine stage quantises a volume that is not uint8 the way the reference's
// callers do before tipl::reg::linear: normalize_upper_lower2(v, 255.999)
// (numerical/numerical.hpp:909-927).
constexpr float kQuantUpper = 255.999f;

void to_u8(const void* d, int dtype, size_t n, DevBuf<uint8_t>& out, cudaStream_t st)
{
    DevBuf<unsigned> mm(2, st);
    out.alloc(n, st);
    REGB_CK(cudaMemsetAsync(out.p, 0, n, st));
    REGB_CK(launch_normalize_to_u8(d, dtype, (long long)n, kQuantUpper, out.p, mm.p, st));
    count_launch(2);
}

void to_f32(const void* d, int dtype, size_t n, DevBuf<float>& out, cudaStream_t st)
{
    out.alloc(n, st);
    REGB_CK(launch_widen_to_f32(d, dtype, (long long)n, out.p, st));
    count_launch();
}

struct EngineJob {
    uint64_t id = 0;
    regb_job spec{};
    regb_result res{};
    int state = 0;  // 0 queued, 1 running, 2 done
    size_t est = 0;
    volatile int cancel = 0;
    Clock::time_point t_submit, t_start, t_end;
};

class Engine {
public:
    explicit Engine(const regb_engine_config& c)
        : cfg_(c), batcher_(c.gather_us > 0 ? c.gather_us : 10, c.affine_workers > 0 ? c.affine_workers : 3), sched_(c.cdm_iters_per_round > 0 ? c.cdm_iters_per_round : 4)
    {
        REGB_CK(cudaGetDevice(&dev_));
        if (cfg_.max_active <= 0)
            cfg_.max_active = 64;
        if (cfg_.hbm_budget_bytes == 0) {
            size_t fr = 0, tot = 0;
            REGB_CK(cudaMemGetInfo(&fr, &tot));
            cfg_.hbm_budget_bytes = (size_t)(0.8 * (double)fr);
        }
    }
    ~Engine()
    {
        {
            std::unique_lock<std::mutex> lk(m_);
            for (auto& kv : jobs_)
                kv.second->cancel = 1;
            queue_.clear();
            cv_.wait(lk, [&] { return running_ == 0; });
        }
        templates_.clear();
        cudaStreamSynchronize(util_.s);
    }

    int add_template(const regb_volume& v, const float* vs)
    {
        auto t = std::make_unique<EngineTemplate>();
        const size_t n = (size_t)v.dim[0] * v.dim[1] * v.dim[2] * pix_size(v.dtype);
        // on the engine's own stream, which outlives every template buffer
        t->data.alloc(n, util_.s);
        REGB_CK(cudaMemcpyAsync(t->data.p, v.ptr, n, v.location == REGB_HOST ? cudaMemcpyHostToDevice
                                                                              : cudaMemcpyDeviceToDevice, util_.s));
        const size_t nv = (size_t)v.dim[0] * v.dim[1] * v.dim[2];
        if (v.dtype != REGB_U8)
            to_u8(t->data.p, v.dtype, nv, t->u8, util_.s);
        if (v.dtype == REGB_U16 || v.dtype == REGB_BF16)
            to_f32(t->data.p, v.dtype, nv, t->f32, util_.s);
        util_.sync();
        std::memcpy(t->dim, v.dim, sizeof(t->dim));
        t->dtype = v.dtype;
        std::memcpy(t->vs, vs, sizeof(t->vs));
        std::lock_guard<std::mutex> g(m_);
        templates_.push_back(std::move(t));
        return (int)templates_.size() - 1;
    }

    uint64_t submit(const regb_job& j)
    {
        auto job = std::make_unique<EngineJob>();
        job->spec = j;
        job->t_submit = Clock::now();
        std::lock_guard<std::mutex> g(m_);
        if (j.template_id >= (int)templates_.size())
            throw Failure(REGB_ERR_ARG, "unknown template id");
        job->est = estimate(j);
        if (job->est > cfg_.hbm_budget_bytes)
            throw Failure(REGB_ERR_BUDGET, "job needs more device memory than the engine's budget");
        job->id = next_id_++;
        EngineJob* p = job.get();
        jobs_[p->id] = std::move(job);
        queue_.push_back(p);
        admit_locked();
        return p->id;
    }

    regb_status poll(uint64_t id, regb_result* out, bool wait)
    {
        std::unique_lock<std::mutex> lk(m_);
        auto it = jobs_.find(id);
        if (it == jobs_.end())
            return REGB_ERR_NOTFOUND;
        EngineJob* j = it->second.get();
        if (wait)
            cv_.wait(lk, [&] { return j->state == 2; });
        if (j->state != 2)
            return REGB_PENDING;
        if (out)
            *out = j->res;
        return REGB_OK;
    }

    regb_status cancel(uint64_t id)
    {
        std::lock_guard<std::mutex> g(m_);
        auto it = jobs_.find(id);
        if (it == jobs_.end())
            return REGB_ERR_NOTFOUND;
        EngineJob* j = it->second.get();
        j->cancel = 1;
        if (j->state == 0) {  // still queued: finish it here
            for (auto q = queue_.begin(); q != queue_.end(); ++q)
                if (*q == j) {
                    queue_.erase(q);
                    break;
                }
            j->res.status = REGB_CANCELLED;
            j->state = 2;
            cv_.notify_all();
        }
        return REGB_OK;
    }

    void forget(uint64_t id)
    {
        std::lock_guard<std::mutex> g(m_);
        auto it = jobs_.find(id);
        if (it != jobs_.end() && it->second->state == 2)
            jobs_.erase(it);
    }

    regb_engine_stats stats()
    {
        std::lock_guard<std::mutex> g(m_);
        regb_engine_stats s{};
        s.queued = (int)queue_.size();
        s.running = running_;
        s.used_bytes = used_;
        s.budget_bytes = cfg_.hbm_budget_bytes;
        s.affine_launches = batcher_.launches();
        s.affine_tasks = batcher_.tasks_evaluated();
        s.cdm_rounds = sched_.rounds();
        s.cdm_round_segments = sched_.round_segments();
        s.cdm_round_ms = sched_.round_ms();
        s.cdm_max_round_segments = sched_.max_round_segments();
        return s;
    }

private:
    // Device memory a job holds while it runs (its own volumes and pyramids, the
    // affine-resampled subject and the CDM fields); the shared batch scratch and
    // resident templates are not counted.
    size_t estimate(const regb_job& j) const
    {
        const int* fd = (j.template_id >= 0) ? templates_.at(j.template_id)->dim : j.fixed.dim;
        const int ftype = (j.template_id >= 0) ? templates_.at(j.template_id)->dtype : j.fixed.dtype;
        const double nf = (double)fd[0] * fd[1] * fd[2];
        const double nm = (double)j.moving.dim[0] * j.moving.dim[1] * j.moving.dim[2];
        const double ps = (double)pix_size(ftype);
        double b = 0.0;
        if (j.template_id < 0)
            b += nf * ps;
        b += nm * (double)pix_size(j.moving.dtype);
        const bool float_cdm = !j.subject_pre && (ftype != REGB_U8 || j.moving.dtype != REGB_U8);
        if (j.moving.dtype != REGB_U8 || j.subject_pre)
            b += nm;                          // uint8 copy for the affine stage
        if (j.subject_pre)
            b += 12.0 * nm;                   // widened copy, smoothed copy, values above the threshold
        if (j.template_id < 0 && ftype != REGB_U8)
            b += nf;
        if (j.run_cdm && float_cdm)
            b += 4.0 * (nm + (j.template_id < 0 ? nf : 0.0));  // float copies for CDM
        if (j.run_linear)
            b += 0.15 * (nf + nm);
        if (j.run_cdm) {
            b += nf * (float_cdm ? 4.0 : ps) + 12.0 * nf;  // resampled subject, output field
            // the largest iterated level: 5 fields + composed image
            int w = fd[0], h = fd[1], d = fd[2];
            float res = j.cdm.resolution;
            double worst = 0.0;
            std::vector<double> lv;
            std::vector<float> lr;
            for (;;) {
                lv.push_back((double)w * h * d);
                lr.push_back(res);
                if (!((unsigned)std::min(w, std::min(h, d)) > j.cdm.min_dimension))
                    break;
                w = (w + 1) / 2;
                h = (h + 1) / 2;
                d = (d + 1) / 2;
                res /= 2.0f;
            }
            for (size_t k = 0; k < lv.size(); ++k)
                if (k + 1 == lv.size() || lr[k] <= 1.0f)
                    worst = std::max(worst, lv[k]);
            b += worst * (60.0 + ps) + 0.3 * nf * ps;
            if (j.mm_reg)  // the reverse CDM, the mappings, the composed subject
                b += worst * (60.0 + ps) + 0.3 * nf * ps + 12.0 * nf + 12.0 * nf + 12.0 * nm + 2.0 * nf;
        }
        return (size_t)b + (16u << 20);
    }

    void admit_locked()
    {
        while (!queue_.empty() && running_ < cfg_.max_active && used_ + queue_.front()->est <= cfg_.hbm_budget_bytes) {
            EngineJob* j = queue_.front();
            queue_.pop_front();
            j->state = 1;
            j->t_start = Clock::now();
            ++running_;
            used_ += j->est;
            std::thread([this, j] { run(j); }).detach();
        }
    }

    void run(EngineJob* j)
    {
        cudaSetDevice(dev_);
        regb_result r{};
        try {
            r = execute(j);
        } catch (const Failure& f) {
            r.status = f.code;
            set_last_error(f.what());
        } catch (const std::exception& e) {
            r.status = REGB_ERR_ARG;
            set_last_error(e.what());
        }
        std::lock_guard<std::mutex> g(m_);
        j->t_end = Clock::now();
        r.queued_ms = std::chrono::duration<double, std::milli>(j->t_start - j->t_submit).count();
        r.run_ms = std::chrono::duration<double, std::milli>(j->t_end - j->t_start).count();
        j->res = r;
        j->state = 2;
        --running_;
        used_ -= j->est;
        admit_locked();
        cv_.notify_all();
    }

    regb_result execute(EngineJob* j)
    {
        const regb_job& s = j->spec;
        regb_result r{};
        std::memcpy(r.arg, s.arg, sizeof(r.arg));
        Stream st;
        // fixed volume: resident template or the job's own
        const void* d_fixed;
        const uint8_t* fixed_u8 = nullptr;  // the affine stage's view
        const float* fixed_f32 = nullptr;   // the float CDM stage's view
        int fdim[3];
        int fdtype;
        float fvs[3];
        DevBuf<uint8_t> own_fixed, own_moving, fixed_q, moving_q;
        DevBuf<float> fixed_w, moving_w;
        if (s.template_id >= 0) {
            const EngineTemplate* t;
            {
                std::lock_guard<std::mutex> g(m_);
                t = templates_.at(s.template_id).get();
            }
            d_fixed = t->data.p;
            fixed_u8 = t->as_u8();
            fixed_f32 = t->as_f32();
            std::memcpy(fdim, t->dim, sizeof(fdim));
            fdtype = t->dtype;
            std::memcpy(fvs, t->vs, sizeof(fvs));
        } else {
            const size_t b = (size_t)s.fixed.dim[0] * s.fixed.dim[1] * s.fixed.dim[2] * pix_size(s.fixed.dtype);
            if (s.fixed.location == REGB_HOST) {
                own_fixed.alloc(b, st.s);
                REGB_CK(cudaMemcpyAsync(own_fixed.p, s.fixed.ptr, b, cudaMemcpyHostToDevice, st.s));
                d_fixed = own_fixed.p;
            } else
                d_fixed = s.fixed.ptr;
            std::memcpy(fdim, s.fixed.dim, sizeof(fdim));
            fdtype = s.fixed.dtype;
            std::memcpy(fvs, s.fixed_vs, sizeof(fvs));
        }
        const size_t nm = (size_t)s.moving.dim[0] * s.moving.dim[1] * s.moving.dim[2];
        const size_t nfx = (size_t)fdim[0] * fdim[1] * fdim[2];
        const size_t mb = nm * pix_size(s.moving.dtype);
        const void* d_moving = s.moving.ptr;
        if (s.moving.location == REGB_HOST) {
            own_moving.alloc(mb, st.s);
            REGB_CK(cudaMemcpyAsync(own_moving.p, s.moving.ptr, mb, cudaMemcpyHostToDevice, st.s));
            d_moving = own_moving.p;
        }
        if (s.template_id < 0) {
            if (fdtype == REGB_U8)
                fixed_u8 = (const uint8_t*)d_fixed;
            else if (s.run_linear) {
                to_u8(d_fixed, fdtype, nfx, fixed_q, st.s);
                fixed_u8 = fixed_q.p;
            }
        }
        const uint8_t* moving_u8 = (const uint8_t*)d_moving;
        if (s.subject_pre) {
            // the mm_reg pipeline: the subject through subject_image_pre, the template
            // through template_image_pre (its uint8 copy), both stages on uint8
            DevBuf<float> wide;
            const float* f = (const float*)d_moving;
            if (s.moving.dtype != REGB_F32) {
                to_f32(d_moving, s.moving.dtype, nm, wide, st.s);
                f = wide.p;
            }
            moving_q.alloc(nm, st.s);
            subject_image_pre(f, s.moving.dim, moving_q.p, st.s);
            moving_u8 = moving_q.p;
            if (!fixed_u8) {
                to_u8(d_fixed, fdtype, nfx, fixed_q, st.s);
                fixed_u8 = fixed_q.p;
            }
        } else if (s.moving.dtype != REGB_U8 && s.run_linear) {
            to_u8(d_moving, s.moving.dtype, nm, moving_q, st.s);
            moving_u8 = moving_q.p;
        }
        // CDM runs on uint8 when both volumes are uint8 or the subject was preprocessed
        // (the reference GPU path's type), otherwise in float on the volumes widened
        // exactly from their storage type
        const bool float_cdm = !s.subject_pre && (fdtype != REGB_U8 || s.moving.dtype != REGB_U8);
        const float* moving_f32 = nullptr;
        if (s.run_cdm && float_cdm) {
            if (!fixed_f32 || s.template_id < 0) {
                if (fdtype == REGB_F32)
                    fixed_f32 = (const float*)d_fixed;
                else {
                    to_f32(d_fixed, fdtype, nfx, fixed_w, st.s);
                    fixed_f32 = fixed_w.p;
                }
            }
            if (s.moving.dtype == REGB_F32)
                moving_f32 = (const float*)d_moving;
            else {
                to_f32(d_moving, s.moving.dtype, nm, moving_w, st.s);
                moving_f32 = moving_w.p;
            }
        }
        st.sync();
        r.status = REGB_OK;
        if (s.run_linear) {
            batcher_.add_client();
            LinearResult lr;
            try {
                lr = linear_register(fixed_u8, fdim, fvs, moving_u8, s.moving.dim, s.moving_vs, r.arg, s.linear,
                                     &j->cancel, st.s, &batcher_);
            } catch (...) {
                batcher_.remove_client();
                throw;
            }
            batcher_.remove_client();
            r.linear_cost = lr.cost;
            r.cost_evals = lr.evals;
        }
        if (j->cancel) {
            r.status = REGB_CANCELLED;
            return r;
        }
        if (s.run_cdm) {
            // the subject resampled onto the template grid with the affine found
            // (the mm_reg pipeline, reg/mm_reg.hpp:379-416)
            const int pix = float_cdm ? 1 : 0;
            const size_t nf = nfx;
            DevBuf<uint8_t> Is(nf * (pix ? 4 : 1), st.s);
            float T[12];
            affine_to_matrix(r.arg, fdim, fvs, s.moving.dim, s.moving_vs, T);
            int shift[3];
            const int* sh = integer_shift(T, shift) ? shift : nullptr;
            const Dim3 md{s.moving.dim[0], s.moving.dim[1], s.moving.dim[2]}, fdd{fdim[0], fdim[1], fdim[2]};
            if (pix)
                REGB_CK(launch_resample<float>(moving_f32, md, (float*)Is.p, fdd, T, sh, st.s));
            else
                REGB_CK(launch_resample<uint8_t>(s.subject_pre ? moving_u8 : (const uint8_t*)d_moving, md, Is.p, fdd,
                                                 T, sh, st.s));
            DevBuf<float> field(3 * nf, st.s);
            int iters = 0;
            const void* It = pix ? (const void*)fixed_f32 : (s.subject_pre ? (const void*)fixed_u8 : d_fixed);
            const uint8_t* I8 = s.subject_pre ? moving_u8 : (const uint8_t*)d_moving;  // uint8 subject (pix 0)
            const bool mm = s.mm_reg && !pix;
            // mm_reg: linear r (calculate_linear_r, reg/mm_reg.hpp:286-311, masked_r), and the
            // reverse CDM -- cdm_common(J, It) beside cdm_common(It, J), reg/mm_reg.hpp:392-407
            DevBuf<float> field_rev;
            std::thread rev;
            regb_status cs_rev = REGB_FALSE;
            int iters_rev = 0;
            std::exception_ptr rev_err;
            DevBuf<uint8_t> It_fov;
            if (mm) {
                r.r_linear = correlation_u8(Is.p, (const uint8_t*)It, (long long)nf, true, st.s);
                // It_match_fov (match_fov is on by default, reg/mm_reg.hpp:309-310): the
                // template outside the subject's field of view is 0 for the nonlinear stage
                It_fov.alloc(nf, st.s);
                REGB_CK(launch_match_fov_u8((const uint8_t*)It, fdd, T, md, It_fov.p, st.s));
                count_launch();
                It = It_fov.p;
                field_rev.alloc(3 * nf, st.s);
                st.sync();  // Is and field_rev are ready before the reverse stream uses them
                rev = std::thread([&] {
                    try {
                        Stream st2;
                        cs_rev = cdm_register(Is.p, It, fdim, 0, field_rev.p, s.cdm, &j->cancel, st2.s, &iters_rev,
                                              &sched_);
                        st2.sync();
                    } catch (...) {
                        rev_err = std::current_exception();
                    }
                });
            }
            regb_status cs = REGB_FALSE;
            std::exception_ptr fwd_err;
            try {
                cs = cdm_register(It, Is.p, fdim, pix, field.p, s.cdm, &j->cancel, st.s, &iters, &sched_);
            } catch (...) {
                fwd_err = std::current_exception();
            }
            if (rev.joinable())
                rev.join();
            if (fwd_err)
                std::rethrow_exception(fwd_err);
            if (rev_err)
                std::rethrow_exception(rev_err);
            r.cdm_ok = (cs == REGB_OK) ? 1 : 0;
            r.cdm_iterations = iters;
            if (cs == REGB_CANCELLED || cs_rev == REGB_CANCELLED)
                r.status = REGB_CANCELLED;
            const cudaMemcpyKind kind =
                s.field_location == REGB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
            if (mm && r.status != REGB_CANCELLED && s.prev_field && s.prev_field_rev) {
                // continue an earlier registration (reg/mm_reg.hpp:408-412): the new
                // fields are accumulated onto the previous ones
                const cudaMemcpyKind in_kind =
                    s.field_location == REGB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
                DevBuf<float> prev(3 * nf, st.s), prev_rev(3 * nf, st.s);
                REGB_CK(cudaMemcpyAsync(prev.p, s.prev_field, sizeof(float) * 3 * nf, in_kind, st.s));
                REGB_CK(cudaMemcpyAsync(prev_rev.p, s.prev_field_rev, sizeof(float) * 3 * nf, in_kind, st.s));
                accumulate_displacement_device(prev.p, field.p, fdim, st.s);
                accumulate_displacement_device(prev_rev.p, field_rev.p, fdim, st.s);
                count_launch(2);
            }
            if (s.field_out && cs != REGB_FALSE)
                REGB_CK(cudaMemcpyAsync(s.field_out, field.p, sizeof(float) * 3 * nf, kind, st.s));
            if (mm && r.status != REGB_CANCELLED) {
                r.cdm_rev_ok = (cs_rev == REGB_OK) ? 1 : 0;
                // compute_mapping_from_displacement (reg/mm_reg.hpp:271-284)
                DevBuf<float> to2from(3 * nf, st.s), from2to(3 * nm, st.s);
                REGB_CK(launch_displacement_to_mapping(field.p, fdd, T, to2from.p, st.s));
                float iT[12];
                std::memcpy(iT, T, sizeof(iT));
                const bool inv_ok = matrix_inverse(iT);
                if (inv_ok)
                    REGB_CK(launch_inv_displacement_to_mapping(field_rev.p, fdd, iT, md, from2to.p, st.s));
                count_launch(inv_ok ? 2 : 1);
                // calculate_nonlinear_r (reg/mm_reg.hpp:330-345): the subject through the mapping
                DevBuf<uint8_t> J2(nf, st.s);
                REGB_CK(launch_compose_mapping_u8(I8, md, to2from.p, fdd, J2.p, st.s));
                count_launch();
                r.r_nonlinear = correlation_u8(J2.p, (const uint8_t*)It, (long long)nf, true, st.s);
                if (s.field_rev_out && cs_rev != REGB_FALSE)
                    REGB_CK(cudaMemcpyAsync(s.field_rev_out, field_rev.p, sizeof(float) * 3 * nf, kind, st.s));
                if (s.mapping_out)
                    REGB_CK(cudaMemcpyAsync(s.mapping_out, to2from.p, sizeof(float) * 3 * nf, kind, st.s));
                if (s.inv_mapping_out && inv_ok)
                    REGB_CK(cudaMemcpyAsync(s.inv_mapping_out, from2to.p, sizeof(float) * 3 * nm, kind, st.s));
            }
            st.sync();
        }
        return r;
    }

    regb_engine_config cfg_;
    int dev_ = 0;
    AffineBatcher batcher_;
    CdmScheduler sched_;
    std::mutex m_;
    std::condition_variable cv_;
    Stream util_;  // declared before templates_: destroyed after their buffers are freed on it
    std::vector<std::unique_ptr<EngineTemplate>> templates_;
    std::map<uint64_t, std::unique_ptr<EngineJob>> jobs_;
    std::deque<EngineJob*> queue_;
    int running_ = 0;
    size_t used_ = 0;
    uint64_t next_id_ = 1;
};

}  // namespace regb

using namespace regb;

struct regb_engine {
    std::unique_ptr<Engine> e;
};

namespace {
template <typename F>
regb_status eguard(F&& f)
{
    try {
        return f();
    } catch (const Failure& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return REGB_ERR_ARG;
    }
}

bool vol_ok(const regb_volume& v)
{
    return v.ptr && v.dim[0] > 0 && v.dim[1] > 0 && v.dim[2] > 0 &&
           (long long)v.dim[0] * v.dim[1] * v.dim[2] < (1LL << 31) && pix_size(v.dtype) &&
           (v.location == REGB_HOST || v.location == REGB_DEVICE);
}
}  // namespace

extern "C" {

void regb_engine_config_default(regb_engine_config* c)
{
    if (!c)
        return;
    c->hbm_budget_bytes = 0;
    c->max_active = 64;
    c->gather_us = 10;
    c->cdm_iters_per_round = 4;
    c->affine_workers = 3;
}

void regb_job_default(regb_job* j)
{
    if (!j)
        return;
    std::memset(j, 0, sizeof(*j));
    j->template_id = -1;
    j->fixed_vs[0] = j->fixed_vs[1] = j->fixed_vs[2] = 1.0f;
    j->moving_vs[0] = j->moving_vs[1] = j->moving_vs[2] = 1.0f;
    j->run_linear = 1;
    regb_linear_param_default(&j->linear);
    regb_cdm_param_default(&j->cdm);
    j->arg[6] = j->arg[7] = j->arg[8] = 1.0f;
    j->field_location = REGB_HOST;
    j->subject_pre = 0;
    j->mm_reg = 0;
}

regb_status regb_engine_create(const regb_engine_config* cfg, regb_engine** out)
{
    return eguard([&] {
        if (!out)
            throw Failure(REGB_ERR_ARG, "null output");
        regb_engine_config c;
        regb_engine_config_default(&c);
        if (cfg)
            c = *cfg;
        ensure_device();
        auto* e = new regb_engine;
        e->e = std::make_unique<Engine>(c);
        *out = e;
        return REGB_OK;
    });
}

regb_status regb_engine_destroy(regb_engine* e)
{
    return eguard([&] {
        delete e;
        return REGB_OK;
    });
}

regb_status regb_engine_add_template(regb_engine* e, const regb_volume* vol, const float vs[3], int* template_id)
{
    return eguard([&] {
        if (!e || !vol || !vs || !template_id || !vol_ok(*vol))
            throw Failure(REGB_ERR_ARG, "bad template arguments");
        *template_id = e->e->add_template(*vol, vs);
        return REGB_OK;
    });
}

regb_status regb_engine_submit(regb_engine* e, const regb_job* job, uint64_t* id)
{
    return eguard([&] {
        if (!e || !job || !id)
            throw Failure(REGB_ERR_ARG, "null argument");
        if (!vol_ok(job->moving) || (job->template_id < 0 && !vol_ok(job->fixed)))
            throw Failure(REGB_ERR_ARG, "bad fixed/moving volume");
        if (job->mm_reg && !job->run_cdm)
            throw Failure(REGB_ERR_ARG, "mm_reg needs run_cdm");
        if ((job->prev_field || job->prev_field_rev) && !(job->mm_reg && job->prev_field && job->prev_field_rev))
            throw Failure(REGB_ERR_ARG, "prev_field and prev_field_rev go together, with mm_reg");
        const int ct = job->linear.cost_type;
        if (job->run_linear && ct != REGB_COST_CORR && ct != REGB_COST_MI && ct != REGB_COST_MI32)
            throw Failure(REGB_ERR_ARG, "cost_type must be MI, MI32 or CORR");
        *id = e->e->submit(*job);
        return REGB_OK;
    });
}

regb_status regb_engine_poll(regb_engine* e, uint64_t id, regb_result* out)
{
    return eguard([&] { return e ? e->e->poll(id, out, false) : REGB_ERR_ARG; });
}

regb_status regb_engine_wait(regb_engine* e, uint64_t id, regb_result* out)
{
    return eguard([&] { return e ? e->e->poll(id, out, true) : REGB_ERR_ARG; });
}

regb_status regb_engine_cancel(regb_engine* e, uint64_t id)
{
    return eguard([&] { return e ? e->e->cancel(id) : REGB_ERR_ARG; });
}

regb_status regb_engine_release_job(regb_engine* e, uint64_t id)
{
    return eguard([&] {
        if (!e)
            return REGB_ERR_ARG;
        e->e->forget(id);
        return REGB_OK;
    });
}

regb_status regb_engine_get_stats(regb_engine* e, regb_engine_stats* out)
{
    return eguard([&] {
        if (!e || !out)
            return REGB_ERR_ARG;
        *out = e->e->stats();
        return REGB_OK;
    });
}

}  // extern "C"
