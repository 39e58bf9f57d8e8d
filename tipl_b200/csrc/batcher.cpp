#include "batcher.h"
#include <chrono>
#include <cstring>

namespace regb {

AffineBatcher::AffineBatcher(int gather_us) : gather_us_(gather_us)
{
    REGB_CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    int dev = 0;
    REGB_CK(cudaGetDevice(&dev));
    th_ = std::thread([this, dev] {
        cudaSetDevice(dev);
        loop();
    });
}

AffineBatcher::~AffineBatcher()
{
    {
        std::lock_guard<std::mutex> g(m_);
        stop_ = true;
    }
    cv_req_.notify_all();
    if (th_.joinable())
        th_.join();
    for (TaskScratch& s : scratch_)
        s.release();
    if (st_) {
        cudaStreamSynchronize(st_);
        cudaStreamDestroy(st_);
    }
}

void AffineBatcher::add_client()
{
    std::lock_guard<std::mutex> g(m_);
    ++clients_;
}

void AffineBatcher::remove_client()
{
    {
        std::lock_guard<std::mutex> g(m_);
        --clients_;
    }
    cv_req_.notify_all();
}

void AffineBatcher::eval(const AffineTask* tasks, int n, int cost_type, double* out)
{
    if (n == 0)
        return;
    if (cost_type < 0 || cost_type >= kCostTypes)
        throw Failure(REGB_ERR_ARG, "unknown cost type");
    Req r{tasks, n, cost_type, out};
    std::unique_lock<std::mutex> lk(m_);
    pending_.push_back(&r);
    cv_req_.notify_all();
    cv_done_.wait(lk, [&] { return r.done; });
    if (r.err)
        std::rethrow_exception(r.err);
}

void AffineBatcher::loop()
{
    std::unique_lock<std::mutex> lk(m_);
    for (;;) {
        cv_req_.wait(lk, [&] { return stop_ || !pending_.empty(); });
        if (stop_ && pending_.empty())
            return;
        // the device is free: give the other jobs a moment to join this batch
        const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(gather_us_);
        cv_req_.wait_until(lk, until, [&] { return stop_ || (int)pending_.size() >= clients_; });
        std::vector<Req*> batch(pending_.begin(), pending_.end());
        pending_.clear();
        lk.unlock();
        for (int ct = 0; ct < kCostTypes; ++ct) {
            int total = 0;
            for (Req* r : batch)
                if (r->cost_type == ct)
                    total += r->n;
            if (!total)
                continue;
            try {
                TaskScratch& s = scratch_[ct];
                s.ensure(total, ct != REGB_COST_CORR, st_);
                int k = 0;
                for (Req* r : batch)
                    if (r->cost_type == ct) {
                        std::memcpy(s.h_tasks.p + k, r->tasks, sizeof(AffineTask) * r->n);
                        k += r->n;
                    }
                std::vector<double> c(total);
                run_affine_tasks(s, total, ct, st_, c.data());
                k = 0;
                for (Req* r : batch)
                    if (r->cost_type == ct) {
                        std::memcpy(r->out, c.data() + k, sizeof(double) * r->n);
                        k += r->n;
                    }
                ++launches_;
                tasks_ += total;
            } catch (...) {
                for (Req* r : batch)
                    if (r->cost_type == ct)
                        r->err = std::current_exception();
            }
        }
        lk.lock();
        for (Req* r : batch)
            r->done = true;
        cv_done_.notify_all();
    }
}

}  // namespace regb
