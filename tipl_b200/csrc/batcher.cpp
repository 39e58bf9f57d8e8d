#include "batcher.h"
#include <chrono>
#include <algorithm>
#include <cstring>

namespace regb {

AffineBatcher::AffineBatcher(int gather_us, int workers)
    : nworkers_(std::min(std::max(workers, 1), kMaxWorkers)), gather_us_(gather_us)
{
    int dev = 0;
    REGB_CK(cudaGetDevice(&dev));
    for (int i = 0; i < nworkers_; ++i)
        REGB_CK(cudaStreamCreateWithFlags(&workers_[i].st, cudaStreamNonBlocking));
    for (int i = 0; i < nworkers_; ++i) {
        Worker& w = workers_[i];
        w.th = std::thread([this, dev, &w] {
            cudaSetDevice(dev);
            loop(w);
        });
    }
}

AffineBatcher::~AffineBatcher()
{
    {
        std::lock_guard<std::mutex> g(m_);
        stop_ = true;
    }
    cv_req_.notify_all();
    for (Worker& w : workers_)
        if (w.th.joinable())
            w.th.join();
    for (Worker& w : workers_) {
        for (TaskScratch& s : w.scratch)
            s.release();
        if (w.st) {
            cudaStreamSynchronize(w.st);
            cudaStreamDestroy(w.st);
        }
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

void AffineBatcher::loop(Worker& w)
{
    std::unique_lock<std::mutex> lk(m_);
    for (;;) {
        cv_req_.wait(lk, [&] { return stop_ || !pending_.empty(); });
        if (stop_ && pending_.empty())
            return;
        // give the jobs that could still submit (those not waiting on the other
        // worker's batch) a moment to join this one
        const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(gather_us_);
        cv_req_.wait_until(lk, until,
                           [&] { return stop_ || (int)pending_.size() >= clients_ - inflight_; });
        if (pending_.empty())
            continue;  // the other worker took them
        std::vector<Req*> batch(pending_.begin(), pending_.end());
        pending_.clear();
        inflight_ += (int)batch.size();
        lk.unlock();
        for (int ct = 0; ct < kCostTypes; ++ct) {
            int total = 0;
            for (Req* r : batch)
                if (r->cost_type == ct)
                    total += r->n;
            if (!total)
                continue;
            try {
                TaskScratch& s = w.scratch[ct];
                s.ensure(total, ct != REGB_COST_CORR, w.st);
                int k = 0;
                for (Req* r : batch)
                    if (r->cost_type == ct) {
                        std::memcpy(s.h_tasks.p + k, r->tasks, sizeof(AffineTask) * r->n);
                        k += r->n;
                    }
                std::vector<double> c(total);
                run_affine_tasks(s, total, ct, w.st, c.data(), false);
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
        inflight_ -= (int)batch.size();
        for (Req* r : batch)
            r->done = true;
        cv_done_.notify_all();
        cv_req_.notify_all();  // the other worker may be waiting for jobs of this batch
    }
}

}  // namespace regb
