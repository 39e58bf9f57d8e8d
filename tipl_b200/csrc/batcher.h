// Cross-job batching of affine cost evaluations (the serving engine's affine stage).
#pragma once
#include <condition_variable>
#include <deque>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>
#include "affine_eval.h"

namespace regb {

constexpr int kCostTypes = 3;  // REGB_COST_CORR, REGB_COST_MI, REGB_COST_MI32

// Collects cost-evaluation requests from many jobs and evaluates all pending ones
// of a cost type in one launch.  A request's tasks carry their own volumes, so
// requests of different jobs, shapes and pyramid levels mix freely; every task's
// cost depends only on its own inputs, whatever it is batched with.
class AffineBatcher {
public:
    explicit AffineBatcher(int gather_us);
    ~AffineBatcher();
    AffineBatcher(const AffineBatcher&) = delete;
    AffineBatcher& operator=(const AffineBatcher&) = delete;

    // Blocks until every task's cost is written to out.
    void eval(const AffineTask* tasks, int n, int cost_type, double* out);
    // Number of jobs currently able to submit (the dispatcher waits a little for the
    // rest of them to join a batch once the device is free).
    void add_client();
    void remove_client();

    long long launches() const { return launches_; }
    long long tasks_evaluated() const { return tasks_; }

private:
    struct Req {
        const AffineTask* tasks;
        int n;
        int cost_type;
        double* out;
        bool done = false;
        std::exception_ptr err;
    };
    void loop();
    std::mutex m_;
    std::condition_variable cv_req_, cv_done_;
    std::deque<Req*> pending_;
    int clients_ = 0;
    bool stop_ = false;
    int gather_us_;
    long long launches_ = 0, tasks_ = 0;
    TaskScratch scratch_[kCostTypes];  // one per cost type (REGB_COST_CORR, _MI, _MI32)
    cudaStream_t st_ = nullptr;
    std::thread th_;
};

}  // namespace regb
