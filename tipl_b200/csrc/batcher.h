// Cross-job batching of affine cost evaluations (the serving engine's affine stage).
#pragma once
#include <atomic>
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
// of a cost type in one launch (one launch per worker may be in flight, each worker
// on its own stream).
// A request's tasks carry their own volumes, so requests of different jobs, shapes
// and pyramid levels mix freely; every task's cost depends only on its own inputs,
// whatever it is batched with.
class AffineBatcher {
public:
    // workers: concurrent launches (1..kMaxWorkers)
    AffineBatcher(int gather_us, int workers);
    ~AffineBatcher();
    AffineBatcher(const AffineBatcher&) = delete;
    AffineBatcher& operator=(const AffineBatcher&) = delete;

    // Blocks until every task's cost is written to out.
    void eval(const AffineTask* tasks, int n, int cost_type, double* out);
    // Number of jobs currently able to submit (the dispatcher waits a little for the
    // rest of them to join a batch once the device is free).
    void add_client();
    void remove_client();

    long long launches() const { return launches_.load(); }
    long long tasks_evaluated() const { return tasks_.load(); }

private:
    struct Req {
        const AffineTask* tasks;
        int n;
        int cost_type;
        double* out;
        bool done = false;
        std::exception_ptr err;
    };
    // Workers, each with its own stream and scratch: while one batch runs on the device,
    // the jobs it does not hold can form the next batch, which another worker launches at
    // once instead of after the first batch's results are back.
    static constexpr int kMaxWorkers = 4;
    int nworkers_;
    struct Worker {
        TaskScratch scratch[kCostTypes];  // one per cost type (REGB_COST_CORR, _MI, _MI32)
        cudaStream_t st = nullptr;
        std::thread th;
    };
    void loop(Worker& w);
    std::mutex m_;
    std::condition_variable cv_req_, cv_done_;
    std::deque<Req*> pending_;
    int clients_ = 0;
    int inflight_ = 0;  // requests taken by a worker and not yet answered
    bool stop_ = false;
    int gather_us_;
    std::atomic<long long> launches_{0}, tasks_{0};
    Worker workers_[kMaxWorkers];
};

}  // namespace regb
