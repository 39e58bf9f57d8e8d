// Cross-job batching of CDM iterations (the serving engine's nonlinear stage).
#pragma once
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>
#include "cdm_level.h"

namespace regb {

// Every registered CDM level is one segment.  A round launches the iteration
// kernel sequence `iters_per_round` times for all active segments of the same
// pixel type and modality gradient types at once, then reads back every segment's done flag
// with one gather.  Levels join and leave between rounds; a level's decisions
// live in its own control block, so its result does not depend on what it was
// batched with.
class CdmScheduler {
public:
    explicit CdmScheduler(int iters_per_round);
    ~CdmScheduler();
    CdmScheduler(const CdmScheduler&) = delete;
    CdmScheduler& operator=(const CdmScheduler&) = delete;
    // Iterates the level until its loop ends (or terminated is set); blocks the caller.
    void run(CdmLevel& lvl, volatile const int* terminated);
    // counters, read under the scheduler's lock
    long long rounds()
    {
        std::lock_guard<std::mutex> g(m_);
        return rounds_;
    }
    long long round_segments()  // levels summed over rounds
    {
        std::lock_guard<std::mutex> g(m_);
        return round_segments_;
    }
    double round_ms()  // device time of the rounds, summed
    {
        std::lock_guard<std::mutex> g(m_);
        return round_ms_;
    }
    int max_round_segments()  // the most levels one round has carried
    {
        std::lock_guard<std::mutex> g(m_);
        return max_round_segments_;
    }

private:
    struct Entry {
        CdmLevel* lvl;
        volatile const int* term;
        bool done = false;
    };
    void loop();
    std::mutex m_;
    std::condition_variable cv_, cv_done_;
    std::vector<Entry*> active_;
    bool stop_ = false;
    int iters_;
    long long rounds_ = 0;
    long long round_segments_ = 0;
    double round_ms_ = 0.0;
    int max_round_segments_ = 0;
    cudaStream_t st_ = nullptr;
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    DevBuf<CdmSeg> segs_;
    PinBuf<CdmSeg> h_segs_;
    DevBuf<int> status_;
    PinBuf<int> h_status_;
    std::thread th_;
};

}  // namespace regb
