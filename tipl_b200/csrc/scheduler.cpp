#include "scheduler.h"
#include <algorithm>
#include <cstring>
#include <string>

namespace regb {

CdmScheduler::CdmScheduler(int iters_per_round) : iters_(std::max(1, iters_per_round))
{
    {
        // the rounds are the serving engine's slower stage: their blocks go first when
        // they and the affine cost launches (default priority) both wait for an SM
        int lo = 0, hi = 0;
        REGB_CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        REGB_CK(cudaStreamCreateWithPriority(&st_, cudaStreamNonBlocking, hi));
    }
    REGB_CK(cudaEventCreate(&ev_[0]));
    REGB_CK(cudaEventCreate(&ev_[1]));
    int dev = 0;
    REGB_CK(cudaGetDevice(&dev));
    th_ = std::thread([this, dev] {
        cudaSetDevice(dev);
        loop();
    });
}

CdmScheduler::~CdmScheduler()
{
    {
        std::lock_guard<std::mutex> g(m_);
        stop_ = true;
    }
    cv_.notify_all();
    if (th_.joinable())
        th_.join();
    segs_.reset();
    status_.reset();
    if (st_) {
        cudaStreamSynchronize(st_);
        cudaStreamDestroy(st_);
    }
    for (cudaEvent_t e : ev_)
        if (e)
            cudaEventDestroy(e);
}

void CdmScheduler::run(CdmLevel& lvl, volatile const int* terminated)
{
    Entry e{&lvl, terminated};
    std::unique_lock<std::mutex> lk(m_);
    active_.push_back(&e);
    cv_.notify_all();
    cv_done_.wait(lk, [&] { return e.done; });
}

void CdmScheduler::loop()
{
    std::unique_lock<std::mutex> lk(m_);
    for (;;) {
        cv_.wait(lk, [&] { return stop_ || !active_.empty(); });
        if (stop_ && active_.empty())
            return;
        std::vector<Entry*> cur(active_);
        lk.unlock();
        bool failed = false;
        try {
            const int n = (int)cur.size();
            if ((int)h_segs_.n < n || (int)segs_.n < n || (int)h_status_.n < n || (int)status_.n < n) {
                const int cap = std::max(n, 2 * (int)h_segs_.n);
                h_segs_.alloc(cap);
                h_status_.alloc(cap);
                segs_.alloc(cap, st_);
                status_.alloc(cap, st_);
            }
            // segments sorted into groups of one (pixel type, modality gradient types)
            std::vector<int> order(n);
            for (int i = 0; i < n; ++i)
                order[i] = i;
            std::vector<std::string> keys(n);
            for (int i = 0; i < n; ++i)
                keys[i] = std::to_string(cur[i]->lvl->pix) + ":" + cur[i]->lvl->gtypes;
            auto key = [&](int i) -> const std::string& { return keys[i]; };
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key(a) < key(b); });
            for (int i = 0; i < n; ++i)
                h_segs_.p[i] = cur[order[i]]->lvl->seg;
            // one launch per group over exactly its blocks: each entry's blk0 counts the
            // blocks of the group's entries before it
            struct Group {
                int g0, g1, blocks;
            };
            std::vector<Group> groups;
            for (int g0 = 0; g0 < n;) {
                int g1 = g0, blocks = 0;
                while (g1 < n && key(order[g1]) == key(order[g0])) {
                    h_segs_.p[g1].blk0 = blocks;
                    blocks += h_segs_.p[g1].nblk;
                    ++g1;
                }
                groups.push_back({g0, g1, blocks});
                g0 = g1;
            }
            REGB_CK(cudaEventRecord(ev_[0], st_));
            REGB_CK(cudaMemcpyAsync(segs_.p, h_segs_.p, sizeof(CdmSeg) * n, cudaMemcpyHostToDevice, st_));
            for (int it = 0; it < iters_; ++it)
                for (const Group& g : groups) {
                    const Entry* e = cur[order[g.g0]];
                    launch_iteration(segs_.p + g.g0, g.g1 - g.g0, g.blocks, e->lvl->pix, e->lvl->gtypes, st_);
                }
            REGB_CK(launch_cdm_status(segs_.p, n, status_.p, st_));
            REGB_CK(cudaMemcpyAsync(h_status_.p, status_.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st_));
            REGB_CK(cudaEventRecord(ev_[1], st_));
            REGB_CK(cudaStreamSynchronize(st_));
            float ms = 0.0f;
            REGB_CK(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
            lk.lock();
            round_ms_ += ms;
            ++rounds_;
            round_segments_ += n;
            max_round_segments_ = std::max(max_round_segments_, n);
            for (int i = 0; i < n; ++i) {
                Entry* e = cur[order[i]];
                if (h_status_.p[i] || (e->term && *e->term)) {
                    e->done = true;
                    active_.erase(std::find(active_.begin(), active_.end(), e));
                }
            }
        } catch (...) {
            failed = true;
            lk.lock();
        }
        if (failed) {
            // leave every level that was in the failed round; its job reads the state
            for (Entry* e : cur) {
                e->done = true;
                auto it = std::find(active_.begin(), active_.end(), e);
                if (it != active_.end())
                    active_.erase(it);
            }
        }
        cv_done_.notify_all();
    }
}

}  // namespace regb
