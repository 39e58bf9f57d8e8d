// The affine search of tipl::reg::linear (reg/linear.hpp:290-561) as host logic:
// the DOF stages, bounds, multi-resolution recursion and the line search beside
// L-BFGS meeting at a rendezvous.  Cost evaluation is a callback (one batch of
// matrices of one pyramid level -> their costs), so the same runner drives the
// device evaluator and, in tests, a CPU one.
#pragma once
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <exception>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include "host.h"
#include "optimizer.h"

namespace regb {

enum { T_TRANS = 1, T_ROT = 2, T_SCALE = 4, T_TILT = 8 };

inline opt::Vec identity_param()
{
    opt::Vec a(12, 0.0f);
    a[6] = a[7] = a[8] = 1.0f;
    return a;
}

// Meeting point of the line-search thread (0) and the L-BFGS thread (1).
//
// The reference runs the two freely in two threads (reg/linear.hpp:459-499): both
// evaluate costs at the same rate, they exchange their best point at every check
// either makes, and which one is ahead decides the trajectory.  Here that timing is
// replayed on a virtual clock instead of the wall clock: a probe set of n costs n
// ticks, so a set submitted at clock t is finished at t + n.  Exactly one thread runs
// at a time; when both are parked at the rendezvous, the set that finishes first
// (L-BFGS on a tie) is handed back and its thread resumes at that set's end time.
// A check (with_other_parked) exchanges best points while the other thread is
// parked, as the reference's checks do while the other thread is mid-evaluation.
// Every parked set not yet evaluated goes to the device in one batch.  The
// trajectory is therefore a function of the inputs alone.
// Clock ticks one line-search task takes, against one tick per L-BFGS probe.  The
// reference's outcome depends on this ratio; 0.5 matched the median final cost of
// repeated reference runs (1 to 16 host threads) best over 23 seeded MI and
// correlation registrations of masked and unmasked phantom pairs (mean difference
// -0.1 %, the rest within the reference's own run-to-run spread).
constexpr double kLineSearchTick = 0.5;

class Rendezvous {
public:
    explicit Rendezvous(opt::BatchFn eval) : eval_(std::move(eval)) {}

    // Parks `who` with the set c, which takes `ticks` of its clock (-1: one per probe).
    std::vector<double> submit(int who, const std::vector<opt::Vec>& c, double ticks = -1.0)
    {
        std::unique_lock<std::mutex> lk(m_);
        req_[who] = &c;
        pending_[who] = true;
        evaluated_[who] = c.empty();
        if (c.empty())
            res_[who].clear();
        released_[who] = false;
        fin_[who] = t_[who] + (ticks < 0 ? (double)c.size() : ticks);
        schedule();
        cv_.notify_all();
        cv_.wait(lk, [&] { return released_[who] || err_; });
        pending_[who] = false;
        released_[who] = false;
        if (err_)
            throw Failure(err_code_, err_msg_);
        return std::move(res_[who]);
    }
    void leave(int who)
    {
        std::unique_lock<std::mutex> lk(m_);
        alive_[who] = false;
        schedule();
        cv_.notify_all();
    }
    // Blocks until the other thread is parked at the rendezvous or has finished,
    // then runs f(other thread alive) under the lock.
    template <typename F>
    void with_other_parked(int who, F&& f)
    {
        const int o = 1 - who;
        std::unique_lock<std::mutex> lk(m_);
        in_check_[who] = true;
        cv_.notify_all();
        // (a thread that is itself waiting at a check counts as parked, so two checks
        // never wait for each other)
        cv_.wait(lk, [&] { return !alive_[o] || parked(o) || in_check_[o] || err_; });
        f(alive_[o]);
        in_check_[who] = false;
    }

private:
    bool parked(int k) const { return pending_[k] && !released_[k]; }
    // Hands back at most one parked set, and only while no thread runs.
    void schedule()
    {
        for (int k = 0; k < 2; ++k)
            if (alive_[k] && !parked(k))
                return;
        int pick = -1;
        if (parked(0) && parked(1))
            pick = (fin_[1] <= fin_[0]) ? 1 : 0;
        else if (parked(0))
            pick = 0;
        else if (parked(1))
            pick = 1;
        if (pick < 0)
            return;
        if (!evaluated_[pick])
            evaluate();
        released_[pick] = true;
        t_[pick] = fin_[pick];
    }
    void evaluate()
    {
        std::vector<opt::Vec> all;
        size_t n[2] = {0, 0};
        bool in[2] = {false, false};
        for (int k = 0; k < 2; ++k)
            if (parked(k) && !evaluated_[k]) {
                all.insert(all.end(), req_[k]->begin(), req_[k]->end());
                n[k] = req_[k]->size();
                in[k] = true;
            }
        std::vector<double> r;
        try {
            if (!all.empty())
                r = eval_(all);
        } catch (const Failure& f) {
            err_ = true;
            err_code_ = f.code;
            err_msg_ = f.what();
            r.assign(all.size(), 0.0);
        }
        size_t off = 0;
        for (int k = 0; k < 2; ++k)
            if (in[k]) {
                res_[k].assign(r.begin() + off, r.begin() + off + n[k]);
                off += n[k];
                evaluated_[k] = true;
            }
    }
    opt::BatchFn eval_;
    std::mutex m_;
    std::condition_variable cv_;
    bool alive_[2] = {true, true};
    bool pending_[2] = {false, false};
    bool evaluated_[2] = {false, false};
    bool released_[2] = {false, false};
    bool in_check_[2] = {false, false};
    double t_[2] = {0.0, 0.0};
    double fin_[2] = {0.0, 0.0};
    const std::vector<opt::Vec>* req_[2] = {nullptr, nullptr};
    std::vector<double> res_[2];
    bool err_ = false;
    regb_status err_code_ = REGB_OK;
    std::string err_msg_;
};

class LinearRunner {
public:
    struct Level {
        const uint8_t* from;
        const uint8_t* to;
        int fd[3], td[3];
        float fvs[3], tvs[3];
    };
    std::vector<Level> levels;  // 0 = full resolution
    opt::Vec arg_upper = identity_param(), arg_lower = identity_param();
    opt::Vec& arg_min;
    std::vector<int> reg_list = {1, 5, 7, 15};
    unsigned int search_count = 16;
    double precision = 0.001;
    int max_iterations = 128;
    int cost_type = REGB_COST_MI;
    volatile const int* terminated = nullptr;
    // costs of n matrices (12 floats each) on pyramid level `level`
    // the summed cost of every image pair, 0.0 + c0 + c1 + ... in pair order
    std::function<std::vector<double>(int level, const float* T, int n)> eval;
    int npairs = 1;
    long long evals = 0;
    // called after each DOF stage with the stage's type, cost and parameters
    std::function<void(int reg, double cost, const opt::Vec& arg)> on_stage;

    explicit LinearRunner(opt::Vec& a) : arg_min(a) {}

    bool term() const { return terminated && *terminated; }

    // set_bound (reg/linear.hpp:370-420)
    void set_bound(int type, const float (*bound)[8], bool absolute)
    {
        if (type == 1) reg_list = {1};
        if (type == 2) reg_list = {2};
        if (type == 3) reg_list = {1, 3};
        if (type == 4) reg_list = {4};
        if (type == 7) reg_list = {1, 5, 7};
        if (type == 15) reg_list = {1, 5, 7, 15};
        if (absolute) {
            arg_upper = identity_param();
            arg_lower = identity_param();
        } else
            arg_upper = arg_lower = arg_min;
        const Level& L = levels[0];
        for (int i = 0; i < 3; ++i) {
            if (type & T_TRANS) {
                const float range = std::max<float>((float)L.fd[i] * L.fvs[i], (float)L.td[i] * L.tvs[i]) * 0.5f;
                arg_upper[i] += range * bound[i][0];
                arg_lower[i] += range * bound[i][1];
            }
            if (type & T_SCALE) {
                arg_upper[6 + i] *= bound[i][4];
                arg_lower[6 + i] *= bound[i][5];
            }
        }
        for (int i = 0; i < 3; ++i) {
            if (type & T_ROT) {
                arg_upper[3 + i] += 1.57079632679f * bound[i][2];
                arg_lower[3 + i] += 1.57079632679f * bound[i][3];
            }
            if (type & T_TILT) {
                arg_upper[9 + i] += bound[i][6];
                arg_lower[9 + i] += bound[i][7];
            }
        }
    }

    // get_current_bound (reg/linear.hpp:334-364)
    void current_bound(int type, opt::Vec& up, opt::Vec& lo) const
    {
        up = arg_upper;
        lo = arg_lower;
        for (int i = 0; i < 3; ++i) {
            if (!(type & T_TRANS)) up[i] = lo[i] = arg_min[i];
            if (!(type & T_SCALE)) up[6 + i] = lo[6 + i] = arg_min[6 + i];
            if (!(type & T_ROT)) up[3 + i] = lo[3 + i] = arg_min[3 + i];
            if (!(type & T_TILT)) up[9 + i] = lo[9 + i] = arg_min[9 + i];
        }
    }

    // fun (reg/linear.hpp:427-444): the cost at a parameter set, divided by
    // 2 * (number of image pairs).
    std::vector<double> fun(int level, const std::vector<opt::Vec>& params)
    {
        const Level& L = levels[level];
        std::vector<float> T(12 * params.size());
        for (size_t k = 0; k < params.size(); ++k)
            affine_to_matrix(params[k].data(), L.fd, L.fvs, L.td, L.tvs, &T[12 * k]);
        std::vector<double> c = eval(level, T.data(), (int)params.size());
        evals += (long long)params.size();
        const float div = (float)npairs * 2.0f;  // cost_fun.size() * 2.0f, a float
        for (double& v : c)
            v /= div;
        return c;
    }

    // run_optimize (reg/linear.hpp:421-516)
    double run_optimize(int level, unsigned int cur_search_count)
    {
        auto f1 = [&](const std::vector<opt::Vec>& p) { return fun(level, p); };
        double optimal_value = fun(level, {arg_min})[0];
        if (cur_search_count) {
            static const std::vector<int> strategy = {0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1};
            for (size_t it = 0; it < reg_list.size() && !term(); ++it) {
                opt::Vec up, lo;
                current_bound(reg_list[it], up, lo);
                opt::Vec arg_min2 = arg_min;
                double optimal_value2 = optimal_value;
                Rendezvous R(f1);
                auto merge = [&] {
                    if (optimal_value2 < optimal_value) {
                        optimal_value = optimal_value2;
                        arg_min = arg_min2;
                    }
                    if (optimal_value < optimal_value2) {
                        optimal_value2 = optimal_value;
                        arg_min2 = arg_min;
                    }
                };
                std::exception_ptr ls_err;
                std::thread ls([&] {
                    try {
                        auto check = [&] {
                            R.with_other_parked(0, [&](bool) { merge(); });
                            return term();
                        };
                        // the line search's sets are charged per applied result (tick),
                        // as the reference's tasks finish one evaluation each
                        const std::vector<opt::Vec> none;
                        opt::line_search(
                            arg_min2, up.data(), lo.data(), strategy,
                            [&](const std::vector<opt::Vec>& c) { return R.submit(0, c, 0.0); }, optimal_value2,
                            (int)cur_search_count, check, [&] { R.submit(0, none, kLineSearchTick); });
                    } catch (...) {
                        ls_err = std::current_exception();
                    }
                    R.leave(0);
                });
                std::exception_ptr lb_err;
                try {
                    auto check = [&] {
                        R.with_other_parked(1, [&](bool) { merge(); });
                        return term();
                    };
                    for (;;) {
                        opt::lbfgs(
                            arg_min, up.data(), lo.data(),
                            [&](const std::vector<opt::Vec>& c) { return R.submit(1, c); }, optimal_value, check,
                            precision, max_iterations);
                        bool ls_alive = true;
                        R.with_other_parked(1, [&](bool alive) { ls_alive = alive; });
                        if (!ls_alive)
                            break;
                    }
                } catch (...) {
                    lb_err = std::current_exception();
                }
                R.leave(1);
                ls.join();
                if (ls_err)
                    std::rethrow_exception(ls_err);
                if (lb_err)
                    std::rethrow_exception(lb_err);
                merge();
                if (on_stage)
                    on_stage(reg_list[it], optimal_value, arg_min);
            }
        } else {
            opt::Vec up, lo;
            current_bound(reg_list.back(), up, lo);
            opt::lbfgs(arg_min, up.data(), lo.data(), f1, optimal_value, [&] { return term(); },
                       precision * 0.2f, max_iterations);
        }
        return optimal_value;
    }

    // run_optimize_mr (reg/linear.hpp:527-550)
    double run_optimize_mr(int level)
    {
        const Level& L = levels[level];
        const long long sz = (long long)L.fd[0] * L.fd[1] * L.fd[2];
        const bool is_large = (double)sz > std::pow(96, 3);
        if (is_large) {
            const double v = run_optimize_mr(level + 1);
            if ((double)sz > std::pow(256, 3))
                return v;
        }
        return run_optimize(level, is_large ? 0 : search_count);
    }
};

}  // namespace regb
