// Affine registration driver: tipl::reg::linear (reg/linear.hpp:290-714) on the
// device.  The runner keeps the reference's structure -- multi-resolution above
// 96^3, the four DOF stages translocation -> translocation_scaling ->
// rigid_scaling -> affine, a line search running beside L-BFGS and sharing the
// best point -- but every probe set becomes one batched cost launch.
//
// Determinism: the reference runs the line search in a second thread and lets it
// exchange its best point with L-BFGS at arbitrary times (reg/linear.hpp:459-499).
// Here the two still run as two threads, but they meet at a rendezvous: their
// probe sets of one round go to the device together, and the best-point exchange
// happens only at L-BFGS's iteration start while the line search is parked at the
// rendezvous.  A job's trajectory is therefore a function of its inputs alone,
// whatever else shares the device.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include "affine_eval.h"
#include "host.h"
#include "optimizer.h"

namespace regb {

// reg_bound / narrow_bound / large_bound (reg/linear.hpp:258-266)
static const float kBound[3][3][8] = {
    {{0.75f, -0.75f, 0.4f, -0.4f, 1.5f, 0.7f, 0.1f, -0.1f},
     {0.75f, -0.75f, 0.25f, -0.25f, 1.5f, 0.7f, 0.1f, -0.1f},
     {0.75f, -0.75f, 0.25f, -0.25f, 1.5f, 0.7f, 0.1f, -0.1f}},
    {{0.2f, -0.2f, 0.2f, -0.2f, 1.2f, 0.8f, 0.05f, -0.05f},
     {0.2f, -0.2f, 0.1f, -0.1f, 1.2f, 0.8f, 0.05f, -0.05f},
     {0.2f, -0.2f, 0.1f, -0.1f, 1.2f, 0.8f, 0.05f, -0.05f}},
    {{1.0f, -1.0f, 0.5f, -0.5f, 2.0f, 0.5f, 0.25f, -0.25f},
     {1.0f, -1.0f, 0.4f, -0.4f, 2.0f, 0.5f, 0.25f, -0.25f},
     {1.0f, -1.0f, 0.4f, -0.4f, 2.0f, 0.5f, 0.25f, -0.25f}}};

enum { T_TRANS = 1, T_ROT = 2, T_SCALE = 4, T_TILT = 8 };

static opt::Vec identity_param()
{
    opt::Vec a(12, 0.0f);
    a[6] = a[7] = a[8] = 1.0f;
    return a;
}

// Meeting point of the line-search thread (0) and the L-BFGS thread (1).
class Rendezvous {
public:
    explicit Rendezvous(opt::BatchFn eval) : eval_(std::move(eval)) {}

    std::vector<double> submit(int who, const std::vector<opt::Vec>& c)
    {
        std::unique_lock<std::mutex> lk(m_);
        req_[who] = &c;
        waiting_[who] = true;
        cv_.notify_all();
        if (ready())
            run();
        else {
            const uint64_t g = gen_;
            cv_.wait(lk, [&] { return gen_ != g; });
        }
        if (err_)
            throw Failure(err_code_, err_msg_);
        return std::move(res_[who]);
    }
    void leave(int who)
    {
        std::unique_lock<std::mutex> lk(m_);
        alive_[who] = false;
        cv_.notify_all();
        if (ready() && (waiting_[0] || waiting_[1]))
            run();
    }
    // Blocks until the line search is parked at the rendezvous or has finished,
    // then runs f under the lock.
    template <typename F>
    void with_other_parked(F&& f)
    {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return !alive_[0] || waiting_[0]; });
        f(alive_[0]);
    }

private:
    bool ready() const
    {
        for (int k = 0; k < 2; ++k)
            if (alive_[k] && !waiting_[k])
                return false;
        return true;
    }
    void run()
    {
        std::vector<opt::Vec> all;
        size_t n0 = 0;
        if (waiting_[0]) {
            all.insert(all.end(), req_[0]->begin(), req_[0]->end());
            n0 = req_[0]->size();
        }
        if (waiting_[1])
            all.insert(all.end(), req_[1]->begin(), req_[1]->end());
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
        if (waiting_[0])
            res_[0].assign(r.begin(), r.begin() + n0);
        if (waiting_[1])
            res_[1].assign(r.begin() + n0, r.end());
        waiting_[0] = waiting_[1] = false;
        ++gen_;
        cv_.notify_all();
    }
    opt::BatchFn eval_;
    std::mutex m_;
    std::condition_variable cv_;
    bool alive_[2] = {true, true};
    bool waiting_[2] = {false, false};
    const std::vector<opt::Vec>* req_[2] = {nullptr, nullptr};
    std::vector<double> res_[2];
    uint64_t gen_ = 0;
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
    AffineEvaluator* eval = nullptr;
    long long evals = 0;

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
        std::vector<double> c = eval->eval(level, T.data(), (int)params.size());
        evals += (long long)params.size();
        for (double& v : c)
            v /= 1 * 2.0f;
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
                        opt::line_search(
                            arg_min2, up.data(), lo.data(), strategy,
                            [&](const std::vector<opt::Vec>& c) { return R.submit(0, c); }, optimal_value2,
                            (int)cur_search_count, [&] { return term(); });
                    } catch (...) {
                        ls_err = std::current_exception();
                    }
                    R.leave(0);
                });
                std::exception_ptr lb_err;
                try {
                    auto check = [&] {
                        R.with_other_parked([&](bool) { merge(); });
                        return term();
                    };
                    for (;;) {
                        opt::lbfgs(
                            arg_min, up.data(), lo.data(),
                            [&](const std::vector<opt::Vec>& c) { return R.submit(1, c); }, optimal_value, check,
                            precision, max_iterations);
                        bool ls_alive = true;
                        R.with_other_parked([&](bool alive) { ls_alive = alive; });
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

// Runs the runner from an explicit state: the reference runner's fields at the
// point its GPU implementation is entered (reg/linear.hpp:597-604).
static LinearResult run_state(const uint8_t* d_from, const int* fdim, const float* from_vs, const uint8_t* d_to,
                              const int* tdim, const float* to_vs, float* arg, const regb_runner_state& s,
                              volatile const int* terminated, cudaStream_t st, AffineBatcher* batcher)
{
    opt::Vec a(arg, arg + 12);
    LinearRunner R(a);
    R.terminated = terminated;
    R.cost_type = s.cost_type;
    R.arg_upper.assign(s.arg_upper, s.arg_upper + 12);
    R.arg_lower.assign(s.arg_lower, s.arg_lower + 12);
    R.reg_list.assign(s.reg_list, s.reg_list + std::max(0, std::min(s.n_reg, 8)));
    if (R.reg_list.empty())
        throw Failure(REGB_ERR_ARG, "empty reg_list");
    R.search_count = s.search_count;
    R.precision = s.precision;
    R.max_iterations = s.max_iterations;

    // pyramid: a level below while the fixed volume exceeds 96^3 (reg/linear.hpp:309-322, 527-545)
    std::vector<DevBuf<uint8_t>> bufs;
    LinearRunner::Level L0;
    L0.from = d_from;
    L0.to = d_to;
    for (int i = 0; i < 3; ++i) {
        L0.fd[i] = fdim[i];
        L0.td[i] = tdim[i];
        L0.fvs[i] = from_vs[i];
        L0.tvs[i] = to_vs[i];
    }
    R.levels.push_back(L0);
    if (s.multi_resolution) {
        for (;;) {
            const LinearRunner::Level& c = R.levels.back();
            const long long sz = (long long)c.fd[0] * c.fd[1] * c.fd[2];
            if (!((double)sz > std::pow(96, 3)))
                break;
            LinearRunner::Level n;
            for (int i = 0; i < 3; ++i) {
                n.fd[i] = (c.fd[i] + 1) / 2;
                n.td[i] = (c.td[i] + 1) / 2;
                n.fvs[i] = c.fvs[i] * 2.0f;
                n.tvs[i] = c.tvs[i] * 2.0f;
            }
            bufs.emplace_back((size_t)n.fd[0] * n.fd[1] * n.fd[2], st);
            bufs.emplace_back((size_t)n.td[0] * n.td[1] * n.td[2], st);
            REGB_CK(launch_downsample(c.from, bufs[bufs.size() - 2].p, c.fd[0], c.fd[1], c.fd[2], 0, st));
            REGB_CK(launch_downsample(c.to, bufs.back().p, c.td[0], c.td[1], c.td[2], 0, st));
            n.from = bufs[bufs.size() - 2].p;
            n.to = bufs.back().p;
            R.levels.push_back(n);
        }
    }
    std::vector<AffineEvaluator::Pair> pairs;
    for (auto& L : R.levels)
        pairs.push_back({L.from, Dim3{L.fd[0], L.fd[1], L.fd[2]}, L.to, Dim3{L.td[0], L.td[1], L.td[2]}});
    AffineEvaluator ev(pairs, s.cost_type, st);
    ev.set_batcher(batcher);
    R.eval = &ev;
    // optimize<cost, mr> (reg/linear.hpp:552-560)
    const double cost = s.multi_resolution ? R.run_optimize_mr(0) : R.run_optimize(0, 0);
    std::copy(a.begin(), a.end(), arg);
    LinearResult out;
    out.cost = (float)cost;
    out.evals = R.evals;
    return out;
}

// The runner state tipl::reg::linear sets up (reg/linear.hpp:631-651, 365-420):
// bounds from the bound table around the identity (absolute) or around arg
// (narrow), the DOF stage list of the registration type, and multi-resolution
// with the line search except for the narrow bound.
void runner_state_from_param(const int* fdim, const float* from_vs, const int* tdim, const float* to_vs,
                             const float* arg, const regb_linear_param& p, regb_runner_state& s)
{
    opt::Vec a(arg, arg + 12);
    LinearRunner R(a);
    LinearRunner::Level L0{};
    for (int i = 0; i < 3; ++i) {
        L0.fd[i] = fdim[i];
        L0.td[i] = tdim[i];
        L0.fvs[i] = from_vs[i];
        L0.tvs[i] = to_vs[i];
    }
    R.levels.push_back(L0);
    const float(*bound)[8] = kBound[(p.bound >= 0 && p.bound < 3) ? p.bound : 0];
    const bool narrow = (p.bound == REGB_BOUND_NARROW);
    R.set_bound(p.reg_type, bound, narrow ? false : true);
    std::memset(&s, 0, sizeof(s));
    std::copy(R.arg_upper.begin(), R.arg_upper.end(), s.arg_upper);
    std::copy(R.arg_lower.begin(), R.arg_lower.end(), s.arg_lower);
    s.n_reg = (int)R.reg_list.size();
    for (int i = 0; i < s.n_reg; ++i)
        s.reg_list[i] = R.reg_list[i];
    s.search_count = narrow ? 0 : p.search_count;
    s.multi_resolution = narrow ? 0 : 1;
    s.cost_type = p.cost_type;
    s.precision = 0.001;
    s.max_iterations = 128;
}

LinearResult linear_register(const uint8_t* d_from, const int* fdim, const float* from_vs, const uint8_t* d_to,
                             const int* tdim, const float* to_vs, float* arg, const regb_linear_param& p,
                             volatile const int* terminated, cudaStream_t st, AffineBatcher* batcher)
{
    regb_runner_state s;
    runner_state_from_param(fdim, from_vs, tdim, to_vs, arg, p, s);
    return run_state(d_from, fdim, from_vs, d_to, tdim, to_vs, arg, s, terminated, st, batcher);
}

LinearResult linear_register_state(const uint8_t* d_from, const int* fdim, const float* from_vs, const uint8_t* d_to,
                                   const int* tdim, const float* to_vs, float* arg, const regb_runner_state& s,
                                   volatile const int* terminated, cudaStream_t st)
{
    return run_state(d_from, fdim, from_vs, d_to, tdim, to_vs, arg, s, terminated, st, nullptr);
}

}  // namespace regb
