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
#include <memory>
#include "affine_eval.h"
#include "host.h"
#include "linear_runner.h"
#include "mask_init.h"
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

// Runs the runner from an explicit state: the reference runner's fields at the
// point its GPU implementation is entered (reg/linear.hpp:597-604).
// npairs image pairs d_from[i] / d_to[i] share the dims fdim / tdim; each has its
// own pyramid and evaluator, and a candidate's cost is their sum in pair order.
static LinearResult run_state(const uint8_t* const* d_from, const uint8_t* const* d_to, int npairs, const int* fdim,
                              const float* from_vs, const int* tdim, const float* to_vs, float* arg,
                              const regb_runner_state& s, volatile const int* terminated, cudaStream_t st,
                              AffineBatcher* batcher)
{
    opt::Vec a(arg, arg + 12);
    LinearRunner R(a);
    R.npairs = npairs;
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
    std::vector<std::vector<const uint8_t*>> pf(1), pt(1);  // [level][pair]
    pf[0].assign(d_from, d_from + npairs);
    pt[0].assign(d_to, d_to + npairs);
    LinearRunner::Level L0;
    L0.from = d_from[0];
    L0.to = d_to[0];
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
            std::vector<const uint8_t*> nf(npairs), nt(npairs);
            for (int k = 0; k < npairs; ++k) {
                bufs.emplace_back((size_t)n.fd[0] * n.fd[1] * n.fd[2], st);
                bufs.emplace_back((size_t)n.td[0] * n.td[1] * n.td[2], st);
                REGB_CK(launch_downsample(pf.back()[k], bufs[bufs.size() - 2].p, c.fd[0], c.fd[1], c.fd[2], 0, st));
                REGB_CK(launch_downsample(pt.back()[k], bufs.back().p, c.td[0], c.td[1], c.td[2], 0, st));
                nf[k] = bufs[bufs.size() - 2].p;
                nt[k] = bufs.back().p;
            }
            n.from = nf[0];
            n.to = nt[0];
            pf.push_back(nf);
            pt.push_back(nt);
            R.levels.push_back(n);
        }
    }
    std::vector<std::unique_ptr<AffineEvaluator>> evs;
    for (int k = 0; k < npairs; ++k) {
        std::vector<AffineEvaluator::Pair> pairs;
        for (size_t l = 0; l < R.levels.size(); ++l) {
            const LinearRunner::Level& L = R.levels[l];
            pairs.push_back({pf[l][k], Dim3{L.fd[0], L.fd[1], L.fd[2]}, pt[l][k], Dim3{L.td[0], L.td[1], L.td[2]}});
        }
        evs.emplace_back(new AffineEvaluator(pairs, s.cost_type, st));
        evs.back()->set_batcher(batcher);
    }
    // run_optimize's fun (reg/linear.hpp:427-440): double cost = 0; cost += each pair's
    R.eval = [&evs](int level, const float* T, int n) {
        std::vector<double> c((size_t)n, 0.0);
        for (auto& ev : evs) {
            const std::vector<double> ck = ev->eval(level, T, n);
            for (int k = 0; k < n; ++k)
                c[k] += ck[k];
        }
        return c;
    };
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

// tipl::reg::linear (reg/linear.hpp:622-700).  An affine search (not narrow-bound)
// whose two volumes both have a mask starts from estimate_affine_param: the search
// runs on a surrogate -- the estimated parameters with unit scaling against the
// moving volume's voxel size divided by the estimated scaling -- and its result is
// converted back to parameters against the true voxel size.
LinearResult linear_register(const uint8_t* d_from, const int* fdim, const float* from_vs, const uint8_t* d_to,
                             const int* tdim, const float* to_vs, float* arg, const regb_linear_param& p,
                             volatile const int* terminated, cudaStream_t st, AffineBatcher* batcher)
{
    return linear_register_multi(&d_from, &d_to, 1, fdim, from_vs, tdim, to_vs, arg, p, terminated, st, batcher);
}

LinearResult linear_register_multi(const uint8_t* const* d_from, const uint8_t* const* d_to, int npairs,
                                   const int* fdim, const float* from_vs, const int* tdim, const float* to_vs,
                                   float* arg, const regb_linear_param& p, volatile const int* terminated,
                                   cudaStream_t st, AffineBatcher* batcher)
{
    if (npairs < 1)
        throw Failure(REGB_ERR_ARG, "linear: no image pair");
    // the mask start looks at the first pair only (reg/linear.hpp:661-663)
    if (p.reg_type == REGB_REG_AFFINE && p.bound != REGB_BOUND_NARROW) {
        MaskCounts cf, ct;
        mask_counts(d_from[0], fdim, cf, st);
        if (has_mask(cf)) {
            mask_counts(d_to[0], tdim, ct, st);
            if (has_mask(ct)) {
                float sur[12], new_to_vs[3];
                estimate_affine_param(cf, from_vs, ct, to_vs, sur);
                for (int i = 0; i < 3; ++i) {
                    new_to_vs[i] = to_vs[i] / std::max<float>(sur[6 + i], 0.01f);
                    sur[6 + i] = 1.0f;
                }
                regb_runner_state s;
                runner_state_from_param(fdim, from_vs, tdim, new_to_vs, sur, p, s);
                LinearResult r = run_state(d_from, d_to, npairs, fdim, from_vs, tdim, new_to_vs, sur, s, terminated,
                                           st, batcher);
                float T[12];
                affine_to_matrix(sur, fdim, from_vs, tdim, new_to_vs, T);
                matrix_to_affine_param(T, fdim, from_vs, tdim, to_vs, arg);
                return r;
            }
        }
    }
    regb_runner_state s;
    runner_state_from_param(fdim, from_vs, tdim, to_vs, arg, p, s);
    return run_state(d_from, d_to, npairs, fdim, from_vs, tdim, to_vs, arg, s, terminated, st, batcher);
}

LinearResult linear_register_state(const uint8_t* d_from, const int* fdim, const float* from_vs, const uint8_t* d_to,
                                   const int* tdim, const float* to_vs, float* arg, const regb_runner_state& s,
                                   volatile const int* terminated, cudaStream_t st)
{
    return run_state(&d_from, &d_to, 1, fdim, from_vs, tdim, to_vs, arg, s, terminated, st, nullptr);
}

LinearResult linear_register_state_multi(const uint8_t* const* d_from, const uint8_t* const* d_to, int npairs,
                                         const int* fdim, const float* from_vs, const int* tdim, const float* to_vs,
                                         float* arg, const regb_runner_state& s, volatile const int* terminated,
                                         cudaStream_t st)
{
    return run_state(d_from, d_to, npairs, fdim, from_vs, tdim, to_vs, arg, s, terminated, st, nullptr);
}

}  // namespace regb
