// Bounded optimisers of the affine search (numerical/optimization.hpp), restated
// with one change of form: every probe set the reference evaluates with par_for
// (the finite-difference probes, the Armijo steps, the grid samples of the line
// search) is handed to a batch evaluator as one set, so the device evaluates it
// in a single launch.  The arithmetic (float parameters, double costs, the order
// of every update) follows the reference.
#pragma once
#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <vector>

namespace regb {
namespace opt {

using Vec = std::vector<float>;
// Evaluates a set of parameter vectors; returns one cost per vector, in order.
using BatchFn = std::function<std::vector<double>(const std::vector<Vec>&)>;
using StopFn = std::function<bool()>;

// norm2 over float values with float accumulation (numerical/matrix.hpp:209-233).
inline float norm2f(const float* b, const float* e)
{
    if (b == e)
        return 0.0f;
    float sum = *b;
    if (++b == e)
        return std::abs(sum);
    sum *= sum;
    for (; b != e; ++b) {
        float x2 = *b;
        x2 *= x2;
        sum += x2;
    }
    return std::sqrt(sum);
}

// calculate_resolution (numerical/optimization.hpp:98-104)
inline double calculate_resolution(Vec& tols, const float* up, const float* lo, double precision)
{
    for (size_t i = 0; i < tols.size(); ++i)
        tols[i] = (float)((up[i] - lo[i]) * precision);
    return norm2f(tols.data(), tols.data() + tols.size());
}

// estimate_change (numerical/optimization.hpp:16-29): fun(x + tol_i e_i) for every
// i with a non-zero tolerance; other entries of fun_ei keep their value.
inline void estimate_change(const Vec& x, const Vec& tol, std::vector<double>& fun_ei, const BatchFn& fun)
{
    std::vector<Vec> c;
    std::vector<size_t> idx;
    for (size_t i = 0; i < x.size(); ++i) {
        if (tol[i] == 0)
            continue;
        Vec v(x);
        v[i] += tol[i];
        c.push_back(std::move(v));
        idx.push_back(i);
    }
    auto r = fun(c);
    for (size_t k = 0; k < idx.size(); ++k)
        fun_ei[idx[k]] = r[k];
}

// gradient (numerical/optimization.hpp:37-52): g = (float(fun_ei) - fun_x) / tol.
inline void gradient(const Vec& tol, double fun_x, const std::vector<double>& fun_ei, Vec& g)
{
    for (size_t i = 0; i < g.size(); ++i)
        g[i] = (float)fun_ei[i];
    for (size_t i = 0; i < g.size(); ++i)
        g[i] = (float)((double)g[i] - fun_x);
    for (size_t i = 0; i < g.size(); ++i)
        g[i] = (tol[i] == 0) ? 0.0f : g[i] / tol[i];
}

// armijo_line_search (numerical/optimization.hpp:59-96): ten steps 2^-6 .. 2^3
// along -g, clamped to the bounds, evaluated as one set; the lowest cost wins.
inline bool armijo(Vec& x, const float* up, const float* lo, const Vec& g, double& fun_x, const BatchFn& fun)
{
    const size_t n = x.size();
    std::vector<Vec> list;
    for (double step = 0.015625; step <= 10.0; step *= 2) {
        Vec nx(x);
        for (size_t j = 0; j < n; ++j)
            nx[j] = (float)((double)nx[j] + (double)g[j] * -step);
        for (size_t j = 0; j < n; ++j)
            nx[j] = (float)std::min<double>(std::max<double>(nx[j], lo[j]), up[j]);
        list.push_back(std::move(nx));
    }
    auto r = fun(list);
    std::vector<double> cost(1 + r.size());
    cost[0] = fun_x;
    for (size_t k = 0; k < r.size(); ++k)
        cost[k + 1] = r[k];
    size_t fin = size_t(std::min_element(cost.begin(), cost.end()) - cost.begin());
    if (fin == 0)
        return false;
    fun_x = cost[fin];
    x = list[fin - 1];
    return true;
}

// lbfgs (numerical/optimization.hpp:137-270), history m = 10.
inline void lbfgs(Vec& x, const float* up, const float* lo, const BatchFn& fun, double& fun_x, const StopFn& terminated,
                  double precision, int max_iteration, size_t m = 10)
{
    const size_t size = x.size();
    Vec tols(size);
    const double tol_length = calculate_resolution(tols, up, lo, precision);
    std::vector<Vec> S, Y;
    std::vector<double> RHO;
    Vec g(size), g_old(size), x_old(size);
    std::vector<double> fun_x_ei(size, 0.0);
    estimate_change(x, tols, fun_x_ei, fun);
    gradient(tols, fun_x, fun_x_ei, g);
    for (int iter = 0; iter < max_iteration && !terminated(); ++iter) {
        Vec q = g;
        std::vector<double> alpha(S.size());
        for (int i = (int)S.size() - 1; i >= 0; --i) {
            double sq = 0.0;
            for (size_t j = 0; j < size; ++j)
                sq += S[i][j] * q[j];
            alpha[i] = RHO[i] * sq;
            for (size_t j = 0; j < size; ++j)
                q[j] = (float)((double)q[j] - alpha[i] * Y[i][j]);
        }
        if (!S.empty()) {
            double yty = 0.0;
            for (size_t j = 0; j < size; ++j)
                yty += Y.back()[j] * Y.back()[j];
            if (yty > 1e-14) {
                const double gamma = (1.0 / RHO.back()) / yty;
                for (size_t j = 0; j < size; ++j) {
                    const double range = up[j] - lo[j];
                    q[j] = (float)((double)q[j] * (gamma * range));
                }
            }
        } else {
            for (size_t j = 0; j < size; ++j) {
                const double range = up[j] - lo[j];
                q[j] = (float)((double)q[j] * range);
            }
            const double length = norm2f(q.data(), q.data() + size);
            if (length > 0.0) {
                const double f = tol_length / length;
                for (size_t j = 0; j < size; ++j)
                    q[j] = (float)((double)q[j] * f);
            }
        }
        for (size_t i = 0; i < S.size(); ++i) {
            double yq = 0.0;
            for (size_t j = 0; j < size; ++j)
                yq += Y[i][j] * q[j];
            const double beta = RHO[i] * yq;
            for (size_t j = 0; j < size; ++j)
                q[j] = (float)((double)q[j] + (double)S[i][j] * (alpha[i] - beta));
        }
        x_old = x;
        g_old = g;
        if (!armijo(x, up, lo, q, fun_x, fun)) {
            if (!S.empty()) {
                S.clear();
                Y.clear();
                RHO.clear();
                continue;
            }
            break;
        }
        estimate_change(x, tols, fun_x_ei, fun);
        gradient(tols, fun_x, fun_x_ei, g);
        Vec s_k(size), y_k(size);
        double sty = 0.0;
        for (size_t i = 0; i < size; ++i) {
            s_k[i] = x[i] - x_old[i];
            y_k[i] = g[i] - g_old[i];
            sty += s_k[i] * y_k[i];
        }
        if (sty > 1e-14) {
            if (S.size() == m) {
                S.erase(S.begin());
                Y.erase(Y.begin());
                RHO.erase(RHO.begin());
            }
            S.push_back(std::move(s_k));
            Y.push_back(std::move(y_k));
            RHO.push_back(1.0 / sty);
        }
    }
}

// line_search (numerical/optimization.hpp:272-512): per active axis a grid of
// grid_samples steps (linear spacing for translations, cubic for the rest), then
// a search along the resultant of the best steps; two rounds with a shrinking
// range.  Each grid is one evaluation set.  The reference runs the samples as
// parallel tasks that each check for termination (the caller's check also
// exchanges best points with the other search thread) and then apply their cost;
// here the results are applied task by task in sample order, each after
// is_terminated() and tick() (the time one evaluation takes).
inline void line_search(Vec& x, const float* up, const float* lo, const std::vector<int>& strategy,
                        const BatchFn& fun, double& optimal_value, int grid_samples, const StopFn& is_terminated,
                        const std::function<void()>& tick = [] {})
{
    const size_t size = x.size();
    const double ftol = 0.05;
    const int search_count = 2;
    std::vector<Vec> xi(size, Vec(size, 0.0f));
    for (size_t i = 0; i < size; ++i)
        xi[i][i] = 1.0f;
    Vec p(x);
    for (int iter = 0; iter < search_count; ++iter) {
        if (is_terminated())
            return;
        const double fp = optimal_value;
        std::vector<double> dim_steps(size, 0.0);
        std::vector<int> active;
        std::vector<double> cu(size, 0.0), cl(size, 0.0);
        for (size_t i = 0; i < size; ++i) {
            double bp = 1e10, bn = -1e10;
            bool movable = false;
            for (size_t j = 0; j < size; ++j)
                if (std::abs(xi[i][j]) > 1e-8 && up[j] != lo[j]) {
                    movable = true;
                    double su = (up[j] - p[j]) / xi[i][j];
                    double sl = (lo[j] - p[j]) / xi[i][j];
                    if (su < sl)
                        std::swap(su, sl);
                    bp = std::min(bp, su);
                    bn = std::max(bn, sl);
                }
            if (!movable)
                continue;
            if (bp < 0.0) bp = 0.0;
            if (bn > 0.0) bn = 0.0;
            if (bp > 1e9) bp = 1.0;
            if (bn < -1e9) bn = -1.0;
            const double scale = 0.5 / (iter + 1.0);
            const double u = bp * scale, l = bn * scale;
            if (u - l > 1e-8) {
                active.push_back((int)i);
                cu[i] = u;
                cl[i] = l;
            }
        }
        if (is_terminated())
            return;
        std::vector<double> costs(size * grid_samples, fp), steps(size * grid_samples, 0.0);
        {
            std::vector<Vec> cand;
            std::vector<int> where;  // per task: its candidate, or -1 (zero step)
            for (size_t a = 0; a < active.size(); ++a)
                for (int s = 0; s < grid_samples; ++s) {
                    const int i = active[a];
                    const int li = i * grid_samples + s;
                    const int strat = (i < (int)strategy.size()) ? strategy[i] : 0;
                    double trial;
                    if (strat == 0) {
                        const double st = (cu[i] - cl[i]) / (grid_samples - 1);
                        trial = cl[i] + s * st;
                    } else {
                        const double uu = (double)(s - (grid_samples - 1) / 2.0) / ((grid_samples - 1) / 2.0);
                        const double v = uu * uu * uu;
                        trial = (v > 0.0) ? (v * cu[i]) : (v * -cl[i]);
                    }
                    steps[li] = trial;
                    if (std::abs(trial) < 1e-8) {
                        where.push_back(-1);
                        continue;
                    }
                    Vec t(p);
                    for (size_t j = 0; j < size; ++j)
                        t[j] = std::min<float>(up[j], std::max<float>(lo[j], (float)(p[j] + trial * xi[i][j])));
                    where.push_back((int)cand.size());
                    cand.push_back(std::move(t));
                }
            std::vector<double> r;
            if (!cand.empty())
                r = fun(cand);
            size_t task = 0;
            for (size_t a = 0; a < active.size(); ++a)
                for (int s = 0; s < grid_samples; ++s, ++task) {
                    if (is_terminated())
                        continue;
                    const int k = where[task];
                    if (k < 0)
                        continue;
                    tick();
                    costs[active[a] * grid_samples + s] = r[k];
                    if (r[k] < optimal_value) {
                        optimal_value = r[k];
                        x = cand[k];
                    }
                }
        }
        if (is_terminated())
            return;
        for (size_t a = 0; a < active.size(); ++a) {
            const int i = active[a];
            double best_f = fp;
            int s_min = (grid_samples - 1) / 2;
            for (int s = 0; s < grid_samples; ++s)
                if (costs[i * grid_samples + s] < best_f) {
                    best_f = costs[i * grid_samples + s];
                    s_min = s;
                }
            dim_steps[i] = steps[i * grid_samples + s_min];
        }
        if (is_terminated())
            return;
        Vec dir(size, 0.0f);
        bool moved = false;
        for (size_t i = 0; i < size; ++i) {
            if (std::abs(dim_steps[i]) > 1e-8)
                moved = true;
            for (size_t j = 0; j < size; ++j)
                dir[j] = (float)((double)dir[j] + dim_steps[i] * xi[i][j]);
        }
        if (moved) {
            double bp = 1e10, bn = -1e10;
            bool movable = false;
            for (size_t j = 0; j < size; ++j)
                if (std::abs(dir[j]) > 1e-8 && up[j] != lo[j]) {
                    movable = true;
                    double su = (up[j] - p[j]) / dir[j];
                    double sl = (lo[j] - p[j]) / dir[j];
                    if (su < sl)
                        std::swap(su, sl);
                    bp = std::min(bp, su);
                    bn = std::max(bn, sl);
                }
            if (movable) {
                if (bp < 0.0) bp = 0.0;
                if (bn > 0.0) bn = 0.0;
                if (bp > 1e9) bp = 1.0;
                if (bn < -1e9) bn = -1.0;
                const double st = (bp - bn) / (grid_samples - 1);
                if (st > 1e-8) {
                    std::vector<Vec> cand;
                    std::vector<int> where;
                    for (int s = 0; s < grid_samples; ++s) {
                        const double trial = bn + s * st;
                        if (std::abs(trial) > 1e-8) {
                            Vec t(p);
                            for (size_t j = 0; j < size; ++j)
                                t[j] = std::min<float>(up[j], std::max<float>(lo[j], (float)(p[j] + trial * dir[j])));
                            where.push_back((int)cand.size());
                            cand.push_back(std::move(t));
                        } else
                            where.push_back(-1);
                    }
                    std::vector<double> r;
                    if (!cand.empty())
                        r = fun(cand);
                    for (int s = 0; s < grid_samples; ++s) {
                        if (is_terminated())
                            continue;
                        const int k = where[s];
                        if (k < 0)
                            continue;
                        tick();
                        if (r[k] < optimal_value) {
                            optimal_value = r[k];
                            x = cand[k];
                        }
                    }
                }
            }
        }
        if (is_terminated())
            return;
        p = x;
        if (2.0 * (fp - optimal_value) <= ftol * (std::abs(fp) + std::abs(optimal_value)) + 1e-10)
            break;
    }
}

}  // namespace opt
}  // namespace regb
