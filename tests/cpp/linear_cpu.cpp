// Test program: the library's affine search (the LinearRunner of
// tipl_b200/csrc/linear_runner.h, the bounds of runner_state_from_param, the
// mask-moment start) driven by the oracle's CPU costs instead of the device.  It
// replays, on the host, exactly the decisions linear_register makes on the GPU, so
// the optimiser's host logic can be checked against the reference's linear() without
// a GPU.  The oracle is the checker here; nothing in the library calls it.
//
//   linear_cpu <w> <h> <d> <from.u8> <w> <h> <d> <to.u8> <cost: 0 corr | 1 MI | 2 MI32>
//              <bound: 0 reg | 1 narrow | 2 large> <out.bin> [12 initial parameters]
// out.bin: float cost, float arg[12], int64 evals.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <thread>
#include <vector>
#include "linear_runner.h"
#include "mask_init.h"
#include "../../oracle/oracle.h"

using namespace regb;

static std::vector<uint8_t> load(const char* path, size_t n)
{
    std::vector<uint8_t> v(n);
    std::ifstream f(path, std::ios::binary);
    f.read((char*)v.data(), (std::streamsize)n);
    if (!f) {
        std::fprintf(stderr, "cannot read %s\n", path);
        std::exit(2);
    }
    return v;
}

static MaskCounts host_counts(const std::vector<uint8_t>& v, const int* dim)
{
    MaskCounts c;
    c.w = dim[0];
    c.h = dim[1];
    c.d = dim[2];
    c.xy.assign((size_t)c.w * c.h, 0);
    c.xz.assign((size_t)c.w * c.d, 0);
    c.yz.assign((size_t)c.h * c.d, 0);
    size_t i = 0;
    for (int z = 0; z < c.d; ++z)
        for (int y = 0; y < c.h; ++y)
            for (int x = 0; x < c.w; ++x, ++i)
                if (v[i]) {
                    ++c.xy[(size_t)y * c.w + x];
                    ++c.xz[(size_t)z * c.w + x];
                    ++c.yz[(size_t)z * c.h + y];
                }
    return c;
}

struct HostLevel {
    std::vector<uint8_t> from, to;
};

int main(int argc, char** argv)
{
    if (argc != 12 && argc != 24) {
        std::fprintf(stderr, "usage: linear_cpu w h d from w h d to cost bound out [arg x 12]\n");
        return 2;
    }
    int fdim[3] = {atoi(argv[1]), atoi(argv[2]), atoi(argv[3])};
    int tdim[3] = {atoi(argv[5]), atoi(argv[6]), atoi(argv[7])};
    const int cost_type = atoi(argv[9]);
    std::vector<uint8_t> from = load(argv[4], (size_t)fdim[0] * fdim[1] * fdim[2]);
    std::vector<uint8_t> to = load(argv[8], (size_t)tdim[0] * tdim[1] * tdim[2]);
    float from_vs[3] = {1, 1, 1}, to_vs[3] = {1, 1, 1};
    float arg[12] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 0, 0, 0};
    if (argc == 24)
        for (int k = 0; k < 12; ++k)
            arg[k] = (float)atof(argv[12 + k]);
    regb_linear_param p;
    p.reg_type = REGB_REG_AFFINE;
    p.cost_type = cost_type;
    p.bound = atoi(argv[10]);
    p.search_count = 16;

    // the mask start of linear_register
    float sur[12], run_to_vs[3];
    bool masked = false;
    {
        MaskCounts cf = host_counts(from, fdim), ct = host_counts(to, tdim);
        if (p.bound != REGB_BOUND_NARROW && has_mask(cf) && has_mask(ct)) {
            masked = true;
            estimate_affine_param(cf, from_vs, ct, to_vs, sur);
            for (int i = 0; i < 3; ++i) {
                run_to_vs[i] = to_vs[i] / std::max<float>(sur[6 + i], 0.01f);
                sur[6 + i] = 1.0f;
            }
        } else {
            std::copy(arg, arg + 12, sur);
            std::copy(to_vs, to_vs + 3, run_to_vs);
        }
    }
    regb_runner_state s;
    runner_state_from_param(fdim, from_vs, tdim, run_to_vs, sur, p, s);

    opt::Vec a(sur, sur + 12);
    LinearRunner R(a);
    R.cost_type = s.cost_type;
    R.arg_upper.assign(s.arg_upper, s.arg_upper + 12);
    R.arg_lower.assign(s.arg_lower, s.arg_lower + 12);
    R.reg_list.assign(s.reg_list, s.reg_list + s.n_reg);
    R.search_count = s.search_count;
    R.precision = s.precision;
    R.max_iterations = s.max_iterations;
    std::vector<HostLevel> host(1);
    host[0].from = from;
    host[0].to = to;
    LinearRunner::Level L0;
    for (int i = 0; i < 3; ++i) {
        L0.fd[i] = fdim[i];
        L0.td[i] = tdim[i];
        L0.fvs[i] = from_vs[i];
        L0.tvs[i] = run_to_vs[i];
    }
    R.levels.push_back(L0);
    for (;;) {
        const LinearRunner::Level c = R.levels.back();
        if (!((double)c.fd[0] * c.fd[1] * c.fd[2] > std::pow(96, 3)))
            break;
        LinearRunner::Level n;
        for (int i = 0; i < 3; ++i) {
            n.fd[i] = (c.fd[i] + 1) / 2;
            n.td[i] = (c.td[i] + 1) / 2;
            n.fvs[i] = c.fvs[i] * 2.0f;
            n.tvs[i] = c.tvs[i] * 2.0f;
        }
        HostLevel hl;
        hl.from.resize((size_t)n.fd[0] * n.fd[1] * n.fd[2]);
        hl.to.resize((size_t)n.td[0] * n.td[1] * n.td[2]);
        orc_downsample_u8(host.back().from.data(), c.fd, hl.from.data());
        orc_downsample_u8(host.back().to.data(), c.td, hl.to.data());
        host.push_back(std::move(hl));
        R.levels.push_back(n);
    }
    for (size_t k = 0; k < R.levels.size(); ++k) {
        R.levels[k].from = host[k].from.data();
        R.levels[k].to = host[k].to.data();
    }
    R.eval = [&](int level, const float* T, int n) {
        const LinearRunner::Level& L = R.levels[level];
        std::vector<double> c(n);
        std::vector<std::thread> th;
        const int nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                for (int k = t; k < n; k += nt)
                    c[k] = cost_type == REGB_COST_MI     ? orc_mi_cost_u8(L.from, L.fd, L.to, L.td, T + 12 * k)
                           : cost_type == REGB_COST_MI32 ? orc_mi32_cost_u8(L.from, L.fd, L.to, L.td, T + 12 * k, nullptr)
                                                         : orc_corr_cost_u8(L.from, L.fd, L.to, L.td, T + 12 * k);
            });
        for (auto& t : th)
            t.join();
        return c;
    };
    R.on_stage = [](int reg, double c, const opt::Vec& v) {
        std::fprintf(stderr, "reg:%d cost:%g t:%.2f %.2f %.2f r:%.3f %.3f %.3f s:%.2f %.2f %.2f a:%.3f %.3f %.3f\n", reg, c,
                     v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10], v[11]);
    };
    const double cost = s.multi_resolution ? R.run_optimize_mr(0) : R.run_optimize(0, 0);
    float out_arg[12];
    if (masked) {
        float T[12];
        affine_to_matrix(a.data(), fdim, from_vs, tdim, run_to_vs, T);
        matrix_to_affine_param(T, fdim, from_vs, tdim, to_vs, out_arg);
    } else
        std::copy(a.begin(), a.end(), out_arg);
    std::FILE* f = std::fopen(argv[11], "wb");
    const float fc = (float)cost;
    const long long ev = R.evals;
    std::fwrite(&fc, 4, 1, f);
    std::fwrite(out_arg, 4, 12, f);
    std::fwrite(&ev, 8, 1, f);
    std::fclose(f);
    std::printf("masked %d cost %.6f evals %lld\n", masked ? 1 : 0, fc, ev);
    return 0;
}
