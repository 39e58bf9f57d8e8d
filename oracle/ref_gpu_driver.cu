// Test infrastructure only: the reference's own CUDA path (TIPL's linear_reg_imp /
// cdm_cuda instantiated by nvcc, as reg/linear_cu.hpp and reg/cdm_cu.hpp do) behind
// extern "C" entry points, built into oracle/_ref/libtipl_ref_gpu.so by oracle/Makefile
// from the reference headers where they lie.  It is timed by bench.py as a secondary
// "reference GPU" figure; nothing in the product path links or loads it.
#include <algorithm>
#include <vector>
#include "reg/linear.hpp"
#include "reg/cdm.hpp"

namespace tipl::reg {
template float linear_reg_imp<void, true, unsigned char, 3>(
    std::true_type, std::shared_ptr<tipl::reg::linear_reg_runner<3, unsigned char, void>>, tipl::reg::cost_type,
    bool&);
template float linear_reg_imp<void, false, unsigned char, 3>(
    std::true_type, std::shared_ptr<tipl::reg::linear_reg_runner<3, unsigned char, void>>, tipl::reg::cost_type,
    bool&);
template bool cdm_cuda<void, unsigned char, 3>(const std::vector<tipl::const_pointer_image<3, unsigned char>>&,
                                               const std::vector<tipl::const_pointer_image<3, unsigned char>>&,
                                               tipl::image<3, tipl::vector<3>>&, bool&, const cdm_param&);
}  // namespace tipl::reg

namespace {
using u8 = unsigned char;
tipl::shape<3> shp(const int* d) { return tipl::shape<3>(d[0], d[1], d[2]); }
tipl::const_pointer_image<3, u8> cview(const u8* p, const int* d) { return tipl::const_pointer_image<3, u8>(p, shp(d)); }
}  // namespace

extern "C" {

void tiplrefgpu_set_threads(int n) { tipl::max_thread_count = std::max(1, n); }

// tipl::reg::linear<void>(..., param.cuda = true) (reg/linear.hpp:622-700) taking the
// reference's GPU runner; returns the final cost.
float tiplrefgpu_linear(const u8* from, const int* from_dim, const float* from_vs, const u8* to, const int* to_dim,
                        const float* to_vs, float* arg_inout, int reg_type, int cost_type)
{
    tipl::affine_param<float, 3> arg(arg_inout);
    tipl::reg::linear_reg_param p;
    p.reg_type = tipl::reg::reg_type(reg_type);
    p.cost_type = tipl::reg::cost_type(cost_type);
    p.cuda = true;
    bool terminated = false;
    float c = tipl::reg::linear<void>(std::vector<tipl::const_pointer_image<3, u8>>{cview(from, from_dim)},
                                      tipl::vector<3>(from_vs),
                                      std::vector<tipl::const_pointer_image<3, u8>>{cview(to, to_dim)},
                                      tipl::vector<3>(to_vs), arg, p, terminated);
    std::copy(arg.begin(), arg.end(), arg_inout);
    return c;
}

// tipl::reg::cdm_common<void, u8, 3>(..., cuda = true) (reg/cdm.hpp:534-558)
int tiplrefgpu_cdm(const u8* It, const u8* Is, const int* dim, float* dis_out, float resolution, float speed,
                   float smoothing, unsigned int min_dimension)
{
    tipl::reg::cdm_param p;
    p.resolution = resolution;
    p.speed = speed;
    p.smoothing = smoothing;
    p.min_dimension = min_dimension;
    tipl::image<3, tipl::vector<3>> d;
    bool terminated = false;
    bool ok = tipl::reg::cdm_common<void>(std::vector<tipl::const_pointer_image<3, u8>>{cview(It, dim)},
                                          std::vector<tipl::const_pointer_image<3, u8>>{cview(Is, dim)}, d, terminated,
                                          p, true);
    if (ok && d.size() == size_t(dim[0]) * dim[1] * dim[2])
        std::copy(&d[0][0], &d[0][0] + 3 * d.size(), dis_out);
    return ok ? 1 : 0;
}

}  // extern "C"
