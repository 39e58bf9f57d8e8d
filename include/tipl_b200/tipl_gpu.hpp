// Drop-in GPU implementation of TIPL's registration hot path, on libregb200.so.
//
// TIPL declares two out-of-line templates for host compilers and expects a CUDA
// translation unit to instantiate them (reg/linear.hpp:605-610 with
// reg/linear_cu.hpp:1-19; reg/cdm.hpp:525-532 with reg/cdm_cu.hpp:1-19):
//
//   tipl::reg::linear_reg_imp<out, mr, unsigned char, 3>(std::true_type, runner, cost_type, terminated)
//   tipl::reg::cdm_cuda<out, T, dim>(It, Is, d, terminated, param)
//
// This header defines both.  Include it in ONE translation unit after the TIPL
// headers, compile that unit with -DTIPL_USE_CUDA by the host compiler (no nvcc),
// and link libregb200.so.  tipl::reg::linear and tipl::reg::cdm_common then run
// their GPU branch here, with their signatures, argument meaning and error
// behaviour unchanged: CUDA failures throw std::runtime_error from linear, and
// make cdm_cuda return false.
//
// Coverage: every image pair of linear's lists and every modality pair of
// cdm_common's lists; linear on 3-D uint8 volumes (the instantiations of
// reg/linear_cu.hpp); cdm on 3-D uint8 or float volumes and on 2-D uint8 images
// (cdm_cuda<out, unsigned char, 2>, the 2-D instantiation of reg/cdm_cu.hpp:12-17).
#pragma once
#include <algorithm>
#include <atomic>
#include <chrono>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>
#include "../regb200.h"

namespace tipl_b200_detail {

// Mirrors a TIPL `bool& terminated` into the int flag the library polls.
class TerminateMirror {
public:
    explicit TerminateMirror(bool& t) : t_(t), flag_(t ? 1 : 0)
    {
        th_ = std::thread([this] {
            while (!done_.load()) {
                if (t_)
                    flag_ = 1;
                std::this_thread::sleep_for(std::chrono::milliseconds(2));
            }
        });
    }
    ~TerminateMirror()
    {
        done_ = true;
        th_.join();
    }
    volatile const int* flag() const { return &flag_; }

private:
    bool& t_;
    volatile int flag_;
    std::atomic<bool> done_{false};
    std::thread th_;
};

template <typename image_type>
regb_volume host_volume(const image_type& I, int dtype)
{
    regb_volume v;
    v.ptr = const_cast<void*>(static_cast<const void*>(&*I.begin()));
    v.dim[0] = int(I.width());
    v.dim[1] = int(I.height());
    if constexpr (image_type::dimension == 3)
        v.dim[2] = int(I.depth());
    else
        v.dim[2] = 1;  // a 2-D image is (w, h, 1)
    v.dtype = dtype;
    v.location = REGB_HOST;
    return v;
}

}  // namespace tipl_b200_detail

namespace tipl {
namespace reg {

template <typename out_type, bool mr, typename value_type, int dim>
float linear_reg_imp(std::true_type, std::shared_ptr<tipl::reg::linear_reg_runner<dim, value_type, out_type> > reg,
                     tipl::reg::cost_type cost_type, bool& terminated)
{
    static_assert(dim == 3, "the GPU registration path is 3-D");
    static_assert(std::is_same<value_type, unsigned char>::value, "tipl::reg::linear takes uint8 volumes");
    regb_runner_state s{};
    for (int i = 0; i < 12; ++i) {
        s.arg_upper[i] = reg->arg_upper[i];
        s.arg_lower[i] = reg->arg_lower[i];
    }
    s.n_reg = int(reg->reg_list.size() < 8 ? reg->reg_list.size() : 8);
    for (int i = 0; i < s.n_reg; ++i)
        s.reg_list[i] = int(reg->reg_list[i]);
    s.search_count = reg->search_count;
    s.multi_resolution = mr ? 1 : 0;
    s.cost_type = (cost_type == tipl::reg::mutual_info) ? REGB_COST_MI : REGB_COST_CORR;
    s.precision = reg->precision;
    s.max_iterations = int(reg->max_iterations);
    // every image pair of the runner's lists (run_optimize makes min(from, to) cost functions)
    std::vector<regb_volume> from, to;
    for (size_t i = 0; i < std::min(reg->from.size(), reg->to.size()); ++i) {
        from.push_back(tipl_b200_detail::host_volume(reg->from[i], REGB_U8));
        to.push_back(tipl_b200_detail::host_volume(reg->to[i], REGB_U8));
    }
    const float fvs[3] = {reg->from_vs[0], reg->from_vs[1], reg->from_vs[2]};
    const float tvs[3] = {reg->to_vs[0], reg->to_vs[1], reg->to_vs[2]};
    float arg[12];
    for (int i = 0; i < 12; ++i)
        arg[i] = reg->arg_min[i];
    float cost = 0.0f;
    long long evals = 0;
    regb_status st;
    {
        tipl_b200_detail::TerminateMirror mirror(terminated);
        st = regb_linear_run_multi(from.data(), fvs, to.data(), tvs, (int)from.size(), arg, &s, mirror.flag(), &cost,
                                   &evals);
    }
    if (st != REGB_OK && st != REGB_CANCELLED)
        throw std::runtime_error(std::string("regb_linear_run_multi: ") + regb_last_error());
    for (int i = 0; i < 12; ++i)
        reg->arg_min[i] = arg[i];
    reg->count += (unsigned int)evals;
    return cost;
}

template <typename out_type, typename value_type, int dim>
bool cdm_cuda(const std::vector<tipl::const_pointer_image<dim, value_type> >& It,
              const std::vector<tipl::const_pointer_image<dim, value_type> >& Is, tipl::image<dim, tipl::vector<dim> >& d,
              bool& terminated, const cdm_param& param)
{
    static_assert(dim == 2 || dim == 3, "cdm registers 2-D or 3-D images");
    static_assert(std::is_same<value_type, unsigned char>::value || std::is_same<value_type, float>::value,
                  "cdm takes uint8 or float volumes");
    static_assert(dim == 3 || std::is_same<value_type, unsigned char>::value,
                  "the 2-D GPU cdm takes uint8 images (cdm_cuda<out, unsigned char, 2>)");
    if (It.empty() || Is.empty())
        return false;
    const int dtype = std::is_same<value_type, float>::value ? REGB_F32 : REGB_U8;
    // every modality pair of the lists (cdm_common has made them one length)
    const size_t nmod = std::min(It.size(), Is.size());
    std::vector<regb_volume> vt, vs;
    for (size_t i = 0; i < nmod; ++i) {
        vt.push_back(tipl_b200_detail::host_volume(It[i], dtype));
        vs.push_back(tipl_b200_detail::host_volume(Is[i], dtype));
    }
    d.resize(It[0].shape());
    regb_field f;
    f.ptr = &d[0][0];  // tipl::vector<dim> is dim packed floats
    f.dim[0] = vt[0].dim[0];
    f.dim[1] = vt[0].dim[1];
    f.dim[2] = vt[0].dim[2];
    f.location = REGB_HOST;
    regb_cdm_param p;
    regb_cdm_param_default(&p);
    p.resolution = param.resolution;
    p.speed = param.speed;
    p.smoothing = param.smoothing;
    p.min_dimension = param.min_dimension;
    p.gradient_type = param.gradient_type.empty() ? 'r' : param.gradient_type[0];
    regb_status st;
    {
        tipl_b200_detail::TerminateMirror mirror(terminated);
        if constexpr (dim == 2)
            st = regb_cdm2d_multi(vt.data(), vs.data(), (int)nmod, &f, &p, param.gradient_type.c_str(), mirror.flag());
        else
            st = regb_cdm_multi(vt.data(), vs.data(), (int)nmod, &f, &p, param.gradient_type.c_str(), mirror.flag());
    }
    if constexpr (!std::is_void<out_type>::value) {
        if (st != REGB_OK && st != REGB_FALSE && st != REGB_CANCELLED)
            out_type() << "cdm: " << regb_last_error();
    }
    return st == REGB_OK || st == REGB_CANCELLED;  // a terminated run still returns its field, as cdm() does
}

}  // namespace reg
}  // namespace tipl
