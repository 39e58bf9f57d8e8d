// Drop-in check: the reference's own tipl::reg::linear and tipl::reg::cdm_common,
// compiled by the host compiler with -DTIPL_USE_CUDA, run their GPU branch through
// include/tipl_b200/tipl_gpu.hpp (libregb200.so) or their CPU branch.
//
//   tipl_drop_in linear|cdm gpu|cpu w h d fixed.u8 moving.u8 out.bin
//   tipl_drop_in cdm2 gpu|cpu w h d fixed.u8 moving.u8 out.bin fixed2.u8 moving2.u8 gradient_types
//   tipl_drop_in linear2 gpu|cpu w h d fixed.u8 moving.u8 out.bin fixed2.u8 moving2.u8
//   tipl_drop_in cdm2d gpu|cpu w h 1 fixed.u8 moving.u8 out.bin resolution min_dimension gradient_types
//                [fixed2.u8 moving2.u8]
// linear writes cost (float) + 12 params; cdm writes ok (int32) + the field; cdm2 runs
// cdm_common on the two-modality lists {fixed, fixed2} / {moving, moving2} at
// resolution 1 with the given cdm_param::gradient_type string; linear2 runs linear on
// the two-pair lists (mm_reg's mm_linear); cdm2d runs cdm_common<void, unsigned char, 2>
// on 2-D images (one or two modality pairs) and writes ok (int32) + the vector<2> field.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>
#include "reg/linear.hpp"
#include "reg/cdm.hpp"
#include "tipl_b200/tipl_gpu.hpp"

static std::vector<unsigned char> read_all(const char* p, size_t n)
{
    std::vector<unsigned char> v(n);
    std::ifstream f(p, std::ios::binary);
    f.read((char*)v.data(), (std::streamsize)n);
    if (!f)
        throw std::runtime_error(std::string("cannot read ") + p);
    return v;
}

int main(int argc, char** argv)
{
    const std::string what = argc > 1 ? argv[1] : "";
    if (what == "cdm2d") {
        if (argc != 12 && argc != 14) {
            std::fprintf(stderr, "usage: %s cdm2d gpu|cpu w h 1 fixed moving out res min_dim types [fixed2 moving2]\n",
                         argv[0]);
            return 2;
        }
        const bool gpu = std::string(argv[2]) == "gpu";
        const tipl::shape<2> sh(std::atoi(argv[3]), std::atoi(argv[4]));
        std::vector<std::vector<unsigned char>> bufs;
        std::vector<tipl::const_pointer_image<2, unsigned char>> F, M;
        for (int k = 6; k < argc; k += (k == 7 ? 5 : 1)) {
            bufs.push_back(read_all(argv[k], sh.size()));
            (bufs.size() % 2 ? F : M).push_back(tipl::const_pointer_image<2, unsigned char>(bufs.back().data(), sh));
        }
        tipl::reg::cdm_param param;
        param.resolution = (float)std::atof(argv[9]);
        param.min_dimension = (unsigned int)std::atoi(argv[10]);
        param.gradient_type = std::string(argv[11]) == "-" ? "" : argv[11];
        tipl::image<2, tipl::vector<2>> dis;
        bool terminated = false;
        bool ok = tipl::reg::cdm_common<void, unsigned char, 2>(F, M, dis, terminated, param, gpu);
        std::ofstream out(argv[8], std::ios::binary);
        int32_t okv = ok ? 1 : 0;
        out.write((const char*)&okv, 4);
        if (ok)
            out.write((const char*)&dis[0][0], (std::streamsize)(dis.size() * 8));
        std::printf("cdm2d %s ok %d\n", gpu ? "gpu" : "cpu", okv);
        return 0;
    }
    if (argc != (what == "cdm2" ? 12 : what == "linear2" ? 11 : 9)) {
        std::fprintf(stderr, "usage: %s linear|cdm|cdm2 gpu|cpu w h d fixed moving out [fixed2 moving2 types]\n",
                     argv[0]);
        return 2;
    }
    const bool gpu = std::string(argv[2]) == "gpu";
    const tipl::shape<3> sh(std::atoi(argv[3]), std::atoi(argv[4]), std::atoi(argv[5]));
    auto fixed = read_all(argv[6], sh.size());
    auto moving = read_all(argv[7], sh.size());
    tipl::const_pointer_image<3, unsigned char> F(fixed.data(), sh), M(moving.data(), sh);
    std::ofstream out(argv[8], std::ios::binary);
    bool terminated = false;
    if (what == "linear2") {
        auto fixed2 = read_all(argv[9], sh.size());
        auto moving2 = read_all(argv[10], sh.size());
        tipl::const_pointer_image<3, unsigned char> F2(fixed2.data(), sh), M2(moving2.data(), sh);
        tipl::affine_param<float, 3> arg;
        tipl::reg::linear_reg_param param;
        param.cuda = gpu;
        float cost = tipl::reg::linear<void>(std::vector<tipl::const_pointer_image<3, unsigned char>>{F, F2},
                                             tipl::vector<3>(1, 1, 1),
                                             std::vector<tipl::const_pointer_image<3, unsigned char>>{M, M2},
                                             tipl::vector<3>(1, 1, 1), arg, param, terminated);
        out.write((const char*)&cost, 4);
        out.write((const char*)arg.data(), 48);
        std::printf("linear2 %s cost %.6f\n", gpu ? "gpu" : "cpu", cost);
    } else if (what == "linear") {
        tipl::affine_param<float, 3> arg;
        tipl::reg::linear_reg_param param;
        param.cuda = gpu;
        float cost = tipl::reg::linear<void>(std::vector<tipl::const_pointer_image<3, unsigned char>>{F},
                                             tipl::vector<3>(1, 1, 1),
                                             std::vector<tipl::const_pointer_image<3, unsigned char>>{M},
                                             tipl::vector<3>(1, 1, 1), arg, param, terminated);
        out.write((const char*)&cost, 4);
        out.write((const char*)arg.data(), 48);
        std::printf("linear %s cost %.6f\n", gpu ? "gpu" : "cpu", cost);
    } else if (what == "cdm2") {
        auto fixed2 = read_all(argv[9], sh.size());
        auto moving2 = read_all(argv[10], sh.size());
        tipl::const_pointer_image<3, unsigned char> F2(fixed2.data(), sh), M2(moving2.data(), sh);
        tipl::reg::cdm_param param;
        param.resolution = 1.0f;
        param.gradient_type = argv[11];
        tipl::image<3, tipl::vector<3>> dis;
        bool ok = tipl::reg::cdm_common<void, unsigned char, 3>({F, F2}, {M, M2}, dis, terminated, param, gpu);
        int32_t okv = ok ? 1 : 0;
        out.write((const char*)&okv, 4);
        if (ok)
            out.write((const char*)&dis[0][0], (std::streamsize)(dis.size() * 12));
        std::printf("cdm2 %s ok %d\n", gpu ? "gpu" : "cpu", okv);
    } else {
        tipl::image<3, tipl::vector<3>> dis;
        bool ok = tipl::reg::cdm_common<void, unsigned char, 3>({F}, {M}, dis, terminated, tipl::reg::cdm_param(), gpu);
        int32_t okv = ok ? 1 : 0;
        out.write((const char*)&okv, 4);
        if (ok)
            out.write((const char*)&dis[0][0], (std::streamsize)(dis.size() * 12));
        std::printf("cdm %s ok %d\n", gpu ? "gpu" : "cpu", okv);
    }
    return 0;
}
