// Test infrastructure only: a thin extern "C" driver over the reference library's
// own header-only C++ implementation (TIPL).  It is compiled from the reference
// headers where they lie (see oracle/Makefile) into oracle/_ref/libtipl_ref.so and
// is used (1) to pin the plain-C restatement in oracle/oracle_core.h, (2) to make
// the golden fixtures under tests/golden/, and (3) as the timed CPU baseline.
// Nothing in the product path links or loads it.
//
// Every entry point forwards to exactly one reference routine; the routine and its
// file:line are named beside each function.
#include <zlib.h>  // before the reference's headers: io/gz_stream.hpp is built only with zlib
#include <map>  // io/gz_stream.hpp uses std::map without including it
#include <algorithm>
#include <vector>
#include <cstring>
#include <cstdint>
#include "io/gz_stream.hpp"
#include "io/nifti.hpp"
#include "reg/linear.hpp"
#include "reg/cdm.hpp"
#include "reg/mm_reg.hpp"

namespace {
using u8 = unsigned char;
using vec3 = tipl::vector<3>;
tipl::shape<3> shp(const int* d) { return tipl::shape<3>(d[0], d[1], d[2]); }
tipl::transformation_matrix<float, 3> to_matrix(const float* T)
{
    tipl::transformation_matrix<float, 3> M;
    std::copy(T, T + 12, M.begin());
    return M;
}
template <typename T>
tipl::const_pointer_image<3, T> cview(const T* p, const int* d) { return tipl::const_pointer_image<3, T>(p, shp(d)); }
tipl::image<3, vec3> field_in(const float* p, const int* d)
{
    tipl::image<3, vec3> f(shp(d));
    std::memcpy(&f[0][0], p, sizeof(float) * 3 * f.size());
    return f;
}
void field_out(const tipl::image<3, vec3>& f, float* p) { std::memcpy(p, &f[0][0], sizeof(float) * 3 * f.size()); }
}  // namespace

// cdm_common<void,T,3> over a list of nmod modalities (reg/cdm.hpp:418-435, 534-558):
// gtypes is cdm_param::gradient_type (modality i uses gtypes[i], 'r' past its end).
template <typename T>
static int cdm_multi(const T* const* It, const T* const* Is, int nmod, const int* dim, float* dis_out,
                     float resolution, float speed, float smoothing, unsigned int min_dimension, const char* gtypes)
{
    tipl::reg::cdm_param p;
    p.resolution = resolution;
    p.speed = speed;
    p.smoothing = smoothing;
    p.min_dimension = min_dimension;
    p.gradient_type = gtypes ? gtypes : "";
    std::vector<tipl::const_pointer_image<3, T> > lt, ls;
    for (int i = 0; i < nmod; ++i) {
        lt.push_back(cview(It[i], dim));
        ls.push_back(cview(Is[i], dim));
    }
    tipl::image<3, vec3> dis;
    bool terminated = false;
    bool ok = tipl::reg::cdm_common<void, T, 3>(lt, ls, dis, terminated, p, false);
    if (ok)
        field_out(dis, dis_out);
    return ok ? 1 : 0;
}
extern "C" {

int tiplref_sizeof_vec3(void) { return int(sizeof(vec3)); }

// tipl::max_thread_count (mt.hpp:89): threads used by every par_for.
void tiplref_set_threads(int n) { tipl::max_thread_count = std::max(1, n); }
int tiplref_get_threads(void) { return tipl::max_thread_count; }

// transformation_matrix(affine_param, from, from_vs, to, to_vs)  (numerical/transformation.hpp:636-701)
void tiplref_affine_to_matrix(const float* param, const int* from_dim, const float* from_vs,
                              const int* to_dim, const float* to_vs, float* T)
{
    tipl::affine_param<float, 3> a(param);
    tipl::transformation_matrix<float, 3> M(a, shp(from_dim), tipl::vector<3>(from_vs), shp(to_dim),
                                            tipl::vector<3>(to_vs));
    std::copy(M.begin(), M.end(), T);
}

// transformation_matrix::inverse (numerical/transformation.hpp:820-832)
int tiplref_matrix_inverse(float* T)
{
    auto M = to_matrix(T);
    bool ok = M.inverse();
    std::copy(M.begin(), M.end(), T);
    return ok ? 1 : 0;
}

// resample<linear>(from, to, trans)  (numerical/resampling.hpp:1239-1269)
void tiplref_resample_u8(const u8* from, const int* from_dim, u8* to, const int* to_dim, const float* T)
{
    tipl::image<3, u8> out(shp(to_dim));
    tipl::resample<tipl::linear>(cview(from, from_dim), out, to_matrix(T));
    std::copy(out.begin(), out.end(), to);
}
void tiplref_resample_f32(const float* from, const int* from_dim, float* to, const int* to_dim, const float* T)
{
    tipl::image<3, float> out(shp(to_dim));
    tipl::resample<tipl::linear>(cview(from, from_dim), out, to_matrix(T));
    std::copy(out.begin(), out.end(), to);
}

// get_mutual_info (reg/linear.hpp:138-146): 256x256 joint histogram, row = template bin.
void tiplref_mi_hist(const u8* from, const int* from_dim, const u8* to, const int* to_dim, const float* T,
                     int32_t* hist)
{
    auto h = tipl::reg::get_mutual_info(cview(to, to_dim), cview(from, from_dim), to_matrix(T));
    std::copy(h.begin(), h.end(), hist);
}

// mutual_information<3>::operator() (reg/linear.hpp:181-202)
double tiplref_mi_cost(const u8* from, const int* from_dim, const u8* to, const int* to_dim, const float* T)
{
    tipl::reg::mutual_information<3> mi;
    return mi(cview(from, from_dim), cview(to, to_dim), to_matrix(T));
}

// correlation::operator() (reg/linear.hpp:23-37)
double tiplref_corr_cost(const u8* from, const int* from_dim, const u8* to, const int* to_dim, const float* T)
{
    tipl::reg::correlation c;
    return c(cview(from, from_dim), cview(to, to_dim), to_matrix(T));
}

// compose_displacement (numerical/dif.hpp:90-107)
void tiplref_compose_u8(const u8* Is, const int* dim, const float* dis, u8* Js)
{
    auto d = field_in(dis, dim);
    tipl::image<3, u8> out;
    tipl::compose_displacement(cview(Is, dim), d, out);
    std::copy(out.begin(), out.end(), Js);
}
void tiplref_compose_f32(const float* Is, const int* dim, const float* dis, float* Js)
{
    auto d = field_in(dis, dim);
    tipl::image<3, float> out;
    tipl::compose_displacement(cview(Is, dim), d, out);
    std::copy(out.begin(), out.end(), Js);
}

// cdm_get_gradient (reg/cdm.hpp:84-106), gradient_type 'r' or 'd'
float tiplref_cdm_gradient_u8(const u8* Js, const u8* It, const int* dim, float* new_d, int gradient_type)
{
    tipl::image<3, vec3> nd;
    float c = tipl::reg::cdm_get_gradient(cview(Js, dim), cview(It, dim), nd, (unsigned char)gradient_type);
    field_out(nd, new_d);
    return c;
}
float tiplref_cdm_gradient_f32(const float* Js, const float* It, const int* dim, float* new_d, int gradient_type)
{
    tipl::image<3, vec3> nd;
    float c = tipl::reg::cdm_get_gradient(cview(Js, dim), cview(It, dim), nd, (unsigned char)gradient_type);
    field_out(nd, new_d);
    return c;
}

// cdm_solve_poisson (reg/cdm.hpp:158-198), in place
void tiplref_cdm_poisson(float* new_d, const int* dim)
{
    auto nd = field_in(new_d, dim);
    bool terminated = false;
    tipl::reg::cdm_solve_poisson(nd, terminated);
    field_out(nd, new_d);
}

// cdm_max_displacement_length (reg/cdm.hpp:269-284)
float tiplref_cdm_max_len(const float* new_d, const int* dim)
{
    auto nd = field_in(new_d, dim);
    return tipl::reg::cdm_max_displacement_length(nd);
}

// accumulate_displacement (numerical/dif.hpp:166-186): new_d <- cur_d o new_d
void tiplref_accumulate(const float* cur_d, float* new_d, const int* dim)
{
    auto cd = field_in(cur_d, dim);
    auto nd = field_in(new_d, dim);
    tipl::accumulate_displacement(cd, nd);
    field_out(nd, new_d);
}

// cdm_smooth (reg/cdm.hpp:328-342): dd <- blend(d)
void tiplref_cdm_smooth(const float* d, float* dd, const int* dim, float smoothing)
{
    auto src = field_in(d, dim);
    tipl::image<3, vec3> out(shp(dim));
    tipl::reg::cdm_smooth(src, out, smoothing);
    field_out(out, dd);
}

// downsample_with_padding (numerical/resampling.hpp:605-632): out shape (d+1)/2
void tiplref_downsample_u8(const u8* in, const int* dim, u8* out)
{
    tipl::image<3, u8> o;
    tipl::downsample_with_padding(cview(in, dim), o);
    std::copy(o.begin(), o.end(), out);
}
void tiplref_downsample_f32(const float* in, const int* dim, float* out)
{
    tipl::image<3, float> o;
    tipl::downsample_with_padding(cview(in, dim), o);
    std::copy(o.begin(), o.end(), out);
}

// best_d *= 2; upsample_with_padding(best_d, shape) (reg/cdm.hpp:402-403, numerical/resampling.hpp:849-859,885-891)
void tiplref_upsample_field_x2(const float* in, const int* in_dim, float* out, const int* out_dim)
{
    auto f = field_in(in, in_dim);
    f *= 2.0f;
    tipl::upsample_with_padding(f, shp(out_dim));
    field_out(f, out);
}

// histogram(from, from_hist, 0, 255, 256) (numerical/basic_op.hpp:1293-1311)
void tiplref_histogram_u8(const u8* in, const int* dim, int32_t* hist)
{
    std::vector<int32_t> h;
    tipl::histogram(cview(in, dim), h, (u8)0, (u8)255, 256);
    std::copy(h.begin(), h.end(), hist);
}

// cdm_common<void,T,3>(It, Is, dis, terminated, param, cuda=false) (reg/cdm.hpp:534-558)
int tiplref_cdm_u8(const u8* It, const u8* Is, const int* dim, float* dis_out, float resolution, float speed,
                   float smoothing, unsigned int min_dimension)
{
    tipl::reg::cdm_param p;
    p.resolution = resolution;
    p.speed = speed;
    p.smoothing = smoothing;
    p.min_dimension = min_dimension;
    tipl::image<3, vec3> dis;
    bool terminated = false;
    bool ok = tipl::reg::cdm_common<void, u8, 3>({cview(It, dim)}, {cview(Is, dim)}, dis, terminated, p, false);
    if (ok)
        field_out(dis, dis_out);
    return ok ? 1 : 0;
}
int tiplref_cdm_f32(const float* It, const float* Is, const int* dim, float* dis_out, float resolution,
                    float speed, float smoothing, unsigned int min_dimension)
{
    tipl::reg::cdm_param p;
    p.resolution = resolution;
    p.speed = speed;
    p.smoothing = smoothing;
    p.min_dimension = min_dimension;
    tipl::image<3, vec3> dis;
    bool terminated = false;
    bool ok = tipl::reg::cdm_common<void, float, 3>({cview(It, dim)}, {cview(Is, dim)}, dis, terminated, p, false);
    if (ok)
        field_out(dis, dis_out);
    return ok ? 1 : 0;
}

int tiplref_cdm_multi_u8(const u8* const* It, const u8* const* Is, int nmod, const int* dim, float* dis_out,
                         float resolution, float speed, float smoothing, unsigned int min_dimension,
                         const char* gtypes)
{
    return cdm_multi(It, Is, nmod, dim, dis_out, resolution, speed, smoothing, min_dimension, gtypes);
}
int tiplref_cdm_multi_f32(const float* const* It, const float* const* Is, int nmod, const int* dim, float* dis_out,
                          float resolution, float speed, float smoothing, unsigned int min_dimension,
                          const char* gtypes)
{
    return cdm_multi(It, Is, nmod, dim, dis_out, resolution, speed, smoothing, min_dimension, gtypes);
}

// cdm_common<void, unsigned char, 2>(It, Is, dis, terminated, param, cuda = false)
// (reg/cdm.hpp:534-558 at dimension 2): 2-D uint8 images of dims (w, h); the field
// out as interleaved (x, y) floats.
int tiplref_cdm2d_multi_u8(const u8* const* It, const u8* const* Is, int nmod, const int* dim, float* dis_out,
                           float resolution, float speed, float smoothing, unsigned int min_dimension,
                           const char* gtypes)
{
    tipl::reg::cdm_param p;
    p.resolution = resolution;
    p.speed = speed;
    p.smoothing = smoothing;
    p.min_dimension = min_dimension;
    p.gradient_type = gtypes ? gtypes : "";
    const tipl::shape<2> sh(dim[0], dim[1]);
    std::vector<tipl::const_pointer_image<2, u8> > lt, ls;
    for (int i = 0; i < nmod; ++i) {
        lt.push_back(tipl::const_pointer_image<2, u8>(It[i], sh));
        ls.push_back(tipl::const_pointer_image<2, u8>(Is[i], sh));
    }
    tipl::image<2, tipl::vector<2> > dis;
    bool terminated = false;
    const bool ok = tipl::reg::cdm_common<void, u8, 2>(lt, ls, dis, terminated, p, false);
    if (ok)
        std::memcpy(dis_out, &dis[0][0], sizeof(float) * 2 * dis.size());
    return ok ? 1 : 0;
}

// linear<void>(from, from_vs, to, to_vs, arg, param) (reg/linear.hpp:622-700); returns the final cost.
float tiplref_linear(const u8* from, const int* from_dim, const float* from_vs, const u8* to, const int* to_dim,
                     const float* to_vs, float* arg_inout, int reg_type, int cost_type)
{
    tipl::affine_param<float, 3> arg(arg_inout);
    tipl::reg::linear_reg_param p;
    p.reg_type = tipl::reg::reg_type(reg_type);
    p.cost_type = tipl::reg::cost_type(cost_type);
    p.cuda = false;
    bool terminated = false;
    float c = tipl::reg::linear<void>(std::vector<tipl::const_pointer_image<3, u8>>{cview(from, from_dim)},
                                      tipl::vector<3>(from_vs),
                                      std::vector<tipl::const_pointer_image<3, u8>>{cview(to, to_dim)},
                                      tipl::vector<3>(to_vs), arg, p, terminated);
    std::copy(arg.begin(), arg.end(), arg_inout);
    return c;
}

// has_mask(img) (numerical/basic_op.hpp:811-830)
int tiplref_has_mask(const u8* img, const int* dim) { return tipl::has_mask(cview(img, dim)) ? 1 : 0; }

// estimate_affine_param(source, source_vs, target, target_vs, arg) (numerical/transformation.hpp:933-1021)
void tiplref_estimate_affine_param(const u8* src, const int* sdim, const float* svs, const u8* tgt, const int* tdim,
                                   const float* tvs, float* arg)
{
    tipl::affine_param<float, 3> a;
    tipl::estimate_affine_param(cview(src, sdim), tipl::vector<3>(svs), cview(tgt, tdim), tipl::vector<3>(tvs), a);
    std::copy(a.begin(), a.end(), arg);
}

// transformation_matrix::to_affine_param(from, from_vs, to, to_vs) (numerical/transformation.hpp:703-741)
void tiplref_matrix_to_affine_param(const float* T, const int* from_dim, const float* from_vs, const int* to_dim,
                                    const float* to_vs, float* arg)
{
    auto a = to_matrix(T).to_affine_param(shp(from_dim), tipl::vector<3>(from_vs), shp(to_dim),
                                          tipl::vector<3>(to_vs));
    std::copy(a.begin(), a.end(), arg);
}

// eigen_decomposition_sym, 3x3 double (numerical/matrix.hpp:1830-1955)
void tiplref_eigen_sym3(const double* A, double* V, double* d)
{
    tipl::mat::eigen_decomposition_sym(A, V, d, tipl::dim<3, 3>());
}

// linear<void> with an explicit bound table: 0 reg_bound, 1 narrow_bound, 2 large_bound
// (reg/linear.hpp:258-266); the narrow bound takes the single-threaded L-BFGS path.
float tiplref_linear_bound(const u8* from, const int* from_dim, const float* from_vs, const u8* to,
                           const int* to_dim, const float* to_vs, float* arg_inout, int reg_type, int cost_type,
                           int bound)
{
    tipl::affine_param<float, 3> arg(arg_inout);
    tipl::reg::linear_reg_param p;
    p.reg_type = tipl::reg::reg_type(reg_type);
    p.cost_type = tipl::reg::cost_type(cost_type);
    p.bound = bound == 1 ? tipl::reg::narrow_bound : (bound == 2 ? tipl::reg::large_bound : tipl::reg::reg_bound);
    p.cuda = false;
    bool terminated = false;
    float c = tipl::reg::linear<void>(std::vector<tipl::const_pointer_image<3, u8>>{cview(from, from_dim)},
                                      tipl::vector<3>(from_vs),
                                      std::vector<tipl::const_pointer_image<3, u8>>{cview(to, to_dim)},
                                      tipl::vector<3>(to_vs), arg, p, terminated);
    std::copy(arg.begin(), arg.end(), arg_inout);
    return c;
}

// normalize_upper_lower2(in, out, upper) (numerical/numerical.hpp:909-927): float -> uint8
void tiplref_normalize_to_u8(const float* in, const int* dim, u8* out, float upper)
{
    tipl::image<3, u8> o;
    tipl::normalize_upper_lower2(cview(in, dim), o, upper);
    if (o.size() == size_t(dim[0]) * dim[1] * dim[2])
        std::copy(o.begin(), o.end(), out);
}

// displacement_to_mapping(dis, mapping, T) (numerical/dif.hpp:42-51)
void tiplref_displacement_to_mapping(const float* dis, const int* dim, const float* T, float* mapping)
{
    auto d = field_in(dis, dim);
    tipl::image<3, vec3> m(shp(dim));
    tipl::displacement_to_mapping(d, m, to_matrix(T));
    field_out(m, mapping);
}

// inv_displacement_to_mapping(inv_dis, inv_mapping, T) (numerical/dif.hpp:53-66)
void tiplref_inv_displacement_to_mapping(const float* inv_dis, const int* dis_dim, const float* T,
                                         const int* map_dim, float* inv_mapping)
{
    auto d = field_in(inv_dis, dis_dim);
    tipl::image<3, vec3> m(shp(map_dim));
    tipl::inv_displacement_to_mapping(d, m, to_matrix(T));
    field_out(m, inv_mapping);
}

// compose_mapping(from, mapping) for a uint8 image (numerical/dif.hpp:70-90)
void tiplref_compose_mapping_u8(const u8* from, const int* fdim, const float* mapping, const int* mdim, u8* to)
{
    auto m = field_in(mapping, mdim);
    auto o = tipl::compose_mapping(cview(from, fdim), m);
    std::copy(o.begin(), o.end(), to);
}

// correlation(x, y) of two uint8 images (numerical/statistics.hpp:585-598)
double tiplref_correlation_u8(const u8* x, const u8* y, long long n)
{
    return tipl::correlation(x, x + n, y);
}

// correlation_ygz(x, y) of two uint8 images (numerical/statistics.hpp:600-619)
double tiplref_correlation_ygz_u8(const u8* x, const u8* y, long long n)
{
    return tipl::correlation_ygz(x, x + n, y);
}

// filter::gaussian(I, bandwidth) on a float image (filter/gaussian.hpp:84-96), in place
void tiplref_gaussian(float* img, const int* dim, int bandwidth)
{
    tipl::image<3> I(img, shp(dim));
    tipl::filter::gaussian(I, (unsigned int)bandwidth);
    std::copy(I.begin(), I.end(), img);
}

// segmentation::otsu_threshold / otsu_median (numerical/otsu.hpp:59-100)
float tiplref_otsu_threshold(const float* img, const int* dim)
{
    return tipl::segmentation::otsu_threshold(tipl::image<3>(img, shp(dim)));
}
float tiplref_otsu_median(const float* img, const int* dim)
{
    return tipl::segmentation::otsu_median(tipl::image<3>(img, shp(dim)));
}

// reg::subject_image_pre (reg/mm_reg.hpp:14-20): float image -> uint8
void tiplref_subject_image_pre(const float* img, const int* dim, u8* out)
{
    auto o = tipl::reg::subject_image_pre(tipl::image<3>(img, shp(dim)));
    std::copy(o.begin(), o.end(), out);
}

// normalize_upper_lower2 of a uint16 volume (numerical/numerical.hpp:909-927)
void tiplref_normalize_u16_to_u8(const unsigned short* in, const int* dim, u8* out, float upper)
{
    tipl::image<3, u8> o;
    tipl::normalize_upper_lower2(cview(in, dim), o, upper);
    if (o.size() == size_t(dim[0]) * dim[1] * dim[2])
        std::copy(o.begin(), o.end(), out);
}


// tipl::io::gz_nifti in(path, std::ios::in); in >> I >> vs >> T (io/nifti.hpp:617-754,
// 1134-1205): I is the first volume as float, reoriented to LPS.  dim_out receives the
// LPS dims, data_out (capacity cap floats) the voxels.  Returns 1 on success.
int tiplref_nifti_load(const char* path, int* dim_out, float* vs_out, float* srow_out, float* data_out,
                       long long cap, int* is_mni)
{
    tipl::io::gz_nifti in(path, std::ios::in);
    if (!in)
        return 0;
    tipl::image<3, float> I;
    tipl::vector<3> vs;
    tipl::matrix<4, 4> T;
    bool mni = false;
    if (!(in >> I >> vs >> T >> mni))
        return 0;
    for (int i = 0; i < 3; ++i) {
        dim_out[i] = int(I.shape()[i]);
        vs_out[i] = vs[i];
    }
    std::copy_n(T.begin(), 12, srow_out);
    *is_mni = mni ? 1 : 0;
    if ((long long)I.size() > cap)
        return 0;
    std::copy(I.begin(), I.end(), data_out);
    return 1;
}

// tipl::io::gz_nifti out(path, std::ios::out); out << vs << T << mni << I
// (io/nifti.hpp:617-635, 969-1030) for a float or uint8 volume.
int tiplref_nifti_save(const char* path, const void* data, int is_u8, const int* dim, const float* vs,
                       const float* srow, int is_mni)
{
    tipl::io::gz_nifti out(path, std::ios::out);
    if (!out)
        return 0;
    tipl::matrix<4, 4> T;
    T.identity();
    std::copy_n(srow, 12, T.begin());
    tipl::vector<3> v(vs[0], vs[1], vs[2]);
    if (is_u8) {
        tipl::image<3, u8> I(shp(dim));
        std::memcpy(I.data(), data, I.size());
        return (out << v << T << bool(is_mni) << I) ? 1 : 0;
    }
    tipl::image<3, float> I(shp(dim));
    std::memcpy(I.data(), data, I.size() * sizeof(float));
    return (out << v << T << bool(is_mni) << I) ? 1 : 0;
}
// gz_nifti(path, out) << vs << T << I for a 4-D float image of dims (w, h, d, t):
// mm_reg::export_nonlinear's dis file (reg/mm_reg.hpp:418-441).
int tiplref_nifti_save4(const char* path, const float* data, const int* dim4, const float* vs, const float* srow)
{
    tipl::io::gz_nifti out(path, std::ios::out);
    if (!out)
        return 0;
    tipl::matrix<4, 4> T;
    T.identity();
    std::copy_n(srow, 12, T.begin());
    tipl::vector<3> v(vs[0], vs[1], vs[2]);
    tipl::image<4, float> I(tipl::shape<4>(dim4[0], dim4[1], dim4[2], dim4[3]));
    std::memcpy(I.data(), data, I.size() * sizeof(float));
    return (out << v << T << I) ? 1 : 0;
}
}  // extern "C"
