/* Test infrastructure only (the checker, never the product path).
 *
 * Plain-C restatement of the reference's CPU registration hot path, built into
 * oracle/liboracle.so by oracle/Makefile.  Volumes are x-fastest,
 * index = (z*h + y)*w + x; displacement fields are AoS xyz per voxel.
 * A transform T is the reference's transformation_matrix storage:
 * T[0..8] = sr (row-major 3x3), T[9..11] = shift (numerical/transformation.hpp:589-605).
 *
 * Suffixes: _u8 / _f32 are reference-exact (bit-identical to the reference's own
 * -O2 -ffp-contract=off build); _f64 computes everything in double and exists only
 * to report how far the FP32 paths are from exact arithmetic.
 */
#ifndef REGB_ORACLE_H
#define REGB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void orc_affine_to_matrix(const float* param, const int* from_dim, const float* from_vs, const int* to_dim,
                          const float* to_vs, float* T);
void orc_affine_to_matrix_f64(const double* param, const int* from_dim, const double* from_vs, const int* to_dim,
                              const double* to_vs, double* T);
int orc_matrix_inverse(float* T);
int orc_is_integer_shift(const float* T, int* shift);

void orc_resample_u8(const uint8_t* from, const int* fdim, uint8_t* to, const int* tdim, const float* T, int allow_crop);
void orc_resample_f32(const float* from, const int* fdim, float* to, const int* tdim, const float* T, int allow_crop);

void orc_histogram_u8(const uint8_t* img, long long n, int32_t* hist256);
void orc_mi_hist_u8(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const float* T,
                    int32_t* hist);
double orc_mi_cost_from_hist(const int32_t* hist, const int32_t* from_hist);
double orc_mi_cost_u8(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const float* T);
/* MI on a 32x32 joint histogram of the volumes quantised to 0..31; hist: optional, 1024 */
double orc_mi32_cost_u8(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const float* T,
                        int32_t* hist);
double orc_corr_cost_u8(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const float* T);
double orc_mi_cost_u8_f64(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const double* T);
double orc_corr_cost_u8_f64(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const double* T);

void orc_compose_u8(const uint8_t* Is, const int* dim, const float* dis, uint8_t* Js);
void orc_compose_f32(const float* Is, const int* dim, const float* dis, float* Js);
void orc_compose_f64(const double* Is, const int* dim, const double* dis, double* Js);
float orc_cdm_gradient_u8(const uint8_t* Js, const uint8_t* It, const int* dim, float* new_d, int gradient_type);
float orc_cdm_gradient_f32(const float* Js, const float* It, const int* dim, float* new_d, int gradient_type);
double orc_cdm_gradient_f64(const double* Js, const double* It, const int* dim, double* new_d, int gradient_type);
void orc_downsample_u8(const uint8_t* in, const int* dim, uint8_t* out);
void orc_downsample_f32(const float* in, const int* dim, float* out);
void orc_downsample_f64(const double* in, const int* dim, double* out);

void orc_cdm_poisson_f32(float* new_d, const int* dim, int sweeps);
void orc_cdm_poisson_f64(double* new_d, const int* dim, int sweeps);
float orc_cdm_max_len_f32(const float* d, const int* dim);
double orc_cdm_max_len_f64(const double* d, const int* dim);
void orc_accumulate_f32(const float* cur_d, float* new_d, const int* dim);
void orc_accumulate_f64(const double* cur_d, double* new_d, const int* dim);
void orc_cdm_smooth_f32(const float* d, float* dd, const int* dim, float smoothing);
void orc_cdm_smooth_f64(const double* d, double* dd, const int* dim, double smoothing);
void orc_upsample_field_x2_f32(const float* in, const int* in_dim, float* out, const int* out_dim);
void orc_upsample_field_x2_f64(const double* in, const int* in_dim, double* out, const int* out_dim);

int orc_cdm_level_u8(const uint8_t* It, const uint8_t* Is, const int* dim, float* best_d, float resolution,
                     float speed, float smoothing, unsigned int min_dimension, int gradient_type, int* iters_out);
int orc_cdm_level_f32(const float* It, const float* Is, const int* dim, float* best_d, float resolution, float speed,
                      float smoothing, unsigned int min_dimension, int gradient_type, int* iters_out);
int orc_cdm_level_f64(const double* It, const double* Is, const int* dim, double* best_d, float resolution,
                      float speed, float smoothing, unsigned int min_dimension, int gradient_type, int* iters_out);
int orc_cdm_multi_u8(const uint8_t* const* It, const uint8_t* const* Is, int nmod, const int* dim, float* best_d,
                     float resolution, float speed, float smoothing, unsigned int min_dimension, const char* gtypes,
                     int* iters_out);
int orc_cdm_multi_f32(const float* const* It, const float* const* Is, int nmod, const int* dim, float* best_d,
                      float resolution, float speed, float smoothing, unsigned int min_dimension, const char* gtypes,
                      int* iters_out);
int orc_cdm_multi_f64(const double* const* It, const double* const* Is, int nmod, const int* dim, double* best_d,
                      float resolution, float speed, float smoothing, unsigned int min_dimension, const char* gtypes,
                      int* iters_out);

/* The CDM at dimension 2 (oracle_cdm2d.h): uint8 images of dims (w, h), fields as
 * interleaved (x, y) floats. */
void orc2_downsample_u8(const uint8_t* in, const int* dim, uint8_t* out);
void orc2_upsample_field_x2(const float* in, const int* in_dim, float* out, const int* out_dim);
void orc2_compose_u8(const uint8_t* Is, const int* dim, const float* d, uint8_t* Js);
float orc2_cdm_gradient_u8(const uint8_t* Js, const uint8_t* It, const int* dim, float* new_d, int gradient_type);
void orc2_cdm_poisson(float* new_d, const int* dim, int sweeps);
float orc2_cdm_max_len(const float* d, const int* dim);
void orc2_accumulate(const float* cur_d, float* new_d, const int* dim);
void orc2_cdm_smooth(const float* d, float* dd, const int* dim, float smoothing);
int orc2_cdm_multi_u8(const uint8_t* const* It, const uint8_t* const* Is, int nmod, const int* dim, float* best_d,
                      float resolution, float speed, float smoothing, unsigned int min_dimension, const char* gtypes,
                      int* iters_out);

int orc_normalize_to_u8_f32(const float* in, long long n, uint8_t* out, float upper);
int orc_normalize_to_u8_u16(const uint16_t* in, long long n, uint8_t* out, float upper);
int orc_normalize_to_u8_u8(const uint8_t* in, long long n, uint8_t* out, float upper);
void orc_displacement_to_mapping_f32(const float* dis, const int* dim, const float* T, float* mapping);
void orc_inv_displacement_to_mapping_f32(const float* inv_dis, const int* dis_dim, const float* T,
                                         const int* map_dim, float* inv_mapping);
void orc_compose_mapping_u8(const uint8_t* from, const int* fdim, const float* mapping, const int* mdim, uint8_t* to);
double orc_correlation_u8(const uint8_t* x, const uint8_t* y, long long n);
double orc_correlation_ygz_u8(const uint8_t* x, const uint8_t* y, long long n);
void orc_match_fov_u8(const uint8_t* It, const int* fdim, const float* T, const int* mdim, uint8_t* out);
void orc_gaussian_f32(float* img, const int* dim, int bandwidth);
float orc_otsu_threshold_f32(const float* img, long long n);
float orc_median_f32(const float* v, long long n);
float orc_otsu_median_f32(const float* img, long long n);
void orc_normalize_otsu_median_f32(float* img, long long n, float upper);
void orc_subject_image_pre_f32(const float* in, const int* dim, uint8_t* out);
int orc_has_mask_u8(const uint8_t* img, const int* dim);
void orc_eigen_sym3(const double* A, double* V, double* d);
void orc_estimate_affine_param_u8(const uint8_t* src, const int* sdim, const float* svs, const uint8_t* tgt,
                                  const int* tdim, const float* tvs, float* arg);
void orc_matrix_to_affine_param(const float* T, const int* from_dim, const float* from_vs, const int* to_dim,
                                const float* to_vs, float* arg);

/* NIfTI volume `vol` of path as float in LPS orientation (the reference's gz_nifti >> I);
 * 1 on success */
int orc_nifti_load(const char* path, int vol, float* out, long long cap, int* dim, float* vs, float* srow,
                   int* steps, int* nsteps);

#ifdef __cplusplus
}
#endif
#endif
