/* Test infrastructure only (the checker, never the product path).
 *
 * Plain-C restatement of the reference's CPU registration hot path.  The generic
 * bodies live in oracle_core.h (pixel passes), oracle_field.h (displacement-field
 * passes) and oracle_cdm.h (the CDM driver); this file holds the transform
 * algebra and the two affine cost functions, then instantiates the generic
 * bodies for uint8/float (reference-exact) and double (error reporting).
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

/* rotation_matrix (numerical/transformation.hpp:143-164), scaling
 * (transformation.hpp:196-208), affine shear (transformation.hpp:220-231) and the
 * voxel-space composition of transformation_matrix(affine_param, ...)
 * (transformation.hpp:636-675).  All in float, in the reference's order. */
void orc_affine_to_matrix(const float* p, const int* fd, const float* fvs, const int* td, const float* tvs, float* T)
{
    const float* tr = p;
    const float* th = p + 3;
    const float* s = p + 6;
    const float* a = p + 9;
    float* m = T;
    float sin_x = sinf(th[0]), cos_x = cosf(th[0]);
    float sin_y = sinf(th[1]), cos_y = cosf(th[1]);
    float sin_z = sinf(th[2]), cos_z = cosf(th[2]);
    float cos_x_sin_z = cos_x * sin_z, cos_x_cos_z = cos_x * cos_z;
    float sin_x_sin_z = sin_x * sin_z, sin_x_cos_z = sin_x * cos_z;
    m[0] = cos_y * cos_z;
    m[1] = cos_y * sin_z;
    m[2] = -sin_y;
    m[3] = -cos_x_sin_z + sin_x_cos_z * sin_y;
    m[4] = cos_x_cos_z + sin_x_sin_z * sin_y;
    m[5] = sin_x * cos_y;
    m[6] = sin_x_sin_z + cos_x_cos_z * sin_y;
    m[7] = -sin_x_cos_z + cos_x_sin_z * sin_y;
    m[8] = cos_x * cos_y;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            m[3 * r + c] *= s[r];
    m[0] += m[3] * a[0] + m[6] * a[1];
    m[1] += m[4] * a[0] + m[7] * a[1];
    m[2] += m[5] * a[0] + m[8] * a[1];
    m[3] += m[6] * a[2];
    m[4] += m[7] * a[2];
    m[5] += m[8] * a[2];
    float t[3] = {(float)fd[0], (float)fd[1], (float)fd[2]};
    for (int i = 0; i < 3; ++i) {
        t[i] *= -0.5f;
    }
    for (int i = 0; i < 3; ++i)
        t[i] *= fvs[i];
    for (int i = 0; i < 3; ++i)
        t[i] += tr[i];
    float* sh = T + 9;
    sh[0] = m[0] * t[0] + m[1] * t[1] + m[2] * t[2];
    sh[1] = m[3] * t[0] + m[4] * t[1] + m[5] * t[2];
    sh[2] = m[6] * t[0] + m[7] * t[1] + m[8] * t[2];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            m[3 * r + c] *= fvs[c];
    for (int r = 0; r < 3; ++r)
        if (tvs[r] != 1.0f) {
            m[3 * r] /= tvs[r];
            m[3 * r + 1] /= tvs[r];
            m[3 * r + 2] /= tvs[r];
            sh[r] /= tvs[r];
        }
    for (int r = 0; r < 3; ++r)
        sh[r] += (float)td[r] * 0.5f;
}

/* The same composition in double (the FP64 4x4 affine path). */
void orc_affine_to_matrix_f64(const double* p, const int* fd, const double* fvs, const int* td, const double* tvs,
                              double* T)
{
    const double* tr = p;
    const double* th = p + 3;
    const double* s = p + 6;
    const double* a = p + 9;
    double* m = T;
    double sin_x = sin(th[0]), cos_x = cos(th[0]);
    double sin_y = sin(th[1]), cos_y = cos(th[1]);
    double sin_z = sin(th[2]), cos_z = cos(th[2]);
    m[0] = cos_y * cos_z;
    m[1] = cos_y * sin_z;
    m[2] = -sin_y;
    m[3] = -cos_x * sin_z + sin_x * cos_z * sin_y;
    m[4] = cos_x * cos_z + sin_x * sin_z * sin_y;
    m[5] = sin_x * cos_y;
    m[6] = sin_x * sin_z + cos_x * cos_z * sin_y;
    m[7] = -sin_x * cos_z + cos_x * sin_z * sin_y;
    m[8] = cos_x * cos_y;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            m[3 * r + c] *= s[r];
    m[0] += m[3] * a[0] + m[6] * a[1];
    m[1] += m[4] * a[0] + m[7] * a[1];
    m[2] += m[5] * a[0] + m[8] * a[1];
    m[3] += m[6] * a[2];
    m[4] += m[7] * a[2];
    m[5] += m[8] * a[2];
    double t[3];
    for (int i = 0; i < 3; ++i)
        t[i] = (double)fd[i] * -0.5 * fvs[i] + tr[i];
    double* sh = T + 9;
    for (int r = 0; r < 3; ++r)
        sh[r] = m[3 * r] * t[0] + m[3 * r + 1] * t[1] + m[3 * r + 2] * t[2];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            m[3 * r + c] *= fvs[c];
    for (int r = 0; r < 3; ++r) {
        m[3 * r] /= tvs[r];
        m[3 * r + 1] /= tvs[r];
        m[3 * r + 2] /= tvs[r];
        sh[r] /= tvs[r];
        sh[r] += (double)td[r] * 0.5;
    }
}

/* transformation_matrix::inverse (numerical/transformation.hpp:820-832) with the
 * cofactor 3x3 inverse of numerical/matrix.hpp:1347-1352,1479-1505.  On a
 * singular sr the matrix is left unchanged and 0 is returned. */
int orc_matrix_inverse(float* T)
{
    const float* a = T;
    float det = a[0] * (a[4] * a[8] - a[5] * a[7]) + a[1] * (a[5] * a[6] - a[3] * a[8]) +
                a[2] * (a[3] * a[7] - a[4] * a[6]);
    if (det + 1.0f == 1.0f)
        return 0;
    float t[9];
    t[0] = a[4] * a[8] - a[5] * a[7];
    t[1] = a[2] * a[7] - a[1] * a[8];
    t[2] = a[1] * a[5] - a[2] * a[4];
    t[3] = a[5] * a[6] - a[3] * a[8];
    t[4] = a[0] * a[8] - a[2] * a[6];
    t[5] = a[2] * a[3] - a[0] * a[5];
    t[6] = a[3] * a[7] - a[4] * a[6];
    t[7] = a[1] * a[6] - a[0] * a[7];
    t[8] = a[0] * a[4] - a[1] * a[3];
    for (int i = 0; i < 9; ++i)
        t[i] = t[i] / det;
    float s[3] = {T[9], T[10], T[11]};
    float ns[3];
    for (int r = 0; r < 3; ++r)
        ns[r] = s[0] * t[3 * r] + s[1] * t[3 * r + 1] + s[2] * t[3 * r + 2];
    for (int r = 0; r < 3; ++r)
        T[9 + r] = -ns[r];
    for (int i = 0; i < 9; ++i)
        T[i] = t[i];
    return 1;
}

/* The integer-shift test of the CPU resample fast path
 * (numerical/resampling.hpp:1243-1258): every shift within 1e-4 of an integer
 * and sr within 1e-4 of the identity. */
int orc_is_integer_shift(const float* T, int* shift)
{
    const double eps = 1.0e-4;
    for (int i = 0; i < 3; ++i) {
        long s = lroundf(T[9 + i]);
        if (fabsf(T[9 + i] - (float)s) > eps)
            return 0;
        shift[i] = (int)s;
        for (int j = 0; j < 3; ++j)
            if (fabsf(T[3 * i + j] - (float)(i == j)) > eps)
                return 0;
    }
    return 1;
}

/* ---- generic instantiations ------------------------------------------------ */
#define SFX _u8
#define PIX uint8_t
#define R float
#define PIX_IS_U8 1
#include "oracle_core.h"
#undef SFX
#undef PIX
#undef R
#undef PIX_IS_U8

#define SFX _f32
#define PIX float
#define R float
#define PIX_IS_U8 0
#include "oracle_core.h"
#undef SFX
#undef PIX
#undef R
#undef PIX_IS_U8

#define SFX _f64
#define PIX double
#define R double
#define PIX_IS_U8 0
#include "oracle_core.h"
#undef SFX
#undef PIX
#undef R
#undef PIX_IS_U8

#define FSFX _f32
#define R float
#include "oracle_field.h"
#undef FSFX
#undef R

#define FSFX _f64
#define R double
#include "oracle_field.h"
#undef FSFX
#undef R

#define SFX _u8
#define FSFX _f32
#define PIX uint8_t
#define R float
#include "oracle_cdm.h"
#undef SFX
#undef FSFX
#undef PIX
#undef R

/* the 2-D CDM (uint8 images; uses regress_u8 and cdm_improved_u8 from above) */
#include "oracle_cdm2d.h"

#define SFX _f32
#define FSFX _f32
#define PIX float
#define R float
#include "oracle_cdm.h"
#undef SFX
#undef FSFX
#undef PIX
#undef R

#define SFX _f64
#define FSFX _f64
#define PIX double
#define R double
#include "oracle_cdm.h"
#undef SFX
#undef FSFX
#undef PIX
#undef R

/* ---- quantisation to uint8 ------------------------------------------------ */

/* normalize_upper_lower2(in, out, upper) (numerical/numerical.hpp:909-927): float
 * min/max, out = uint8((v - min) * (upper / (max - min))) truncated; returns 0 and
 * leaves out untouched for a constant volume. */
#define ORC_NORMALIZE(NAME, T)                                                  \
    int NAME(const T* in, long long n, uint8_t* out, float upper)               \
    {                                                                           \
        if (n <= 0)                                                             \
            return 0;                                                           \
        float mn = (float)in[0], mx = (float)in[0];                             \
        for (long long i = 1; i < n; ++i) {                                     \
            const float v = (float)in[i];                                       \
            if (v < mn) mn = v;                                                 \
            if (v > mx) mx = v;                                                 \
        }                                                                       \
        const float range = mx - mn;                                            \
        if (range == 0.0f)                                                      \
            return 0;                                                           \
        upper /= range;                                                         \
        for (long long i = 0; i < n; ++i)                                       \
            out[i] = (uint8_t)(((float)in[i] - mn) * upper);                    \
        return 1;                                                               \
    }
ORC_NORMALIZE(orc_normalize_to_u8_f32, float)
ORC_NORMALIZE(orc_normalize_to_u8_u16, uint16_t)
ORC_NORMALIZE(orc_normalize_to_u8_u8, uint8_t)
#undef ORC_NORMALIZE

/* ---- mapping steps of the mm_reg pipeline --------------------------------- */
#include "oracle_map.h"

/* ---- subject preprocessing of the mm_reg pipeline ------------------------- */
#include "oracle_pre.h"

/* ---- mask-moment initialisation of linear() ------------------------------- */
#include "oracle_mask.h"

/* ---- NIfTI volumes read as float ------------------------------------------ */
#include "oracle_nifti.h"

/* ---- affine costs ---------------------------------------------------------- */

/* histogram(img, hist, 0, 255, 256) (numerical/basic_op.hpp:1293-1311): bin =
 * clamp(floor(v * (256/255)), 0, 255), which for uint8 is the value itself. */
void orc_histogram_u8(const uint8_t* img, long long n, int32_t* hist)
{
    float range = 256.0f / 255.0f;
    memset(hist, 0, 256 * sizeof(int32_t));
    for (long long i = 0; i < n; ++i) {
        float v = (float)img[i] * range;
        int b = (int)floorf(v);
        if (b < 0) b = 0;
        if (b > 255) b = 255;
        ++hist[b];
    }
}

/* get_mutual_info CPU (reg/linear.hpp:138-146): for every template voxel x,
 * H[(from[x] << 8) + to(T x)]++, where to(T x) is the uint8 trilinear sample of the
 * moving volume (0 outside). */
void orc_mi_hist_u8(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const float* T,
                    int32_t* hist)
{
    memset(hist, 0, 65536 * sizeof(int32_t));
    size_t i = 0;
    for (int z = 0; z < fdim[2]; ++z)
        for (int y = 0; y < fdim[1]; ++y)
            for (int x = 0; x < fdim[0]; ++x, ++i) {
                float p[3];
                apply_T_u8(T, (float)x, (float)y, (float)z, p);
                uint8_t v = 0;
                trilinear_u8(to, tdim, p[0], p[1], p[2], &v);
                ++hist[((uint32_t)from[i] << 8) + v];
            }
}

/* get_mutual_info_mean CPU (reg/linear.hpp:87-104): column sums of H, then
 * sum over non-zero bins of n*ln(n/row/col), divided by 65536; the functor
 * returns its negative (linear.hpp:201). */
double orc_mi_cost_from_hist(const int32_t* hist, const int32_t* from_hist)
{
    uint32_t to_hist[256];
    memset(to_hist, 0, sizeof(to_hist));
    for (int i = 0; i < 65536; ++i)
        to_hist[i & 255] += (uint32_t)hist[i];
    double sum = 0.0;
    for (int i = 0; i < 65536; ++i) {
        double mu = hist[i];
        if (mu == 0.0f)
            continue;
        sum += mu * log(mu / (double)from_hist[i >> 8] / (double)to_hist[i & 255]);
    }
    return -(sum / (double)65536.0f);
}

double orc_mi_cost_u8(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const float* T)
{
    int32_t* hist = (int32_t*)malloc(65536 * sizeof(int32_t));
    int32_t fh[256];
    orc_histogram_u8(from, (long long)fdim[0] * fdim[1] * fdim[2], fh);
    orc_mi_hist_u8(from, fdim, to, tdim, T, hist);
    double c = orc_mi_cost_from_hist(hist, fh);
    free(hist);
    return c;
}

/* MI on a 32x32 joint histogram.  No counterpart in the reference, whose
 * mi_band_width is fixed at 8 (reg/linear.hpp:84-85); these are its
 * mutual_information steps (reg/linear.hpp:173-203) with 5 bits:
 *   - both volumes quantised by normalize_upper_lower2(v, 32 - 0.01f) (:195-196,
 *     the reference's step for non-uint8 inputs); a constant volume becomes all 0;
 *   - from_hist = histogram(from, 0, 31, 32) (:198, numerical/basic_op.hpp:1293-1311);
 *   - H[(from[x] << 5) + to(T x)]++ with the uint8 trilinear sample (:138-146);
 *   - -sum(n ln(n / row / col)) / 1024 (:87-104).
 * hist (optional, 1024 entries) receives H. */
double orc_mi32_cost_u8(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const float* T,
                        int32_t* hist)
{
    const long long nf = (long long)fdim[0] * fdim[1] * fdim[2], nt = (long long)tdim[0] * tdim[1] * tdim[2];
    uint8_t* qf = (uint8_t*)calloc((size_t)(nf > 0 ? nf : 1), 1);
    uint8_t* qt = (uint8_t*)calloc((size_t)(nt > 0 ? nt : 1), 1);
    const float upper = 32.0f - 0.01f;
    orc_normalize_to_u8_u8(from, nf, qf, upper);
    orc_normalize_to_u8_u8(to, nt, qt, upper);
    int32_t fh[32], H[1024];
    const float range = 32.0f / 31.0f;
    memset(fh, 0, sizeof(fh));
    for (long long i = 0; i < nf; ++i) {
        int b = (int)floorf((float)qf[i] * range);
        if (b < 0) b = 0;
        if (b > 31) b = 31;
        ++fh[b];
    }
    memset(H, 0, sizeof(H));
    size_t i = 0;
    for (int z = 0; z < fdim[2]; ++z)
        for (int y = 0; y < fdim[1]; ++y)
            for (int x = 0; x < fdim[0]; ++x, ++i) {
                float p[3];
                apply_T_u8(T, (float)x, (float)y, (float)z, p);
                uint8_t v = 0;
                trilinear_u8(qt, tdim, p[0], p[1], p[2], &v);
                ++H[((uint32_t)qf[i] << 5) + v];
            }
    uint32_t col[32];
    memset(col, 0, sizeof(col));
    for (int k = 0; k < 1024; ++k)
        col[k & 31] += (uint32_t)H[k];
    double sum = 0.0;
    for (int k = 0; k < 1024; ++k) {
        double mu = H[k];
        if (mu == 0.0f)
            continue;
        sum += mu * log(mu / (double)fh[k >> 5] / (double)col[k & 31]);
    }
    if (hist)
        memcpy(hist, H, sizeof(H));
    free(qf);
    free(qt);
    return -(sum / (double)1024.0f);
}

/* ---- FP64 restatement of the affine costs (error reporting only) ----------
 * The same algorithm as orc_mi_cost_u8 / orc_corr_cost_u8 with every float step in
 * double: the transform (given in double), the trilinear weights and the weighted
 * sum; the uint8 quantisation of the sampled value stays (it is part of the
 * algorithm: the joint histogram bins and the resampled volume are uint8). */
static int trilinear_u8_f64(const uint8_t* I, const int* dim, double x, double y, double z, uint8_t* out)
{
    if (x < 0 || y < 0 || z < 0)
        return 0;
    size_t ix = (size_t)x, iy = (size_t)y, iz = (size_t)z;
    size_t w = (size_t)dim[0];
    if (ix + 1 >= w || iy + 1 >= (size_t)dim[1] || iz + 1 >= (size_t)dim[2])
        return 0;
    double p0 = x - (double)ix, p1 = y - (double)iy, p2 = z - (double)iz;
    double n0 = 1 - p0, n1 = 1 - p1, n2 = 1 - p2;
    size_t wh = w * (size_t)dim[1];
    size_t d0 = iz * wh + iy * w + ix;
    size_t d[8] = {d0, d0 + 1, d0 + w, d0 + w + 1, d0 + wh, d0 + 1 + wh, d0 + w + wh, d0 + w + 1 + wh};
    double r[8] = {n0 * n1 * n2, p0 * n1 * n2, n0 * p1 * n2, p0 * p1 * n2,
                   n0 * n1 * p2, p0 * n1 * p2, n0 * p1 * p2, p0 * p1 * p2};
    double acc = 0.0;
    for (int i = 0; i < 8; ++i)
        acc += (double)I[d[i]] * r[i];
    *out = (uint8_t)(acc <= 0.0 ? 0 : (unsigned)acc);
    return 1;
}

double orc_mi_cost_u8_f64(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const double* T)
{
    int32_t* hist = (int32_t*)calloc(65536, sizeof(int32_t));
    int32_t fh[256];
    orc_histogram_u8(from, (long long)fdim[0] * fdim[1] * fdim[2], fh);
    size_t i = 0;
    for (int z = 0; z < fdim[2]; ++z)
        for (int y = 0; y < fdim[1]; ++y)
            for (int x = 0; x < fdim[0]; ++x, ++i) {
                const double px = x * T[0] + y * T[1] + z * T[2] + T[9];
                const double py = x * T[3] + y * T[4] + z * T[5] + T[10];
                const double pz = x * T[6] + y * T[7] + z * T[8] + T[11];
                uint8_t v = 0;
                trilinear_u8_f64(to, tdim, px, py, pz, &v);
                ++hist[((uint32_t)from[i] << 8) + v];
            }
    double c = orc_mi_cost_from_hist(hist, fh);
    free(hist);
    return c;
}

/* correlation in FP64 on the fixed grid (no role swap, no integer-shift copy): r from
 * the template and the double-interpolated, uint8-quantised moving volume; 1 - r^2. */
double orc_corr_cost_u8_f64(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const double* T)
{
    long long nf = (long long)fdim[0] * fdim[1] * fdim[2];
    double sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0;
    size_t i = 0;
    for (int z = 0; z < fdim[2]; ++z)
        for (int y = 0; y < fdim[1]; ++y)
            for (int x = 0; x < fdim[0]; ++x, ++i) {
                const double px = x * T[0] + y * T[1] + z * T[2] + T[9];
                const double py = x * T[3] + y * T[4] + z * T[5] + T[10];
                const double pz = x * T[6] + y * T[7] + z * T[8] + T[11];
                uint8_t v = 0;
                trilinear_u8_f64(to, tdim, px, py, pz, &v);
                const double a = from[i], b = v;
                sx += a; sy += b; sxx += a * a; syy += b * b; sxy += a * b;
            }
    const double n = (double)nf, mx = sx / n, my = sy / n;
    const double vx = sxx / n - mx * mx, vy = syy / n - my * my;
    if (vx <= 0 || vy <= 0)
        return 1.0;
    const double r = (sxy / n - mx * my) / sqrt(vx) / sqrt(vy);
    return 1.0 - r * r;
}

/* correlation functor CPU (reg/linear.hpp:23-37): the smaller volume is the
 * fixed grid (the transform is inverted when the roles swap); the other is
 * resampled onto it with the CPU resample (integer-shift copy included) and
 * cost = 1 - r^2, r formed in double from exact integer sums
 * (numerical/statistics.hpp:569-580, 311-322, 257-309, 491-567) and squared in float. */
double orc_corr_cost_u8(const uint8_t* from, const int* fdim, const uint8_t* to, const int* tdim, const float* T)
{
    long long nf = (long long)fdim[0] * fdim[1] * fdim[2];
    long long nt = (long long)tdim[0] * tdim[1] * tdim[2];
    if (nf > nt) {
        float Ti[12];
        memcpy(Ti, T, sizeof(Ti));
        orc_matrix_inverse(Ti);
        return orc_corr_cost_u8(to, tdim, from, fdim, Ti);
    }
    uint8_t* y = (uint8_t*)malloc((size_t)nf);
    orc_resample_u8(to, tdim, y, fdim, T, 1);
    long long sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0;
    for (long long i = 0; i < nf; ++i) {
        sx += from[i];
        sy += y[i];
        sxx += (long long)from[i] * from[i];
        syy += (long long)y[i] * y[i];
        sxy += (long long)from[i] * y[i];
    }
    free(y);
    double n = (double)nf;
    double mx = (double)sx / n, my = (double)sy / n;
    double vx = (double)sxx / n - mx * mx, vy = (double)syy / n - my * my;
    double sd1 = vx > 0.0 ? sqrt(vx) : 0.0, sd2 = vy > 0.0 ? sqrt(vy) : 0.0;
    double c = 0.0;
    if (!(sd1 == 0 || sd2 == 0))
        c = ((double)sxy / n - mx * my) / sd1 / sd2;
    float cf = (float)c;
    return (double)(1.0f - cf * cf);
}
