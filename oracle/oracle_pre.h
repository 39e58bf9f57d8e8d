/* Test infrastructure only (the checker, never the product path).
 *
 * Plain-C restatement of the subject preprocessing of the mm_reg pipeline
 * (reg/mm_reg.hpp:14-20, subject_image_pre): the separable [1 2 1] Gaussian
 * (filter/gaussian.hpp:18-88), the Otsu threshold and median
 * (numerical/otsu.hpp:14-107), normalize_otsu_median (numerical/otsu.hpp:110-136)
 * and the conversion of the float image to uint8.  Included once by oracle.c.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* gaussian_impl (filter/gaussian.hpp:18-81) for a float image: bandwidth rounds of
 * x, y, z passes of (a[left] + 2a[i]) + a[right] with the edge sample repeated, then
 * the exact scale 2^-(2 * bandwidth * 3). */
void orc_gaussian_f32(float* img, const int* dim, int bandwidth)
{
    const size_t w = (size_t)dim[0], h = (size_t)dim[1], d = (size_t)dim[2], wh = w * h, n = wh * d;
    if (!n || !bandwidth)
        return;
    float* a = (float*)malloc(n * sizeof(float));
    float* b = (float*)malloc(n * sizeof(float));
    memcpy(a, img, n * sizeof(float));
    for (int k = 0; k < bandwidth; ++k) {
        for (size_t i = 0; i < n; ++i) {
            size_t x = i % w;
            float c = a[i];
            c += c;
            b[i] = a[x ? i - 1 : i] + c + a[x + 1 < w ? i + 1 : i];
        }
        { float* t = a; a = b; b = t; }
        for (size_t i = 0; i < n; ++i) {
            size_t y = (i / w) % h;
            float c = a[i];
            c += c;
            b[i] = a[y ? i - w : i] + c + a[y + 1 < h ? i + w : i];
        }
        { float* t = a; a = b; b = t; }
        for (size_t i = 0; i < n; ++i) {
            size_t z = i / wh;
            float c = a[i];
            c += c;
            b[i] = a[z ? i - wh : i] + c + a[z + 1 < d ? i + wh : i];
        }
        { float* t = a; a = b; b = t; }
    }
    const double scale = ldexp(1.0, -(int)(2 * (size_t)bandwidth * 3));
    for (size_t i = 0; i < n; ++i)
        img[i] = (float)(a[i] * scale);
    free(a);
    free(b);
}

/* otsu_threshold (numerical/otsu.hpp:59-71) with otsu_threshold_from_hist (:14-57):
 * a 256-bin histogram over [min, max] (numerical/basic_op.hpp:1293-1311), bin 0
 * cleared, the between-class variance scan in float. */
float orc_otsu_threshold_f32(const float* img, long long n)
{
    if (n <= 0)
        return 0.0f;
    float mn = img[0], mx = img[0];
    for (long long i = 1; i < n; ++i) {
        if (img[i] < mn) mn = img[i];
        if (img[i] > mx) mx = img[i];
    }
    if (mn >= mx)
        return mn;
    unsigned int hist[256];
    memset(hist, 0, sizeof(hist));
    float range = mx - mn;
    if (range == 0.0f)
        range = 1.0f;
    range = 256.0f / range;
    for (long long i = 0; i < n; ++i) {
        float v = (img[i] - mn) * range;
        int b = (int)floorf(v);
        b = b < 0 ? 0 : (b > 255 ? 255 : b);
        ++hist[b];
    }
    hist[0] = 0;
    float total_w = 0.0f, total_sum = 0.0f;
    for (int i = 0; i < 256; ++i) {
        float val = (float)hist[i];
        total_w += val;
        total_sum += val * (float)i;
    }
    if (total_w == 0.0f)
        return mn;
    float max_sig_b = 0.0f, w_b = 0.0f, sum_b = 0.0f;
    size_t opt = 0;
    for (size_t i = 0; i < 255; ++i) {
        w_b += (float)hist[i];
        if (w_b == 0.0f)
            continue;
        float w_f = total_w - w_b;
        if (w_f == 0.0f)
            break;
        sum_b += (float)hist[i] * (float)i;
        float dd = (sum_b * total_w) - (total_sum * w_b);
        float sig_b = (dd * dd) / (w_b * w_f);
        if (sig_b > max_sig_b) {
            max_sig_b = sig_b;
            opt = i;
        }
    }
    return mn + (float)opt * (mx - mn) / (float)256;
}

static int orc_cmp_f32(const void* a, const void* b)
{
    const float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}

/* The element nth_element places at begin + size/2 (numerical/statistics.hpp:326-333). */
static float orc_mid_f32(float* v, size_t n)
{
    qsort(v, n, sizeof(float), orc_cmp_f32);
    return v[n / 2];
}

/* median(container) (numerical/statistics.hpp:343-363): below 2048 values the middle
 * element; otherwise the middle of the 256 middles of 256 contiguous chunks. */
float orc_median_f32(const float* v, long long n)
{
    float* t = (float*)malloc((size_t)(n > 0 ? n : 1) * sizeof(float));
    memcpy(t, v, (size_t)n * sizeof(float));
    float r;
    if (n < 2048)
        r = orc_mid_f32(t, (size_t)n);
    else {
        const size_t cc = 256, cs = (size_t)n / cc, rem = (size_t)n % cc;
        float chunk[256];
        for (size_t i = 0; i < cc; ++i) {
            size_t s = i * cs + (i < rem ? i : rem);
            size_t len = cs + (i < rem ? 1 : 0);
            chunk[i] = orc_mid_f32(t + s, len);
        }
        r = orc_mid_f32(chunk, cc);
    }
    free(t);
    return r;
}

/* otsu_median (numerical/otsu.hpp:86-100): the median of the values above the Otsu
 * threshold, kept in voxel order. */
float orc_otsu_median_f32(const float* img, long long n)
{
    float ot = orc_otsu_threshold_f32(img, n);
    float* buf = (float*)malloc((size_t)(n > 0 ? n : 1) * sizeof(float));
    long long m = 0;
    for (long long i = 0; i < n; ++i)
        if (img[i] > ot)
            buf[m++] = img[i];
    float r = m ? orc_median_f32(buf, m) : ot;
    free(buf);
    return r;
}

/* normalize_otsu_median, float image (numerical/otsu.hpp:126-135) */
void orc_normalize_otsu_median_f32(float* img, long long n, float upper)
{
    float ot = orc_otsu_median_f32(img, n);
    if (ot == 0.0f)
        return;
    const float s = upper * 0.5f / ot;
    long long pos = 0;
    for (long long i = 0; i < n; ++i) {
        img[i] = img[i] * s;
        pos += img[i] > 0.0f;
    }
    if ((double)pos > 0.5 * (double)n) {
        const float c = upper * 0.1f;
        for (long long i = 0; i < n; ++i)
            img[i] = img[i] - c;
    }
    for (long long i = 0; i < n; ++i)
        img[i] = img[i] > upper ? upper : (img[i] < 0.0f ? 0.0f : img[i]);
}

/* subject_image_pre (reg/mm_reg.hpp:14-20): gaussian (bandwidth 1), then
 * normalize_otsu_median(I, 255.99), then the float -> uint8 conversion. */
void orc_subject_image_pre_f32(const float* in, const int* dim, uint8_t* out)
{
    const long long n = (long long)dim[0] * dim[1] * dim[2];
    float* t = (float*)malloc((size_t)(n > 0 ? n : 1) * sizeof(float));
    memcpy(t, in, (size_t)n * sizeof(float));
    orc_gaussian_f32(t, dim, 1);
    orc_normalize_otsu_median_f32(t, n, 255.99f);
    for (long long i = 0; i < n; ++i)
        out[i] = (uint8_t)t[i];
    free(t);
}
