// Subject preprocessing of the mm_reg pipeline on the device (reg/mm_reg.hpp:14-20):
// subject_image_pre = filter::gaussian (bandwidth 1), normalize_otsu_median(I, 255.99),
// conversion to uint8.  The per-voxel passes are preprocess_kernels.cu; the 256-bin
// Otsu scan, the final middle of the 256 chunk middles and the scalar decisions are
// host arithmetic in the reference's float/double types.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "host.h"
#include "kernels.h"
#include "preprocess.h"
#include "stats.h"

namespace regb {

namespace {

float key_to_float(unsigned k)
{
    const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// otsu_threshold_from_hist (numerical/otsu.hpp:14-57): between-class variance scan in
// float over the histogram (bin 0 already cleared by the caller).
float otsu_from_hist(const unsigned* hist, float min_v, float max_v)
{
    float total_w = 0.0f, total_sum = 0.0f;
    for (int i = 0; i < 256; ++i) {
        const float val = (float)hist[i];
        total_w += val;
        total_sum += val * (float)i;
    }
    if (total_w == 0.0f)
        return min_v;
    float max_sig_b = 0.0f, w_b = 0.0f, sum_b = 0.0f;
    size_t best = 0;
    for (size_t i = 0; i + 1 < 256; ++i) {
        w_b += (float)hist[i];
        if (w_b == 0.0f)
            continue;
        const float w_f = total_w - w_b;
        if (w_f == 0.0f)
            break;
        sum_b += (float)hist[i] * (float)i;
        const float dd = (sum_b * total_w) - (total_sum * w_b);
        const float sig_b = (dd * dd) / (w_b * w_f);
        if (sig_b > max_sig_b) {
            max_sig_b = sig_b;
            best = i;
        }
    }
    return min_v + (float)best * (max_v - min_v) / (float)256;
}

float middle(std::vector<float>& v)
{
    std::nth_element(v.begin(), v.begin() + v.size() / 2, v.end());
    return v[v.size() / 2];
}

}  // namespace

void gaussian(const float* d_in, const int* dim, int bandwidth, float* d_out, cudaStream_t st)
{
    const long long n = (long long)dim[0] * dim[1] * dim[2];
    if (bandwidth <= 0) {
        if (d_out != d_in)
            REGB_CK(cudaMemcpyAsync(d_out, d_in, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
        return;
    }
    const float scale = (float)std::ldexp(1.0, -(2 * bandwidth * 3));
    DevBuf<float> tmp;
    if (bandwidth > 1)
        tmp.alloc((size_t)n, st);
    // rounds ping-pong so that the last one lands in d_out
    const float* src = d_in;
    for (int k = 0; k < bandwidth; ++k) {
        const bool last = (k + 1 == bandwidth);
        float* dst = ((bandwidth - 1 - k) % 2 == 0) ? d_out : tmp.p;
        REGB_CK(launch_gaussian_round(src, dst, dim[0], dim[1], dim[2], scale, last ? 1 : 0, st));
        count_launch();
        src = dst;
    }
}

float otsu_median(const float* d_img, long long n, cudaStream_t st)
{
    DevBuf<unsigned> mm(2, st), hist(256, st);
    REGB_CK(launch_minmax(d_img, REGB_F32, n, mm.p, st));
    count_launch();
    unsigned hmm[2];
    REGB_CK(cudaMemcpyAsync(hmm, mm.p, sizeof(hmm), cudaMemcpyDeviceToHost, st));
    REGB_CK(cudaStreamSynchronize(st));
    const float mn = key_to_float(hmm[0]), mx = key_to_float(hmm[1]);
    // otsu_threshold (numerical/otsu.hpp:59-71) with histogram (basic_op.hpp:1293-1311)
    float ot = mn;
    if (mn < mx) {
        float range = mx - mn;
        if (range == 0.0f)
            range = 1.0f;
        range = 256.0f / range;
        REGB_CK(launch_otsu_hist(d_img, n, mn, range, hist.p, st));
        count_launch();
        unsigned h[256];
        REGB_CK(cudaMemcpyAsync(h, hist.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        REGB_CK(cudaStreamSynchronize(st));
        h[0] = 0;
        ot = otsu_from_hist(h, mn, mx);
    }
    // the median of the values above it, in voxel order (otsu.hpp:86-100)
    const long long nt = compact_tiles(n);
    DevBuf<unsigned> counts((size_t)nt + 1, st);
    DevBuf<float> above((size_t)std::max<long long>(n, 1), st);
    REGB_CK(launch_compact_above(d_img, n, ot, counts.p, above.p, st));
    count_launch(3);
    unsigned m = 0;
    REGB_CK(cudaMemcpyAsync(&m, counts.p + nt, sizeof(m), cudaMemcpyDeviceToHost, st));
    REGB_CK(cudaStreamSynchronize(st));
    if (m == 0)
        return ot;
    std::vector<float> v;
    if (m < 2048) {
        v.resize(m);
        REGB_CK(cudaMemcpyAsync(v.data(), above.p, m * sizeof(float), cudaMemcpyDeviceToHost, st));
    } else {
        DevBuf<float> med(256, st);
        REGB_CK(launch_chunk_medians(above.p, m, med.p, st));
        count_launch();
        v.resize(256);
        REGB_CK(cudaMemcpyAsync(v.data(), med.p, 256 * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    REGB_CK(cudaStreamSynchronize(st));
    return middle(v);
}

// correlation(x, y) (numerical/statistics.hpp:569-598), or correlation_ygz (:600-619:
// only the voxels with y > 0): means, deviations and covariance in double from the
// exact integer sums (the reference widens its sums the same way).
double correlation_u8(const uint8_t* d_x, const uint8_t* d_y, long long n, bool masked, cudaStream_t st)
{
    DevBuf<unsigned long long> m(6, st);
    REGB_CK(launch_moments_u8(d_x, d_y, n, masked ? 1 : 0, m.p, st));
    count_launch();
    unsigned long long h[6];
    REGB_CK(cudaMemcpyAsync(h, m.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    REGB_CK(cudaStreamSynchronize(st));
    if (h[5] == 0)
        return 0.0;
    const double dn = (double)h[5], mx = (double)h[0] / dn, my = (double)h[1] / dn;
    const double vx = (double)h[2] / dn - mx * mx, vy = (double)h[3] / dn - my * my;
    const double sd1 = vx > 0.0 ? std::sqrt(vx) : 0.0, sd2 = vy > 0.0 ? std::sqrt(vy) : 0.0;
    if (sd1 == 0 || sd2 == 0)
        return 0.0;
    return ((double)h[4] / dn - mx * my) / sd1 / sd2;
}

void subject_image_pre(const float* d_in, const int* dim, uint8_t* d_out, cudaStream_t st)
{
    const long long n = (long long)dim[0] * dim[1] * dim[2];
    const float upper = 255.99f;
    DevBuf<float> g((size_t)n, st);
    gaussian(d_in, dim, 1, g.p, st);
    const float ot = otsu_median(g.p, n, st);
    // normalize_otsu_median (otsu.hpp:126-135); a zero median leaves the image as it is
    const float s = (ot == 0.0f) ? 1.0f : upper * 0.5f / ot;
    int shift = 0;
    if (ot != 0.0f) {
        DevBuf<unsigned long long> cnt(1, st);
        REGB_CK(launch_positive_count(g.p, n, s, cnt.p, st));
        count_launch();
        unsigned long long pos = 0;
        REGB_CK(cudaMemcpyAsync(&pos, cnt.p, sizeof(pos), cudaMemcpyDeviceToHost, st));
        REGB_CK(cudaStreamSynchronize(st));
        shift = ((double)pos > 0.5 * (double)n) ? 1 : 0;
    }
    REGB_CK(launch_otsu_normalize(g.p, n, s, shift, upper * 0.1f, ot == 0.0f ? 255.0f : upper, d_out, st));
    count_launch();
}

}  // namespace regb
