/* Test infrastructure only (the checker, never the product path).
 *
 * The reference's CDM at dimension 2 -- tipl::reg::cdm over 2-D uint8 images, whose
 * GPU instantiation is cdm_cuda<tipl::out, unsigned char, 2> (reg/cdm_cu.hpp:12-17) --
 * restated in plain C.  Fields are interleaved (x, y) floats (tipl::vector<2>).
 * Included by oracle.c after the uint8 instantiations of oracle_core.h and
 * oracle_cdm.h, whose regress_u8 (linear_regression) and cdm_improved_u8 it uses.
 */

/* interpolator::linear<2>::get_location (numerical/interpolation.hpp:274-305): cell
 * test and weights n0*n1, p0*n1, n0*p1, p0*p1 of the 2x2 cell. */
static int orc2_cell(const int* dim, float x, float y, size_t* d, float* r)
{
    if (x < 0 || y < 0)
        return 0;
    size_t ix = (size_t)x, iy = (size_t)y, w = (size_t)dim[0];
    if (ix + 1 >= w || iy + 1 >= (size_t)dim[1])
        return 0;
    d[0] = iy * w + ix;
    d[1] = d[0] + 1;
    d[2] = d[0] + w;
    d[3] = d[2] + 1;
    float p0 = x - (float)ix, p1 = y - (float)iy;
    float n0 = 1.0f - p0, n1 = 1.0f - p1;
    r[0] = n0 * n1;
    r[1] = p0 * n1;
    r[2] = n0 * p1;
    r[3] = p0 * p1;
    return 1;
}

/* estimate<linear> of a uint8 image (interpolation.hpp:61-73 weighted_sum, 28-34
 * assign): 0 and *out untouched where the cell test fails. */
static int orc2_bilinear_u8(const uint8_t* I, const int* dim, float x, float y, uint8_t* out)
{
    size_t d[4];
    float r[4];
    if (!orc2_cell(dim, x, y, d, r))
        return 0;
    float acc = (float)I[d[0]] * r[0];
    for (int i = 1; i < 4; ++i) {
        float v = (float)I[d[i]];
        v *= r[i];
        acc += v;
    }
    *out = (uint8_t)(acc <= 0.0f ? 0 : (uint8_t)acc);
    return 1;
}

/* estimate<linear> of a vector<2> image: components accumulated as the scalar case. */
static int orc2_bilinear_vec(const float* I, const int* dim, float x, float y, float* out)
{
    size_t d[4];
    float r[4];
    if (!orc2_cell(dim, x, y, d, r))
        return 0;
    for (int c = 0; c < 2; ++c) {
        float acc = I[2 * d[0] + c] * r[0];
        for (int i = 1; i < 4; ++i) {
            float v = I[2 * d[i] + c];
            v *= r[i];
            acc += v;
        }
        out[c] = acc;
    }
    return 1;
}

/* downsample_with_padding (numerical/resampling.hpp:575-603) at dimension 2: the
 * 2x2 mean with a missing +1 neighbour replaced by the nearest present one, the
 * integer sum shifted by 2. */
void orc2_downsample_u8(const uint8_t* in, const int* dim, uint8_t* out)
{
    int od[2] = {(dim[0] + 1) / 2, (dim[1] + 1) / 2};
    size_t w = dim[0];
    size_t shift[4] = {0, 1, w, 1 + w};
    size_t o = 0;
    for (int y = 0; y < od[1]; ++y)
        for (int x = 0; x < od[0]; ++x, ++o) {
            int x2 = 2 * x, y2 = 2 * y;
            int has = 0;
            if (x2 + 1 < dim[0]) has += 1;
            if (y2 + 1 < dim[1]) has += 2;
            size_t base = (size_t)y2 * dim[0] + x2;
            uint8_t buf[4];
            unsigned int acc = buf[0] = in[base];
            for (int i = 1; i < 4; ++i) {
                int h = has & i;
                acc += (buf[i] = (h == i) ? in[base + shift[i]] : buf[h]);
            }
            out[o] = (uint8_t)(acc >> 2);
        }
}

/* best_d *= 2 then upsample_with_padding (reg/cdm.hpp:402-403,
 * numerical/resampling.hpp:849-859) at dimension 2: out(x, y) = bilinear(2*in,
 * (x, y)*0.5), zero where the sample fails. */
void orc2_upsample_field_x2(const float* in, const int* in_dim, float* out, const int* out_dim)
{
    long long nin = 2LL * in_dim[0] * in_dim[1];
    float* d2 = (float*)malloc(sizeof(float) * nin);
    for (long long i = 0; i < nin; ++i)
        d2[i] = in[i] * 2.0f;
    long long i = 0;
    for (int y = 0; y < out_dim[1]; ++y)
        for (int x = 0; x < out_dim[0]; ++x, ++i) {
            float o[2] = {0, 0};
            float vx = (float)x, vy = (float)y;
            vx *= 0.5f;
            vy *= 0.5f;
            orc2_bilinear_vec(d2, in_dim, vx, vy, o);
            out[2 * i] = o[0];
            out[2 * i + 1] = o[1];
        }
    free(d2);
}

/* compose_displacement (numerical/dif.hpp:90-107) at dimension 2: Js = Is where the
 * displacement is zero, else the bilinear sample at (x, y) + d; failed samples 0. */
void orc2_compose_u8(const uint8_t* Is, const int* dim, const float* d, uint8_t* Js)
{
    long long i = 0;
    for (int y = 0; y < dim[1]; ++y)
        for (int x = 0; x < dim[0]; ++x, ++i) {
            Js[i] = 0;
            if (d[2 * i] == 0.0f && d[2 * i + 1] == 0.0f)
                Js[i] = Is[i];
            else {
                float px = (float)x, py = (float)y;
                px += d[2 * i];
                py += d[2 * i + 1];
                orc2_bilinear_u8(Is, dim, px, py, Js + i);
            }
        }
}

/* get_window_at_width<2> (numerical/window.hpp:76-91 with iterate_xy / iterate_x):
 * the clipped 5x5 window in the reference's visiting order (rows y..y+2 then
 * y-1, y-2; in each row x..x+2 then x-1, x-2).  Returns the count. */
static int orc2_window5(const uint8_t* I, const int* dim, int x, int y, uint8_t* out)
{
    int xu = dim[0] - x - 1, yu = dim[1] - y - 1, xl = x, yl = y;
    if (xu > 2) xu = 2;
    if (yu > 2) yu = 2;
    if (xl > 2) xl = 2;
    if (yl > 2) yl = 2;
    int n = 0;
    long long w = dim[0], idx = (long long)y * w + x;
    for (int pass = 0; pass < 2; ++pass) {
        int lo = pass ? 1 : 0, hi = pass ? yl : yu;
        for (int dy = lo; dy <= hi; ++dy) {
            long long row = idx + (pass ? -dy : dy) * w;
            for (int dx = 0; dx <= xu; ++dx)
                out[n++] = I[row + dx];
            for (int dx = 1; dx <= xl; ++dx)
                out[n++] = I[row - dx];
        }
    }
    return n;
}

/* cdm_get_gradient (reg/cdm.hpp:46-106) at dimension 2; gradient_at's 2-D form
 * (numerical/numerical.hpp:111-116).  new_d (2 per pixel) is overwritten with the
 * term; returns mean(cost_map) as float. */
float orc2_cdm_gradient_u8(const uint8_t* Js, const uint8_t* It, const int* dim, float* new_d, int gradient_type)
{
    size_t n = (size_t)dim[0] * dim[1], w = (size_t)dim[0];
    for (size_t i = 0; i < 2 * n; ++i)
        new_d[i] = 0;
    double cost_sum = 0.0;
    uint8_t wj[25], wi[25];
    size_t pos = 0;
    for (int y = 0; y < dim[1]; ++y)
        for (int x = 0; x < dim[0]; ++x, ++pos) {
            float cost = 0;
            float* nd = new_d + 2 * pos;
            float g[2];
            g[0] = (x + 1 < dim[0] && x) ? (float)(Js[pos + 1] - Js[pos - 1]) : 0.0f;
            g[1] = (y + 1 < dim[1] && y) ? (float)(Js[pos + w] - Js[pos - w]) : 0.0f;
            if (gradient_type == 'd') {
                int dif = (int)Js[pos] - (int)It[pos];
                g[0] *= dif;
                g[1] *= dif;
                nd[0] += g[0];
                nd[1] += g[1];
                cost = (float)(dif * dif);
            } else {
                if (Js[pos] == 0 || It[pos] == 0)
                    continue;
                orc2_window5(It, dim, x, y, wi);
                int m = orc2_window5(Js, dim, x, y, wj);
                float a, b, r2;
                regress_u8(wj, wi, m, &a, &b, &r2);
                if (a > 0) {
                    float s = r2 * ((float)Js[pos] * a + b - (float)It[pos]);
                    g[0] *= s;
                    g[1] *= s;
                    nd[0] += g[0];
                    nd[1] += g[1];
                    cost = -r2;
                }
            }
            cost_sum += (double)cost;
        }
    return (float)(cost_sum / (double)n);
}

/* cdm_solve_poisson (reg/cdm.hpp:158-198) at dimension 2: solve = new_d * (-1/4);
 * 12 sweeps of (new_d - s[-1] - s[+1] - s[-w] - s[+w]) * (-1/4) with flat-index
 * neighbours and flat-index bounds.  The result replaces new_d. */
void orc2_cdm_poisson(float* new_d, const int* dim, int sweeps)
{
    long long n = (long long)dim[0] * dim[1], w = dim[0];
    const float inv_d2 = -0.5f / 2.0f;
    float* s = (float*)malloc(sizeof(float) * 2 * n);
    float* t = (float*)malloc(sizeof(float) * 2 * n);
    for (long long i = 0; i < 2 * n; ++i)
        s[i] = new_d[i] * inv_d2;
    for (int it = 0; it < sweeps; ++it) {
        for (long long p = 0; p < n; ++p)
            for (int c = 0; c < 2; ++c) {
                float v = new_d[2 * p + c];
                if (p >= 1) v -= s[2 * (p - 1) + c];
                if (p < n - 1) v -= s[2 * (p + 1) + c];
                if (p >= w) v -= s[2 * (p - w) + c];
                if (p < n - w) v -= s[2 * (p + w) + c];
                v *= inv_d2;
                t[2 * p + c] = v;
            }
        float* x = s;
        s = t;
        t = x;
    }
    memcpy(new_d, s, sizeof(float) * 2 * n);
    free(s);
    free(t);
}

/* cdm_max_displacement_length (reg/cdm.hpp:260-280): max of vector<2>::length(),
 * sqrt of the float x*x + y*y (utility/pixel_index.hpp:340). */
float orc2_cdm_max_len(const float* d, const int* dim)
{
    long long n = (long long)dim[0] * dim[1];
    float m = 0;
    for (long long i = 0; i < n; ++i) {
        float l = sqrtf(d[2 * i] * d[2 * i] + d[2 * i + 1] * d[2 * i + 1]);
        if (l > m)
            m = l;
    }
    return m;
}

/* accumulate_displacement (numerical/dif.hpp:166-186) with displacement_to_mapping
 * (dif.hpp:19-28) at dimension 2: mapping = cur_d + (x, y); where new_d != 0 and
 * (x, y) + new_d samples inside, new_d = mapping(sample) - (x, y), else cur_d. */
void orc2_accumulate(const float* cur_d, float* new_d, const int* dim)
{
    long long n = (long long)dim[0] * dim[1];
    float* map = (float*)malloc(sizeof(float) * 2 * n);
    long long i = 0;
    for (int y = 0; y < dim[1]; ++y)
        for (int x = 0; x < dim[0]; ++x, ++i) {
            map[2 * i] = cur_d[2 * i] + (float)x;
            map[2 * i + 1] = cur_d[2 * i + 1] + (float)y;
        }
    i = 0;
    for (int y = 0; y < dim[1]; ++y)
        for (int x = 0; x < dim[0]; ++x, ++i) {
            float* nd = new_d + 2 * i;
            float dx = nd[0], dy = nd[1];
            int ok = 0;
            if (dx != 0 || dy != 0) {
                dx += (float)x;
                dy += (float)y;
                float o[2];
                if (orc2_bilinear_vec(map, dim, dx, dy, o)) {
                    nd[0] = o[0] - (float)x;
                    nd[1] = o[1] - (float)y;
                    ok = 1;
                }
            }
            if (!ok) {
                nd[0] = cur_d[2 * i];
                nd[1] = cur_d[2 * i + 1];
            }
        }
    free(map);
}

/* cdm_smooth (reg/cdm.hpp:302-342) at dimension 2: dd = d*(1-s) + (s/4)*(d[+1] +
 * d[-1] + d[+w] + d[-w]) by flat index; a zero smoothing leaves dd untouched. */
void orc2_cdm_smooth(const float* d, float* dd, const int* dim, float smoothing)
{
    if (smoothing == 0)
        return;
    long long n = (long long)dim[0] * dim[1], w = dim[0];
    float w_6 = smoothing / (2.0f * 2);
    float w_1 = 1.0f - smoothing;
    for (long long p = 0; p < n; ++p)
        for (int c = 0; c < 2; ++c) {
            float v = 0;
            if (p + 1 < n) v += d[2 * (p + 1) + c];
            if (p >= 1) v += d[2 * (p - 1) + c];
            if (p + w < n) v += d[2 * (p + w) + c];
            if (p >= w) v += d[2 * (p - w) + c];
            v *= w_6;
            dd[2 * p + c] = d[2 * p + c] * w_1 + v;
        }
}

/* cdm(It, Is, best_d, terminated, param) (reg/cdm.hpp:373-474) at dimension 2 over
 * nmod modality pairs of one shape (dim[0] x dim[1]); the loop is the 3-D driver's
 * (oracle_cdm.h), the pyramid recurses while min(w, h) > min_dimension.  best_d holds
 * 2 * w * h zeroed floats.  Returns 0 where the reference returns false. */
int orc2_cdm_multi_u8(const uint8_t* const* It, const uint8_t* const* Is, int nmod, const int* dim, float* best_d,
                      float resolution, float speed, float smoothing, unsigned int min_dimension, const char* gtypes,
                      int* iters_out)
{
    long long n = (long long)dim[0] * dim[1];
    int ntype = gtypes ? (int)strlen(gtypes) : 0;
    int mn = dim[0] < dim[1] ? dim[0] : dim[1];
    if ((unsigned int)mn > min_dimension) {
        int rd[2] = {(dim[0] + 1) / 2, (dim[1] + 1) / 2};
        long long rn = (long long)rd[0] * rd[1];
        uint8_t** rIt = (uint8_t**)malloc(sizeof(uint8_t*) * nmod);
        uint8_t** rIs = (uint8_t**)malloc(sizeof(uint8_t*) * nmod);
        for (int i = 0; i < nmod; ++i) {
            rIt[i] = (uint8_t*)malloc(rn);
            rIs[i] = (uint8_t*)malloc(rn);
            orc2_downsample_u8(It[i], dim, rIt[i]);
            orc2_downsample_u8(Is[i], dim, rIs[i]);
        }
        float* rfield = (float*)calloc(2 * rn, sizeof(float));
        int ok = orc2_cdm_multi_u8((const uint8_t* const*)rIt, (const uint8_t* const*)rIs, nmod, rd, rfield,
                                   resolution / 2.0f, speed, smoothing, min_dimension, gtypes, iters_out);
        for (int i = 0; i < nmod; ++i) {
            free(rIt[i]);
            free(rIs[i]);
        }
        free(rIt);
        free(rIs);
        if (!ok) {
            free(rfield);
            return 0;
        }
        orc2_upsample_field_x2(rfield, rd, best_d, dim);
        free(rfield);
        if (resolution > 1.0f)
            return 1;
    }
    float theta = 0;
    float cost[8];
    int ncost = 0;
    float best_cost = 3.402823466e+38f;
    float* cur_d = (float*)malloc(sizeof(float) * 2 * n);
    float* new_d = (float*)malloc(sizeof(float) * 2 * n);
    float* dd = nmod > 1 ? (float*)malloc(sizeof(float) * 2 * n) : NULL;
    uint8_t* Js = (uint8_t*)malloc(n);
    memcpy(cur_d, best_d, sizeof(float) * 2 * n);
    float cur_smoothing = 0.8f;
    int ok = 1;
    for (unsigned int index = 0; index < 200 && ok; ++index) {
        float sum_cost = 0;
        for (int i = 0; i < nmod; ++i) {
            orc2_compose_u8(Is[i], dim, cur_d, Js);
            float* out = i ? dd : new_d;
            sum_cost += orc2_cdm_gradient_u8(Js, It[i], dim, out, i < ntype ? gtypes[i] : 'r');
            if (sum_cost == 0) {
                ok = 0;
                break;
            }
            if (i)
                for (long long k = 0; k < 2 * n; ++k)
                    new_d[k] += dd[k];
        }
        if (!ok)
            break;
        if (iters_out)
            ++*iters_out;
        cost[ncost++] = sum_cost / (float)nmod;
        if (cost[ncost - 1] < best_cost) {
            best_cost = cost[ncost - 1];
            if (index)
                memcpy(best_d, cur_d, sizeof(float) * 2 * n);
        }
        if (!cdm_improved_u8(cost, &ncost)) {
            if (cur_smoothing <= smoothing)
                break;
            memcpy(cur_d, best_d, sizeof(float) * 2 * n);
            cur_smoothing *= 0.5f;
            ncost = 0;
        }
        orc2_cdm_poisson(new_d, dim, 12);
        if (theta == 0)
            theta = orc2_cdm_max_len(new_d, dim);
        if (theta == 0)
            break;
        const float sc = speed / theta;
        for (long long k = 0; k < 2 * n; ++k)
            new_d[k] *= sc;
        orc2_accumulate(cur_d, new_d, dim);
        orc2_cdm_smooth(new_d, cur_d, dim, cur_smoothing);
    }
    free(cur_d);
    free(new_d);
    free(dd);
    free(Js);
    return ok;
}
