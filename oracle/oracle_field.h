/* Test infrastructure only (the checker, never the product path).
 *
 * Displacement-field passes of the reference's CDM iteration, restated in plain C.
 * Included by oracle.c with R = float (suffix _f32, reference-exact) and
 * R = double (suffix _f64, error reporting).  A field is AoS xyz, x-fastest,
 * index = (z*h + y)*w + x (utility/basic_image.hpp:160-161).
 */
#ifndef FSFX
#error "define FSFX and R before including"
#endif

#define FCAT_(a, b) a##b
#define FCAT(a, b) FCAT_(a, b)
#define FF(name) FCAT(name, FSFX)

/* linear<3> estimate on a vector image (numerical/interpolation.hpp:337-383,
 * 61-73 with interp_type<vector>): the same cell test and weights as the scalar
 * case, components accumulated independently in the same order. */
static int FF(trilinear_vec)(const R* I, const int* dim, R x, R y, R z, R* out)
{
    if (x < 0 || y < 0 || z < 0)
        return 0;
    size_t ix = (size_t)x, iy = (size_t)y, iz = (size_t)z;
    size_t w = (size_t)dim[0];
    if (ix + 1 >= w || iy + 1 >= (size_t)dim[1] || iz + 1 >= (size_t)dim[2])
        return 0;
    R p0 = x - (R)ix, p1 = y - (R)iy, p2 = z - (R)iz;
    R n0 = (R)1 - p0, n1 = (R)1 - p1, n2 = (R)1 - p2;
    size_t wh = w * (size_t)dim[1];
    size_t d0 = iz * wh + iy * w + ix;
    size_t d[8] = {d0, d0 + 1, d0 + w, d0 + w + 1, d0 + wh, d0 + 1 + wh, d0 + w + wh, d0 + w + 1 + wh};
    R n0n1 = n0 * n1, p0n1 = p0 * n1, n0p1 = n0 * p1, p0p1 = p0 * p1;
    R r[8] = {n0n1 * n2, p0n1 * n2, n0p1 * n2, p0p1 * n2, n0n1 * p2, p0n1 * p2, n0p1 * p2, p0p1 * p2};
    for (int c = 0; c < 3; ++c) {
        R acc = I[3 * d[0] + c] * r[0];
        for (int i = 1; i < 8; ++i) {
            R v = I[3 * d[i] + c];
            v *= r[i];
            acc += v;
        }
        out[c] = acc;
    }
    return 1;
}

/* cdm_solve_poisson CPU (reg/cdm.hpp:158-198): solve = new_d * (-1/6); then 12
 * Jacobi sweeps solve' = (new_d - s[-1] - s[+1] - s[-w] - s[+w] - s[-wh] - s[+wh]) * (-1/6),
 * neighbours taken by flat index with bounds on the flat index only, so the
 * x/y edges wrap into the previous/next row or plane.  Result replaces new_d. */
void FF(orc_cdm_poisson)(R* new_d, const int* dim, int sweeps)
{
    long long n = (long long)dim[0] * dim[1] * dim[2];
    long long w = dim[0], wh = (long long)dim[0] * dim[1];
    const R inv_d2 = (R)(-0.5f / 3.0f);
    R* s = (R*)malloc(sizeof(R) * 3 * n);
    R* t = (R*)malloc(sizeof(R) * 3 * n);
    for (long long i = 0; i < 3 * n; ++i)
        s[i] = new_d[i] * inv_d2;
    for (int it = 0; it < sweeps; ++it) {
        for (long long p = 0; p < n; ++p)
            for (int c = 0; c < 3; ++c) {
                R v = new_d[3 * p + c];
                if (p >= 1) v -= s[3 * (p - 1) + c];
                if (p < n - 1) v -= s[3 * (p + 1) + c];
                if (p >= w) v -= s[3 * (p - w) + c];
                if (p < n - w) v -= s[3 * (p + w) + c];
                if (p >= wh) v -= s[3 * (p - wh) + c];
                if (p < n - wh) v -= s[3 * (p + wh) + c];
                v *= inv_d2;
                t[3 * p + c] = v;
            }
        R* tmp = s;
        s = t;
        t = tmp;
    }
    for (long long i = 0; i < 3 * n; ++i)
        new_d[i] = s[i];
    free(s);
    free(t);
}

/* cdm_max_displacement_length (reg/cdm.hpp:260-284): max over voxels of
 * sqrt(double(x*x + y*y + z*z)) with the squared length formed in R. */
R FF(orc_cdm_max_len)(const R* d, const int* dim)
{
    long long n = (long long)dim[0] * dim[1] * dim[2];
    R m = 0;
    for (long long i = 0; i < n; ++i) {
        R x = d[3 * i], y = d[3 * i + 1], z = d[3 * i + 2];
        R l2 = x * x + y * y + z * z;
        R l = (R)sqrt((double)l2);
        if (l > m)
            m = l;
    }
    return m;
}

/* field *= c (numerical/numerical.hpp multiply_constant / vector::operator*=). */
void FF(orc_field_scale)(R* d, const int* dim, R c)
{
    long long n = 3LL * dim[0] * dim[1] * dim[2];
    for (long long i = 0; i < n; ++i)
        d[i] *= c;
}

/* accumulate_displacement CPU (numerical/dif.hpp:166-186) with
 * displacement_to_mapping (dif.hpp:19-28): mapping = cur_d + x; for each voxel
 * with new_d != 0 whose x + new_d samples inside the volume,
 * new_d = mapping(x + new_d) - x; otherwise new_d = cur_d. */
void FF(orc_accumulate)(const R* cur_d, R* new_d, const int* dim)
{
    long long n = (long long)dim[0] * dim[1] * dim[2];
    R* map = (R*)malloc(sizeof(R) * 3 * n);
    long long i = 0;
    for (int z = 0; z < dim[2]; ++z)
        for (int y = 0; y < dim[1]; ++y)
            for (int x = 0; x < dim[0]; ++x, ++i) {
                map[3 * i] = cur_d[3 * i] + (R)x;
                map[3 * i + 1] = cur_d[3 * i + 1] + (R)y;
                map[3 * i + 2] = cur_d[3 * i + 2] + (R)z;
            }
    i = 0;
    for (int z = 0; z < dim[2]; ++z)
        for (int y = 0; y < dim[1]; ++y)
            for (int x = 0; x < dim[0]; ++x, ++i) {
                R* nd = new_d + 3 * i;
                R dx = nd[0], dy = nd[1], dz = nd[2];
                int ok = 0;
                if (dx != 0 || dy != 0 || dz != 0) {
                    dx += (R)x;
                    dy += (R)y;
                    dz += (R)z;
                    R o[3];
                    if (FF(trilinear_vec)(map, dim, dx, dy, dz, o)) {
                        nd[0] = o[0] - (R)x;
                        nd[1] = o[1] - (R)y;
                        nd[2] = o[2] - (R)z;
                        ok = 1;
                    }
                }
                if (!ok) {
                    nd[0] = cur_d[3 * i];
                    nd[1] = cur_d[3 * i + 1];
                    nd[2] = cur_d[3 * i + 2];
                }
            }
    free(map);
}

/* cdm_smooth CPU (reg/cdm.hpp:302-342): dd = d*(1-s) + (s/6)*sum of the six
 * flat-index neighbours, summed in the order +1, -1, +w, -w, +wh, -wh.  A zero
 * smoothing leaves dd untouched. */
void FF(orc_cdm_smooth)(const R* d, R* dd, const int* dim, R smoothing)
{
    if (smoothing == 0)
        return;
    long long n = (long long)dim[0] * dim[1] * dim[2];
    long long w = dim[0], wh = (long long)dim[0] * dim[1];
    R w_6 = smoothing / (R)(2.0f * 3);
    R w_1 = (R)1 - smoothing;
    for (long long p = 0; p < n; ++p)
        for (int c = 0; c < 3; ++c) {
            R v = 0;
            if (p + 1 < n) v += d[3 * (p + 1) + c];
            if (p >= 1) v += d[3 * (p - 1) + c];
            if (p + w < n) v += d[3 * (p + w) + c];
            if (p >= w) v += d[3 * (p - w) + c];
            if (p + wh < n) v += d[3 * (p + wh) + c];
            if (p >= wh) v += d[3 * (p - wh) + c];
            v *= w_6;
            dd[3 * p + c] = d[3 * p + c] * w_1 + v;
        }
}

/* best_d *= 2 then upsample_with_padding(best_d, shape) (reg/cdm.hpp:402-403,
 * numerical/resampling.hpp:849-859,885-891): out(x) = trilinear(2*in, x*0.5),
 * zero where the sample fails. */
void FF(orc_upsample_field_x2)(const R* in, const int* in_dim, R* out, const int* out_dim)
{
    long long nin = 3LL * in_dim[0] * in_dim[1] * in_dim[2];
    R* d2 = (R*)malloc(sizeof(R) * nin);
    for (long long i = 0; i < nin; ++i)
        d2[i] = in[i] * (R)2;
    long long i = 0;
    for (int z = 0; z < out_dim[2]; ++z)
        for (int y = 0; y < out_dim[1]; ++y)
            for (int x = 0; x < out_dim[0]; ++x, ++i) {
                R o[3] = {0, 0, 0};
                R vx = (R)x, vy = (R)y, vz = (R)z;
                vx *= (R)0.5f;
                vy *= (R)0.5f;
                vz *= (R)0.5f;
                FF(trilinear_vec)(d2, in_dim, vx, vy, vz, o);
                out[3 * i] = o[0];
                out[3 * i + 1] = o[1];
                out[3 * i + 2] = o[2];
            }
    free(d2);
}

#undef FF
#undef FCAT
#undef FCAT_
