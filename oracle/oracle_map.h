/* Test infrastructure only (the checker, never the product path).
 *
 * Plain-C restatement of the mapping steps of the mm_reg pipeline
 * (reg/mm_reg.hpp:271-345): displacement_to_mapping with an affine
 * (numerical/dif.hpp:42-51), inv_displacement_to_mapping (:53-66), compose_mapping
 * for uint8 images (:70-80), and the Pearson correlation of two uint8 images
 * (numerical/statistics.hpp:569-598).  Included once by oracle.c after the float
 * field instantiation (trilinear_vec_f32).
 */

/* mapping[i] = T(dis[i] + index): the component sums in float, then the transform
 * ((v0*r0 + v1*r1) + v2*r2) + s (numerical/transformation.hpp:58-73, 846-850). */
void orc_displacement_to_mapping_f32(const float* dis, const int* dim, const float* T, float* mapping)
{
    size_t i = 0;
    for (int z = 0; z < dim[2]; ++z)
        for (int y = 0; y < dim[1]; ++y)
            for (int x = 0; x < dim[0]; ++x, ++i) {
                const float v0 = dis[3 * i] + (float)x, v1 = dis[3 * i + 1] + (float)y, v2 = dis[3 * i + 2] + (float)z;
                for (int a = 0; a < 3; ++a)
                    mapping[3 * i + a] = v0 * T[3 * a] + v1 * T[3 * a + 1] + v2 * T[3 * a + 2] + T[9 + a];
            }
}

/* inv_mapping[i] = p + estimate(inv_dis, p), p = T^-1(index) over the inv_mapping grid;
 * the estimate is the zero vector where the 2x2x2 cell leaves inv_dis. */
void orc_inv_displacement_to_mapping_f32(const float* inv_dis, const int* dis_dim, const float* T,
                                         const int* map_dim, float* inv_mapping)
{
    float iT[12];
    memcpy(iT, T, sizeof(iT));
    orc_matrix_inverse(iT);
    size_t i = 0;
    for (int z = 0; z < map_dim[2]; ++z)
        for (int y = 0; y < map_dim[1]; ++y)
            for (int x = 0; x < map_dim[0]; ++x, ++i) {
                float p[3], dv[3] = {0.0f, 0.0f, 0.0f};
                for (int a = 0; a < 3; ++a)
                    p[a] = (float)x * iT[3 * a] + (float)y * iT[3 * a + 1] + (float)z * iT[3 * a + 2] + iT[9 + a];
                trilinear_vec_f32(inv_dis, dis_dim, p[0], p[1], p[2], dv);
                for (int a = 0; a < 3; ++a)
                    inv_mapping[3 * i + a] = p[a] + dv[a];
            }
}

/* to[i] = trilinear(from, mapping[i]) with the uint8 assign, 0 where the cell leaves from */
void orc_compose_mapping_u8(const uint8_t* from, const int* fdim, const float* mapping, const int* mdim, uint8_t* to)
{
    const size_t n = (size_t)mdim[0] * mdim[1] * mdim[2];
    for (size_t i = 0; i < n; ++i) {
        uint8_t v = 0;
        if (!trilinear_u8(from, fdim, mapping[3 * i], mapping[3 * i + 1], mapping[3 * i + 2], &v))
            v = 0;
        to[i] = v;
    }
}

/* correlation(x, y) of two uint8 images (numerical/statistics.hpp:569-598): means,
 * standard deviations and covariance in double from exact integer sums; 0 when either
 * deviation is 0. */
double orc_correlation_u8(const uint8_t* x, const uint8_t* y, long long n)
{
    long long sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0;
    for (long long i = 0; i < n; ++i) {
        sx += x[i];
        sy += y[i];
        sxx += (long long)x[i] * x[i];
        syy += (long long)y[i] * y[i];
        sxy += (long long)x[i] * y[i];
    }
    const double dn = (double)n, mx = (double)sx / dn, my = (double)sy / dn;
    const double vx = (double)sxx / dn - mx * mx, vy = (double)syy / dn - my * my;
    const double sd1 = vx > 0.0 ? sqrt(vx) : 0.0, sd2 = vy > 0.0 ? sqrt(vy) : 0.0;
    if (sd1 == 0 || sd2 == 0)
        return 0.0;
    return ((double)sxy / dn - mx * my) / sd1 / sd2;
}

/* correlation_ygz (numerical/statistics.hpp:600-619): correlation over the voxels with y > 0 */
double orc_correlation_ygz_u8(const uint8_t* x, const uint8_t* y, long long n)
{
    if (n <= 0)
        return 0.0;
    uint8_t* nx = (uint8_t*)malloc((size_t)n);
    uint8_t* ny = (uint8_t*)malloc((size_t)n);
    long long m = 0;
    for (long long i = 0; i < n; ++i)
        if (y[i] > 0) {
            nx[m] = x[i];
            ny[m] = y[i];
            ++m;
        }
    double r = m ? orc_correlation_u8(nx, ny, m) : 0.0;
    free(nx);
    free(ny);
    return r;
}

/* It_match_fov (reg/mm_reg.hpp:313-329): 0 where T(x) is outside a volume of mdim
 * (shape::is_valid, utility/shape.hpp:116-122) */
void orc_match_fov_u8(const uint8_t* It, const int* fdim, const float* T, const int* mdim, uint8_t* out)
{
    size_t i = 0;
    for (int z = 0; z < fdim[2]; ++z)
        for (int y = 0; y < fdim[1]; ++y)
            for (int x = 0; x < fdim[0]; ++x, ++i) {
                float p[3];
                apply_T_u8(T, (float)x, (float)y, (float)z, p);
                int ok = 1;
                for (int a = 0; a < 3; ++a)
                    if (p[a] < 0 || p[a] >= (float)(unsigned)mdim[a])
                        ok = 0;
                out[i] = ok ? It[i] : 0;
            }
}
