/* Test infrastructure only (the checker, never the product path).
 *
 * Plain-C restatement of the mask-moment initialisation tipl::reg::linear runs
 * before an affine search (reg/linear.hpp:658-684): has_mask, estimate_affine_param
 * and the conversion of the search's matrix back to an affine_param
 * (transformation_matrix::to_affine_param).  Included once by oracle.c.
 *
 * Types follow the reference exactly: coordinate products are float (int * float),
 * sums and moments double, the 3x3 QR of to_affine_param float with a double Q.
 */
#include <math.h>

/* bounding_box(I, min, max, background = 0) (numerical/basic_op.hpp:697-730) and
 * has_mask (numerical/basic_op.hpp:811-830). */
int orc_has_mask_u8(const uint8_t* img, const int* dim)
{
    const int w = dim[0], h = dim[1], d = dim[2];
    const size_t sz = (size_t)w * h * d;
    const size_t threshold = sz / 5;
    size_t zero_count = 0;
    for (size_t i = 0; i < sz && zero_count <= threshold; ++i)
        if (img[i] == 0)
            ++zero_count;
    if (zero_count > threshold)
        return 1;
    int shape[3] = {w, h, d}, rmin[3], rmax[3];
    for (int k = 0; k < 3; ++k) {
        rmin[k] = shape[k] - 1;
        rmax[k] = 0;
    }
    size_t i = 0;
    for (int z = 0; z < d; ++z)
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x, ++i) {
                if (img[i] <= 0)
                    continue;
                const int p[3] = {x, y, z};
                for (int k = 0; k < 3; ++k) {
                    if (p[k] < rmin[k]) rmin[k] = p[k];
                    if (p[k] > rmax[k]) rmax[k] = p[k];
                }
            }
    for (int k = 0; k < 3; ++k) {
        if (rmax[k] == 0)
            rmax[k] = rmin[k] = 0;
        ++rmax[k];
    }
    for (int k = 0; k < 3; ++k)
        if (rmin[k] > 0 && rmax[k] < shape[k])
            return 1;
    return 0;
}

/* compute_moments of estimate_affine_param (numerical/transformation.hpp:943-982):
 * centroid and covariance of the voxels > 0, in physical units. */
static size_t orc_moments(const uint8_t* img, const int* dim, const float* vs, double* c, double* cov)
{
    const int w = dim[0], h = dim[1], d = dim[2];
    size_t sum = 0, i = 0;
    c[0] = c[1] = c[2] = 0.0;
    for (int z = 0; z < d; ++z)
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x, ++i)
                if (img[i] > 0) {
                    c[0] += x * vs[0];
                    c[1] += y * vs[1];
                    c[2] += z * vs[2];
                    ++sum;
                }
    if (sum == 0)
        return 0;
    for (int k = 0; k < 3; ++k)
        c[k] /= (double)sum;
    for (int k = 0; k < 9; ++k)
        cov[k] = 0.0;
    i = 0;
    for (int z = 0; z < d; ++z)
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x, ++i)
                if (img[i] > 0) {
                    const double dd[3] = {x * vs[0] - c[0], y * vs[1] - c[1], z * vs[2] - c[2]};
                    cov[0] += dd[0] * dd[0];
                    cov[1] += dd[0] * dd[1];
                    cov[2] += dd[0] * dd[2];
                    cov[4] += dd[1] * dd[1];
                    cov[5] += dd[1] * dd[2];
                    cov[8] += dd[2] * dd[2];
                }
    cov[3] = cov[1];
    cov[6] = cov[2];
    cov[7] = cov[5];
    for (int k = 0; k < 9; ++k)
        cov[k] /= (double)sum;
    return sum;
}

/* eigen_decomposition_sym for a symmetric 3x3 (numerical/matrix.hpp:1830-1955):
 * closed-form eigenvalues from the invariants, eigenvector i in V[3i..3i+2]. */
void orc_eigen_sym3(const double* A, double* V, double* d)
{
    int k;
    if (A[1] == 0.0) {
        if (A[2] == 0.0) {
            if (A[5] == 0.0) {
                d[0] = A[0];
                d[1] = A[4];
                d[2] = A[8];
                for (k = 0; k < 9; ++k) V[k] = 0.0;
                V[0] = V[4] = V[8] = 1.0;
                return;
            }
            double A5A5 = A[5] * A[5];
            d[0] = A[0];
            d[1] = d[2] = (A[4] + A[8]) * 0.5;
            double A4_A8 = (A[4] - A[8]) * 0.5;
            double l = sqrt(A4_A8 * A4_A8 + A5A5);
            d[1] += l;
            d[2] -= l;
            for (k = 0; k < 9; ++k) V[k] = 0.0;
            V[0] = 1.0;
            double A4_d1 = A[4] - d[1];
            double length = sqrt(A5A5 + A4_d1 * A4_d1);
            V[4] = V[8] = -A[5] / length;
            V[5] = A4_d1 / length;
            V[7] = -V[5];
            return;
        }
        if (A[5] == 0.0) {
            double A2A2 = A[2] * A[2];
            d[0] = A[4];
            d[1] = d[2] = (A[0] + A[8]) * 0.5;
            double A0_A8 = (A[0] - A[8]) * 0.5;
            double l = sqrt(A0_A8 * A0_A8 + A2A2);
            d[1] += l;
            d[2] -= l;
            for (k = 0; k < 9; ++k) V[k] = 0.0;
            V[1] = 1.0;
            double A0_d1 = A[0] - d[1];
            double length = sqrt(A2A2 + A0_d1 * A0_d1);
            V[3] = V[8] = -A[2] / length;
            V[5] = A0_d1 / length;
            V[6] = -V[5];
            return;
        }
    } else if (A[2] == 0.0 && A[5] == 0.0) {
        double A1A1 = A[1] * A[1];
        d[0] = A[8];
        d[1] = d[2] = (A[0] + A[4]) * 0.5;
        double A0_A4 = (A[0] - A[4]) * 0.5;
        double l = sqrt(A0_A4 * A0_A4 + A1A1);
        d[1] += l;
        d[2] -= l;
        for (k = 0; k < 9; ++k) V[k] = 0.0;
        V[2] = 1.0;
        double A0_d1 = A[0] - d[1];
        double length = sqrt(A1A1 + A0_d1 * A0_d1);
        V[3] = V[7] = -A[1] / length;
        V[4] = A0_d1 / length;
        V[6] = -V[4];
        return;
    }
    double A2A1 = A[2] * A[1];
    double A1A5 = A[1] * A[5];
    double A2A5 = A[2] * A[5];
    double A0A4 = A[0] * A[4];
    double A1A1 = A[1] * A[1];
    double A2A2 = A[2] * A[2];
    double A5A5 = A[5] * A[5];
    double A0_A4 = A[0] + A[4];
    {
        double I1 = A0_A4 + A[8];
        double I2 = A0A4 + A0_A4 * A[8] - A1A1 - A2A2 - A5A5;
        double I3 = A0A4 * A[8] + 2.0 * A2A1 * A[5] - (A[8] * A1A1 + A[4] * A2A2 + A[0] * A5A5);
        double I1_3 = (I1 / 3.0);
        double I1_3_I1_3 = I1_3 * I1_3;
        double v = I1_3_I1_3 - I2 / 3.0;
        double s = I1_3_I1_3 * I1_3 - I1 * I2 / 6.0 + I3 / 2.0;
        if (v == 0.0) {
            d[0] = d[1] = d[2] = 0.0;
            for (k = 0; k < 9; ++k) V[k] = 0.0;
            V[0] = V[4] = V[8] = 1.0;
            return;
        }
        double sqrt_v = sqrt(v);
        double r = s / v / sqrt_v;
        r = r < 1.0 ? r : 1.0;   /* std::min(1.0, r) */
        r = -1.0 < r ? r : -1.0; /* std::max(-1.0, r) */
        double angle = acos(r) / 3.0;
        d[0] = I1_3 + 2.0 * sqrt_v * cos(angle);
        d[1] = I1_3 - 2.0 * sqrt_v * cos(3.14159265358979323846 / 3.0 + angle);
        d[2] = I1 - d[0] - d[1];
    }
    for (int i = 0; i < 3; ++i, V += 3) {
        double Ai = A[0] - d[i];
        double Bi = A[4] - d[i];
        double Ci = A[8] - d[i];
        double q1 = (A2A1 - Ai * A[5]);
        double q2 = (A1A5 - Bi * A[2]);
        double q3 = (A2A5 - Ci * A[1]);
        V[0] = q2 * q3;
        V[1] = q3 * q1;
        V[2] = q2 * q1;
        double length = sqrt(V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
        V[0] /= length;
        V[1] /= length;
        V[2] /= length;
    }
}

/* determinant, 3x3 (numerical/matrix.hpp:1347-1353) */
static double orc_det3(const double* m)
{
    return m[0] * (m[4] * m[8] - m[5] * m[7]) + m[1] * (m[5] * m[6] - m[3] * m[8]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}

/* estimate_affine_param(source, source_vs, target, target_vs, arg)
 * (numerical/transformation.hpp:933-1021); arg = translocation, rotation, scaling, affine. */
void orc_estimate_affine_param_u8(const uint8_t* src, const int* sdim, const float* svs, const uint8_t* tgt,
                                  const int* tdim, const float* tvs, float* arg)
{
    const float pi_half = 1.570796327f;
    double c_s[3], c_t[3], cov_s[9], cov_t[9];
    for (int k = 0; k < 12; ++k)
        arg[k] = 0.0f;
    arg[6] = arg[7] = arg[8] = 1.0f;
    if (orc_moments(src, sdim, svs, c_s, cov_s) <= 0 || orc_moments(tgt, tdim, tvs, c_t, cov_t) <= 0)
        return;
    double Vs[9] = {0}, Vt[9] = {0}, Ls[3] = {0}, Lt[3] = {0}, R[9] = {0};
    orc_eigen_sym3(cov_s, Vs, Ls);
    orc_eigen_sym3(cov_t, Vt, Lt);
    for (int i = 0; i < 3; ++i) {
        const double lt = Lt[i] < 0.0 ? 0.0 : Lt[i]; /* std::max(a, b) = a < b ? b : a */
        const double ls = Ls[i] < 1e-6 ? 1e-6 : Ls[i];
        arg[6 + i] = (float)sqrt(lt / ls);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                R[i * 3 + j] += Vt[i + k * 3] * Vs[j + k * 3];
    if (orc_det3(R) < 0.0)
        for (int i = 0; i < 3; ++i)
            R[i * 3 + 2] = -R[i * 3 + 2];
    arg[3] = (float)atan2(R[7], R[8]);
    arg[4] = (float)atan2(-R[6], sqrt(R[7] * R[7] + R[8] * R[8]));
    arg[5] = (float)atan2(R[3], R[0]);
    for (int i = 0; i < 3; ++i)
        arg[3 + i] = remainderf(arg[3 + i], pi_half);
    double dt[3];
    for (int i = 0; i < 3; ++i) {
        const double sc = (double)arg[6 + i] < 1e-6 ? 1e-6 : (double)arg[6 + i];
        dt[i] = (c_t[i] - (float)((unsigned)tdim[i] * tvs[i]) * 0.5) / sc;
    }
    for (int i = 0; i < 3; ++i) {
        double dt_rot = R[0 * 3 + i] * dt[0] + R[1 * 3 + i] * dt[1] + R[2 * 3 + i] * dt[2];
        arg[i] = (float)(dt_rot - (c_s[i] - (float)((unsigned)sdim[i] * svs[i]) * 0.5));
    }
}

/* mat::inverse, 3x3 in place (numerical/matrix.hpp:1480-1507), float */
static int orc_inverse3f(float* m)
{
    const float det = m[0] * (m[4] * m[8] - m[5] * m[7]) + m[1] * (m[5] * m[6] - m[3] * m[8]) +
                      m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (det + 1.0f == 1.0f)
        return 0;
    float t[9];
    t[0] = m[4] * m[8] - m[5] * m[7];
    t[1] = m[2] * m[7] - m[1] * m[8];
    t[2] = m[1] * m[5] - m[2] * m[4];
    t[3] = m[5] * m[6] - m[3] * m[8];
    t[4] = m[0] * m[8] - m[2] * m[6];
    t[5] = m[2] * m[3] - m[0] * m[5];
    t[6] = m[3] * m[7] - m[4] * m[6];
    t[7] = m[1] * m[6] - m[0] * m[7];
    t[8] = m[0] * m[4] - m[1] * m[3];
    for (int k = 0; k < 9; ++k)
        m[k] = t[k] / det;
    return 1;
}

/* qr_decomposition(A, Q, dim<3,3>) (numerical/matrix.hpp:903-962, 1022-1043, 985-1000,
 * 1090-1100): Householder QR of a float 3x3 with the Q factor in double; A becomes R. */
static void orc_qr3(float* A, double* Q)
{
    const int m = 3, n = 3;
    float c[3] = {0, 0, 0}, d[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
        float* Ak = A + k * n;
        if (k == 2) {
            d[k] = Ak[k];
            c[k] = 0.0f;
            break;
        }
        float scale = 0.0f;
        for (int i = k; i < m; ++i) {
            const float a = fabsf(A[i * n + k]);
            scale = scale < a ? a : scale;
        }
        if (scale == 0.0f) {
            c[k] = d[k] = 0.0f;
        } else {
            float sum = 0.0f;
            for (int i = k; i < m; ++i) {
                float t = (A[i * n + k] /= scale);
                sum += t * t;
            }
            float sigma = (Ak[k] >= 0) ? sqrtf(sum) : -sqrtf(sum);
            Ak[k] += sigma;
            c[k] = sigma * Ak[k];
            d[k] = -scale * sigma;
            for (int j = k + 1; j < n; ++j) {
                float s2 = 0.0f;
                for (int i = k; i < m; ++i)
                    s2 += A[i * n + k] * A[i * n + j];
                s2 /= c[k];
                for (int i = k; i < m; ++i)
                    A[i * n + j] -= s2 * A[i * n + k];
            }
        }
    }
    /* qr_compute_q, square case: Qt accumulated in place */
    for (int k = 0; k < 9; ++k)
        Q[k] = 0.0;
    Q[0] = Q[4] = Q[8] = 1.0;
    for (int k = 0; k < n; ++k)
        if (c[k] != 0.0f)
            for (int j = 0; j < m; ++j) {
                float sum = 0.0f;
                for (int i = k; i < m; ++i)
                    sum += A[i * n + k] * Q[j * m + i];
                sum /= c[k];
                for (int i = k; i < m; ++i)
                    Q[j * m + i] -= sum * A[i * n + k];
            }
    /* qr_get_r: diagonal from d, zeros below */
    for (int i = 0; i < 3; ++i) {
        const int pos = i * (n + 1);
        A[pos] = d[i];
        for (int j = 1; j <= i; ++j)
            A[pos - j] = 0.0f;
    }
}

/* inverse_upper, 3x3 float (numerical/matrix.hpp:1621-1650) */
static int orc_inverse_upper3f(float* U)
{
    const int n = 3, n_1 = 4;
    int pos = 0;
    for (int col = 0; col < n; ++col, pos += n_1) {
        if (U[pos] + 1.0f == 1.0f)
            return 0;
        U[pos] = 1.0f / U[pos];
    }
    /* off-diagonals, last column first, rows upward */
    for (int col = n - 1; col >= 0; --col)
        for (int row = col - 1; row >= 0; --row) {
            float sum = 0.0f;
            for (int i = row + 1; i <= col; ++i)
                sum += U[row * n + i] * U[i * n + col];
            U[row * n + col] = -sum * U[row * n + row];
        }
    return 1;
}

/* transformation_matrix::to_affine_param (numerical/transformation.hpp:703-741) with
 * matrix_to_rotation_scaling_affine (:234-272) and rotation_matrix_to_angles (:167-181). */
void orc_matrix_to_affine_param(const float* T, const int* from_dim, const float* from_vs, const int* to_dim,
                                const float* to_vs, float* rb)
{
    float R[9], iR[9], t[3];
    for (int k = 0; k < 12; ++k)
        rb[k] = 0.0f;
    rb[6] = rb[7] = rb[8] = 1.0f;
    for (int k = 0; k < 9; ++k)
        R[k] = T[k];
    t[0] = T[9] - (float)to_dim[0] * 0.5f;
    t[1] = T[10] - (float)to_dim[1] * 0.5f;
    t[2] = T[11] - (float)to_dim[2] * 0.5f;
    if (to_vs[2] != 1.0f) {
        R[6] *= to_vs[2]; R[7] *= to_vs[2]; R[8] *= to_vs[2]; t[2] *= to_vs[2];
    }
    if (to_vs[1] != 1.0f) {
        R[3] *= to_vs[1]; R[4] *= to_vs[1]; R[5] *= to_vs[1]; t[1] *= to_vs[1];
    }
    if (to_vs[0] != 1.0f) {
        R[0] *= to_vs[0]; R[1] *= to_vs[0]; R[2] *= to_vs[0]; t[0] *= to_vs[0];
    }
    R[0] /= from_vs[0]; R[1] /= from_vs[1]; R[2] /= from_vs[2];
    R[3] /= from_vs[0]; R[4] /= from_vs[1]; R[5] /= from_vs[2];
    R[6] /= from_vs[0]; R[7] /= from_vs[1]; R[8] /= from_vs[2];
    for (int k = 0; k < 9; ++k)
        iR[k] = R[k];
    if (!orc_inverse3f(iR))
        for (int k = 0; k < 9; ++k)
            iR[k] = 0.0f;
    rb[0] = (iR[0] * t[0] + iR[1] * t[1] + iR[2] * t[2]) + (float)from_dim[0] * 0.5f * from_vs[0];
    rb[1] = (iR[3] * t[0] + iR[4] * t[1] + iR[5] * t[2]) + (float)from_dim[1] * 0.5f * from_vs[1];
    rb[2] = (iR[6] * t[0] + iR[7] * t[1] + iR[8] * t[2]) + (float)from_dim[2] * 0.5f * from_vs[2];

    /* matrix_to_rotation_scaling_affine(R, rotation, scaling, affine) */
    float* m = R;
    double Q[9];
    orc_inverse3f(m);
    orc_qr3(m, Q);
    orc_inverse_upper3f(m);
    {
        double Qt[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                Qt[i * 3 + j] = Q[j * 3 + i];
        for (int k = 0; k < 9; ++k)
            Q[k] = Qt[k];
    }
    if (m[0] < 0) {
        m[0] = -m[0];
        Q[0] = -Q[0]; Q[1] = -Q[1]; Q[2] = -Q[2];
    }
    if (m[4] < 0) {
        m[1] = -m[1];
        m[4] = -m[4];
        Q[3] = -Q[3]; Q[4] = -Q[4]; Q[5] = -Q[5];
    }
    if (m[8] < 0) {
        m[2] = -m[2];
        m[5] = -m[5];
        m[8] = -m[8];
        Q[6] = -Q[6]; Q[7] = -Q[7]; Q[8] = -Q[8];
    }
    rb[6] = m[0];
    rb[7] = m[4];
    rb[8] = m[8];
    rb[9] = m[1] / m[4];
    rb[10] = m[2] / m[8];
    rb[11] = m[5] / m[8];
    {
        double sy = sqrt(Q[0] * Q[0] + Q[1] * Q[1]);
        if (sy > 1.0e-6) {
            rb[3] = (float)atan2(Q[5], Q[8]);
            rb[5] = (float)atan2(Q[1], Q[0]);
        } else {
            rb[3] = (float)atan2(-Q[7], Q[4]);
            rb[5] = 0.0f;
        }
        rb[4] = (float)atan2(-Q[2], sy);
    }
}
