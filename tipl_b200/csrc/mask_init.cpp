// Mask-moment initialisation of an affine registration (tipl::reg::linear,
// reg/linear.hpp:658-684): has_mask on both volumes, estimate_affine_param from
// their masks' centroids and principal axes, and the conversion of the search's
// matrix back to an affine_param (transformation_matrix::to_affine_param).
//
// The per-voxel pass is mask_count_kernel (exact integer counts per (x,y), (x,z),
// (y,z) line); everything here is host arithmetic on those tables and 3x3 matrices,
// with the reference's types (coordinate products float, moments double, the QR of
// to_affine_param float with a double Q factor).
#include <algorithm>
#include <cmath>
#include <vector>
#include "host.h"
#include "kernels.h"
#include "mask_init.h"
#include "stats.h"

namespace regb {

void mask_counts(const uint8_t* d_vol, const int* dim, MaskCounts& out, cudaStream_t st)
{
    out.w = dim[0];
    out.h = dim[1];
    out.d = dim[2];
    const size_t nxy = (size_t)out.w * out.h, nxz = (size_t)out.w * out.d, nyz = (size_t)out.h * out.d;
    DevBuf<uint32_t> buf(nxy + nxz + nyz, st);
    REGB_CK(launch_mask_counts(d_vol, Dim3{out.w, out.h, out.d}, buf.p, buf.p + nxy, buf.p + nxy + nxz, st));
    count_launch();
    out.xy.resize(nxy);
    out.xz.resize(nxz);
    out.yz.resize(nyz);
    REGB_CK(cudaMemcpyAsync(out.xy.data(), buf.p, nxy * 4, cudaMemcpyDeviceToHost, st));
    REGB_CK(cudaMemcpyAsync(out.xz.data(), buf.p + nxy, nxz * 4, cudaMemcpyDeviceToHost, st));
    REGB_CK(cudaMemcpyAsync(out.yz.data(), buf.p + nxy + nxz, nyz * 4, cudaMemcpyDeviceToHost, st));
    REGB_CK(cudaStreamSynchronize(st));
}

namespace {

// Voxels > 0 per x, per y, per z.
void axis_counts(const MaskCounts& c, std::vector<double>& cx, std::vector<double>& cy, std::vector<double>& cz,
                 unsigned long long& n)
{
    cx.assign(c.w, 0.0);
    cy.assign(c.h, 0.0);
    cz.assign(c.d, 0.0);
    n = 0;
    for (int y = 0; y < c.h; ++y)
        for (int x = 0; x < c.w; ++x) {
            const uint32_t v = c.xy[(size_t)y * c.w + x];
            cx[x] += v;
            cy[y] += v;
            n += v;
        }
    for (int z = 0; z < c.d; ++z)
        for (int x = 0; x < c.w; ++x)
            cz[z] += c.xz[(size_t)z * c.w + x];
}

}  // namespace

// has_mask (numerical/basic_op.hpp:811-830) with bounding_box(I, min, max, 0)
// (:697-730): more than a fifth of the voxels zero, or the non-zero voxels' box
// inside the volume on some axis.
bool has_mask(const MaskCounts& c)
{
    std::vector<double> cx, cy, cz;
    unsigned long long n;
    axis_counts(c, cx, cy, cz, n);
    const unsigned long long sz = (unsigned long long)c.w * c.h * c.d;
    if (sz - n > sz / 5)
        return true;
    const int shape[3] = {c.w, c.h, c.d};
    const std::vector<double>* cnt[3] = {&cx, &cy, &cz};
    for (int k = 0; k < 3; ++k) {
        int lo = shape[k] - 1, hi = 0;
        for (int i = 0; i < shape[k]; ++i)
            if ((*cnt[k])[i] > 0) {
                lo = std::min(lo, i);
                hi = std::max(hi, i);
            }
        if (hi == 0)
            lo = hi = 0;
        ++hi;
        if (lo > 0 && hi < shape[k])
            return true;
    }
    return false;
}

namespace {

// compute_moments of estimate_affine_param (numerical/transformation.hpp:943-982) from
// the count tables: every voxel > 0 contributes its coordinate x*vs (a float product)
// to the centroid and (p - c)(p - c)^T to the covariance; the per-line counts weight
// each distinct coordinate (pair) once.
unsigned long long moments(const MaskCounts& c, const float* vs, double* ctr, double* cov)
{
    std::vector<double> cx, cy, cz;
    unsigned long long n;
    axis_counts(c, cx, cy, cz, n);
    if (n == 0)
        return 0;
    std::vector<double> px(c.w), py(c.h), pz(c.d);
    for (int i = 0; i < c.w; ++i) px[i] = i * vs[0];
    for (int i = 0; i < c.h; ++i) py[i] = i * vs[1];
    for (int i = 0; i < c.d; ++i) pz[i] = i * vs[2];
    double s[3] = {0, 0, 0};
    for (int i = 0; i < c.w; ++i) s[0] += cx[i] * px[i];
    for (int i = 0; i < c.h; ++i) s[1] += cy[i] * py[i];
    for (int i = 0; i < c.d; ++i) s[2] += cz[i] * pz[i];
    for (int k = 0; k < 3; ++k)
        ctr[k] = s[k] / double(n);
    for (int i = 0; i < c.w; ++i) px[i] -= ctr[0];
    for (int i = 0; i < c.h; ++i) py[i] -= ctr[1];
    for (int i = 0; i < c.d; ++i) pz[i] -= ctr[2];
    double m[6] = {0, 0, 0, 0, 0, 0};  // xx xy xz yy yz zz
    for (int i = 0; i < c.w; ++i) m[0] += cx[i] * (px[i] * px[i]);
    for (int i = 0; i < c.h; ++i) m[3] += cy[i] * (py[i] * py[i]);
    for (int i = 0; i < c.d; ++i) m[5] += cz[i] * (pz[i] * pz[i]);
    for (int y = 0; y < c.h; ++y)
        for (int x = 0; x < c.w; ++x)
            m[1] += c.xy[(size_t)y * c.w + x] * (px[x] * py[y]);
    for (int z = 0; z < c.d; ++z)
        for (int x = 0; x < c.w; ++x)
            m[2] += c.xz[(size_t)z * c.w + x] * (px[x] * pz[z]);
    for (int z = 0; z < c.d; ++z)
        for (int y = 0; y < c.h; ++y)
            m[4] += c.yz[(size_t)z * c.h + y] * (py[y] * pz[z]);
    cov[0] = m[0];
    cov[1] = cov[3] = m[1];
    cov[2] = cov[6] = m[2];
    cov[4] = m[3];
    cov[5] = cov[7] = m[4];
    cov[8] = m[5];
    for (int k = 0; k < 9; ++k)
        cov[k] /= double(n);
    return n;
}

double det3(const double* m)
{
    return m[0] * (m[4] * m[8] - m[5] * m[7]) + m[1] * (m[5] * m[6] - m[3] * m[8]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// One 2x2 block of a symmetric 3x3 whose other off-diagonals are zero: the lone
// diagonal entry `solo` is eigenvalue 0, the block (a, b; b, c) gives the other two.
void eigen_block(double solo, double a, double b, double c, double* d, double& l_sq_term, double& a_d1)
{
    d[0] = solo;
    d[1] = d[2] = (a + c) * 0.5;
    const double half = (a - c) * 0.5;
    const double l = std::sqrt(half * half + b * b);
    d[1] += l;
    d[2] -= l;
    l_sq_term = b * b;
    a_d1 = a - d[1];
}

}  // namespace

// eigen_decomposition_sym for a symmetric 3x3 (numerical/matrix.hpp:1830-1955):
// eigenvalues in closed form from the invariants (trigonometric solution of the
// characteristic cubic), eigenvector i in V[3i..3i+2] from the cross products of
// two rows of A - d_i I; the block-diagonal cases solve the 2x2 block directly.
void eigen_sym3(const double* A, double* V, double* d)
{
    const auto identity = [&] {
        for (int k = 0; k < 9; ++k)
            V[k] = 0.0;
        V[0] = V[4] = V[8] = 1.0;
    };
    if (A[1] == 0.0 && A[2] == 0.0 && A[5] == 0.0) {
        d[0] = A[0];
        d[1] = A[4];
        d[2] = A[8];
        identity();
        return;
    }
    if (A[1] == 0.0 && A[2] == 0.0) {  // yz block
        double bb, ad;
        eigen_block(A[0], A[4], A[5], A[8], d, bb, ad);
        for (int k = 0; k < 9; ++k) V[k] = 0.0;
        V[0] = 1.0;
        const double len = std::sqrt(bb + ad * ad);
        V[4] = V[8] = -A[5] / len;
        V[5] = ad / len;
        V[7] = -V[5];
        return;
    }
    if (A[1] == 0.0 && A[5] == 0.0) {  // xz block
        double bb, ad;
        eigen_block(A[4], A[0], A[2], A[8], d, bb, ad);
        for (int k = 0; k < 9; ++k) V[k] = 0.0;
        V[1] = 1.0;
        const double len = std::sqrt(bb + ad * ad);
        V[3] = V[8] = -A[2] / len;
        V[5] = ad / len;
        V[6] = -V[5];
        return;
    }
    if (A[1] != 0.0 && A[2] == 0.0 && A[5] == 0.0) {  // xy block
        double bb, ad;
        eigen_block(A[8], A[0], A[1], A[4], d, bb, ad);
        for (int k = 0; k < 9; ++k) V[k] = 0.0;
        V[2] = 1.0;
        const double len = std::sqrt(bb + ad * ad);
        V[3] = V[7] = -A[1] / len;
        V[4] = ad / len;
        V[6] = -V[4];
        return;
    }
    const double A2A1 = A[2] * A[1], A1A5 = A[1] * A[5], A2A5 = A[2] * A[5], A0A4 = A[0] * A[4];
    const double A1A1 = A[1] * A[1], A2A2 = A[2] * A[2], A5A5 = A[5] * A[5], A0_A4 = A[0] + A[4];
    // invariants: trace, sum of principal 2x2 minors, determinant
    const double I1 = A0_A4 + A[8];
    const double I2 = A0A4 + A0_A4 * A[8] - A1A1 - A2A2 - A5A5;
    const double I3 = A0A4 * A[8] + 2.0 * A2A1 * A[5] - (A[8] * A1A1 + A[4] * A2A2 + A[0] * A5A5);
    const double I1_3 = I1 / 3.0;
    const double I1_3sq = I1_3 * I1_3;
    const double v = I1_3sq - I2 / 3.0;
    const double s = I1_3sq * I1_3 - I1 * I2 / 6.0 + I3 / 2.0;
    if (v == 0.0) {
        d[0] = d[1] = d[2] = 0.0;
        identity();
        return;
    }
    const double sqrt_v = std::sqrt(v);
    const double angle = std::acos(std::max<double>(-1.0, std::min<double>(1.0, s / v / sqrt_v))) / 3.0;
    d[0] = I1_3 + 2.0 * sqrt_v * std::cos(angle);
    d[1] = I1_3 - 2.0 * sqrt_v * std::cos(3.14159265358979323846 / 3.0 + angle);
    d[2] = I1 - d[0] - d[1];
    for (int i = 0; i < 3; ++i) {
        double* e = V + 3 * i;
        const double q1 = A2A1 - (A[0] - d[i]) * A[5];
        const double q2 = A1A5 - (A[4] - d[i]) * A[2];
        const double q3 = A2A5 - (A[8] - d[i]) * A[1];
        e[0] = q2 * q3;
        e[1] = q3 * q1;
        e[2] = q2 * q1;
        const double len = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        e[0] /= len;
        e[1] /= len;
        e[2] /= len;
    }
}

// estimate_affine_param(source, source_vs, target, target_vs, arg)
// (numerical/transformation.hpp:933-1021): scaling from the eigenvalue ratios,
// rotation from the eigenvector frames (reflection removed, angles folded into
// [-pi/4, pi/4]), translation aligning the centroids.  arg = translocation[3],
// rotation[3], scaling[3], affine[3].  Returns false (arg = identity) when either
// volume has no voxel > 0.
bool estimate_affine_param(const MaskCounts& src, const float* svs, const MaskCounts& tgt, const float* tvs,
                           float* arg)
{
    for (int k = 0; k < 12; ++k)
        arg[k] = 0.0f;
    arg[6] = arg[7] = arg[8] = 1.0f;
    double c_s[3], c_t[3], cov_s[9], cov_t[9];
    if (moments(src, svs, c_s, cov_s) == 0 || moments(tgt, tvs, c_t, cov_t) == 0)
        return false;
    double Vs[9], Vt[9], Ls[3], Lt[3], R[9] = {0};
    eigen_sym3(cov_s, Vs, Ls);
    eigen_sym3(cov_t, Vt, Lt);
    for (int i = 0; i < 3; ++i)
        arg[6 + i] = (float)std::sqrt(std::max(Lt[i], 0.0) / std::max(Ls[i], 1e-6));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                R[i * 3 + j] += Vt[i + k * 3] * Vs[j + k * 3];
    if (det3(R) < 0.0)
        for (int i = 0; i < 3; ++i)
            R[i * 3 + 2] = -R[i * 3 + 2];
    arg[3] = (float)std::atan2(R[7], R[8]);
    arg[4] = (float)std::atan2(-R[6], std::sqrt(R[7] * R[7] + R[8] * R[8]));
    arg[5] = (float)std::atan2(R[3], R[0]);
    const float quarter_turn = 1.570796327f;
    for (int i = 0; i < 3; ++i)
        arg[3 + i] = std::remainder(arg[3 + i], quarter_turn);
    const int sdim[3] = {src.w, src.h, src.d}, tdim[3] = {tgt.w, tgt.h, tgt.d};
    double dt[3];
    for (int i = 0; i < 3; ++i)
        dt[i] = (c_t[i] - (unsigned)tdim[i] * tvs[i] * 0.5) / std::max<double>(arg[6 + i], 1e-6);
    for (int i = 0; i < 3; ++i) {
        const double rot = R[0 * 3 + i] * dt[0] + R[1 * 3 + i] * dt[1] + R[2 * 3 + i] * dt[2];
        arg[i] = (float)(rot - (c_s[i] - (unsigned)sdim[i] * svs[i] * 0.5));
    }
    return true;
}

namespace {

// 3x3 inverse by cofactors over the determinant, float (numerical/matrix.hpp:1480-1507);
// m is left unchanged when |det| is below float resolution.
bool inverse3f(float* m)
{
    const float det = m[0] * (m[4] * m[8] - m[5] * m[7]) + m[1] * (m[5] * m[6] - m[3] * m[8]) +
                      m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (det + 1.0f == 1.0f)
        return false;
    const float c[9] = {m[4] * m[8] - m[5] * m[7], m[2] * m[7] - m[1] * m[8], m[1] * m[5] - m[2] * m[4],
                        m[5] * m[6] - m[3] * m[8], m[0] * m[8] - m[2] * m[6], m[2] * m[3] - m[0] * m[5],
                        m[3] * m[7] - m[4] * m[6], m[1] * m[6] - m[0] * m[7], m[0] * m[4] - m[1] * m[3]};
    for (int k = 0; k < 9; ++k)
        m[k] = c[k] / det;
    return true;
}

// Householder QR of a float 3x3 (numerical/matrix.hpp:903-962): A becomes R (diagonal
// from d, zeros below); Qt (double) is accumulated by applying the reflections to
// the identity (:1022-1043, the square case).
void qr3(float* A, double* Qt)
{
    float c[3] = {0, 0, 0}, d[3] = {0, 0, 0};
    for (int k = 0; k < 2; ++k) {
        float scale = 0.0f;
        for (int i = k; i < 3; ++i)
            scale = std::max<float>(scale, std::fabs(A[i * 3 + k]));
        if (scale == 0.0f)
            continue;
        float ss = 0.0f;
        for (int i = k; i < 3; ++i) {
            const float t = (A[i * 3 + k] /= scale);
            ss += t * t;
        }
        const float sigma = (A[k * 3 + k] >= 0) ? std::sqrt(ss) : -std::sqrt(ss);
        A[k * 3 + k] += sigma;
        c[k] = sigma * A[k * 3 + k];
        d[k] = -scale * sigma;
        for (int j = k + 1; j < 3; ++j) {
            float dot = 0.0f;
            for (int i = k; i < 3; ++i)
                dot += A[i * 3 + k] * A[i * 3 + j];
            dot /= c[k];
            for (int i = k; i < 3; ++i)
                A[i * 3 + j] -= dot * A[i * 3 + k];
        }
    }
    d[2] = A[8];
    for (int k = 0; k < 9; ++k)
        Qt[k] = (k % 4 == 0) ? 1.0 : 0.0;
    for (int k = 0; k < 3; ++k) {
        if (c[k] == 0.0f)
            continue;
        for (int j = 0; j < 3; ++j) {
            float dot = 0.0f;
            for (int i = k; i < 3; ++i)
                dot += A[i * 3 + k] * Qt[j * 3 + i];  // float += double product
            dot /= c[k];
            for (int i = k; i < 3; ++i)
                Qt[j * 3 + i] -= dot * A[i * 3 + k];
        }
    }
    for (int i = 0; i < 3; ++i) {
        A[i * 4] = d[i];
        for (int j = 1; j <= i; ++j)
            A[i * 4 - j] = 0.0f;
    }
}

// Inverse of an upper-triangular float 3x3 in place (numerical/matrix.hpp:1621-1650).
void inverse_upper3f(float* U)
{
    for (int k = 0; k < 3; ++k) {
        if (U[k * 4] + 1.0f == 1.0f)
            return;
        U[k * 4] = 1.0f / U[k * 4];
    }
    for (int col = 2; col >= 0; --col)
        for (int row = col - 1; row >= 0; --row) {
            float sum = 0.0f;
            for (int i = row + 1; i <= col; ++i)
                sum += U[row * 3 + i] * U[i * 3 + col];
            U[row * 3 + col] = -sum * U[row * 3 + row];
        }
}

}  // namespace

// transformation_matrix::to_affine_param (numerical/transformation.hpp:703-741): the
// physical-space linear part R (voxel sizes folded in) and the centred shift give the
// translocation; matrix_to_rotation_scaling_affine (:234-272) factors R^-1 = Q * U
// (QR), U^-1's diagonal is the scaling, its ratios the shears, and Q's Euler angles
// (rotation_matrix_to_angles, :167-181) the rotation.
void matrix_to_affine_param(const float* T, const int* from_dim, const float* from_vs, const int* to_dim,
                            const float* to_vs, float* rb)
{
    for (int k = 0; k < 12; ++k)
        rb[k] = 0.0f;
    rb[6] = rb[7] = rb[8] = 1.0f;
    float R[9], t[3];
    for (int k = 0; k < 9; ++k)
        R[k] = T[k];
    for (int i = 0; i < 3; ++i)
        t[i] = T[9 + i] - float(to_dim[i]) * 0.5f;
    for (int i = 2; i >= 0; --i)
        if (to_vs[i] != 1.0f) {
            R[3 * i] *= to_vs[i];
            R[3 * i + 1] *= to_vs[i];
            R[3 * i + 2] *= to_vs[i];
            t[i] *= to_vs[i];
        }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            R[3 * r + c] /= from_vs[c];
    float iR[9];
    std::copy(R, R + 9, iR);
    if (!inverse3f(iR))
        std::fill(iR, iR + 9, 0.0f);
    for (int i = 0; i < 3; ++i)
        rb[i] = (iR[3 * i] * t[0] + iR[3 * i + 1] * t[1] + iR[3 * i + 2] * t[2]) +
                float(from_dim[i]) * 0.5f * from_vs[i];

    float* m = R;
    double Qt[9], Q[9];
    inverse3f(m);
    qr3(m, Qt);
    inverse_upper3f(m);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            Q[i * 3 + j] = Qt[j * 3 + i];
    // positive diagonal of U^-1: flip the matching row of U^-1's upper part and of Q
    for (int k = 0; k < 3; ++k)
        if (m[4 * k] < 0) {
            for (int c = 0; c <= k; ++c)
                m[3 * c + k] = -m[3 * c + k];
            Q[3 * k] = -Q[3 * k];
            Q[3 * k + 1] = -Q[3 * k + 1];
            Q[3 * k + 2] = -Q[3 * k + 2];
        }
    rb[6] = m[0];
    rb[7] = m[4];
    rb[8] = m[8];
    rb[9] = m[1] / m[4];
    rb[10] = m[2] / m[8];
    rb[11] = m[5] / m[8];
    const double sy = std::sqrt(Q[0] * Q[0] + Q[1] * Q[1]);
    if (sy > 1.0e-6) {
        rb[3] = (float)std::atan2(Q[5], Q[8]);
        rb[5] = (float)std::atan2(Q[1], Q[0]);
    } else {
        rb[3] = (float)std::atan2(-Q[7], Q[4]);
        rb[5] = 0.0f;
    }
    rb[4] = (float)std::atan2(-Q[2], sy);
}

}  // namespace regb
