/* Test infrastructure only (the checker, never the product path).
 *
 * Plain-C restatement of the reference's CPU algorithm for the registration hot
 * path.  This header is included by oracle.c once per (pixel type, real type)
 * combination:
 *   PIX = uint8_t, R = float   suffix _u8   reference-exact for uint8 volumes
 *   PIX = float,   R = float   suffix _f32  reference-exact for float volumes
 *   PIX = double,  R = double  suffix _f64  all-double restatement, used only to
 *                                           report the FP32 paths' error
 * Field-only passes (Poisson, smooth, accumulate, ...) depend on R alone and live
 * in oracle_field.h; the CDM driver lives in oracle_cdm.h.
 *
 * Every float operation is written in the reference's order; oracle.c is built
 * with -ffp-contract=off so no multiply-add is fused, which is what makes the
 * _u8/_f32 instantiations bit-identical to the reference's own build.
 */
#ifndef SFX
#error "define SFX, PIX, R, PIX_IS_U8 before including"
#endif

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)


/* interp_type<T>::assign (numerical/interpolation.hpp:28-34): unsigned outputs
 * clamp negatives to 0 and truncate; signed/floating outputs convert. */
static inline PIX FN(assign_pix)(R v)
{
#if PIX_IS_U8
    return (PIX)(v <= (R)0 ? 0 : (PIX)v);
#else
    return (PIX)v;
#endif
}

/* interpolator::linear<3>::get_location + weighted_sum
 * (numerical/interpolation.hpp:337-383, 61-73).  Returns 0 and leaves *out
 * untouched when the 2x2x2 cell leaves the volume. */
static int FN(trilinear)(const PIX* I, const int* dim, R x, R y, R z, PIX* out)
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
    R acc = (R)I[d[0]] * r[0];
    for (int i = 1; i < 8; ++i) {
        R v = (R)I[d[i]];
        v *= r[i];
        acc += v;
    }
    *out = FN(assign_pix)(acc);
    return 1;
}

/* vector_transformation with sr/shift (numerical/transformation.hpp:58-73):
 * ((x*r0 + y*r1) + z*r2) + s0, evaluated left to right. */
static inline void FN(apply_T)(const float* T, R x, R y, R z, R* o)
{
    o[0] = x * (R)T[0] + y * (R)T[1] + z * (R)T[2] + (R)T[9];
    o[1] = x * (R)T[3] + y * (R)T[4] + z * (R)T[5] + (R)T[10];
    o[2] = x * (R)T[6] + y * (R)T[7] + z * (R)T[8] + (R)T[11];
}

/* resample<linear> CPU (numerical/resampling.hpp:1239-1269).  With allow_crop the
 * reference's integer-shift fast path is taken when every shift is within 1e-4
 * of an integer and sr within 1e-4 of identity: a plain copy of the overlap,
 * other voxels left as they were (zero for a fresh output). */
void FN(orc_resample)(const PIX* from, const int* fdim, PIX* to, const int* tdim, const float* T, int allow_crop)
{
    size_t n = (size_t)tdim[0] * tdim[1] * tdim[2];
    int shift[3];
    if (allow_crop && orc_is_integer_shift(T, shift)) {
        for (size_t i = 0; i < n; ++i)
            to[i] = (PIX)0;
        for (int z = 0; z < tdim[2]; ++z)
            for (int y = 0; y < tdim[1]; ++y)
                for (int x = 0; x < tdim[0]; ++x) {
                    int sx = x + shift[0], sy = y + shift[1], sz = z + shift[2];
                    if (sx < 0 || sy < 0 || sz < 0 || sx >= fdim[0] || sy >= fdim[1] || sz >= fdim[2])
                        continue;
                    to[((size_t)z * tdim[1] + y) * tdim[0] + x] =
                        from[((size_t)sz * fdim[1] + sy) * fdim[0] + sx];
                }
        return;
    }
    size_t i = 0;
    for (int z = 0; z < tdim[2]; ++z)
        for (int y = 0; y < tdim[1]; ++y)
            for (int x = 0; x < tdim[0]; ++x, ++i) {
                R p[3];
                FN(apply_T)(T, (R)x, (R)y, (R)z, p);
                PIX v = (PIX)0;
                FN(trilinear)(from, fdim, p[0], p[1], p[2], &v);
                to[i] = v;
            }
}

/* compose_displacement CPU (numerical/dif.hpp:90-107): Js = Is where d == 0,
 * else trilinear(Is, x + d); failed samples stay 0. */
void FN(orc_compose)(const PIX* Is, const int* dim, const R* dis, PIX* Js)
{
    size_t i = 0;
    for (int z = 0; z < dim[2]; ++z)
        for (int y = 0; y < dim[1]; ++y)
            for (int x = 0; x < dim[0]; ++x, ++i) {
                const R* d = dis + 3 * i;
                Js[i] = (PIX)0;
                if (d[0] == 0 && d[1] == 0 && d[2] == 0) {
                    Js[i] = Is[i];
                    continue;
                }
                R vx = (R)x, vy = (R)y, vz = (R)z;
                vx += d[0];
                vy += d[1];
                vz += d[2];
                FN(trilinear)(Is, dim, vx, vy, vz, &Js[i]);
            }
}

/* get_window_at_width<2> (numerical/window.hpp:92-110) + iterate_xyz/xy/x
 * (window.hpp:25-72): visiting order z = 0..up, -1..-lo; inside each z the same
 * for y; inside each y, x = 0..up, -1..-lo. */
static int FN(window5)(const PIX* I, const int* dim, int x, int y, int z, PIX* out)
{
    int xu = dim[0] - x - 1, yu = dim[1] - y - 1, zu = dim[2] - z - 1, xl = x, yl = y, zl = z;
    if (xu > 2) xu = 2;
    if (yu > 2) yu = 2;
    if (zu > 2) zu = 2;
    if (xl > 2) xl = 2;
    if (yl > 2) yl = 2;
    if (zl > 2) zl = 2;
    int n = 0;
    long long w = dim[0], wh = (long long)dim[0] * dim[1];
    long long idx = ((long long)z * dim[1] + y) * dim[0] + x;
    for (int pz = 0; pz < 2; ++pz) {
        int zc = pz ? zl : zu;
        for (int dz = pz; dz <= zc; ++dz) {
            long long zi = idx + (pz ? -dz : dz) * wh;
            for (int py = 0; py < 2; ++py) {
                int yc = py ? yl : yu;
                for (int dy = py; dy <= yc; ++dy) {
                    long long yi = zi + (py ? -dy : dy) * w;
                    for (int dx = 0; dx <= xu; ++dx)
                        out[n++] = I[yi + dx];
                    for (int dx = 1; dx <= xl; ++dx)
                        out[n++] = I[yi - dx];
                }
            }
        }
    }
    return n;
}

/* linear_regression(x, y, a, b, r2) (numerical/statistics.hpp:694-713) with the
 * reference's sum types: integer pixels sum exactly in int64, floating pixels
 * sum in double, and the cross products are formed in the pixel product type
 * before being widened (statistics.hpp:186-197, 491-502). */
static void FN(regress)(const PIX* xs, const PIX* ys, int n, R* a, R* b, R* r2)
{
#if PIX_IS_U8
    long long sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0;
    for (int i = 0; i < n; ++i) {
        sx += xs[i];
        sy += ys[i];
        sxx += (long long)xs[i] * xs[i];
        syy += (long long)ys[i] * ys[i];
        sxy += (int)xs[i] * (int)ys[i];
    }
    double dsx = (double)sx, dsy = (double)sy, dsxx = (double)sxx, dsyy = (double)syy, dsxy = (double)sxy;
#else
    double dsx = xs[0], dsy = ys[0], dsxx = 0, dsyy = 0, dsxy = (double)(xs[0] * ys[0]);
    for (int i = 1; i < n; ++i) {
        dsx += xs[i];
        dsy += ys[i];
        dsxy += (double)(xs[i] * ys[i]);
    }
    for (int i = 0; i < n; ++i) {
        double t = xs[i];
        dsxx += t * t;
        t = ys[i];
        dsyy += t * t;
    }
#endif
    double mx = dsx / (double)n, my = dsy / (double)n;
    double xv = dsxx / (double)n - mx * mx;
    double yv = dsyy / (double)n - my * my;
    if (xv == 0 || yv == 0) {
        *a = 0;
        *b = (R)my;
        *r2 = 0;
        return;
    }
    double cov = dsxy / (double)n - mx * my;
    /* a, b, r2 are written through the caller's float references, so b is formed
     * from the already-rounded a (statistics.hpp:708-710). */
    *a = (R)(cov / xv);
    *b = (R)(my - *a * mx);
    *r2 = (R)(cov * cov / xv / yv);
}

/* gradient_at (numerical/numerical.hpp:102-109): central difference, 0 on the
 * first/last voxel of each axis. */
static void FN(grad_at)(const PIX* I, const int* dim, int x, int y, int z, size_t pos, R* g)
{
    size_t w = dim[0], wh = (size_t)dim[0] * dim[1];
    g[0] = (x + 1 < dim[0] && x) ? (R)(I[pos + 1] - I[pos - 1]) : (R)0;
    g[1] = (y + 1 < dim[1] && y) ? (R)(I[pos + w] - I[pos - w]) : (R)0;
    g[2] = (z + 1 < dim[2] && z) ? (R)(I[pos + wh] - I[pos - wh]) : (R)0;
}

/* cdm_get_gradient CPU (reg/cdm.hpp:46-106): new_d (zeroed) += gradient term,
 * returns mean(cost_map) over every voxel as float. */
R FN(orc_cdm_gradient)(const PIX* Js, const PIX* It, const int* dim, R* new_d, int gradient_type)
{
    size_t n = (size_t)dim[0] * dim[1] * dim[2];
    for (size_t i = 0; i < 3 * n; ++i)
        new_d[i] = 0;
    double cost_sum = 0.0;
    PIX wj[125], wi[125];
    size_t pos = 0;
    for (int z = 0; z < dim[2]; ++z)
        for (int y = 0; y < dim[1]; ++y)
            for (int x = 0; x < dim[0]; ++x, ++pos) {
                R cost = 0;
                R* nd = new_d + 3 * pos;
                if (gradient_type == 'd') {
                    R g[3];
                    FN(grad_at)(Js, dim, x, y, z, pos, g);
#if PIX_IS_U8
                    int dif = (int)Js[pos] - (int)It[pos];
#else
                    PIX dif = Js[pos] - It[pos];
#endif
                    g[0] *= dif;
                    g[1] *= dif;
                    g[2] *= dif;
                    nd[0] += g[0];
                    nd[1] += g[1];
                    nd[2] += g[2];
                    cost = (R)(dif * dif);
                } else {
                    if (Js[pos] == 0 || It[pos] == 0) {
                        cost_sum += 0.0;
                        continue;
                    }
                    FN(window5)(It, dim, x, y, z, wi);
                    int m = FN(window5)(Js, dim, x, y, z, wj);
                    R a, b, r2;
                    FN(regress)(wj, wi, m, &a, &b, &r2);
                    if (a > 0) {
                        R g[3];
                        FN(grad_at)(Js, dim, x, y, z, pos, g);
#if PIX_IS_U8
                        float s = r2 * ((float)Js[pos] * a + b - (float)It[pos]);
#else
                        R s = r2 * (Js[pos] * a + b - It[pos]);
#endif
                        g[0] *= s;
                        g[1] *= s;
                        g[2] *= s;
                        nd[0] += g[0];
                        nd[1] += g[1];
                        nd[2] += g[2];
                        cost = -r2;
                    }
                }
                cost_sum += (double)cost;
            }
    return (R)(cost_sum / (double)n);
}

/* downsample_with_padding CPU (numerical/resampling.hpp:575-632): 2x box mean,
 * the missing +1 neighbours replaced by the nearest present one; integer pixels
 * sum in uint16 and shift by 3, floating pixels divide by 8. */
void FN(orc_downsample)(const PIX* in, const int* dim, PIX* out)
{
    int od[3] = {(dim[0] + 1) / 2, (dim[1] + 1) / 2, (dim[2] + 1) / 2};
    size_t w = dim[0], wh = (size_t)dim[0] * dim[1];
    size_t shift[8] = {0, 1, w, 1 + w, wh, wh + 1, wh + w, wh + 1 + w};
    size_t o = 0;
    for (int z = 0; z < od[2]; ++z)
        for (int y = 0; y < od[1]; ++y)
            for (int x = 0; x < od[0]; ++x, ++o) {
                int x2 = 2 * x, y2 = 2 * y, z2 = 2 * z;
                int has = 0;
                if (x2 + 1 < dim[0]) has += 1;
                if (y2 + 1 < dim[1]) has += 2;
                if (z2 + 1 < dim[2]) has += 4;
                size_t base = ((size_t)z2 * dim[1] + y2) * dim[0] + x2;
                PIX buf[8];
                buf[0] = in[base];
#if PIX_IS_U8
                unsigned short acc = buf[0];
#else
                PIX acc = buf[0];
#endif
                for (int i = 1; i < 8; ++i) {
                    int h = has & i;
                    buf[i] = (h == i) ? in[base + shift[i]] : buf[h];
                    acc += buf[i];
                }
#if PIX_IS_U8
                out[o] = (PIX)(acc >> 3);
#else
                out[o] = acc / 8;
#endif
            }
}


#undef FN
#undef CAT
#undef CAT_
