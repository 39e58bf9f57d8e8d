/* Test infrastructure only (the checker, never the product path).
 *
 * Plain-C restatement of the reference's NIfTI reader for one volume read as float
 * (io/nifti.hpp, io/gz_stream.hpp): header (NIfTI-1 or -2, either byte order,
 * .nii / .nii.gz / .hdr+.img), handle_qform (:1223-1260), toLPS (:129-160), the
 * element conversion of save_to_buffer (:1044-1131), scl_slope / scl_inter
 * (:1152-1158), then the flips and swaps applied one after another to the image
 * (numerical/basic_op.hpp:1030-1205), as the reference applies them.  gzip files
 * are read through zlib's gz interface.  Included once by oracle.c.
 */
#include <stdio.h>
#include <zlib.h>

static unsigned char* orc_read_file(const char* path, size_t* size)
{
    gzFile g = gzopen(path, "rb");
    if (!g)
        return NULL;
    size_t cap = 1 << 20, n = 0;
    unsigned char* b = (unsigned char*)malloc(cap);
    for (;;) {
        if (n == cap) {
            cap *= 2;
            b = (unsigned char*)realloc(b, cap);
        }
        int r = gzread(g, b + n, (unsigned)(cap - n > (1u << 30) ? (1u << 30) : cap - n));
        if (r <= 0)
            break;
        n += (size_t)r;
    }
    gzclose(g);
    *size = n;
    return b;
}

static void orc_swap_bytes(void* p, int n)
{
    unsigned char* c = (unsigned char*)p;
    for (int i = 0; i < n / 2; ++i) {
        unsigned char t = c[i];
        c[i] = c[n - 1 - i];
        c[n - 1 - i] = t;
    }
}

#define ORC_GET(T, name)                                                         \
    static T name(const unsigned char* p, int sw)                                \
    {                                                                            \
        T v;                                                                     \
        memcpy(&v, p, sizeof(T));                                                \
        if (sw)                                                                  \
            orc_swap_bytes(&v, sizeof(T));                                       \
        return v;                                                                \
    }
ORC_GET(int16_t, orc_i16)
ORC_GET(int32_t, orc_i32)
ORC_GET(int64_t, orc_i64)
ORC_GET(float, orc_f32)
ORC_GET(double, orc_f64)
#undef ORC_GET

/* one image operation (op 0..2 flip x/y/z, 3 swap xy, 4 swap yz, 5 swap xz) on a
 * (d[0], d[1], d[2]) float volume; d is updated */
static void orc_flip_op(float** img, int* d, int op)
{
    const size_t w = (size_t)d[0], h = (size_t)d[1], z = (size_t)d[2], n = w * h * z;
    float* I = *img;
    float* O = (float*)malloc(n * sizeof(float));
    for (size_t k = 0; k < z; ++k)
        for (size_t j = 0; j < h; ++j)
            for (size_t i = 0; i < w; ++i) {
                const float v = I[(k * h + j) * w + i];
                size_t o = 0;
                switch (op) {
                case 0: o = (k * h + j) * w + (w - 1 - i); break;
                case 1: o = (k * h + (h - 1 - j)) * w + i; break;
                case 2: o = ((z - 1 - k) * h + j) * w + i; break;
                case 3: o = (k * w + i) * h + j; break;         /* new dims (h, w, z) */
                case 4: o = (j * z + k) * w + i; break;         /* new dims (w, z, h) */
                case 5: o = (i * h + j) * z + k; break;         /* new dims (z, h, w) */
                }
                O[o] = v;
            }
    if (op == 3) { int t = d[0]; d[0] = d[1]; d[1] = t; }
    if (op == 4) { int t = d[1]; d[1] = d[2]; d[2] = t; }
    if (op == 5) { int t = d[0]; d[0] = d[2]; d[2] = t; }
    free(I);
    *img = O;
}

/* Loads volume `vol` of path as float in LPS orientation.  out: capacity cap floats;
 * dim, vs, srow (12), steps (8) and nsteps receive the geometry.  Returns 1 on
 * success, 0 on any failure. */
int orc_nifti_load(const char* path, int vol, float* out, long long cap, int* dim, float* vs, float* srow,
                   int* steps, int* nsteps)
{
    size_t fsize = 0;
    unsigned char* f = orc_read_file(path, &fsize);
    if (!f || fsize < 348) {
        free(f);
        return 0;
    }
    int sw = 0;
    int32_t hs = orc_i32(f, 0);
    if (hs != 348 && hs != 540) {
        hs = orc_i32(f, 1);
        if (hs != 348 && hs != 540) {
            free(f);
            return 0;
        }
        sw = 1;
    }
    int16_t dt, bp, d[8];
    float pix[8], vox_offset, slope, inter, qb, qc, qd, qx, qy, qz, R[12];
    int16_t qform, sform;
    int pair = 0;
    if (hs == 540) {
        if (fsize < 540 || !(f[4] == 'n' && f[5] == '+' && f[6] == '2')) {
            free(f);
            return 0;
        }
        dt = orc_i16(f + 12, sw);
        bp = orc_i16(f + 14, sw);
        for (int i = 0; i < 8; ++i) {
            d[i] = (int16_t)orc_i64(f + 16 + 8 * i, sw);
            pix[i] = (float)orc_f64(f + 104 + 8 * i, sw);
        }
        vox_offset = (float)orc_i64(f + 168, sw);
        slope = (float)orc_f64(f + 176, sw);
        inter = (float)orc_f64(f + 184, sw);
        qform = (int16_t)orc_i32(f + 344, sw);
        sform = (int16_t)orc_i32(f + 348, sw);
        qb = (float)orc_f64(f + 352, sw);
        qc = (float)orc_f64(f + 360, sw);
        qd = (float)orc_f64(f + 368, sw);
        qx = (float)orc_f64(f + 376, sw);
        qy = (float)orc_f64(f + 384, sw);
        qz = (float)orc_f64(f + 392, sw);
        for (int i = 0; i < 12; ++i)
            R[i] = (float)orc_f64(f + 400 + 8 * i, sw);
    } else {
        dt = orc_i16(f + 70, sw);
        bp = orc_i16(f + 72, sw);
        for (int i = 0; i < 8; ++i) {
            d[i] = orc_i16(f + 40 + 2 * i, sw);
            pix[i] = orc_f32(f + 76 + 4 * i, sw);
        }
        vox_offset = orc_f32(f + 108, sw);
        slope = orc_f32(f + 112, sw);
        inter = orc_f32(f + 116, sw);
        qform = orc_i16(f + 252, sw);
        sform = orc_i16(f + 254, sw);
        qb = orc_f32(f + 256, sw);
        qc = orc_f32(f + 260, sw);
        qd = orc_f32(f + 264, sw);
        qx = orc_f32(f + 268, sw);
        qy = orc_f32(f + 272, sw);
        qz = orc_f32(f + 276, sw);
        for (int i = 0; i < 12; ++i)
            R[i] = orc_f32(f + 280 + 4 * i, sw);
        const unsigned char* m = f + 344;
        const int is_nii = m[0] == 'n' && (m[2] == '1' || m[2] == '2') && (m[1] == 'i' || m[1] == '+');
        pair = !(is_nii && m[1] == '+');
    }
    /* handle_qform */
    if (qform > 0 && sform == 0) {
        const float b2 = qb * qb, c2 = qc * qc, d2 = qd * qd, sum = b2 + c2 + d2;
        const float a2 = (sum > 1.0f) ? 0.0f : 1.0f - sum;
        const float a = sqrtf(a2);
        const float ab2 = 2.0f * a * qb, ac2 = 2.0f * a * qc, ad2 = 2.0f * a * qd;
        const float bc2 = 2.0f * qb * qc, bd2 = 2.0f * qb * qd, cd2 = 2.0f * qc * qd;
        float qfac = pix[0];
        if (qfac == 0.0f)
            qfac = 1.0f;
        R[0] = (a2 + b2 - c2 - d2) * pix[1];
        R[1] = (bc2 - ad2) * pix[2];
        R[2] = (bd2 + ac2) * pix[3] * qfac;
        R[3] = qx;
        R[4] = (bc2 + ad2) * pix[1];
        R[5] = (a2 + c2 - b2 - d2) * pix[2];
        R[6] = (cd2 - ab2) * pix[3] * qfac;
        R[7] = qy;
        R[8] = (bd2 - ac2) * pix[1];
        R[9] = (cd2 + ab2) * pix[2];
        R[10] = (a2 + d2 - c2 - b2) * pix[3] * qfac;
        R[11] = qz;
    }
    /* the voxels of volume vol, as stored */
    const int16_t fd[3] = {d[1], d[2], d[3]};
    const int bpv = bp / 8;
    if (fd[0] <= 0 || fd[1] <= 0 || fd[2] <= 0 || bpv <= 0) {
        free(f);
        return 0;
    }
    const size_t n = (size_t)fd[0] * fd[1] * fd[2];
    unsigned char* data = f;
    size_t dsize = fsize, start = (size_t)vox_offset;
    if (pair) {
        char img[4096];
        snprintf(img, sizeof(img), "%s", path);
        char* dot = strrchr(img, '.');
        char* slash = strrchr(img, '/');
        if (dot && (!slash || dot > slash))
            strcpy(dot, ".img");
        else
            strcat(img, ".img");
        data = orc_read_file(img, &dsize);
        start = 0;
        if (!data) {
            free(f);
            return 0;
        }
    }
    start += (size_t)vol * n * bpv;
    if (dsize < start + n * bpv) {
        if (data != f)
            free(data);
        free(f);
        return 0;
    }
    float* I = (float*)malloc(n * sizeof(float));
    const unsigned char* p = data + start;
    for (size_t i = 0; i < n; ++i, p += bpv) {
        float v = 0.0f;
        switch (dt) {
        case 2: v = (float)p[0]; break;
        case 256: v = (float)(signed char)p[0]; break;
        case 4: v = (float)orc_i16(p, sw); break;
        case 512: v = (float)(uint16_t)orc_i16(p, sw); break;
        case 8: v = (float)orc_i32(p, sw); break;
        case 768: v = (float)(uint32_t)orc_i32(p, sw); break;
        case 16: v = orc_f32(p, sw); break;
        case 64: v = (float)orc_f64(p, sw); break;
        case 1024: v = (float)orc_i64(p, sw); break;
        case 1280: v = (float)(uint64_t)orc_i64(p, sw); break;
        case 128: /* tipl::rgb(r, g, b) as uint32: b low byte, alpha 0 (io/nifti.hpp:1113-1115) */
            v = (float)(((uint32_t)p[0] << 16) | ((uint32_t)p[1] << 8) | (uint32_t)p[2]);
            break;
        default: /* no conversion in the reference's float read: the voxel stays 0 */
            v = 0.0f;
            break;
        }
        if (slope != 0.0f) {
            if (slope != 1.0f)
                v = v * slope;
            if (inter != 0.0f)
                v = v + inter;
        }
        I[i] = v;
    }
    if (data != f)
        free(data);
    free(f);
    /* toLPS on the header, then the same steps on the image */
    int D[3] = {fd[0], fd[1], fd[2]};
    int16_t hd[3] = {fd[0], fd[1], fd[2]};
    float px[3] = {pix[1], pix[2], pix[3]};
    int seq[8], ns = 0;
#define ORC_SWP(a, b, op)                                                                  \
    do {                                                                                   \
        seq[ns++] = op;                                                                    \
        for (int r = 0; r < 12; r += 4) {                                                  \
            float t = R[r + a]; R[r + a] = R[r + b]; R[r + b] = t;                          \
        }                                                                                  \
        { float t = px[a]; px[a] = px[b]; px[b] = t; }                                     \
        { int16_t t = hd[a]; hd[a] = hd[b]; hd[b] = t; }                                   \
    } while (0)
#define ORC_FLP(a, op)                                                                     \
    do {                                                                                   \
        seq[ns++] = op;                                                                    \
        for (int r = 0; r < 12; r += 4) {                                                  \
            R[r + 3] += R[r + a] * (float)(hd[a] - 1);                                     \
            R[r + a] = -R[r + a];                                                          \
        }                                                                                  \
    } while (0)
    if (fabsf(R[5]) < fabsf(R[1]) && fabsf(R[9]) < fabsf(R[1])) ORC_SWP(0, 1, 3);
    if (fabsf(R[6]) < fabsf(R[2]) && fabsf(R[10]) < fabsf(R[2])) ORC_SWP(0, 2, 5);
    if (fabsf(R[2]) < fabsf(R[6]) && fabsf(R[10]) < fabsf(R[6])) ORC_SWP(1, 2, 4);
    if (R[0] > 0.0f) ORC_FLP(0, 0);
    if (R[5] > 0.0f) ORC_FLP(1, 1);
    if (R[10] < 0.0f) ORC_FLP(2, 2);
#undef ORC_SWP
#undef ORC_FLP
    for (int k = 0; k < ns; ++k)
        orc_flip_op(&I, D, seq[k]);
    if ((long long)n > cap) {
        free(I);
        return 0;
    }
    memcpy(out, I, n * sizeof(float));
    free(I);
    for (int i = 0; i < 3; ++i) {
        dim[i] = D[i];
        vs[i] = px[i];
    }
    memcpy(srow, R, sizeof(R));
    for (int k = 0; k < ns; ++k)
        steps[k] = seq[k];
    *nsteps = ns;
    return 1;
}
