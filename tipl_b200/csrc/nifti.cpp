// NIfTI reading and writing on the host (io/nifti.hpp, io/gz_stream.hpp of the
// reference).  Files are read through zlib's gz interface, which passes an
// uncompressed file through unchanged, so .nii and .nii.gz take the same path.
#include "nifti.h"
#include <zlib.h>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

namespace regb {

namespace {

struct GzFile {
    gzFile f = nullptr;
    ~GzFile()
    {
        if (f)
            gzclose(f);
    }
};

// The first n bytes of the (decompressed) file; fewer if the file is shorter.
std::vector<uint8_t> read_prefix(const std::string& path, size_t n)
{
    GzFile g;
    g.f = gzopen(path.c_str(), "rb");
    if (!g.f)
        throw Failure(REGB_ERR_ARG, "cannot open file: " + path);
    gzbuffer(g.f, 1 << 20);
    std::vector<uint8_t> out(n);
    size_t got = 0;
    while (got < n) {
        const unsigned chunk = (unsigned)std::min<size_t>(n - got, 1u << 30);
        const int r = gzread(g.f, out.data() + got, chunk);
        if (r < 0)
            throw Failure(REGB_ERR_ARG, "cannot read file: " + path);
        if (r == 0)
            break;
        got += (size_t)r;
    }
    out.resize(got);
    return out;
}

template <typename T>
T get(const uint8_t* p, bool swap)
{
    uint8_t b[sizeof(T)];
    std::memcpy(b, p, sizeof(T));
    if (swap)
        std::reverse(b, b + sizeof(T));
    T v;
    std::memcpy(&v, b, sizeof(T));
    return v;
}

// handle_qform (io/nifti.hpp:1223-1260): a qform-only header gets its srow rows from
// the quaternion, in float
void handle_qform(NiftiHeader& h)
{
    if (!(h.qform_code > 0 && h.sform_code == 0))
        return;
    const float b = h.quatern_b, c = h.quatern_c, d = h.quatern_d;
    const float b2 = b * b, c2 = c * c, d2 = d * d;
    const float sum = b2 + c2 + d2;
    const float a2 = (sum > 1.0f) ? 0.0f : 1.0f - sum;
    const float a = std::sqrt(a2);
    const float ab2 = 2.0f * a * b, ac2 = 2.0f * a * c, ad2 = 2.0f * a * d;
    const float bc2 = 2.0f * b * c, bd2 = 2.0f * b * d, cd2 = 2.0f * c * d;
    float qfac = h.pixdim[0];
    if (qfac == 0.0f)
        qfac = 1.0f;
    float* R = h.srow;
    R[0] = (a2 + b2 - c2 - d2) * h.pixdim[1];
    R[1] = (bc2 - ad2) * h.pixdim[2];
    R[2] = (bd2 + ac2) * h.pixdim[3] * qfac;
    R[3] = h.qoffset_x;
    R[4] = (bc2 + ad2) * h.pixdim[1];
    R[5] = (a2 + c2 - b2 - d2) * h.pixdim[2];
    R[6] = (cd2 - ab2) * h.pixdim[3] * qfac;
    R[7] = h.qoffset_y;
    R[8] = (bd2 - ac2) * h.pixdim[1];
    R[9] = (cd2 + ab2) * h.pixdim[2];
    R[10] = (a2 + d2 - c2 - b2) * h.pixdim[3] * qfac;
    R[11] = h.qoffset_z;
    h.sform_code = h.qform_code;
}

// toLPS (io/nifti.hpp:129-160): swaps to make each voxel axis the dominant one of its
// space axis, then flips toward L, P, S; updates dims, voxel sizes and rows
std::vector<char> to_lps(int16_t* dim, float* pixdim, float* R)
{
    std::vector<char> seq;
    auto swp = [&](int a, int b, char op) {
        seq.push_back(op);
        for (int r : {0, 4, 8})
            std::swap(R[r + a], R[r + b]);
        std::swap(pixdim[a], pixdim[b]);
        std::swap(dim[a], dim[b]);
    };
    auto flp = [&](int a, char op) {
        seq.push_back(op);
        for (int r : {0, 4, 8}) {
            R[r + 3] += R[r + a] * float(dim[a] - 1);
            R[r + a] = -R[r + a];
        }
    };
    if (std::fabs(R[5]) < std::fabs(R[1]) && std::fabs(R[9]) < std::fabs(R[1]))
        swp(0, 1, 3);
    if (std::fabs(R[6]) < std::fabs(R[2]) && std::fabs(R[10]) < std::fabs(R[2]))
        swp(0, 2, 5);
    if (std::fabs(R[2]) < std::fabs(R[6]) && std::fabs(R[10]) < std::fabs(R[6]))
        swp(1, 2, 4);
    if (R[0] > 0.0f)
        flp(0, 0);
    if (R[5] > 0.0f)
        flp(1, 1);
    if (R[10] < 0.0f)
        flp(2, 2);
    return seq;
}

// The voxel map of a flip/swap sequence (numerical/basic_op.hpp:1030-1205 applied in
// order): file voxel = M * (voxel of the reoriented volume) + o.
void sequence_map(const std::vector<char>& seq, const int16_t* file_dim, int* M, long long* o)
{
    long long D[3] = {file_dim[1], file_dim[2], file_dim[3]};
    int m[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    long long off[3] = {0, 0, 0};
    for (char op : seq) {
        if (op <= 2) {
            // flip axis a: current voxel c = (new voxel with c[a] = D[a] - 1 - n[a])
            const int a = op;
            for (int r = 0; r < 3; ++r) {
                off[r] += (long long)m[3 * r + a] * (D[a] - 1);
                m[3 * r + a] = -m[3 * r + a];
            }
        } else {
            // swap axes a, b: current voxel c = new voxel with components a, b exchanged
            const int a = op == 3 ? 0 : (op == 4 ? 1 : 0);
            const int b = op == 3 ? 1 : 2;
            for (int r = 0; r < 3; ++r)
                std::swap(m[3 * r + a], m[3 * r + b]);
            std::swap(D[a], D[b]);
        }
    }
    std::memcpy(M, m, sizeof(m));
    for (int r = 0; r < 3; ++r)
        o[r] = off[r];
}

std::string img_path(const std::string& path)
{
    // the .img beside a .hdr (std::filesystem::path::replace_extension)
    const size_t slash = path.find_last_of("/\\");
    const size_t dot = path.find_last_of('.');
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash))
        return path + ".img";
    return path.substr(0, dot) + ".img";
}

}  // namespace

int nifti_bytes_per_voxel(int datatype, int bitpix)
{
    // the datatypes the reference's float read converts (io/nifti.hpp:1096-1131) keep
    // their element size; every other code is read as bitpix / 8 bytes and left at 0
    // (that read has no conversion for them: complex, float128, RGBA32, ...)
    int size = 0;
    switch (datatype) {
    case 2: case 256: size = 1; break;
    case 4: case 512: size = 2; break;
    case 128: size = 3; break;  // RGB: r, g, b bytes
    case 8: case 16: case 768: size = 4; break;
    case 64: case 1024: case 1280: size = 8; break;
    default: return bitpix >= 8 ? bitpix / 8 : 0;
    }
    return bitpix == 8 * size ? size : 0;
}

NiftiFile nifti_open(const std::string& path)
{
    std::vector<uint8_t> b = read_prefix(path, 540);
    if (b.size() < 348)
        throw Failure(REGB_ERR_ARG, "invalid NIFTI format: file shorter than a header: " + path);
    NiftiFile f;
    NiftiHeader& h = f.h;
    int size = get<int32_t>(b.data(), false);
    if (size != 540 && size != 348) {
        size = get<int32_t>(b.data(), true);
        if (size != 540 && size != 348)
            throw Failure(REGB_ERR_ARG, "invalid NIFTI format: size of header is not 540 or 348");
        h.big_endian = true;
    }
    const bool sw = h.big_endian;
    const uint8_t* p = b.data();
    if (size == 540) {
        if (b.size() < 540)
            throw Failure(REGB_ERR_ARG, "invalid NIFTI format: truncated NIfTI-2 header");
        if (!(p[4] == 'n' && p[5] == '+' && p[6] == '2'))
            throw Failure(REGB_ERR_ARG, "invalid NIFTI format: no NIFTI tag found.");
        h.nifti2 = true;
        h.datatype = get<int16_t>(p + 12, sw);
        h.bitpix = get<int16_t>(p + 14, sw);
        for (int i = 0; i < 8; ++i) {
            h.dim[i] = (int16_t)get<int64_t>(p + 16 + 8 * i, sw);
            h.pixdim[i] = (float)get<double>(p + 104 + 8 * i, sw);
        }
        h.vox_offset = (float)get<int64_t>(p + 168, sw);
        h.scl_slope = (float)get<double>(p + 176, sw);
        h.scl_inter = (float)get<double>(p + 184, sw);
        std::memcpy(h.descrip, p + 240, 80);
        h.qform_code = (int16_t)get<int32_t>(p + 344, sw);
        h.sform_code = (int16_t)get<int32_t>(p + 348, sw);
        h.quatern_b = (float)get<double>(p + 352, sw);
        h.quatern_c = (float)get<double>(p + 360, sw);
        h.quatern_d = (float)get<double>(p + 368, sw);
        h.qoffset_x = (float)get<double>(p + 376, sw);
        h.qoffset_y = (float)get<double>(p + 384, sw);
        h.qoffset_z = (float)get<double>(p + 392, sw);
        for (int i = 0; i < 12; ++i)
            h.srow[i] = (float)get<double>(p + 400 + 8 * i, sw);
    } else {
        h.datatype = get<int16_t>(p + 70, sw);
        h.bitpix = get<int16_t>(p + 72, sw);
        for (int i = 0; i < 8; ++i) {
            h.dim[i] = get<int16_t>(p + 40 + 2 * i, sw);
            h.pixdim[i] = get<float>(p + 76 + 4 * i, sw);
        }
        h.vox_offset = get<float>(p + 108, sw);
        h.scl_slope = get<float>(p + 112, sw);
        h.scl_inter = get<float>(p + 116, sw);
        std::memcpy(h.descrip, p + 148, 80);
        h.qform_code = get<int16_t>(p + 252, sw);
        h.sform_code = get<int16_t>(p + 254, sw);
        h.quatern_b = get<float>(p + 256, sw);
        h.quatern_c = get<float>(p + 260, sw);
        h.quatern_d = get<float>(p + 264, sw);
        h.qoffset_x = get<float>(p + 268, sw);
        h.qoffset_y = get<float>(p + 272, sw);
        h.qoffset_z = get<float>(p + 276, sw);
        for (int i = 0; i < 12; ++i)
            h.srow[i] = get<float>(p + 280 + 4 * i, sw);
        const char* mg = (const char*)p + 344;
        const bool is_nii = mg[0] == 'n' && (mg[2] == '1' || mg[2] == '2') && (mg[1] == 'i' || mg[1] == '+');
        h.pair = !(is_nii && mg[1] == '+');
    }
    std::memcpy(f.file_dim, h.dim, sizeof(h.dim));
    handle_qform(h);
    f.seq = to_lps(h.dim + 1, h.pixdim + 1, h.srow);
    sequence_map(f.seq, f.file_dim, f.M, f.o);
    return f;
}

std::vector<uint8_t> nifti_read_voxels(const std::string& path, const NiftiFile& f, int vol)
{
    const int bpv = nifti_bytes_per_voxel(f.h.datatype, f.h.bitpix);
    if (bpv == 0)
        throw Failure(REGB_ERR_ARG, "unsupported NIfTI datatype " + std::to_string(f.h.datatype) + " / bitpix " +
                                        std::to_string(f.h.bitpix));
    const long long n = (long long)f.file_dim[1] * f.file_dim[2] * f.file_dim[3];
    if (f.file_dim[1] <= 0 || f.file_dim[2] <= 0 || f.file_dim[3] <= 0)
        throw Failure(REGB_ERR_ARG, "invalid dim value");
    long long nvol = 1;
    for (int i = 4; i <= 7 && i <= f.file_dim[0]; ++i)
        nvol *= std::max<int16_t>(f.file_dim[i], 1);
    if (vol < 0 || vol >= nvol)
        throw Failure(REGB_ERR_ARG, "volume index out of range");
    const size_t vbytes = (size_t)n * bpv;
    const size_t start = f.h.pair ? 0 : (size_t)f.h.vox_offset;
    const size_t begin = start + (size_t)vol * vbytes;
    std::vector<uint8_t> all = read_prefix(f.h.pair ? img_path(path) : path, begin + vbytes);
    if (all.size() < begin + vbytes)
        throw Failure(REGB_ERR_ARG, "end of file reached. The file is smaller than expected.");
    return std::vector<uint8_t>(all.begin() + begin, all.begin() + begin + vbytes);
}

void nifti_write(const std::string& path, const void* data, int datatype, int bitpix, const int dim[3],
                 const float vs[3], const float srow[12], int sform_code, const char* descrip, int nvol)
{
    uint8_t hdr[352];
    std::memset(hdr, 0, sizeof(hdr));
    auto put = [&](size_t off, const void* v, size_t n) { std::memcpy(hdr + off, v, n); };
    const int32_t sizeof_hdr = 348;
    put(0, &sizeof_hdr, 4);
    // a 4-D image (nvol > 1) carries its volumes in dim[4] (set_dim, io/nifti.hpp:787-792)
    int16_t d[8] = {(int16_t)(nvol > 1 ? 4 : 3), (int16_t)dim[0], (int16_t)dim[1], (int16_t)dim[2],
                    (int16_t)(nvol > 1 ? nvol : 1), 1, 1, 1};
    put(40, d, 16);
    const int16_t dt = (int16_t)datatype, bp = (int16_t)bitpix;
    put(70, &dt, 2);
    put(72, &bp, 2);
    float pix[8] = {3.0f, vs[0], vs[1], vs[2], 1.0f, 1.0f, 1.0f, 1.0f};
    put(76, pix, 32);
    const float vox_offset = 352.0f, slope = 1.0f;
    put(108, &vox_offset, 4);
    put(112, &slope, 4);
    if (descrip)
        std::memcpy(hdr + 148, descrip, std::min<size_t>(80, std::strlen(descrip)));
    const int16_t qc = 0, sc = (int16_t)sform_code;
    put(252, &qc, 2);
    put(254, &sc, 2);
    const float qc_c = 1.0f;  // the writer's initial quaternion (io/nifti.hpp:889-908)
    put(260, &qc_c, 4);
    put(280, srow, 48);
    const char magic[4] = {'n', '+', '1', 0};
    put(344, magic, 4);
    const size_t bytes = (size_t)dim[0] * dim[1] * dim[2] * (size_t)(bitpix / 8) * (size_t)(nvol > 1 ? nvol : 1);
    // the reference's output stream is always gzip (io/gz_stream.hpp:535-580), whatever
    // the file name says; its reader and this one take either form
    GzFile g;
    g.f = gzopen(path.c_str(), "wb");
    if (!g.f)
        throw Failure(REGB_ERR_ARG, "cannot write to " + path);
    if (gzwrite(g.f, hdr, sizeof(hdr)) != (int)sizeof(hdr))
        throw Failure(REGB_ERR_ARG, "cannot write to " + path);
    size_t done = 0;
    while (done < bytes) {
        const unsigned chunk = (unsigned)std::min<size_t>(bytes - done, 1u << 30);
        if (gzwrite(g.f, (const char*)data + done, chunk) != (int)chunk)
            throw Failure(REGB_ERR_ARG, "cannot write to " + path);
        done += chunk;
    }
    const int rc = gzclose(g.f);
    g.f = nullptr;
    if (rc != Z_OK)
        throw Failure(REGB_ERR_ARG, "cannot write to " + path);
}

}  // namespace regb
