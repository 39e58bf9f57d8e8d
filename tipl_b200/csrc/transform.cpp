// Transform algebra on the host, in the reference's float arithmetic so the
// transforms handed to the kernels are bit-identical to the ones the reference
// would build from the same parameters.  Compiled without FMA contraction.
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include "host.h"

namespace regb {

static thread_local std::string g_last_error;

void set_last_error(const std::string& s) { g_last_error = s; }
const std::string& last_error() { return g_last_error; }

void throw_cuda(cudaError_t e, const char* what)
{
    (void)cudaGetLastError();
    throw Failure(REGB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Size classes are powers of two from 256 bytes; at most kPinnedCacheBytes stay cached.
namespace {
constexpr size_t kPinnedCacheBytes = size_t(256) << 20;
std::mutex g_pin_m;
std::map<size_t, std::vector<void*>> g_pin_free;
size_t g_pin_cached = 0;
size_t pin_class(size_t b)
{
    size_t c = 256;
    while (c < b)
        c <<= 1;
    return c;
}
}  // namespace

void* pinned_get(size_t& bytes)
{
    bytes = pin_class(bytes);
    {
        std::lock_guard<std::mutex> g(g_pin_m);
        auto it = g_pin_free.find(bytes);
        if (it != g_pin_free.end() && !it->second.empty()) {
            void* p = it->second.back();
            it->second.pop_back();
            g_pin_cached -= bytes;
            return p;
        }
    }
    void* p = nullptr;
    REGB_CK(cudaMallocHost(&p, bytes));
    return p;
}

void pinned_put(void* p, size_t bytes)
{
    {
        std::lock_guard<std::mutex> g(g_pin_m);
        if (g_pin_cached + bytes <= kPinnedCacheBytes) {
            g_pin_free[bytes].push_back(p);
            g_pin_cached += bytes;
            return;
        }
    }
    cudaFreeHost(p);
}

void pinned_trim()
{
    std::map<size_t, std::vector<void*>> all;
    {
        std::lock_guard<std::mutex> g(g_pin_m);
        all.swap(g_pin_free);
        g_pin_cached = 0;
    }
    for (auto& kv : all)
        for (void* p : kv.second)
            cudaFreeHost(p);
}

size_t pix_size(int dtype)
{
    switch (dtype) {
    case REGB_U8: return 1;
    case REGB_F32: return 4;
    case REGB_U16:
    case REGB_BF16: return 2;
    default: return 0;
    }
}

void ensure_device()
{
    static std::mutex m;
    static bool done[64] = {false};
    int dev = 0;
    REGB_CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(m);
    if (dev < 64 && !done[dev]) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;  // keep freed blocks pooled instead of returning them each sync
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        (void)cudaGetLastError();
        done[dev] = true;
    }
}

// transformation_matrix(affine_param, from, from_vs, to, to_vs)
// (numerical/transformation.hpp:636-675): rotation_matrix (transformation.hpp:143-164),
// row scaling (196-208), shear (220-231), then the voxel-space composition.
void affine_to_matrix(const float* p, const int* fd, const float* fvs, const int* td, const float* tvs, float* T)
{
    const float* tr = p;
    const float* th = p + 3;
    const float* s = p + 6;
    const float* a = p + 9;
    float* m = T;
    const float sin_x = std::sin(th[0]), cos_x = std::cos(th[0]);
    const float sin_y = std::sin(th[1]), cos_y = std::cos(th[1]);
    const float sin_z = std::sin(th[2]), cos_z = std::cos(th[2]);
    const float cxsz = cos_x * sin_z, cxcz = cos_x * cos_z, sxsz = sin_x * sin_z, sxcz = sin_x * cos_z;
    m[0] = cos_y * cos_z;
    m[1] = cos_y * sin_z;
    m[2] = -sin_y;
    m[3] = -cxsz + sxcz * sin_y;
    m[4] = cxcz + sxsz * sin_y;
    m[5] = sin_x * cos_y;
    m[6] = sxsz + cxcz * sin_y;
    m[7] = -sxcz + cxsz * sin_y;
    m[8] = cos_x * cos_y;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            m[3 * r + c] *= s[r];
    m[0] += m[3] * a[0] + m[6] * a[1];
    m[1] += m[4] * a[0] + m[7] * a[1];
    m[2] += m[5] * a[0] + m[8] * a[1];
    m[3] += m[6] * a[2];
    m[4] += m[7] * a[2];
    m[5] += m[8] * a[2];
    float t[3] = {(float)fd[0], (float)fd[1], (float)fd[2]};
    for (int i = 0; i < 3; ++i)
        t[i] *= -0.5f;
    for (int i = 0; i < 3; ++i)
        t[i] *= fvs[i];
    for (int i = 0; i < 3; ++i)
        t[i] += tr[i];
    float* sh = T + 9;
    for (int r = 0; r < 3; ++r)
        sh[r] = m[3 * r] * t[0] + m[3 * r + 1] * t[1] + m[3 * r + 2] * t[2];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            m[3 * r + c] *= fvs[c];
    for (int r = 0; r < 3; ++r)
        if (tvs[r] != 1.0f) {
            m[3 * r] /= tvs[r];
            m[3 * r + 1] /= tvs[r];
            m[3 * r + 2] /= tvs[r];
            sh[r] /= tvs[r];
        }
    for (int r = 0; r < 3; ++r)
        sh[r] += (float)td[r] * 0.5f;
}

void affine_to_matrix_f64(const double* p, const int* fd, const double* fvs, const int* td, const double* tvs,
                          double* T)
{
    const double* th = p + 3;
    const double* s = p + 6;
    const double* a = p + 9;
    double* m = T;
    const double sx = std::sin(th[0]), cx = std::cos(th[0]);
    const double sy = std::sin(th[1]), cy = std::cos(th[1]);
    const double sz = std::sin(th[2]), cz = std::cos(th[2]);
    m[0] = cy * cz;
    m[1] = cy * sz;
    m[2] = -sy;
    m[3] = -cx * sz + sx * cz * sy;
    m[4] = cx * cz + sx * sz * sy;
    m[5] = sx * cy;
    m[6] = sx * sz + cx * cz * sy;
    m[7] = -sx * cz + cx * sz * sy;
    m[8] = cx * cy;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            m[3 * r + c] *= s[r];
    m[0] += m[3] * a[0] + m[6] * a[1];
    m[1] += m[4] * a[0] + m[7] * a[1];
    m[2] += m[5] * a[0] + m[8] * a[1];
    m[3] += m[6] * a[2];
    m[4] += m[7] * a[2];
    m[5] += m[8] * a[2];
    double t[3];
    for (int i = 0; i < 3; ++i)
        t[i] = (double)fd[i] * -0.5 * fvs[i] + p[i];
    double* sh = T + 9;
    for (int r = 0; r < 3; ++r)
        sh[r] = m[3 * r] * t[0] + m[3 * r + 1] * t[1] + m[3 * r + 2] * t[2];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            m[3 * r + c] = m[3 * r + c] * fvs[c] / tvs[r];
    for (int r = 0; r < 3; ++r)
        sh[r] = sh[r] / tvs[r] + (double)td[r] * 0.5;
}

// transformation_matrix::inverse (numerical/transformation.hpp:820-832), cofactor
// inverse of numerical/matrix.hpp:1479-1505; false (T unchanged) when singular.
bool matrix_inverse(float* T)
{
    const float* a = T;
    const float det = a[0] * (a[4] * a[8] - a[5] * a[7]) + a[1] * (a[5] * a[6] - a[3] * a[8]) +
                      a[2] * (a[3] * a[7] - a[4] * a[6]);
    if (det + 1.0f == 1.0f)
        return false;
    float t[9] = {a[4] * a[8] - a[5] * a[7], a[2] * a[7] - a[1] * a[8], a[1] * a[5] - a[2] * a[4],
                  a[5] * a[6] - a[3] * a[8], a[0] * a[8] - a[2] * a[6], a[2] * a[3] - a[0] * a[5],
                  a[3] * a[7] - a[4] * a[6], a[1] * a[6] - a[0] * a[7], a[0] * a[4] - a[1] * a[3]};
    for (float& v : t)
        v = v / det;
    float ns[3];
    for (int r = 0; r < 3; ++r)
        ns[r] = T[9] * t[3 * r] + T[10] * t[3 * r + 1] + T[11] * t[3 * r + 2];
    for (int r = 0; r < 3; ++r)
        T[9 + r] = -ns[r];
    for (int i = 0; i < 9; ++i)
        T[i] = t[i];
    return true;
}

// The CPU resample's integer-shift test (numerical/resampling.hpp:1243-1258).
bool integer_shift(const float* T, int* shift)
{
    const double eps = 1.0e-4;
    for (int i = 0; i < 3; ++i) {
        const long s = std::lround(T[9 + i]);
        if (std::fabs(T[9 + i] - (float)s) > eps)
            return false;
        shift[i] = (int)s;
        for (int j = 0; j < 3; ++j)
            if (std::fabs(T[3 * i + j] - (float)(i == j)) > eps)
                return false;
    }
    return true;
}

}  // namespace regb
