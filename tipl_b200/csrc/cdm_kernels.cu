// CDM nonlinear registration passes (reg/cdm.hpp) and the displacement algebra
// they use (numerical/dif.hpp), as segment kernels: a launch covers one or more job
// levels (CdmSeg entries), each owning nblk consecutive blocks of a 1-D grid that
// stride over its voxels.
//
// One iteration of a level (reg/cdm.hpp:418-470) is the launch sequence
//   compose -> gradient (+ loop decisions in its last block) -> 12 Poisson sweeps
//   (the first also saves/restores best_d, the last forms theta) -> accumulate -> smooth
// The reference's host-side decisions (cost bookkeeping, cdm_improved, the
// smoothing schedule, best_d save/restore, theta, the iteration cap) run on the
// device against CdmCtl, so a level runs without any host round trip; every
// kernel of an iteration reads ctl->done and returns once a level has left its loop.
#include <atomic>
#include <cfloat>
#include "common.cuh"
#include "stats.h"

namespace regb {

constexpr int kCdmThreads = 256;

int cdm_blocks_for(long long nvox)
{
    long long b = (nvox + kCdmThreads - 1) / kCdmThreads;
    if (b > 148 * 8)
        b = 148 * 8;
    return (int)(b < 1 ? 1 : b);
}

// The segment entry a block of a launch over nseg entries works on: the last one
// whose blk0 <= blockIdx.x.  Every warp finds it on its own with one ballot per 32
// entries (all lanes active: this runs first in each kernel); a launch of one entry
// reads nothing to find it.
__device__ __forceinline__ int seg_of_block(const CdmSeg* __restrict__ segs, int nseg)
{
    if (nseg <= 1)
        return 0;
    const int b = (int)blockIdx.x, lane = threadIdx.x & 31;
    int k = 0;
    for (int base = 0; base < nseg; base += 32) {
        const int i = base + lane;
        const unsigned m = __ballot_sync(0xffffffffu, i < nseg && segs[i].blk0 <= b);
        k += __popc(m);
        if (m != 0xffffffffu)
            break;
    }
    return k - 1;
}

// MULTI: the kernel's instantiation for launches over several entries; a launch of one
// entry takes the other, which has no lookup in its code at all.
#define SEG_BEGIN                                                  \
    const CdmSeg& S = segs[MULTI ? seg_of_block(segs, nseg) : 0];  \
    const int blk = (int)blockIdx.x - (MULTI ? S.blk0 : 0);        \
    if (blk >= S.nblk)                                             \
        return;                                                    \
    const Dim3 D{S.w, S.h, S.d};                                   \
    const long long n = D.n();                                     \
    const long long stride = (long long)S.nblk * blockDim.x;       \
    const long long first = (long long)blk * blockDim.x + threadIdx.x;

// ------------------------------------------------------------------ compose
// compose_displacement (numerical/dif.hpp:90-107, 260-285): Js = Is[mod] where the
// displacement is exactly zero, else the trilinear sample at x + d; failed
// samples are 0.
template <typename T, bool MULTI>
__global__ void __launch_bounds__(kCdmThreads) cdm_compose_kernel(const CdmSeg* __restrict__ segs, int nseg, int mod)
{
    SEG_BEGIN
    if (S.ctl->done || mod >= max(S.nmod, 1))
        return;
    const T* __restrict__ Is = (const T*)S.Is[mod];
    T* __restrict__ Js = (T*)S.Js;
    const float* __restrict__ cd = S.cur_d;
    if (S.ndim == 2) {
        // the 2-D form: vector<2> field, bilinear sample at (x + dx, y + dy)
        for (long long i = first; i < n; i += stride) {
            const float dx = cd[3 * i], dy = cd[3 * i + 1];
            T v;
            if (dx == 0.0f && dy == 0.0f)
                v = Is[i];
            else {
                const int x = (int)(i % D.w), y = (int)(i / D.w);
                float px = (float)x, py = (float)y;
                px += dx;
                py += dy;
                Cell2 c;
                v = T(0);
                if (bilinear_cell(D, px, py, c))
                    v = assign_pix<T>(cell_sum2(Is, D, c));
            }
            Js[i] = v;
        }
        return;
    }
    for (long long i = first; i < n; i += stride) {
        const float dx = cd[3 * i], dy = cd[3 * i + 1], dz = cd[3 * i + 2];
        T v;
        if (dx == 0.0f && dy == 0.0f && dz == 0.0f)
            v = Is[i];
        else {
            int x, y, z;
            unflat((int)i, D, x, y, z);
            float px = (float)x, py = (float)y, pz = (float)z;
            px += dx;
            py += dy;
            pz += dz;
            Cell c;
            v = T(0);
            if (trilinear_cell(D, px, py, pz, c))
                v = assign_pix<T>(cell_sum(Is, D, c));
        }
        Js[i] = v;
    }
}

__device__ void control_block(const CdmSeg& S, int mod);
__device__ __forceinline__ bool last_block_of_segment(const CdmSeg& S);

// ------------------------------------------------------------------ gradient
// Window sums of linear_regression over the clipped 5^3 window
// (numerical/window.hpp:92-110, numerical/statistics.hpp:694-713).  Integer
// pixels: exact integer sums (the reference sums in int64).  Float pixels: double
// sums in the reference's visiting order with float cross products.
struct Reg {
    float a, b, r2;
};

__device__ __forceinline__ void regress_finish(double sx, double sy, double sxx, double syy, double sxy, int m,
                                               Reg& r)
{
    const double dn = (double)m;
    const double mx = sx / dn, my = sy / dn;
    const double xv = sxx / dn - mx * mx;
    const double yv = syy / dn - my * my;
    if (xv == 0.0 || yv == 0.0) {
        r.a = 0.0f;
        r.b = (float)my;
        r.r2 = 0.0f;
        return;
    }
    const double cov = sxy / dn - mx * my;
    r.a = (float)(cov / xv);
    r.b = (float)(my - (double)r.a * mx);  // b uses the float-rounded slope
    r.r2 = (float)(cov * cov / xv / yv);
}

template <typename T>
struct WindowAcc;

template <>
struct WindowAcc<uint8_t> {
    int sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0, m = 0;
    __device__ __forceinline__ void add(uint8_t j, uint8_t t)
    {
        const int a = j, b = t;
        sx += a;
        sy += b;
        sxx += a * a;
        syy += b * b;
        sxy += a * b;
        ++m;
    }
    __device__ __forceinline__ void finish(Reg& r) const
    {
        regress_finish((double)sx, (double)sy, (double)sxx, (double)syy, (double)sxy, m, r);
    }
};

template <>
struct WindowAcc<float> {
    double sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0;
    int m = 0;
    __device__ __forceinline__ void add(float j, float t)
    {
        // sum(): first element then +=; square_sum(): 0 + t*t in double;
        // inner_product(): float product widened to double.
        if (m == 0) {
            sx = (double)j;
            sy = (double)t;
            sxy = (double)(j * t);
        } else {
            sx += (double)j;
            sy += (double)t;
            sxy += (double)(j * t);
        }
        const double dj = j, dt = t;
        sxx += dj * dj;
        syy += dt * dt;
        ++m;
    }
    __device__ __forceinline__ void finish(Reg& r) const { regress_finish(sx, sy, sxx, syy, sxy, m, r); }
};

template <typename T>
__device__ __forceinline__ float pix_diff(T a, T b)
{
    return (float)(a - b);
}
template <>
__device__ __forceinline__ float pix_diff<uint8_t>(uint8_t a, uint8_t b)
{
    return (float)((int)a - (int)b);
}

// gradient_at (numerical/numerical.hpp:102-109)
template <typename T>
__device__ __forceinline__ float3 grad_at(const T* __restrict__ I, const Dim3& D, int x, int y, int z, long long i)
{
    float3 g;
    const long long w = D.w, wh = D.wh();
    g.x = (x + 1 < D.w && x) ? pix_diff(I[i + 1], I[i - 1]) : 0.0f;
    g.y = (y + 1 < D.h && y) ? pix_diff(I[i + w], I[i - w]) : 0.0f;
    g.z = (z + 1 < D.d && z) ? pix_diff(I[i + wh], I[i - wh]) : 0.0f;
    return g;
}

// Stores modality mod's gradient term dd = 0 + g: new_d = dd for the first modality,
// new_d += dd for the others (reg/cdm.hpp:430-433).
__device__ __forceinline__ void store_term(float* __restrict__ nd, long long i, float3 out, int mod)
{
    if (mod) {
        out.x = nd[3 * i] + out.x;
        out.y = nd[3 * i + 1] + out.y;
        out.z = nd[3 * i + 2] + out.z;
    }
    nd[3 * i] = out.x;
    nd[3 * i + 1] = out.y;
    nd[3 * i + 2] = out.z;
}

// cdm_get_gradient_r_imp / _d_imp (reg/cdm.hpp:46-78) of modality mod: the term is
// 0 + gradient term; the cost of every voxel (0 where skipped) is summed per block in
// double.
template <typename T, bool MULTI>
__global__ void __launch_bounds__(kCdmThreads) cdm_gradient_kernel(const CdmSeg* __restrict__ segs, int nseg, int gtype,
                                                                   int mod)
{
    SEG_BEGIN
    if (S.ctl->done || mod >= max(S.nmod, 1))
        return;
    const T* __restrict__ Js = (const T*)S.Js;
    const T* __restrict__ It = (const T*)S.It[mod];
    float* __restrict__ nd = S.new_d;
    double csum = 0.0;
    for (long long i = first; i < n; i += stride) {
        int x, y, z;
        unflat((int)i, D, x, y, z);
        float3 out = make_float3(0.0f, 0.0f, 0.0f);
        float cost = 0.0f;
        const T js = Js[i], it = It[i];
        if (gtype == 'd') {
            float3 g = grad_at(Js, D, x, y, z, i);
            const float dif = pix_diff(js, it);
            g.x *= dif;
            g.y *= dif;
            g.z *= dif;
            out.x = 0.0f + g.x;
            out.y = 0.0f + g.y;
            out.z = 0.0f + g.z;
            cost = dif * dif;
        } else if (!(js == T(0) || it == T(0))) {
            const int xu = min(D.w - x - 1, 2), yu = min(D.h - y - 1, 2), zu = min(D.d - z - 1, 2);
            const int xl = min(x, 2), yl = min(y, 2), zl = min(z, 2);
            const long long w = D.w, wh = D.wh();
            WindowAcc<T> acc;
            // (float pixels only: the uint8 'r' gradient is the box-sum kernel below)
            if (sizeof(T) == 4 && xu == 2 && xl == 2 && yu == 2 && yl == 2 && zu == 2 && zl == 2) {
                // an interior voxel: the whole 5^3 window, visited in the same order
                // with every offset known -- no loop bounds, no index arithmetic per tap
                const T* __restrict__ pj = Js + i;
                const T* __restrict__ pt = It + i;
                constexpr int kOrd[5] = {0, 1, 2, -1, -2};
#pragma unroll
                for (int a = 0; a < 5; ++a) {
#pragma unroll
                    for (int b = 0; b < 5; ++b) {
                        const long long row = kOrd[a] * wh + kOrd[b] * w;
                        const T* __restrict__ rj = pj + row;
                        const T* __restrict__ rt = pt + row;
#pragma unroll
                        for (int c = 0; c < 5; ++c)
                            acc.add(rj[kOrd[c]], rt[kOrd[c]]);
                    }
                }
            } else
            // iterate_xyz order (numerical/window.hpp:54-72)
            for (int pz = 0; pz < 2; ++pz) {
                const int zc = pz ? zl : zu;
                for (int dz = pz; dz <= zc; ++dz) {
                    const long long zi = i + (pz ? -dz : dz) * wh;
                    for (int py = 0; py < 2; ++py) {
                        const int yc = py ? yl : yu;
                        for (int dy = py; dy <= yc; ++dy) {
                            const long long yi = zi + (py ? -dy : dy) * w;
                            for (int dx = 0; dx <= xu; ++dx)
                                acc.add(Js[yi + dx], It[yi + dx]);
                            for (int dx = 1; dx <= xl; ++dx)
                                acc.add(Js[yi - dx], It[yi - dx]);
                        }
                    }
                }
            }
            Reg r;
            acc.finish(r);
            if (r.a > 0.0f) {
                float3 g = grad_at(Js, D, x, y, z, i);
                const float s = r.r2 * ((float)js * r.a + r.b - (float)it);
                g.x *= s;
                g.y *= s;
                g.z *= s;
                out.x = 0.0f + g.x;
                out.y = 0.0f + g.y;
                out.z = 0.0f + g.z;
                cost = -r.r2;
            }
        }
        store_term(nd, i, out, mod);
        csum += (double)cost;
    }
    __shared__ double red[32];
    csum = block_sum(csum, red);
    if (threadIdx.x == 0)
        S.cost_part[blk] = csum;
    if (last_block_of_segment(S))
        control_block(S, mod);
}

// Tiled uint8 'r' gradient.  For integer pixels the regression's window sums
// (sum Js, sum It, sum Js^2, sum It^2, sum Js*It over the clipped 5^3 window) are
// exact integers, so they are formed here as separable 5-tap box sums over a
// shared-memory tile (zero outside the volume, the window size m from the clipped
// extents) -- the same integers the reference sums voxel by voxel, hence
// bit-identical results at a fraction of the loads.
constexpr int kTX = 32, kTY = 4, kTZ = 4, kBoxThreads = 128;
constexpr int kHX = kTX + 4, kHY = kTY + 4, kHZ = kTZ + 4;
struct BoxSmem {
    uint8_t J[kHZ][kHY][kHX];
    uint8_t I[kHZ][kHY][kHX];
    int p1[5][kHZ][kHY][kTX];  // x-summed
    int p2[5][kHZ][kTY][kTX];  // x,y-summed
};

template <bool MULTI>
__global__ void __launch_bounds__(kBoxThreads) cdm_gradient_box_u8_kernel(const CdmSeg* __restrict__ segs, int nseg,
                                                                                    int mod)
{
    const CdmSeg& S = segs[MULTI ? seg_of_block(segs, nseg) : 0];
    const int blk = (int)blockIdx.x - (MULTI ? S.blk0 : 0);
    if (blk >= S.nblk)
        return;
    if (S.ctl->done || mod >= max(S.nmod, 1))
        return;
    extern __shared__ __align__(16) unsigned char smraw[];
    BoxSmem& sm = *reinterpret_cast<BoxSmem*>(smraw);
    const Dim3 D{S.w, S.h, S.d};
    const uint8_t* __restrict__ Js = (const uint8_t*)S.Js;
    const uint8_t* __restrict__ It = (const uint8_t*)S.It[mod];
    float* __restrict__ nd = S.new_d;
    const int ntx = (D.w + kTX - 1) / kTX, nty = (D.h + kTY - 1) / kTY, ntz = (D.d + kTZ - 1) / kTZ;
    const int ntiles = ntx * nty * ntz;
    const long long wl = D.w, whl = D.wh();
    double csum = 0.0;
    for (int tile = blk; tile < ntiles; tile += S.nblk) {
        const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
        const int x0 = tx * kTX, y0 = ty * kTY, z0 = tz * kTZ;
        __syncthreads();  // the previous tile's readers are done with the buffers
        for (int k = threadIdx.x; k < kHZ * kHY * kHX; k += blockDim.x) {
            const int hx = k % kHX, hy = (k / kHX) % kHY, hz = k / (kHX * kHY);
            const int gx = x0 + hx - 2, gy = y0 + hy - 2, gz = z0 + hz - 2;
            uint8_t a = 0, b = 0;
            if (gx >= 0 && gy >= 0 && gz >= 0 && gx < D.w && gy < D.h && gz < D.d) {
                const long long gi = (gz * whl) + gy * wl + gx;
                a = Js[gi];
                b = It[gi];
            }
            sm.J[hz][hy][hx] = a;
            sm.I[hz][hy][hx] = b;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < kHZ * kHY * kTX; k += blockDim.x) {
            const int xo = k % kTX, hy = (k / kTX) % kHY, hz = k / (kTX * kHY);
            int s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
#pragma unroll
            for (int dx = 0; dx < 5; ++dx) {
                const int a = sm.J[hz][hy][xo + dx], b = sm.I[hz][hy][xo + dx];
                s0 += a;
                s1 += b;
                s2 += a * a;
                s3 += b * b;
                s4 += a * b;
            }
            sm.p1[0][hz][hy][xo] = s0;
            sm.p1[1][hz][hy][xo] = s1;
            sm.p1[2][hz][hy][xo] = s2;
            sm.p1[3][hz][hy][xo] = s3;
            sm.p1[4][hz][hy][xo] = s4;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < kHZ * kTY * kTX; k += blockDim.x) {
            const int xo = k % kTX, yo = (k / kTX) % kTY, hz = k / (kTX * kTY);
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                int v = 0;
#pragma unroll
                for (int dy = 0; dy < 5; ++dy)
                    v += sm.p1[c][hz][yo + dy][xo];
                sm.p2[c][hz][yo][xo] = v;
            }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < kTZ * kTY * kTX; k += blockDim.x) {
            const int xo = k % kTX, yo = (k / kTX) % kTY, zo = k / (kTX * kTY);
            const int x = x0 + xo, y = y0 + yo, z = z0 + zo;
            if (x >= D.w || y >= D.h || z >= D.d)
                continue;
            const long long i = (z * whl) + y * wl + x;
            const int js = sm.J[zo + 2][yo + 2][xo + 2], it = sm.I[zo + 2][yo + 2][xo + 2];
            float3 out = make_float3(0.0f, 0.0f, 0.0f);
            float cost = 0.0f;
            if (!(js == 0 || it == 0)) {
                int t[5];
#pragma unroll
                for (int c = 0; c < 5; ++c) {
                    int v = 0;
#pragma unroll
                    for (int dz = 0; dz < 5; ++dz)
                        v += sm.p2[c][zo + dz][yo][xo];
                    t[c] = v;
                }
                const int m = (min(D.w - 1, x + 2) - max(0, x - 2) + 1) * (min(D.h - 1, y + 2) - max(0, y - 2) + 1) *
                              (min(D.d - 1, z + 2) - max(0, z - 2) + 1);
                Reg r;
                regress_finish((double)t[0], (double)t[1], (double)t[2], (double)t[3], (double)t[4], m, r);
                if (r.a > 0.0f) {
                    // gradient_at from the tile (neighbours are inside the halo)
                    float3 g;
                    g.x = (x + 1 < D.w && x) ? (float)((int)sm.J[zo + 2][yo + 2][xo + 3] - (int)sm.J[zo + 2][yo + 2][xo + 1]) : 0.0f;
                    g.y = (y + 1 < D.h && y) ? (float)((int)sm.J[zo + 2][yo + 3][xo + 2] - (int)sm.J[zo + 2][yo + 1][xo + 2]) : 0.0f;
                    g.z = (z + 1 < D.d && z) ? (float)((int)sm.J[zo + 3][yo + 2][xo + 2] - (int)sm.J[zo + 1][yo + 2][xo + 2]) : 0.0f;
                    const float sc = r.r2 * ((float)js * r.a + r.b - (float)it);
                    g.x *= sc;
                    g.y *= sc;
                    g.z *= sc;
                    out.x = 0.0f + g.x;
                    out.y = 0.0f + g.y;
                    out.z = 0.0f + g.z;
                    cost = -r.r2;
                }
            }
            store_term(nd, i, out, mod);
            csum += (double)cost;
        }
    }
    __shared__ double red[32];
    csum = block_sum(csum, red);
    if (threadIdx.x == 0)
        S.cost_part[blk] = csum;
    if (last_block_of_segment(S))
        control_block(S, mod);
}

// ------------------------------------------------------------------ control
// cdm_improved (reg/cdm.hpp:19-34): regression of the last costs on their index
// (int x, float y; statistics.hpp:694-713); a positive slope means "not improved".
__device__ bool cdm_improved_dev(CdmCtl* c)
{
    const int n = c->ncost;
    if (n > 5) {
        long long sx = 0, sxx = 0;
        double sy = (double)c->cost[0], syy = 0.0, sxy = (double)(0.0f * c->cost[0]);
        for (int i = 0; i < n; ++i) {
            sx += i;
            sxx += (long long)i * i;
        }
        for (int i = 1; i < n; ++i) {
            sy += (double)c->cost[i];
            sxy += (double)((float)i * c->cost[i]);
        }
        for (int i = 0; i < n; ++i) {
            const double t = c->cost[i];
            syy += t * t;
        }
        const double mx = (double)sx / n, my = sy / n;
        const double xv = (double)sxx / n - mx * mx, yv = syy / n - my * my;
        float a = 0.0f;
        if (!(xv == 0.0 || yv == 0.0))
            a = (float)((sxy / n - mx * my) / xv);
        if (a > 0.0f)
            return false;
        if (n > 7) {
            for (int i = 1; i < n; ++i)
                c->cost[i - 1] = c->cost[i];
            c->ncost = n - 1;
        }
    }
    return true;
}

// Mean of the per-block cost partials, summed in a fixed order.
__device__ float seg_cost_mean(const CdmSeg& S)
{
    __shared__ double red[32];
    double s = 0.0;
    for (int k = threadIdx.x; k < S.nblk; k += blockDim.x)
        s += S.cost_part[k];
    s = block_sum(s, red);
    __shared__ float out;
    if (threadIdx.x == 0)
        out = (float)(s / (double)((long long)S.w * S.h * S.d));
    __syncthreads();
    return out;
}

// The body of the reference's iteration loop between the gradient and the
// Poisson solve (reg/cdm.hpp:418-460), run by one block of the segment (the
// gradient kernel's last block).  Each modality's launch keeps its mean cost; the
// last modality's sums them in modality order (float), failing the level as soon
// as a partial sum is exactly zero, and records sum / nmod.
__device__ void control_block(const CdmSeg& S, int mod)
{
    CdmCtl* c = S.ctl;
    const float mean_cost = seg_cost_mean(S);
    if (threadIdx.x != 0)
        return;
    const int nm = S.nmod > 1 ? S.nmod : 1;
    c->mod_cost[mod] = mean_cost;
    if (mod + 1 < nm)
        return;
    c->save_best = 0;
    c->restore = 0;
    if (c->index >= c->max_iter) {
        c->done = 1;
        return;
    }
    float sum_cost = 0.0f;
    for (int k = 0; k < nm; ++k) {
        sum_cost += c->mod_cost[k];
        if (sum_cost == 0.0f) {
            c->last_cost = sum_cost;
            c->done = 2;
            return;
        }
    }
    c->last_cost = sum_cost;
    c->cost[c->ncost++] = sum_cost / (float)nm;
    const float cur = c->cost[c->ncost - 1];
    if (cur < c->best_cost) {
        c->best_cost = cur;
        if (c->index)
            c->save_best = 1;
    }
    if (!cdm_improved_dev(c)) {
        if (c->cur_smoothing <= c->smoothing) {
            c->done = 1;
            ++c->iters_run;
            return;
        }
        c->restore = 1;
        c->cur_smoothing *= 0.5f;
        c->ncost = 0;
    }
    ++c->index;
    ++c->iters_run;
}

// Completion ticket of a segment's blocks: true in the one block that finishes
// last (all other blocks' global writes are visible to it).
__device__ __forceinline__ bool last_block_of_segment(const CdmSeg& S)
{
    __shared__ unsigned int last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        last = (atomicAdd(&S.ctl->ticket, 1u) == (unsigned)S.nblk - 1u);
        if (last)
            S.ctl->ticket = 0u;
    }
    __syncthreads();
    if (last)
        __threadfence();
    return last;
}

// ------------------------------------------------------------------ Poisson
// cdm_solve_poisson (reg/cdm.hpp:158-253): s0 = new_d * (-1/6); then Jacobi sweeps
// s' = (new_d - s[-1] - s[+1] - s[-w] - s[+w] - s[-wh] - s[+wh]) * (-1/6) with the
// neighbours taken by flat index, bounds on the flat index only (2-D: -1/4 and no
// +-wh taps).
// mode 0: the first sweep, reading s0 = new_d * (-1/6) formed on the fly (the same
//         float product the reference stores), writing B; it also applies this
//         iteration's best_d save / restore (reg/cdm.hpp:447-457), which the
//         reference performs before its Poisson solve -- even on the iteration
//         that leaves the loop;
// mode 1: a middle sweep, parity picks A->B or B->A;
// mode 2: the last sweep (B->A) with the first-iteration max |result| (theta,
//         reg/cdm.hpp:463-467) formed from the values it writes.
__device__ __forceinline__ void poisson_point(const float* __restrict__ s, const float* __restrict__ rhs, long long p,
                                              long long n, long long w, long long wh, bool scale_s, float c6, float* v)
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float acc = rhs[3 * p + c];
        if (scale_s) {
            if (p >= 1) acc -= s[3 * (p - 1) + c] * c6;
            if (p < n - 1) acc -= s[3 * (p + 1) + c] * c6;
            if (p >= w) acc -= s[3 * (p - w) + c] * c6;
            if (p < n - w) acc -= s[3 * (p + w) + c] * c6;
            if (p >= wh) acc -= s[3 * (p - wh) + c] * c6;
            if (p < n - wh) acc -= s[3 * (p + wh) + c] * c6;
        } else {
            if (p >= 1) acc -= s[3 * (p - 1) + c];
            if (p < n - 1) acc -= s[3 * (p + 1) + c];
            if (p >= w) acc -= s[3 * (p - w) + c];
            if (p < n - w) acc -= s[3 * (p + w) + c];
            if (p >= wh) acc -= s[3 * (p - wh) + c];
            if (p < n - wh) acc -= s[3 * (p + wh) + c];
        }
        acc *= c6;
        v[c] = acc;
    }
}

// inv_d2 = -0.5 / dimension (reg/cdm.hpp:163,175): -1/6 in 3-D, -1/4 in 2-D.  A 2-D
// level's plane is the whole image (d == 1), so its +-wh taps fall outside the flat
// index range and drop out, as the reference's 2-D stencil has none.
__device__ __forceinline__ float poisson_weight(const CdmSeg& S)
{
    return S.ndim == 2 ? -0.5f / 2.0f : -0.5f / 3.0f;
}

template <bool MULTI>
__global__ void __launch_bounds__(kCdmThreads) cdm_poisson_kernel(const CdmSeg* __restrict__ segs, int nseg, int mode,
                                                                  int parity)
{
    SEG_BEGIN
    CdmCtl* c = S.ctl;
    if (mode == 0) {
        const float* src = nullptr;
        float* dst = nullptr;
        if (c->save_best) {
            src = S.cur_d;
            dst = S.best_d;
        } else if (c->restore) {
            src = S.best_d;
            dst = S.cur_d;
        }
        if (dst)
            for (long long i = first; i < 3 * n; i += stride)
                dst[i] = src[i];
    }
    if (c->done)
        return;
    const float* __restrict__ rhs = S.new_d;
    const float* __restrict__ in;
    float* __restrict__ out;
    if (mode == 0) {
        in = rhs;
        out = S.tmp_d;
    } else if (mode == 2) {
        in = S.tmp_d;
        out = S.aux_d;
    } else {
        in = parity ? S.tmp_d : S.aux_d;
        out = parity ? S.aux_d : S.tmp_d;
    }
    const long long w = D.w, wh = D.wh();
    if (mode != 2) {
        // one float of the interleaved xyz array per thread: the component's
        // neighbours at voxel offsets 1, w, wh are float offsets 3, 3w, 3wh, and
        // the reference's flat-index bounds p >= k / p < n - k are f >= 3k / f < 3(n - k)
        // -- every tap is a coalesced load, the arithmetic per component unchanged
        const float c6 = poisson_weight(S);
        const long long N3 = 3 * n, w3 = 3 * w, wh3 = 3 * wh;
        const bool sc = (mode == 0);
        for (long long f = first; f < N3; f += stride) {
            float acc = rhs[f];
            if (sc) {
                if (f >= 3) acc -= in[f - 3] * c6;
                if (f < N3 - 3) acc -= in[f + 3] * c6;
                if (f >= w3) acc -= in[f - w3] * c6;
                if (f < N3 - w3) acc -= in[f + w3] * c6;
                if (f >= wh3) acc -= in[f - wh3] * c6;
                if (f < N3 - wh3) acc -= in[f + wh3] * c6;
            } else {
                if (f >= 3) acc -= in[f - 3];
                if (f < N3 - 3) acc -= in[f + 3];
                if (f >= w3) acc -= in[f - w3];
                if (f < N3 - w3) acc -= in[f + w3];
                if (f >= wh3) acc -= in[f - wh3];
                if (f < N3 - wh3) acc -= in[f + wh3];
            }
            acc *= c6;
            out[f] = acc;
        }
        return;
    }
    const bool want_theta = (c->theta == 0.0f);
    float m = 0.0f;
    for (long long p = first; p < n; p += stride) {
        float v[3];
        poisson_point(in, rhs, p, n, w, wh, mode == 0, poisson_weight(S), v);
        out[3 * p] = v[0];
        out[3 * p + 1] = v[1];
        out[3 * p + 2] = v[2];
        if (want_theta) {
            // cdm_max_displacement_length: sqrt(double(x*x + y*y + z*z)) as float
            const float l2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            m = fmaxf(m, (float)sqrt((double)l2));
        }
    }
    if (!want_theta)
        return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(&c->theta_bits, __float_as_uint(m));
    if (!last_block_of_segment(S) || threadIdx.x != 0)
        return;
    const float theta = __uint_as_float(atomicAdd(&c->theta_bits, 0u));
    c->theta = theta;
    if (theta == 0.0f)
        c->done = 1;
    else
        c->scale = c->speed / theta;
}

// ------------------------------------------------------------------ theta
// cdm_max_displacement_length (reg/cdm.hpp:260-295), only while theta == 0 (the
// first iteration of a level); the last block sets theta and speed/theta, or
// leaves the loop when theta is 0 (reg/cdm.hpp:463-467).
template <bool MULTI>
__global__ void __launch_bounds__(kCdmThreads) cdm_theta_kernel(const CdmSeg* __restrict__ segs, int nseg)
{
    SEG_BEGIN
    CdmCtl* c = S.ctl;
    if (c->done || c->theta != 0.0f)
        return;
    const float* __restrict__ d = S.aux_d;
    float m = 0.0f;
    for (long long i = first; i < n; i += stride) {
        const float x = d[3 * i], y = d[3 * i + 1], z = d[3 * i + 2];
        const float l2 = x * x + y * y + z * z;
        const float l = (float)sqrt((double)l2);
        m = fmaxf(m, l);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(&c->theta_bits, __float_as_uint(m));
    if (!last_block_of_segment(S) || threadIdx.x != 0)
        return;
    const float theta = __uint_as_float(atomicAdd(&c->theta_bits, 0u));
    c->theta = theta;
    if (theta == 0.0f)
        c->done = 1;
    else
        c->scale = c->speed / theta;
}

// ------------------------------------------------------------------ accumulate
// new_d *= speed/theta (reg/cdm.hpp:467) fused with accumulate_displacement
// (numerical/dif.hpp:166-186): out = (cur_d + id)(x + new_d) - x where new_d is
// non-zero and the sample lands inside, else cur_d.  The mapping cur_d + id is
// formed per corner exactly as displacement_to_mapping stores it.
template <bool MULTI>
__global__ void __launch_bounds__(kCdmThreads) cdm_accumulate_kernel(const CdmSeg* __restrict__ segs, int nseg)
{
    SEG_BEGIN
    const CdmCtl* c = S.ctl;
    if (c->done)
        return;
    const float scale = c->scale;
    const float* __restrict__ nd = S.aux_d;
    const float* __restrict__ cd = S.cur_d;
    float* __restrict__ out = S.tmp_d;
    const int w = D.w, wh = D.wh();
    if (S.ndim == 2) {
        // the 2-D form: bilinear sample of the mapping cur_d + (x, y); z stays 0
        for (long long i = first; i < n; i += stride) {
            float dx = nd[3 * i] * scale, dy = nd[3 * i + 1] * scale;
            const int x = (int)(i % w), y = (int)(i / w);
            bool ok = false;
            if (dx != 0.0f || dy != 0.0f) {
                dx += (float)x;
                dy += (float)y;
                Cell2 cl;
                if (bilinear_cell(D, dx, dy, cl)) {
                    const int b = cl.base, bx = b % w, by = b / w;
                    const int off[4] = {0, 1, w, w + 1};
                    const int ox[4] = {0, 1, 0, 1};
                    const int oy[4] = {0, 0, 1, 1};
                    float ax = 0.f, ay = 0.f;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const float* q = cd + 3LL * (b + off[k]);
                        const float mx = q[0] + (float)(bx + ox[k]);
                        const float my = q[1] + (float)(by + oy[k]);
                        if (k == 0) {
                            ax = mx * cl.r[0];
                            ay = my * cl.r[0];
                        } else {
                            ax += mx * cl.r[k];
                            ay += my * cl.r[k];
                        }
                    }
                    out[3 * i] = ax - (float)x;
                    out[3 * i + 1] = ay - (float)y;
                    ok = true;
                }
            }
            if (!ok) {
                out[3 * i] = cd[3 * i];
                out[3 * i + 1] = cd[3 * i + 1];
            }
            out[3 * i + 2] = 0.0f;
        }
        return;
    }
    for (long long i = first; i < n; i += stride) {
        float dx = nd[3 * i] * scale, dy = nd[3 * i + 1] * scale, dz = nd[3 * i + 2] * scale;
        int x, y, z;
        unflat((int)i, D, x, y, z);
        bool ok = false;
        if (dx != 0.0f || dy != 0.0f || dz != 0.0f) {
            dx += (float)x;
            dy += (float)y;
            dz += (float)z;
            Cell cl;
            if (trilinear_cell(D, dx, dy, dz, cl)) {
                const int b = cl.base;
                const int bx = b % w, by = (b / w) % D.h, bz = b / wh;
                const int off[8] = {0, 1, w, w + 1, wh, wh + 1, wh + w, wh + w + 1};
                const int ox[8] = {0, 1, 0, 1, 0, 1, 0, 1};
                const int oy[8] = {0, 0, 1, 1, 0, 0, 1, 1};
                const int oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float* q = cd + 3LL * (b + off[k]);
                    const float mx = q[0] + (float)(bx + ox[k]);
                    const float my = q[1] + (float)(by + oy[k]);
                    const float mz = q[2] + (float)(bz + oz[k]);
                    if (k == 0) {
                        ax = mx * cl.r[0];
                        ay = my * cl.r[0];
                        az = mz * cl.r[0];
                    } else {
                        ax += mx * cl.r[k];
                        ay += my * cl.r[k];
                        az += mz * cl.r[k];
                    }
                }
                out[3 * i] = ax - (float)x;
                out[3 * i + 1] = ay - (float)y;
                out[3 * i + 2] = az - (float)z;
                ok = true;
            }
        }
        if (!ok) {
            out[3 * i] = cd[3 * i];
            out[3 * i + 1] = cd[3 * i + 1];
            out[3 * i + 2] = cd[3 * i + 2];
        }
    }
}

// ------------------------------------------------------------------ smooth
// cdm_smooth (reg/cdm.hpp:302-366): cur_d = d*(1-s) + (s/6) * (d[+1] + d[-1] +
// d[+w] + d[-w] + d[+wh] + d[-wh]) by flat index; s == 0 leaves cur_d as it is.
// 2-D: s/4 and four neighbours (the +-wh taps of a d == 1 level fall outside).
template <bool MULTI>
__global__ void __launch_bounds__(kCdmThreads) cdm_smooth_kernel(const CdmSeg* __restrict__ segs, int nseg)
{
    SEG_BEGIN
    const CdmCtl* c = S.ctl;
    if (c->done)
        return;
    const float sm = c->cur_smoothing;
    if (sm == 0.0f)
        return;
    const float w_6 = sm / (2.0f * (S.ndim == 2 ? 2.0f : 3.0f));  // smoothing / (2 * dimension)
    const float w_1 = 1.0f - sm;
    const float* __restrict__ d = S.tmp_d;
    float* __restrict__ dd = S.cur_d;
    // one float of the interleaved array per thread (see the Poisson sweep)
    const long long N3 = 3 * n, w3 = 3 * (long long)D.w, wh3 = 3 * (long long)D.wh();
    for (long long f = first; f < N3; f += stride) {
        float v = 0.0f;
        if (f + 3 < N3) v += d[f + 3];
        if (f >= 3) v += d[f - 3];
        if (f + w3 < N3) v += d[f + w3];
        if (f >= w3) v += d[f - w3];
        if (f + wh3 < N3) v += d[f + wh3];
        if (f >= wh3) v += d[f - wh3];
        v *= w_6;
        dd[f] = d[f] * w_1 + v;
    }
}

// ------------------------------------------------------------------ pyramid
// downsample_with_padding (numerical/resampling.hpp:575-603): 2x box mean; a
// missing +1 neighbour repeats the nearest present one; integer pixels sum in
// 16 bits and shift by 3, float pixels divide by 8.
template <typename T>
__global__ void downsample_kernel(const T* __restrict__ in, Dim3 di, T* __restrict__ out, Dim3 dout)
{
    const long long n = dout.n();
    const long long w = di.w, wh = (long long)di.wh();
    const long long shift[8] = {0, 1, w, 1 + w, wh, wh + 1, wh + w, wh + 1 + w};
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        unflat((int)o, dout, x, y, z);
        const int x2 = 2 * x, y2 = 2 * y, z2 = 2 * z;
        int has = 0;
        if (x2 + 1 < di.w) has += 1;
        if (y2 + 1 < di.h) has += 2;
        if (z2 + 1 < di.d) has += 4;
        const long long base = ((long long)z2 * di.h + y2) * di.w + x2;
        T buf[8];
        buf[0] = in[base];
        if constexpr (sizeof(T) == 1) {
            unsigned int acc = buf[0];
#pragma unroll
            for (int k = 1; k < 8; ++k) {
                const int h = has & k;
                buf[k] = (h == k) ? in[base + shift[k]] : buf[h];
                acc = (acc + buf[k]) & 0xffffu;
            }
            out[o] = (T)(acc >> 3);
        } else {
            T acc = buf[0];
#pragma unroll
            for (int k = 1; k < 8; ++k) {
                const int h = has & k;
                buf[k] = (h == k) ? in[base + shift[k]] : buf[h];
                acc += buf[k];
            }
            out[o] = acc / 8;
        }
    }
}

cudaError_t launch_downsample(const void* in, void* out, int w, int h, int d, int pix, cudaStream_t st)
{
    Dim3 di{w, h, d}, dout{(w + 1) / 2, (h + 1) / 2, (d + 1) / 2};
    int blocks = cdm_blocks_for(dout.n());
    if (pix == 0)
        downsample_kernel<uint8_t><<<blocks, kCdmThreads, 0, st>>>((const uint8_t*)in, di, (uint8_t*)out, dout);
    else
        downsample_kernel<float><<<blocks, kCdmThreads, 0, st>>>((const float*)in, di, (float*)out, dout);
    count_launch();
    return cudaGetLastError();
}

// best_d *= 2; upsample_with_padding (reg/cdm.hpp:402-403,
// numerical/resampling.hpp:849-891): out(x) = trilinear(2*in, x * 0.5), 0 where the
// sample fails.  The doubling is exact, so it is applied to the corner values.
__global__ void upsample_x2_kernel(const float* __restrict__ in, Dim3 di, float* __restrict__ out, Dim3 dout)
{
    const long long n = dout.n();
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        unflat((int)o, dout, x, y, z);
        float vx = (float)x, vy = (float)y, vz = (float)z;
        vx *= 0.5f;
        vy *= 0.5f;
        vz *= 0.5f;
        Cell c;
        float3 v = make_float3(0.f, 0.f, 0.f);
        if (trilinear_cell(di, vx, vy, vz, c)) {
            const int w = di.w, wh = di.wh(), b = c.base;
            const int off[8] = {0, 1, w, w + 1, wh, wh + 1, wh + w, wh + w + 1};
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float* q = in + 3LL * (b + off[k]);
                const float qx = q[0] * 2.0f, qy = q[1] * 2.0f, qz = q[2] * 2.0f;
                if (k == 0) {
                    v.x = qx * c.r[0];
                    v.y = qy * c.r[0];
                    v.z = qz * c.r[0];
                } else {
                    v.x += qx * c.r[k];
                    v.y += qy * c.r[k];
                    v.z += qz * c.r[k];
                }
            }
        }
        out[3 * o] = v.x;
        out[3 * o + 1] = v.y;
        out[3 * o + 2] = v.z;
    }
}

// The 2-D form (vector<2> field of a d == 1 level): bilinear at (x, y) * 0.5; z is 0.
__global__ void upsample_x2_2d_kernel(const float* __restrict__ in, Dim3 di, float* __restrict__ out, Dim3 dout)
{
    const long long n = dout.n();
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(o % dout.w), y = (int)(o / dout.w);
        float vx = (float)x, vy = (float)y;
        vx *= 0.5f;
        vy *= 0.5f;
        Cell2 c;
        float2 v = make_float2(0.f, 0.f);
        if (bilinear_cell(di, vx, vy, c)) {
            const int w = di.w, b = c.base;
            const int off[4] = {0, 1, w, w + 1};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float* q = in + 3LL * (b + off[k]);
                const float qx = q[0] * 2.0f, qy = q[1] * 2.0f;
                if (k == 0) {
                    v.x = qx * c.r[0];
                    v.y = qy * c.r[0];
                } else {
                    v.x += qx * c.r[k];
                    v.y += qy * c.r[k];
                }
            }
        }
        out[3 * o] = v.x;
        out[3 * o + 1] = v.y;
        out[3 * o + 2] = 0.0f;
    }
}

cudaError_t launch_upsample_field_x2(const float* in, int iw, int ih, int id, float* out, int ow, int oh, int od,
                                     cudaStream_t st, int ndim)
{
    Dim3 di{iw, ih, id}, dout{ow, oh, od};
    if (ndim == 2)
        upsample_x2_2d_kernel<<<cdm_blocks_for(dout.n()), kCdmThreads, 0, st>>>(in, di, out, dout);
    else
        upsample_x2_kernel<<<cdm_blocks_for(dout.n()), kCdmThreads, 0, st>>>(in, di, out, dout);
    count_launch();
    return cudaGetLastError();
}

__global__ void field_xy_kernel(const float* __restrict__ xyz, long long n, float* __restrict__ xy)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        xy[2 * i] = xyz[3 * i];
        xy[2 * i + 1] = xyz[3 * i + 1];
    }
}

cudaError_t launch_field_xy(const float* xyz, long long n, float* xy, cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    field_xy_kernel<<<cdm_blocks_for(n), kCdmThreads, 0, st>>>(xyz, n, xy);
    count_launch();
    return cudaGetLastError();
}

__global__ void cost_mean_kernel(const CdmSeg* __restrict__ segs, float* __restrict__ out)
{
    const float m = seg_cost_mean(segs[blockIdx.y]);
    if (threadIdx.x == 0)
        out[blockIdx.y] = m;
}

cudaError_t launch_cost_mean(const CdmSeg* segs, int nseg, float* out, cudaStream_t st)
{
    cost_mean_kernel<<<dim3(1, nseg), 256, 0, st>>>(segs, out);
    count_launch();
    return cudaGetLastError();
}

// done flags of many segments gathered into one array (one read-back per round)
__global__ void cdm_status_kernel(const CdmSeg* __restrict__ segs, int n, int* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = segs[i].ctl->done;
}

cudaError_t launch_cdm_status(const CdmSeg* segs, int nseg, int* out, cudaStream_t st)
{
    if (nseg <= 0)
        return cudaSuccess;
    cdm_status_kernel<<<(nseg + 127) / 128, 128, 0, st>>>(segs, nseg, out);
    count_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------------------ launchers
// blocks: the launch's blocks, sum(nblk) over its nseg segment entries (their blk0 set
// accordingly); one entry alone: its nblk.
#define SEG_GRID dim3(blocks)
#define SEG_LAUNCH(multi, single, threads, smem, ...)                                  \
    do {                                                                               \
        if (nseg > 1)                                                                  \
            multi<<<SEG_GRID, threads, smem, st>>>(segs, nseg, ##__VA_ARGS__);         \
        else                                                                           \
            single<<<SEG_GRID, threads, smem, st>>>(segs, nseg, ##__VA_ARGS__);        \
    } while (0)

cudaError_t launch_cdm_compose(const CdmSeg* segs, int nseg, int blocks, int pix, cudaStream_t st, int mod)
{
    if (mod < 0 || mod >= kCdmMaxModalities)
        return cudaErrorInvalidValue;
    if (pix == 0)
        SEG_LAUNCH((cdm_compose_kernel<uint8_t, true>), (cdm_compose_kernel<uint8_t, false>), kCdmThreads, 0, mod);
    else
        SEG_LAUNCH((cdm_compose_kernel<float, true>), (cdm_compose_kernel<float, false>), kCdmThreads, 0, mod);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_cdm_gradient(const CdmSeg* segs, int nseg, int blocks, int pix, int gradient_type,
                                cudaStream_t st, int mod)
{
    if (mod < 0 || mod >= kCdmMaxModalities)
        return cudaErrorInvalidValue;
    if (pix == 0 && gradient_type == 'r') {
        static std::atomic<unsigned long long> attr_set{0};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess)
            return e;
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(attr_set.load() & bit)) {
            e = cudaFuncSetAttribute(cdm_gradient_box_u8_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(BoxSmem));
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(cdm_gradient_box_u8_kernel<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BoxSmem));
            if (e != cudaSuccess)
                return e;
            attr_set.fetch_or(bit);
        }
        SEG_LAUNCH(cdm_gradient_box_u8_kernel<true>, cdm_gradient_box_u8_kernel<false>, kBoxThreads,
                   sizeof(BoxSmem), mod);
    } else if (pix == 0)
        SEG_LAUNCH((cdm_gradient_kernel<uint8_t, true>), (cdm_gradient_kernel<uint8_t, false>), kCdmThreads, 0,
                   gradient_type, mod);
    else
        SEG_LAUNCH((cdm_gradient_kernel<float, true>), (cdm_gradient_kernel<float, false>), kCdmThreads, 0,
                   gradient_type, mod);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_cdm_poisson(const CdmSeg* segs, int nseg, int blocks, int sweeps, cudaStream_t st)
{
    // sweeps is 12 (reg/cdm.hpp:165): first (B), 10 middle (B->A, A->B, ...), last (B->A)
    SEG_LAUNCH(cdm_poisson_kernel<true>, cdm_poisson_kernel<false>, kCdmThreads, 0, 0, 0);
    for (int k = 1; k < sweeps - 1; ++k)
        SEG_LAUNCH(cdm_poisson_kernel<true>, cdm_poisson_kernel<false>, kCdmThreads, 0, 1, k & 1);
    SEG_LAUNCH(cdm_poisson_kernel<true>, cdm_poisson_kernel<false>, kCdmThreads, 0, 2, 1);
    count_launch(sweeps);
    return cudaGetLastError();
}

cudaError_t launch_cdm_theta(const CdmSeg* segs, int nseg, int blocks, cudaStream_t st)
{
    SEG_LAUNCH(cdm_theta_kernel<true>, cdm_theta_kernel<false>, kCdmThreads, 0);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_cdm_accumulate(const CdmSeg* segs, int nseg, int blocks, cudaStream_t st)
{
    SEG_LAUNCH(cdm_accumulate_kernel<true>, cdm_accumulate_kernel<false>, kCdmThreads, 0);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_cdm_smooth(const CdmSeg* segs, int nseg, int blocks, cudaStream_t st)
{
    SEG_LAUNCH(cdm_smooth_kernel<true>, cdm_smooth_kernel<false>, kCdmThreads, 0);
    count_launch();
    return cudaGetLastError();
}

}  // namespace regb
