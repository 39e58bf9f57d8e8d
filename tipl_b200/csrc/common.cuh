// Shared device helpers for the registration kernels.
//
// Arithmetic rule: every kernel file is compiled with -fmad=false and the float
// expressions below are written in the reference's evaluation order, so products
// and sums round exactly as the reference's CPU build (-ffp-contract=off) does.
// That is what makes uint8 outputs and histogram counts bit-identical.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "kernels.h"

namespace regb {

// p' = sr * p + shift with the reference's left-to-right sums
// (numerical/transformation.hpp:58-73): ((x*r0 + y*r1) + z*r2) + s0.
struct Xform {
    float m[12];  // sr[9] row-major, shift[3]
};

__device__ __forceinline__ void apply_xform(const float* __restrict__ T, float x, float y, float z, float& ox,
                                            float& oy, float& oz)
{
    ox = x * T[0] + y * T[1] + z * T[2] + T[9];
    oy = x * T[3] + y * T[4] + z * T[5] + T[10];
    oz = x * T[6] + y * T[7] + z * T[8] + T[11];
}

// Cell test of interpolator::linear<3>::get_location
// (numerical/interpolation.hpp:337-350): reject negative coordinates and any
// cell whose +1 neighbour leaves the volume.  For x >= 0, trunc(x)+1 >= w is the
// same as x >= w-1, and w-1 is exact in float for every accepted extent.
struct Cell {
    int base;      // flat index of the (ix, iy, iz) corner
    float r[8];    // weights in the reference's order
};

__device__ __forceinline__ bool trilinear_cell(const Dim3& D, float x, float y, float z, Cell& c)
{
    if (x < 0.0f || y < 0.0f || z < 0.0f)
        return false;
    if (!(x < (float)(D.w - 1)) || !(y < (float)(D.h - 1)) || !(z < (float)(D.d - 1)))
        return false;
    int ix = (int)x, iy = (int)y, iz = (int)z;
    float p0 = x - (float)ix, p1 = y - (float)iy, p2 = z - (float)iz;
    float n0 = 1.0f - p0, n1 = 1.0f - p1, n2 = 1.0f - p2;
    float n0n1 = n0 * n1, p0n1 = p0 * n1, n0p1 = n0 * p1, p0p1 = p0 * p1;
    c.r[0] = n0n1 * n2;
    c.r[1] = p0n1 * n2;
    c.r[2] = n0p1 * n2;
    c.r[3] = p0p1 * n2;
    c.r[4] = n0n1 * p2;
    c.r[5] = p0n1 * p2;
    c.r[6] = n0p1 * p2;
    c.r[7] = p0p1 * p2;
    c.base = (iz * D.h + iy) * D.w + ix;
    return true;
}

// Cell test and weights of interpolator::linear<2>::get_location
// (numerical/interpolation.hpp:274-305): reject negative coordinates and cells
// whose +1 neighbour leaves the image; weights n0*n1, p0*n1, n0*p1, p0*p1.
struct Cell2 {
    int base;
    float r[4];
};

__device__ __forceinline__ bool bilinear_cell(const Dim3& D, float x, float y, Cell2& c)
{
    if (x < 0.0f || y < 0.0f)
        return false;
    if (!(x < (float)(D.w - 1)) || !(y < (float)(D.h - 1)))
        return false;
    const int ix = (int)x, iy = (int)y;
    const float p0 = x - (float)ix, p1 = y - (float)iy;
    const float n0 = 1.0f - p0, n1 = 1.0f - p1;
    c.r[0] = n0 * n1;
    c.r[1] = p0 * n1;
    c.r[2] = n0 * p1;
    c.r[3] = p0 * p1;
    c.base = iy * D.w + ix;
    return true;
}

template <typename T>
__device__ __forceinline__ float ld_pix(const T* __restrict__ p, int i)
{
    return (float)__ldg(p + i);
}

// weighted_sum (numerical/interpolation.hpp:61-73): r = I0*w0; r += I1*w1; ...
template <typename T>
__device__ __forceinline__ float cell_sum(const T* __restrict__ I, const Dim3& D, const Cell& c)
{
    const int w = D.w, wh = D.wh(), b = c.base;
    float acc = ld_pix(I, b) * c.r[0];
    acc += ld_pix(I, b + 1) * c.r[1];
    acc += ld_pix(I, b + w) * c.r[2];
    acc += ld_pix(I, b + w + 1) * c.r[3];
    acc += ld_pix(I, b + wh) * c.r[4];
    acc += ld_pix(I, b + wh + 1) * c.r[5];
    acc += ld_pix(I, b + wh + w) * c.r[6];
    acc += ld_pix(I, b + wh + w + 1) * c.r[7];
    return acc;
}

// weighted_sum over the 2-D cell (numerical/interpolation.hpp:61-73).
template <typename T>
__device__ __forceinline__ float cell_sum2(const T* __restrict__ I, const Dim3& D, const Cell2& c)
{
    const int w = D.w, b = c.base;
    float acc = ld_pix(I, b) * c.r[0];
    acc += ld_pix(I, b + 1) * c.r[1];
    acc += ld_pix(I, b + w) * c.r[2];
    acc += ld_pix(I, b + w + 1) * c.r[3];
    return acc;
}

// interp_type<T>::assign (numerical/interpolation.hpp:28-34).
template <typename T>
__device__ __forceinline__ T assign_pix(float v);
template <>
__device__ __forceinline__ uint8_t assign_pix<uint8_t>(float v)
{
    return v <= 0.0f ? (uint8_t)0 : (uint8_t)v;
}
template <>
__device__ __forceinline__ float assign_pix<float>(float v)
{
    return v;
}

// Vector-field cell sum: each component accumulated as the scalar case.
__device__ __forceinline__ float3 cell_sum_vec(const float* __restrict__ F, const Dim3& D, const Cell& c)
{
    const int w = D.w, wh = D.wh(), b = c.base;
    const int off[8] = {0, 1, w, w + 1, wh, wh + 1, wh + w, wh + w + 1};
    const float* p = F + 3LL * b;
    float3 acc;
    acc.x = __ldg(p) * c.r[0];
    acc.y = __ldg(p + 1) * c.r[0];
    acc.z = __ldg(p + 2) * c.r[0];
#pragma unroll
    for (int k = 1; k < 8; ++k) {
        const float* q = F + 3LL * (b + off[k]);
        acc.x += __ldg(q) * c.r[k];
        acc.y += __ldg(q + 1) * c.r[k];
        acc.z += __ldg(q + 2) * c.r[k];
    }
    return acc;
}

// ---- exact conversions on the FP/ALU pipes (the conversion unit is the
// bottleneck of the sampling loops otherwise) ----
constexpr float kTwo23 = 8388608.0f;

// float(v) for 0 <= v < 2^23: the bits of 2^23 + v, minus 2^23 (both steps exact).
__device__ __forceinline__ float u8_to_f(uint32_t v) { return __uint_as_float(0x4B000000u | v) - kTwo23; }

// floor(x) for 0 <= x < 2^23: x + 2^23 rounded toward zero is 2^23 + floor(x);
// returns floor(x) as float and sets i to it as an integer.
__device__ __forceinline__ float floor_pos(float x, int& i)
{
    const float r = __fadd_rz(x, kTwo23);
    i = __float_as_int(r) - 0x4B000000;
    return r - kTwo23;
}

// Extent of a sampled volume with the float upper limits of the cell test.
struct SampleGeo {
    int w, h, wh;
    float wl, hl, dl;  // w-1, h-1, d-1
};
__device__ __forceinline__ SampleGeo sample_geo(const Dim3& D)
{
    return SampleGeo{D.w, D.h, D.w * D.h, (float)(D.w - 1), (float)(D.h - 1), (float)(D.d - 1)};
}

// The reference's uint8 trilinear estimate (interpolation.hpp:337-383 with the
// uint8 assign of 28-34) at (x, y, z); 0 where the cell test fails.  Same values as
// trilinear_cell + cell_sum + assign_pix<uint8_t>, with every float<->int
// conversion done by the exact tricks above.
__device__ __forceinline__ uint32_t sample_u8(const uint8_t* __restrict__ I, const SampleGeo& g, float x, float y,
                                              float z)
{
    if (x < 0.0f || y < 0.0f || z < 0.0f)
        return 0u;
    if (!(x < g.wl) || !(y < g.hl) || !(z < g.dl))
        return 0u;
    int ix, iy, iz;
    const float fx = floor_pos(x, ix), fy = floor_pos(y, iy), fz = floor_pos(z, iz);
    const float p0 = x - fx, p1 = y - fy, p2 = z - fz;
    const float n0 = 1.0f - p0, n1 = 1.0f - p1, n2 = 1.0f - p2;
    const float n0n1 = n0 * n1, p0n1 = p0 * n1, n0p1 = n0 * p1, p0p1 = p0 * p1;
    const uint8_t* q = I + ((iz * g.h + iy) * g.w + ix);
    const int w = g.w, wh = g.wh;
    float acc = u8_to_f(__ldg(q)) * (n0n1 * n2);
    acc += u8_to_f(__ldg(q + 1)) * (p0n1 * n2);
    acc += u8_to_f(__ldg(q + w)) * (n0p1 * n2);
    acc += u8_to_f(__ldg(q + w + 1)) * (p0p1 * n2);
    acc += u8_to_f(__ldg(q + wh)) * (n0n1 * p2);
    acc += u8_to_f(__ldg(q + wh + 1)) * (p0n1 * p2);
    acc += u8_to_f(__ldg(q + wh + w)) * (n0p1 * p2);
    acc += u8_to_f(__ldg(q + wh + w + 1)) * (p0p1 * p2);
    if (acc <= 0.0f)
        return 0u;
    return (uint32_t)(__float_as_int(__fadd_rz(acc, kTwo23)) - 0x4B000000);  // trunc of acc in (0, 256)
}

// The same estimate split in two halves so a thread can keep several samples'
// loads in flight: prepare() runs the cell test and forms the weights' factors,
// load() issues the eight corner loads, finish() sums them and truncates.
struct U8Sample {
    const uint8_t* q;
    float p0, p1, p2, n0, n1, n2;
    uint32_t v[8];
    bool ok;
    __device__ __forceinline__ void prepare(const uint8_t* __restrict__ I, const SampleGeo& g, float x, float y,
                                            float z)
    {
        ok = !(x < 0.0f || y < 0.0f || z < 0.0f) && (x < g.wl) && (y < g.hl) && (z < g.dl);
        if (!ok)
            return;
        int ix, iy, iz;
        const float fx = floor_pos(x, ix), fy = floor_pos(y, iy), fz = floor_pos(z, iz);
        p0 = x - fx;
        p1 = y - fy;
        p2 = z - fz;
        n0 = 1.0f - p0;
        n1 = 1.0f - p1;
        n2 = 1.0f - p2;
        q = I + ((iz * g.h + iy) * g.w + ix);
    }
    __device__ __forceinline__ void load(const SampleGeo& g)
    {
        if (!ok)
            return;
        const int w = g.w, wh = g.wh;
        v[0] = __ldg(q);
        v[1] = __ldg(q + 1);
        v[2] = __ldg(q + w);
        v[3] = __ldg(q + w + 1);
        v[4] = __ldg(q + wh);
        v[5] = __ldg(q + wh + 1);
        v[6] = __ldg(q + wh + w);
        v[7] = __ldg(q + wh + w + 1);
    }
    __device__ __forceinline__ uint32_t finish() const
    {
        if (!ok)
            return 0u;
        const float n0n1 = n0 * n1, p0n1 = p0 * n1, n0p1 = n0 * p1, p0p1 = p0 * p1;
        float acc = u8_to_f(v[0]) * (n0n1 * n2);
        acc += u8_to_f(v[1]) * (p0n1 * n2);
        acc += u8_to_f(v[2]) * (n0p1 * n2);
        acc += u8_to_f(v[3]) * (p0p1 * n2);
        acc += u8_to_f(v[4]) * (n0n1 * p2);
        acc += u8_to_f(v[5]) * (p0n1 * p2);
        acc += u8_to_f(v[6]) * (n0p1 * p2);
        acc += u8_to_f(v[7]) * (p0p1 * p2);
        if (acc <= 0.0f)
            return 0u;
        return (uint32_t)(__float_as_int(__fadd_rz(acc, kTwo23)) - 0x4B000000);
    }
};

// ---- packed pairs: sm_100 executes two FP32 adds/multiplies as one instruction,
// each lane rounded exactly like the scalar IEEE operation, so two voxels can
// share arithmetic instructions without changing a bit of either result.
// One rule keeps that true: a packed product must never feed a packed add or
// subtract, because the assembler contracts that pair into a fused multiply-add
// (explicit .rn does not stop it for the packed forms).  Products that feed sums
// are formed with the scalar __fmul_rn, which is never contracted. ----
#define REGB_F32X2_OP(name, op)                                                                  \
    __device__ __forceinline__ float2 name(float2 a, float2 b)                                  \
    {                                                                                            \
        float2 r;                                                                                \
        asm("{\n\t.reg .b64 ra, rb, rd;\n\t"                                                   \
            "mov.b64 ra, {%2, %3};\n\t"                                                          \
            "mov.b64 rb, {%4, %5};\n\t" op " rd, ra, rb;\n\t"                                  \
            "mov.b64 {%0, %1}, rd;\n\t}"                                                         \
            : "=f"(r.x), "=f"(r.y)                                                               \
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                           \
        return r;                                                                                \
    }
REGB_F32X2_OP(add2, "add.rn.f32x2")
REGB_F32X2_OP(sub2, "sub.rn.f32x2")
REGB_F32X2_OP(mul2, "mul.rn.f32x2")
REGB_F32X2_OP(addrz2, "add.rz.f32x2")
#undef REGB_F32X2_OP
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }

// Two uint8 trilinear estimates (the reference's interpolation of sample_u8) at
// (px.x, py.x, pz.x) and (px.y, py.y, pz.y), sharing every FP instruction.
// enA/enB disable a lane; a disabled or rejected lane returns 0 and loads
// nothing outside the volume.
__device__ __forceinline__ void sample_u8_pair(const uint8_t* __restrict__ I, const SampleGeo& g, float2 px,
                                               float2 py, float2 pz, bool enA, bool enB, uint32_t& oA,
                                               uint32_t& oB)
{
    const bool okA = enA && !(px.x < 0.0f || py.x < 0.0f || pz.x < 0.0f) && (px.x < g.wl) && (py.x < g.hl) &&
                     (pz.x < g.dl);
    const bool okB = enB && !(px.y < 0.0f || py.y < 0.0f || pz.y < 0.0f) && (px.y < g.wl) && (py.y < g.hl) &&
                     (pz.y < g.dl);
    const float2 t23 = bc2(kTwo23);
    // 2^23 + floor, per lane with the scalar round-toward-zero add
    const float2 rx = make_float2(__fadd_rz(px.x, kTwo23), __fadd_rz(px.y, kTwo23));
    const float2 ry = make_float2(__fadd_rz(py.x, kTwo23), __fadd_rz(py.y, kTwo23));
    const float2 rz = make_float2(__fadd_rz(pz.x, kTwo23), __fadd_rz(pz.y, kTwo23));
    const float2 fx = sub2(rx, t23), fy = sub2(ry, t23), fz = sub2(rz, t23);
    const float2 p0 = sub2(px, fx), p1 = sub2(py, fy), p2 = sub2(pz, fz);
    const float2 one = bc2(1.0f);
    const float2 n0 = sub2(one, p0), n1 = sub2(one, p1), n2 = sub2(one, p2);
    const float2 n0n1 = mul2(n0, n1), p0n1 = mul2(p0, n1), n0p1 = mul2(n0, p1), p0p1 = mul2(p0, p1);
    const int w = g.w, wh = g.wh;
    const uint8_t* qa = okA ? I + (((__float_as_int(rz.x) - 0x4B000000) * g.h + (__float_as_int(ry.x) - 0x4B000000)) *
                                       w + (__float_as_int(rx.x) - 0x4B000000))
                            : I;
    const uint8_t* qb = okB ? I + (((__float_as_int(rz.y) - 0x4B000000) * g.h + (__float_as_int(ry.y) - 0x4B000000)) *
                                       w + (__float_as_int(rx.y) - 0x4B000000))
                            : I;
    uint32_t a[8], b[8];
    a[0] = __ldg(qa);
    b[0] = __ldg(qb);
    a[1] = __ldg(qa + 1);
    b[1] = __ldg(qb + 1);
    a[2] = __ldg(qa + w);
    b[2] = __ldg(qb + w);
    a[3] = __ldg(qa + w + 1);
    b[3] = __ldg(qb + w + 1);
    a[4] = __ldg(qa + wh);
    b[4] = __ldg(qb + wh);
    a[5] = __ldg(qa + wh + 1);
    b[5] = __ldg(qb + wh + 1);
    a[6] = __ldg(qa + wh + w);
    b[6] = __ldg(qb + wh + w);
    a[7] = __ldg(qa + wh + w + 1);
    b[7] = __ldg(qb + wh + w + 1);
    const float2 wt[8] = {mul2(n0n1, n2), mul2(p0n1, n2), mul2(n0p1, n2), mul2(p0p1, n2),
                          mul2(n0n1, p2), mul2(p0n1, p2), mul2(n0p1, p2), mul2(p0p1, p2)};
    float2 acc;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float2 v = sub2(make_float2(__uint_as_float(0x4B000000u | a[k]), __uint_as_float(0x4B000000u | b[k])),
                              t23);
        const float2 m = make_float2(__fmul_rn(v.x, wt[k].x), __fmul_rn(v.y, wt[k].y));  // feeds a sum: scalar
        acc = (k == 0) ? m : add2(acc, m);
    }
    const float2 tr = make_float2(__fadd_rz(acc.x, kTwo23), __fadd_rz(acc.y, kTwo23));
    oA = (okA && acc.x > 0.0f) ? (uint32_t)(__float_as_int(tr.x) - 0x4B000000) : 0u;
    oB = (okB && acc.y > 0.0f) ? (uint32_t)(__float_as_int(tr.y) - 0x4B000000) : 0u;
}

// sample_u8_pair with the cell's corners read by 2-D texture gathers instead of
// eight byte loads.  The volume is held as a (w, h*d) texture of halves (exact for
// 0..255, returned as float by the texture unit): slice z, row y is texture row
// z*h + y.  With unnormalised coordinates, a gather at (ix + 1, r + 1) returns the
// 2x2 block with lower corner (ix, r) as x = (ix, r+1), y = (ix+1, r+1),
// z = (ix+1, r), w = (ix, r); a second gather h rows further down gives slice z+1.
// Both coordinates are exact integers below 2^24.  Lanes whose cell test fails
// gather at (1, 1) and return 0.
__device__ __forceinline__ void sample_tex_pair(cudaTextureObject_t tex, const SampleGeo& g, float hf, float2 px,
                                                float2 py, float2 pz, bool enA, bool enB, uint32_t& oA, uint32_t& oB)
{
    const bool okA = enA && !(px.x < 0.0f || py.x < 0.0f || pz.x < 0.0f) && (px.x < g.wl) && (py.x < g.hl) &&
                     (pz.x < g.dl);
    const bool okB = enB && !(px.y < 0.0f || py.y < 0.0f || pz.y < 0.0f) && (px.y < g.wl) && (py.y < g.hl) &&
                     (pz.y < g.dl);
    const float2 t23 = bc2(kTwo23);
    const float2 rx = make_float2(__fadd_rz(px.x, kTwo23), __fadd_rz(px.y, kTwo23));
    const float2 ry = make_float2(__fadd_rz(py.x, kTwo23), __fadd_rz(py.y, kTwo23));
    const float2 rz = make_float2(__fadd_rz(pz.x, kTwo23), __fadd_rz(pz.y, kTwo23));
    const float2 fx = sub2(rx, t23), fy = sub2(ry, t23), fz = sub2(rz, t23);
    const float2 p0 = sub2(px, fx), p1 = sub2(py, fy), p2 = sub2(pz, fz);
    const float2 one = bc2(1.0f);
    const float2 n0 = sub2(one, p0), n1 = sub2(one, p1), n2 = sub2(one, p2);
    const float2 n0n1 = mul2(n0, n1), p0n1 = mul2(p0, n1), n0p1 = mul2(n0, p1), p0p1 = mul2(p0, p1);
    // texture coordinates (exact integers): u = ix + 1, v = iz*h + iy + 1
    const float2 zh = make_float2(__fmul_rn(fz.x, hf), __fmul_rn(fz.y, hf));
    const float2 u = add2(fx, one), v = add2(add2(zh, fy), one);
    const float uA = okA ? u.x : 1.0f, vA = okA ? v.x : 1.0f;
    const float uB = okB ? u.y : 1.0f, vB = okB ? v.y : 1.0f;
    const float4 a0 = tex2Dgather<float4>(tex, uA, vA, 0);
    const float4 b0 = tex2Dgather<float4>(tex, uB, vB, 0);
    const float4 a1 = tex2Dgather<float4>(tex, uA, vA + hf, 0);
    const float4 b1 = tex2Dgather<float4>(tex, uB, vB + hf, 0);
    const float2 c[8] = {make_float2(a0.w, b0.w), make_float2(a0.z, b0.z), make_float2(a0.x, b0.x),
                         make_float2(a0.y, b0.y), make_float2(a1.w, b1.w), make_float2(a1.z, b1.z),
                         make_float2(a1.x, b1.x), make_float2(a1.y, b1.y)};
    const float2 wt[8] = {mul2(n0n1, n2), mul2(p0n1, n2), mul2(n0p1, n2), mul2(p0p1, n2),
                          mul2(n0n1, p2), mul2(p0n1, p2), mul2(n0p1, p2), mul2(p0p1, p2)};
    float2 acc;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float2 m = make_float2(__fmul_rn(c[k].x, wt[k].x), __fmul_rn(c[k].y, wt[k].y));  // feeds a sum: scalar
        acc = (k == 0) ? m : add2(acc, m);
    }
    const float2 tr = make_float2(__fadd_rz(acc.x, kTwo23), __fadd_rz(acc.y, kTwo23));
    oA = (okA && acc.x > 0.0f) ? (uint32_t)(__float_as_int(tr.x) - 0x4B000000) : 0u;
    oB = (okB && acc.y > 0.0f) ? (uint32_t)(__float_as_int(tr.y) - 0x4B000000) : 0u;
}

// Per-row part of the transform: for a fixed row (y, z), y*T[3a+1] and z*T[3a+2]
// of each axis a; the per-voxel remainder ((x*T0 + yT1) + zT2) + s keeps the
// reference's summation order.  The x column and the shift are held once (ColXform)
// and shared by every row a thread works on.
struct ColXform {
    float t0[3], s[3];
    __device__ __forceinline__ void set(const float* T)
    {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            t0[a] = T[3 * a];
            s[a] = T[9 + a];
        }
    }
};
struct RowXform {
    float yt[3], zt[3];
    __device__ __forceinline__ void set(const float* T, int y, int z)
    {
        const float fy = (float)y, fz = (float)z;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            yt[a] = fy * T[3 * a + 1];
            zt[a] = fz * T[3 * a + 2];
        }
    }
    __device__ __forceinline__ void at(const ColXform& c, float fx, float& px, float& py, float& pz) const
    {
        px = fx * c.t0[0] + yt[0] + zt[0] + c.s[0];
        py = fx * c.t0[1] + yt[1] + zt[1] + c.s[1];
        pz = fx * c.t0[2] + yt[2] + zt[2] + c.s[2];
    }
};

__device__ __forceinline__ void unflat(int i, const Dim3& D, int& x, int& y, int& z)
{
    x = i % D.w;
    int t = i / D.w;
    y = t % D.h;
    z = t / D.h;
}

// Block-wide reductions over a power-of-two block (<= 1024 threads).
template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ T block_sum(T v, T* scratch /* >= 32 */)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0)
        scratch[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? scratch[threadIdx.x] : T(0);
    if (wid == 0)
        v = warp_sum(v);
    return v;  // valid in thread 0
}

}  // namespace regb
