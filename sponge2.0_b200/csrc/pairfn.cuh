// Device-side pair arithmetic shared by the cluster-list force kernels and
// the reference-layout kernels: the packed FP32x2 LJ + screened-Coulomb pair
// function, the exact 22-bit cluster-centre difference, warp reductions and
// the PME excluded-pair kernel h(x).
#pragma once

#include "common.cuh"
#include "ewald_fit.h"

namespace spgnb
{
namespace
{

constexpr float kTwoPow32 = 4294967296.0f;

__device__ __forceinline__ float3 pair_offset(float ex, float ey, float ez, float4 pi, float4 pj, bool image,
                                              const SysDesc& D)
{
    float dx = (ex - pi.x) + pj.x;
    float dy = (ey - pi.y) + pj.y;
    float dz = (ez - pi.z) + pj.z;
    if (image)
    {
        const float sx = rintf(dx * D.rcell.a11 + dy * D.rcell.a21 + dz * D.rcell.a31);
        const float sy = rintf(dy * D.rcell.a22 + dz * D.rcell.a32);
        const float sz = rintf(dz * D.rcell.a33);
        dx -= sx * D.cell.a11 + sy * D.cell.a21 + sz * D.cell.a31;
        dy -= sy * D.cell.a22 + sz * D.cell.a32;
        dz -= sz * D.cell.a33;
    }
    return make_float3(dx, dy, dz);
}

// Transpose of an 8x8 bit matrix held as 64 bits, row r in byte r (bit 8r + c
// moves to bit 8c + r): three rounds of swapping off-diagonal blocks of
// 1x1, 2x2 and 4x4 bits (H. S. Warren, Hacker's Delight, 2nd ed., section 7-3).
__device__ __forceinline__ unsigned long long transpose8x8(unsigned long long x)
{
    unsigned long long t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
    x ^= t ^ (t << 7);
    t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
    x ^= t ^ (t << 14);
    t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
    x ^= t ^ (t << 28);
    return x;
}

// ------------------------------------------------ packed FP32x2 pair math
__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }

// Fixed (c, c) constants of the packed arithmetic in constant memory, so the
// FP32x2 instructions read them as constant-bank operands instead of
// building register pairs each time.
static __constant__ float2 kPk[1] = {{-1.0f, -1.0f}};
enum PackedConst
{
    kPkMinusOne = 0
};
// pair_scalar2's LJ energy is -12 times the energy (A/(12 r^12) - B/(6 r^6)):
// the kernels scale the sums once
constexpr float kLjEnergyScale = -1.0f / 12.0f;

__device__ __forceinline__ float2 poly5x2(float2 x, const float2* c)
{
    float2 p = __ffma2_rn(c[5], x, c[4]);
    p = __ffma2_rn(p, x, c[3]);
    p = __ffma2_rn(p, x, c[2]);
    p = __ffma2_rn(p, x, c[1]);
    return __ffma2_rn(p, x, c[0]);
}

__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The hardware approximations with subnormals flushed (PTX rsqrt.approx.ftz,
// rcp.approx.ftz): r^2 of a listed pair and the fits' denominators (>= 1)
// are far from the subnormal range, so the range handling of rsqrtf and
// __fdividef is not needed.
__device__ __forceinline__ float rsqrt_approx(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// One system's pair-function parameters as (v, v) pairs, made once per atom
// pair and kept in registers over its list.
struct PairParams2
{
    float2 w_scale, nbeta3, nbeta, beta_2_sqrtpi, nb2_log2e;
    float rc2, beta;
};

__device__ __forceinline__ PairParams2 pack_params(const ForceParams& pc)
{
    PairParams2 q;
    q.w_scale = f2(pc.w_scale);
    q.nbeta3 = f2(-pc.beta3);
    q.nbeta = f2(-pc.beta);
    q.beta_2_sqrtpi = f2(pc.beta * 1.1283791670955126f);
    q.nb2_log2e = f2(-pc.beta * pc.beta * 1.4426950408889634f);  // -w log2(e) = -beta^2 r^2 log2(e)
    q.rc2 = pc.rc2;
    q.beta = pc.beta;
    return q;
}

// pair_scalar for two pairs at once; nA = -A.  Without energies the screened
// Coulomb force uses the K fit; with energies it uses the M fit and
// exp(-w): beta^3 K(w) = beta (M(w) - 2/sqrt(pi) exp(-w)) / r^2, so
//   F_c/qq = (t + beta 2/sqrt(pi) exp(-w)) / r^2,  E_c/qq = t,  t = 1/r - beta M(w).
template <bool ENERGY, int FIT>
__device__ __forceinline__ float2 pair_scalar2(float2 r2, float2 qq, float2 nA, float2 B, const PairParams2& pc,
                                               float2& e_lj, float2& e_c)
{
    // the hardware reciprocal square root alone: a Newton step on top of it
    // moves the forces' error against FP64 by 1e-8 relative RMS and costs
    // four packed instructions a word
    const float2 rinv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    const float2 r2inv = __fmul2_rn(rinv, rinv);
    const float2 r6inv = __fmul2_rn(__fmul2_rn(r2inv, r2inv), r2inv);
    // u = (-A/r^6 + B)/r^6 serves the force and, plus B/r^6, the energy
    const float2 u = __fmul2_rn(__ffma2_rn(nA, r6inv, B), r6inv);
    const float2 flj = __fmul2_rn(u, r2inv);
    float2 fc;
    if (FIT == 1)
    {
        const float2 x = __fmul2_rn(r2, pc.w_scale);
        if (!ENERGY)
        {
            const float2 kp = poly5x2(x, kEwaldKP2), kq = poly5x2(x, kEwaldKQ2);
            const float2 K = __fmul2_rn(kp, make_float2(rcp_approx(kq.x), rcp_approx(kq.y)));
            fc = __fmul2_rn(qq, __ffma2_rn(pc.nbeta3, K, __fmul2_rn(rinv, r2inv)));
        }
        else
        {
            const float2 mp = poly5x2(x, kEwaldMP2), mq = poly5x2(x, kEwaldMQ2);
            const float2 M = __fmul2_rn(mp, make_float2(rcp_approx(mq.x), rcp_approx(mq.y)));
            const float2 wl = __fmul2_rn(r2, pc.nb2_log2e);
            const float2 E = make_float2(ex2_approx(wl.x), ex2_approx(wl.y));
            const float2 t = __ffma2_rn(pc.nbeta, M, rinv);
            e_c = __fmul2_rn(qq, t);
            fc = __fmul2_rn(__fmul2_rn(qq, r2inv), __ffma2_rn(pc.beta_2_sqrtpi, E, t));
        }
    }
    else
    {
        float c[2], e[2];
        const float rr[2] = {r2.x, r2.y}, ri[2] = {rinv.x, rinv.y}, q[2] = {qq.x, qq.y};
        for (int h2 = 0; h2 < 2; h2++)
        {
            const float r = rr[h2] * ri[h2];
            const float br = pc.beta * r;
            const float erfcv = erfcf(br);
            c[h2] = q[h2] * ri[h2] * ri[h2] * ri[h2] * __fmaf_rn(br * 1.1283791670955126f, __expf(-br * br), erfcv);
            e[h2] = q[h2] * erfcv * ri[h2];
        }
        fc = make_float2(c[0], c[1]);
        if (ENERGY) e_c = make_float2(e[0], e[1]);
    }
    if (ENERGY) e_lj = __ffma2_rn(B, r6inv, u);  // -A/r^12 + 2B/r^6 = -12 E_lj
    return __ffma2_rn(fc, kPk[kPkMinusOne], flj);
}

// A difference of two 22-bit cluster-centre coordinates, wrapped to
// [-2^21, 2^21) (minimum image of the centres) and converted exactly: the
// wrapped value plus 2^23 + 2^21 is an integer below 2^23 + 2^22, whose float
// bit pattern is 0x4B000000 | value.
__device__ __forceinline__ float centre_step(int qj, int qi)
{
    return __int_as_float(((qj - qi + 0x200000) & 0x3fffff) | 0x4b000000) - 10485760.0f;
}


__device__ __forceinline__ void cp_async(void* smem, const void* gmem, int bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    if (bytes == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem));
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Sums eight per-lane values over the warp: after three halving exchanges
// (lane bit 4, 3, 2 picks the half it keeps) and two full ones, lanes
// 4v..4v+3 hold the total of value v.  Nine shuffles instead of forty.
template <typename T>
__device__ __forceinline__ T reduce_scatter8(const T (&v)[8], int lane)
{
    const bool h4 = (lane & 16) != 0, h3 = (lane & 8) != 0, h2 = (lane & 4) != 0;
    T u[4], x[2];
#pragma unroll
    for (int k = 0; k < 4; k++)
    {
        const T send = h4 ? v[k] : v[k + 4];
        u[k] = (h4 ? v[k + 4] : v[k]) + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int k = 0; k < 2; k++)
    {
        const T send = h3 ? u[k] : u[k + 2];
        x[k] = (h3 ? u[k + 2] : u[k]) + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    const T send = h2 ? x[0] : x[1];
    T y = (h2 ? x[1] : x[0]) + __shfl_xor_sync(0xffffffffu, send, 4);
    y += __shfl_xor_sync(0xffffffffu, y, 2);
    y += __shfl_xor_sync(0xffffffffu, y, 1);
    return y;
}

// PME excluded-pair correction (Particle_Mesh::PME_Excluded_Force_With_Atom_Energy,
// PM_force.cpp:918-997): reciprocal space includes every pair, excluded ones
// too, so their smooth part erf(beta r)/r is taken back out.  One thread per
// atom walks its (upper-triangular) exclusion list, as the reference does:
//   dr = min image(r_j - r_i),  x = beta r,
//   F_i += q_i q_j beta^3 h(x) dr,  F_j -= the same,  E_i -= q_i q_j erf(x)/r,
//   W_i -= F (x) dr (the reference's symmetric virial form),
// with h(x) = (erf(x) - 2/sqrt(pi) x exp(-x^2)) / x^3.  Below x = 0.7, h is
// summed from its Taylor series (the series of erf and of x exp(-x^2)
// combined: h = 2/sqrt(pi) sum_{n>=1} (-1)^(n+1) 2n x^(2n-2) / ((2n+1) n!))
// instead of the difference of two nearly equal numbers, so the correction
// keeps FP32 precision at bonded distances.  Forces accumulate in int64 fixed
// point (the partner's share by atomics), the energy total likewise, so the
// result does not depend on the order.
__device__ __forceinline__ float excl_h(float x)
{
    const float x2 = x * x;
    if (x < 0.7f)
    {
        // 2/sqrt(pi) * (2/3 - 2/5 x^2 + 1/7 x^4 - 1/27 x^6 + 1/132 x^8 - 1/780 x^10 + 1/5400 x^12
        //               - 1/42840 x^14)
        float p = -1.0f / 42840.0f;
        p = __fmaf_rn(p, x2, 1.0f / 5400.0f);
        p = __fmaf_rn(p, x2, -1.0f / 780.0f);
        p = __fmaf_rn(p, x2, 1.0f / 132.0f);
        p = __fmaf_rn(p, x2, -1.0f / 27.0f);
        p = __fmaf_rn(p, x2, 1.0f / 7.0f);
        p = __fmaf_rn(p, x2, -0.4f);
        p = __fmaf_rn(p, x2, 2.0f / 3.0f);
        return 1.1283791670955126f * p;
    }
    return (erff(x) - 1.1283791670955126f * x * expf(-x2)) / (x2 * x);
}

}  // namespace
}  // namespace spgnb
