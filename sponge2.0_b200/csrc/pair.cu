// LJ + PME direct-space pair force, energy and virial:
// LENNARD_JONES_INFORMATION and SOLVENT_LENNARD_JONES of
// SPONGE/Lennard_Jones_force/{Lennard_Jones_force,solvent_LJ}.cpp.
//
// Pair function (Lennard_Jones_force.h:44-73), evaluated in FP32:
//   F/r = (B - A r^-6) r^-8 - q_i q_j [r^-3 - beta^3 K(beta^2 r^2)]
//   E_lj = (A/12 r^-6 - B/6) r^-6,  E_c = q_i q_j [r^-1 - beta M(beta^2 r^2)]
// where K, M are the smooth parts of the screened Coulomb kernels
// (ewald_fit.h).  Over an spgnb list every atom is one warp walking its full
// partner list, so its force is complete in registers and written once, with
// no atomics; energy/virial totals accumulate in int64 fixed point.  Over a
// reference-layout (half) list the force accumulates in int64 fixed point.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace spgnb
{
namespace
{

constexpr int kForceWarps = 8;  // warps per block of the full-list kernel: one cluster per block pass
constexpr float kTwoPow32 = 4294967296.0f;

using PairConst = ForceParams;

__device__ __forceinline__ float poly5(float x, const float* c)
{
    float p = c[5];
    p = __fmaf_rn(p, x, c[4]);
    p = __fmaf_rn(p, x, c[3]);
    p = __fmaf_rn(p, x, c[2]);
    p = __fmaf_rn(p, x, c[1]);
    return __fmaf_rn(p, x, c[0]);
}

// Scalar pair force F/r (and energies when requested) for r2 > 0.
// FIT: 1 the rational fits (beta*rc inside their range), 0 erfcf/expf,
// 2 chosen at run time from pc.use_fit.
template <bool ENERGY, int FIT = 2>
__device__ __forceinline__ float pair_scalar(float r2, float qq, float A, float B, const PairConst& pc,
                                             float& e_lj, float& e_c)
{
    float rinv = rsqrtf(r2);
    rinv = rinv * __fmaf_rn(-0.5f * r2 * rinv, rinv, 1.5f);  // one Newton step
    const float r2inv = rinv * rinv;
    const float r6inv = r2inv * r2inv * r2inv;
    const float flj = __fmaf_rn(-A, r6inv, B) * r6inv * r2inv;
    float fc;
    if (FIT == 1 || (FIT == 2 && pc.use_fit))
    {
        const float x = r2 * pc.w_scale;
        const float K = __fdividef(poly5(x, kEwaldKP), poly5(x, kEwaldKQ));
        fc = qq * __fmaf_rn(-pc.beta3, K, rinv * r2inv);
        if (ENERGY)
        {
            const float M = __fdividef(poly5(x, kEwaldMP), poly5(x, kEwaldMQ));
            e_c = qq * __fmaf_rn(-pc.beta, M, rinv);
        }
    }
    else
    {
        const float r = r2 * rinv;
        const float br = pc.beta * r;
        const float erfcv = erfcf(br);
        fc = qq * rinv * r2inv * __fmaf_rn(br * 1.1283791670955126f, __expf(-br * br), erfcv);
        if (ENERGY) e_c = qq * erfcv * rinv;
    }
    if (ENERGY) e_lj = __fmaf_rn(A * (1.0f / 12.0f), r6inv, -B * (1.0f / 6.0f)) * r6inv;
    return flj - fc;
}

__device__ __forceinline__ void red_fixed(long long* acc, float v)
{
    long long q = __float2ll_rn(v * kTwoPow32);
    if (q != 0) atomicAdd((unsigned long long*)acc, (unsigned long long)q);
}

// Per-step slot pack: each slot's offset from the build-time cluster centre
// moved by the displacement since the build (minimum image in the system's
// box, so a caller that wraps coordinates between builds is fine), with the
// charge, and its LJ type.  Slot slots_cap is a null slot: 10^4 A away from
// everything, charge 0.  With pruning on
// (pref set) the kernel also flags a re-pruning when some atom moved more
// than half the prune buffer since the last one.
__global__ void k_pack_slots(int slots_cap, int* counters, const int* __restrict__ slot_atom,
                             const int* __restrict__ cl_sys, const SysDesc* __restrict__ sys,
                             const float4* __restrict__ x0, const float4* __restrict__ d0,
                             const float3* __restrict__ crd, const float* __restrict__ charge,
                             const int* __restrict__ local_type, float4* __restrict__ pos, int* __restrict__ ptype,
                             const float4* __restrict__ pref, float half_buffer2, int* __restrict__ prune)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    if (s == slots_cap)
    {
        pos[s] = make_float4(1.0e4f, 1.0e4f, 1.0e4f, 0.0f);
        ptype[s] = 0;
    }
    else if (s < slots_cap)
    {
        const int a = slot_atom[s];
        const float4 d = d0[s];
        float4 p = make_float4(d.x, d.y, d.z, 0.0f);
        int t = 0;
        if (a >= 0)
        {
            const SysDesc& D = sys[cl_sys[s >> 3]];
            const float3 c = crd[a];
            const float4 o = x0[s];
            float dx = c.x - o.x, dy = c.y - o.y, dz = c.z - o.z;
            const float sx = rintf(dx * D.rcell.a11 + dy * D.rcell.a21 + dz * D.rcell.a31);
            const float sy = rintf(dy * D.rcell.a22 + dz * D.rcell.a32);
            const float sz = rintf(dz * D.rcell.a33);
            dx -= sx * D.cell.a11 + sy * D.cell.a21 + sz * D.cell.a31;
            dy -= sy * D.cell.a22 + sz * D.cell.a32;
            dz -= sz * D.cell.a33;
            p = make_float4(d.x + dx, d.y + dy, d.z + dz, charge[a]);
            t = local_type[a];
            if (pref)
            {
                const float4 r = pref[s];
                const float ex = p.x - r.x, ey = p.y - r.y, ez = p.z - r.z;
                moved = ex * ex + ey * ey + ez * ez > half_buffer2;
                if (moved) prune[cl_sys[s >> 3]] = 1;
            }
        }
        pos[s] = p;
        ptype[s] = t;
    }
    if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) counters[kCntPrune] = 1;
}

// Pruning (no reference counterpart; results unchanged).  Runs after every
// rebuild and whenever some atom of a system moved more than buffer/2 since
// its last one (the pack kernel checks).  The lists belong to slot pairs: the
// two atoms of slots 2p and 2p+1 of a cluster share one list, the union of
// their partners within cutoff + buffer, so the force kernel evaluates both
// atoms against each partner it loads.  One warp per cluster walks its
// neighbour table, expands the union of the eight atoms' mask rows 32
// elements at a time into shared memory, loads each candidate partner once,
// tests it against all eight atoms without branches (packed FP32x2, two atoms
// an instruction) and keeps, for each of the four slot pairs in table order, every partner
// within cutoff + buffer of either of the pair's atoms, as a 32-bit word
//   {partner slot - system's first slot (22 bits) | LJ type << 22 |
//    pairs with the first atom << 29 | with the second << 30 | image flag << 31}
// (an atom's bit is clear for itself, its exclusions and other
// non-partners).  The list is padded to a multiple of 32 words with words
// whose atom bits are clear.  Any pair within the cutoff before the next
// pruning was within cutoff + buffer at this one, so the copy misses none.
// buffer <= 0 keeps every listed pair.  The last block to finish clears the
// flags.
constexpr int kPruneWarps = 8;
constexpr int kWindow = 32;                    // lists are padded to whole 32-word windows
constexpr int kWordSlotBits = 22;                  // partner slot field of a list word
constexpr unsigned kWordSlotMask = (1u << kWordSlotBits) - 1u;
constexpr int kWordTypeShift = 22;                 // 7-bit LJ type
constexpr unsigned kWordFirst = 1u << 29, kWordSecond = 1u << 30, kWordImage = 1u << 31;

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

__global__ void __launch_bounds__(kPruneWarps * 32)
    k_prune(ForceParams p0, const ForceParams* __restrict__ fps, float buffer, int* counters, int clusters_cap,
            int table_cap, int slot_cap, const int* __restrict__ cl_sys, const SysDesc* __restrict__ sys,
            const int* __restrict__ tcount, const float4* __restrict__ tab, const uint2* __restrict__ tmask,
            const float4* __restrict__ pos, const int* __restrict__ ptype, float4* __restrict__ pref,
            int* __restrict__ pcount, unsigned* __restrict__ pwords, int n_sys, int* __restrict__ prune)
{
    if (counters[kCntPrune] == 0) return;
    // a chunk's candidates {partner slot | image flag, element lane | own-atom bits << 5}
    __shared__ uint2 buf[kPruneWarps][kChunk * kClusterSize];
    __shared__ float4 own_all[kPruneWarps][kClusterSize];
    // the cluster's atoms negated, per coordinate, as the four slot pairs'
    // {first, second} float2
    __shared__ __align__(16) float nown_all[kPruneWarps][3][kClusterSize];
    __shared__ float4 ent_all[kPruneWarps][32];  // the window's table elements (centre differences)
    __shared__ unsigned long long kept_total;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    if (threadIdx.x == 0) kept_total = 0;
    __syncthreads();
    uint2* __restrict__ mybuf = buf[w];
    float4* __restrict__ own = own_all[w];
    const float2* __restrict__ nown = reinterpret_cast<const float2*>(&nown_all[w][0][0]);
    float4* __restrict__ ent = ent_all[w];
    // one warp per cluster, taken from a shared counter (tables differ in
    // length): each candidate partner is loaded once and tested against the
    // cluster's eight atoms, feeding the four slot pairs' lists
    for (;;)
    {
        int c = 0;
        if (lane == 0) c = atomicAdd(&counters[kCntPruneNext], 1);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= clusters_cap) break;
        const int sy = cl_sys[c];
        if (!prune[sy]) continue;
        const int s0 = c * kClusterSize;
        if (lane < kClusterSize)
        {
            const float4 pl = pos[s0 + lane];
            own[lane] = pl;
            nown_all[w][0][lane] = -pl.x;
            nown_all[w][1][lane] = -pl.y;
            nown_all[w][2][lane] = -pl.z;
            pref[s0 + lane] = pl;
        }
        __syncwarp();
        const SysDesc& D = sys[sy];
        const unsigned slot0 = (unsigned)D.cl_begin * kClusterSize;
        const ForceParams P = fps ? fps[sy] : p0;
        const float rp = sqrtf(P.rc2) + buffer + 1e-3f;
        const float rp2 = buffer > 0.0f ? rp * rp : 3.0e38f;
        const int T = tcount[c];
        const float4* __restrict__ tb = tab + (size_t)c * table_cap;
        const uint2* __restrict__ tm = tmask + (size_t)c * table_cap;
        const int usable = 2 * slot_cap - kWindow;
        int kept[4] = {0, 0, 0, 0};
        for (int t0 = 0; t0 < T; t0 += 32)
        {
            const int t = t0 + lane;
            uint2 mm = make_uint2(0u, 0u);
            float4 e = make_float4(0, 0, 0, 0);
            if (t < T)
            {
                e = tb[t];
                mm = tm[t];
            }
            // partners of any of the eight atoms
            unsigned u = mm.x | mm.y;
            u |= u >> 16;
            u |= u >> 8;
            const unsigned row = u & 0xffu;
            const int cnt = __popc(row);
            int incl = cnt;
            for (int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            const int eb = __float_as_int(e.w);
            const unsigned flag = (eb & (1 << 30)) ? kWordImage : 0u;
            const unsigned base = (unsigned)(eb & 0x3fffffff) | flag;
            int k = incl - cnt;
            // own atom a pairs with neighbour slot b when bit 8a + b is set;
            // transposed, byte b holds neighbour b's own-atom bits
            const unsigned long long tm8 = transpose8x8(((unsigned long long)mm.y << 32) | mm.x);
            ent[lane] = e;
#pragma unroll
            for (int b = 0; b < kClusterSize; b++)
                if ((row >> b) & 1u)
                {
                    const unsigned am = (unsigned)(tm8 >> (8 * b)) & 0xffu;
                    mybuf[k++] = make_uint2(base + b, (unsigned)lane | (am << 5));
                }
            __syncwarp();
            for (int q0 = 0; q0 < total; q0 += 32)
            {
                const int q = q0 + lane;
                const uint2 wv = mybuf[q < total ? q : 0];
                // the element's centre difference, staged by the lane that read it
                const float4 es = ent[wv.y & 31u];
                const float ex = es.x, ey = es.y, ez = es.z;
                const unsigned am = q < total ? (wv.y >> 5) & 0xffu : 0u;
                const int js = (int)(wv.x & 0x7fffffffu);
                const bool img = (wv.x & 0x80000000u) != 0;
                float4 pj = make_float4(0, 0, 0, 0);
                int tj = 0;
                if (am)
                {
                    pj = pos[js];
                    tj = ptype[js];
                }
                const unsigned wbase =
                    ((unsigned)js - slot0) | ((unsigned)tj << kWordTypeShift) | (img ? kWordImage : 0u);
                // bit a: own atom a lies within the pruning radius of the
                // partner.  All eight are tested without branches; the
                // minimum-image path (small boxes) only when a lane needs it.
                unsigned hit = 0;
                if (!__any_sync(0xffffffffu, img && am != 0u))
                {
                    // the partner in the cluster's frame, then two own atoms
                    // at a time in packed FP32x2
                    const float2 cx = make_float2(ex + pj.x, ex + pj.x), cy = make_float2(ey + pj.y, ey + pj.y),
                                 cz = make_float2(ez + pj.z, ez + pj.z);
#pragma unroll
                    for (int p = 0; p < 4; p++)
                    {
                        const float2 dx = __fadd2_rn(cx, nown[p]), dy = __fadd2_rn(cy, nown[4 + p]),
                                     dz = __fadd2_rn(cz, nown[8 + p]);
                        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                        hit |= ((r2.x < rp2 ? 1u : 0u) | (r2.y < rp2 ? 2u : 0u)) << (2 * p);
                    }
                }
                else
                {
#pragma unroll 1
                    for (int a = 0; a < kClusterSize; a++)
                    {
                        const float3 d = pair_offset(ex, ey, ez, own[a], pj, img, D);
                        if (__fmaf_rn(d.z, d.z, __fmaf_rn(d.y, d.y, d.x * d.x)) < rp2) hit |= 1u << a;
                    }
                }
                hit &= am;
#pragma unroll
                for (int p = 0; p < 4; p++)
                {
                    // kept when either atom of the slot pair is in range; the
                    // word's atom bits stay those of the full list
                    const bool keep = ((hit >> (2 * p)) & 3u) != 0u;
                    const unsigned m = __ballot_sync(0xffffffffu, keep);
                    if (keep)
                    {
                        const int kk = kept[p] + __popc(m & ((1u << lane) - 1u));
                        if (kk < usable)
                            pwords[(size_t)(s0 + 2 * p) * slot_cap + kk] = wbase | (((am >> (2 * p)) & 3u) << 29);
                        else
                            atomicOr(&counters[kCntOverflow], kOvfWords);
                    }
                    kept[p] += __popc(m);
                }
            }
            __syncwarp();
        }
        // pad to whole windows: the first atom against itself, no atom bit set
        unsigned long long kept_sum = 0;
#pragma unroll
        for (int p = 0; p < 4; p++)
        {
            const int s1 = s0 + 2 * p;
            const int kp = min(kept[p], usable);
            const int padded = (kp + kWindow - 1) & ~(kWindow - 1);
            for (int k2 = kp + lane; k2 < padded; k2 += 32) pwords[(size_t)s1 * slot_cap + k2] = (unsigned)s1 - slot0;
            if (lane == 0)
            {
                pcount[s1] = padded;
                pcount[s1 + 1] = 0;
            }
            kept_sum += (unsigned long long)kp;
        }
        if (lane == 0) atomicAdd(&kept_total, kept_sum);
        __syncwarp();
    }
    __shared__ int is_last;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        atomicAdd((unsigned long long*)&counters[kCntPWords], kept_total);
        __threadfence();
        is_last = atomicAdd(&counters[kCntPruneDone], 1) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    for (int q = threadIdx.x; q < n_sys; q += blockDim.x) prune[q] = 0;
    if (threadIdx.x == 0)
    {
        unsigned long long* wp = (unsigned long long*)&counters[kCntPWords];
        *(unsigned long long*)&counters[kCntPWordsLast] = atomicExch(wp, 0ull);
        counters[kCntPruneDone] = 0;
        counters[kCntPruneNext] = 0;
        counters[kCntPrune] = 0;
        counters[kCntPrunes] += 1;
    }
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

// Pruned-list force kernel.  A warp takes one slot pair (the two atoms of
// slots 2p, 2p+1 of a cluster) at a time, strided over the grid's warps, and
// walks the pair's shared list, one word per lane per iteration (32-word
// windows).  The next item's header (list length, system, types, the two
// atoms' offsets, the cluster centre) and first window are staged in shared
// memory by cp.async while the warp works on the current one, and the list's
// later windows are loaded kPrefetch iterations ahead.  A word names the
// partner slot, so its offset {delta + displacement, q} and its cluster's
// 22-bit centre load side by side, once for both atoms:
//   dr = (c_j - c_i) * cell / 2^22 + p_j - p_{i1,i2},
// and the two pairs are evaluated with packed FP32x2 arithmetic; the LJ
// coefficients of both come from the warp's shared-memory row for the two
// atoms' types {-A1, -A2, B1, B2} indexed by the partner's type.  Each
// lane's partial forces are converted to int64 fixed point (2^-32
// kcal/mol/A) and summed over the lanes exactly, so an atom's force does not
// depend on the reduction order; one lane per component adds it to the
// caller's array, once per call: bitwise reproducible.
//
// MODE 0: forces.  MODE 1: + energy and virial totals (each pair is seen
// from both atoms, so the sums are halved).  MODE 2: + per-atom energy and
// virial of the pairs the atom owns (the lower global index; water sites
// hand theirs to the residue's first atom, as SOLVENT_LENNARD_JONES does),
// and the totals summed from those (each pair once).
// One item's header and first list window, staged in shared memory by
// asynchronous copies (cp.async) while the warp works on the item before.
struct alignas(16) ItemStage
{
    int n, sy, t1, t2;     // list words, system, LJ types of the two atoms
    int4 ci;               // the cluster's 22-bit centre
    float4 p1, p2;         // the two atoms' slot offsets and charges
    unsigned words[32];    // first window of the list
};

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

#ifndef SPGNB_PAIR_MINB2
#define SPGNB_PAIR_MINB2 3
#endif
#ifndef SPGNB_PAIR_MINB0
#define SPGNB_PAIR_MINB0 4
#endif
#ifndef SPGNB_PAIR_PREFETCH
#define SPGNB_PAIR_PREFETCH 2
#endif
constexpr int kPrefetch = SPGNB_PAIR_PREFETCH;  // list windows in flight per warp
__device__ __forceinline__ float excl_h(float x);

template <int MODE, int FIT, bool TRI, bool EXCL>
__global__ void __launch_bounds__(kForceWarps * 32, MODE == 0 ? SPGNB_PAIR_MINB0 : (MODE == 1 ? 3 : SPGNB_PAIR_MINB2))
    k_pair_fast(ForceParams p0, const ForceParams* __restrict__ fps, const SysDesc* __restrict__ sys,
                int n_clusters, int slot_cap,
                const int* __restrict__ cl_sys, const int* __restrict__ pcount, const unsigned* __restrict__ pwords,
                const int* __restrict__ slot_atom, const int* __restrict__ slot_gid, const int4* __restrict__ cl_q,
                const float4* __restrict__ pos, const int* __restrict__ ptype,
                const float2* __restrict__ gtable, int n_types, float3* __restrict__ frc,
                long long* __restrict__ totals, OwnerMap om, PerAtomOut pa, const int* __restrict__ only,
                ExclFuse xf)
{
    extern __shared__ float4 rows_all[];        // per warp: n_types rows {-A1, -A2, B1, B2}
    __shared__ long long red[kForceWarps][8];  // per-warp fixed-point totals (lane 0)
    __shared__ int row_of[kForceWarps][2];     // table rows the warp's shared row was built from
    constexpr bool EN = MODE >= 1;
    constexpr bool PA = MODE >= 2;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    float4* __restrict__ rows = rows_all + w * n_types;
    if (EN && lane < 8) red[w][lane] = 0;
    if (lane < 2) row_of[w][lane] = -1;
    __syncwarp();
    int cur_sys = -1;              // the system red[w] accumulates for
    const int items = n_clusters * 4;
    __shared__ ItemStage stage_all[kForceWarps][2];
    ItemStage* stage = stage_all[w];
    const int stride = gridDim.x * kForceWarps;
    // stages item `it` (nothing past the end: an empty group keeps the count)
    auto prefetch = [&](int it, ItemStage& S) {
        if (it < items)
        {
            const int c = it >> 2;
            const int s1 = c * kClusterSize + 2 * (it & 3);
            if (lane == 0) cp_async(&S.n, pcount + s1, 4);
            if (lane == 1) cp_async(&S.sy, cl_sys + c, 4);
            if (lane == 2) cp_async(&S.t1, ptype + s1, 8);
            if (lane == 3) cp_async(&S.ci, cl_q + c, 16);
            if (lane == 4) cp_async(&S.p1, pos + s1, 16);
            if (lane == 5) cp_async(&S.p2, pos + s1 + 1, 16);
            cp_async(&S.words[lane], pwords + (size_t)s1 * slot_cap + lane, 4);
        }
        cp_async_commit();
    };
    int kk = 0;
    prefetch(blockIdx.x * kForceWarps + w, stage[0]);
    for (int it = blockIdx.x * kForceWarps + w; it < items; it += stride, kk++)
    {
        // every lane has read the buffer the next prefetch overwrites
        __syncwarp();
        prefetch(it + stride, stage[(kk + 1) & 1]);
        cp_async_wait_prior();
        __syncwarp();
        const ItemStage& S = stage[kk & 1];
        const int c = it >> 2;
        const int s1 = c * kClusterSize + 2 * (it & 3);
        const int n = S.n;  // a multiple of the window
        if (n == 0) continue;
        const int sy = S.sy;
        if (only && !only[sy]) continue;
        if (EN && sy != cur_sys)
        {
            // totals belong to one system each: flush this warp's share
            __syncwarp();
            if (lane == 0 && cur_sys >= 0)
                for (int q = 0; q < 8; q++)
                {
                    const long long v = red[w][q];
                    if (v) atomicAdd((unsigned long long*)&totals[8 * cur_sys + q], (unsigned long long)v);
                    red[w][q] = 0;
                }
            __syncwarp();
            cur_sys = sy;
        }
        const ForceParams P = fps ? fps[sy] : p0;
        const PairParams2 pp = pack_params(P);
        const SysDesc& D = sys[sy];
        const Cell qc = D.qcell;
        const int slot0 = D.cl_begin * kClusterSize;
        const float4 pi1 = S.p1, pi2 = S.p2;
        const int4 ci = S.ci;
        const int r1 = S.t1 * n_types + P.table_begin, r2i = S.t2 * n_types + P.table_begin;
        if (r1 != row_of[w][0] || r2i != row_of[w][1])
        {
            __syncwarp();
            for (int t = lane; t < n_types; t += 32)
            {
                const float2 g1 = gtable[r1 + t], g2 = gtable[r2i + t];
                rows[t] = make_float4(-g1.x, -g2.x, g1.y, g2.y);
            }
            if (lane == 0)
            {
                row_of[w][0] = r1;
                row_of[w][1] = r2i;
            }
            __syncwarp();
        }
        int gi1 = 0, gi2 = 0;
        if (PA)
        {
            gi1 = slot_gid[s1];
            gi2 = slot_gid[s1 + 1];
        }
        const unsigned* __restrict__ wl = pwords + (size_t)s1 * slot_cap;
        const float2 npx = make_float2(-pi1.x, -pi2.x), npy = make_float2(-pi1.y, -pi2.y),
                     npz = make_float2(-pi1.z, -pi2.z), qi2 = make_float2(pi1.w, pi2.w);
        float2 fx = f2(0.0f), fy = f2(0.0f), fz = f2(0.0f);
        float2 acc[PA ? 1 : 8], own[PA ? 8 : 1];  // totals (MODE 1) or owned sums (MODE 2)
#pragma unroll
        for (int q = 0; q < (PA ? 1 : 8); q++) acc[q] = f2(0.0f);
#pragma unroll
        for (int q = 0; q < (PA ? 8 : 1); q++) own[q] = f2(0.0f);
        // one list word: the partner against both atoms
        auto eval_word = [&](unsigned cw, int j, float4 pj, int4 cj) {
            const float4 ab = rows[(cw >> kWordTypeShift) & 0x7fu];
            const float ux = centre_step(cj.x, ci.x), uy = centre_step(cj.y, ci.y), uz = centre_step(cj.z, ci.z);
            // the partner in the frame of the pair's cluster centre
            float sx = __fmaf_rn(ux, qc.a11, pj.x);
            float sy2 = __fmaf_rn(uy, qc.a22, pj.y);
            const float sz = __fmaf_rn(uz, qc.a33, pj.z);
            if (TRI)
            {
                sx = __fmaf_rn(uy, qc.a21, sx);
                sx = __fmaf_rn(uz, qc.a31, sx);
                sy2 = __fmaf_rn(uz, qc.a32, sy2);
            }
            float2 dx = __fadd2_rn(f2(sx), npx), dy = __fadd2_rn(f2(sy2), npy), dz = __fadd2_rn(f2(sz), npz);
            if (cw & kWordImage)
            {
                // small box: these pairs need their own image
                float ddx[2] = {dx.x, dx.y}, ddy[2] = {dy.x, dy.y}, ddz[2] = {dz.x, dz.y};
                for (int h = 0; h < 2; h++)
                {
                    const float tx = rintf(ddx[h] * D.rcell.a11 + ddy[h] * D.rcell.a21 + ddz[h] * D.rcell.a31);
                    const float ty = rintf(ddy[h] * D.rcell.a22 + ddz[h] * D.rcell.a32);
                    const float tz = rintf(ddz[h] * D.rcell.a33);
                    ddx[h] -= tx * D.cell.a11 + ty * D.cell.a21 + tz * D.cell.a31;
                    ddy[h] -= ty * D.cell.a22 + tz * D.cell.a32;
                    ddz[h] -= tz * D.cell.a33;
                }
                dx = make_float2(ddx[0], ddx[1]);
                dy = make_float2(ddy[0], ddy[1]);
                dz = make_float2(ddz[0], ddz[1]);
            }
            const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
            const bool inA = (cw & kWordFirst) && r2.x < pp.rc2;
            const bool inB = (cw & kWordSecond) && r2.y < pp.rc2;
            float2 elj, ec;
            float2 f = pair_scalar2<EN, FIT>(r2, __fmul2_rn(f2(pj.w), qi2), make_float2(ab.x, ab.y),
                                             make_float2(ab.z, ab.w), pp, elj, ec);
            f = make_float2(inA ? f.x : 0.0f, inB ? f.y : 0.0f);
            if (!EN)
            {
                fx = __ffma2_rn(f, dx, fx);
                fy = __ffma2_rn(f, dy, fy);
                fz = __ffma2_rn(f, dz, fz);
            }
            else
            {
                const float2 gx = __fmul2_rn(f, dx), gy = __fmul2_rn(f, dy), gz = __fmul2_rn(f, dz);
                fx = __fadd2_rn(fx, gx);
                fy = __fadd2_rn(fy, gy);
                fz = __fadd2_rn(fz, gz);
                if (!PA)
                {
                    elj = make_float2(inA ? elj.x : 0.0f, inB ? elj.y : 0.0f);
                    ec = make_float2(inA ? ec.x : 0.0f, inB ? ec.y : 0.0f);
                    acc[0] = __fadd2_rn(acc[0], elj);
                    acc[1] = __fadd2_rn(acc[1], ec);
                    acc[2] = __ffma2_rn(gx, dx, acc[2]);
                    acc[3] = __ffma2_rn(gx, dy, acc[3]);
                    acc[4] = __ffma2_rn(gy, dy, acc[4]);
                    acc[5] = __ffma2_rn(gx, dz, acc[5]);
                    acc[6] = __ffma2_rn(gy, dz, acc[6]);
                    acc[7] = __ffma2_rn(gz, dz, acc[7]);
                }
                else
                {
                    // only the pair's owner (the lower global index) keeps its
                    // energy and virial; the totals are summed from these, so
                    // every pair counts once
                    const int gj = __ldg(slot_gid + j);
                    const bool oA = inA && gi1 < gj, oB = inB && gi2 < gj;
                    own[0] = __fadd2_rn(own[0], make_float2(oA ? elj.x : 0.0f, oB ? elj.y : 0.0f));
                    own[1] = __fadd2_rn(own[1], make_float2(oA ? ec.x : 0.0f, oB ? ec.y : 0.0f));
                    const float2 mgx = make_float2(oA ? gx.x : 0.0f, oB ? gx.y : 0.0f);
                    const float2 mgy = make_float2(oA ? gy.x : 0.0f, oB ? gy.y : 0.0f);
                    const float2 mgz = make_float2(oA ? gz.x : 0.0f, oB ? gz.y : 0.0f);
                    own[2] = __ffma2_rn(mgx, dx, own[2]);
                    own[3] = __ffma2_rn(mgx, dy, own[3]);
                    own[4] = __ffma2_rn(mgy, dy, own[4]);
                    own[5] = __ffma2_rn(mgx, dz, own[5]);
                    own[6] = __ffma2_rn(mgy, dz, own[6]);
                    own[7] = __ffma2_rn(mgz, dz, own[7]);
                }
            }
        };
        auto partner = [&](unsigned cw) { return slot0 + (int)(cw & kWordSlotMask); };
        // the list streams from memory: its windows are loaded kPrefetch
        // iterations ahead of their use (a ring of registers)
        unsigned ring[kPrefetch];
        ring[0] = S.words[lane];
#pragma unroll
        for (int q = 1; q < kPrefetch; q++) ring[q] = q * 32 < n ? wl[q * 32 + lane] : 0u;
#pragma unroll 1
        for (int k0 = 0; k0 < n; k0 += 32)
        {
            const unsigned cw = ring[0];
#pragma unroll
            for (int q = 0; q + 1 < kPrefetch; q++) ring[q] = ring[q + 1];
            if (k0 + kPrefetch * 32 < n) ring[kPrefetch - 1] = wl[k0 + kPrefetch * 32 + lane];
            const int j = partner(cw);
            eval_word(cw, j, pos[j], cl_q[j >> 3]);
        }
        if (EXCL)
        {
            // PME's excluded-pair correction for the two atoms (each atom's
            // excluded partners on both sides, one pair per lane), as
            // k_pme_excluded computes it; the force joins the lane's partial
            // sums, the energy and per-atom outputs go to the pair's owner
            // (lower global index)
            const int a1 = slot_atom[s1], a2 = slot_atom[s1 + 1];
            const int2 sn1 = a1 >= 0 ? xf.sn[a1] : make_int2(0, 0), sn2 = a2 >= 0 ? xf.sn[a2] : make_int2(0, 0);
            const int n1 = sn1.y, n2 = sn2.y;
            float eown = 0.0f;
            for (int k = lane; k < n1 + n2; k += 32)
            {
                const bool sec = k >= n1;
                const int ia = sec ? a2 : a1;
                const int jx = xf.list[sec ? sn2.x + k - n1 : sn1.x + k];
                const float3 ri = xf.crd[ia], rj = xf.crd[jx];
                float ex = rj.x - ri.x, ey = rj.y - ri.y, ez = rj.z - ri.z;
                const float tx = floorf(ex * D.rcell.a11 + ey * D.rcell.a21 + ez * D.rcell.a31 + 0.5f);
                const float ty = floorf(ey * D.rcell.a22 + ez * D.rcell.a32 + 0.5f);
                const float tz = floorf(ez * D.rcell.a33 + 0.5f);
                ex -= tx * D.cell.a11 + ty * D.cell.a21 + tz * D.cell.a31;
                ey -= ty * D.cell.a22 + tz * D.cell.a32;
                ez -= tz * D.cell.a33;
                const float er = sqrtf(ex * ex + ey * ey + ez * ez);
                const float x = xf.beta * er;
                const float qq = xf.charge[ia] * xf.charge[jx];
                const float fa = qq * xf.beta3 * excl_h(x);
                const float gx = fa * ex, gy = fa * ey, gz = fa * ez;
                if (sec)
                {
                    fx.y += gx;
                    fy.y += gy;
                    fz.y += gz;
                }
                else
                {
                    fx.x += gx;
                    fy.x += gy;
                    fz.x += gz;
                }
                if (EN && xf.atom_local[ia] < xf.atom_local[jx])
                {
                    const float e = -qq * erff(x) / er;
                    eown += e;
                    if (PA)
                    {
                        if (xf.energy) atomicAdd(xf.energy + ia, e);
                        if (xf.virial)
                        {
                            float* v = xf.virial + 6 * (size_t)ia;
                            atomicAdd(v + 0, -gx * ex);
                            atomicAdd(v + 1, -(gx * ey + gy * ex));
                            atomicAdd(v + 2, -gy * ey);
                            atomicAdd(v + 3, -(gx * ez + gz * ex));
                            atomicAdd(v + 4, -(gy * ez + gz * ey));
                            atomicAdd(v + 5, -gz * ez);
                        }
                    }
                }
            }
            if (EN && n1 + n2 > 0)
            {
                long long qe = __double2ll_rn((double)eown * kEnergyScale);
                for (int o = 16; o > 0; o >>= 1) qe += __shfl_xor_sync(0xffffffffu, qe, o);
                if (lane == 0 && qe) atomicAdd((unsigned long long*)xf.total, (unsigned long long)qe);
            }
        }
        // forces of both atoms: int64 fixed point per lane, summed over the
        // lanes by a reduce-scatter (lanes 4v..4v+3 end with value v)
        long long fq[8] = {__float2ll_rn(fx.x * kTwoPow32), __float2ll_rn(fy.x * kTwoPow32),
                           __float2ll_rn(fz.x * kTwoPow32), __float2ll_rn(fx.y * kTwoPow32),
                           __float2ll_rn(fy.y * kTwoPow32), __float2ll_rn(fz.y * kTwoPow32), 0, 0};
        const long long fsum = reduce_scatter8(fq, lane);
        const int vidx = lane >> 2;  // the value this lane holds
        if ((lane & 3) == 0 && vidx < 6)
        {
            const int ai = slot_atom[s1 + (vidx >= 3 ? 1 : 0)];
            if (ai >= 0)  // one add per component and call: the same as a read-modify-write, without the wait
                atomicAdd(&frc[ai].x + (vidx % 3), (float)((double)fsum * kForceUnscale));
        }
        if (EN && !PA)
        {
            float ev[8];
#pragma unroll
            for (int q = 0; q < 8; q++)
                ev[q] = (q >= 2 ? -1.0f : (q == 0 ? kLjEnergyScale : 1.0f)) * (acc[q].x + acc[q].y);
            const float esum = reduce_scatter8(ev, lane);
            if ((lane & 3) == 0)
            {
                // halve the double-counted sums; the symmetric off-diagonal
                // terms (xy + yx etc.) are twice the one accumulated
                const double sc = (vidx == 3 || vidx == 5 || vidx == 6) ? 1.0 : 0.5;
                red[w][vidx] += __double2ll_rn((double)esum * sc * kEnergyScale);
            }
        }
        if (PA)
        {
            float own1[8], own2[8];
#pragma unroll
            for (int q = 0; q < 8; q++)
            {
                // the virial terms were accumulated as +g (x) d: the virial is -g (x) d
                const float sg = q >= 2 ? -1.0f : (q == 0 ? kLjEnergyScale : 1.0f);
                own1[q] = sg * own[q].x;
                own2[q] = sg * own[q].y;
            }
            // both atoms' sums over the lanes: lanes 4q..4q+3 end with value q
            const float a = reduce_scatter8(own1, lane), b = reduce_scatter8(own2, lane);
            // an atom's energy is value 0 + value 1 (lanes 0 and 4)
            const float a1 = __shfl_down_sync(0xffffffffu, a, 4), b1 = __shfl_down_sync(0xffffffffu, b, 4);
            if ((lane & 3) == 0)
            {
                // the item's totals: each pair once; the symmetric off-diagonal
                // terms (xy + yx etc.) are twice the one accumulated
                const bool twice = vidx == 3 || vidx == 5 || vidx == 6;
                red[w][vidx] += __double2ll_rn((double)(a + b) * (twice ? 2.0 : 1.0) * kEnergyScale);
#pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const int ai = slot_atom[s1 + h];
                    if (ai < 0) continue;
                    const float val = h ? b : a;
                    const int o = om.remap(ai);
                    if (vidx == 0)
                    {
                        if (pa.energy) atomicAdd(pa.energy + o, val + (h ? b1 : a1));
                        if (pa.lj_energy) atomicAdd(pa.lj_energy + o, val);
                    }
                    else if (vidx == 1)
                    {
                        if (pa.direct) atomicAdd(pa.direct + o, val);
                    }
                    else if (pa.virial)
                        atomicAdd(pa.virial + 6 * (size_t)o + (vidx - 2), twice ? 2.0f * val : val);
                }
            }
        }
    }
    cp_async_wait_all();
    __syncwarp();
    if (EN && lane == 0 && cur_sys >= 0)
        for (int q = 0; q < 8; q++)
        {
            const long long v = red[w][q];
            if (v) atomicAdd((unsigned long long*)&totals[8 * cur_sys + q], (unsigned long long)v);
        }
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

__global__ void k_pme_excluded(int n, const float3* __restrict__ crd, Cell cell, Cell rcell,
                               const float* __restrict__ charge, float beta, const int* __restrict__ ex_start,
                               const int* __restrict__ ex_list, const int* __restrict__ ex_num,
                               long long* __restrict__ acc, float* __restrict__ atom_ene,
                               float* __restrict__ atom_virial, long long* __restrict__ total)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float ene = 0.0f;
    if (i < n && ex_num[i] > 0)
    {
        const int k0 = ex_start[i], k1 = k0 + ex_num[i];
        const float3 ri = crd[i];
        const float qi = charge[i];
        const float beta3 = beta * beta * beta;
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        float w[6] = {0, 0, 0, 0, 0, 0};
        for (int t = k0; t < k1; t++)
        {
            const int j = ex_list[t];
            const float3 rj = crd[j];
            // Get_Periodic_Displacement(r_j, r_i) (utils/vector.hpp:322-327)
            float dx = rj.x - ri.x, dy = rj.y - ri.y, dz = rj.z - ri.z;
            const float sx = floorf(dx * rcell.a11 + dy * rcell.a21 + dz * rcell.a31 + 0.5f);
            const float sy = floorf(dy * rcell.a22 + dz * rcell.a32 + 0.5f);
            const float sz = floorf(dz * rcell.a33 + 0.5f);
            dx -= sx * cell.a11 + sy * cell.a21 + sz * cell.a31;
            dy -= sy * cell.a22 + sz * cell.a32;
            dz -= sz * cell.a33;
            const float r2 = dx * dx + dy * dy + dz * dz;
            const float r = sqrtf(r2);
            const float x = beta * r;
            const float qq = qi * charge[j];
            const float fa = qq * beta3 * excl_h(x);
            const float gx = fa * dx, gy = fa * dy, gz = fa * dz;
            ene -= qq * erff(x) / r;
            fx += gx;
            fy += gy;
            fz += gz;
            atomicAdd((unsigned long long*)&acc[4 * (size_t)j + 0], (unsigned long long)__float2ll_rn(-gx * kTwoPow32));
            atomicAdd((unsigned long long*)&acc[4 * (size_t)j + 1], (unsigned long long)__float2ll_rn(-gy * kTwoPow32));
            atomicAdd((unsigned long long*)&acc[4 * (size_t)j + 2], (unsigned long long)__float2ll_rn(-gz * kTwoPow32));
            // Get_Virial_From_Force_Dis(F, dr), subtracted
            w[0] -= gx * dx;
            w[1] -= gx * dy + gy * dx;
            w[2] -= gy * dy;
            w[3] -= gx * dz + gz * dx;
            w[4] -= gy * dz + gz * dy;
            w[5] -= gz * dz;
        }
        atomicAdd((unsigned long long*)&acc[4 * (size_t)i + 0], (unsigned long long)__float2ll_rn(fx * kTwoPow32));
        atomicAdd((unsigned long long*)&acc[4 * (size_t)i + 1], (unsigned long long)__float2ll_rn(fy * kTwoPow32));
        atomicAdd((unsigned long long*)&acc[4 * (size_t)i + 2], (unsigned long long)__float2ll_rn(fz * kTwoPow32));
        if (atom_virial)
            for (int q = 0; q < 6; q++) atom_virial[6 * (size_t)i + q] += w[q];
        if (atom_ene) atom_ene[i] += ene;
    }
    // the energy total: one atomic per warp
    long long qe = __double2ll_rn((double)ene * kEnergyScale);
    for (int o = 16; o > 0; o >>= 1) qe += __shfl_xor_sync(0xffffffffu, qe, o);
    if ((threadIdx.x & 31) == 0 && qe) atomicAdd((unsigned long long*)total, (unsigned long long)qe);
}

// Fixed point -> caller's float force (+=) for the reference-layout path,
// accumulators cleared for the next call.
__global__ void k_finalize(int n, long long* __restrict__ acc, float3* __restrict__ frc)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long* a = acc + 4 * (size_t)i;
    long long x = a[0], y = a[1], z = a[2];
    if (x | y | z)
    {
        float3 f = frc[i];
        f.x += (float)((double)x * kForceUnscale);
        f.y += (float)((double)y * kForceUnscale);
        f.z += (float)((double)z * kForceUnscale);
        frc[i] = f;
        a[0] = 0;
        a[1] = 0;
        a[2] = 0;
    }
}

// 20-byte {float3 crd; int type; float charge} records
__global__ void k_vector_lj(int n, const float3* __restrict__ crd, const float* __restrict__ charge,
                            const int* __restrict__ local_type, float* __restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 c = crd[i];
    float* o = out + 5 * (size_t)i;
    o[0] = c.x;
    o[1] = c.y;
    o[2] = c.z;
    o[3] = __int_as_float(local_type[i]);
    o[4] = charge[i];
}

__global__ void k_local_types(int n, const int* __restrict__ atom_local, const int* __restrict__ atom_type,
                              int* __restrict__ local_type)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) local_type[i] = atom_type[atom_local[i]];
}

// ------------------------------------------------ reference-layout lists
__global__ void k_pack_atoms(int n, const float3* __restrict__ crd, const float* __restrict__ charge,
                             const int* __restrict__ local_type, float4* __restrict__ pos, int* __restrict__ ptype)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 c = crd[i];
    pos[i] = make_float4(c.x, c.y, c.z, charge[i]);
    ptype[i] = local_type[i];
}

// Reference minimum image (vector.hpp:322-327), dr = b - a.
__device__ __forceinline__ void ref_image(float& dx, float& dy, float& dz, const Cell& c, const Cell& r)
{
    float sx = floorf(dx * r.a11 + dy * r.a21 + dz * r.a31 + 0.5f);
    float sy = floorf(dy * r.a22 + dz * r.a32 + 0.5f);
    float sz = floorf(dz * r.a33 + 0.5f);
    dx -= sx * c.a11 + sy * c.a21 + sz * c.a31;
    dy -= sy * c.a22 + sz * c.a32;
    dz -= sz * c.a33;
}

// Warp per owner atom over its reference-layout half list
// (Lennard_Jones_force.cpp:43-136 semantics, int64 accumulation).
template <int MODE>
__global__ void k_pair_atom_groups(PairConst pc, Cell cell, Cell rcell, int n_owner, int local_atoms,
                                   const spgnb_atom_group* __restrict__ nl, const float4* __restrict__ pos,
                                   const int* __restrict__ ptype, const float2* __restrict__ table,
                                   long long* __restrict__ acc, long long* __restrict__ totals, PerAtomOut pa)
{
    constexpr bool EN = MODE >= 1;
    const int lane = threadIdx.x & 31;
    const int total_warps = gridDim.x * (blockDim.x >> 5);
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n_owner; i += total_warps)
    {
        const spgnb_atom_group g = nl[i];
        const float4 pi = pos[i];
        const int ti = ptype[i] * pc.n_types;
        float fx = 0, fy = 0, fz = 0;
        float acc8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = lane; k < g.atom_numbers; k += 32)
        {
            const int j = g.atom_serial[k];
            const float4 pj = pos[j];
            float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            ref_image(dx, dy, dz, cell, rcell);
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (!(r2 < pc.rc2)) continue;
            const float2 AB = table[ti + ptype[j]];
            float elj = 0, ec = 0;
            const float fs = pair_scalar<EN>(r2, pi.w * pj.w, AB.x, AB.y, pc, elj, ec);
            const float ij = j < local_atoms ? 1.0f : 0.5f;
            const float gx = fs * dx, gy = fs * dy, gz = fs * dz;
            fx += gx;
            fy += gy;
            fz += gz;
            if (j < local_atoms)
            {
                red_fixed(acc + 4 * (size_t)j + 0, -gx);
                red_fixed(acc + 4 * (size_t)j + 1, -gy);
                red_fixed(acc + 4 * (size_t)j + 2, -gz);
            }
            if (EN)
            {
                acc8[0] += ij * elj;
                acc8[1] += ij * ec;
                acc8[2] -= ij * gx * dx;
                acc8[3] -= ij * (gx * dy + gy * dx);
                acc8[4] -= ij * gy * dy;
                acc8[5] -= ij * (gx * dz + gz * dx);
                acc8[6] -= ij * (gy * dz + gz * dy);
                acc8[7] -= ij * gz * dz;
            }
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
            if (EN)
                for (int q = 0; q < 8; q++) acc8[q] += __shfl_xor_sync(0xffffffffu, acc8[q], o);
        }
        if (lane == 0)
        {
            red_fixed(acc + 4 * (size_t)i + 0, fx);
            red_fixed(acc + 4 * (size_t)i + 1, fy);
            red_fixed(acc + 4 * (size_t)i + 2, fz);
            if (EN)
            {
                for (int q = 0; q < 8; q++)
                {
                    long long v = __double2ll_rn((double)acc8[q] * kEnergyScale);
                    if (v) atomicAdd((unsigned long long*)&totals[q], (unsigned long long)v);
                }
                if (MODE >= 2)
                {
                    if (pa.energy) atomicAdd(pa.energy + i, acc8[0] + acc8[1]);
                    if (pa.lj_energy) atomicAdd(pa.lj_energy + i, acc8[0]);
                    if (pa.direct) atomicAdd(pa.direct + i, acc8[1]);
                    if (pa.virial)
                        for (int q = 0; q < 6; q++) atomicAdd(pa.virial + 6 * (size_t)i + q, acc8[2 + q]);
                }
            }
        }
    }
}

// Water residues over the first site's reference-layout list
// (solvent_LJ.cpp:25-145 semantics): every site of residue r against each j
// of the first site's list; energy and virial to the first site.
template <int MODE, int WP>
__global__ void k_pair_solvent(PairConst pc, Cell cell, Cell rcell, int res_begin, int res_end, int local_atoms,
                               const int* __restrict__ res_start, const spgnb_atom_group* __restrict__ nl,
                               const float4* __restrict__ pos, const int* __restrict__ ptype,
                               const float2* __restrict__ table, long long* __restrict__ acc,
                               long long* __restrict__ totals, PerAtomOut pa)
{
    constexpr bool EN = MODE >= 1;
    const int lane = threadIdx.x & 31;
    const int total_warps = gridDim.x * (blockDim.x >> 5);
    for (int r = res_begin + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < res_end; r += total_warps)
    {
        const int a0 = res_start[r];
        float4 si[WP];
        int ti[WP];
        float fs_[WP][3];
        for (int s = 0; s < WP; s++)
        {
            si[s] = pos[a0 + s];
            ti[s] = ptype[a0 + s] * pc.n_types;
            fs_[s][0] = fs_[s][1] = fs_[s][2] = 0.0f;
        }
        float acc8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const spgnb_atom_group g = nl[a0];
        for (int k = lane; k < g.atom_numbers; k += 32)
        {
            const int j = g.atom_serial[k];
            const float4 pj = pos[j];
            const int tj = ptype[j];
            const float ij = j < local_atoms ? 1.0f : 0.5f;
            float gjx = 0, gjy = 0, gjz = 0;
            for (int s = 0; s < WP; s++)
            {
                float dx = pj.x - si[s].x, dy = pj.y - si[s].y, dz = pj.z - si[s].z;
                ref_image(dx, dy, dz, cell, rcell);
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (!(r2 < pc.rc2)) continue;
                const float2 AB = table[ti[s] + tj];
                float elj = 0, ec = 0;
                const float f = pair_scalar<EN>(r2, si[s].w * pj.w, AB.x, AB.y, pc, elj, ec);
                const float gx = f * dx, gy = f * dy, gz = f * dz;
                fs_[s][0] += gx;
                fs_[s][1] += gy;
                fs_[s][2] += gz;
                gjx -= gx;
                gjy -= gy;
                gjz -= gz;
                if (EN)
                {
                    acc8[0] += ij * elj;
                    acc8[1] += ij * ec;
                    acc8[2] -= ij * gx * dx;
                    acc8[3] -= ij * (gx * dy + gy * dx);
                    acc8[4] -= ij * gy * dy;
                    acc8[5] -= ij * (gx * dz + gz * dx);
                    acc8[6] -= ij * (gy * dz + gz * dy);
                    acc8[7] -= ij * gz * dz;
                }
            }
            if (j < local_atoms)
            {
                red_fixed(acc + 4 * (size_t)j + 0, gjx);
                red_fixed(acc + 4 * (size_t)j + 1, gjy);
                red_fixed(acc + 4 * (size_t)j + 2, gjz);
            }
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            for (int s = 0; s < WP; s++)
                for (int d = 0; d < 3; d++) fs_[s][d] += __shfl_xor_sync(0xffffffffu, fs_[s][d], o);
            if (EN)
                for (int q = 0; q < 8; q++) acc8[q] += __shfl_xor_sync(0xffffffffu, acc8[q], o);
        }
        if (lane == 0)
        {
            for (int s = 0; s < WP; s++)
                for (int d = 0; d < 3; d++) red_fixed(acc + 4 * (size_t)(a0 + s) + d, fs_[s][d]);
            if (EN)
            {
                for (int q = 0; q < 8; q++)
                {
                    long long v = __double2ll_rn((double)acc8[q] * kEnergyScale);
                    if (v) atomicAdd((unsigned long long*)&totals[q], (unsigned long long)v);
                }
                if (MODE >= 2)
                {
                    if (pa.energy) atomicAdd(pa.energy + a0, acc8[0] + acc8[1]);
                    if (pa.lj_energy) atomicAdd(pa.lj_energy + a0, acc8[0]);
                    if (pa.direct) atomicAdd(pa.direct + a0, acc8[1]);
                    if (pa.virial)
                        for (int q = 0; q < 6; q++) atomicAdd(pa.virial + 6 * (size_t)a0 + q, acc8[2 + q]);
                }
            }
        }
    }
}

__global__ void k_long_range(int need_pressure, float* virial, int need_potential, float* potential, float vfac,
                             float efac)
{
    if (need_pressure)
    {
        virial[0] += vfac;
        virial[2] += vfac;
        virial[5] += vfac;
    }
    if (need_potential) potential[0] += efac;
}

__global__ void k_solvent_count(int local_res_numbers, const int* __restrict__ res_len, int water_points,
                                int atom_numbers, const float* __restrict__ mass, int* out)
{
    // SOLVENT_LENNARD_JONES get_local_device (solvent_LJ.cpp:433-467)
    int start = local_res_numbers, cnt = 0;
    for (int i = local_res_numbers - 1; i >= 0; i--)
    {
        int rs = atom_numbers - water_points * (cnt + 1);
        if (rs < 0) break;
        float mo = mass[rs], m1 = mass[rs + 1], m2 = mass[rs + 2];
        if (res_len[i] == water_points && mo > 15.8f && mo < 16.2f && m1 > 1.007f && m1 < 1.009f && m2 > 1.007f &&
            m2 < 1.009f)
        {
            start--;
            cnt++;
        }
        else
            break;
    }
    out[0] = start;
    out[1] = cnt * water_points;
}

PairConst make_pair_const(const spgnb_lj* lj, float beta)
{
    PairConst pc;
    pc.rc2 = lj->cutoff * lj->cutoff;
    pc.beta = beta;
    pc.beta3 = beta * beta * beta;
    pc.w_scale = beta * beta * SPGNB_EWALD_INV_W_MAX;
    pc.n_types = lj->n_types;
    float z = beta * lj->cutoff;
    pc.use_fit = (z * z <= SPGNB_EWALD_W_MAX * 0.999f) ? 1 : 0;
    pc.table_begin = 0;
    pc.pad = 0;
    return pc;
}

// Slot offsets and types plus the null slot.
int ensure_slots(spgnb_lj* lj, int slots)
{
    if (slots + 1 <= lj->sdata_cap) return SPGNB_OK;
    dfree(lj->d_sdata);
    dfree(lj->d_slot_type);
    int st;
    if ((st = dalloc(&lj->d_sdata, (size_t)(slots + 1)))) return st;
    if ((st = dalloc(&lj->d_slot_type, (size_t)(slots + 1)))) return st;
    lj->sdata_cap = slots + 1;
    return SPGNB_OK;
}

int ensure_pos(spgnb_lj* lj, int count)
{
    if (count <= lj->pos_cap) return SPGNB_OK;
    dfree(lj->d_pos);
    dfree(lj->d_pos_type);
    int st;
    if ((st = dalloc(&lj->d_pos, count))) return st;
    if ((st = dalloc(&lj->d_pos_type, count))) return st;
    lj->pos_cap = count;
    return SPGNB_OK;
}

// A persistent grid: as many blocks as can be resident on every SM.
template <typename K>
int pair_blocks(K kernel, int threads, size_t smem)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess ||
        per_sm <= 0)
    {
        cudaGetLastError();
        per_sm = 4;
    }
    return per_sm * num_sms();
}


// Launches the pruned-list force kernel for the given mode / pair-function /
// box-shape variant.
struct FastArgs
{
    ForceParams p0;
    const ForceParams* fps;
    const spgnb_nl* nl;
    const float4* pos;
    const int* ptype;
    const float2* table;
    int n_types;
    float3* frc;
    long long* totals;
    OwnerMap om;
    PerAtomOut pa;
    const int* only;
    ExclFuse xf;
};

template <int M, int F, bool T, bool E>
int launch_fast(const FastArgs& x, size_t smem, cudaStream_t s)
{
    const spgnb_nl* nl = x.nl;
    const int grid =
        std::max(1, std::min(pair_blocks(k_pair_fast<M, F, T, E>, kForceWarps * 32, smem), nl->clusters_cap));
    k_pair_fast<M, F, T, E><<<grid, kForceWarps * 32, smem, s>>>(
        x.p0, x.fps, nl->d_sys, nl->clusters_cap, nl->slot_cap, nl->d_cl_sys, nl->d_pcount, nl->d_pwords,
        nl->d_slot_atom, nl->d_slot_gid, nl->d_cl_q, x.pos, x.ptype, x.table, x.n_types, x.frc, x.totals, x.om, x.pa,
        x.only, x.xf);
    SPGNB_CHECK_LAUNCH("k_pair_fast");
    return SPGNB_OK;
}

template <int M, int F>
int launch_fast_t(const FastArgs& x, bool tri, size_t smem, cudaStream_t s)
{
    if (x.xf.list) return tri ? launch_fast<M, F, true, true>(x, smem, s) : launch_fast<M, F, false, true>(x, smem, s);
    return tri ? launch_fast<M, F, true, false>(x, smem, s) : launch_fast<M, F, false, false>(x, smem, s);
}

template <int M>
int launch_fast_ft(const FastArgs& x, bool fit, bool tri, size_t smem, cudaStream_t s)
{
    return fit ? launch_fast_t<M, 1>(x, tri, smem, s) : launch_fast_t<M, 0>(x, tri, smem, s);
}

int launch_fast_any(const FastArgs& x, int mode, bool fit, bool tri, size_t smem, cudaStream_t s)
{
    if (mode == 0) return launch_fast_ft<0>(x, fit, tri, smem, s);
    if (mode == 1) return launch_fast_ft<1>(x, fit, tri, smem, s);
    return launch_fast_ft<2>(x, fit, tri, smem, s);
}

}  // namespace

int force_kernels_init(int table_size)
{
    (void)table_size;  // the pair kernel's rows take at most kForceWarps * kMaxTypes * 16 bytes
    return SPGNB_OK;
}

int lj_finalize_forces(spgnb_lj* lj, int n, float3* frc, cudaStream_t s)
{
    if (n <= 0) return SPGNB_OK;
    k_finalize<<<(n + 255) / 256, 256, 0, s>>>(n, lj->d_frc_acc, frc);
    SPGNB_CHECK_LAUNCH("k_finalize");
    return SPGNB_OK;
}

int force_pipeline(const ForceInputs& in, cudaStream_t s)
{
    spgnb_nl* nl = in.nl;
    const int slots = nl->clusters_cap * kClusterSize;
    const bool track = nl->opt.prune_buffer > 0.0f;
    const float half = 0.5f * nl->opt.prune_buffer;
    k_pack_slots<<<(slots + 256) / 256, 256, 0, s>>>(slots, nl->d_counters, nl->d_slot_atom, nl->d_cl_sys, nl->d_sys,
                                                     nl->d_slot_x0, nl->d_slot_d0, in.crd, in.charge, in.atom_type,
                                                     in.slot_pos, in.slot_type, track ? nl->d_pref : nullptr,
                                                     half * half, nl->d_prune);
    SPGNB_CHECK_LAUNCH("k_pack_slots");
    const int grid = std::max(1, std::min(num_sms() * 5, (nl->clusters_cap + kPruneWarps - 1) / kPruneWarps));
    k_prune<<<grid, kPruneWarps * 32, 0, s>>>(in.p0, in.d_fps, nl->opt.prune_buffer, nl->d_counters, nl->clusters_cap,
                                              nl->table_cap, nl->slot_cap, nl->d_cl_sys, nl->d_sys, nl->d_tcount,
                                              nl->d_tab, nl->d_tmask, in.slot_pos, in.slot_type, nl->d_pref,
                                              nl->d_pcount, nl->d_pwords, nl->S, nl->d_prune);
    SPGNB_CHECK_LAUNCH("k_prune");
    cudaEvent_t ev0, ev1;
    pair_events(&ev0, &ev1);
    if (ev0) SPGNB_CUDA(cudaEventRecord(ev0, s));
    const int T = (int)lrint(sqrt((double)in.table_size));
    if (T <= 0 || T * T != in.table_size || T > kMaxTypes)
        return fail(SPGNB_E_UNSUPPORTED, "force: the LJ table is not square or has more than %d types", kMaxTypes);
    const FastArgs fa{in.p0, in.d_fps, nl, in.slot_pos, in.slot_type, in.table, T, in.frc,
                      in.totals, in.om, in.pa, in.only, in.xf};
    const int st = launch_fast_any(fa, in.mode, in.fit, nl->triclinic, sizeof(float4) * kForceWarps * T, s);
    if (st) return st;
    if (ev1) SPGNB_CUDA(cudaEventRecord(ev1, s));
    return SPGNB_OK;
}

namespace
{

int check_common(spgnb_lj* lj, int local_atom_numbers, int ghost_numbers, const spgnb_vector* d_crd,
                 const float* d_charge, spgnb_vector* d_frc)
{
    if (!lj) return fail(SPGNB_E_ARG, "LJ handle is NULL");
    if (ghost_numbers != 0)
        return fail(SPGNB_E_UNSUPPORTED, "ghost atoms (multi-rank domain decomposition) are not supported");
    if (local_atom_numbers > lj->atom_numbers)
        return fail(SPGNB_E_ARG, "%d local atoms exceed the %d the module was created for", local_atom_numbers,
                    lj->atom_numbers);
    if (!lj->d_local_type) return fail(SPGNB_E_STATE, "LJ: Get_Local has not been called");
    if (local_atom_numbers > lj->local_atoms)
        return fail(SPGNB_E_STATE, "LJ: %d local atoms but Get_Local saw %d", local_atom_numbers, lj->local_atoms);
    if (!d_crd || !d_charge || !d_frc) return fail(SPGNB_E_ARG, "LJ: NULL device pointer");
    return SPGNB_OK;
}

}  // namespace
}  // namespace spgnb

using namespace spgnb;

extern "C" {

int spgnb_lj_create(int atom_numbers, int atom_type_numbers, const int* h_atom_type, const float* h_pair_A,
                    const float* h_pair_B, float cutoff, spgnb_lj** out)
{
    if (!out) return fail(SPGNB_E_ARG, "spgnb_lj_create: out is NULL");
    *out = nullptr;
    if (atom_numbers <= 0 || atom_type_numbers <= 0 || !h_atom_type || !h_pair_A || !h_pair_B || !(cutoff > 0))
        return fail(SPGNB_E_ARG, "spgnb_lj_create: bad arguments");
    const int T = atom_type_numbers;
    if (T * T * (int)sizeof(float2) > 96 * 1024 || T > kMaxTypes)
        return fail(SPGNB_E_UNSUPPORTED, "spgnb_lj_create: %d LJ types exceed the shared-memory pair table", T);
    std::vector<double> hist(T, 0.0);
    for (int i = 0; i < atom_numbers; i++)
    {
        int t = h_atom_type[i];
        if (t < 0 || t >= T) return fail(SPGNB_E_ARG, "spgnb_lj_create: atom %d has type %d outside [0,%d)", i, t, T);
        hist[t] += 1.0;
    }
    std::vector<float2> table((size_t)T * T);
    double c6 = 0.0;
    for (int a = 0; a < T; a++)
        for (int b = 0; b < T; b++)
        {
            int hi = a > b ? a : b, lo = a > b ? b : a;
            int p = hi * (hi + 1) / 2 + lo;
            table[(size_t)a * T + b] = make_float2(h_pair_A[p], h_pair_B[p]);
            c6 += hist[a] * hist[b] * (double)h_pair_B[p];
        }
    spgnb_lj* lj = new spgnb_lj();
    lj->atom_numbers = atom_numbers;
    lj->n_types = T;
    lj->cutoff = cutoff;
    // Lennard_Jones_force.cpp:263-268 in float arithmetic
    float f = (float)c6;
    f *= -2.0f / 3.0f * 3.1415926535897932f / cutoff / cutoff / cutoff / 6.0f;
    lj->long_range_factor = f;
    int st;
    if ((st = dalloc(&lj->d_atom_type, atom_numbers)) || (st = dalloc(&lj->d_table, table.size())) ||
        (st = dalloc(&lj->d_lj_energy_atom, atom_numbers)) || (st = dalloc(&lj->d_frc_acc, 4 * (size_t)atom_numbers)) ||
        (st = dalloc(&lj->d_totals, 8)) || (st = dalloc(&lj->d_excl_total, 1)))
    {
        spgnb_lj_destroy(lj);
        return st;
    }
    cudaMemset(lj->d_excl_total, 0, sizeof(long long));
    force_kernels_init(T * T);
    cudaMemcpy(lj->d_atom_type, h_atom_type, sizeof(int) * atom_numbers, cudaMemcpyHostToDevice);
    cudaMemcpy(lj->d_table, table.data(), sizeof(float2) * table.size(), cudaMemcpyHostToDevice);
    cudaMemset(lj->d_frc_acc, 0, sizeof(long long) * 4 * (size_t)atom_numbers);
    cudaMemset(lj->d_totals, 0, sizeof(long long) * 8);
    cudaMemset(lj->d_lj_energy_atom, 0, sizeof(float) * atom_numbers);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
    {
        spgnb_lj_destroy(lj);
        return cuda_fail(e, "spgnb_lj_create");
    }
    *out = lj;
    return SPGNB_OK;
}

int spgnb_lj_get_local(spgnb_lj* lj, const int* d_atom_local, int local_atom_numbers, int ghost_numbers)
{
    if (!lj || !d_atom_local) return fail(SPGNB_E_ARG, "spgnb_lj_get_local: NULL argument");
    const int n = local_atom_numbers + ghost_numbers;
    if (n > lj->atom_numbers) return fail(SPGNB_E_ARG, "spgnb_lj_get_local: too many local atoms");
    if (!lj->d_local_type)
    {
        int st = dalloc(&lj->d_local_type, lj->atom_numbers);
        if (st) return st;
    }
    k_local_types<<<(n + 255) / 256, 256, 0, stream()>>>(n, d_atom_local, lj->d_atom_type, lj->d_local_type);
    SPGNB_CHECK_LAUNCH("k_local_types");
    lj->local_atoms = local_atom_numbers;
    lj->d_atom_local = d_atom_local;
    return SPGNB_OK;
}

int spgnb_lj_pme_direct_force(spgnb_lj* lj, int atom_numbers, int local_atom_numbers, int solvent_numbers,
                              int ghost_numbers, const spgnb_vector* d_crd, const float* d_charge,
                              spgnb_vector* d_frc, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, const spgnb_nl* nl,
                              float pme_beta, int need_atom_energy, float* d_atom_energy, int need_virial,
                              spgnb_ltmatrix3* d_atom_virial, float* d_atom_direct_pme_energy)
{
    (void)atom_numbers;
    int st = check_common(lj, local_atom_numbers, ghost_numbers, d_crd, d_charge, d_frc);
    if (st) return st;
    if (!nl) return fail(SPGNB_E_ARG, "spgnb_lj_pme_direct_force: nl is NULL");
    if (!nl->built) return fail(SPGNB_E_STATE, "spgnb_lj_pme_direct_force: the neighbour list was never built");
    if (local_atom_numbers != nl->local_atoms)
        return fail(SPGNB_E_STATE, "spgnb_lj_pme_direct_force: list built for %d atoms, called with %d",
                    nl->local_atoms, local_atom_numbers);
    if (local_atom_numbers == 0) return SPGNB_OK;
    if (nl->S != 1) return fail(SPGNB_E_STATE, "spgnb_lj_pme_direct_force: the list holds several systems");
    if (memcmp(&cell, &nl->cell, sizeof(cell)) != 0)
        return fail(SPGNB_E_STATE, "spgnb_lj_pme_direct_force: the box differs from the one of the last list "
                                   "update; update the list after a box change");
    cudaStream_t s = stream();
    const int slots = nl->clusters_cap * kClusterSize;
    if ((st = ensure_slots(lj, slots))) return st;
    SPGNB_CUDA(cudaMemsetAsync(lj->d_totals, 0, sizeof(long long) * 8, s));
    if (need_atom_energy)
    {
        SPGNB_CUDA(cudaMemsetAsync(lj->d_lj_energy_atom, 0, sizeof(float) * lj->atom_numbers, s));
        if (d_atom_direct_pme_energy)
            SPGNB_CUDA(cudaMemsetAsync(d_atom_direct_pme_energy, 0, sizeof(float) * lj->atom_numbers, s));
    }
    if ((st = nl_set_prune_rc(const_cast<spgnb_nl*>(nl), lj->cutoff, s))) return st;
    ForceInputs in;
    in.nl = const_cast<spgnb_nl*>(nl);
    in.crd = (const float3*)d_crd;
    in.charge = d_charge;
    in.atom_type = lj->d_local_type;
    in.slot_pos = lj->d_sdata;
    in.slot_type = lj->d_slot_type;
    in.p0 = make_pair_const(lj, pme_beta);
    in.fit = in.p0.use_fit != 0;
    in.table = lj->d_table;
    in.table_size = lj->n_types * lj->n_types;
    in.frc = (float3*)d_frc;
    in.totals = lj->d_totals;
    int mode = 0;
    if (need_atom_energy || need_virial) mode = 1;
    if ((need_atom_energy && (d_atom_energy || d_atom_direct_pme_energy)) || (need_virial && d_atom_virial))
        mode = 2;
    in.mode = mode;
    if (mode == 2)
    {
        in.om.atom_local = lj->d_atom_local;
        in.om.solvent_start = local_atom_numbers - (solvent_numbers > 0 ? solvent_numbers : 0);
        in.om.water_points = 3;
        in.pa.energy = need_atom_energy ? d_atom_energy : nullptr;
        in.pa.lj_energy = need_atom_energy ? lj->d_lj_energy_atom : nullptr;
        in.pa.direct = need_atom_energy ? d_atom_direct_pme_energy : nullptr;
        in.pa.virial = need_virial ? (float*)d_atom_virial : nullptr;
    }
    else
    {
        in.om.solvent_start = local_atom_numbers;
    }
    if (lj->xs_on)
    {
        // PME's excluded-pair correction in the same pass
        in.xf.sn = lj->d_xs_sn;
        in.xf.list = lj->d_xs_list;
        in.xf.crd = in.crd;
        in.xf.charge = d_charge;
        in.xf.atom_local = lj->d_atom_local;
        in.xf.beta = pme_beta;
        in.xf.beta3 = pme_beta * pme_beta * pme_beta;
        in.xf.total = lj->d_excl_total;
        if (mode == 2)
        {
            in.xf.energy = need_atom_energy ? d_atom_energy : nullptr;
            in.xf.virial = need_virial ? (float*)d_atom_virial : nullptr;
        }
        if (mode >= 1) SPGNB_CUDA(cudaMemsetAsync(lj->d_excl_total, 0, sizeof(long long), s));
    }
    if ((st = force_pipeline(in, s))) return st;
    lj->have_energy = need_atom_energy != 0;
    lj->have_virial = need_virial != 0;
    return SPGNB_OK;
}

int spgnb_lj_fuse_pme_excluded(spgnb_lj* lj, int atom_numbers, const int* d_excluded_list_start,
                               const int* d_excluded_list, const int* d_excluded_numbers, int excluded_total)
{
    if (!lj) return fail(SPGNB_E_ARG, "spgnb_lj_fuse_pme_excluded: NULL handle");
    lj->xs_on = false;
    if (atom_numbers <= 0 || !d_excluded_list_start || !d_excluded_list || !d_excluded_numbers) return SPGNB_OK;
    if (atom_numbers > lj->atom_numbers)
        return fail(SPGNB_E_ARG, "spgnb_lj_fuse_pme_excluded: %d atoms, the module holds %d", atom_numbers,
                    lj->atom_numbers);
    if (excluded_total < 0) return fail(SPGNB_E_ARG, "spgnb_lj_fuse_pme_excluded: negative list size");
    const int n = atom_numbers;
    std::vector<int> start(n), num(n), list(std::max(excluded_total, 1));
    cudaStream_t s = stream();
    SPGNB_CUDA(cudaMemcpyAsync(start.data(), d_excluded_list_start, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    SPGNB_CUDA(cudaMemcpyAsync(num.data(), d_excluded_numbers, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    if (excluded_total > 0)
        SPGNB_CUDA(cudaMemcpyAsync(list.data(), d_excluded_list, sizeof(int) * excluded_total, cudaMemcpyDeviceToHost,
                                   s));
    SPGNB_CUDA(cudaStreamSynchronize(s));
    // both directions of every excluded pair, each atom's partners ascending
    std::vector<int> cnt(n, 0);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < num[i]; k++)
        {
            const int e = start[i] + k;
            if (num[i] < 0 || start[i] < 0 || e >= excluded_total)
                return fail(SPGNB_E_ARG, "spgnb_lj_fuse_pme_excluded: atom %d's list runs past the %d entries", i,
                            excluded_total);
            const int j = list[e];
            if (j < 0 || j >= n || j == i)
                return fail(SPGNB_E_ARG, "spgnb_lj_fuse_pme_excluded: atom %d excludes %d", i, j);
            cnt[i]++;
            cnt[j]++;
        }
    std::vector<int> sym_start(n), fill(n);
    int total = 0;
    for (int i = 0; i < n; i++)
    {
        sym_start[i] = total;
        fill[i] = total;
        total += cnt[i];
    }
    std::vector<int> sym(std::max(total, 1));
    for (int i = 0; i < n; i++)
        for (int k = 0; k < num[i]; k++)
        {
            const int j = list[start[i] + k];
            sym[fill[i]++] = j;
            sym[fill[j]++] = i;
        }
    for (int i = 0; i < n; i++) std::sort(sym.begin() + sym_start[i], sym.begin() + sym_start[i] + cnt[i]);
    dfree(lj->d_xs_sn);
    dfree(lj->d_xs_list);
    int st;
    if ((st = dalloc(&lj->d_xs_sn, lj->atom_numbers)) || (st = dalloc(&lj->d_xs_list, sym.size()))) return st;
    std::vector<int2> sn(lj->atom_numbers, make_int2(0, 0));
    for (int i = 0; i < n; i++) sn[i] = make_int2(sym_start[i], cnt[i]);
    SPGNB_CUDA(cudaMemcpyAsync(lj->d_xs_sn, sn.data(), sizeof(int2) * sn.size(), cudaMemcpyHostToDevice, s));
    SPGNB_CUDA(cudaMemcpyAsync(lj->d_xs_list, sym.data(), sizeof(int) * sym.size(), cudaMemcpyHostToDevice, s));
    SPGNB_CUDA(cudaStreamSynchronize(s));
    lj->xs_on = true;
    return SPGNB_OK;
}

int spgnb_lj_pme_direct_force_atom_groups(spgnb_lj* lj, int atom_numbers, int local_atom_numbers,
                                          int solvent_numbers, int ghost_numbers, const spgnb_vector* d_crd,
                                          const float* d_charge, spgnb_vector* d_frc, spgnb_ltmatrix3 cell,
                                          spgnb_ltmatrix3 rcell, const spgnb_atom_group* d_nl, float pme_beta,
                                          int need_atom_energy, float* d_atom_energy, int need_virial,
                                          spgnb_ltmatrix3* d_atom_virial, float* d_atom_direct_pme_energy)
{
    (void)atom_numbers;
    int st = check_common(lj, local_atom_numbers, ghost_numbers, d_crd, d_charge, d_frc);
    if (st) return st;
    if (!d_nl) return fail(SPGNB_E_ARG, "spgnb_lj_pme_direct_force_atom_groups: d_nl is NULL");
    cudaStream_t s = stream();
    if ((st = ensure_pos(lj, lj->atom_numbers))) return st;
    const Cell c = make_cell(cell), rc = make_cell(rcell);
    SPGNB_CUDA(cudaMemsetAsync(lj->d_totals, 0, sizeof(long long) * 8, s));
    if (need_atom_energy)
    {
        SPGNB_CUDA(cudaMemsetAsync(lj->d_lj_energy_atom, 0, sizeof(float) * lj->atom_numbers, s));
        if (d_atom_direct_pme_energy)
            SPGNB_CUDA(cudaMemsetAsync(d_atom_direct_pme_energy, 0, sizeof(float) * lj->atom_numbers, s));
    }
    const int n = local_atom_numbers;
    if (n == 0) return SPGNB_OK;
    k_pack_atoms<<<(n + 255) / 256, 256, 0, s>>>(n, (const float3*)d_crd, d_charge, lj->d_local_type, lj->d_pos,
                                                 lj->d_pos_type);
    SPGNB_CHECK_LAUNCH("k_pack_atoms");
    PairConst pc = make_pair_const(lj, pme_beta);
    PerAtomOut pa{need_atom_energy ? d_atom_energy : nullptr, need_atom_energy ? lj->d_lj_energy_atom : nullptr,
                  need_atom_energy ? d_atom_direct_pme_energy : nullptr, need_virial ? (float*)d_atom_virial : nullptr};
    const int owners = n - (solvent_numbers > 0 ? solvent_numbers : 0);
    const int blocks = std::max(1, std::min((owners + 3) / 4, num_sms() * 8));
    const int mode = (need_atom_energy || need_virial) ? 2 : 0;
    if (owners > 0)
    {
        if (mode == 0)
            k_pair_atom_groups<0><<<blocks, 128, 0, s>>>(pc, c, rc, owners, n, d_nl, lj->d_pos, lj->d_pos_type,
                                                         lj->d_table, lj->d_frc_acc, lj->d_totals, pa);
        else
            k_pair_atom_groups<2><<<blocks, 128, 0, s>>>(pc, c, rc, owners, n, d_nl, lj->d_pos, lj->d_pos_type,
                                                         lj->d_table, lj->d_frc_acc, lj->d_totals, pa);
        SPGNB_CHECK_LAUNCH("k_pair_atom_groups");
    }
    k_finalize<<<(n + 255) / 256, 256, 0, s>>>(n, lj->d_frc_acc, (float3*)d_frc);
    SPGNB_CHECK_LAUNCH("k_finalize");
    lj->have_energy = need_atom_energy != 0;
    lj->have_virial = need_virial != 0;
    return SPGNB_OK;
}

int spgnb_lj_long_range_correction(spgnb_lj* lj, int need_pressure, spgnb_ltmatrix3* d_virial,
                                   int need_potential, float* d_potential, float volume)
{
    if (!lj) return fail(SPGNB_E_ARG, "spgnb_lj_long_range_correction: NULL handle");
    if ((need_pressure && !d_virial) || (need_potential && !d_potential))
        return fail(SPGNB_E_ARG, "spgnb_lj_long_range_correction: NULL output");
    if (!(volume > 0)) return fail(SPGNB_E_ARG, "spgnb_lj_long_range_correction: volume must be positive");
    float f = (float)lj->long_range_factor;
    float vfac = 2 * f / volume;
    float efac = f / volume;
    lj->last_volume = volume;
    if (need_potential) lj->h_last_long_energy = efac;
    k_long_range<<<1, 1, 0, stream()>>>(need_pressure, (float*)d_virial, need_potential, d_potential, vfac, efac);
    SPGNB_CHECK_LAUNCH("k_long_range");
    return SPGNB_OK;
}

int spgnb_lj_pme_excluded_force(spgnb_lj* lj, int atom_numbers, const spgnb_vector* d_crd, spgnb_ltmatrix3 cell,
                                spgnb_ltmatrix3 rcell, const float* d_charge, float pme_beta,
                                const int* d_excluded_list_start, const int* d_excluded_list,
                                const int* d_excluded_numbers, spgnb_vector* d_frc, int need_energy,
                                float* d_atom_energy, spgnb_ltmatrix3* d_atom_virial)
{
    if (!lj) return fail(SPGNB_E_ARG, "spgnb_lj_pme_excluded_force: NULL handle");
    if (atom_numbers < 0 || atom_numbers > lj->atom_numbers)
        return fail(SPGNB_E_ARG, "spgnb_lj_pme_excluded_force: %d atoms, the module holds %d", atom_numbers,
                    lj->atom_numbers);
    if (atom_numbers == 0) return SPGNB_OK;
    if (!d_crd || !d_charge || !d_frc || !d_excluded_list_start || !d_excluded_list || !d_excluded_numbers)
        return fail(SPGNB_E_ARG, "spgnb_lj_pme_excluded_force: NULL device pointer");
    if (need_energy && !d_atom_energy) return fail(SPGNB_E_ARG, "spgnb_lj_pme_excluded_force: NULL atom_energy");
    cudaStream_t s = stream();
    SPGNB_CUDA(cudaMemsetAsync(lj->d_excl_total, 0, sizeof(long long), s));
    const int n = atom_numbers;
    k_pme_excluded<<<(n + 255) / 256, 256, 0, s>>>(n, (const float3*)d_crd, make_cell(cell), make_cell(rcell),
                                                   d_charge, pme_beta, d_excluded_list_start, d_excluded_list,
                                                   d_excluded_numbers, lj->d_frc_acc,
                                                   need_energy ? d_atom_energy : nullptr, (float*)d_atom_virial,
                                                   lj->d_excl_total);
    SPGNB_CHECK_LAUNCH("k_pme_excluded");
    k_finalize<<<(n + 255) / 256, 256, 0, s>>>(n, lj->d_frc_acc, (float3*)d_frc);
    SPGNB_CHECK_LAUNCH("k_finalize");
    return SPGNB_OK;
}

int spgnb_lj_pme_excluded_energy(spgnb_lj* lj, double* energy)
{
    if (!lj || !energy) return fail(SPGNB_E_ARG, "spgnb_lj_pme_excluded_energy: NULL argument");
    long long h = 0;
    SPGNB_CUDA(cudaMemcpyAsync(&h, lj->d_excl_total, sizeof(h), cudaMemcpyDeviceToHost, stream()));
    SPGNB_CUDA(cudaStreamSynchronize(stream()));
    *energy = (double)h / kEnergyScale;
    return SPGNB_OK;
}

int spgnb_lj_totals(spgnb_lj* lj, double out[8])
{
    if (!lj || !out) return fail(SPGNB_E_ARG, "spgnb_lj_totals: NULL argument");
    long long h[8];
    SPGNB_CUDA(cudaMemcpyAsync(h, lj->d_totals, sizeof(h), cudaMemcpyDeviceToHost, stream()));
    SPGNB_CUDA(cudaStreamSynchronize(stream()));
    for (int q = 0; q < 8; q++) out[q] = (double)h[q] / kEnergyScale;
    for (int q = 0; q < 8; q++) lj->totals[q] = out[q];
    return SPGNB_OK;
}

int spgnb_lj_energies(spgnb_lj* lj, double* lj_short, double* lj_long, double* lj_total, double* direct_coulomb)
{
    double t[8];
    int st = spgnb_lj_totals(lj, t);
    if (st) return st;
    if (lj_short) *lj_short = t[0];
    if (lj_long) *lj_long = lj->h_last_long_energy;
    if (lj_total) *lj_total = t[0] + lj->h_last_long_energy;
    if (direct_coulomb) *direct_coulomb = t[1];
    return SPGNB_OK;
}

double spgnb_lj_long_range_factor(const spgnb_lj* lj) { return lj ? lj->long_range_factor : 0.0; }

int spgnb_lj_atom_lj_energy(spgnb_lj* lj, float** d_atom_lj_energy)
{
    if (!lj || !d_atom_lj_energy) return fail(SPGNB_E_ARG, "spgnb_lj_atom_lj_energy: NULL argument");
    *d_atom_lj_energy = lj->d_lj_energy_atom;
    return SPGNB_OK;
}

int spgnb_lj_export_vector_lj(spgnb_lj* lj, const spgnb_vector* d_crd, const float* d_charge, void* d_vector_lj,
                              int n)
{
    if (!lj || !d_crd || !d_charge || !d_vector_lj) return fail(SPGNB_E_ARG, "spgnb_lj_export_vector_lj: NULL argument");
    if (!lj->d_local_type) return fail(SPGNB_E_STATE, "spgnb_lj_export_vector_lj: Get_Local has not been called");
    if (n <= 0) return SPGNB_OK;
    if (n > lj->atom_numbers) return fail(SPGNB_E_ARG, "spgnb_lj_export_vector_lj: n exceeds the module's atoms");
    k_vector_lj<<<(n + 255) / 256, 256, 0, stream()>>>(n, (const float3*)d_crd, d_charge, lj->d_local_type,
                                                       (float*)d_vector_lj);
    SPGNB_CHECK_LAUNCH("k_vector_lj");
    return SPGNB_OK;
}

int spgnb_lj_destroy(spgnb_lj* lj)
{
    if (!lj) return SPGNB_OK;
    dfree(lj->d_atom_type);
    dfree(lj->d_local_type);
    dfree(lj->d_table);
    dfree(lj->d_lj_energy_atom);
    dfree(lj->d_frc_acc);
    dfree(lj->d_totals);
    dfree(lj->d_excl_total);
    dfree(lj->d_xs_sn);
    dfree(lj->d_xs_list);
    dfree(lj->d_pos);
    dfree(lj->d_pos_type);
    dfree(lj->d_sdata);
    dfree(lj->d_slot_type);
    delete lj;
    return SPGNB_OK;
}

// ----------------------------------------------------- SOLVENT_LENNARD_JONES
int spgnb_solvent_create(spgnb_lj* lj, int water_points, spgnb_solvent** out)
{
    if (!out || !lj) return fail(SPGNB_E_ARG, "spgnb_solvent_create: NULL argument");
    *out = nullptr;
    if (water_points != 3 && water_points != 4)
        return fail(SPGNB_E_ARG, "spgnb_solvent_create: water_points must be 3 or 4");
    spgnb_solvent* s = new spgnb_solvent();
    s->lj = lj;
    s->water_points = water_points;
    int st = dalloc(&s->d_scratch, 2);
    if (st)
    {
        delete s;
        return st;
    }
    *out = s;
    return SPGNB_OK;
}

int spgnb_solvent_get_local(spgnb_solvent* s, int local_res_numbers, const int* d_res_len, int atom_numbers,
                            const float* d_mass, int* local_solvent_numbers)
{
    if (!s || !d_res_len || !d_mass) return fail(SPGNB_E_ARG, "spgnb_solvent_get_local: NULL argument");
    k_solvent_count<<<1, 1, 0, stream()>>>(local_res_numbers, d_res_len, s->water_points, atom_numbers, d_mass,
                                           s->d_scratch);
    SPGNB_CHECK_LAUNCH("k_solvent_count");
    int h[2];
    SPGNB_CUDA(cudaMemcpyAsync(h, s->d_scratch, sizeof(h), cudaMemcpyDeviceToHost, stream()));
    SPGNB_CUDA(cudaStreamSynchronize(stream()));
    s->solvent_start_local = h[0];
    s->local_solvent_numbers = h[1];
    if (local_solvent_numbers) *local_solvent_numbers = h[1];
    return SPGNB_OK;
}

int spgnb_solvent_pme_direct_force(spgnb_solvent* sv, int atom_numbers, int residue_numbers,
                                   const int* d_res_start, const spgnb_vector* d_crd, const float* d_charge,
                                   spgnb_vector* d_frc, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                                   const spgnb_nl* nl, const spgnb_atom_group* d_nl, float pme_beta,
                                   int need_atom_energy, float* d_atom_energy, int need_virial,
                                   spgnb_ltmatrix3* d_atom_virial, float* d_atom_direct_pme_energy)
{
    (void)d_charge;
    if (!sv) return fail(SPGNB_E_ARG, "spgnb_solvent_pme_direct_force: NULL handle");
    if (nl) return SPGNB_OK;  // evaluated by spgnb_lj_pme_direct_force over the spgnb list
    if (!d_nl || !d_res_start || !d_crd || !d_frc)
        return fail(SPGNB_E_ARG, "spgnb_solvent_pme_direct_force: NULL device pointer");
    spgnb_lj* lj = sv->lj;
    if (residue_numbers <= sv->solvent_start_local || sv->local_solvent_numbers == 0) return SPGNB_OK;
    // positions were packed per atom by spgnb_lj_pme_direct_force_atom_groups of this step
    if (lj->pos_cap < atom_numbers)
        return fail(SPGNB_E_STATE, "solvent module: call the LJ module's force first (it packs the coordinates)");
    cudaStream_t s = stream();
    // the LJ call already converted and cleared its accumulators; reuse them
    PairConst pc = make_pair_const(lj, pme_beta);
    PerAtomOut pa{need_atom_energy ? d_atom_energy : nullptr, need_atom_energy ? lj->d_lj_energy_atom : nullptr,
                  need_atom_energy ? d_atom_direct_pme_energy : nullptr, need_virial ? (float*)d_atom_virial : nullptr};
    const Cell c = make_cell(cell), rc = make_cell(rcell);
    const int nres = residue_numbers - sv->solvent_start_local;
    const int blocks = std::max(1, std::min((nres + 3) / 4, num_sms() * 8));
    const bool en = need_atom_energy || need_virial;
    if (sv->water_points == 3)
    {
        if (en)
            k_pair_solvent<2, 3><<<blocks, 128, 0, s>>>(pc, c, rc, sv->solvent_start_local, residue_numbers,
                                                        atom_numbers, d_res_start, d_nl, lj->d_pos, lj->d_pos_type,
                                                        lj->d_table, lj->d_frc_acc, lj->d_totals, pa);
        else
            k_pair_solvent<0, 3><<<blocks, 128, 0, s>>>(pc, c, rc, sv->solvent_start_local, residue_numbers,
                                                        atom_numbers, d_res_start, d_nl, lj->d_pos, lj->d_pos_type,
                                                        lj->d_table, lj->d_frc_acc, lj->d_totals, pa);
    }
    else
    {
        if (en)
            k_pair_solvent<2, 4><<<blocks, 128, 0, s>>>(pc, c, rc, sv->solvent_start_local, residue_numbers,
                                                        atom_numbers, d_res_start, d_nl, lj->d_pos, lj->d_pos_type,
                                                        lj->d_table, lj->d_frc_acc, lj->d_totals, pa);
        else
            k_pair_solvent<0, 4><<<blocks, 128, 0, s>>>(pc, c, rc, sv->solvent_start_local, residue_numbers,
                                                        atom_numbers, d_res_start, d_nl, lj->d_pos, lj->d_pos_type,
                                                        lj->d_table, lj->d_frc_acc, lj->d_totals, pa);
    }
    SPGNB_CHECK_LAUNCH("k_pair_solvent");
    k_finalize<<<(atom_numbers + 255) / 256, 256, 0, s>>>(atom_numbers, lj->d_frc_acc, (float3*)d_frc);
    SPGNB_CHECK_LAUNCH("k_finalize");
    return SPGNB_OK;
}

int spgnb_solvent_destroy(spgnb_solvent* s)
{
    if (!s) return SPGNB_OK;
    dfree(s->d_scratch);
    delete s;
    return SPGNB_OK;
}

}  // extern "C"
