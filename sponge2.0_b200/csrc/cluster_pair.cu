// Short-range force over the cluster lists: the per-step slot pack, the
// pruning of the neighbour tables into per-cluster partner lists, the
// cluster-pair force kernel and its finishing pass.  Together they are the
// B200 form of Lennard_Jones_And_Direct_Coulomb_Device and its dispatcher
// (SPONGE/Lennard_Jones_force/Lennard_Jones_force.cpp:43-136, 359-417) and of
// the solvent kernel (solvent_LJ.cpp:25-145), which evaluate the same pairs.
//
// List layout.  A cluster is 8 slots.  Each cluster I has one partner list:
// 32-bit words {partner slot - system's first slot (22 bits) | mask of the
// cluster's atoms the partner pairs with (8 bits) << 22 | image flag << 30}.
// A word's partner is evaluated against all eight atoms of I at once, so the
// partner's gathers and the word's decoding are paid once per eight pairs.
// The list holds partners in clusters J > I, and in I itself the pairs
// a < b: every pair once (a half list), the partner's share of each pair
// scattered by int64 atomics.  Words are kept when the partner lies within
// rc + buffer of one of the atoms at the last pruning, and a pruning is
// redone when an atom has moved half the buffer since, so no pair within rc
// is ever missing.
#include <math.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "pairfn.cuh"

namespace spgnb
{
namespace
{

constexpr int kPruneWarps = 8;
constexpr int kWindow = 32;                        // list parts are padded to whole 32-word windows
constexpr unsigned kWordSlotMask = (1u << 22) - 1u; // partner slot field of a list word
constexpr int kWordMaskShift = 22;                  // the 8-bit atom mask
constexpr unsigned kWordImage = 1u << 30;           // the pair needs its own periodic image
constexpr int kPairWarps = 4;                       // warps per block of the force kernel

// Per-step slot pack: each slot's offset from the build-time cluster centre
// moved by the displacement since the build (minimum image in the system's
// box, so a caller that wraps coordinates between builds is fine), with the
// charge; and the slot's aux record {cluster centre x | LJ type << 22, centre
// y, centre z, global index}, the 22-bit centre the force kernel takes
// differences of (its high bits are masked off there).  Slot slots_cap is a
// null slot: 10^4 A away from everything, charge 0.  With pruning on (pref
// set) the kernel also flags a re-pruning when some atom moved more than half
// the prune buffer since the last one.  It also clears the outputs the force
// call must start from zero (totals, module-owned per-atom energies).  With
// a gate it runs only when *gate is non-zero (after a rebuild, in the
// batched step).
__global__ void k_pack_slots(int slots_cap, int* counters, const int* __restrict__ slot_atom,
                             const int* __restrict__ slot_gid, const int* __restrict__ cl_sys,
                             const SysDesc* __restrict__ sys, const int4* __restrict__ cl_q,
                             const float4* __restrict__ x0, const float4* __restrict__ d0,
                             const float3* __restrict__ crd, const float* __restrict__ charge,
                             const int* __restrict__ local_type, float4* __restrict__ pos, int4* __restrict__ aux,
                             const float4* __restrict__ pref, float half_buffer2, int* __restrict__ prune,
                             long long* __restrict__ clear_totals, long long* __restrict__ clear_one,
                             float* __restrict__ clear_a, float* __restrict__ clear_b, int clear_n,
                             const int* __restrict__ gate)
{
    grid_dep_wait();
    if (gate && *gate == 0) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    // the outputs the force call zeroes first
    if (clear_totals && s < 8) clear_totals[s] = 0;
    if (clear_one && s == 0) *clear_one = 0;
    for (int k = s; k < clear_n; k += gridDim.x * blockDim.x)
    {
        if (clear_a) clear_a[k] = 0.0f;
        if (clear_b) clear_b[k] = 0.0f;
    }
    if (s == slots_cap)
    {
        pos[s] = make_float4(1.0e4f, 1.0e4f, 1.0e4f, 0.0f);
        aux[s] = make_int4(0, 0, 0, -1);
    }
    else if (s < slots_cap)
    {
        const int a = slot_atom[s];
        const float4 d = d0[s];
        const int4 q = cl_q[s >> 3];
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
        aux[s] = make_int4((q.x & 0x3fffff) | (t << 22), q.y, q.z, a >= 0 ? slot_gid[s] : -1);
    }
    if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) counters[kCntPrune] = 1;
}

// Pruning (no reference counterpart; results unchanged).  Runs after every
// rebuild and whenever some atom of a system moved more than buffer/2 since
// its last one (the pack kernel checks).  One warp per cluster I walks the
// elements of its neighbour table with J >= I (a table built one-sided holds
// no others), expands the union of the eight atoms' mask rows 32 elements at
// a time into shared memory, loads each candidate partner once, tests it
// against all eight atoms without branches (packed FP32x2, two atoms an
// instruction) and writes one word per partner within cutoff + buffer of any
// of them, in table order, padded to a whole window with words whose mask is
// empty.  The last block to finish clears the flags.
__global__ void __launch_bounds__(kPruneWarps * 32)
    k_prune8(ForceParams p0, const ForceParams* __restrict__ fps, float buffer, int* counters, int clusters_cap,
             int table_cap, int list_cap, const int* __restrict__ cl_sys, const SysDesc* __restrict__ sys,
             const int* __restrict__ tcount, const float4* __restrict__ tab, const uint2* __restrict__ tmask,
             const float4* __restrict__ pos, float4* __restrict__ pref, int* __restrict__ lcount,
             unsigned* __restrict__ words, int n_sys, int* __restrict__ prune)
{
    grid_dep_wait();
    if (counters[kCntPrune] == 0) return;
    // a chunk's candidates {partner slot | image flag, element lane | own-atom bits << 5}
    __shared__ uint2 buf[kPruneWarps][kChunk * kClusterSize];
    __shared__ float4 own_all[kPruneWarps][kClusterSize];
    // the cluster's atoms negated, per coordinate, as four {even, odd} float2
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
    const unsigned below = (1u << lane) - 1u;
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
        unsigned* __restrict__ wc = words + (size_t)c * list_cap;
        const int usable = list_cap - kWindow;  // room left for the padding
        int kh = 0;
        for (int t0 = 0; t0 < T; t0 += 32)
        {
            const int t = t0 + lane;
            uint2 mm = make_uint2(0u, 0u);
            float4 e = make_float4(0, 0, 0, 0);
            if (t < T)
            {
                e = tb[t];
                mm = tm[t];
                // clusters below I hold the other side of its pairs
                if (((__float_as_int(e.w) & 0x3fffffff) >> 3) < c) mm = make_uint2(0u, 0u);
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
            const unsigned flag = (eb & (1 << 30)) ? 0x80000000u : 0u;
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
            // a lane's candidate of an iteration: its record and own-atom
            // bits; the partner's position is loaded an iteration ahead
            auto candidate = [&](int q, uint2& wv, unsigned& am, float4& pj) {
                wv = mybuf[q < total ? q : 0];
                am = q < total ? (wv.y >> 5) & 0xffu : 0u;
                pj = make_float4(0, 0, 0, 0);
                if (am) pj = pos[wv.x & 0x7fffffffu];
            };
            uint2 wv_next;
            unsigned am_next;
            float4 pj_next;
            candidate(lane, wv_next, am_next, pj_next);
            for (int q0 = 0; q0 < total; q0 += 32)
            {
                const uint2 wv = wv_next;
                const unsigned am = am_next;
                const float4 pj = pj_next;
                if (q0 + 32 < total) candidate(q0 + 32 + lane, wv_next, am_next, pj_next);
                // the element's centre difference, staged by the lane that read it
                const float4 es = ent[wv.y & 31u];
                const float ex = es.x, ey = es.y, ez = es.z;
                const int js = (int)(wv.x & 0x7fffffffu);
                const bool img = (wv.x & 0x80000000u) != 0;
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
                // partners in later clusters pair with every atom they reach;
                // within the cluster only the pairs a < b
                if ((js >> 3) == c) hit &= (1u << (js & 7)) - 1u;
                const unsigned wb = ((unsigned)js - slot0) | (img ? kWordImage : 0u);
                const unsigned mh = __ballot_sync(0xffffffffu, hit != 0u);
                const int kh_next = kh + __popc(mh);
                if (kh_next <= usable)
                {
                    if (hit) wc[kh + __popc(mh & below)] = wb | (hit << kWordMaskShift);
                }
                else if (lane == 0)
                    atomicOr(&counters[kCntOverflow], kOvfWords);
                kh = kh_next;
            }
            __syncwarp();
        }
        // an overflowed cluster keeps no list (the flag makes the caller regrow
        // and rebuild); otherwise pad it to a whole window
        if (kh > usable) kh = 0;
        const int hp = (kh + kWindow - 1) & ~(kWindow - 1);
        const unsigned null_word = (unsigned)s0 - slot0;
        for (int k2 = kh + lane; k2 < hp; k2 += 32) wc[k2] = null_word;
        if (lane == 0)
        {
            lcount[s0] = hp;
            atomicAdd(&kept_total, (unsigned long long)kh);
        }
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

// Cluster-pair force kernel.  A warp takes clusters from a counter and walks
// the cluster's list, one word per lane per iteration; the partner's offset
// {delta + displacement, q} and aux record {22-bit centre, LJ type, global
// index} load once for all of the cluster's atoms the lane holds, and
//   dr = (c_J - c_I) * cell / 2^22 + p_j - p_i
// is formed with the exact integer centre difference.  The cluster's atoms
// are staged in shared memory as packed pairs, so every instruction of the
// pair function serves two pairs (FP32x2) and the registers stay few enough
// for 6 resident blocks per SM (5 with energy/virial totals, 3 with per-atom
// outputs).  The LJ coefficients of a pair of cluster atoms
// against the partner's type come as one float4 {-A_a, -A_b, B_a, B_b} of
// the T^3 table.  Partner records are copied into shared memory by
// asynchronous copies (cp.async) one iteration ahead of their use, list words
// two, so their latency overlaps the pair arithmetic.
//
// Each pair is evaluated once; a lane holds all 8 atoms, the partner's force
// (summed over the 8 in a fixed order) goes to its int64 fixed-point
// accumulator by one atomic add per component and word, and the cluster's
// forces are summed over the lanes as int64 and added the same way.  Integer
// addition does not depend on order, so the forces are bitwise reproducible;
// the finishing pass converts them.
//
// MODE 0: forces.  MODE 1: + energy and virial totals.  MODE 2: + per-atom
// energy and virial: a pair's terms belong to its owner, the atom with the
// lower global index, as the reference's half list credits them (water
// sites hand theirs to the residue's first atom, as SOLVENT_LENNARD_JONES
// does).  Cluster-owned sums stay in registers over the list; a word's
// partner-owned sums go to the partner's int64 staging, 8 atomic adds; the
// finishing pass turns the staging into the per-atom arrays and totals.
template <int MODE, int FIT, bool TRI>
__global__ void __launch_bounds__(kPairWarps * 32, MODE == 2 ? 3 : (MODE == 1 ? 5 : 7))
    k_pair8(ForceParams p0, const ForceParams* __restrict__ fps, const SysDesc* __restrict__ sys, int n_clusters,
            int list_cap, const int* __restrict__ cl_sys, const int* __restrict__ lcount,
            const unsigned* __restrict__ words, const int4* __restrict__ cl_q, const float4* __restrict__ pos,
            const int4* __restrict__ aux, const float4* __restrict__ t4, long long* __restrict__ facc,
            long long* __restrict__ oacc, long long* __restrict__ totals, const int* __restrict__ only,
            int* __restrict__ counters, int max_types)
{
    grid_dep_wait();
    constexpr bool EN = MODE >= 1;
    constexpr bool PA = MODE >= 2;
    constexpr int NP = 4;        // the cluster's 8 atoms as packed pairs
    __shared__ long long red[kPairWarps][8];  // per-warp fixed-point totals
    __shared__ int is_last;
    extern __shared__ float4 rows_all[];      // per warp: 4 x max_types coefficient rows
    __shared__ unsigned wring_all[kPairWarps][3][32];       // per warp: list words in flight
    // per warp: the cluster's atom pairs {-x, -y | -z, q} and global indices
    __shared__ float4 iat_all[kPairWarps][4][2];
    __shared__ int2 igid_all[kPairWarps][4];
    __shared__ __align__(16) float4 jpos_all[kPairWarps][2][32];  // partner offsets and charges in flight
    __shared__ __align__(16) int4 jaux_all[kPairWarps][2][32];    // partner aux records in flight
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    float4* __restrict__ rows = rows_all + w * 4 * max_types;
    unsigned(&wring)[3][32] = wring_all[w];
    float4(&iat)[4][2] = iat_all[w];
    int2(&igid)[4] = igid_all[w];
    float4(&jpos)[2][32] = jpos_all[w];
    int4(&jaux)[2][32] = jaux_all[w];
    if (EN && lane < 8) red[w][lane] = 0;
    __syncwarp();
    int cur_sys = -1;  // the system red[w] accumulates for
    for (;;)
    {
        int c = 0;
        if (lane == 0) c = atomicAdd(&counters[kCntPairNext], 1);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= n_clusters) break;
        const int s0 = c * kClusterSize;
        const int total = lcount[s0];  // a multiple of the window
        if (total == 0) continue;
        const int sy = cl_sys[c];
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
        const int4 ci = cl_q[c];
        const int nt = P.n_types;
        // the cluster's atoms, negated, as packed pairs
        __syncwarp();  // the previous cluster's atoms are no longer read
        if (lane < 4)
        {
            const int a = 2 * lane;
            const float4 u0 = pos[s0 + a], u1 = pos[s0 + a + 1];
            iat[lane][0] = make_float4(-u0.x, -u1.x, -u0.y, -u1.y);
            iat[lane][1] = make_float4(-u0.z, -u1.z, u0.w, u1.w);
            igid[lane] = make_int2(aux[s0 + a].w, aux[s0 + a + 1].w);
        }
        __syncwarp();
        // the coefficient rows of the cluster's four atom pairs against every
        // partner type, {-A_a, -A_b, B_a, B_b}, staged in shared memory
        {
            int rq[4];
#pragma unroll
            for (int q = 0; q < 4; q++)
                rq[q] = P.t4_begin + (((aux[s0 + 2 * q].x >> 22) & 0x7f) * nt + ((aux[s0 + 2 * q + 1].x >> 22) & 0x7f)) * nt;
            __syncwarp();  // the previous cluster's rows are no longer read
            for (int e = lane; e < 4 * nt; e += 32)
            {
                const int q = e / nt;
                const int r = q == 0 ? rq[0] : (q == 1 ? rq[1] : (q == 2 ? rq[2] : rq[3]));
                rows[e] = __ldg(t4 + r + (e - q * nt));
            }
            __syncwarp();
        }
        float2 fx[NP], fy[NP], fz[NP];
#pragma unroll
        for (int p = 0; p < NP; p++) fx[p] = fy[p] = fz[p] = f2(0.0f);
        float2 acc[(EN && !PA) ? 8 : 1];
#pragma unroll
        for (int q = 0; q < ((EN && !PA) ? 8 : 1); q++) acc[q] = f2(0.0f);
        float2 own[PA ? NP : 1][PA ? 8 : 1];
#pragma unroll
        for (int p = 0; p < (PA ? NP : 1); p++)
#pragma unroll
            for (int q = 0; q < (PA ? 8 : 1); q++) own[p][q] = f2(0.0f);

        const unsigned* __restrict__ wb = words + (size_t)c * list_cap;
        // a three-deep ring of list words and a two-deep ring of partner
        // records in shared memory, filled by asynchronous copies: a lane
        // only ever reads what it copied itself, so no warp barrier is needed
        auto stage_word = [&](int it) {
            if (it * 32 < total) cp_async(&wring[it % 3][lane], wb + it * 32 + lane, 4);
            cp_async_commit();
        };
        auto stage_partner = [&](int it, unsigned w) {
            if (it * 32 < total)
            {
                const int j = slot0 + (int)(w & kWordSlotMask);
                cp_async(&jpos[it & 1][lane], pos + j, 16);
                cp_async(&jaux[it & 1][lane], aux + j, 16);
            }
            cp_async_commit();
        };
        const int iters = total / 32;
        stage_word(0);
        stage_word(1);
        cp_async_wait_prior();
        unsigned wc = wring[0][lane];
        stage_partner(0, wc);
#pragma unroll 1
        for (int it = 0; it < iters; it++)
        {
            // in flight, oldest first: word it+1, partner it, then word it+2
            stage_word(it + 2);
            cp_async_wait_prior();
            const unsigned wn = wring[(it + 1) % 3][lane];
            const float4 pjc = jpos[it & 1][lane];
            const int4 xjc = jaux[it & 1][lane];
            const int jc = slot0 + (int)(wc & kWordSlotMask);
            stage_partner(it + 1, wn);

            const unsigned mi = (wc >> kWordMaskShift) & 0xffu;
            const float ux = centre_step(xjc.x, ci.x), uy = centre_step(xjc.y, ci.y), uz = centre_step(xjc.z, ci.z);
            // the partner in the frame of the cluster's centre
            float sx = __fmaf_rn(ux, qc.a11, pjc.x);
            float sy2 = __fmaf_rn(uy, qc.a22, pjc.y);
            const float sz = __fmaf_rn(uz, qc.a33, pjc.z);
            if (TRI)
            {
                sx = __fmaf_rn(uy, qc.a21, sx);
                sx = __fmaf_rn(uz, qc.a31, sx);
                sy2 = __fmaf_rn(uz, qc.a32, sy2);
            }
            const bool img = (wc & kWordImage) != 0u;
            const bool any_img = __any_sync(0xffffffffu, img);
            const int tj = (xjc.x >> 22) & 0x7f;
            const int gj = xjc.w;
            const float2 qj = f2(pjc.w);
            float2 hx = f2(0.0f), hy = f2(0.0f), hz = f2(0.0f);  // the partner's force, negated
            float2 jo[PA ? 8 : 1];                                  // the partner's owned sums
#pragma unroll
            for (int q = 0; q < (PA ? 8 : 1); q++) jo[q] = f2(0.0f);
#pragma unroll
            for (int p = 0; p < NP; p++)
            {
                const float4 A = iat[p][0], B = iat[p][1];
                const float2 pnx = make_float2(A.x, A.y), pny = make_float2(A.z, A.w), pnz = make_float2(B.x, B.y),
                             pq = make_float2(B.z, B.w);
                float2 dx = __fadd2_rn(f2(sx), pnx), dy = __fadd2_rn(f2(sy2), pny), dz = __fadd2_rn(f2(sz), pnz);
                if (any_img && img)
                {
                    // small box: the pair takes its own minimum image
                    float ddx[2] = {dx.x, dx.y}, ddy[2] = {dy.x, dy.y}, ddz[2] = {dz.x, dz.y};
#pragma unroll
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
                const bool inA = ((mi >> (2 * p)) & 1u) && r2.x < pp.rc2;
                const bool inB = ((mi >> (2 * p + 1)) & 1u) && r2.y < pp.rc2;
                const float4 ab = rows[p * nt + tj];
                float2 elj, ec;
                float2 f = pair_scalar2<EN, FIT>(r2, __fmul2_rn(qj, pq), make_float2(ab.x, ab.y),
                                                 make_float2(ab.z, ab.w), pp, elj, ec);
                f = make_float2(inA ? f.x : 0.0f, inB ? f.y : 0.0f);
                const float2 gx = __fmul2_rn(f, dx), gy = __fmul2_rn(f, dy), gz = __fmul2_rn(f, dz);
                fx[p] = __fadd2_rn(fx[p], gx);
                fy[p] = __fadd2_rn(fy[p], gy);
                fz[p] = __fadd2_rn(fz[p], gz);
                hx = __fadd2_rn(hx, gx);
                hy = __fadd2_rn(hy, gy);
                hz = __fadd2_rn(hz, gz);
                if (EN && !PA)
                {
                    acc[0] = __fadd2_rn(acc[0], make_float2(inA ? elj.x : 0.0f, inB ? elj.y : 0.0f));
                    acc[1] = __fadd2_rn(acc[1], make_float2(inA ? ec.x : 0.0f, inB ? ec.y : 0.0f));
                    acc[2] = __ffma2_rn(gx, dx, acc[2]);
                    acc[3] = __ffma2_rn(gx, dy, acc[3]);
                    acc[4] = __ffma2_rn(gy, dy, acc[4]);
                    acc[5] = __ffma2_rn(gx, dz, acc[5]);
                    acc[6] = __ffma2_rn(gy, dz, acc[6]);
                    acc[7] = __ffma2_rn(gz, dz, acc[7]);
                }
                if (PA)
                {
                    // the pair's owner is the lower global index: this lane's
                    // atom (kept over the list) or the partner (summed over
                    // the word's atoms)
                    const int2 pg = igid[p];
                    const float2 wi = make_float2(pg.x < gj ? 1.0f : 0.0f, pg.y < gj ? 1.0f : 0.0f);
                    const float2 v[8] = {make_float2(inA ? elj.x : 0.0f, inB ? elj.y : 0.0f),
                                         make_float2(inA ? ec.x : 0.0f, inB ? ec.y : 0.0f),
                                         __fmul2_rn(gx, dx), __fmul2_rn(gx, dy), __fmul2_rn(gy, dy),
                                         __fmul2_rn(gx, dz), __fmul2_rn(gy, dz), __fmul2_rn(gz, dz)};
#pragma unroll
                    for (int q = 0; q < 8; q++) own[p][q] = __ffma2_rn(v[q], wi, own[p][q]);
                    const float2 wj = __fadd2_rn(f2(1.0f), __fmul2_rn(wi, kPk[kPkMinusOne]));
#pragma unroll
                    for (int q = 0; q < 8; q++) jo[q] = __ffma2_rn(v[q], wj, jo[q]);
                }
            }
            if (PA)
            {
                // the partner's owned sums over this word: raw fixed point to
                // its staging (scaled in the finishing pass), one quantity
                // after another so that a warp's adds fall on few lines
                float js[8];
                bool any = false;
#pragma unroll
                for (int q = 0; q < 8; q++)
                {
                    js[q] = jo[q].x + jo[q].y;
                    any |= js[q] != 0.0f;
                }
                if (any)
                {
                    unsigned long long* oa = (unsigned long long*)(oacc + jc);
                    const size_t ostride = (size_t)n_clusters * kClusterSize;
#pragma unroll
                    for (int q = 0; q < 8; q++)
                    {
                        const long long v = __float2ll_rn(js[q] * kTwoPow32);
                        if (v) atomicAdd(oa + q * ostride, (unsigned long long)v);
                    }
                }
            }
            {
                // the partner's force: minus the sum over the cluster's atoms
                const long long qx = __float2ll_rn(-(hx.x + hx.y) * kTwoPow32);
                const long long qy = __float2ll_rn(-(hy.x + hy.y) * kTwoPow32);
                const long long qz = __float2ll_rn(-(hz.x + hz.y) * kTwoPow32);
                unsigned long long* fa = (unsigned long long*)(facc + 3 * (size_t)jc);
                if (qx) atomicAdd(fa + 0, (unsigned long long)qx);
                if (qy) atomicAdd(fa + 1, (unsigned long long)qy);
                if (qz) atomicAdd(fa + 2, (unsigned long long)qz);
            }
            wc = wn;
        }
        cp_async_wait_all();

        // the cluster's forces: int64 per lane, summed over the lanes by a
        // reduce-scatter (lanes 4a..4a+3 end with atom a)
        long long vx[8], vy[8], vz[8];
#pragma unroll
        for (int a = 0; a < 8; a++)
        {
            const int p = a / 2;
            const float sxv = (a & 1) ? fx[p].y : fx[p].x, syv = (a & 1) ? fy[p].y : fy[p].x,
                        szv = (a & 1) ? fz[p].y : fz[p].x;
            vx[a] = __float2ll_rn(sxv * kTwoPow32);
            vy[a] = __float2ll_rn(syv * kTwoPow32);
            vz[a] = __float2ll_rn(szv * kTwoPow32);
        }
        const long long Fx = reduce_scatter8(vx, lane), Fy = reduce_scatter8(vy, lane),
                        Fz = reduce_scatter8(vz, lane);
        const int va = lane >> 2;
        if ((lane & 3) == 0)
        {
            unsigned long long* fa = (unsigned long long*)(facc + 3 * (size_t)(s0 + va));
            if (Fx) atomicAdd(fa + 0, (unsigned long long)Fx);
            if (Fy) atomicAdd(fa + 1, (unsigned long long)Fy);
            if (Fz) atomicAdd(fa + 2, (unsigned long long)Fz);
        }
        if (EN && !PA)
        {
            float ev[8];
#pragma unroll
            for (int q = 0; q < 8; q++) ev[q] = acc[q].x + acc[q].y;
            const float esum = reduce_scatter8(ev, lane);
            if ((lane & 3) == 0)
            {
                // each pair once; the virial is -g (x) d, its symmetric
                // off-diagonal terms (xy + yx etc.) twice the one accumulated
                const double sc = va == 0 ? (double)kLjEnergyScale
                                          : (va == 1 ? 1.0 : ((va == 3 || va == 5 || va == 6) ? -2.0 : -1.0));
                red[w][va] += __double2ll_rn((double)esum * sc * kEnergyScale);
            }
        }
        if (PA)
        {
            // the cluster's owned sums: raw fixed point to each atom's
            // staging (scaled in the finishing pass)
#pragma unroll
            for (int a = 0; a < 8; a++)
            {
                const int p = a / 2;
                float v[8];
#pragma unroll
                for (int q = 0; q < 8; q++) v[q] = (a & 1) ? own[p][q].y : own[p][q].x;
                // lanes 4q..4q+3 end with value q of atom a
                const float val = reduce_scatter8(v, lane);
                const long long r = __float2ll_rn(val * kTwoPow32);
                if ((lane & 3) == 0 && r)
                    atomicAdd((unsigned long long*)(oacc + (size_t)va * n_clusters * kClusterSize + (s0 + a)),
                              (unsigned long long)r);
            }
        }
    }
    __syncwarp();
    if (EN && lane == 0 && cur_sys >= 0)
        for (int q = 0; q < 8; q++)
        {
            const long long v = red[w][q];
            if (v) atomicAdd((unsigned long long*)&totals[8 * cur_sys + q], (unsigned long long)v);
        }
    // the last block resets the cluster counter for the next launch
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        is_last = atomicAdd(&counters[kCntPairDone], 1) == gridDim.x - 1;
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0)
    {
        counters[kCntPairNext] = 0;
        counters[kCntPairDone] = 0;
    }
}

// The fused PME excluded-pair correction of atom a
// (Particle_Mesh::PME_Excluded_Force_With_Atom_Energy, PM_force.cpp:918-997):
// its symmetric exclusion list holds both sides of every pair, so each atom
// computes its own share, F_a += q_a q_x beta^3 h(beta r) dr with dr = the
// reference's minimum image of r_x - r_a, and the pair's owner (lower global
// index) adds -q_a q_x erf(beta r)/r to the energy and -F (x) dr to its
// virial (wv: xx, xy, yy, xz, yz, zz).
template <bool EN>
__device__ __forceinline__ void excl_terms(int a, const SysDesc& D, const ExclFuse& xf, float& fx, float& fy,
                                           float& fz, float& eown, float (&wv)[6])
{
    const int2 sn = xf.sn[a];
    const float3 ri = xf.crd[a];
    const float qa = xf.charge[a];
    const int ga = xf.atom_local[a];
    for (int k = 0; k < sn.y; k++)
    {
        const int jx = xf.list[sn.x + k];
        const float3 rj = xf.crd[jx];
        float ex = rj.x - ri.x, ey = rj.y - ri.y, ez = rj.z - ri.z;
        const float tx = floorf(ex * D.rcell.a11 + ey * D.rcell.a21 + ez * D.rcell.a31 + 0.5f);
        const float ty = floorf(ey * D.rcell.a22 + ez * D.rcell.a32 + 0.5f);
        const float tz = floorf(ez * D.rcell.a33 + 0.5f);
        ex -= tx * D.cell.a11 + ty * D.cell.a21 + tz * D.cell.a31;
        ey -= ty * D.cell.a22 + tz * D.cell.a32;
        ez -= tz * D.cell.a33;
        const float er = sqrtf(ex * ex + ey * ey + ez * ez);
        const float xb = xf.beta * er;
        const float qq = qa * xf.charge[jx];
        const float fa = qq * xf.beta3 * excl_h(xb);
        const float gx = fa * ex, gy = fa * ey, gz = fa * ez;
        fx += gx;
        fy += gy;
        fz += gz;
        if (EN && ga < xf.atom_local[jx])
        {
            eown -= qq * erff(xb) / er;
            wv[0] -= gx * ex;
            wv[1] -= gx * ey + gy * ex;
            wv[2] -= gy * ey;
            wv[3] -= gx * ez + gz * ex;
            wv[4] -= gy * ez + gz * ey;
            wv[5] -= gz * ez;
        }
    }
}

// Finishing pass of the force and totals modes, one thread per slot: the
// half-list kernel's int64 force sums go to the caller's float array, the
// staging cleared for the next call; with EXCL each atom also adds its
// excluded pairs' correction (and, with EN, its owned energy to the total).
// A thread touches only its own atom's force.
template <bool EXCL, bool EN>
__global__ void k_fin8(int slots, const int* __restrict__ slot_atom, const int* __restrict__ cl_sys,
                       const SysDesc* __restrict__ sys, long long* __restrict__ facc, float3* __restrict__ frc,
                       ExclFuse xf)
{
    grid_dep_wait();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    float ene = 0.0f;
    if (s < slots)
    {
        const int a = slot_atom[s];
        long long* q = facc + 3 * (size_t)s;
        const long long x = q[0], y = q[1], z = q[2];
        if (x | y | z)
        {
            q[0] = 0;
            q[1] = 0;
            q[2] = 0;
        }
        if (a >= 0)
        {
            float fx = (float)((double)x * kForceUnscale), fy = (float)((double)y * kForceUnscale),
                  fz = (float)((double)z * kForceUnscale);
            if (EXCL)
            {
                float wv[6] = {0, 0, 0, 0, 0, 0};
                excl_terms<EN>(a, sys[cl_sys[s >> 3]], xf, fx, fy, fz, ene, wv);
            }
            if (fx != 0.0f || fy != 0.0f || fz != 0.0f)
            {
                float3 f = frc[a];
                f.x += fx;
                f.y += fy;
                f.z += fz;
                frc[a] = f;
            }
        }
    }
    if (EXCL && EN)
    {
        // the correction's energy total: one atomic per warp
        long long qe = __double2ll_rn((double)ene * kEnergyScale);
        for (int o = 16; o > 0; o >>= 1) qe += __shfl_xor_sync(0xffffffffu, qe, o);
        if ((threadIdx.x & 31) == 0 && qe) atomicAdd((unsigned long long*)xf.total, (unsigned long long)qe);
    }
}

// Finishing pass of the per-atom mode (one system), one thread per local
// atom a: its force from its slot's staging; the owned energy and virial of
// a itself, or, for the first atom of a water of the solvent tail, of every
// site of the residue (SOLVENT_LENNARD_JONES credits the residue's first
// atom; three or four sites), summed exactly in int64 from the sites'
// slots, go to the per-atom arrays by plain read-modify-writes (each element
// has one writer, so the result does not depend on thread order) and to the
// totals; the staging read is cleared for the next call.  With EXCL the
// atom's excluded-pair correction is added as in k_fin8.
template <bool EXCL>
__global__ void k_fin8_atoms(int n, int slots, const int* __restrict__ atom_slot, const int* __restrict__ cl_sys,
                             const SysDesc* __restrict__ sys, long long* __restrict__ facc,
                             long long* __restrict__ oacc, float3* __restrict__ frc, long long* __restrict__ totals,
                             OwnerMap om, PerAtomOut pa, ExclFuse xf)
{
    grid_dep_wait();
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    float ene = 0.0f;
    long long tq[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // this atom's share of the totals
    if (a < n)
    {
        // every load first (they do not depend on each other beyond the
        // slots), then the arithmetic, then the stores: a thread waits for
        // memory about twice
        int sites = 1;  // the sites whose owned sums a receives
        if (a >= om.solvent_start)
            sites = (a - om.solvent_start) % om.water_points ? 0 : min(min(om.water_points, n - a), 4);
        int sl[4];
        sl[0] = atom_slot[a];
#pragma unroll
        for (int k = 1; k < 4; k++) sl[k] = k < sites ? atom_slot[a + k] : 0;
        long long* q = facc + 3 * (size_t)sl[0];
        const long long x = q[0], y = q[1], z = q[2];
        long long r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (k < sites)
            {
#pragma unroll
                for (int u = 0; u < 8; u++) r[u] += oacc[(size_t)u * slots + sl[k]];
            }
        const float3 f0 = frc[a];
        const bool own = sites > 0;
        const float e0 = own && pa.energy ? pa.energy[a] : 0.0f;
        const float l0 = own && pa.lj_energy ? pa.lj_energy[a] : 0.0f;
        const float d0 = own && pa.direct ? pa.direct[a] : 0.0f;
        float w0[6] = {0, 0, 0, 0, 0, 0};
        if (own && pa.virial)
        {
#pragma unroll
            for (int u = 0; u < 6; u++) w0[u] = pa.virial[6 * (size_t)a + u];
        }
        // the staging read is cleared for the next call
        if (x | y | z)
        {
            q[0] = 0;
            q[1] = 0;
            q[2] = 0;
        }
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (k < sites)
            {
#pragma unroll
                for (int u = 0; u < 8; u++) oacc[(size_t)u * slots + sl[k]] = 0;
            }
        // raw sums: -12 E_lj, E_c, and +g (x) d; the virial is -g (x) d with
        // the symmetric off-diagonal terms twice the one summed
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++)
        {
            const double sg = u == 0 ? (double)kLjEnergyScale
                                     : (u == 1 ? 1.0 : ((u == 3 || u == 5 || u == 6) ? -2.0 : -1.0));
            v[u] = (double)r[u] * sg;
            tq[u] = __double2ll_rn(v[u]);
        }
        const float elj = (float)(v[0] * kForceUnscale), ec = (float)(v[1] * kForceUnscale);
        float fx = (float)((double)x * kForceUnscale), fy = (float)((double)y * kForceUnscale),
              fz = (float)((double)z * kForceUnscale);
        float xe = 0.0f;
        float xw[6] = {0, 0, 0, 0, 0, 0};
        if (EXCL) excl_terms<true>(a, sys[cl_sys[sl[0] >> 3]], xf, fx, fy, fz, xe, xw);
        ene = xe;
        if (fx != 0.0f || fy != 0.0f || fz != 0.0f) frc[a] = make_float3(f0.x + fx, f0.y + fy, f0.z + fz);
        if (own)
        {
            if (pa.energy) pa.energy[a] = e0 + (elj + ec);
            if (pa.lj_energy) pa.lj_energy[a] = l0 + elj;
            if (pa.direct) pa.direct[a] = d0 + ec;
            if (pa.virial)
            {
#pragma unroll
                for (int u = 0; u < 6; u++) pa.virial[6 * (size_t)a + u] = w0[u] + (float)(v[2 + u] * kForceUnscale);
            }
        }
        if (EXCL)
        {
            // the correction's own adds (its arrays may be the same ones)
            if (xf.energy && xe != 0.0f) xf.energy[a] += xe;
            if (xf.virial && xf.sn[a].y > 0)
            {
                float* w = xf.virial + 6 * (size_t)a;
#pragma unroll
                for (int u = 0; u < 6; u++) w[u] += xw[u];
            }
        }
    }
    // the totals: summed over the warp by shuffles, over the block in shared
    // memory, one atomic per value and block
    __shared__ long long bsum[8];
    if (threadIdx.x < 8) bsum[threadIdx.x] = 0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 8; k++)
    {
        long long v = tq[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd((unsigned long long*)&bsum[k], (unsigned long long)v);
    }
    __syncthreads();
    if (threadIdx.x < 8 && bsum[threadIdx.x])
        atomicAdd((unsigned long long*)&totals[threadIdx.x], (unsigned long long)bsum[threadIdx.x]);
    if (EXCL)
    {
        // the correction's energy total: one atomic per warp
        long long qe = __double2ll_rn((double)ene * kEnergyScale);
        for (int o = 16; o > 0; o >>= 1) qe += __shfl_xor_sync(0xffffffffu, qe, o);
        if ((threadIdx.x & 31) == 0 && qe) atomicAdd((unsigned long long*)xf.total, (unsigned long long)qe);
    }
}

// A persistent grid: as many blocks as can be resident on every SM.
template <typename K>
int resident_blocks(K kernel, int threads, size_t smem)
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

template <int M, int F, bool T>
int launch_pair(const ForceInputs& in, cudaStream_t s)
{
    const spgnb_nl* nl = in.nl;
    const int mt = in.max_types > 0 ? in.max_types : in.p0.n_types;
    const size_t smem = sizeof(float4) * kPairWarps * 4 * mt;
    int resident = resident_blocks(k_pair8<M, F, T>, kPairWarps * 32, smem);
    if (in.pair_blocks_per_sm > 0) resident = std::min(resident, in.pair_blocks_per_sm * num_sms());
    const int grid = std::max(1, std::min(resident, (nl->clusters_cap + kPairWarps - 1) / kPairWarps));
    if (smem > 48 * 1024)
        SPGNB_CUDA(cudaFuncSetAttribute(k_pair8<M, F, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    launch_dependent(k_pair8<M, F, T>, grid, kPairWarps * 32, smem, s,
        in.p0, in.d_fps, nl->d_sys, nl->clusters_cap, nl->list_cap, nl->d_cl_sys, nl->d_pcount, nl->d_pwords,
        nl->d_cl_q, in.slot_pos, in.slot_aux, in.t4, nl->d_facc, nl->d_oacc, in.totals, in.only, nl->d_counters, mt);
    SPGNB_CHECK_LAUNCH("k_pair8");
    return SPGNB_OK;
}

template <int M, int F>
int launch_pair_t(const ForceInputs& in, bool tri, cudaStream_t s)
{
    return tri ? launch_pair<M, F, true>(in, s) : launch_pair<M, F, false>(in, s);
}

template <int M>
int launch_pair_ft(const ForceInputs& in, bool tri, cudaStream_t s)
{
    return in.fit ? launch_pair_t<M, 1>(in, tri, s) : launch_pair_t<M, 0>(in, tri, s);
}

}  // namespace

std::vector<float4> coefficient_table(const float2* table, int T)
{
    std::vector<float4> t4((size_t)T * T * T);
    for (int a = 0; a < T; a++)
        for (int b = 0; b < T; b++)
            for (int j = 0; j < T; j++)
            {
                const float2 ga = table[(size_t)a * T + j], gb = table[(size_t)b * T + j];
                t4[((size_t)a * T + b) * T + j] = make_float4(-ga.x, -gb.x, ga.y, gb.y);
            }
    return t4;
}

int build_t4(const float2* table, int T, float4** d_t4)
{
    const std::vector<float4> t4 = coefficient_table(table, T);
    dfree(*d_t4);
    int st = dalloc(d_t4, t4.size());
    if (st) return st;
    SPGNB_CUDA(cudaMemcpy(*d_t4, t4.data(), sizeof(float4) * t4.size(), cudaMemcpyHostToDevice));
    return SPGNB_OK;
}

int force_check(const ForceInputs& in)
{
    if (!in.t4) return fail(SPGNB_E_STATE, "force: the LJ module has no pair table");
    if (in.mode == 2 && in.nl->S != 1)
        return fail(SPGNB_E_UNSUPPORTED, "force: per-atom energy/virial outputs are for a one-system list");
    if (in.p0.n_types <= 0 || in.p0.n_types > kMaxTypes)
        return fail(SPGNB_E_UNSUPPORTED, "force: %d LJ types (at most %d)", in.p0.n_types, kMaxTypes);
    return SPGNB_OK;
}

int launch_pack(const ForceInputs& in, cudaStream_t s, const int* gate)
{
    spgnb_nl* nl = in.nl;
    const int slots = nl->clusters_cap * kClusterSize;
    const bool track = nl->opt.prune_buffer > 0.0f;
    const float half = 0.5f * nl->opt.prune_buffer;
    launch_dependent(k_pack_slots, (slots + 256) / 256, 256, 0, s, slots, nl->d_counters, nl->d_slot_atom, nl->d_slot_gid,
                                                     nl->d_cl_sys, nl->d_sys, nl->d_cl_q, nl->d_slot_x0,
                                                     nl->d_slot_d0, in.crd, in.charge, in.atom_type, in.slot_pos,
                                                     in.slot_aux, track ? nl->d_pref : nullptr, half * half,
                                                     nl->d_prune, in.clear.totals, in.clear.one, in.clear.a, in.clear.b,
                                                     in.clear.n, gate);
    SPGNB_CHECK_LAUNCH("k_pack_slots");
    return SPGNB_OK;
}

int launch_prune(const ForceInputs& in, cudaStream_t s)
{
    spgnb_nl* nl = in.nl;
    const int prune_bps = in.prune_blocks_per_sm > 0 ? in.prune_blocks_per_sm : 5;
    const int grid = std::max(1, std::min(num_sms() * prune_bps, (nl->clusters_cap + kPruneWarps - 1) / kPruneWarps));
    launch_dependent(k_prune8, grid, kPruneWarps * 32, 0, s, in.p0, in.d_fps, nl->opt.prune_buffer, nl->d_counters,
                                               nl->clusters_cap, nl->table_cap, nl->list_cap,
                                               nl->d_cl_sys, nl->d_sys, nl->d_tcount, nl->d_tab, nl->d_tmask,
                                               in.slot_pos, nl->d_pref, nl->d_pcount, nl->d_pwords, nl->S,
                                               nl->d_prune);
    SPGNB_CHECK_LAUNCH("k_prune8");
    return SPGNB_OK;
}

int launch_pair_kernel(const ForceInputs& in, cudaStream_t s)
{
    spgnb_nl* nl = in.nl;
    cudaEvent_t ev0, ev1;
    pair_events(&ev0, &ev1);
    if (ev0) SPGNB_CUDA(cudaEventRecord(ev0, s));
    int st;
    if (in.mode == 0)
        st = launch_pair_ft<0>(in, nl->triclinic, s);
    else if (in.mode == 1)
        st = launch_pair_ft<1>(in, nl->triclinic, s);
    else
        st = launch_pair_ft<2>(in, nl->triclinic, s);
    if (st) return st;
    if (ev1) SPGNB_CUDA(cudaEventRecord(ev1, s));
    return SPGNB_OK;
}

int force_pipeline(const ForceInputs& in, cudaStream_t s)
{
    spgnb_nl* nl = in.nl;
    const int slots = nl->clusters_cap * kClusterSize;
    int st = force_check(in);
    if (!st) st = launch_pack(in, s, nullptr);
    if (!st) st = launch_prune(in, s);
    if (!st) st = launch_pair_kernel(in, s);
    if (st) return st;
    const bool excl = in.xf.list != nullptr;
    const int blocks = (slots + 255) / 256;
    if (in.mode == 2)
    {
        const int n = nl->local_atoms;
        const int ab = (n + 255) / 256;
        if (excl)
            launch_dependent(k_fin8_atoms<true>, ab, 256, 0, s, n, slots, nl->d_atom_slot, nl->d_cl_sys, nl->d_sys, nl->d_facc,
                                                  nl->d_oacc, in.frc, in.totals, in.om, in.pa, in.xf);
        else
            launch_dependent(k_fin8_atoms<false>, ab, 256, 0, s, n, slots, nl->d_atom_slot, nl->d_cl_sys, nl->d_sys, nl->d_facc,
                                                   nl->d_oacc, in.frc, in.totals, in.om, in.pa, in.xf);
    }
    else if (excl && in.mode == 1)
        launch_dependent(k_fin8<true, true>, blocks, 256, 0, s, slots, nl->d_slot_atom, nl->d_cl_sys, nl->d_sys, nl->d_facc, in.frc,
                                                  in.xf);
    else if (excl)
        launch_dependent(k_fin8<true, false>, blocks, 256, 0, s, slots, nl->d_slot_atom, nl->d_cl_sys, nl->d_sys, nl->d_facc,
                                                   in.frc, in.xf);
    else
        launch_dependent(k_fin8<false, false>, blocks, 256, 0, s, slots, nl->d_slot_atom, nl->d_cl_sys, nl->d_sys, nl->d_facc,
                                                    in.frc, in.xf);
    SPGNB_CHECK_LAUNCH("k_fin8");
    return SPGNB_OK;
}

}  // namespace spgnb
