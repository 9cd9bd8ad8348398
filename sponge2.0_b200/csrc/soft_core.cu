// LJ_SOFT_CORE: alchemical LJ + PME direct space with soft cores
// (SPONGE/Lennard_Jones_force/LJ_soft_core.{h,cpp}).
//
// Work split.  Only pairs with a perturbed atom can differ between the two
// states, and in a free-energy run those are a few dozen atoms out of tens of
// thousands.  So the module holds a regular spgnb_lj whose table is state A
// plus one null type: the pruned-list pair kernel evaluates every pair of the
// system with the perturbed atoms given the null type and charge 0 (their
// pairs come out exactly zero), and k_soft_pairs adds the perturbed atoms'
// pairs with the reference's two-state formula, one warp per perturbed atom
// over its cluster-table neighbours (the full neighbour set of the last
// build, exclusions removed).  A pair of two perturbed atoms is evaluated
// once, by the atom with the lower global index.
//
// Which atoms are perturbed is decided at creation from the types alone: two
// (type A, type B) combinations interact alike in both states when
// AA == BA and AB == BB for their pair (the reference then mixes equal terms,
// (1 - lambda) F + lambda F); the perturbed combinations are a small vertex
// cover of the combinations that do not, so every pair outside it is a pair
// the plain kernel reproduces.  Any cover is correct; a small one is fast.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <map>
#include <utility>
#include <vector>

#include "common.cuh"

namespace spgnb
{
namespace
{

constexpr float kTwoOverSqrtPi = 1.1283791670955126f;
constexpr int kSoftWarps = 4;

struct SoftConst
{
    float rc2, beta;
    float lam, lam_;      // lambda and 1 - lambda (float, as the reference)
    float alp_a, alp_b;   // alpha lambda^p, alpha (1 - lambda)^p
    float dua, dub;       // p alpha (1 - lambda) (lambda + FLT_MIN)^(p-1) / 6 and the state-B mirror
    float s6, s6min;      // sigma^6, sigma_min^6
};

struct SoftPair
{
    float f, elj, ec, dlj, dc;
};

__device__ __forceinline__ int tri_index(int a, int b)
{
    const int hi = a > b ? a : b, lo = a > b ? b : a;
    return hi * (hi + 1) / 2 + lo;
}

// Reference minimum image (vector.hpp:322-327), dr = r_j - r_i on entry.
__device__ __forceinline__ void min_image(float& dx, float& dy, float& dz, const Cell& c, const Cell& r)
{
    const float sx = floorf(dx * r.a11 + dy * r.a21 + dz * r.a31 + 0.5f);
    const float sy = floorf(dy * r.a22 + dz * r.a32 + 0.5f);
    const float sz = floorf(dz * r.a33 + 0.5f);
    dx -= sx * c.a11 + sy * c.a21 + sz * c.a31;
    dy -= sy * c.a22 + sz * c.a32;
    dz -= sz * c.a33;
}

__device__ __forceinline__ void red_fixed(long long* acc, float v)
{
    const long long q = __float2ll_rn(v * 4294967296.0f);
    if (q != 0) atomicAdd((unsigned long long*)acc, (unsigned long long)q);
}

// One pair, LJ_soft_core.cpp:247-414 with LJ_soft_core.h:33-150.  qq = q_i q_j;
// dq = q_i^BA q_j + q_i q_j^BA (the charge derivative, DHC only).  f is the
// scalar that multiplies dr = r_j - r_i for the force on i.
template <bool EN, bool DH, bool DHC>
__device__ __forceinline__ SoftPair soft_pair(const SoftConst& k, float r2, float qq, float dq, float AA, float AB,
                                              float BA, float BB)
{
    SoftPair o{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const float r = sqrtf(r2);
    if (BA * AA != 0.0f || BA + AA == 0.0f)
    {
        // both states have (or both lack) the r^-12 term: linear mixing at r
        const float i2 = 1.0f / r2;
        const float i6 = i2 * i2 * i2;
        const float i8 = i6 * i2;
        const float fa = (AB - AA * i6) * i8;
        const float fb = (BB - BA * i6) * i8;
        const float br = k.beta * r;
        const float erfc_r = erfcf(br);
        const float fc = qq * i2 / r * (br * kTwoOverSqrtPi * expf(-br * br) + erfc_r);
        o.f = k.lam_ * fa + k.lam * fb - fc;
        if (EN || DH)
        {
            const float ea = (AA * (1.0f / 12.0f) * i6 - AB * (1.0f / 6.0f)) * i6;
            const float eb = (BA * (1.0f / 12.0f) * i6 - BB * (1.0f / 6.0f)) * i6;
            if (EN)
            {
                o.elj = k.lam_ * ea + k.lam * eb;
                o.ec = qq * erfc_r / r;
            }
            if (DH)
            {
                o.dlj = eb - ea;
                if (DHC) o.dc = erfc_r * dq / r;
            }
        }
        return o;
    }
    // one state lacks the r^-12 term: each state at its soft-core distance
    // r_X^6 = r^6 + alpha lambda_X^p sigma_X (rs^-6 = 1 / r_X^6 exactly)
    const float sa = (AA == 0.0f || AB == 0.0f) ? k.s6 : fmaxf(0.5f * AA / AB, k.s6min);
    const float sb = (BA == 0.0f || BB == 0.0f) ? k.s6 : fmaxf(0.5f * BA / BB, k.s6min);
    const float r4 = r2 * r2;
    const float r6 = r4 * r2;
    const float xa = r6 + k.alp_a * sa;
    const float xb = r6 + k.alp_b * sb;
    const float ra = sqrtf(cbrtf(xa));
    const float rb = sqrtf(cbrtf(xb));
    const float ia = 1.0f / xa;
    const float ib = 1.0f / xb;
    // LJ: r^4 (B - A rs^-6) rs^-12; Coulomb: qq r^4 (2/sqrt(pi) beta e^-(beta rs)^2 + erfc(beta rs)/rs) rs^-6
    const float la = (AB - AA * ia) * ia * ia;
    const float lb = (BB - BA * ib) * ib * ib;
    const float bra = k.beta * ra, brb = k.beta * rb;
    const float erfc_a = erfcf(bra), erfc_b = erfcf(brb);
    const float exp_a = expf(-bra * bra), exp_b = expf(-brb * brb);
    const float ca = qq * (kTwoOverSqrtPi * k.beta * exp_a + erfc_a / ra) * ia;
    const float cb = qq * (kTwoOverSqrtPi * k.beta * exp_b + erfc_b / rb) * ib;
    o.f = r4 * (k.lam_ * la + k.lam * lb) - r4 * (k.lam_ * ca + k.lam * cb);
    if (EN || DH)
    {
        const float ea = (AA * (1.0f / 12.0f) * ia - AB * (1.0f / 6.0f)) * ia;
        const float eb = (BA * (1.0f / 12.0f) * ib - BB * (1.0f / 6.0f)) * ib;
        const float cea = qq * erfc_a / ra;
        const float ceb = qq * erfc_b / rb;
        if (EN)
        {
            o.elj = k.lam_ * ea + k.lam * eb;
            o.ec = k.lam_ * cea + k.lam * ceb;
        }
        if (DH)
        {
            // dU/dr_X dr_X/dlambda: F(r_X) r_X^-4 sigma_X times the state's constant,
            // F(r_X) r_X^-4 = (B - A rs^-6) rs^-12 for LJ
            o.dlj = eb - ea + k.dua * la * sa - k.dub * lb * sb;
            if (DHC)
            {
                // Coulomb F(rs) rs^-4 = qq rs^-7 (2/sqrt(pi) beta rs e^-(beta rs)^2 + erfc(beta rs))
                const float fa = qq * (kTwoOverSqrtPi * bra * exp_a + erfc_a) * ia / ra;
                const float fb = qq * (kTwoOverSqrtPi * brb * exp_b + erfc_b) * ib / rb;
                o.dc = ceb - cea + k.dub * fb * sb - k.dua * fa * sa + k.lam * erfc_b * dq / rb +
                       k.lam_ * erfc_a * dq / ra;
            }
        }
    }
    return o;
}

// One thread per candidate pair: a warp takes a listed atom i and four
// elements of the table of i's cluster (list == nullptr: the atoms are the
// local atoms, flag selects), lane 8e + b the neighbour slot b of element e,
// kept when the element's pair mask pairs it with i.  So an atom's pairs
// spread over many warps and no lane evaluates more than one: the kernel's
// time is one pair's latency, not a list's.  A partner that is itself
// flagged and has the lower global index owns the pair and skips it here.
// Forces go to int64 accumulators; energy and virial to the pair's owner
// (lower global index), the totals in fixed point.
constexpr int kSoftElems = 4;   // table elements per warp

template <bool FORCE, bool EN, bool PA, bool DH, bool DHC>
__global__ void __launch_bounds__(kSoftWarps * 32)
    k_soft_pairs(SoftConst k, Cell cell, Cell rcell, long long n_items, int chunks, const int* __restrict__ list,
                 const unsigned char* __restrict__ flag,
                 const int* __restrict__ atom_local, const int* __restrict__ atom_slot,
                 const int* __restrict__ slot_atom, const int* __restrict__ tcount, const float4* __restrict__ tab,
                 const uint2* __restrict__ tmask, int table_cap, const float3* __restrict__ crd,
                 const float* __restrict__ charge, const float* __restrict__ charge_ba,
                 const int2* __restrict__ types, const float* __restrict__ tAA, const float* __restrict__ tAB,
                 const float* __restrict__ tBA, const float* __restrict__ tBB, long long* __restrict__ acc,
                 long long* __restrict__ totals, PerAtomOut pa, long long* __restrict__ dh)
{
    grid_dep_wait();
    const int lane = threadIdx.x & 31;
    const long long item = (long long)blockIdx.x * kSoftWarps + (threadIdx.x >> 5);
    if (item >= n_items) return;  // whole warps
    const int ia = (int)(item / chunks);
    const int t0 = (int)(item % chunks) * kSoftElems;
    const int i = list ? list[ia] : ia;
    if (!flag[i]) return;
    const int s = atom_slot[i];
    if (s < 0) return;
    const int c = s / kClusterSize, a = s % kClusterSize;
    const int T = tcount[c];
    if (t0 >= T) return;
    const float3 ri = crd[i];
    const float qi = charge[i];
    const float qbi = DHC ? charge_ba[i] : 0.0f;
    const int2 ti = types[i];
    const int gi = atom_local[i];
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    float tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // this lane's pair: E_lj, E_c, virial
    float own[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // the part owned by i
    float dl = 0.0f, dc = 0.0f;
    do
    {
        const int t = t0 + (lane >> 3), b = lane & 7;
        if (t >= T) break;
        const uint2 mm = tmask[(size_t)c * table_cap + t];
        if (!((((a < 4 ? mm.x : mm.y) >> (8 * (a & 3))) >> b) & 1u)) break;
        const int base = __float_as_int(tab[(size_t)c * table_cap + t].w) & 0x3fffffff;
        const int j = slot_atom[base + b];
        if (j < 0 || j == i) break;
        const int gj = atom_local[j];
        if (flag[j] && gj < gi) break;
        const float3 rj = crd[j];
        float dx = rj.x - ri.x, dy = rj.y - ri.y, dz = rj.z - ri.z;
        min_image(dx, dy, dz, cell, rcell);
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < k.rc2)) break;
        const int2 tj = types[j];
        const int pa_ = tri_index(ti.x, tj.x), pb_ = tri_index(ti.y, tj.y);
        const float qj = charge[j];
        const float dq = DHC ? qbi * qj + qi * charge_ba[j] : 0.0f;
        const SoftPair o = soft_pair<EN, DH, DHC>(k, r2, qi * qj, dq, tAA[pa_], tAB[pa_], tBA[pb_], tBB[pb_]);
        if (DH)
        {
            dl = o.dlj;
            dc = o.dc;
        }
        if (!FORCE) break;
        const float gx = o.f * dx, gy = o.f * dy, gz = o.f * dz;
        fx = gx;
        fy = gy;
        fz = gz;
        red_fixed(acc + 4 * (size_t)j + 0, -gx);
        red_fixed(acc + 4 * (size_t)j + 1, -gy);
        red_fixed(acc + 4 * (size_t)j + 2, -gz);
        if (EN)
        {
            // Get_Virial_From_Force_Dis(F, dr) (vector.hpp:337-347), subtracted
            const float w[8] = {o.elj, o.ec, -gx * dx, -(gx * dy + gy * dx), -gy * dy, -(gx * dz + gz * dx),
                                -(gy * dz + gz * dy), -gz * dz};
#pragma unroll
            for (int q = 0; q < 8; q++) tot[q] = w[q];
            if (PA)
            {
                if (gi < gj)
                {
#pragma unroll
                    for (int q = 0; q < 8; q++) own[q] = w[q];
                }
                else
                {
                    if (pa.energy) atomicAdd(pa.energy + j, w[0] + w[1]);
                    if (pa.lj_energy) atomicAdd(pa.lj_energy + j, w[0]);
                    if (pa.direct) atomicAdd(pa.direct + j, w[1]);
                    if (pa.virial)
                        for (int q = 0; q < 6; q++) atomicAdd(pa.virial + 6 * (size_t)j + q, w[2 + q]);
                }
            }
        }
    } while (false);
    if (FORCE)
    {
        for (int o = 16; o > 0; o >>= 1)
        {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
        }
        if (lane == 0)
        {
            red_fixed(acc + 4 * (size_t)i + 0, fx);
            red_fixed(acc + 4 * (size_t)i + 1, fy);
            red_fixed(acc + 4 * (size_t)i + 2, fz);
        }
    }
    if (EN)
    {
#pragma unroll
        for (int q = 0; q < 8; q++)
        {
            long long v = __double2ll_rn((double)tot[q] * kEnergyScale);
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0 && v) atomicAdd((unsigned long long*)&totals[q], (unsigned long long)v);
        }
    }
    if (PA)
    {
#pragma unroll
        for (int q = 0; q < 8; q++)
            for (int o = 16; o > 0; o >>= 1) own[q] += __shfl_xor_sync(0xffffffffu, own[q], o);
        if (lane == 0)
        {
            if (pa.energy) atomicAdd(pa.energy + i, own[0] + own[1]);
            if (pa.lj_energy) atomicAdd(pa.lj_energy + i, own[0]);
            if (pa.direct) atomicAdd(pa.direct + i, own[1]);
            if (pa.virial)
                for (int q = 0; q < 6; q++) atomicAdd(pa.virial + 6 * (size_t)i + q, own[2 + q]);
        }
    }
    if (DH)
    {
        long long v0 = __double2ll_rn((double)dl * kEnergyScale);
        long long v1 = __double2ll_rn((double)dc * kEnergyScale);
        for (int o = 16; o > 0; o >>= 1)
        {
            v0 += __shfl_xor_sync(0xffffffffu, v0, o);
            v1 += __shfl_xor_sync(0xffffffffu, v1, o);
        }
        if (lane == 0)
        {
            if (v0) atomicAdd((unsigned long long*)&dh[0], (unsigned long long)v0);
            if (v1) atomicAdd((unsigned long long*)&dh[1], (unsigned long long)v1);
        }
    }
}

// Local copies of the per-atom state (LJ_soft_core.cpp:892-904).
__global__ void k_soft_local(int n, const int* __restrict__ atom_local, const int2* __restrict__ types_g,
                             const unsigned char* __restrict__ pert_g, int2* __restrict__ types,
                             unsigned char* __restrict__ flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int g = atom_local[i];
    types[i] = types_g[g];
    flag[i] = pert_g[g];
}

// Charges seen by the plain kernel: perturbed atoms carry none.
__global__ void k_mask_charge(int n, const float* __restrict__ q, const unsigned char* __restrict__ flag,
                              float* __restrict__ out)
{
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = flag[i] ? 0.0f : q[i];
}

// Atoms whose pairs enter dH/dlambda with charge perturbation on: the
// perturbed ones and every atom whose charge changes; flagged and listed (in
// any order: the sums are fixed point).
__global__ void k_dh_flags(int n, const unsigned char* __restrict__ flag, const float* __restrict__ charge_ba,
                           unsigned char* __restrict__ out, int* __restrict__ list, int* __restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool on = flag[i] || charge_ba[i] != 0.0f;
    out[i] = on ? 1 : 0;
    if (on) list[atomicAdd(count, 1)] = i;
}

template <bool FORCE, bool EN, bool PA, bool DH, bool DHC>
int launch_soft(const SoftConst& k, const spgnb_ltmatrix3& cell, const spgnb_ltmatrix3& rcell, int n_items,
                const int* list, const unsigned char* flag, const int* atom_local, const spgnb_nl* nl,
                const float3* crd, const float* charge, const float* charge_ba, const int2* types, const float* AA,
                const float* AB, const float* BA, const float* BB, long long* acc, long long* totals,
                PerAtomOut pa, long long* dh, cudaStream_t s)
{
    if (n_items <= 0) return SPGNB_OK;
    const int chunks = (nl->table_cap + kSoftElems - 1) / kSoftElems;
    const long long warps = (long long)n_items * chunks;
    const long long grid = (warps + kSoftWarps - 1) / kSoftWarps;
    if (grid > 0x7fffffffLL) return fail(SPGNB_E_UNSUPPORTED, "soft-core kernel: %lld blocks", grid);
    launch_dependent(k_soft_pairs<FORCE, EN, PA, DH, DHC>, (unsigned)grid, kSoftWarps * 32, 0, s,
        k, make_cell(cell), make_cell(rcell), warps, chunks, list, flag, atom_local, nl->d_atom_slot,
        nl->d_slot_atom,
        nl->d_tcount, nl->d_tab, nl->d_tmask, nl->table_cap, crd, charge, charge_ba, types, AA, AB, BA, BB, acc,
        totals, pa, dh);
    SPGNB_CHECK_LAUNCH("k_soft_pairs");
    return SPGNB_OK;
}

// Small vertex cover of the combinations whose pairs differ between the
// states: combinations that differ with themselves first, then greedily the
// one covering the most remaining edges per atom.
std::vector<char> cover_combos(const std::vector<std::pair<int, int>>& combos, const std::vector<double>& count,
                               const std::vector<float>& AA, const std::vector<float>& AB,
                               const std::vector<float>& BA, const std::vector<float>& BB)
{
    const int C = (int)combos.size();
    auto tri = [](int a, int b) { return a > b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; };
    auto differ = [&](int u, int v) {
        const int p = tri(combos[u].first, combos[v].first), q = tri(combos[u].second, combos[v].second);
        return !(AA[p] == BA[q] && AB[p] == BB[q]);
    };
    std::vector<char> in(C, 0);
    std::vector<std::vector<int>> adj(C);
    for (int u = 0; u < C; u++)
    {
        if (differ(u, u)) in[u] = 1;
        for (int v = u + 1; v < C; v++)
            if (differ(u, v))
            {
                adj[u].push_back(v);
                adj[v].push_back(u);
            }
    }
    for (;;)
    {
        int best = -1;
        double best_score = 0.0;
        for (int u = 0; u < C; u++)
        {
            if (in[u]) continue;
            int deg = 0;
            for (int v : adj[u]) deg += !in[v];
            if (deg == 0) continue;
            const double score = deg / std::max(count[u], 1.0);
            if (best < 0 || score > best_score)
            {
                best = u;
                best_score = score;
            }
        }
        if (best < 0) break;
        in[best] = 1;
    }
    return in;
}

}  // namespace
}  // namespace spgnb

struct spgnb_lj_soft
{
    int atom_numbers = 0;
    int nA = 0, nB = 0;
    float cutoff = 0;
    spgnb_soft_core_params prm{};
    spgnb_lj* inner = nullptr;           // state A + null type, perturbed atoms masked
    std::vector<char> h_pert;            // per global atom
    std::vector<int> pert_atoms;         // global indices, ascending
    double factor = 0, factor_ti = 0;
    int2* d_types_g = nullptr;           // per global atom {type A, type B}
    unsigned char* d_pert_g = nullptr;
    float *d_AA = nullptr, *d_AB = nullptr, *d_BA = nullptr, *d_BB = nullptr;
    int2* d_types = nullptr;             // per local atom
    unsigned char* d_flag = nullptr;
    unsigned char* d_dh_flag = nullptr;
    int* d_dh_list = nullptr;            // atoms of the charge-perturbed dH/dlambda
    int* d_dh_count = nullptr;
    float* d_masked_q = nullptr;
    int* d_list = nullptr;               // perturbed local atoms
    int n_list = 0;
    int local_atoms = 0;
    const int* d_atom_local = nullptr;
    long long* d_dh = nullptr;           // dH/dlambda LJ, direct (fixed point)
};

using namespace spgnb;

namespace
{

SoftConst soft_const(const spgnb_lj_soft* lj, float beta)
{
    const spgnb_soft_core_params& p = lj->prm;
    SoftConst k;
    k.rc2 = lj->cutoff * lj->cutoff;
    k.beta = beta;
    k.lam = p.lambda;
    k.lam_ = 1.0f - p.lambda;
    k.alp_a = p.alpha * powf(p.lambda, p.p);
    k.alp_b = p.alpha * powf(k.lam_, p.p);
    k.dua = (1.0f / 6.0f) * p.p * p.alpha * (1.0f - p.lambda) * powf(p.lambda + FLT_MIN, p.p - 1.0f);
    k.dub = (1.0f / 6.0f) * p.p * p.alpha * (1.0f - k.lam_) * powf(k.lam_ + FLT_MIN, p.p - 1.0f);
    k.s6 = powf(p.sigma, 6.0f);
    k.s6min = powf(p.sigma_min, 6.0f);
    return k;
}

int check_list(const spgnb_lj_soft* lj, const spgnb_nl* nl, int local_atom_numbers, const char* who)
{
    if (!nl) return fail(SPGNB_E_ARG, "%s: nl is NULL", who);
    if (!nl->built) return fail(SPGNB_E_STATE, "%s: the neighbour list was never built", who);
    if (nl->S != 1) return fail(SPGNB_E_STATE, "%s: the list holds several systems", who);
    if (local_atom_numbers != nl->local_atoms)
        return fail(SPGNB_E_STATE, "%s: list built for %d atoms, called with %d", who, nl->local_atoms,
                    local_atom_numbers);
    if (!lj->d_types) return fail(SPGNB_E_STATE, "%s: Get_Local has not been called", who);
    if (local_atom_numbers > lj->local_atoms)
        return fail(SPGNB_E_STATE, "%s: %d local atoms but Get_Local saw %d", who, local_atom_numbers, lj->local_atoms);
    return SPGNB_OK;
}

}  // namespace

extern "C" {

void spgnb_lj_soft_default_params(spgnb_soft_core_params* prm)
{
    if (!prm) return;
    prm->lambda = 0.0f;
    prm->alpha = 0.5f;
    prm->p = 1.0f;
    prm->sigma = 3.0f;
    prm->sigma_min = 0.0f;
}

int spgnb_lj_soft_create(int atom_numbers, int atom_type_numbers_A, int atom_type_numbers_B,
                         const int* h_atom_LJ_type_A, const int* h_atom_LJ_type_B, const float* h_LJ_AA,
                         const float* h_LJ_AB, const float* h_LJ_BA, const float* h_LJ_BB,
                         const spgnb_soft_core_params* prm, float cutoff, spgnb_lj_soft** out)
{
    if (!out) return fail(SPGNB_E_ARG, "spgnb_lj_soft_create: out is NULL");
    *out = nullptr;
    if (atom_numbers <= 0 || atom_type_numbers_A <= 0 || atom_type_numbers_B <= 0 || !h_atom_LJ_type_A ||
        !h_atom_LJ_type_B || !h_LJ_AA || !h_LJ_AB || !h_LJ_BA || !h_LJ_BB || !prm || !(cutoff > 0))
        return fail(SPGNB_E_ARG, "spgnb_lj_soft_create: bad arguments");
    const int nA = atom_type_numbers_A, nB = atom_type_numbers_B;
    if (nA + 1 > kMaxTypes)
        return fail(SPGNB_E_UNSUPPORTED, "spgnb_lj_soft_create: %d state-A types (at most %d)", nA, kMaxTypes - 1);
    const size_t pA = (size_t)nA * (nA + 1) / 2, pB = (size_t)nB * (nB + 1) / 2;
    std::vector<float> AA(h_LJ_AA, h_LJ_AA + pA), AB(h_LJ_AB, h_LJ_AB + pA);
    std::vector<float> BA(h_LJ_BA, h_LJ_BA + pB), BB(h_LJ_BB, h_LJ_BB + pB);

    // (type A, type B) combinations and their atom counts
    std::map<std::pair<int, int>, int> id_of;
    std::vector<std::pair<int, int>> combos;
    std::vector<double> count;
    std::vector<int> combo_of(atom_numbers);
    for (int i = 0; i < atom_numbers; i++)
    {
        const int ta = h_atom_LJ_type_A[i], tb = h_atom_LJ_type_B[i];
        if (ta < 0 || ta >= nA || tb < 0 || tb >= nB)
            return fail(SPGNB_E_ARG, "spgnb_lj_soft_create: atom %d has types (%d, %d) outside [0,%d) x [0,%d)", i,
                        ta, tb, nA, nB);
        auto it = id_of.find({ta, tb});
        if (it == id_of.end())
        {
            it = id_of.emplace(std::make_pair(ta, tb), (int)combos.size()).first;
            combos.push_back({ta, tb});
            count.push_back(0.0);
        }
        combo_of[i] = it->second;
        count[it->second] += 1.0;
    }
    const std::vector<char> cover = cover_combos(combos, count, AA, AB, BA, BB);

    spgnb_lj_soft* lj = new spgnb_lj_soft();
    lj->atom_numbers = atom_numbers;
    lj->nA = nA;
    lj->nB = nB;
    lj->cutoff = cutoff;
    lj->prm = *prm;
    lj->h_pert.resize(atom_numbers);
    std::vector<int> inner_type(atom_numbers);
    std::vector<int2> types(atom_numbers);
    for (int i = 0; i < atom_numbers; i++)
    {
        lj->h_pert[i] = cover[combo_of[i]];
        if (lj->h_pert[i]) lj->pert_atoms.push_back(i);
        inner_type[i] = lj->h_pert[i] ? nA : h_atom_LJ_type_A[i];
        types[i] = make_int2(h_atom_LJ_type_A[i], h_atom_LJ_type_B[i]);
    }

    // Total_C6_Get / Total_C6_B_A_Get (LJ_soft_core.cpp:83-181) over combination pairs:
    // sum_ij (1 - lambda) AB_ij + lambda BB_ij and sum_ij BB_ij - AB_ij, products in float
    const float lam = prm->lambda, lam_ = 1.0f - prm->lambda;
    double c6 = 0.0, c6_ti = 0.0;
    auto tri = [](int a, int b) { return a > b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; };
    for (size_t u = 0; u < combos.size(); u++)
        for (size_t v = 0; v < combos.size(); v++)
        {
            const int p = tri(combos[u].first, combos[v].first), q = tri(combos[u].second, combos[v].second);
            const double w = count[u] * count[v];
            c6 += w * ((double)(lam_ * AB[p]) + (double)(lam * BB[q]));
            c6_ti += w * (double)(BB[q] - AB[p]);
        }
    const float scale = -2.0f / 3.0f * 3.1415926535897932f / cutoff / cutoff / cutoff / 6.0f;
    lj->factor = (float)c6 * scale;
    lj->factor_ti = (float)c6_ti * scale;

    // the plain kernel's table: state A plus the null type nA
    std::vector<float> iA((size_t)(nA + 1) * (nA + 2) / 2, 0.0f), iB(iA.size(), 0.0f);
    for (size_t p = 0; p < pA; p++)
    {
        iA[p] = AA[p];
        iB[p] = AB[p];
    }
    int st = spgnb_lj_create(atom_numbers, nA + 1, inner_type.data(), iA.data(), iB.data(), cutoff, &lj->inner);
    if (st)
    {
        delete lj;
        return st;
    }
    lj->inner->long_range_factor = lj->factor;
    std::vector<unsigned char> pert_u8(lj->h_pert.begin(), lj->h_pert.end());
    if ((st = dalloc(&lj->d_types_g, atom_numbers)) || (st = dalloc(&lj->d_pert_g, atom_numbers)) ||
        (st = dalloc(&lj->d_AA, pA)) || (st = dalloc(&lj->d_AB, pA)) || (st = dalloc(&lj->d_BA, pB)) ||
        (st = dalloc(&lj->d_BB, pB)) || (st = dalloc(&lj->d_dh, 2)))
    {
        spgnb_lj_soft_destroy(lj);
        return st;
    }
    cudaMemcpy(lj->d_types_g, types.data(), sizeof(int2) * atom_numbers, cudaMemcpyHostToDevice);
    cudaMemcpy(lj->d_pert_g, pert_u8.data(), atom_numbers, cudaMemcpyHostToDevice);
    cudaMemcpy(lj->d_AA, AA.data(), sizeof(float) * pA, cudaMemcpyHostToDevice);
    cudaMemcpy(lj->d_AB, AB.data(), sizeof(float) * pA, cudaMemcpyHostToDevice);
    cudaMemcpy(lj->d_BA, BA.data(), sizeof(float) * pB, cudaMemcpyHostToDevice);
    cudaMemcpy(lj->d_BB, BB.data(), sizeof(float) * pB, cudaMemcpyHostToDevice);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
    {
        spgnb_lj_soft_destroy(lj);
        return cuda_fail(e, "spgnb_lj_soft_create");
    }
    *out = lj;
    return SPGNB_OK;
}

int spgnb_lj_soft_get_local(spgnb_lj_soft* lj, const int* d_atom_local, int local_atom_numbers, int ghost_numbers)
{
    if (!lj || !d_atom_local) return fail(SPGNB_E_ARG, "spgnb_lj_soft_get_local: NULL argument");
    const int n = local_atom_numbers + ghost_numbers;
    if (ghost_numbers != 0)
        return fail(SPGNB_E_UNSUPPORTED, "spgnb_lj_soft_get_local: ghost atoms (multi-rank) are not supported");
    if (n > lj->atom_numbers) return fail(SPGNB_E_ARG, "spgnb_lj_soft_get_local: too many local atoms");
    int st = spgnb_lj_get_local(lj->inner, d_atom_local, local_atom_numbers, ghost_numbers);
    if (st) return st;
    if (!lj->d_types)
    {
        const int N = lj->atom_numbers;
        if ((st = dalloc(&lj->d_types, N)) || (st = dalloc(&lj->d_flag, N)) || (st = dalloc(&lj->d_dh_flag, N)) ||
            (st = dalloc(&lj->d_masked_q, N)) || (st = dalloc(&lj->d_list, N)) || (st = dalloc(&lj->d_dh_list, N)) ||
            (st = dalloc(&lj->d_dh_count, 1)))
            return st;
    }
    cudaStream_t s = stream();
    if (n > 0)
    {
        k_soft_local<<<(n + 255) / 256, 256, 0, s>>>(n, d_atom_local, lj->d_types_g, lj->d_pert_g, lj->d_types,
                                                    lj->d_flag);
        SPGNB_CHECK_LAUNCH("k_soft_local");
    }
    // the perturbed local atoms, listed once on the host
    std::vector<int> local(n);
    if (n > 0)
    {
        SPGNB_CUDA(cudaMemcpyAsync(local.data(), d_atom_local, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        SPGNB_CUDA(cudaStreamSynchronize(s));
    }
    std::vector<int> list;
    for (int i = 0; i < n; i++)
    {
        if (local[i] < 0 || local[i] >= lj->atom_numbers)
            return fail(SPGNB_E_ARG, "spgnb_lj_soft_get_local: atom_local[%d] = %d outside the system", i, local[i]);
        if (lj->h_pert[local[i]]) list.push_back(i);
    }
    if (!list.empty())
        SPGNB_CUDA(cudaMemcpyAsync(lj->d_list, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, s));
    SPGNB_CUDA(cudaStreamSynchronize(s));
    lj->n_list = (int)list.size();
    lj->local_atoms = local_atom_numbers;
    lj->d_atom_local = d_atom_local;
    return SPGNB_OK;
}

int spgnb_lj_soft_pme_direct_force(spgnb_lj_soft* lj, int atom_numbers, int local_atom_numbers,
                                   int solvent_numbers, int ghost_numbers, const spgnb_vector* d_crd,
                                   const float* d_charge, spgnb_vector* d_frc, spgnb_ltmatrix3 cell,
                                   spgnb_ltmatrix3 rcell, const spgnb_nl* nl, float pme_beta, int need_atom_energy,
                                   float* d_atom_energy, int need_virial, spgnb_ltmatrix3* d_atom_virial,
                                   float* d_atom_direct_pme_energy)
{
    static const char* who = "spgnb_lj_soft_pme_direct_force";
    if (!lj) return fail(SPGNB_E_ARG, "%s: NULL handle", who);
    if (!d_crd || !d_charge || !d_frc) return fail(SPGNB_E_ARG, "%s: NULL device pointer", who);
    if (ghost_numbers != 0) return fail(SPGNB_E_UNSUPPORTED, "%s: ghost atoms are not supported", who);
    if (local_atom_numbers == 0) return SPGNB_OK;
    int st = check_list(lj, nl, local_atom_numbers, who);
    if (st) return st;
    cudaStream_t s = stream();
    // the perturbed atoms' pairs come from their clusters' two-sided tables
    if ((st = nl_two_sided_atoms(nl, lj->d_flag, s))) return st;
    const int n = local_atom_numbers;
    launch_dependent(k_mask_charge, (n + 255) / 256, 256, 0, s, n, d_charge, lj->d_flag, lj->d_masked_q);
    SPGNB_CHECK_LAUNCH("k_mask_charge");
    st = spgnb_lj_pme_direct_force(lj->inner, atom_numbers, local_atom_numbers, solvent_numbers, ghost_numbers, d_crd,
                                   lj->d_masked_q, d_frc, cell, rcell, nl, pme_beta, need_atom_energy, d_atom_energy,
                                   need_virial, d_atom_virial, d_atom_direct_pme_energy);
    if (st) return st;
    if (lj->n_list == 0) return SPGNB_OK;
    int mode = 0;
    if (need_atom_energy || need_virial) mode = 1;
    if ((need_atom_energy && (d_atom_energy || d_atom_direct_pme_energy)) || (need_virial && d_atom_virial))
        mode = 2;
    PerAtomOut pa{nullptr, nullptr, nullptr, nullptr};
    if (mode == 2)
    {
        pa.energy = need_atom_energy ? d_atom_energy : nullptr;
        pa.lj_energy = need_atom_energy ? lj->inner->d_lj_energy_atom : nullptr;
        pa.direct = need_atom_energy ? d_atom_direct_pme_energy : nullptr;
        pa.virial = need_virial ? (float*)d_atom_virial : nullptr;
    }
    const SoftConst k = soft_const(lj, pme_beta);
    const float3* crd = (const float3*)d_crd;
    long long* acc = lj->inner->d_frc_acc;
    long long* tot = lj->inner->d_totals;
    if (mode == 0)
        st = launch_soft<true, false, false, false, false>(k, cell, rcell, lj->n_list, lj->d_list, lj->d_flag,
                                                           lj->d_atom_local, nl, crd, d_charge, nullptr, lj->d_types,
                                                           lj->d_AA, lj->d_AB, lj->d_BA, lj->d_BB, acc, tot, pa,
                                                           nullptr, s);
    else if (mode == 1)
        st = launch_soft<true, true, false, false, false>(k, cell, rcell, lj->n_list, lj->d_list, lj->d_flag,
                                                          lj->d_atom_local, nl, crd, d_charge, nullptr, lj->d_types,
                                                          lj->d_AA, lj->d_AB, lj->d_BA, lj->d_BB, acc, tot, pa,
                                                          nullptr, s);
    else
        st = launch_soft<true, true, true, false, false>(k, cell, rcell, lj->n_list, lj->d_list, lj->d_flag,
                                                         lj->d_atom_local, nl, crd, d_charge, nullptr, lj->d_types,
                                                         lj->d_AA, lj->d_AB, lj->d_BA, lj->d_BB, acc, tot, pa,
                                                         nullptr, s);
    if (st) return st;
    return lj_finalize_forces(lj->inner, n, (float3*)d_frc, s);
}

int spgnb_lj_soft_partial_h_partial_lambda(spgnb_lj_soft* lj, int solvent_numbers, const spgnb_vector* d_crd,
                                           spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, const float* d_charge,
                                           const spgnb_nl* nl, const float* d_charge_B_A, float pme_beta,
                                           int charge_perturbated, double* dh_dlambda, double* dh_dlambda_direct)
{
    static const char* who = "spgnb_lj_soft_partial_h_partial_lambda";
    (void)solvent_numbers;
    if (!lj || !dh_dlambda) return fail(SPGNB_E_ARG, "%s: NULL argument", who);
    if (!d_crd || !d_charge) return fail(SPGNB_E_ARG, "%s: NULL device pointer", who);
    if (charge_perturbated && !d_charge_B_A) return fail(SPGNB_E_ARG, "%s: charge_B_A is NULL", who);
    int st = check_list(lj, nl, lj->local_atoms, who);
    if (st) return st;
    cudaStream_t s = stream();
    // the atoms whose pairs it sums (the perturbed ones, and with charge
    // perturbation every atom whose charge changes) read their clusters'
    // tables: two-sided ones for this call (a rare one: output steps)
    if ((st = nl_symmetrize(nl, s))) return st;
    SPGNB_CUDA(cudaMemsetAsync(lj->d_dh, 0, 2 * sizeof(long long), s));
    const SoftConst k = soft_const(lj, pme_beta);
    const float3* crd = (const float3*)d_crd;
    PerAtomOut pa{nullptr, nullptr, nullptr, nullptr};
    const int n = lj->local_atoms;
    if (charge_perturbated)
    {
        SPGNB_CUDA(cudaMemsetAsync(lj->d_dh_count, 0, sizeof(int), s));
        k_dh_flags<<<(n + 255) / 256, 256, 0, s>>>(n, lj->d_flag, d_charge_B_A, lj->d_dh_flag, lj->d_dh_list,
                                                   lj->d_dh_count);
        SPGNB_CHECK_LAUNCH("k_dh_flags");
        int m = 0;
        SPGNB_CUDA(cudaMemcpyAsync(&m, lj->d_dh_count, sizeof(int), cudaMemcpyDeviceToHost, s));
        SPGNB_CUDA(cudaStreamSynchronize(s));
        st = launch_soft<false, false, false, true, true>(k, cell, rcell, m, lj->d_dh_list, lj->d_dh_flag,
                                                          lj->d_atom_local,
                                                          nl, crd, d_charge, d_charge_B_A, lj->d_types, lj->d_AA,
                                                          lj->d_AB, lj->d_BA, lj->d_BB, nullptr, nullptr, pa, lj->d_dh,
                                                          s);
    }
    else
    {
        st = launch_soft<false, false, false, true, false>(k, cell, rcell, lj->n_list, lj->d_list, lj->d_flag,
                                                           lj->d_atom_local, nl, crd, d_charge, nullptr, lj->d_types,
                                                           lj->d_AA, lj->d_AB, lj->d_BA, lj->d_BB, nullptr, nullptr,
                                                           pa, lj->d_dh, s);
    }
    if (st) return st;
    long long h[2];
    SPGNB_CUDA(cudaMemcpyAsync(h, lj->d_dh, sizeof(h), cudaMemcpyDeviceToHost, s));
    SPGNB_CUDA(cudaStreamSynchronize(s));
    // LJ_soft_core.cpp:840-841: + long_range_factor_TI / (a11 a22 a33), in float
    const float tail = (float)lj->factor_ti / cell.a11 / cell.a22 / cell.a33;
    *dh_dlambda = (double)h[0] / kEnergyScale + (double)tail;
    if (dh_dlambda_direct) *dh_dlambda_direct = charge_perturbated ? (double)h[1] / kEnergyScale : 0.0;
    return SPGNB_OK;
}

int spgnb_lj_soft_long_range_correction(spgnb_lj_soft* lj, int need_pressure, spgnb_ltmatrix3* d_virial,
                                        int need_potential, float* d_potential, float volume)
{
    if (!lj) return fail(SPGNB_E_ARG, "spgnb_lj_soft_long_range_correction: NULL handle");
    return spgnb_lj_long_range_correction(lj->inner, need_pressure, d_virial, need_potential, d_potential, volume);
}

int spgnb_lj_soft_energies(spgnb_lj_soft* lj, double* lj_short, double* lj_long, double* lj_total,
                           double* direct_coulomb)
{
    if (!lj) return fail(SPGNB_E_ARG, "spgnb_lj_soft_energies: NULL handle");
    return spgnb_lj_energies(lj->inner, lj_short, lj_long, lj_total, direct_coulomb);
}

int spgnb_lj_soft_totals(spgnb_lj_soft* lj, double out[8])
{
    if (!lj) return fail(SPGNB_E_ARG, "spgnb_lj_soft_totals: NULL handle");
    return spgnb_lj_totals(lj->inner, out);
}

int spgnb_lj_soft_long_range_factors(const spgnb_lj_soft* lj, double* factor, double* factor_ti)
{
    if (!lj) return fail(SPGNB_E_ARG, "spgnb_lj_soft_long_range_factors: NULL handle");
    if (factor) *factor = lj->factor;
    if (factor_ti) *factor_ti = lj->factor_ti;
    return SPGNB_OK;
}

int spgnb_lj_soft_atom_lj_energy(spgnb_lj_soft* lj, float** d_atom_lj_energy)
{
    if (!lj) return fail(SPGNB_E_ARG, "spgnb_lj_soft_atom_lj_energy: NULL handle");
    return spgnb_lj_atom_lj_energy(lj->inner, d_atom_lj_energy);
}

int spgnb_lj_soft_perturbed_atoms(const spgnb_lj_soft* lj, int* count, int* h_atoms, int capacity)
{
    if (!lj || !count) return fail(SPGNB_E_ARG, "spgnb_lj_soft_perturbed_atoms: NULL argument");
    *count = (int)lj->pert_atoms.size();
    if (h_atoms && capacity >= *count) std::copy(lj->pert_atoms.begin(), lj->pert_atoms.end(), h_atoms);
    return SPGNB_OK;
}

int spgnb_solvent_create_soft(spgnb_lj_soft* lj, int water_points, spgnb_solvent** out)
{
    if (!lj) return fail(SPGNB_E_ARG, "spgnb_solvent_create_soft: NULL handle");
    return spgnb_solvent_create(lj->inner, water_points, out);
}

int spgnb_lj_soft_destroy(spgnb_lj_soft* lj)
{
    if (!lj) return SPGNB_OK;
    spgnb_lj_destroy(lj->inner);
    dfree(lj->d_types_g);
    dfree(lj->d_pert_g);
    dfree(lj->d_AA);
    dfree(lj->d_AB);
    dfree(lj->d_BA);
    dfree(lj->d_BB);
    dfree(lj->d_types);
    dfree(lj->d_flag);
    dfree(lj->d_dh_flag);
    dfree(lj->d_dh_list);
    dfree(lj->d_dh_count);
    dfree(lj->d_masked_q);
    dfree(lj->d_list);
    dfree(lj->d_dh);
    delete lj;
    return SPGNB_OK;
}

}  // extern "C"
