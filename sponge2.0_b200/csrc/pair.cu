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
#include "pairfn.cuh"

namespace spgnb
{
namespace
{

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
    grid_dep_wait();
    if (need_pressure)
    {
        virial[0] += vfac;
        virial[2] += vfac;
        virial[5] += vfac;
    }
    if (need_potential) potential[0] += efac;
}

// SOLVENT_LENNARD_JONES get_local_device (solvent_LJ.cpp:433-467): the
// solvent is the longest run of residues at the end of the local atoms that
// are waters of water_points atoms (O mass about 16, H masses about 1.008),
// counted from the last residue backwards.  Residue i of that run starts at
// atom_numbers - water_points * (local_res_numbers - i); one thread per
// residue tests it, and the run starts after the last residue that fails.
__global__ void k_solvent_count(int local_res_numbers, const int* __restrict__ res_len, int water_points,
                                int atom_numbers, const float* __restrict__ mass, int* last_fail)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= local_res_numbers) return;
    const int rs = atom_numbers - water_points * (local_res_numbers - i);
    bool water = rs >= 0 && res_len[i] == water_points;
    if (water)
    {
        const float mo = mass[rs], m1 = mass[rs + 1], m2 = mass[rs + 2];
        water = mo > 15.8f && mo < 16.2f && m1 > 1.007f && m1 < 1.009f && m2 > 1.007f && m2 < 1.009f;
    }
    if (!water) atomicMax(last_fail, i);
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
    pc.t4_begin = 0;
    return pc;
}

// Slot offsets and types plus the null slot.
int ensure_slots(spgnb_lj* lj, int slots)
{
    if (slots + 1 <= lj->sdata_cap) return SPGNB_OK;
    dfree(lj->d_sdata);
    dfree(lj->d_slot_aux);
    int st;
    if ((st = dalloc(&lj->d_sdata, (size_t)(slots + 1)))) return st;
    if ((st = dalloc(&lj->d_slot_aux, (size_t)(slots + 1)))) return st;
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

}  // namespace

int lj_finalize_forces(spgnb_lj* lj, int n, float3* frc, cudaStream_t s)
{
    if (n <= 0) return SPGNB_OK;
    k_finalize<<<(n + 255) / 256, 256, 0, s>>>(n, lj->d_frc_acc, frc);
    SPGNB_CHECK_LAUNCH("k_finalize");
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
    cudaMemcpy(lj->d_atom_type, h_atom_type, sizeof(int) * atom_numbers, cudaMemcpyHostToDevice);
    cudaMemcpy(lj->d_table, table.data(), sizeof(float2) * table.size(), cudaMemcpyHostToDevice);
    if ((st = build_t4(table.data(), T, &lj->d_t4)))
    {
        spgnb_lj_destroy(lj);
        return st;
    }
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
    if ((st = nl_set_prune_rc(const_cast<spgnb_nl*>(nl), lj->cutoff, s))) return st;
    ForceInputs in;
    in.nl = const_cast<spgnb_nl*>(nl);
    // what the callee zeroes (Lennard_Jones_force.cpp:376-382) is cleared by
    // the slot pack at the head of the force pass, not by separate memsets
    in.clear.totals = lj->d_totals;
    if (need_atom_energy)
    {
        in.clear.a = lj->d_lj_energy_atom;
        in.clear.b = d_atom_direct_pme_energy;
        in.clear.n = lj->atom_numbers;
    }
    in.crd = (const float3*)d_crd;
    in.charge = d_charge;
    in.atom_type = lj->d_local_type;
    in.slot_pos = lj->d_sdata;
    in.slot_aux = lj->d_slot_aux;
    in.p0 = make_pair_const(lj, pme_beta);
    in.fit = in.p0.use_fit != 0;
    in.t4 = lj->d_t4;
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
        if (mode >= 1) in.clear.one = lj->d_excl_total;
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
    launch_dependent(k_long_range, 1, 1, 0, stream(), need_pressure, (float*)d_virial, need_potential, d_potential,
                     vfac, efac);
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
    dfree(lj->d_slot_aux);
    dfree(lj->d_t4);
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
    SPGNB_CUDA(cudaMemsetAsync(s->d_scratch, 0xff, sizeof(int), stream()));  // no failing residue: -1
    if (local_res_numbers > 0)
    {
        k_solvent_count<<<(local_res_numbers + 255) / 256, 256, 0, stream()>>>(
            local_res_numbers, d_res_len, s->water_points, atom_numbers, d_mass, s->d_scratch);
        SPGNB_CHECK_LAUNCH("k_solvent_count");
    }
    int last_fail = -1;
    SPGNB_CUDA(cudaMemcpyAsync(&last_fail, s->d_scratch, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    SPGNB_CUDA(cudaStreamSynchronize(stream()));
    s->solvent_start_local = last_fail + 1;
    s->local_solvent_numbers = (local_res_numbers - (last_fail + 1)) * s->water_points;
    if (local_solvent_numbers) *local_solvent_numbers = s->local_solvent_numbers;
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
