// Batched engine: many independent periodic systems stepped together.
//
// No reference counterpart (the reference runs one system per process); the
// per-system physics is the reference path's: the neighbour list of
// NEIGHBOR_LIST (per system, skin-triggered as in neighbor_list.cpp:166-180),
// LJ + PME direct space of LENNARD_JONES_INFORMATION / SOLVENT_LENNARD_JONES,
// and the long-range LJ correction (Lennard_Jones_force.cpp:320-341).  The
// integrator is leap-frog velocity Verlet with SETTLE for rigid 3-site waters
// (Miyamoto & Kollman, J. Comput. Chem. 13, 952 (1992)).
//
// Layout: the systems' atoms are concatenated; every system owns fixed
// ranges of cells, clusters and slots of one multi-system neighbour list, and
// its rebuild and pruning decisions look at its own atoms only, so a system's
// trajectory is the same alone and in any batch.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

// reference units: kcal/mol, A, g/mol; one internal time unit is 1/20.455 ps
// (AKMA), in which F/m is an acceleration in A per unit^2
static constexpr float kTimeUnitsPerPs = 20.455f;

struct SysRec
{
    bool live = false;
    int atom_begin = 0, atom_count = 0;
    long long ex_begin = 0, ex_count = 0;
    int w_begin = 0, w_count = 0;
    double lr_factor = 0, volume = 0;
    long long t4_begin = 0, t4_count = 0;  // the system's own coefficient table, when it has one
};

// A pool of systems: fixed capacities, every system in ranges of its own.
struct spgnb_batch
{
    int S = 0;          // system ids
    int n = 0;          // atom capacity
    long long ex_cap = 0;
    int w_cap = 0;
    RangePool atom_pool, ex_pool, water_pool;
    RangePool t4_pool;  // coefficient-table elements: the batch's table first, then systems' own
    std::vector<SysRec> rec;
    std::vector<float> h_pair_A, h_pair_B;  // the batch's type table, reference layout
    spgnb_batch_options opt{};
    spgnb_nl* nl = nullptr;
    cudaStream_t stream = nullptr;
    // per atom (parked atoms: zero velocity and inverse mass)
    float3* d_crd = nullptr;
    float3* d_vel = nullptr;
    float3* d_frc = nullptr;
    float3* d_crd_old = nullptr;
    float* d_charge = nullptr;
    float* d_inv_mass = nullptr;
    int* d_type = nullptr;
    int* d_atom_local = nullptr;  // the atom's own index (exclusions hold pool indices)
    int* d_ex_start = nullptr;
    int* d_ex_num = nullptr;
    int* d_ex_list = nullptr;
    int* d_waters = nullptr;  // oxygen of each rigid water, -1 for a free entry
    unsigned char* d_in_water = nullptr;  // per atom: moved with its water (SETTLE)
    // force field
    int T = 0;                    // types of the batch's table
    int max_T = 0;                // most types of any table (the force kernel's shared rows)
    long long t4_cap = 0;
    float4* d_t4 = nullptr;       // the force kernel's T^3 tables
    spgnb::ForceParams* d_fps = nullptr;  // S + 1
    std::vector<spgnb::ForceParams> h_fps;
    bool fit = true;                  // the rational fits (every admitted system inside their range)
    long long* d_totals = nullptr;    // 8 per system id
    long long* d_kin = nullptr;       // per system: sum of m v^2, fixed point
    float* d_lambda = nullptr;        // per system: the thermostat's velocity scale for the next step
    int* d_skin_hit = nullptr;        // per system: an atom moved past the skin this step
    int* d_done = nullptr;            // blocks of the step kernel finished
    float* d_ndof = nullptr;          // per system: degrees of freedom
    int* d_steps = nullptr;           // per system: steps done
    int* d_left = nullptr;            // per system: steps left (-1 unlimited, 0 stopped or parked)
    int* d_flags = nullptr;           // per system: evaluate now
    std::vector<int> h_flags;
    float4* d_slot_pos = nullptr;
    int4* d_slot_aux = nullptr;
    // stepping
    bool have_water = false;
    float ra = 0, rb = 0, rc = 0, mO = 0, mH = 0;
    cudaGraphExec_t g_plain = nullptr, g_energy = nullptr;
    // kernel launches inside each graph: those of every step, and those of
    // the list builds, which run only on steps where some system rebuilds
    long long kernels_plain = 0, kernels_energy = 0, kernels_build = 0;
    bool graph_tri = false;
    long long steps_done = 0;
    // launch configuration (spgnb_batch_autotune)
    int pair_bps = 0, prune_bps = 0;
    float tuned_ms = 0.0f;
    bool pending = false;  // admitted systems wait for their first lists and forces
    std::vector<spgnb::PinnedStage> stages;  // upload buffers of admissions, reused when their copies are done
};

namespace spgnb
{
namespace
{

__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 unit3(float3 a) { return mul3(a, rsqrtf(dot3(a, a))); }

// SETTLE for one rigid water (oxygen o, hydrogens o+1, o+2): moves the
// unconstrained new positions onto the water's geometry, keeping its centre
// of mass, from the old (constrained) ones.  The triangle in its own frame
// has O at (0, ra, 0) and the hydrogens at (-+rc, -rb, 0); the new plane
// orientation comes from rotations about the frame axes solved in closed
// form (Miyamoto & Kollman 1992).  Velocities follow from the displacement.
// Old positions o0..o2 (constrained), new ones n0..n2 (unconstrained) in;
// the constrained new positions and their velocities out (in n and v).
__device__ __forceinline__ void settle_water(float3 o0, float3 o1, float3 o2, float3 (&n)[3], float3 (&v)[3],
                                             float mO, float mH, float ra, float rb, float rc, float inv_dt)
{
    const float3 origin = o0;
    // everything relative to the old oxygen, for precision
    const float3 b0 = sub3(o1, origin), c0 = sub3(o2, origin);
    const float3 a1 = sub3(n[0], origin), b1 = sub3(n[1], origin), c1 = sub3(n[2], origin);
    const float wt = mO + 2.0f * mH;
    const float3 com = mul3(add3(mul3(a1, mO), mul3(add3(b1, c1), mH)), 1.0f / wt);
    const float3 xa1 = sub3(a1, com), xb1 = sub3(b1, com), xc1 = sub3(c1, com);
    // frame: z normal to the old plane, x normal to the new oxygen and z
    const float3 ez = unit3(cross3(b0, c0));
    const float3 ex = unit3(cross3(xa1, ez));
    const float3 ey = cross3(ez, ex);
    const float xb0 = dot3(ex, b0), yb0 = dot3(ey, b0);
    const float xc0 = dot3(ex, c0), yc0 = dot3(ey, c0);
    const float za1 = dot3(ez, xa1);
    const float xb1d = dot3(ex, xb1), yb1d = dot3(ey, xb1), zb1 = dot3(ez, xb1);
    const float xc1d = dot3(ex, xc1), yc1d = dot3(ey, xc1), zc1 = dot3(ez, xc1);
    const float sinphi = fminf(fmaxf(za1 / ra, -1.0f), 1.0f);
    const float cosphi = sqrtf(fmaxf(1.0f - sinphi * sinphi, 0.0f));
    const float sinpsi = fminf(fmaxf((zb1 - zc1) / (2.0f * rc * cosphi), -1.0f), 1.0f);
    const float cospsi = sqrtf(fmaxf(1.0f - sinpsi * sinpsi, 0.0f));
    const float ya2 = ra * cosphi;
    const float xb2 = -rc * cospsi;
    const float t1 = -rb * cosphi, t2 = rc * sinpsi * sinphi;
    const float yb2 = t1 - t2, yc2 = t1 + t2;
    // rotation about z that best matches the old triangle
    const float alpha = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2;
    const float beta = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2;
    const float gamma = xb0 * yb1d - xb1d * yb0 + xc0 * yc1d - xc1d * yc0;
    const float ab2 = alpha * alpha + beta * beta;
    const float sintheta = (alpha * gamma - beta * sqrtf(fmaxf(ab2 - gamma * gamma, 0.0f))) / ab2;
    const float costheta = sqrtf(fmaxf(1.0f - sintheta * sintheta, 0.0f));
    const float xa3 = -ya2 * sintheta, ya3 = ya2 * costheta;
    const float xb3 = xb2 * costheta - yb2 * sintheta, yb3 = xb2 * sintheta + yb2 * costheta;
    const float xc3 = -xb2 * costheta - yc2 * sintheta, yc3 = -xb2 * sintheta + yc2 * costheta;
    const float3 a3 = add3(com, add3(add3(mul3(ex, xa3), mul3(ey, ya3)), mul3(ez, za1)));
    const float3 b3 = add3(com, add3(add3(mul3(ex, xb3), mul3(ey, yb3)), mul3(ez, zb1)));
    const float3 c3 = add3(com, add3(add3(mul3(ex, xc3), mul3(ey, yc3)), mul3(ez, zc1)));
    n[0] = add3(origin, a3);
    n[1] = add3(origin, b3);
    n[2] = add3(origin, c3);
    v[0] = mul3(a3, inv_dt);  // a0 is the origin
    v[1] = mul3(sub3(b3, b0), inv_dt);
    v[2] = mul3(sub3(c3, c0), inv_dt);
}

// What one step of the batched engine's integrator needs (k_step_begin).
struct StepArgs
{
    int n, w_cap, S;
    const int* atom_sys;            // system of each atom (parked atoms: a system that is not live)
    const int* atom_slot;           // slot of each atom in its system's last build
    const unsigned char* in_water;  // atoms moved by their water's thread
    const int* waters;              // oxygen of each rigid water, -1 for a free entry
    const int* live;
    int* left;
    int* steps;
    float3* crd;
    float3* vel;
    float3* frc;
    float3* crd_old;
    const float* inv_mass;
    const float* charge;
    long long* facc;                // the force pass's int64 staging per slot, taken and cleared here
    float dt, inv_dt;
    int settle;
    float mO, mH, ra, rb, rc;
    int thermostat;                 // Berendsen: lambda from the last step's kinetic energy
    long long* kin;
    float* lambda;
    const float* ndof;
    float kT0, coupling;
    int interval;                   // > 0: rebuild by step count; 0: by the skin check
    const spgnb::SysDesc* sys;
    const float4* slot_x0;
    const float4* slot_d0;
    float4* slot_pos;
    const float4* pref;             // positions at the last pruning (null: pruning off)
    float half_buffer2;
    int* prune;
    int* skin_hit;
    int* need;
    int* counters;
    int* done;                      // blocks finished (the last one decides)
    cudaGraphConditionalHandle h_build, h_prune;  // 0 outside a captured graph
};

// One atom's state for a step, every load issued before any use (the
// loads do not depend on each other beyond the slot index), so a thread waits
// for memory about twice instead of once per access.
struct AtomIn
{
    int slot;
    long long f[3];  // the force pass's int64 sums for the atom's slot
    float3 x, v;
    float im, q;
    float4 x0, d0, pref;
};

__device__ __forceinline__ void load_atom(const StepArgs& a, int i, AtomIn& t)
{
    t.slot = a.atom_slot[i];
    const long long* f = a.facc + 3 * (size_t)t.slot;
    t.f[0] = f[0];
    t.f[1] = f[1];
    t.f[2] = f[2];
    t.x = a.crd[i];
    t.v = a.vel[i];
    t.im = a.inv_mass[i];
    t.q = a.charge[i];
    t.x0 = a.slot_x0[t.slot];
    t.d0 = a.slot_d0[t.slot];
    t.pref = a.pref ? a.pref[t.slot] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// F(t) from the staging, which is cleared for the next force pass; also the
// caller-visible float force.
__device__ __forceinline__ float3 take_force(const StepArgs& a, int i, const AtomIn& t)
{
    long long* f = a.facc + 3 * (size_t)t.slot;
    f[0] = 0;
    f[1] = 0;
    f[2] = 0;
    const float3 r = make_float3((float)((double)t.f[0] * kForceUnscale), (float)((double)t.f[1] * kForceUnscale),
                                 (float)((double)t.f[2] * kForceUnscale));
    a.frc[i] = r;
    return r;
}

// Leap-frog kick with F(t) (velocities first scaled by the thermostat's
// lambda) and drift, in registers: t.x becomes the new position.
__device__ __forceinline__ void kick_drift(const StepArgs& a, AtomIn& t, float3 f, float lam)
{
    const float im = t.im * a.dt;
    t.v.x = fmaf(f.x, im, t.v.x * lam);
    t.v.y = fmaf(f.y, im, t.v.y * lam);
    t.v.z = fmaf(f.z, im, t.v.z * lam);
    t.x = make_float3(fmaf(t.v.x, a.dt, t.x.x), fmaf(t.v.y, a.dt, t.x.y), fmaf(t.v.z, a.dt, t.x.z));
}

struct BoxOf
{
    spgnb::Cell cell, rcell;
    float permit2;
};

__device__ __forceinline__ BoxOf box_of(const StepArgs& a, int sy)
{
    const spgnb::SysDesc& D = a.sys[sy];
    BoxOf b;
    b.cell = D.cell;
    b.rcell = D.rcell;
    b.permit2 = D.permit2;
    return b;
}

// The moved atom's slot record {offset from the build-time cluster centre
// moved by the displacement since the build, charge} for the force pass, and
// the checks that follow a move: a pruning when it moved more than half the
// prune buffer since the last one, a rebuild (skin trigger) when it moved
// more than the permitted skin since the build (UPDATOR::Check_Refresh,
// neighbor_list.cpp:166-180, in the same expression as k_check_refresh).
__device__ __forceinline__ void pack_atom(const StepArgs& a, const AtomIn& t, int sy, const BoxOf& D, bool& moved)
{
    const float3 c = t.x;
    const float4 o = t.x0;
    {
        float dx = c.x - o.x, dy = c.y - o.y, dz = c.z - o.z;
        const float sx = rintf(dx * D.rcell.a11 + dy * D.rcell.a21 + dz * D.rcell.a31);
        const float sy2 = rintf(dy * D.rcell.a22 + dz * D.rcell.a32);
        const float sz = rintf(dz * D.rcell.a33);
        dx -= sx * D.cell.a11 + sy2 * D.cell.a21 + sz * D.cell.a31;
        dy -= sy2 * D.cell.a22 + sz * D.cell.a32;
        dz -= sz * D.cell.a33;
        const float4 p = make_float4(t.d0.x + dx, t.d0.y + dy, t.d0.z + dz, t.q);
        a.slot_pos[t.slot] = p;
        if (a.pref)
        {
            const float ex = p.x - t.pref.x, ey = p.y - t.pref.y, ez = p.z - t.pref.z;
            if (ex * ex + ey * ey + ez * ez > a.half_buffer2)
            {
                a.prune[sy] = 1;
                moved = true;
            }
        }
    }
    if (a.interval <= 0)
    {
        float dx = c.x - o.x, dy = c.y - o.y, dz = c.z - o.z;
        const float sx = floorf(dx * D.rcell.a11 + dy * D.rcell.a21 + dz * D.rcell.a31 + 0.5f);
        const float sy2 = floorf(dy * D.rcell.a22 + dz * D.rcell.a32 + 0.5f);
        const float sz = floorf(dz * D.rcell.a33 + 0.5f);
        dx -= sx * D.cell.a11 + sy2 * D.cell.a21 + sz * D.cell.a31;
        dy -= sy2 * D.cell.a22 + sz * D.cell.a32;
        dz -= sz * D.cell.a33;
        if (dx * dx + dy * dy + dz * dz > D.permit2) a.skin_hit[sy] = 1;
    }
}

__device__ __forceinline__ double mv2(const AtomIn& t)
{
    return t.im != 0.0f ? (double)((t.v.x * t.v.x + t.v.y * t.v.y + t.v.z * t.v.z) / t.im) : 0.0;
}

// The start of a batched step, one kernel: threads [0, n) the atoms outside
// rigid waters, [n, n + w_cap) the waters (their three atoms, then SETTLE).
// Each takes its atoms' forces F(t) from the force pass's staging, kicks and
// drifts them, writes their slot records for this step's force pass and
// checks how far they moved, and adds m v^2 to its system's fixed-point sum.
// Systems with no steps left keep their state (their forces are still taken).
// The last block to finish, once every atom has moved, ends the step for
// each system: its step counter, the thermostat's lambda for the next step,
// the rebuild decision (refresh interval or skin trigger), and sets the
// graph's conditionals: the list build when some system rebuilds, the
// pruning when some system prunes.
__global__ void k_step_begin(StepArgs a)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    int sy = -1;
    double e = 0.0;
    bool moved = false;
    if (u < a.n)
    {
        const int i = u;
        const int s = a.atom_sys[i];
        if (!a.in_water[i] && s < a.S && a.live[s])
        {
            AtomIn t;
            load_atom(a, i, t);
            const float3 f = take_force(a, i, t);
            if (a.left[s] != 0)
            {
                const BoxOf box = box_of(a, s);
                const float3 x_old = t.x;
                kick_drift(a, t, f, a.thermostat ? a.lambda[s] : 1.0f);
                a.crd_old[i] = x_old;
                a.crd[i] = t.x;
                a.vel[i] = t.v;
                pack_atom(a, t, s, box, moved);
                e = mv2(t);
                sy = s;
            }
        }
    }
    else if (u < a.n + a.w_cap)
    {
        const int o = a.waters[u - a.n];
        const int s = o >= 0 ? a.atom_sys[o] : a.S;
        if (s < a.S && a.live[s])
        {
            AtomIn t[3];
            load_atom(a, o, t[0]);
            load_atom(a, o + 1, t[1]);
            load_atom(a, o + 2, t[2]);
            const float3 f0 = take_force(a, o, t[0]), f1 = take_force(a, o + 1, t[1]),
                         f2 = take_force(a, o + 2, t[2]);
            if (a.left[s] != 0)
            {
                const BoxOf box = box_of(a, s);
                const float lam = a.thermostat ? a.lambda[s] : 1.0f;
                const float3 x0 = t[0].x, x1 = t[1].x, x2 = t[2].x;
                kick_drift(a, t[0], f0, lam);
                kick_drift(a, t[1], f1, lam);
                kick_drift(a, t[2], f2, lam);
                if (a.settle)
                {
                    float3 n[3] = {t[0].x, t[1].x, t[2].x}, v[3];
                    settle_water(x0, x1, x2, n, v, a.mO, a.mH, a.ra, a.rb, a.rc, a.inv_dt);
                    for (int k = 0; k < 3; k++)
                    {
                        t[k].x = n[k];
                        t[k].v = v[k];
                    }
                }
                a.crd_old[o] = x0;
                a.crd_old[o + 1] = x1;
                a.crd_old[o + 2] = x2;
                for (int k = 0; k < 3; k++)
                {
                    a.crd[o + k] = t[k].x;
                    a.vel[o + k] = t[k].v;
                    pack_atom(a, t[k], s, box, moved);
                }
                e = mv2(t[0]) + mv2(t[1]) + mv2(t[2]);
                sy = s;
            }
        }
    }
    if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) a.counters[kCntPrune] = 1;
    if (a.thermostat)
    {
        // twice the kinetic energy in fixed point (the same in any order):
        // one atomic per warp when its atoms belong to one system
        long long q = sy >= 0 ? __double2ll_rn(e * kEnergyScale) : 0ll;
        const unsigned valid = __ballot_sync(0xffffffffu, sy >= 0);
        if (valid)
        {
            const int s0 = __shfl_sync(0xffffffffu, sy, __ffs(valid) - 1);
            if (__all_sync(0xffffffffu, sy < 0 || sy == s0))
            {
#pragma unroll
                for (int k = 16; k > 0; k >>= 1) q += __shfl_xor_sync(0xffffffffu, q, k);
                if ((threadIdx.x & 31) == 0) atomicAdd((unsigned long long*)&a.kin[s0], (unsigned long long)q);
            }
            else if (sy >= 0)
                atomicAdd((unsigned long long*)&a.kin[sy], (unsigned long long)q);
        }
    }
    // the last block ends the step for every system (the block's writes
    // ordered before its count by the barrier and one fence)
    __shared__ int is_last;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        is_last = atomicAdd(a.done, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    int any_need = 0, any_prune = 0;
    for (int s = threadIdx.x; s < a.S; s += blockDim.x)
    {
        const bool active = a.live[s] && a.left[s] != 0;
        const bool due = active && (a.interval > 0 ? (a.steps[s] + 1) % a.interval == 0 : a.skin_hit[s] != 0);
        a.skin_hit[s] = 0;
        a.need[s] = due ? 1 : 0;
        any_need |= due ? 1 : 0;
        any_prune |= a.prune[s] != 0 ? 1 : 0;
        if (a.thermostat)
        {
            // Berendsen: lambda^2 = 1 + dt/tau (T0/T - 1), clamped to [0.64, 1.5625]
            const double kT = (double)a.kin[s] / kEnergyScale / fmax((double)a.ndof[s], 1.0);
            const float lam2 = kT > 0.0 ? 1.0f + a.coupling * (float)(a.kT0 / kT - 1.0) : 1.0f;
            a.lambda[s] = sqrtf(fminf(fmaxf(lam2, 0.64f), 1.5625f));
            a.kin[s] = 0;
        }
        if (active)
        {
            a.steps[s] += 1;
            if (a.left[s] > 0) a.left[s] -= 1;
        }
    }
    any_need = __syncthreads_or(any_need);
    any_prune = __syncthreads_or(any_prune);
    if (threadIdx.x == 0)
    {
        a.counters[kCntNeed] = any_need;
        if (any_prune) a.counters[kCntPrune] = 1;
        *a.done = 0;
        if (a.h_build) cudaGraphSetConditional(a.h_build, any_need ? 1u : 0u);
        if (a.h_prune) cudaGraphSetConditional(a.h_prune, (any_need || any_prune) ? 1u : 0u);
    }
}

// Clears the force staging of the chosen systems' slots (all with flags
// null), and their energy totals, before a force pass for them alone.
__global__ void k_clear_staged(int slots, const int* __restrict__ cl_sys, const int* __restrict__ flags,
                               long long* __restrict__ facc, int S, long long* __restrict__ totals)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < slots && (!flags || flags[cl_sys[s >> 3]]))
    {
        facc[3 * (size_t)s] = 0;
        facc[3 * (size_t)s + 1] = 0;
        facc[3 * (size_t)s + 2] = 0;
    }
    if (totals && s < 8 * S && (!flags || flags[s >> 3])) totals[s] = 0;
}

// The forces of atoms [first, first + count) from their slots' staging
// (left in place for the next step).
__global__ void k_forces_out(int first, int count, const int* __restrict__ atom_slot,
                             const long long* __restrict__ facc, float3* __restrict__ frc)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int i = first + k;
    const long long* f = facc + 3 * (size_t)atom_slot[i];
    frc[i] = make_float3((float)((double)f[0] * kForceUnscale), (float)((double)f[1] * kForceUnscale),
                         (float)((double)f[2] * kForceUnscale));
}

ForceInputs batch_inputs(spgnb_batch* b, int mode, const int* only)
{
    ForceInputs in;
    in.nl = b->nl;
    in.crd = b->d_crd;
    in.charge = b->d_charge;
    in.atom_type = b->d_type;
    in.slot_pos = b->d_slot_pos;
    in.slot_aux = b->d_slot_aux;
    in.p0 = b->h_fps[0];
    in.d_fps = b->d_fps;
    in.fit = b->fit;
    in.t4 = b->d_t4;
    in.max_types = b->max_T;
    in.frc = b->d_frc;
    in.totals = b->d_totals;
    in.mode = mode;
    in.pair_blocks_per_sm = b->pair_bps;
    in.prune_blocks_per_sm = b->prune_bps;
    in.om.solvent_start = b->n;
    in.only = only;
    return in;
}

// A force pass outside the step, for the flagged systems (all with only
// null): their staging cleared, slot pack, pruning, pair kernel.  The forces
// stay in the staging for the next step to take (k_forces_out reads them).
int batch_force(spgnb_batch* b, int mode, cudaStream_t s, const int* only = nullptr)
{
    const int slots = b->nl->clusters_cap * kClusterSize;
    const int m = std::max(slots, 8 * b->S);
    k_clear_staged<<<(m + 255) / 256, 256, 0, s>>>(slots, b->nl->d_cl_sys, only, b->nl->d_facc, b->S,
                                                   mode ? b->d_totals : nullptr);
    SPGNB_CHECK_LAUNCH("k_clear_staged");
    const ForceInputs in = batch_inputs(b, mode, only);
    int st = force_check(in);
    if (!st) st = launch_pack(in, s, nullptr);
    if (!st) st = launch_prune(in, s);
    if (!st) st = launch_pair_kernel(in, s);
    return st;
}

// During a graph capture: an 'if' node on handle h after the work captured
// so far on s, its body captured on the side stream (open .. close).
struct CaptureIf
{
    cudaStream_t side = nullptr;
    bool open_ = false;
    static int handle(cudaStream_t s, cudaGraphConditionalHandle* h)
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        SPGNB_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
        *h = 0;
        if (cs == cudaStreamCaptureStatusActive)
            SPGNB_CUDA(cudaGraphConditionalHandleCreate(h, g, 0, cudaGraphCondAssignDefault));
        return SPGNB_OK;
    }
    int open(cudaStream_t s, cudaGraphConditionalHandle h)
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        SPGNB_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeIf;
        p.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        SPGNB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
        SPGNB_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
        SPGNB_CUDA(cudaStreamBeginCaptureToGraph(side, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeThreadLocal));
        open_ = true;
        return SPGNB_OK;
    }
    int close()
    {
        if (!open_) return SPGNB_OK;
        open_ = false;
        cudaGraph_t g = nullptr;
        SPGNB_CUDA(cudaStreamEndCapture(side, &g));
        return SPGNB_OK;
    }
};

// One step: k_step_begin (forces taken, kick, drift, SETTLE, slot records,
// decisions), the list build (when some system rebuilds), the pruning (when
// some system prunes), the pair kernel.  In a capture (cap set) the build
// and the pruning are the bodies of conditional nodes the step kernel sets;
// otherwise they are launched and return at once unless needed.  Counts the
// kernels of the build and pruning bodies into *cond_kernels.
int batch_step(spgnb_batch* b, bool energy, cudaStream_t s, CaptureIf* cap = nullptr,
               long long* cond_kernels = nullptr)
{
    spgnb_nl* nl = b->nl;
    StepArgs a{};
    a.n = b->n;
    a.w_cap = b->have_water ? b->w_cap : 0;
    a.S = b->S;
    a.atom_sys = nl->d_atom_sys;
    a.atom_slot = nl->d_atom_slot;
    a.in_water = b->d_in_water;
    a.waters = b->d_waters;
    a.live = nl->d_live;
    a.left = b->d_left;
    a.steps = b->d_steps;
    a.crd = b->d_crd;
    a.vel = b->d_vel;
    a.frc = b->d_frc;
    a.crd_old = b->d_crd_old;
    a.inv_mass = b->d_inv_mass;
    a.charge = b->d_charge;
    a.facc = nl->d_facc;
    a.dt = b->opt.dt * kTimeUnitsPerPs;
    a.inv_dt = 1.0f / a.dt;
    a.settle = b->have_water ? 1 : 0;
    a.mO = b->mO;
    a.mH = b->mH;
    a.ra = b->ra;
    a.rb = b->rb;
    a.rc = b->rc;
    a.thermostat = b->opt.thermostat_tau > 0.0f ? 1 : 0;
    a.kin = b->d_kin;
    a.lambda = b->d_lambda;
    a.ndof = b->d_ndof;
    a.kT0 = 0.00198716f * b->opt.temperature;  // kcal/mol
    a.coupling = b->opt.thermostat_tau > 0.0f ? b->opt.dt / b->opt.thermostat_tau : 0.0f;
    a.interval = b->opt.refresh_interval;
    a.sys = nl->d_sys;
    a.slot_x0 = nl->d_slot_x0;
    a.slot_d0 = nl->d_slot_d0;
    a.slot_pos = b->d_slot_pos;
    const bool track = nl->opt.prune_buffer > 0.0f;
    a.pref = track ? nl->d_pref : nullptr;
    const float half = 0.5f * nl->opt.prune_buffer;
    a.half_buffer2 = half * half;
    a.prune = nl->d_prune;
    a.skin_hit = b->d_skin_hit;
    a.need = nl->d_need;
    a.counters = nl->d_counters;
    a.done = b->d_done;
    int st;
    if (cap && ((st = CaptureIf::handle(s, &a.h_build)) || (st = CaptureIf::handle(s, &a.h_prune)))) return st;
    const int units = a.n + a.w_cap;
    k_step_begin<<<(units + 255) / 256, 256, 0, s>>>(a);
    SPGNB_CHECK_LAUNCH("k_step_begin");
    const ForceInputs in = batch_inputs(b, energy ? 1 : 0, nullptr);
    if ((st = force_check(in))) return st;
    // the list build, then the slot records in the new slots
    cudaStream_t bs = s;
    if (cap && a.h_build)
    {
        if ((st = cap->open(s, a.h_build))) return st;
        bs = cap->side;
    }
    const unsigned long long c0 = launches_so_far();
    st = nl_queue_build_body(nl, b->n, b->d_crd, b->d_atom_local, b->d_ex_start, b->d_ex_list, b->d_ex_num, bs);
    if (!st) st = launch_pack(in, bs, nl->d_counters + kCntNeed);
    if (cap && a.h_build)
    {
        const int st2 = cap->close();
        if (!st) st = st2;
    }
    if (st) return st;
    // the pruning
    cudaStream_t ps = s;
    if (cap && a.h_prune)
    {
        if ((st = cap->open(s, a.h_prune))) return st;
        ps = cap->side;
    }
    st = launch_prune(in, ps);
    if (cap && a.h_prune)
    {
        const int st2 = cap->close();
        if (!st) st = st2;
    }
    if (st) return st;
    if (cond_kernels) *cond_kernels += (long long)(launches_so_far() - c0);
    if (energy) SPGNB_CUDA(cudaMemsetAsync(b->d_totals, 0, sizeof(long long) * 8 * b->S, s));
    return launch_pair_kernel(in, s);
}

// Lists and forces (with energies) of the systems admitted since the last
// run; the other systems' state is untouched.
int settle_pending(spgnb_batch* b)
{
    if (!b->pending) return SPGNB_OK;
    cudaStream_t s = b->stream;
    // d_flags: set for each admitted system by its admission
    int st = nl_queue_build(b->nl, b->n, b->d_crd, b->d_atom_local, b->d_ex_start, b->d_ex_list, b->d_ex_num,
                            kBuildPreset, s, b->d_flags);
    if (!st) st = batch_force(b, 1, s, b->d_flags);
    if (st) return st;
    SPGNB_CUDA(cudaMemsetAsync(b->d_flags, 0, sizeof(int) * b->S, s));
    std::fill(b->h_flags.begin(), b->h_flags.end(), 0);
    b->pending = false;
    return SPGNB_OK;
}

void free_graphs(spgnb_batch* b)
{
    if (b->g_plain) cudaGraphExecDestroy(b->g_plain);
    if (b->g_energy) cudaGraphExecDestroy(b->g_energy);
    b->g_plain = b->g_energy = nullptr;
}

int capture(spgnb_batch* b, bool energy_last, cudaGraphExec_t* out, long long* kernels)
{
    cudaGraph_t g = nullptr;
    CaptureIf cap;
    SPGNB_CUDA(cudaStreamCreateWithFlags(&cap.side, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
    {
        cudaStreamDestroy(cap.side);
        return cuda_fail(e, "cudaStreamBeginCapture");
    }
    int st = SPGNB_OK;
    long long cond = 0;
    const unsigned long long c0 = launches_so_far();
    for (int k = 0; k < b->opt.steps_per_graph && !st; k++)
        st = batch_step(b, energy_last && k == b->opt.steps_per_graph - 1, b->stream, &cap, &cond);
    // captured, not run: counted when the graph is launched (the conditional
    // bodies, which run only on rebuild and pruning steps, apart)
    const long long all = (long long)(launches_so_far() - c0);
    count_launches(-all);
    *kernels = all - cond;
    b->kernels_build = cond / std::max(1, b->opt.steps_per_graph);
    cap.close();
    e = cudaStreamEndCapture(b->stream, &g);
    cudaStreamDestroy(cap.side);
    if (st)
    {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    return SPGNB_OK;
}

int ensure_graphs(spgnb_batch* b)
{
    if (!b->opt.use_graphs) return SPGNB_OK;
    if (b->g_plain && b->g_energy && b->graph_tri == b->nl->triclinic) return SPGNB_OK;
    free_graphs(b);
    b->graph_tri = b->nl->triclinic;
    int st = capture(b, false, &b->g_plain, &b->kernels_plain);
    if (!st) st = capture(b, true, &b->g_energy, &b->kernels_energy);
    return st;
}

void free_batch(spgnb_batch* b)
{
    free_graphs(b);
    if (b->nl) spgnb_nl_destroy(b->nl);
    b->nl = nullptr;
    dfree(b->d_crd);
    dfree(b->d_vel);
    dfree(b->d_frc);
    dfree(b->d_crd_old);
    dfree(b->d_charge);
    dfree(b->d_inv_mass);
    dfree(b->d_type);
    dfree(b->d_atom_local);
    dfree(b->d_ex_start);
    dfree(b->d_ex_num);
    dfree(b->d_ex_list);
    dfree(b->d_waters);
    dfree(b->d_in_water);
    dfree(b->d_lambda);
    dfree(b->d_skin_hit);
    dfree(b->d_done);
    dfree(b->d_fps);
    dfree(b->d_totals);
    dfree(b->d_kin);
    dfree(b->d_ndof);
    dfree(b->d_steps);
    dfree(b->d_left);
    dfree(b->d_flags);
    dfree(b->d_slot_pos);
    dfree(b->d_slot_aux);
    dfree(b->d_t4);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (PinnedStage& ps : b->stages)
    {
        if (ps.ev) cudaEventDestroy(ps.ev);
        if (ps.p) cudaFreeHost(ps.p);
    }
    b->stages.clear();
    if (b->stream) cudaStreamDestroy(b->stream);
    b->stream = nullptr;
}

// A pinned upload buffer of at least `bytes` whose earlier copies are done.
int take_stage(spgnb_batch* b, size_t bytes, PinnedStage** out)
{
    PinnedStage* pick = nullptr;
    for (PinnedStage& ps : b->stages)
    {
        if (ps.busy && cudaEventQuery(ps.ev) == cudaSuccess) ps.busy = false;
        if (!ps.busy && ps.cap >= bytes && (!pick || ps.cap < pick->cap)) pick = &ps;
    }
    if (!pick)
    {
        for (PinnedStage& ps : b->stages)
            if (!ps.busy && (!pick || ps.cap > pick->cap)) pick = &ps;
        if (!pick)
        {
            b->stages.emplace_back();
            pick = &b->stages.back();
            SPGNB_CUDA(cudaEventCreateWithFlags(&pick->ev, cudaEventDisableTiming));
        }
        if (pick->p) SPGNB_CUDA(cudaFreeHost(pick->p));
        pick->p = nullptr;
        pick->cap = std::max(bytes, (size_t)1 << 20);
        cudaError_t e = cudaHostAlloc((void**)&pick->p, pick->cap, cudaHostAllocDefault);
        if (e != cudaSuccess)
        {
            pick->cap = 0;
            return cuda_fail(e, "cudaHostAlloc (upload staging)");
        }
    }
    pick->used = 0;
    *out = pick;
    return SPGNB_OK;
}

__global__ void k_set_flag(int* flags, int id) { flags[id] = 1; }

template <typename T>
int zalloc(T** d, size_t count)
{
    int st = dalloc(d, count);
    if (st) return st;
    SPGNB_CUDA(cudaMemset(*d, 0, sizeof(T) * std::max<size_t>(count, 1)));
    return SPGNB_OK;
}


// One system checked and laid out on the host, indices local to it.
struct Staged
{
    int N = 0;
    std::vector<float3> crd, vel;
    std::vector<float> charge, inv_mass;
    std::vector<int> type, ex_start, ex_num, ex_list;
    int water_begin = 0, water_numbers = 0;
    float mO = 0, mH = 0;
    ForceParams fp{};
    std::vector<float4> t4;  // the system's own coefficient table (empty: the batch's)
    double lr_factor = 0, volume = 0;
    float ndof = 1;
    SysHost sh;
    std::vector<int> run_start;
    std::vector<int2> runs;
};

int check_type_table(int T, const float* A, const float* B)
{
    if (T <= 0 || !A || !B) return fail(SPGNB_E_ARG, "batch: bad LJ type table");
    if (T > kMaxTypes) return fail(SPGNB_E_UNSUPPORTED, "batch: %d LJ types (at most %d)", T, kMaxTypes);
    return SPGNB_OK;
}

// The reference's triangular pair_A / pair_B as the square table.
std::vector<float2> square_table(int T, const float* A, const float* B)
{
    std::vector<float2> table((size_t)T * T);
    for (int p = 0; p < T; p++)
        for (int q = 0; q < T; q++)
        {
            const int hi = p > q ? p : q, lo = p > q ? q : p;
            table[(size_t)p * T + q] = make_float2(A[hi * (hi + 1) / 2 + lo], B[hi * (hi + 1) / 2 + lo]);
        }
    return table;
}

int stage(const spgnb_batch_system& y, int T0, const float* pair_A0, const float* pair_B0, int index, Staged& z)
{
    if (y.atom_type_numbers < 0)
        return fail(SPGNB_E_ARG, "batch: system %d has %d LJ types", index, y.atom_type_numbers);
    const bool own = y.atom_type_numbers > 0;
    const int T = own ? y.atom_type_numbers : T0;
    const float* pair_A = own ? y.h_pair_A : pair_A0;
    const float* pair_B = own ? y.h_pair_B : pair_B0;
    if (own)
    {
        const int st = check_type_table(T, pair_A, pair_B);
        if (st) return st;
        z.t4 = coefficient_table(square_table(T, pair_A, pair_B).data(), T);
    }
    if (y.atom_numbers <= 0 || !y.h_crd || !y.h_charge || !y.h_mass || !y.h_atom_type || !y.h_excluded_start ||
        !y.h_excluded_numbers || (y.excluded_total > 0 && !y.h_excluded_list) || y.water_begin < 0 ||
        y.water_numbers < 0 || y.water_begin + 3LL * y.water_numbers > y.atom_numbers || y.excluded_total < 0)
        return fail(SPGNB_E_ARG, "batch: system %d is incomplete", index);
    const int N = y.atom_numbers;
    z.N = N;
    z.crd.resize(N);
    z.vel.resize(N);
    z.charge.resize(N);
    z.inv_mass.resize(N);
    z.type.resize(N);
    z.ex_start.resize(N);
    z.ex_num.resize(N);
    std::vector<double> hist(T, 0.0);
    int moving = 0;
    for (int i = 0; i < N; i++)
    {
        z.crd[i] = make_float3(y.h_crd[3 * i], y.h_crd[3 * i + 1], y.h_crd[3 * i + 2]);
        z.vel[i] = y.h_vel ? make_float3(y.h_vel[3 * i], y.h_vel[3 * i + 1], y.h_vel[3 * i + 2]) : make_float3(0, 0, 0);
        z.charge[i] = y.h_charge[i];
        z.inv_mass[i] = y.h_mass[i] > 0.0f ? 1.0f / y.h_mass[i] : 0.0f;
        moving += y.h_mass[i] > 0.0f;
        const int t = y.h_atom_type[i];
        if (t < 0 || t >= T) return fail(SPGNB_E_ARG, "batch: system %d atom %d has type %d outside [0,%d)", index, i, t, T);
        z.type[i] = t;
        hist[t] += 1.0;
        const int cnt = y.h_excluded_numbers[i], st0 = y.h_excluded_start[i];
        if (cnt < 0 || (cnt > 0 && (st0 < 0 || st0 + cnt > y.excluded_total)))
            return fail(SPGNB_E_ARG, "batch: system %d atom %d has a bad exclusion range", index, i);
        z.ex_num[i] = cnt;
        z.ex_start[i] = (int)z.ex_list.size();
        for (int k = 0; k < cnt; k++)
        {
            const int j = y.h_excluded_list[st0 + k];
            if (j < 0 || j >= N) return fail(SPGNB_E_ARG, "batch: system %d excludes atom %d outside it", index, j);
            z.ex_list.push_back(j);
        }
    }
    z.water_begin = y.water_begin;
    z.water_numbers = y.water_numbers;
    if (y.water_numbers > 0)
    {
        z.mO = y.h_mass[y.water_begin];
        z.mH = y.h_mass[y.water_begin + 1];
    }
    z.ndof = (float)std::max(1, 3 * moving - 3 * y.water_numbers - 3);
    ForceParams& f = z.fp;
    f.rc2 = y.cutoff * y.cutoff;
    f.beta = y.pme_beta;
    f.beta3 = y.pme_beta * y.pme_beta * y.pme_beta;
    f.w_scale = y.pme_beta * y.pme_beta * SPGNB_EWALD_INV_W_MAX;
    const float zz = y.pme_beta * y.cutoff;
    f.use_fit = (zz * zz <= SPGNB_EWALD_W_MAX * 0.999f) ? 1 : 0;
    f.n_types = T;
    f.table_begin = 0;
    f.t4_begin = 0;  // a table of its own gets its place on admission
    // Total_C6_Get and the factor of Lennard_Jones_force.cpp:263-268
    double c6 = 0.0;
    for (int p = 0; p < T; p++)
        for (int q = 0; q < T; q++)
        {
            const int hi = p > q ? p : q, lo = p > q ? q : p;
            c6 += hist[p] * hist[q] * (double)pair_B[hi * (hi + 1) / 2 + lo];
        }
    float fac = (float)c6;
    fac *= -2.0f / 3.0f * 3.1415926535897932f / y.cutoff / y.cutoff / y.cutoff / 6.0f;
    z.lr_factor = fac;
    z.volume = (double)y.cell.a11 * y.cell.a22 * y.cell.a33;
    int st = nl_init_system(z.sh, N, y.cell, y.rcell, y.cutoff, y.skin, index);
    if (st) return st;
    return nl_system_runs(z.sh, z.run_start, z.runs);
}

// Device arrays for the capacities; every range free.
int create_common(spgnb_batch* b, const NLPoolSpec& spec, long long ex_cap, int w_cap, int T, const float* pair_A,
                  const float* pair_B, long long t4_cap)
{
    int st;
    b->S = spec.systems;
    b->n = spec.atoms;
    b->ex_cap = std::max(1LL, ex_cap);
    b->w_cap = std::max(1, w_cap);
    b->T = T;
    b->atom_pool.reset(b->n);
    b->ex_pool.reset(b->ex_cap);
    b->water_pool.reset(b->w_cap);
    b->rec.assign(b->S, SysRec{});
    b->h_flags.assign(b->S, 0);
    b->h_fps.assign(b->S + 1, ForceParams{});
    const std::vector<float4> t4 = coefficient_table(square_table(T, pair_A, pair_B).data(), T);
    b->t4_cap = std::max<long long>(t4_cap, (long long)t4.size());
    b->t4_pool.reset(b->t4_cap);
    b->t4_pool.alloc((long long)t4.size());  // the batch's table at element 0
    spgnb_nl_options nlo;
    spgnb_nl_default_options(&nlo);
    nlo.refresh_interval = 0;
    // the reference's grid gives each row's last cell the remainder of the
    // box, so in small boxes edge cells hold well over the reference's
    // 150-atom buckets; this engine has no such buckets, only the in-cell sort
    // capacity, so the grid flag is raised at that capacity
    nlo.max_atom_in_grid_numbers = kMaxCellAtoms;
    nlo.skin_permit = b->opt.skin_permit;
    nlo.export_atom_groups = 0;
    nlo.prune_buffer = b->opt.prune_buffer;
    const size_t n = b->n, S1 = b->S + 1;
    if ((st = nl_create_pool(spec, &nlo, &b->nl)) || (st = zalloc(&b->d_crd, n)) || (st = zalloc(&b->d_vel, n)) ||
        (st = zalloc(&b->d_frc, n)) || (st = zalloc(&b->d_crd_old, n)) || (st = zalloc(&b->d_charge, n)) ||
        (st = zalloc(&b->d_inv_mass, n)) || (st = zalloc(&b->d_type, n)) || (st = zalloc(&b->d_atom_local, n)) ||
        (st = zalloc(&b->d_ex_start, n)) || (st = zalloc(&b->d_ex_num, n)) ||
        (st = zalloc(&b->d_ex_list, (size_t)b->ex_cap)) || (st = dalloc(&b->d_waters, (size_t)b->w_cap)) ||
        (st = dalloc(&b->d_t4, (size_t)b->t4_cap)) || (st = zalloc(&b->d_fps, S1)) ||
        (st = zalloc(&b->d_totals, 8 * S1)) || (st = zalloc(&b->d_kin, S1)) || (st = zalloc(&b->d_ndof, S1)) ||
        (st = zalloc(&b->d_in_water, n)) || (st = dalloc(&b->d_lambda, S1)) || (st = zalloc(&b->d_skin_hit, S1)) ||
        (st = zalloc(&b->d_done, 1)) ||
        (st = zalloc(&b->d_steps, S1)) || (st = zalloc(&b->d_left, S1)) || (st = zalloc(&b->d_flags, S1)) ||
        (st = dalloc(&b->d_slot_pos, (size_t)b->nl->clusters_cap * kClusterSize + 1)) ||
        (st = dalloc(&b->d_slot_aux, (size_t)b->nl->clusters_cap * kClusterSize + 1)))
        return st;
    SPGNB_CUDA(cudaMemcpy(b->d_t4, t4.data(), sizeof(float4) * t4.size(), cudaMemcpyHostToDevice));
    SPGNB_CUDA(cudaMemset(b->d_waters, 0xff, sizeof(int) * b->w_cap));
    {
        const std::vector<float> ones(S1, 1.0f);
        SPGNB_CUDA(cudaMemcpy(b->d_lambda, ones.data(), sizeof(float) * S1, cudaMemcpyHostToDevice));
    }
    SPGNB_CUDA(cudaDeviceSynchronize());
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    return SPGNB_OK;
}

int admit_staged(spgnb_batch* b, Staged& z, int steps, int* id)
{
    int st;
    if (b->fit && !z.fp.use_fit)
        return fail(SPGNB_E_UNSUPPORTED, "batch: beta * cutoff of this system is outside the pool's fitted range");
    if (z.water_numbers > 0 && b->have_water && (z.mO != b->mO || z.mH != b->mH))
        return fail(SPGNB_E_ARG, "batch: the rigid waters of a pool share one mass pair");
    if (z.fp.n_types > b->max_T)
        return fail(SPGNB_E_UNSUPPORTED, "batch: a type table of %d types (the pool takes at most %d)", z.fp.n_types,
                    b->max_T);
    cudaStream_t s = b->stream;
    const long long nt4 = (long long)z.t4.size();
    const long long tb = nt4 ? b->t4_pool.alloc(nt4) : 0;
    if (tb < 0) return fail(SPGNB_E_OOM, "batch: no room for the system's type table now");
    const long long ab = b->atom_pool.alloc(z.N);
    if (ab < 0)
    {
        b->t4_pool.release(tb, nt4);
        return fail(SPGNB_E_OOM, "batch: no room for %d atoms now", z.N);
    }
    const long long ne = (long long)z.ex_list.size();
    const long long eb = b->ex_pool.alloc(ne);
    const long long wb = eb < 0 ? -1 : b->water_pool.alloc(z.water_numbers);
    if (eb < 0 || wb < 0)
    {
        if (eb >= 0) b->ex_pool.release(eb, ne);
        b->atom_pool.release(ab, z.N);
        b->t4_pool.release(tb, nt4);
        return fail(SPGNB_E_OOM, "batch: no room for the exclusions or waters now");
    }
    z.fp.t4_begin = (int)tb;
    z.sh.atom_begin = (int)ab;
    // every upload of this admission goes through one pinned buffer, so the
    // copies queue behind the work in flight instead of waiting for it
    const size_t N = z.N;
    const size_t need = N * (2 * sizeof(float3) + 6 * sizeof(int) + 1) + ne * sizeof(int) +
                        z.water_numbers * sizeof(int) + sizeof(ForceParams) + 3 * sizeof(int) + sizeof(float) + 16 * 24 +
                        nt4 * sizeof(float4) + nl_admit_upload_bytes(z.sh, z.runs.size());
    PinnedStage* ps = nullptr;
    if ((st = take_stage(b, need, &ps)))
    {
        b->water_pool.release(wb, z.water_numbers);
        b->ex_pool.release(eb, ne);
        b->atom_pool.release(ab, z.N);
        b->t4_pool.release(tb, nt4);
        return st;
    }
    Uploader up{ps};
    int sid = -1;
    // after the first queued copy a failure must keep the pinned buffer from
    // being reused until the copies already queued from it have run, and hand
    // back the ranges (and the system id, when one was taken)
    auto bail = [&](int code) {
        cudaEventRecord(ps->ev, s);
        ps->busy = true;
        if (sid >= 0) nl_retire(b->nl, sid, s);
        b->water_pool.release(wb, z.water_numbers);
        b->ex_pool.release(eb, ne);
        b->atom_pool.release(ab, z.N);
        b->t4_pool.release(tb, nt4);
        return code;
    };
    st = nl_admit(b->nl, z.sh, &z.run_start, &z.runs, s, &sid, up);
    if (st)
    {
        sid = -1;  // nl_admit has released what it took
        return bail(st == SPGNB_E_OOM ? fail(SPGNB_E_OOM, "batch: no free system id, cells or clusters now") : st);
    }
    if (z.water_numbers > 0 && !b->have_water)
    {
        b->have_water = true;
        b->mO = z.mO;
        b->mH = z.mH;
        b->rc = 0.5f * b->opt.water_dhh;
        const float h = sqrtf(b->opt.water_doh * b->opt.water_doh - b->rc * b->rc);
        b->ra = 2.0f * b->mH * h / (b->mO + 2.0f * b->mH);
        b->rb = h - b->ra;
        free_graphs(b);  // the step now includes SETTLE
    }
    const int a0 = (int)ab;
    std::vector<int> own(z.N), ex_start(z.N), ex_list(ne), waters(z.water_numbers);
    std::vector<unsigned char> in_water(z.N, 0);
    for (int k = 0; k < 3 * z.water_numbers; k++) in_water[z.water_begin + k] = 1;
    for (int i = 0; i < z.N; i++)
    {
        own[i] = a0 + i;
        ex_start[i] = (int)eb + z.ex_start[i];
    }
    for (long long k = 0; k < ne; k++) ex_list[k] = a0 + z.ex_list[k];
    for (int w = 0; w < z.water_numbers; w++) waters[w] = a0 + z.water_begin + 3 * w;
    const std::vector<ForceParams> fp(1, z.fp);
    const std::vector<float> ndof(1, z.ndof);
    const std::vector<int> left(1, steps > 0 ? steps : -1);
    const std::vector<float> lambda(1, 1.0f);
    auto putv = [&](auto* dst, size_t off, const auto& v) { return up.put(dst + off, v.data(), sizeof(v[0]) * v.size(), s); };
    if ((st = putv(b->d_crd, ab, z.crd)) || (st = putv(b->d_vel, ab, z.vel)) ||
        (st = putv(b->d_charge, ab, z.charge)) || (st = putv(b->d_inv_mass, ab, z.inv_mass)) ||
        (st = putv(b->d_type, ab, z.type)) || (st = putv(b->d_atom_local, ab, own)) ||
        (st = putv(b->d_in_water, ab, in_water)) || (st = putv(b->d_lambda, sid, lambda)) ||
        (st = putv(b->d_ex_start, ab, ex_start)) || (st = putv(b->d_ex_num, ab, z.ex_num)) ||
        (st = putv(b->d_ex_list, eb, ex_list)) || (st = putv(b->d_waters, wb, waters)) ||
        (st = putv(b->d_fps, sid, fp)) || (st = putv(b->d_ndof, sid, ndof)) || (st = putv(b->d_left, sid, left)) ||
        (nt4 && (st = putv(b->d_t4, tb, z.t4))))
        return bail(st);
    SPGNB_CUDA(cudaMemsetAsync(b->d_frc + ab, 0, sizeof(float3) * z.N, s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_steps + sid, 0, sizeof(int), s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_kin + sid, 0, sizeof(long long), s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_skin_hit + sid, 0, sizeof(int), s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_totals + 8 * (size_t)sid, 0, sizeof(long long) * 8, s));
    k_set_flag<<<1, 1, 0, s>>>(b->d_flags, sid);
    SPGNB_CHECK_LAUNCH("k_set_flag");
    SPGNB_CUDA(cudaEventRecord(ps->ev, s));
    ps->busy = true;
    b->h_fps[sid] = z.fp;
    SysRec& r = b->rec[sid];
    r.live = true;
    r.atom_begin = a0;
    r.atom_count = z.N;
    r.ex_begin = eb;
    r.ex_count = ne;
    r.w_begin = (int)wb;
    r.w_count = z.water_numbers;
    r.lr_factor = z.lr_factor;
    r.volume = z.volume;
    r.t4_begin = tb;
    r.t4_count = nt4;
    b->h_flags[sid] = 1;
    b->pending = true;
    *id = sid;
    return SPGNB_OK;
}

// Batch-side device bytes for the capacities.
double batch_bytes(long long atoms, long long ex, long long waters, long long slots, int S, long long t4_cap)
{
    return (double)atoms * (12 * 4 + 4 * 6) + ex * 4.0 + waters * 4.0 + slots * 32.0 + (S + 1.0) * (32 + 64 + 8 + 16) +
           t4_cap * 16.0;
}

// Pool capacities for `atoms` atoms under the pool options.
NLPoolSpec pool_spec(const spgnb_batch_pool_options& po, float prune_buffer, int atoms)
{
    NLPoolSpec sp;
    const double gl = 0.5 * (po.min_cutoff + po.skin);
    const double cells_per_atom = 1.25 / (po.density * gl * gl * gl);
    sp.systems = po.max_systems;
    sp.atoms = atoms;
    sp.cells = (int)std::min<double>(atoms * cells_per_atom + 2.0 * po.max_systems + 64, (1 << 28) - 1);
    sp.clusters = (int)std::min<double>(atoms / (double)kClusterSize + sp.cells + po.max_systems, 0x7fffffff);
    sp.runs = (long long)sp.cells * 48;
    double pc, pa;
    nl_capacity_for(po.density * 1.1, 1e30, po.max_cutoff, po.skin, prune_buffer, &pc, &pa);
    sp.table_cap = std::max((int)(pc * 1.3) + 64, 128);
    sp.list_cap = list_cap_for(pa);
    sp.prune_rc = po.max_cutoff;
    return sp;
}

double pool_bytes(const spgnb_batch_pool_options& po, float prune_buffer, int atoms, long long t4_cap)
{
    const NLPoolSpec sp = pool_spec(po, prune_buffer, atoms);
    spgnb_nl probe;
    probe.S = sp.systems;
    probe.n_cap = sp.atoms;
    probe.G = sp.cells;
    probe.clusters_cap = sp.clusters;
    probe.runs_cap = sp.runs;
    probe.table_cap = sp.table_cap;
    probe.list_cap = sp.list_cap;
    probe.opt.export_atom_groups = 0;
    const long long ex = po.max_excluded > 0 ? po.max_excluded : 2LL * atoms;
    const long long w = po.max_waters > 0 ? po.max_waters : atoms / 3;
    return (double)nl_device_bytes(&probe) +
           batch_bytes(atoms, ex, w, (long long)sp.clusters * kClusterSize, sp.systems, t4_cap);
}

}  // namespace
}  // namespace spgnb

using namespace spgnb;

extern "C" {

void spgnb_batch_default_options(spgnb_batch_options* o)
{
    if (!o) return;
    o->dt = 0.002f;
    o->water_doh = 0.9572f;
    o->water_dhh = 1.5139f;
    o->skin_permit = 0.5f;
    o->prune_buffer = 1.0f;
    o->steps_per_graph = 10;
    o->use_graphs = 1;
    o->thermostat_tau = 0.0f;
    o->temperature = 300.0f;
    o->refresh_interval = 0;
}

void spgnb_batch_pool_default_options(spgnb_batch_pool_options* o)
{
    if (!o) return;
    o->max_systems = 1024;
    o->max_atoms = 0;
    o->max_excluded = 0;
    o->max_waters = 0;
    o->max_cutoff = 12.0f;
    o->min_cutoff = 8.0f;
    o->skin = 2.0f;
    o->density = 0.1003f;
    o->hbm_budget_bytes = 120e9;
    o->max_types = 0;
    o->type_table_bytes = 64.0 * (1 << 20);
}

int spgnb_batch_set_thermostat(spgnb_batch* b, float tau, float temperature)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_set_thermostat: NULL handle");
    if (!(tau >= 0.0f) || !(temperature >= 0.0f)) return fail(SPGNB_E_ARG, "spgnb_batch_set_thermostat: bad values");
    b->opt.thermostat_tau = tau;
    b->opt.temperature = temperature;
    free_graphs(b);
    // the velocity scale starts again from 1 (the sums from zero)
    const std::vector<float> ones(b->S + 1, 1.0f);
    SPGNB_CUDA(cudaMemcpyAsync(b->d_lambda, ones.data(), sizeof(float) * ones.size(), cudaMemcpyHostToDevice,
                               b->stream));
    SPGNB_CUDA(cudaMemsetAsync(b->d_kin, 0, sizeof(long long) * (b->S + 1), b->stream));
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    return SPGNB_OK;
}

static spgnb_batch* new_batch(const spgnb_batch_options* opt, int T, const float* A, const float* B)
{
    spgnb_batch* b = new spgnb_batch();
    if (opt)
        b->opt = *opt;
    else
        spgnb_batch_default_options(&b->opt);
    if (b->opt.steps_per_graph <= 0) b->opt.steps_per_graph = 1;
    const int P = T * (T + 1) / 2;
    b->h_pair_A.assign(A, A + P);
    b->h_pair_B.assign(B, B + P);
    return b;
}

int spgnb_batch_create(int n_systems, const spgnb_batch_system* systems, int atom_type_numbers,
                       const float* h_pair_A, const float* h_pair_B, const spgnb_batch_options* opt,
                       spgnb_batch** out)
{
    if (!out) return fail(SPGNB_E_ARG, "spgnb_batch_create: out is NULL");
    *out = nullptr;
    if (n_systems <= 0 || !systems) return fail(SPGNB_E_ARG, "spgnb_batch_create: bad arguments");
    const int T = atom_type_numbers;
    int st = check_type_table(T, h_pair_A, h_pair_B);
    if (st) return st;
    spgnb_batch* b = new_batch(opt, T, h_pair_A, h_pair_B);
    const std::vector<float>& pa = b->h_pair_A;
    const std::vector<float>& pb = b->h_pair_B;
    std::vector<Staged> z(n_systems);
    long long atoms = 0, ex = 0, waters = 0, cells = 0, clusters = 0, runs = 0;
    long long t4_cap = (long long)T * T * T;
    b->max_T = T;
    double per_cluster = 0, per_list = 0;
    float rcmax = 0;
    for (int k = 0; k < n_systems && !st; k++)
    {
        if ((st = stage(systems[k], T, pa.data(), pb.data(), k, z[k]))) break;
        const Staged& y = z[k];
        t4_cap += (long long)y.t4.size();
        b->max_T = std::max(b->max_T, y.fp.n_types);
        atoms += y.N;
        ex += (long long)y.ex_list.size();
        waters += y.water_numbers;
        const int G = y.sh.cells();
        cells += G + 1;
        clusters += y.N / kClusterSize + G + 1;
        runs += (long long)y.runs.size();
        double pc, pw;
        nl_capacity_for(y.N / y.volume, y.N, systems[k].cutoff, systems[k].skin, b->opt.prune_buffer, &pc, &pw);
        per_cluster = std::max(per_cluster, pc);
        per_list = std::max(per_list, pw);
        rcmax = std::max(rcmax, systems[k].cutoff);
        if (!y.fp.use_fit) b->fit = false;
    }
    if (!st && atoms > (1LL << 28)) st = fail(SPGNB_E_UNSUPPORTED, "spgnb_batch_create: %lld atoms in total", atoms);
    if (!st && (clusters + 1) * kClusterSize > kMaxSlots)
        st = fail(SPGNB_E_UNSUPPORTED, "batch: %lld atoms in %lld cells exceed the %d-slot limit of the lists", atoms,
                  cells, kMaxSlots);
    if (st)
    {
        delete b;
        return st;
    }
    NLPoolSpec spec;
    spec.systems = n_systems;
    spec.atoms = (int)atoms;
    spec.cells = (int)cells;
    spec.clusters = (int)clusters;
    spec.runs = std::max(1LL, runs);
    spec.table_cap = std::max((int)(per_cluster * 1.3) + 64, 128);
    spec.list_cap = list_cap_for(per_list);
    spec.prune_rc = rcmax;
    if (!(st = create_common(b, spec, ex, (int)waters, T, pa.data(), pb.data(), t4_cap)))
        for (int k = 0; k < n_systems && !st; k++)
        {
            int id = -1;
            st = admit_staged(b, z[k], 0, &id);
            if (!st && id != k) st = fail(SPGNB_E_STATE, "spgnb_batch_create: system %d got id %d", k, id);
            z[k] = Staged{};
        }
    if (!st) st = settle_pending(b);
    if (!st)
    {
        cudaError_t e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "spgnb_batch_create");
    }
    if (st)
    {
        free_batch(b);
        delete b;
        return st;
    }
    *out = b;
    return SPGNB_OK;
}

int spgnb_batch_create_pool(const spgnb_batch_pool_options* pool, int atom_type_numbers, const float* h_pair_A,
                            const float* h_pair_B, const spgnb_batch_options* opt, spgnb_batch** out)
{
    if (!out) return fail(SPGNB_E_ARG, "spgnb_batch_create_pool: out is NULL");
    *out = nullptr;
    const int T = atom_type_numbers;
    int st = check_type_table(T, h_pair_A, h_pair_B);
    if (st) return st;
    spgnb_batch_pool_options po;
    if (pool)
        po = *pool;
    else
        spgnb_batch_pool_default_options(&po);
    if (po.max_systems <= 0 || !(po.max_cutoff > 0.0f) || !(po.min_cutoff > 0.0f) || po.min_cutoff > po.max_cutoff ||
        !(po.skin >= 0.0f) || !(po.density > 0.0f) || (po.max_atoms <= 0 && !(po.hbm_budget_bytes > 0.0)) ||
        po.max_types < 0 || po.max_types > kMaxTypes || !(po.type_table_bytes >= 0.0))
        return fail(SPGNB_E_ARG, "spgnb_batch_create_pool: bad pool options");
    spgnb_batch* b = new_batch(opt, T, h_pair_A, h_pair_B);
    b->max_T = std::max(T, po.max_types);
    const long long t4_cap = (long long)T * T * T + (long long)(po.type_table_bytes / sizeof(float4));
    int atoms = po.max_atoms;
    // the largest atom count whose clusters fit the slot field of the lists
    {
        int lo = 1024, hi = 1 << 28;
        while (hi - lo > 1024)
        {
            const int mid = lo + (hi - lo) / 2;
            const NLPoolSpec sp = pool_spec(po, b->opt.prune_buffer, mid);
            if (((long long)sp.clusters + 1) * kClusterSize <= kMaxSlots)
                lo = mid;
            else
                hi = mid;
        }
        const int slot_limit = lo;
        if (atoms <= 0)
        {
            // linear in the atom count: solve bytes(atoms) = budget
            const double b1 = pool_bytes(po, b->opt.prune_buffer, 1 << 20, t4_cap);
            const double b2 = pool_bytes(po, b->opt.prune_buffer, 1 << 21, t4_cap);
            const double per_atom = (b2 - b1) / (double)(1 << 20);
            const double fixed = b1 - per_atom * (1 << 20);
            atoms = (int)std::min<double>((po.hbm_budget_bytes - fixed) / per_atom, (double)(1 << 28));
        }
        atoms = std::min(atoms, slot_limit);
        atoms &= ~1023;
    }
    if (atoms < 1024)
    {
        delete b;
        return fail(SPGNB_E_ARG, "spgnb_batch_create_pool: the budget holds fewer than 1024 atoms");
    }
    const NLPoolSpec spec = pool_spec(po, b->opt.prune_buffer, atoms);
    const long long ex = po.max_excluded > 0 ? po.max_excluded : 2LL * atoms;
    const int w = po.max_waters > 0 ? po.max_waters : atoms / 3;
    b->fit = true;
    if ((st = create_common(b, spec, ex, w, T, b->h_pair_A.data(), b->h_pair_B.data(), t4_cap)))
    {
        free_batch(b);
        delete b;
        return st;
    }
    *out = b;
    return SPGNB_OK;
}

int spgnb_batch_admit(spgnb_batch* b, const spgnb_batch_system* sys, int steps, int* id)
{
    if (!b || !sys || !id) return fail(SPGNB_E_ARG, "spgnb_batch_admit: NULL argument");
    *id = -1;
    Staged z;
    int st = stage(*sys, b->T, b->h_pair_A.data(), b->h_pair_B.data(), -1, z);
    if (st) return st;
    return admit_staged(b, z, steps, id);
}

int spgnb_batch_retire(spgnb_batch* b, int id)
{
    if (!b || id < 0 || id >= b->S || !b->rec[id].live) return fail(SPGNB_E_ARG, "spgnb_batch_retire: bad system id");
    cudaStream_t s = b->stream;
    SysRec& r = b->rec[id];
    int st = nl_retire(b->nl, id, s);
    if (st) return st;
    // parked atoms: at rest, massless, no force; free water entries -1
    SPGNB_CUDA(cudaMemsetAsync(b->d_vel + r.atom_begin, 0, sizeof(float3) * r.atom_count, s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_frc + r.atom_begin, 0, sizeof(float3) * r.atom_count, s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_inv_mass + r.atom_begin, 0, sizeof(float) * r.atom_count, s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_charge + r.atom_begin, 0, sizeof(float) * r.atom_count, s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_ex_num + r.atom_begin, 0, sizeof(int) * r.atom_count, s));
    if (r.w_count) SPGNB_CUDA(cudaMemsetAsync(b->d_waters + r.w_begin, 0xff, sizeof(int) * r.w_count, s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_left + id, 0, sizeof(int), s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_steps + id, 0, sizeof(int), s));
    SPGNB_CUDA(cudaMemsetAsync(b->d_totals + 8 * (size_t)id, 0, sizeof(long long) * 8, s));
    b->atom_pool.release(r.atom_begin, r.atom_count);
    b->ex_pool.release(r.ex_begin, r.ex_count);
    b->water_pool.release(r.w_begin, r.w_count);
    b->t4_pool.release(r.t4_begin, r.t4_count);
    b->h_flags[id] = 0;
    r = SysRec{};
    return SPGNB_OK;
}

int spgnb_batch_evaluate(spgnb_batch* b, const int* ids, int n)
{
    if (!b || (n > 0 && !ids)) return fail(SPGNB_E_ARG, "spgnb_batch_evaluate: NULL argument");
    int st = settle_pending(b);
    if (st) return st;
    bool any = false;
    for (int k = 0; k < n; k++)
    {
        if (ids[k] < 0 || ids[k] >= b->S || !b->rec[ids[k]].live)
            return fail(SPGNB_E_ARG, "spgnb_batch_evaluate: system %d is not in the pool", ids[k]);
        b->h_flags[ids[k]] = 1;
        any = true;
    }
    if (!any) return SPGNB_OK;
    cudaStream_t s = b->stream;
    SPGNB_CUDA(cudaMemcpyAsync(b->d_flags, b->h_flags.data(), sizeof(int) * b->S, cudaMemcpyHostToDevice, s));
    st = batch_force(b, 1, s, b->d_flags);
    if (st) return st;
    SPGNB_CUDA(cudaMemsetAsync(b->d_flags, 0, sizeof(int) * b->S, s));
    SPGNB_CUDA(cudaStreamSynchronize(s));  // h_flags is the copy's source
    std::fill(b->h_flags.begin(), b->h_flags.end(), 0);
    return SPGNB_OK;
}

int spgnb_batch_progress(spgnb_batch* b, int* steps_done, int* steps_left)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_progress: NULL handle");
    std::vector<int> d(b->S), l(b->S);
    SPGNB_CUDA(cudaMemcpyAsync(d.data(), b->d_steps, sizeof(int) * b->S, cudaMemcpyDeviceToHost, b->stream));
    SPGNB_CUDA(cudaMemcpyAsync(l.data(), b->d_left, sizeof(int) * b->S, cudaMemcpyDeviceToHost, b->stream));
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    for (int k = 0; k < b->S; k++)
    {
        const bool live = b->rec[k].live;
        if (steps_done) steps_done[k] = live ? d[k] : 0;
        if (steps_left) steps_left[k] = live ? l[k] : 0;
    }
    return SPGNB_OK;
}

int spgnb_batch_capacity(spgnb_batch* b, int* max_systems, long long* max_atoms, long long* free_atoms,
                         double* device_bytes)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_capacity: NULL handle");
    if (max_systems) *max_systems = b->S;
    if (max_atoms) *max_atoms = b->n;
    if (free_atoms) *free_atoms = b->atom_pool.available();
    if (device_bytes)
        *device_bytes = (double)nl_device_bytes(b->nl) +
                        batch_bytes(b->n, b->ex_cap, b->w_cap, (long long)b->nl->clusters_cap * kClusterSize, b->S, b->t4_cap);
    return SPGNB_OK;
}

int spgnb_batch_run(spgnb_batch* b, int steps, int energy_interval)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_run: NULL handle");
    int st = settle_pending(b);
    if (st) return st;
    if (steps <= 0) return SPGNB_OK;
    if ((st = ensure_graphs(b))) return st;
    const int K = b->opt.steps_per_graph;
    int done = 0;
    while (done < steps)
    {
        const long long at = b->steps_done;
        if (b->opt.use_graphs && steps - done >= K)
        {
            const bool en = energy_interval > 0 && (at + K) % energy_interval == 0;
            bool any_inside = false;
            if (energy_interval > 0)
                for (int k = 1; k < K; k++)
                    if ((at + k) % energy_interval == 0) any_inside = true;
            if (!any_inside)
            {
                SPGNB_CUDA(cudaGraphLaunch(en ? b->g_energy : b->g_plain, b->stream));
                count_launches(en ? b->kernels_energy : b->kernels_plain);
                b->steps_done += K;
                done += K;
                continue;
            }
        }
        const bool en = energy_interval > 0 && (at + 1) % energy_interval == 0;
        if ((st = batch_step(b, en, b->stream))) return st;
        b->steps_done += 1;
        done += 1;
    }
    return SPGNB_OK;
}

int spgnb_batch_energies(spgnb_batch* b, double* out)
{
    if (!b || !out) return fail(SPGNB_E_ARG, "spgnb_batch_energies: NULL argument");
    int st = settle_pending(b);
    if (st) return st;
    std::vector<long long> h(8 * (size_t)b->S);
    SPGNB_CUDA(cudaMemcpyAsync(h.data(), b->d_totals, sizeof(long long) * h.size(), cudaMemcpyDeviceToHost, b->stream));
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    for (int s = 0; s < b->S; s++)
    {
        const long long* t = &h[8 * (size_t)s];
        double* o = out + 9 * (size_t)s;
        const SysRec& r = b->rec[s];
        o[0] = (double)t[0] / kEnergyScale;
        o[1] = r.live ? r.lr_factor / r.volume : 0.0;
        o[2] = (double)t[1] / kEnergyScale;
        for (int q = 0; q < 6; q++) o[3 + q] = (double)t[2 + q] / kEnergyScale;
    }
    return SPGNB_OK;
}

int spgnb_batch_download(spgnb_batch* b, int sys, float* h_crd, float* h_vel, float* h_frc)
{
    if (!b || sys < 0 || sys >= b->S || !b->rec[sys].live) return fail(SPGNB_E_ARG, "spgnb_batch_download: bad system");
    int st = settle_pending(b);
    if (st) return st;
    const size_t off = b->rec[sys].atom_begin, cnt = b->rec[sys].atom_count;
    if (h_crd)
        SPGNB_CUDA(cudaMemcpyAsync(h_crd, b->d_crd + off, sizeof(float3) * cnt, cudaMemcpyDeviceToHost, b->stream));
    if (h_vel)
        SPGNB_CUDA(cudaMemcpyAsync(h_vel, b->d_vel + off, sizeof(float3) * cnt, cudaMemcpyDeviceToHost, b->stream));
    if (h_frc)
    {
        // the last force pass's forces, still in the staging for the next step
        k_forces_out<<<((int)cnt + 255) / 256, 256, 0, b->stream>>>((int)off, (int)cnt, b->nl->d_atom_slot,
                                                                     b->nl->d_facc, b->d_frc);
        SPGNB_CHECK_LAUNCH("k_forces_out");
        SPGNB_CUDA(cudaMemcpyAsync(h_frc, b->d_frc + off, sizeof(float3) * cnt, cudaMemcpyDeviceToHost, b->stream));
    }
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    return SPGNB_OK;
}

int spgnb_batch_stats(spgnb_batch* b, long long* steps, long long* rebuilds, long long* prunings, int* overflow)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_stats: NULL handle");
    int h[kCntSize];
    SPGNB_CUDA(cudaMemcpyAsync(h, b->nl->d_counters, sizeof(h), cudaMemcpyDeviceToHost, b->stream));
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    if (steps) *steps = b->steps_done;
    if (rebuilds) *rebuilds = h[kCntBuilds];
    if (prunings) *prunings = h[kCntPrunes];
    if (overflow) *overflow = h[kCntOverflow];
    return SPGNB_OK;
}

int spgnb_batch_autotune(spgnb_batch* b, int steps_per_candidate, float* chosen_buffer)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_autotune: NULL handle");
    if (steps_per_candidate <= 0) steps_per_candidate = 20;
    cudaEvent_t e0, e1;
    SPGNB_CUDA(cudaEventCreate(&e0));
    SPGNB_CUDA(cudaEventCreate(&e1));
    // steps of the current configuration per ms, warmed up (graphs captured,
    // a pruning with a changed buffer done) before the timed steps; the
    // timed count is a whole number of graphs
    auto time_steps = [&](float* ms_per_step) -> int {
        free_graphs(b);
        int st = spgnb_batch_run(b, b->opt.steps_per_graph, 0);
        if (st) return st;
        const int K = std::max(1, steps_per_candidate / b->opt.steps_per_graph) * b->opt.steps_per_graph;
        SPGNB_CUDA(cudaEventRecord(e0, b->stream));
        if ((st = spgnb_batch_run(b, K, 0))) return st;
        SPGNB_CUDA(cudaEventRecord(e1, b->stream));
        SPGNB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        SPGNB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        *ms_per_step = ms / K;
        return SPGNB_OK;
    };
    int st = SPGNB_OK;
    float best_ms = 1e30f;
    // one setting at a time, the others at their best so far
    auto tune = [&](auto set, const auto& candidates) {
        auto best = candidates[0];
        bool any = false;
        for (auto c : candidates)
        {
            if (!set(c)) continue;
            float ms = 0;
            if ((st = time_steps(&ms))) return;
            if (!any || ms < best_ms)
            {
                best_ms = ms;
                best = c;
                any = true;
            }
        }
        set(best);
    };
    // the prune buffer, up to the one the lists were sized for
    const float maxb = b->opt.prune_buffer;
    const std::vector<float> buffers = {0.4f, 0.6f, 0.8f, 1.0f, 1.3f, 1.6f};
    tune([&](float c) {
        if (c > maxb + 1e-6f) return false;
        b->nl->opt.prune_buffer = c;
        b->opt.prune_buffer = c;
        return nl_prune_all(b->nl, b->stream) == SPGNB_OK;
    }, buffers);
    if (!st)
    {
        // the force kernel's resident blocks per SM (0: all that fit)
        const std::vector<int> pair_bps = {0, 3, 2};
        best_ms = 1e30f;
        tune([&](int c) { b->pair_bps = c; return true; }, pair_bps);
    }
    if (!st)
    {
        // the pruning kernel's blocks per SM
        const std::vector<int> prune_bps = {5, 3, 8};
        best_ms = 1e30f;
        tune([&](int c) { b->prune_bps = c; return true; }, prune_bps);
    }
    if (!st)
    {
        const std::vector<int> graph_steps = {10, 5, 20};
        best_ms = 1e30f;
        tune([&](int c) { b->opt.steps_per_graph = c; return true; }, graph_steps);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    b->tuned_ms = best_ms;
    free_graphs(b);
    if ((st = nl_prune_all(b->nl, b->stream))) return st;
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    if (chosen_buffer) *chosen_buffer = b->opt.prune_buffer;
    return SPGNB_OK;
}

int spgnb_batch_set_tuning(spgnb_batch* b, const spgnb_batch_tuning* t)
{
    if (!b || !t) return fail(SPGNB_E_ARG, "spgnb_batch_set_tuning: NULL argument");
    if (!(t->prune_buffer > 0.0f) || t->prune_buffer > b->opt.prune_buffer + 1e-6f || t->pair_blocks_per_sm < 0 ||
        t->prune_blocks_per_sm < 0 || t->steps_per_graph <= 0)
        return fail(SPGNB_E_ARG, "spgnb_batch_set_tuning: bad values (prune buffer in (0, %g])", b->opt.prune_buffer);
    b->nl->opt.prune_buffer = t->prune_buffer;
    b->opt.prune_buffer = t->prune_buffer;
    b->pair_bps = t->pair_blocks_per_sm;
    b->prune_bps = t->prune_blocks_per_sm;
    b->opt.steps_per_graph = t->steps_per_graph;
    free_graphs(b);
    return nl_prune_all(b->nl, b->stream);
}

int spgnb_batch_launch_counts(spgnb_batch* b, int* per_step, int* per_rebuild)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_launch_counts: NULL handle");
    int st = ensure_graphs(b);
    if (st) return st;
    if (per_step) *per_step = (int)(b->kernels_plain / std::max(1, b->opt.steps_per_graph));
    if (per_rebuild) *per_rebuild = (int)b->kernels_build;
    return SPGNB_OK;
}

int spgnb_batch_get_tuning(spgnb_batch* b, spgnb_batch_tuning* out)
{
    if (!b || !out) return fail(SPGNB_E_ARG, "spgnb_batch_get_tuning: NULL argument");
    out->prune_buffer = b->opt.prune_buffer;
    out->pair_blocks_per_sm = b->pair_bps;
    out->prune_blocks_per_sm = b->prune_bps > 0 ? b->prune_bps : 5;
    out->steps_per_graph = b->opt.steps_per_graph;
    out->ms_per_step = b->tuned_ms;
    return SPGNB_OK;
}

void* spgnb_batch_stream(spgnb_batch* b) { return b ? (void*)b->stream : nullptr; }

int spgnb_batch_check_overflow(spgnb_batch* b, int* regrown)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_check_overflow: NULL handle");
    if (regrown) *regrown = 0;
    int flags = 0;
    SPGNB_CUDA(cudaMemcpyAsync(&flags, b->nl->d_counters + kCntOverflow, sizeof(int), cudaMemcpyDeviceToHost,
                               b->stream));
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    if (!flags) return SPGNB_OK;
    if (flags & kOvfCellHard)
        return fail(SPGNB_E_OVERFLOW, "batch: a grid cell holds more than %d atoms (a system collapsed?)",
                    kMaxCellAtoms);
    int st = nl_regrow(b->nl, flags);
    if (st) return st;
    free_graphs(b);
    if ((st = nl_queue_build(b->nl, b->n, b->d_crd, b->d_atom_local, b->d_ex_start, b->d_ex_list, b->d_ex_num,
                             kBuildForced, b->stream)) ||
        (st = batch_force(b, 0, b->stream)))
        return st;
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    if (regrown) *regrown = 1;
    return SPGNB_OK;
}

int spgnb_batch_destroy(spgnb_batch* b)
{
    if (!b) return SPGNB_OK;
    free_batch(b);
    delete b;
    return SPGNB_OK;
}

}  // extern "C"
