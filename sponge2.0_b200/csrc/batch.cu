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

struct spgnb_batch
{
    int S = 0;
    int n = 0;
    int n_waters = 0;
    spgnb_batch_options opt{};
    spgnb_nl* nl = nullptr;
    cudaStream_t stream = nullptr;
    // per atom
    float3* d_crd = nullptr;
    float3* d_vel = nullptr;
    float3* d_frc = nullptr;
    float3* d_crd_old = nullptr;
    float* d_charge = nullptr;
    float* d_inv_mass = nullptr;
    int* d_type = nullptr;
    int* d_atom_local = nullptr;
    int* d_ex_start = nullptr;
    int* d_ex_num = nullptr;
    int* d_ex_list = nullptr;
    int* d_waters = nullptr;  // oxygen of each rigid water
    // force field
    int T = 0;
    float2* d_table = nullptr;
    spgnb::ForceParams* d_fps = nullptr;
    std::vector<spgnb::ForceParams> h_fps;
    bool fit = true;
    long long* d_totals = nullptr;  // 8 per system
    int* d_atom_sys = nullptr;      // system of each atom (thermostat)
    double* d_kin = nullptr;        // per system: sum of m v^2
    int* d_step = nullptr;          // steps done, on the device (interval refresh)
    float* d_ndof = nullptr;        // per system: degrees of freedom
    float4* d_slot_pos = nullptr;
    int* d_slot_type = nullptr;
    // per system, host
    std::vector<int> atom_begin, atom_count;
    std::vector<double> lr_factor, volume;
    // stepping
    float ra = 0, rb = 0, rc = 0, mO = 0, mH = 0;
    cudaGraphExec_t g_plain = nullptr, g_energy = nullptr;
    long long kernels_plain = 0, kernels_energy = 0;  // kernel launches inside each graph
    long long steps_done = 0;
};

namespace spgnb
{
namespace
{

__global__ void k_leapfrog(int n, float3* __restrict__ crd, float3* __restrict__ vel, const float3* __restrict__ frc,
                           const float* __restrict__ inv_mass, float3* __restrict__ crd_old, float dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 x = crd[i];
    const float3 f = frc[i];
    const float im = inv_mass[i] * dt;
    float3 v = vel[i];
    v.x = fmaf(f.x, im, v.x);
    v.y = fmaf(f.y, im, v.y);
    v.z = fmaf(f.z, im, v.z);
    crd_old[i] = x;
    vel[i] = v;
    crd[i] = make_float3(fmaf(v.x, dt, x.x), fmaf(v.y, dt, x.y), fmaf(v.z, dt, x.z));
}

__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 unit3(float3 a) { return mul3(a, rsqrtf(dot3(a, a))); }

// SETTLE: moves the unconstrained new positions of one rigid water onto its
// geometry, keeping its centre of mass, from the old (constrained) ones.  The
// triangle in its own frame has O at (0, ra, 0) and the hydrogens at
// (-+rc, -rb, 0); the new plane orientation comes from rotations about the
// frame axes solved in closed form.  Velocities follow from the displacement.
__global__ void k_settle(int n_waters, const int* __restrict__ waters, float3* __restrict__ crd,
                         float3* __restrict__ vel, const float3* __restrict__ crd_old, float mO, float mH, float ra,
                         float rb, float rc, float inv_dt)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_waters) return;
    const int o = waters[w];
    const float3 origin = crd_old[o];
    // everything relative to the old oxygen, for precision
    const float3 b0 = sub3(crd_old[o + 1], origin), c0 = sub3(crd_old[o + 2], origin);
    const float3 a1 = sub3(crd[o], origin), b1 = sub3(crd[o + 1], origin), c1 = sub3(crd[o + 2], origin);
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
    crd[o] = add3(origin, a3);
    crd[o + 1] = add3(origin, b3);
    crd[o + 2] = add3(origin, c3);
    vel[o] = mul3(a3, inv_dt);  // a0 is the origin
    vel[o + 1] = mul3(sub3(b3, b0), inv_dt);
    vel[o + 2] = mul3(sub3(c3, c0), inv_dt);
}

// Berendsen weak coupling per system: twice the kinetic energy, then every
// velocity scaled by sqrt(1 + dt/tau (T0/T - 1)) (clamped to [0.8, 1.25]).
__global__ void k_kinetic(int n, const float3* __restrict__ vel, const float* __restrict__ inv_mass,
                          const int* __restrict__ atom_sys, double* __restrict__ kin)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || inv_mass[i] == 0.0f) return;
    const float3 v = vel[i];
    atomicAdd(&kin[atom_sys[i]], (double)((v.x * v.x + v.y * v.y + v.z * v.z) / inv_mass[i]));
}

__global__ void k_rescale(int n, float3* __restrict__ vel, const int* __restrict__ atom_sys,
                          const double* __restrict__ kin, const float* __restrict__ ndof, float kT0, float coupling)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = atom_sys[i];
    const double kT = kin[s] / fmax((double)ndof[s], 1.0);  // k_B T = 2 E_kin / dof
    const float lam2 = kT > 0.0 ? 1.0f + coupling * (float)(kT0 / kT - 1.0) : 1.0f;
    const float lam = sqrtf(fminf(fmaxf(lam2, 0.64f), 1.5625f));
    float3 v = vel[i];
    vel[i] = make_float3(v.x * lam, v.y * lam, v.z * lam);
}

int batch_force(spgnb_batch* b, int mode, cudaStream_t s)
{
    SPGNB_CUDA(cudaMemsetAsync(b->d_frc, 0, sizeof(float3) * b->n, s));
    if (mode) SPGNB_CUDA(cudaMemsetAsync(b->d_totals, 0, sizeof(long long) * 8 * b->S, s));
    ForceInputs in;
    in.nl = b->nl;
    in.crd = b->d_crd;
    in.charge = b->d_charge;
    in.atom_type = b->d_type;
    in.slot_pos = b->d_slot_pos;
    in.slot_type = b->d_slot_type;
    in.p0 = b->h_fps[0];
    in.d_fps = b->S > 1 ? b->d_fps : nullptr;
    in.fit = b->fit;
    in.table = b->d_table;
    in.table_size = b->T * b->T;
    in.frc = b->d_frc;
    in.totals = b->d_totals;
    in.mode = mode;
    in.om.solvent_start = b->n;
    return force_pipeline(in, s);
}

// One step: kick-drift, SETTLE, list update, forces.
int batch_step(spgnb_batch* b, bool energy, cudaStream_t s)
{
    const float dt = b->opt.dt * kTimeUnitsPerPs;
    k_leapfrog<<<(b->n + 255) / 256, 256, 0, s>>>(b->n, b->d_crd, b->d_vel, b->d_frc, b->d_inv_mass, b->d_crd_old,
                                                   dt);
    SPGNB_CHECK_LAUNCH("k_leapfrog");
    if (b->n_waters > 0)
    {
        k_settle<<<(b->n_waters + 127) / 128, 128, 0, s>>>(b->n_waters, b->d_waters, b->d_crd, b->d_vel,
                                                            b->d_crd_old, b->mO, b->mH, b->ra, b->rb, b->rc,
                                                            1.0f / dt);
        SPGNB_CHECK_LAUNCH("k_settle");
    }
    if (b->opt.thermostat_tau > 0.0f)
    {
        SPGNB_CUDA(cudaMemsetAsync(b->d_kin, 0, sizeof(double) * b->S, s));
        k_kinetic<<<(b->n + 255) / 256, 256, 0, s>>>(b->n, b->d_vel, b->d_inv_mass, b->d_atom_sys, b->d_kin);
        SPGNB_CHECK_LAUNCH("k_kinetic");
        const float kT0 = 0.00198716f * b->opt.temperature;  // kcal/mol
        k_rescale<<<(b->n + 255) / 256, 256, 0, s>>>(b->n, b->d_vel, b->d_atom_sys, b->d_kin, b->d_ndof, kT0,
                                                      b->opt.dt / b->opt.thermostat_tau);
        SPGNB_CHECK_LAUNCH("k_rescale");
    }
    int st = nl_queue_build(b->nl, b->n, b->d_crd, b->d_atom_local, b->d_ex_start, b->d_ex_list, b->d_ex_num,
                            b->opt.refresh_interval > 0 ? kBuildInterval : kBuildSkin, s, b->d_step,
                            b->opt.refresh_interval);
    if (st) return st;
    return batch_force(b, energy ? 1 : 0, s);
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
    SPGNB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int st = SPGNB_OK;
    const unsigned long long c0 = launches_so_far();
    for (int k = 0; k < b->opt.steps_per_graph && !st; k++)
        st = batch_step(b, energy_last && k == b->opt.steps_per_graph - 1, b->stream);
    // captured, not run: counted when the graph is launched
    *kernels = (long long)(launches_so_far() - c0);
    count_launches(-*kernels);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
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
    if (!b->opt.use_graphs || (b->g_plain && b->g_energy)) return SPGNB_OK;
    free_graphs(b);
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
    dfree(b->d_table);
    dfree(b->d_fps);
    dfree(b->d_totals);
    dfree(b->d_atom_sys);
    dfree(b->d_kin);
    dfree(b->d_ndof);
    dfree(b->d_step);
    dfree(b->d_slot_pos);
    dfree(b->d_slot_type);
    if (b->stream) cudaStreamDestroy(b->stream);
    b->stream = nullptr;
}

template <typename T>
int upload(T** d, const std::vector<T>& h)
{
    int st = dalloc(d, h.size());
    if (st) return st;
    if (!h.empty()) SPGNB_CUDA(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return SPGNB_OK;
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

int spgnb_batch_set_thermostat(spgnb_batch* b, float tau, float temperature)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_set_thermostat: NULL handle");
    if (!(tau >= 0.0f) || !(temperature >= 0.0f)) return fail(SPGNB_E_ARG, "spgnb_batch_set_thermostat: bad values");
    b->opt.thermostat_tau = tau;
    b->opt.temperature = temperature;
    free_graphs(b);
    return SPGNB_OK;
}

int spgnb_batch_create(int n_systems, const spgnb_batch_system* systems, int atom_type_numbers,
                       const float* h_pair_A, const float* h_pair_B, const spgnb_batch_options* opt,
                       spgnb_batch** out)
{
    if (!out) return fail(SPGNB_E_ARG, "spgnb_batch_create: out is NULL");
    *out = nullptr;
    if (n_systems <= 0 || !systems || atom_type_numbers <= 0 || !h_pair_A || !h_pair_B)
        return fail(SPGNB_E_ARG, "spgnb_batch_create: bad arguments");
    const int T = atom_type_numbers;
    if (T > kMaxTypes || T * T * (int)sizeof(float2) > 96 * 1024)
        return fail(SPGNB_E_UNSUPPORTED, "spgnb_batch_create: %d LJ types exceed the shared-memory pair table", T);
    spgnb_batch* b = new spgnb_batch();
    if (opt)
        b->opt = *opt;
    else
        spgnb_batch_default_options(&b->opt);
    if (b->opt.steps_per_graph <= 0) b->opt.steps_per_graph = 1;
    b->S = n_systems;
    b->T = T;
    // host staging
    long long ntot = 0;
    for (int s = 0; s < n_systems; s++)
    {
        const spgnb_batch_system& y = systems[s];
        if (y.atom_numbers <= 0 || !y.h_crd || !y.h_charge || !y.h_mass || !y.h_atom_type || !y.h_excluded_start ||
            !y.h_excluded_numbers || (y.excluded_total > 0 && !y.h_excluded_list) || y.water_begin < 0 ||
            y.water_numbers < 0 || y.water_begin + 3LL * y.water_numbers > y.atom_numbers)
        {
            delete b;
            return fail(SPGNB_E_ARG, "spgnb_batch_create: system %d is incomplete", s);
        }
        b->atom_begin.push_back((int)ntot);
        b->atom_count.push_back(y.atom_numbers);
        ntot += y.atom_numbers;
    }
    if (ntot > (1LL << 28))
    {
        delete b;
        return fail(SPGNB_E_UNSUPPORTED, "spgnb_batch_create: %lld atoms in total", ntot);
    }
    b->n = (int)ntot;
    std::vector<float3> crd(b->n), vel(b->n);
    std::vector<float> charge(b->n), inv_mass(b->n);
    std::vector<int> type(b->n), iota(b->n), ex_start(b->n), ex_num(b->n), ex_list, waters;
    std::vector<int> counts(n_systems), atom_sys(b->n);
    std::vector<float> ndof(n_systems);
    std::vector<spgnb_ltmatrix3> cells(n_systems), rcells(n_systems);
    std::vector<float> cutoffs(n_systems), skins(n_systems);
    b->h_fps.resize(n_systems);
    b->lr_factor.resize(n_systems);
    b->volume.resize(n_systems);
    for (int s = 0; s < n_systems; s++)
    {
        const spgnb_batch_system& y = systems[s];
        const int a0 = b->atom_begin[s];
        std::vector<double> hist(T, 0.0);
        for (int i = 0; i < y.atom_numbers; i++)
        {
            const int g = a0 + i;
            crd[g] = make_float3(y.h_crd[3 * i], y.h_crd[3 * i + 1], y.h_crd[3 * i + 2]);
            vel[g] = y.h_vel ? make_float3(y.h_vel[3 * i], y.h_vel[3 * i + 1], y.h_vel[3 * i + 2]) : make_float3(0, 0, 0);
            charge[g] = y.h_charge[i];
            inv_mass[g] = y.h_mass[i] > 0.0f ? 1.0f / y.h_mass[i] : 0.0f;
            const int t = y.h_atom_type[i];
            if (t < 0 || t >= T)
            {
                delete b;
                return fail(SPGNB_E_ARG, "spgnb_batch_create: system %d atom %d has type %d outside [0,%d)", s, i, t, T);
            }
            type[g] = t;
            hist[t] += 1.0;
            iota[g] = g;
            ex_num[g] = y.h_excluded_numbers[i];
            ex_start[g] = (int)ex_list.size();
            for (int k = 0; k < y.h_excluded_numbers[i]; k++)
                ex_list.push_back(a0 + y.h_excluded_list[y.h_excluded_start[i] + k]);
        }
        for (int w = 0; w < y.water_numbers; w++) waters.push_back(a0 + y.water_begin + 3 * w);
        for (int i = 0; i < y.atom_numbers; i++) atom_sys[a0 + i] = s;
        int moving = 0;
        for (int i = 0; i < y.atom_numbers; i++) moving += y.h_mass[i] > 0.0f;
        ndof[s] = (float)std::max(1, 3 * moving - 3 * y.water_numbers - 3);
        counts[s] = y.atom_numbers;
        cells[s] = y.cell;
        rcells[s] = y.rcell;
        cutoffs[s] = y.cutoff;
        skins[s] = y.skin;
        ForceParams& f = b->h_fps[s];
        f.rc2 = y.cutoff * y.cutoff;
        f.beta = y.pme_beta;
        f.beta3 = y.pme_beta * y.pme_beta * y.pme_beta;
        f.w_scale = y.pme_beta * y.pme_beta * SPGNB_EWALD_INV_W_MAX;
        const float z = y.pme_beta * y.cutoff;
        f.use_fit = (z * z <= SPGNB_EWALD_W_MAX * 0.999f) ? 1 : 0;
        f.n_types = T;
        f.table_begin = 0;
        f.pad = 0;
        if (!f.use_fit) b->fit = false;
        // Total_C6_Get and the factor of Lennard_Jones_force.cpp:263-268
        double c6 = 0.0;
        for (int p = 0; p < T; p++)
            for (int q = 0; q < T; q++)
            {
                const int hi = p > q ? p : q, lo = p > q ? q : p;
                c6 += hist[p] * hist[q] * (double)h_pair_B[hi * (hi + 1) / 2 + lo];
            }
        float fac = (float)c6;
        fac *= -2.0f / 3.0f * 3.1415926535897932f / y.cutoff / y.cutoff / y.cutoff / 6.0f;
        b->lr_factor[s] = fac;
        b->volume[s] = (double)y.cell.a11 * y.cell.a22 * y.cell.a33;
    }
    if (ex_list.empty()) ex_list.push_back(0);
    b->n_waters = (int)waters.size();
    std::vector<float2> table((size_t)T * T);
    for (int p = 0; p < T; p++)
        for (int q = 0; q < T; q++)
        {
            const int hi = p > q ? p : q, lo = p > q ? q : p;
            table[(size_t)p * T + q] = make_float2(h_pair_A[hi * (hi + 1) / 2 + lo], h_pair_B[hi * (hi + 1) / 2 + lo]);
        }
    // rigid water geometry (first water's masses)
    b->mO = 16.0f;
    b->mH = 1.008f;
    for (int s = 0; s < n_systems; s++)
        if (systems[s].water_numbers > 0)
        {
            b->mO = systems[s].h_mass[systems[s].water_begin];
            b->mH = systems[s].h_mass[systems[s].water_begin + 1];
            break;
        }
    b->rc = 0.5f * b->opt.water_dhh;
    const float h = sqrtf(b->opt.water_doh * b->opt.water_doh - b->rc * b->rc);
    b->ra = 2.0f * b->mH * h / (b->mO + 2.0f * b->mH);
    b->rb = h - b->ra;

    int st = SPGNB_OK;
    spgnb_nl_options nlo;
    spgnb_nl_default_options(&nlo);
    nlo.refresh_interval = 0;
    nlo.skin_permit = b->opt.skin_permit;
    nlo.export_atom_groups = 0;
    nlo.prune_buffer = b->opt.prune_buffer;
    if ((st = nl_create_multi(n_systems, counts.data(), cells.data(), rcells.data(), cutoffs.data(), skins.data(),
                              &nlo, &b->nl)) ||
        (st = upload(&b->d_crd, crd)) || (st = upload(&b->d_vel, vel)) || (st = dalloc(&b->d_frc, b->n)) ||
        (st = dalloc(&b->d_crd_old, b->n)) || (st = upload(&b->d_charge, charge)) ||
        (st = upload(&b->d_inv_mass, inv_mass)) || (st = upload(&b->d_type, type)) ||
        (st = upload(&b->d_atom_local, iota)) || (st = upload(&b->d_ex_start, ex_start)) ||
        (st = upload(&b->d_ex_num, ex_num)) || (st = upload(&b->d_ex_list, ex_list)) ||
        (st = upload(&b->d_waters, waters)) || (st = upload(&b->d_table, table)) ||
        (st = upload(&b->d_fps, b->h_fps)) || (st = dalloc(&b->d_totals, 8 * (size_t)n_systems)) ||
        (st = upload(&b->d_atom_sys, atom_sys)) || (st = upload(&b->d_ndof, ndof)) ||
        (st = dalloc(&b->d_kin, (size_t)n_systems)) || (st = dalloc(&b->d_step, 1)) ||
        (st = dalloc(&b->d_slot_pos, (size_t)b->nl->clusters_cap * kClusterSize + 1)) ||
        (st = dalloc(&b->d_slot_type, (size_t)b->nl->clusters_cap * kClusterSize + 1)))
    {
        free_batch(b);
        delete b;
        return st;
    }
    force_kernels_init(T * T);
    cudaMemset(b->d_step, 0, sizeof(int));
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess)
    {
        free_batch(b);
        delete b;
        return cuda_fail(e, "cudaStreamCreate");
    }
    // first lists and F(0) with energies
    if ((st = nl_queue_build(b->nl, b->n, b->d_crd, b->d_atom_local, b->d_ex_start, b->d_ex_list, b->d_ex_num, kBuildForced,
                             b->stream)) ||
        (st = batch_force(b, 1, b->stream)))
    {
        free_batch(b);
        delete b;
        return st;
    }
    e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess)
    {
        free_batch(b);
        delete b;
        return cuda_fail(e, "spgnb_batch_create");
    }
    *out = b;
    return SPGNB_OK;
}

int spgnb_batch_run(spgnb_batch* b, int steps, int energy_interval)
{
    if (!b) return fail(SPGNB_E_ARG, "spgnb_batch_run: NULL handle");
    if (steps <= 0) return SPGNB_OK;
    int st = ensure_graphs(b);
    if (st) return st;
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
    std::vector<long long> h(8 * (size_t)b->S);
    SPGNB_CUDA(cudaMemcpyAsync(h.data(), b->d_totals, sizeof(long long) * h.size(), cudaMemcpyDeviceToHost, b->stream));
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    for (int s = 0; s < b->S; s++)
    {
        const long long* t = &h[8 * (size_t)s];
        double* o = out + 9 * (size_t)s;
        o[0] = (double)t[0] / kEnergyScale;
        o[1] = b->lr_factor[s] / b->volume[s];
        o[2] = (double)t[1] / kEnergyScale;
        for (int q = 0; q < 6; q++) o[3 + q] = (double)t[2 + q] / kEnergyScale;
    }
    return SPGNB_OK;
}

int spgnb_batch_download(spgnb_batch* b, int sys, float* h_crd, float* h_vel, float* h_frc)
{
    if (!b || sys < 0 || sys >= b->S) return fail(SPGNB_E_ARG, "spgnb_batch_download: bad system");
    const size_t off = b->atom_begin[sys], cnt = b->atom_count[sys];
    if (h_crd)
        SPGNB_CUDA(cudaMemcpyAsync(h_crd, b->d_crd + off, sizeof(float3) * cnt, cudaMemcpyDeviceToHost, b->stream));
    if (h_vel)
        SPGNB_CUDA(cudaMemcpyAsync(h_vel, b->d_vel + off, sizeof(float3) * cnt, cudaMemcpyDeviceToHost, b->stream));
    if (h_frc)
        SPGNB_CUDA(cudaMemcpyAsync(h_frc, b->d_frc + off, sizeof(float3) * cnt, cudaMemcpyDeviceToHost, b->stream));
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
    // candidates up to the buffer the list was sized for
    const float maxb = b->opt.prune_buffer;
    const float cand[] = {0.4f, 0.6f, 0.8f, 1.0f, 1.3f, 1.6f};
    float best = maxb;
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    SPGNB_CUDA(cudaEventCreate(&e0));
    SPGNB_CUDA(cudaEventCreate(&e1));
    int st = SPGNB_OK;
    for (float c : cand)
    {
        if (c > maxb + 1e-6f) continue;
        b->nl->opt.prune_buffer = c;
        const std::vector<int> ones(b->S, 1);
        SPGNB_CUDA(cudaMemcpyAsync(b->nl->d_prune, ones.data(), sizeof(int) * b->S, cudaMemcpyHostToDevice, b->stream));
        const int one = 1;
        SPGNB_CUDA(cudaMemcpyAsync(b->nl->d_counters + kCntPrune, &one, sizeof(int), cudaMemcpyHostToDevice, b->stream));
        free_graphs(b);
        if ((st = spgnb_batch_run(b, b->opt.steps_per_graph, 0))) break;  // warm-up, includes the pruning
        SPGNB_CUDA(cudaEventRecord(e0, b->stream));
        if ((st = spgnb_batch_run(b, steps_per_candidate, 0))) break;
        SPGNB_CUDA(cudaEventRecord(e1, b->stream));
        SPGNB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        SPGNB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms)
        {
            best_ms = ms;
            best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    b->nl->opt.prune_buffer = best;
    b->opt.prune_buffer = best;
    free_graphs(b);
    const std::vector<int> ones(b->S, 1);
    SPGNB_CUDA(cudaMemcpyAsync(b->nl->d_prune, ones.data(), sizeof(int) * b->S, cudaMemcpyHostToDevice, b->stream));
    const int one = 1;
    SPGNB_CUDA(cudaMemcpyAsync(b->nl->d_counters + kCntPrune, &one, sizeof(int), cudaMemcpyHostToDevice, b->stream));
    SPGNB_CUDA(cudaStreamSynchronize(b->stream));
    if (chosen_buffer) *chosen_buffer = best;
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
    const int S = b->S;
    if (b->d_slot_pos) dfree(b->d_slot_pos);
    if (b->d_slot_type) dfree(b->d_slot_type);
    if ((st = dalloc(&b->d_slot_pos, (size_t)b->nl->clusters_cap * kClusterSize + 1)) ||
        (st = dalloc(&b->d_slot_type, (size_t)b->nl->clusters_cap * kClusterSize + 1)))
        return st;
    (void)S;
    if ((st = nl_queue_build(b->nl, b->n, b->d_crd, b->d_atom_local, b->d_ex_start, b->d_ex_list, b->d_ex_num, kBuildForced,
                             b->stream)) ||
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
