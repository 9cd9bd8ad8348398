// LJ + PME direct-space force over a reference-layout neighbour list that
// allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc at the point where the
// force is needed -- a SPONGE plugin's Calculate_Force hook, which runs
// inside the MD step after other modules have queued work (cudaMalloc
// synchronises the whole device and stalls that queue), or a serving process
// whose device memory is carved up in advance by an admission budget and
// must not grow.  The regular entry points allocate their scratch in
// spgnb_lj_create / on first use; this one keeps its scratch in a file-scope
// device array instead, so it has neither a create call nor an allocation.
//
// Limits and behaviour:
//   * at most kNoAllocMaxAtoms atoms and kNoAllocMaxTypes LJ types; larger
//     inputs are rejected with SPGNB_E_ARG before any work is queued;
//   * the scratch array (~2.6 MB) is part of the library image: every GPU
//     that loads libspgnb.so holds it until the process exits;
//   * every call shares that one array and leaves its contents behind; each
//     call clears what must start at zero, but two calls whose kernels
//     overlap on the GPU (different streams, or different host threads on
//     one device) race on it -- serialise them;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before capturing any stream on that device.
#include <math.h>

#include "common.cuh"

namespace spgnb
{
namespace
{

constexpr int kNoAllocMaxAtoms = 65536;
constexpr int kNoAllocMaxTypes = 64;
constexpr int kMaxDevices = 64;

// Scratch layout: int64 force accumulators x, y, z (3 * max atoms), the
// packed {x, y, z, q} records, the square {A, B} pair table.
constexpr size_t kAccBytes = sizeof(long long) * 3 * kNoAllocMaxAtoms;
constexpr size_t kPosBytes = sizeof(float4) * kNoAllocMaxAtoms;
constexpr size_t kTableBytes = sizeof(float2) * kNoAllocMaxTypes * kNoAllocMaxTypes;
constexpr size_t kScratchBytes = kAccBytes + kPosBytes + kTableBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of the scratch array per device, looked up on a device's
// first call.  Written without a lock: every writer for a device stores the
// same address, so a racing second lookup only repeats the first.
void* g_scratch_addr[kMaxDevices] = {nullptr};

struct Params
{
    float rc2, beta, beta3, w_scale;
    int n_types, use_fit;
};

__device__ __forceinline__ float poly5(float x, const float* c)
{
    float p = c[5];
    p = __fmaf_rn(p, x, c[4]);
    p = __fmaf_rn(p, x, c[3]);
    p = __fmaf_rn(p, x, c[2]);
    p = __fmaf_rn(p, x, c[1]);
    return __fmaf_rn(p, x, c[0]);
}

// F/r of the pair (Lennard_Jones_force.h:50-73 forms), FP32.
__device__ __forceinline__ float force_over_r(float r2, float qq, float A, float B, const Params& p)
{
    float rinv = rsqrtf(r2);
    rinv = rinv * __fmaf_rn(-0.5f * r2 * rinv, rinv, 1.5f);
    const float r2inv = rinv * rinv;
    const float r6inv = r2inv * r2inv * r2inv;
    const float flj = __fmaf_rn(-A, r6inv, B) * r6inv * r2inv;
    float fc;
    if (p.use_fit)
    {
        const float x = r2 * p.w_scale;
        fc = qq * __fmaf_rn(-p.beta3, __fdividef(poly5(x, kEwaldKP), poly5(x, kEwaldKQ)), rinv * r2inv);
    }
    else
    {
        const float br = p.beta * r2 * rinv;
        fc = qq * rinv * r2inv * __fmaf_rn(br * 1.1283791670955126f, __expf(-br * br), erfcf(br));
    }
    return flj - fc;
}

__device__ __forceinline__ void add_fixed(long long* a, float v)
{
    const long long q = __float2ll_rn(v * 4294967296.0f);
    if (q != 0) atomicAdd((unsigned long long*)a, (unsigned long long)q);
}

// Clears the accumulators, packs positions/charges and the type table.
__global__ void k_noalloc_prepare(unsigned char* scratch, int n, const float3* __restrict__ crd,
                                  const float* __restrict__ charge, int n_types, const float* __restrict__ pair_A,
                                  const float* __restrict__ pair_B)
{
    long long* acc = (long long*)scratch;
    float4* pos = (float4*)(scratch + kAccBytes);
    float2* table = (float2*)(scratch + kAccBytes + kPosBytes);
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        acc[i] = 0;
        acc[kNoAllocMaxAtoms + i] = 0;
        acc[2 * kNoAllocMaxAtoms + i] = 0;
        const float3 c = crd[i];
        pos[i] = make_float4(c.x, c.y, c.z, charge[i]);
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_types * n_types; k += stride)
    {
        const int a = k / n_types, b = k % n_types;
        const int hi = a > b ? a : b, lo = a > b ? b : a;
        const int t = hi * (hi + 1) / 2 + lo;
        table[k] = make_float2(pair_A[t], pair_B[t]);
    }
}

// Warp per owner atom over its half list; the reference's minimum image and
// cutoff test (Lennard_Jones_force.cpp:74-98); forces into the scratch
// accumulators in int64 fixed point.
__global__ void k_noalloc_pairs(unsigned char* scratch, Params p, Cell c, Cell r, int n_owner, int n,
                                const spgnb_atom_group* __restrict__ nl, const int* __restrict__ atom_type)
{
    long long* acc = (long long*)scratch;
    const float4* pos = (const float4*)(scratch + kAccBytes);
    const float2* table = (const float2*)(scratch + kAccBytes + kPosBytes);
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n_owner; i += warps)
    {
        const spgnb_atom_group g = nl[i];
        const float4 pi = pos[i];
        // types outside [0, n_types) and partners outside [0, n) are caller
        // errors: types are clamped and such partners skipped, so every read
        // stays inside the scratch array and the caller's arrays
        const int ti = min(max(atom_type[i], 0), p.n_types - 1) * p.n_types;
        float fx = 0, fy = 0, fz = 0;
        for (int k = lane; k < g.atom_numbers; k += 32)
        {
            const int j = g.atom_serial[k];
            if (j < 0 || j >= n) continue;
            const float4 pj = pos[j];
            float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            const float sx = floorf(dx * r.a11 + dy * r.a21 + dz * r.a31 + 0.5f);
            const float sy = floorf(dy * r.a22 + dz * r.a32 + 0.5f);
            const float sz = floorf(dz * r.a33 + 0.5f);
            dx -= sx * c.a11 + sy * c.a21 + sz * c.a31;
            dy -= sy * c.a22 + sz * c.a32;
            dz -= sz * c.a33;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (!(r2 < p.rc2)) continue;
            const float2 AB = table[ti + min(max(atom_type[j], 0), p.n_types - 1)];
            const float f = force_over_r(r2, pi.w * pj.w, AB.x, AB.y, p);
            fx += f * dx;
            fy += f * dy;
            fz += f * dz;
            add_fixed(acc + j, -f * dx);
            add_fixed(acc + kNoAllocMaxAtoms + j, -f * dy);
            add_fixed(acc + 2 * kNoAllocMaxAtoms + j, -f * dz);
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
        }
        if (lane == 0)
        {
            add_fixed(acc + i, fx);
            add_fixed(acc + kNoAllocMaxAtoms + i, fy);
            add_fixed(acc + 2 * kNoAllocMaxAtoms + i, fz);
        }
    }
}

__global__ void k_noalloc_finish(const unsigned char* scratch, int n, float3* __restrict__ frc)
{
    const long long* acc = (const long long*)scratch;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 f = frc[i];
    f.x += (float)((double)acc[i] * (1.0 / 4294967296.0));
    f.y += (float)((double)acc[kNoAllocMaxAtoms + i] * (1.0 / 4294967296.0));
    f.z += (float)((double)acc[2 * kNoAllocMaxAtoms + i] * (1.0 / 4294967296.0));
    frc[i] = f;
}

int scratch_address(void** out)
{
    int dev = 0;
    SPGNB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(SPGNB_E_UNSUPPORTED, "device index %d out of range", dev);
    if (!g_scratch_addr[dev])
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return SPGNB_OK;
}

}  // namespace
}  // namespace spgnb

using namespace spgnb;

extern "C" {

int spgnb_lj_pme_direct_force_noalloc(int local_atom_numbers, int solvent_numbers, int ghost_numbers,
                                      int atom_type_numbers,
                                      const int* d_atom_type, const float* d_pair_A, const float* d_pair_B,
                                      const spgnb_vector* d_crd, const float* d_charge, spgnb_vector* d_frc,
                                      spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, const spgnb_atom_group* d_nl,
                                      float cutoff, float pme_beta)
{
    if (local_atom_numbers < 0 || local_atom_numbers > kNoAllocMaxAtoms)
        return fail(SPGNB_E_ARG,
                    "spgnb_lj_pme_direct_force_noalloc: %d atoms; this entry point handles at most %d "
                    "(its scratch is a fixed device array)",
                    local_atom_numbers, kNoAllocMaxAtoms);
    if (atom_type_numbers <= 0 || atom_type_numbers > kNoAllocMaxTypes)
        return fail(SPGNB_E_ARG, "spgnb_lj_pme_direct_force_noalloc: %d LJ types; at most %d", atom_type_numbers,
                    kNoAllocMaxTypes);
    if (solvent_numbers < 0 || solvent_numbers > local_atom_numbers)
        return fail(SPGNB_E_ARG, "spgnb_lj_pme_direct_force_noalloc: bad solvent_numbers");
    if (ghost_numbers != 0)
        return fail(SPGNB_E_UNSUPPORTED,
                    "spgnb_lj_pme_direct_force_noalloc: ghost atoms (multi-rank domain decomposition) are not "
                    "supported");
    if (!d_atom_type || !d_pair_A || !d_pair_B || !d_crd || !d_charge || !d_frc || !d_nl)
        return fail(SPGNB_E_ARG, "spgnb_lj_pme_direct_force_noalloc: NULL device pointer");
    if (!(cutoff > 0.0f)) return fail(SPGNB_E_ARG, "spgnb_lj_pme_direct_force_noalloc: cutoff must be positive");
    if (local_atom_numbers == 0) return SPGNB_OK;
    void* scratch = nullptr;
    int st = scratch_address(&scratch);
    if (st) return st;
    Params p;
    p.rc2 = cutoff * cutoff;
    p.beta = pme_beta;
    p.beta3 = pme_beta * pme_beta * pme_beta;
    p.w_scale = pme_beta * pme_beta * SPGNB_EWALD_INV_W_MAX;
    p.n_types = atom_type_numbers;
    const float z = pme_beta * cutoff;
    p.use_fit = (z * z <= SPGNB_EWALD_W_MAX * 0.999f) ? 1 : 0;
    cudaStream_t s = stream();
    const int n = local_atom_numbers;
    k_noalloc_prepare<<<std::max(1, std::min((n + 255) / 256, num_sms() * 4)), 256, 0, s>>>(
        (unsigned char*)scratch, n, (const float3*)d_crd, d_charge, atom_type_numbers, d_pair_A, d_pair_B);
    SPGNB_CHECK_LAUNCH("k_noalloc_prepare");
    const int owners = n - solvent_numbers;
    if (owners > 0)
    {
        k_noalloc_pairs<<<std::max(1, std::min((owners + 3) / 4, num_sms() * 8)), 128, 0, s>>>(
            (unsigned char*)scratch, p, make_cell(cell), make_cell(rcell), owners, n, d_nl, d_atom_type);
        SPGNB_CHECK_LAUNCH("k_noalloc_pairs");
    }
    k_noalloc_finish<<<(n + 255) / 256, 256, 0, s>>>((const unsigned char*)scratch, n, (float3*)d_frc);
    SPGNB_CHECK_LAUNCH("k_noalloc_finish");
    return SPGNB_OK;
}

}  // extern "C"
