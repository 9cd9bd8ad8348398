// Diagnostics used by the benchmark: pair counts of a built list and an
// FP32 fused-multiply-add throughput probe (the denominator of the FP32
// roofline, measured on the device the benchmark runs on).
#include <algorithm>

#include "common.cuh"

namespace spgnb
{
namespace
{

// Counts listed pairs (each once) and those inside the cutoff at the given
// coordinates, from the neighbour tables (one- or two-sided).
__global__ void k_count_pairs(const int* __restrict__ counters, int clusters_cap, int table_cap,
                              const int* __restrict__ tcount, const float4* __restrict__ tab,
                              const uint2* __restrict__ tmask, const int* __restrict__ slot_atom,
                              const float4* __restrict__ x0, const float4* __restrict__ d0,
                              const float3* __restrict__ crd, Cell cell, Cell rcell, float rc2,
                              unsigned long long* out)
{
    const int lane = threadIdx.x & 31;
    const int nc = clusters_cap;
    (void)counters;
    const int warps = gridDim.x * (blockDim.x >> 5);
    unsigned long long listed = 0, inside = 0;
    auto pos = [&](int s) {
        const int a = slot_atom[s];
        const float4 d = d0[s];
        if (a < 0) return make_float3(d.x, d.y, d.z);
        const float3 c = crd[a];
        const float4 o = x0[s];
        float dx = c.x - o.x, dy = c.y - o.y, dz = c.z - o.z;
        const float sx = rintf(dx * rcell.a11 + dy * rcell.a21 + dz * rcell.a31);
        const float sy = rintf(dy * rcell.a22 + dz * rcell.a32);
        const float sz = rintf(dz * rcell.a33);
        dx -= sx * cell.a11 + sy * cell.a21 + sz * cell.a31;
        dy -= sy * cell.a22 + sz * cell.a32;
        dz -= sz * cell.a33;
        return make_float3(d.x + dx, d.y + dy, d.z + dz);
    };
    for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nc; c += warps)
    {
        const int T = tcount[c];
        for (int t = lane; t < T; t += 32)
        {
            const float4 e = tab[(size_t)c * table_cap + t];
            const uint2 mm = tmask[(size_t)c * table_cap + t];
            unsigned long long m = ((unsigned long long)mm.y << 32) | mm.x;
            const int base = __float_as_int(e.w) & 0x3fffffff;
            while (m)
            {
                const int k = __ffsll((long long)m) - 1;
                m &= m - 1;
                const int si = c * kClusterSize + (k >> 3), sj = base + (k & 7);
                // every pair once: from the lower cluster's table (a
                // two-sided table also holds the lower clusters), and
                // within a cluster from its lower-index atom
                const int J = sj >> 3;
                if (J < c || (J == c && !(__float_as_int(x0[si].w) < __float_as_int(x0[sj].w)))) continue;
                const float3 pi = pos(si), pj = pos(sj);
                float dx = e.x + pj.x - pi.x, dy = e.y + pj.y - pi.y, dz = e.z + pj.z - pi.z;
                const float sx = rintf(dx * rcell.a11 + dy * rcell.a21 + dz * rcell.a31);
                const float sy = rintf(dy * rcell.a22 + dz * rcell.a32);
                const float sz = rintf(dz * rcell.a33);
                dx -= sx * cell.a11 + sy * cell.a21 + sz * cell.a31;
                dy -= sy * cell.a22 + sz * cell.a32;
                dz -= sz * cell.a33;
                listed++;
                if (dx * dx + dy * dy + dz * dz < rc2) inside++;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1)
    {
        listed += __shfl_xor_sync(0xffffffffu, listed, o);
        inside += __shfl_xor_sync(0xffffffffu, inside, o);
    }
    if (lane == 0)
    {
        atomicAdd(&out[0], listed);
        atomicAdd(&out[1], inside);
    }
}

// Independent FMA chains, eight per thread, so the pipe never waits on a
// dependency; the result is stored to keep the work alive.
__global__ void k_fma_probe(int iters, float* out)
{
    float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
    float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; i++)
    {
#pragma unroll
        for (int k = 0; k < 16; k++)
        {
            a0 = __fmaf_rn(a0, m, c);
            a1 = __fmaf_rn(a1, m, c);
            a2 = __fmaf_rn(a2, m, c);
            a3 = __fmaf_rn(a3, m, c);
            a4 = __fmaf_rn(a4, m, c);
            a5 = __fmaf_rn(a5, m, c);
            a6 = __fmaf_rn(a6, m, c);
            a7 = __fmaf_rn(a7, m, c);
        }
    }
    float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.0f) out[blockIdx.x] = s;
}

}  // namespace
}  // namespace spgnb

using namespace spgnb;

extern "C" {

int spgnb_nl_count_pairs(spgnb_nl* nl, const spgnb_vector* d_crd, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                         float cutoff, long long* listed, long long* in_cutoff)
{
    if (!nl || !d_crd) return fail(SPGNB_E_ARG, "spgnb_nl_count_pairs: NULL argument");
    if (!nl->built) return fail(SPGNB_E_STATE, "spgnb_nl_count_pairs: list never built");
    unsigned long long* d = nullptr;
    int st = dalloc(&d, 2);
    if (st) return st;
    cudaStream_t s = stream();
    cudaMemsetAsync(d, 0, 16, s);
    k_count_pairs<<<num_sms() * 8, 128, 0, s>>>(nl->d_counters, nl->clusters_cap, nl->table_cap, nl->d_tcount,
                                                nl->d_tab, nl->d_tmask, nl->d_slot_atom, nl->d_slot_x0, nl->d_slot_d0,
                                                (const float3*)d_crd, make_cell(cell), make_cell(rcell),
                                                cutoff * cutoff, d);
    cudaError_t e = cudaGetLastError();
    unsigned long long h[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "spgnb_nl_count_pairs");
    if (listed) *listed = (long long)h[0];
    if (in_cutoff) *in_cutoff = (long long)h[1];
    return SPGNB_OK;
}

int spgnb_probe_fp32_fma_tflops(int repeats, double* tflops)
{
    if (!tflops) return fail(SPGNB_E_ARG, "spgnb_probe_fp32_fma_tflops: NULL output");
    const int blocks = num_sms() * 8, threads = 256, iters = 4096;
    float* out = nullptr;
    int st = dalloc(&out, blocks);
    if (st) return st;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaStream_t s = stream();
    k_fma_probe<<<blocks, threads, 0, s>>>(iters, out);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < std::max(1, repeats); r++)
    {
        cudaEventRecord(a, s);
        k_fma_probe<<<blocks, threads, 0, s>>>(iters, out);
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        best = std::min(best, ms);
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (e != cudaSuccess) return cuda_fail(e, "spgnb_probe_fp32_fma_tflops");
    double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return SPGNB_OK;
}

}  // extern "C"
