// Neighbour-list rebuild: NEIGHBOR_LIST::Initial / Update / Check_Overflow /
// Clear of SPONGE/neighbor_list/neighbor_list.cpp, over one or many
// independent periodic systems, built around 8-atom clusters.
//
// The listed set is the reference's, pair for pair: atoms are binned into the
// reference grid (cells of (rc+skin)/2, same wrap and clamp, :206-275), pairs
// are considered between a cell and its stencil (:5-49), and a pair (i, j)
// with atom_local[i] < atom_local[j] is listed when the FP32 expression
// Get_Periodic_Displacement(crd_i, crd_j)^2 (vector.hpp:322-327) is below
// 4*grid_length^2 (:367-372, :705) and j is not in i's exclusion list
// (:594-665).
//
// Stages of one rebuild (every kernel returns at once when no rebuild is due,
// so a step never synchronises with the host):
//   bin -> scan -> scatter -> in-cell sort -> cluster centres   (clusters)
//   search  -> per cluster, its neighbour clusters with exact 64-bit masks
// The force call prunes the tables into per-atom lists (pair.cu); the
// reference-layout export reads the tables.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace spgnb
{
namespace
{

__device__ __forceinline__ int pack_shift(int k1, int k2, int k3)
{
    k1 = max(-511, min(511, k1));
    k2 = max(-511, min(511, k2));
    k3 = max(-511, min(511, k3));
    return ((k1 + 512) << 20) | ((k2 + 512) << 10) | (k3 + 512);
}

__device__ __forceinline__ void unpack_shift(int p, int& k1, int& k2, int& k3)
{
    k1 = ((p >> 20) & 1023) - 512;
    k2 = ((p >> 10) & 1023) - 512;
    k3 = (p & 1023) - 512;
}

// FP32 squared distance of the reference's candidate test, crd_a - crd_b,
// with the rounding sequence a CUDA build of vector.hpp:322-327 followed by
// the dot product produces (orc_pair_dr2, mode 1, in the oracle).
__device__ __forceinline__ float ref_pair_dr2(float3 a, float3 b, const Cell& c, const Cell& r)
{
    float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
    float sx = __fmaf_rn(dz, r.a31, __fmaf_rn(dx, r.a11, __fmul_rn(dy, r.a21)));
    float sy = __fmaf_rn(dy, r.a22, __fmul_rn(dz, r.a32));
    sx = floorf(__fadd_rn(sx, 0.5f));
    sy = floorf(__fadd_rn(sy, 0.5f));
    float sz = floorf(__fmaf_rn(dz, r.a33, 0.5f));
    float tx = __fmaf_rn(sz, c.a31, __fmaf_rn(sx, c.a11, __fmul_rn(sy, c.a21)));
    float ty = __fmaf_rn(sy, c.a22, __fmul_rn(sz, c.a32));
    dx = __fsub_rn(dx, tx);
    dy = __fsub_rn(dy, ty);
    dz = __fmaf_rn(-sz, c.a33, dz);
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// ---------------------------------------------------------------- kernels

// Check_Refresh (neighbor_list.cpp:166-180), per system: a system rebuilds
// when one of its atoms moved more than skin*skin_permit since its last build.
__global__ void k_check_refresh(int n_slots, const int* __restrict__ slot_atom, const int* __restrict__ cl_sys,
                                const SysDesc* __restrict__ sys, const float3* __restrict__ crd,
                                const float4* __restrict__ x0, int* __restrict__ need, int* counters)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    bool move = false;
    if (s < n_slots)
    {
        const int a = slot_atom[s];
        if (a >= 0)
        {
            const int sy = cl_sys[s >> 3];
            const SysDesc& D = sys[sy];
            const float3 c = crd[a];
            const float4 o = x0[s];
            float dx = c.x - o.x, dy = c.y - o.y, dz = c.z - o.z;
            const float sx = floorf(dx * D.rcell.a11 + dy * D.rcell.a21 + dz * D.rcell.a31 + 0.5f);
            const float sy2 = floorf(dy * D.rcell.a22 + dz * D.rcell.a32 + 0.5f);
            const float sz = floorf(dz * D.rcell.a33 + 0.5f);
            dx -= sx * D.cell.a11 + sy2 * D.cell.a21 + sz * D.cell.a31;
            dy -= sy2 * D.cell.a22 + sz * D.cell.a32;
            dz -= sz * D.cell.a33;
            move = dx * dx + dy * dy + dz * dz > D.permit2;
            if (move) need[sy] = 1;
        }
    }
    if (__any_sync(0xffffffffu, move) && (threadIdx.x & 31) == 0) counters[kCntNeed] = 1;
}

// Put_Atom_In_Grids (neighbor_list.cpp:206-275): brick wrap, cell index
// nx*Ny*Nz + ny*Nz + nz with clamping, per-cell count.
__global__ void k_bin(int n, const float3* __restrict__ crd, const int* __restrict__ atom_sys,
                      const SysDesc* __restrict__ sys, int* __restrict__ atom_cell, int* __restrict__ atom_shift,
                      float4* __restrict__ wrapped, int* __restrict__ cell_count, const int* __restrict__ need,
                      const int* __restrict__ counters)
{
    if (counters[kCntNeed] == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !need[atom_sys[i]]) return;
    const SysDesc& g = sys[atom_sys[i]];
    const float3 c = crd[i];
    float x = c.x, y = c.y, z = c.z;
    const float k3 = floorf(__fdiv_rn(z, g.cell.a33));
    z = __fsub_rn(z, __fmul_rn(k3, g.cell.a33));
    y = __fsub_rn(y, __fmul_rn(k3, g.cell.a32));
    const float k2 = floorf(__fdiv_rn(y, g.cell.a22));
    y = __fsub_rn(y, __fmul_rn(k2, g.cell.a22));
    x = __fsub_rn(x, __fadd_rn(__fmul_rn(k3, g.cell.a31), __fmul_rn(k2, g.cell.a21)));
    const float k1 = floorf(__fdiv_rn(x, g.cell.a11));
    x = __fsub_rn(x, __fmul_rn(k1, g.cell.a11));
    int nx = (int)__fdiv_rn(x, g.gl);
    int ny = (int)__fdiv_rn(y, g.gl);
    int nz = (int)__fdiv_rn(z, g.gl);
    nx = nx < 0 ? 0 : (nx < g.Nx ? nx : g.Nx - 1);
    ny = ny < 0 ? 0 : (ny < g.Ny ? ny : g.Ny - 1);
    nz = nz < 0 ? 0 : (nz < g.Nz ? nz : g.Nz - 1);
    const int cid = g.cell_begin + nx * g.Ny * g.Nz + ny * g.Nz + nz;
    atom_cell[i] = cid;
    atom_shift[i] = pack_shift((int)k1, (int)k2, (int)k3);
    wrapped[i] = make_float4(x, y, z, 0.0f);
    atomicAdd(&cell_count[cid], 1);
}

// Cluster counts per cell (ceil(count/8)), their exclusive scan from the
// system's first cluster, overflow checks of the cells; one block per system.
__global__ void k_scan_cells(const SysDesc* __restrict__ sys, const int* __restrict__ cell_count,
                             int2* __restrict__ cell_cl, int max_atom_in_grid, const int* __restrict__ need,
                             int* __restrict__ ncl, int* counters)
{
    const int sy = blockIdx.x;
    if (counters[kCntNeed] == 0 || !need[sy]) return;
    const SysDesc& g = sys[sy];
    const int G = g.Nx * g.Ny * g.Nz;
    const int* cc = cell_count + g.cell_begin;
    __shared__ int max_cell;
    if (threadIdx.x == 0) max_cell = 0;
    __syncthreads();
    int local_max = 0;
    for (int c = threadIdx.x; c < G; c += blockDim.x) local_max = max(local_max, cc[c]);
    atomicMax(&max_cell, local_max);
    int2* out = cell_cl + g.cell_begin;
    const int base = g.cl_begin;
    auto clusters = [&](int c) { return (min(cc[c], kMaxCellAtoms) + kClusterSize - 1) / kClusterSize; };
    const int total = block_scan_to<int>(G, clusters, [&](int c, int excl) {
        out[c] = make_int2(base + excl, base + excl + clusters(c));
    });
    if (threadIdx.x == 0)
    {
        // (cannot exceed the system's capacity atoms/8 + cells; if it did, build nothing)
        ncl[sy] = total <= g.cl_cap ? total : 0;
        atomicMax(&counters[kCntMaxCell], max_cell);
        int flags = 0;
        if (max_cell > max_atom_in_grid) flags |= kOvfGrid;
        if (total > g.cl_cap) flags |= kOvfPairs;
        if (max_cell > kMaxCellAtoms) flags |= kOvfCellHard;
        if (flags) atomicOr(&counters[kCntOverflow], flags);
    }
}

__global__ void k_scatter(int n, const int* __restrict__ atom_sys, const int* __restrict__ atom_cell,
                          const int2* __restrict__ cell_cl, const int* __restrict__ ncl,
                          const SysDesc* __restrict__ sys, int* __restrict__ cell_cursor, int* __restrict__ tmp_atoms,
                          const int* __restrict__ need, const int* __restrict__ counters)
{
    if (counters[kCntNeed] == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int sy = atom_sys[i];
    if (!need[sy] || ncl[sy] == 0) return;
    const int c = atom_cell[i];
    const int pos = atomicAdd(&cell_cursor[c], 1);
    const int2 r = cell_cl[c];
    if (pos < kMaxCellAtoms && r.y <= sys[sy].cl_begin + ncl[sy]) tmp_atoms[r.x * kClusterSize + pos] = i;
}

__device__ __forceinline__ unsigned spread3(unsigned v)
{
    // 2-bit value -> bits 0 and 3
    return (v & 1u) | ((v & 2u) << 2);
}

// Deterministic in-cell order: by a 4x4x4 Morton sub-cell key, then by atom
// index, so clusters are spatially compact and the build reproducible.
__global__ void k_sort_cells(int G, const int* __restrict__ cell_sys, const SysDesc* __restrict__ sys,
                             const int* __restrict__ cell_count, const int2* __restrict__ cell_cl,
                             const int* __restrict__ ncl, const int* __restrict__ tmp_atoms,
                             const float4* __restrict__ wrapped, int* __restrict__ slot_atom, int* __restrict__ cl_cell,
                             int* __restrict__ atom_slot, const int* __restrict__ need, const int* __restrict__ counters)
{
    if (counters[kCntNeed] == 0) return;
    extern __shared__ unsigned long long keys[];
    for (int c = blockIdx.x; c < G; c += gridDim.x)
    {
        const int sy = cell_sys[c];
        if (!need[sy]) continue;
        const SysDesc& g = sys[sy];
        const int n = min(cell_count[c], kMaxCellAtoms);
        const int2 r = cell_cl[c];
        if (ncl[sy] == 0 || r.y > g.cl_begin + ncl[sy]) continue;
        const int base = r.x * kClusterSize;
        const int nslots = (r.y - r.x) * kClusterSize;
        const int local = c - g.cell_begin;
        const int nz = local % g.Nz, ny = (local / g.Nz) % g.Ny, nx = local / (g.Ny * g.Nz);
        const float inv = 4.0f / g.gl;
        for (int e = threadIdx.x; e < n; e += blockDim.x)
        {
            const int a = tmp_atoms[base + e];
            const float4 w = wrapped[a];
            const int sx = min(3, max(0, (int)((w.x - nx * g.gl) * inv)));
            const int syy = min(3, max(0, (int)((w.y - ny * g.gl) * inv)));
            const int sz = min(3, max(0, (int)((w.z - nz * g.gl) * inv)));
            const unsigned key = (spread3(sx) << 2) | (spread3(syy) << 1) | spread3(sz);
            keys[e] = ((unsigned long long)key << 32) | (unsigned)a;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nslots; e += blockDim.x)
        {
            if (e < n)
            {
                const unsigned long long k = keys[e];
                int rank = 0;
                for (int f = 0; f < n; f++) rank += keys[f] < k;
                const int a = (int)(k & 0xffffffffu);
                slot_atom[base + rank] = a;
                atom_slot[a] = base + rank;
            }
            else
            {
                slot_atom[base + e] = -1;
            }
        }
        for (int k = r.x + threadIdx.x; k < r.y; k += blockDim.x) cl_cell[k] = c;
        __syncthreads();
    }
}

// Per cluster: centre (double, bounding-box middle of the wrapped positions),
// radius, fractional fixed-point centre, per-slot offsets and build
// coordinates (w = the atom's global index, -1 for padding).  Eight lanes per
// cluster.
__global__ void k_cluster_props(const float3* __restrict__ crd, int* __restrict__ slot_atom,
                                const int* __restrict__ atom_shift, const int* __restrict__ atom_local,
                                const int* __restrict__ cl_sys, const SysDesc* __restrict__ sys, int* counters,
                                uint4* __restrict__ cl_u, int4* __restrict__ cl_q, float4* __restrict__ cl_c,
                                float4* __restrict__ slot_x0, int* __restrict__ slot_gid, float4* __restrict__ slot_d0,
                                int2* __restrict__ slot_ex, const int* __restrict__ ex_start,
                                const int* __restrict__ ex_list, const int* __restrict__ ex_num, int clusters_cap,
                                const int* __restrict__ need, const int* __restrict__ ncl, int* __restrict__ tcount,
                                int* __restrict__ slot_count, int* __restrict__ pcount)
{
    if (counters[kCntNeed] == 0) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t >> 3;
    const int l8 = t & 7;
    const int sy = k < clusters_cap ? cl_sys[k] : 0;
    // every lane takes part in the shuffles below; only clusters of systems
    // being rebuilt write anything
    const bool active = k < clusters_cap && need[sy];
    const bool live = active && k - sys[sy].cl_begin < ncl[sy];
    const int s = k * kClusterSize + l8;
    if (active && !live)
    {
        // a cluster of the system's range that this build does not use
        slot_atom[s] = -1;
        slot_count[s] = 0;
        pcount[s] = 0;
        if (l8 == 0) tcount[k] = 0;
    }
    const int a = live ? slot_atom[s] : -1;
    Cell cell{1, 0, 1, 0, 0, 1};
    if (live) cell = sys[sy].cell;
    double w[3] = {0, 0, 0};
    float3 x = make_float3(0, 0, 0);
    if (a >= 0)
    {
        x = crd[a];
        int k1, k2, k3;
        unpack_shift(atom_shift[a], k1, k2, k3);
        w[0] = (double)x.x - (double)k3 * cell.a31 - (double)k2 * cell.a21 - (double)k1 * cell.a11;
        w[1] = (double)x.y - (double)k3 * cell.a32 - (double)k2 * cell.a22;
        w[2] = (double)x.z - (double)k3 * cell.a33;
    }
    double lo[3], hi[3];
    for (int d = 0; d < 3; d++)
    {
        lo[d] = a >= 0 ? w[d] : 1e300;
        hi[d] = a >= 0 ? w[d] : -1e300;
        for (int o = 1; o < 8; o <<= 1)
        {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
    }
    double cen[3];
    for (int d = 0; d < 3; d++) cen[d] = (lo[d] <= hi[d]) ? 0.5 * (lo[d] + hi[d]) : 0.0;
    // fractional centre on the double inverse of the float cell
    const double c11 = cell.a11, c21 = cell.a21, c22 = cell.a22, c31 = cell.a31, c32 = cell.a32, c33 = cell.a33;
    const double r33 = 1.0 / c33, r22 = 1.0 / c22, r11 = 1.0 / c11;
    const double r32 = -c32 * r33 / c22;
    const double r31 = (c32 * c21 * r33 - c31 * c22) / (c11 * c22 * c33);
    const double r21 = -c21 * r22 / c11;
    const double sfr[3] = {cen[0] * r11 + cen[1] * r21 + cen[2] * r31, cen[1] * r22 + cen[2] * r32, cen[2] * r33};
    // the centre is rounded to 2^-22 of each box vector, so centre
    // differences are exact 22-bit integers (the force kernel converts them
    // without a table); the 32-bit form is the same value shifted by 10
    unsigned u[3], u22[3];
    double q[3];
    for (int d = 0; d < 3; d++)
    {
        const double f = floor(sfr[d]);
        const double frac = sfr[d] - f;
        double scaled = floor(frac * 4194304.0);
        if (scaled >= 4194304.0) scaled = 4194303.0;
        if (!(scaled >= 0.0)) scaled = 0.0;
        u22[d] = (unsigned)scaled;
        u[d] = u22[d] << 10;
        q[d] = scaled / 4194304.0 + f;  // the quantised centre, unwrapped
    }
    const double cq[3] = {q[0] * c11 + q[1] * c21 + q[2] * c31, q[1] * c22 + q[2] * c32, q[2] * c33};
    double r2 = 0;
    if (a >= 0)
    {
        const double d0 = w[0] - cq[0], d1 = w[1] - cq[1], d2 = w[2] - cq[2];
        r2 = d0 * d0 + d1 * d1 + d2 * d2;
        slot_d0[s] = make_float4((float)d0, (float)d1, (float)d2, 0.0f);
        const int g = atom_local[a];
        slot_x0[s] = make_float4(x.x, x.y, x.z, __int_as_float(g));
        slot_gid[s] = g;
        // [first, last] of the atom's (sorted) exclusion list, empty when none
        const int k = ex_num[g];
        slot_ex[s] = k > 0 ? make_int2(ex_list[ex_start[g]], ex_list[ex_start[g] + k - 1]) : make_int2(0x7fffffff, -1);
    }
    else if (active)
    {
        const float p = kPadCoordinate + (float)s;
        slot_d0[s] = make_float4(p, p, p, 0.0f);
        slot_x0[s] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
        slot_gid[s] = -1;
        slot_ex[s] = make_int2(0x7fffffff, -1);
    }
    for (int o = 1; o < 8; o <<= 1) r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, o));
    if (live && l8 == 0)
    {
        const float rad = (float)(sqrt(r2) * (1.0 + 1e-6) + 1e-5);
        cl_u[k] = make_uint4(u[0], u[1], u[2], __float_as_uint(rad));
        cl_q[k] = make_int4((int)u22[0], (int)u22[1], (int)u22[2], 0);
        // bounding box about the quantised centre (its offset from the box
        // middle included), with a little slack
        float h[3];
        for (int d = 0; d < 3; d++)
            h[d] = lo[d] <= hi[d] ? (float)(0.5 * (hi[d] - lo[d]) + fabs(cq[d] - cen[d]) + 1e-4) : 0.0f;
        cl_c[k] = make_float4(h[0], h[1], h[2], rad);
    }
}

__device__ __forceinline__ float3 frac_delta(uint4 ui, uint4 uj)
{
    const float s = 2.3283064365386963e-10f;  // 2^-32
    return make_float3((float)(int)(uj.x - ui.x) * s, (float)(int)(uj.y - ui.y) * s, (float)(int)(uj.z - ui.z) * s);
}

__device__ __forceinline__ float3 frac_to_cart(float3 f, const Cell& c)
{
    return make_float3(f.x * c.a11 + f.y * c.a21 + f.z * c.a31, f.y * c.a22 + f.z * c.a32, f.z * c.a33);
}

// Neighbour search, one warp per cluster, its table in a deterministic order
// (candidate runs, then cluster index) with no sorting or atomics.
// One-sided tables (half set): a cluster keeps only neighbour clusters
// J >= I, so each cluster pair is searched once; the pruned half list needs
// no more, and the exports reach the lower side through the reverse index.
// Symmetric (two-sided) tables, every neighbour cluster lower and higher:
// for the clusters holding a flagged atom (the soft-core kernel's perturbed
// atoms), or all clusters (dH/dlambda).  For each candidate cluster that passes a
// conservative sphere test, the 64 atom pairs are decided as the reference
// decides them: a pair needs the higher-index atom's cell in the stencil of
// the lower-index atom's cell, squared distance below 4*grid_length^2 in the
// reference's FP32 expression, and no exclusion.  The distance is first
// evaluated from the cluster-relative offsets; only pairs within 1e-4*cs2 of
// the threshold (or of clusters whose spheres reach half a box) are
// re-evaluated with the reference's exact expression, so every decision is the
// reference's.  Exclusion lists are scanned only when the partner lies within
// the list's [first, last] range (the reference's pre-check).  A cluster pair
// with any listed pair becomes a table element {centre difference, neighbour
// slot base | image flag} plus its 64-bit mask (bit a*8 + b: own slot a with
// neighbour slot b); the per-slot partner counts come out with it.
constexpr int kSearchWarps = 4;
constexpr float kBorderBand = 1.0e-4f;

__device__ bool excluded_scan(int glo, int ghi, const int* __restrict__ ex_start, const int* __restrict__ ex_list,
                              const int* __restrict__ ex_num)
{
    const int k = ex_num[glo];
    const int* l = ex_list + ex_start[glo];
    for (int t = 0; t < k; t++)
        if (l[t] == ghi) return true;
    return false;
}

__global__ void __launch_bounds__(kSearchWarps * 32, 5)
    k_search(const SysDesc* __restrict__ sys, int clusters_cap, int table_cap, const int* __restrict__ need,
             const int* __restrict__ ncl, const int* __restrict__ run_start, const int2* __restrict__ runs,
             const int2* __restrict__ cell_cl, const int* __restrict__ cl_cell,
             const int* __restrict__ cl_sys, const uint4* __restrict__ cl_u, const int4* __restrict__ cl_q,
             const float4* __restrict__ cl_c, const float4* __restrict__ slot_x0, const float4* __restrict__ slot_d0,
             const int2* __restrict__ slot_ex,
             const int* __restrict__ ex_start, const int* __restrict__ ex_list, const int* __restrict__ ex_num,
             int* __restrict__ tcount, float4* __restrict__ tab, uint2* __restrict__ tmask,
             int* __restrict__ slot_count, int* counters, const int* __restrict__ go, int half,
             const int* __restrict__ slot_atom, const unsigned char* __restrict__ two_sided_atoms)
{
    if (go && *go == 0) return;
    __shared__ float4 stage_t[kSearchWarps][kChunk];
    __shared__ uint2 stage_m[kSearchWarps][kChunk];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned long long elements = 0, listed = 0;

    // clusters are taken from a counter (their tables differ in length)
    for (;;)
    {
        int c = 0;
        if (lane == 0) c = atomicAdd(&counters[kCntSearchNext], 1);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= clusters_cap) break;
        const int sy = cl_sys[c];
        if (!need[sy] || c - sys[sy].cl_begin >= ncl[sy]) continue;
        const SysDesc& p = sys[sy];
        const int cellA = cl_cell[c];
        const uint4 ui = cl_u[c];
        const int4 qc = cl_q[c];
        const float ri = __uint_as_float(ui.w);
        const float4 hc = cl_c[c];
        const float band = kBorderBand * p.cs2;
        // one-sided table, unless the cluster holds an atom flagged for two sides
        bool one_sided = half != 0;
        if (one_sided && two_sided_atoms)
        {
            const int sa = slot_atom[c * kClusterSize + (lane & 7)];
            one_sided = !__any_sync(0xffffffffu, sa >= 0 && two_sided_atoms[sa]);
        }
        // the two own atoms this lane tests (rounds h = 0, 1)
        int ga[2];
        float3 xa[2], da[2];
        int2 ea[2];
        for (int h = 0; h < 2; h++)
        {
            const int a = h * 4 + (lane >> 3);
            const float4 x = slot_x0[c * kClusterSize + a];
            const float4 d = slot_d0[c * kClusterSize + a];
            ga[h] = __float_as_int(x.w);
            xa[h] = make_float3(x.x, x.y, x.z);
            da[h] = make_float3(d.x, d.y, d.z);
            ea[h] = slot_ex[c * kClusterSize + a];
        }
        unsigned row_count = 0;  // lanes 0-7: partners of own slot `lane`
        int written = 0, staged = 0;
        float4* __restrict__ my_tab = tab + (size_t)c * table_cap;
        uint2* __restrict__ my_mask = tmask + (size_t)c * table_cap;
        auto flush = [&](int count) {
            const int k = written + lane;
            if (lane < count && k < table_cap)
            {
                my_tab[k] = stage_t[wib][lane];
                my_mask[k] = stage_m[wib][lane];
            }
            if (lane == 0 && written + count > table_cap) atomicOr(&counters[kCntOverflow], kOvfPairs);
            written = min(written + count, table_cap);
            __syncwarp();
        };

        for (int r = run_start[cellA]; r < run_start[cellA + 1]; r++)
        {
            const int2 run = runs[r];
            const bool fwd = (run.x >> 28) & 1;  // the run's cells are in stencil(cellA)
            const bool rev = (run.x >> 29) & 1;  // cellA is in their stencils
            int b0 = cell_cl[run.x & 0x0fffffff].x;
            const int b1 = cell_cl[run.y - 1].y;
            for (; b0 < b1; b0 += 32)
            {
                const int cj = b0 + lane;
                bool ok = false;
                if (cj < b1 && (!one_sided || cj >= c))
                {
                    const uint4 uj = cl_u[cj];
                    const float3 f = frac_delta(ui, uj);
                    if (!p.triclinic)
                    {
                        // bounding boxes within the list radius
                        const float3 d = frac_to_cart(f, p.cell);
                        const float4 hj = cl_c[cj];
                        const float gx = fmaxf(fabsf(d.x) - (hc.x + hj.x), 0.0f);
                        const float gy = fmaxf(fabsf(d.y) - (hc.y + hj.y), 0.0f);
                        const float gz = fmaxf(fabsf(d.z) - (hc.z + hj.z), 0.0f);
                        ok = gx * gx + gy * gy + gz * gz < p.list_radius * p.list_radius;
                    }
                    else
                    {
                        const float rsum = ri + __uint_as_float(uj.w) + p.list_radius;
                        for (int im = 0; im < 27 && !ok; im++)
                        {
                            const float3 fi = make_float3(f.x + (float)(im / 9 - 1), f.y + (float)((im / 3) % 3 - 1),
                                                          f.z + (float)(im % 3 - 1));
                            const float3 d = frac_to_cart(fi, p.cell);
                            ok = d.x * d.x + d.y * d.y + d.z * d.z < rsum * rsum;
                        }
                    }
                }
                unsigned surv = __ballot_sync(0xffffffffu, ok);
                while (surv)
                {
                    const int cjs = b0 + __ffs(surv) - 1;
                    surv &= surv - 1;
                    const int b = lane & 7;
                    const float4 xj = slot_x0[cjs * kClusterSize + b];
                    const float4 dj = slot_d0[cjs * kClusterSize + b];
                    const int2 ej = slot_ex[cjs * kClusterSize + b];
                    const int gb = __float_as_int(xj.w);
                    const float3 xb = make_float3(xj.x, xj.y, xj.z);
                    // centre difference: minimum image of the 22-bit centres
                    const uint4 uj = cl_u[cjs];
                    const int4 qj = cl_q[cjs];
                    const float ux = (float)(((qj.x - qc.x + 0x200000) & 0x3fffff) - 0x200000);
                    const float uy = (float)(((qj.y - qc.y + 0x200000) & 0x3fffff) - 0x200000);
                    const float uz = (float)(((qj.z - qc.z + 0x200000) & 0x3fffff) - 0x200000);
                    const float Dx = ux * p.qcell.a11 + uy * p.qcell.a21 + uz * p.qcell.a31;
                    const float Dy = uy * p.qcell.a22 + uz * p.qcell.a32;
                    const float Dz = uz * p.qcell.a33;
                    // one image per cluster pair is enough when every pair of the
                    // two spheres stays inside half a box in fractional terms
                    bool safe = true;
                    if (!p.all_safe)
                    {
                        const float3 fd = frac_delta(ui, uj);
                        const float rr = ri + __uint_as_float(uj.w);
                        safe = fabsf(fd.x) + rr * p.frac_norm[0] < 0.49f && fabsf(fd.y) + rr * p.frac_norm[1] < 0.49f &&
                               fabsf(fd.z) + rr * p.frac_norm[2] < 0.49f;
                    }
                    unsigned bits[2];
                    // both rounds' distances first, then one vote for the border
                    // cases (the cheap distance only decides pairs well away
                    // from the threshold, so its rounding does not matter)
                    const float ex = Dx + dj.x, ey = Dy + dj.y, ez = Dz + dj.z;
                    const bool gb_ok = gb >= 0, self = cjs == c;
                    bool in_h[2], border_h[2], rule_h[2];
#pragma unroll
                    for (int h = 0; h < 2; h++)
                    {
                        const int a = h * 4 + (lane >> 3);
                        const bool a_lo = ga[h] < gb;
                        rule_h[h] = ga[h] >= 0 && gb_ok && (!self || b != a) && (a_lo ? fwd : rev);
                        const float dx = ex - da[h].x, dy = ey - da[h].y, dz = ez - da[h].z;
                        const float d2 = dx * dx + dy * dy + dz * dz;
                        border_h[h] = rule_h[h] && (!safe || fabsf(d2 - p.cs2) < band);
                        in_h[h] = d2 < p.cs2;
                    }
                    if (__any_sync(0xffffffffu, border_h[0] || border_h[1]))
                    {
#pragma unroll
                        for (int h = 0; h < 2; h++)
                            if (border_h[h])
                            {
                                const float e2 = ga[h] < gb ? ref_pair_dr2(xa[h], xb, p.cell, p.rcell)
                                                            : ref_pair_dr2(xb, xa[h], p.cell, p.rcell);
                                in_h[h] = e2 < p.cs2;
                            }
                    }
#pragma unroll
                    for (int h = 0; h < 2; h++)
                    {
                        const bool a_lo = ga[h] < gb;
                        bool in = in_h[h] && rule_h[h];
                        if (in)
                        {
                            // the lower index's exclusion list, scanned only within its range
                            const int2 e = a_lo ? ea[h] : ej;
                            const int glo = a_lo ? ga[h] : gb, ghi = a_lo ? gb : ga[h];
                            if (ghi >= e.x && ghi <= e.y) in = !excluded_scan(glo, ghi, ex_start, ex_list, ex_num);
                        }
                        bits[h] = __ballot_sync(0xffffffffu, in);
                    }
                    if (bits[0] | bits[1])
                    {
                        const unsigned long long m = ((unsigned long long)bits[1] << 32) | bits[0];
                        if (written + staged < table_cap && lane < 8) row_count += __popc((unsigned)(m >> (8 * lane)) & 0xffu);
                        if (lane == 0)
                        {
                            stage_t[wib][staged] = make_float4(Dx, Dy, Dz,
                                                               __int_as_float((cjs * kClusterSize) | (safe ? 0 : (1 << 30))));
                            stage_m[wib][staged] = make_uint2(bits[0], bits[1]);
                        }
                        staged++;
                        __syncwarp();
                        if (staged == kChunk)
                        {
                            flush(kChunk);
                            staged = 0;
                        }
                    }
                }
            }
        }
        if (staged > 0) flush(staged);
        if (lane < 8) slot_count[c * kClusterSize + lane] = (int)row_count;
        unsigned long long words = lane < 8 ? row_count : 0u;
        for (int o = 16; o > 0; o >>= 1) words += __shfl_xor_sync(0xffffffffu, words, o);
        if (lane == 0)
        {
            tcount[c] = written;
            elements += (unsigned long long)written;
            listed += words;
        }
    }
    if (lane == 0)
    {
        if (elements) atomicAdd((unsigned long long*)&counters[kCntEntries], elements);
        if (listed) atomicAdd((unsigned long long*)&counters[kCntWords], listed);
    }
}

// Reverse index of the tables, made after a search: k_rev_clear and
// k_rev_fill append every element (c, t) whose neighbour cluster J lies
// above c to J's list (an atomic cursor), then k_rev_sort puts each list in
// ascending element order (c, then t), so the index is the same on every
// call.  A list longer than table_cap sets the table overflow flag (the
// tables grow, as for the search's own overflow).  With need, only after a
// rebuild.
__global__ void k_rev_clear(int clusters_cap, int* __restrict__ rev_count, const int* __restrict__ need)
{
    if (need && *need == 0) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < clusters_cap) rev_count[c] = 0;
}

__global__ void k_rev_fill(int clusters_cap, int table_cap, const int* __restrict__ tcount,
                           const float4* __restrict__ tab, int* __restrict__ rev, int* __restrict__ rev_count,
                           int* counters, const int* __restrict__ need)
{
    if (need && *need == 0) return;
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < clusters_cap; c += warps)
    {
        const int T = tcount[c];
        for (int t = lane; t < T; t += 32)
        {
            const int J = (__float_as_int(tab[(size_t)c * table_cap + t].w) & 0x3fffffff) / kClusterSize;
            if (J <= c) continue;
            const int pos = atomicAdd(&rev_count[J], 1);
            if (pos < table_cap)
                rev[(size_t)J * table_cap + pos] = c * table_cap + t;
            else
                atomicOr(&counters[kCntOverflow], kOvfPairs);
        }
    }
}

constexpr int kRevWarps = 4;

// One warp per cluster: its list staged in shared memory; each entry's place
// is the number of entries below it (the entries differ).
__global__ void k_rev_sort(int clusters_cap, int table_cap, int* __restrict__ rev, const int* __restrict__ rev_count,
                           const int* __restrict__ need)
{
    if (need && *need == 0) return;
    extern __shared__ int rev_buf[];  // kRevWarps x table_cap
    const int lane = threadIdx.x & 31;
    int* b = rev_buf + (threadIdx.x >> 5) * table_cap;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < clusters_cap; c += warps)
    {
        const int m = min(rev_count[c], table_cap);
        int* r = rev + (size_t)c * table_cap;
        for (int k = lane; k < m; k += 32) b[k] = r[k];
        __syncwarp();
        for (int k = lane; k < m; k += 32)
        {
            const int v = b[k];
            int rank = 0;
            for (int q = 0; q < m; q++) rank += b[q] < v ? 1 : 0;
            r[rank] = v;
        }
        __syncwarp();
    }
}

// Reference-layout export: zero the counts, then every listed pair goes to
// its owner (the lower atom_local index) as the reference stores it.
__global__ void k_export_zero(int n, spgnb_atom_group* __restrict__ nl, const int* __restrict__ counters)
{
    if (counters[kCntNeed] == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        nl[i].atom_numbers = 0;
        nl[i].ghost_numbers = 0;
    }
}

// ATOM_GROUP lists from the cluster tables: one warp per cluster walks its
// own elements with J >= the cluster (its atoms' upper partners) and then
// its reverse index (the lower clusters' elements that hold it, whose masks
// give each own atom's column), a chunk of 32 elements at a time loaded once
// for the cluster's eight atoms; each atom's kept partners are compacted and
// appended to its list, so every partner on both sides comes once, in the
// same order on every call, with no atomics.
//   HALF: the reference-layout half list of NEIGHBOR_LIST::d_nl, each listed
//   pair with its owner (the lower atom_local index) as the reference stores
//   it; runs after a rebuild only (need: the device's rebuild flag).
//   full: FULL_NEIGHBOR_LIST::Build_From_Half / Build_From_Half_With_Cutoff
//   (full_neighbor_list.cpp:27-147), every listed pair in both atoms' lists.
//   With a cutoff, a pair is kept when its distance at d_crd is within it,
//   measured from the lower-index atom as the reference does
//   (Get_Periodic_Displacement(r_i, r_j)).
// A list longer than max_nb is cut and ovf_bits set in *overflow.
template <bool HALF>
__global__ void k_export_lists(int clusters_cap, int table_cap, const int* __restrict__ tcount,
                               const float4* __restrict__ tab, const uint2* __restrict__ tmask,
                               const int* __restrict__ slot_atom, const float4* __restrict__ slot_x0,
                               const int* __restrict__ slot_gid, const float3* __restrict__ crd, Cell cell,
                               Cell rcell, float cut2,
                               spgnb_atom_group* __restrict__ full, int max_nb, int* __restrict__ overflow,
                               int ovf_bits, const int* __restrict__ need, const int* __restrict__ rev,
                               const int* __restrict__ rev_count)
{
    if (HALF && *need == 0) return;
    // an atom's kept partners of a chunk, compacted here so that its list is
    // written with contiguous stores (blocks of 128 threads)
    __shared__ int staged[4][32 * kClusterSize];
    const int lane = threadIdx.x & 31;
    int* const stage = staged[threadIdx.x >> 5];
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < clusters_cap; c += warps)
    {
        const int T = tcount[c];
        const int V = T + min(rev_count[c], table_cap);  // own elements, then the reverse index
        // the cluster's own atoms (the same in every lane)
        int ia[kClusterSize], gia[kClusterSize], count[kClusterSize];
#pragma unroll
        for (int a = 0; a < kClusterSize; a++)
        {
            ia[a] = slot_atom[c * kClusterSize + a];
            gia[a] = __float_as_int(slot_x0[c * kClusterSize + a].w);
            count[a] = 0;
        }
        for (int t0 = 0; t0 < V; t0 += 32)
        {
            const int t = t0 + lane;
            uint2 mm = make_uint2(0u, 0u);
            bool col = false;  // a reverse element: the own atom's column of the mask
            int base = 0;
            if (t < T)
            {
                // a neighbour cluster below this one (a two-sided table) comes
                // from the reverse index
                base = __float_as_int(tab[(size_t)c * table_cap + t].w) & 0x3fffffff;
                if (base >= c * kClusterSize) mm = tmask[(size_t)c * table_cap + t];
            }
            else if (t < V)
            {
                const int e = rev[(size_t)c * table_cap + (t - T)];
                mm = tmask[e];
                base = (e / table_cap) * kClusterSize;
                col = true;
            }
            // the neighbour cluster's eight atoms (and global indices), in two
            // 16-byte loads each: a cluster's slots start on an 8-slot boundary
            int4 na0 = make_int4(-1, -1, -1, -1), na1 = na0, g0 = na0, g1 = na0;
            if (mm.x | mm.y)
            {
                const int4* sa = reinterpret_cast<const int4*>(slot_atom + base);
                na0 = sa[0];
                na1 = sa[1];
                if (HALF)
                {
                    const int4* sg = reinterpret_cast<const int4*>(slot_gid + base);
                    g0 = sg[0];
                    g1 = sg[1];
                }
            }
            const int nb[kClusterSize] = {na0.x, na0.y, na0.z, na0.w, na1.x, na1.y, na1.z, na1.w};
            const int gb[kClusterSize] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
#pragma unroll
            for (int a = 0; a < kClusterSize; a++)
            {
                if (ia[a] < 0) continue;  // warp-uniform
                unsigned row;
                if (col)
                {
                    // bit a' * 8 + a of the lower cluster's element
                    row = 0;
#pragma unroll
                    for (int q = 0; q < 4; q++)
                    {
                        row |= ((mm.x >> (8 * q + a)) & 1u) << q;
                        row |= ((mm.y >> (8 * q + a)) & 1u) << (q + 4);
                    }
                }
                else
                    row = ((a < 4 ? mm.x : mm.y) >> (8 * (a & 3))) & 0xffu;
                unsigned keep = row;
                if (HALF && row)
                {
                    unsigned above = 0;
#pragma unroll
                    for (int b = 0; b < kClusterSize; b++) above |= (gia[a] < gb[b] ? 1u : 0u) << b;
                    keep = row & above;
                }
                else if (!HALF && cut2 >= 0.0f && row)
                {
                    const float3 xi = crd[ia[a]];
                    keep = 0;
                    for (unsigned r = row; r; r &= r - 1)
                    {
                        const int b = __ffs(r) - 1;
                        const float3 xj = crd[nb[b]];
                        const bool i_lo = gia[a] < __float_as_int(slot_x0[base + b].w);
                        const float d2 = i_lo ? ref_pair_dr2(xi, xj, cell, rcell) : ref_pair_dr2(xj, xi, cell, rcell);
                        if (d2 <= cut2) keep |= 1u << b;
                    }
                }
                const int k = __popc(keep);
                int incl = k;
                for (int o = 1; o < 32; o <<= 1)
                {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                if (total == 0) continue;  // warp-uniform
                int pos = incl - k;
#pragma unroll
                for (int b = 0; b < kClusterSize; b++)
                    if ((keep >> b) & 1u) stage[pos++] = nb[b];
                __syncwarp();
                int* list = full[ia[a]].atom_serial;
                for (int q = lane; q < total; q += 32)
                {
                    if (count[a] + q < max_nb)
                        list[count[a] + q] = stage[q];
                    else
                        atomicOr(overflow, ovf_bits);
                }
                __syncwarp();
                count[a] += total;
            }
        }
        if (lane < kClusterSize)
        {
            int ca = 0, ja = -1;
#pragma unroll
            for (int a = 0; a < kClusterSize; a++)
                if (a == lane)
                {
                    ca = count[a];
                    ja = ia[a];
                }
            if (ja >= 0)
            {
                full[ja].atom_numbers = ca;
                full[ja].ghost_numbers = 0;
            }
        }
    }
}

__global__ void k_zero_groups(int n, spgnb_atom_group* __restrict__ g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        g[i].atom_numbers = 0;
        g[i].ghost_numbers = 0;
    }
}

__global__ void k_finish(int G, int S, const int* __restrict__ cell_sys, const int* __restrict__ need,
                         int* __restrict__ prune, int* __restrict__ cell_count, int* __restrict__ cell_cursor,
                         int* counters)
{
    if (counters[kCntNeed] == 0) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < G && need[cell_sys[c]])
    {
        cell_count[c] = 0;
        cell_cursor[c] = 0;
    }
    if (c < S && need[c])
    {
        prune[c] = 1;  // its pruned lists belong to the old build
        atomicAdd(&counters[kCntBuilds], 1);
        counters[kCntPrune] = 1;
    }
}

// Refresh by a fixed interval of steps (NEIGHBOR_LIST::Update with
// refresh_interval > 0), counted on the device per system: a system rebuilds
// when its own step count reaches a multiple of the interval, so a system's
// rebuilds do not depend on when it joined a batch.
__global__ void k_interval_need(int S, int interval, const int* __restrict__ steps, const int* __restrict__ live,
                                const int* __restrict__ active, int* __restrict__ need, int* counters)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const bool due = interval > 0 && live[s] && (!active || active[s] != 0) && (steps[s] + 1) % interval == 0;
    need[s] = due ? 1 : 0;
    if (due) counters[kCntNeed] = 1;
}

__global__ void k_set_need(int S, const int* __restrict__ live, const int* __restrict__ active,
                           int* __restrict__ need, int* counters)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const bool due = live[s] && (!active || active[s] != 0);
    need[s] = due ? 1 : 0;
    if (due) counters[kCntNeed] = 1;
}

__global__ void k_need_preset(int S, const int* __restrict__ flags, const int* __restrict__ live,
                              int* __restrict__ need, int* counters)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const bool due = live[s] && flags[s];
    need[s] = due ? 1 : 0;
    if (due) counters[kCntNeed] = 1;
}

__global__ void k_prune_live(int S, const int* __restrict__ live, int* __restrict__ prune, int* counters)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    prune[s] = live[s] ? 1 : 0;
    if (live[s]) counters[kCntPrune] = 1;
}

__global__ void k_fill_int(int* __restrict__ p, long long n, int v)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

// Before a search that re-makes the last build's tables two-sided: the
// cluster counter and the table statistics start again.
__global__ void k_sym_begin(int* counters)
{
    counters[kCntEntries] = 0;
    counters[kCntEntries + 1] = 0;
    counters[kCntWords] = 0;
    counters[kCntWords + 1] = 0;
    counters[kCntSearchNext] = 0;
}

__global__ void k_reset_list_counters(int* counters)
{
    if (counters[kCntNeed] == 0) return;
    counters[kCntItems] = 0;
    counters[kCntEntries] = 0;
    counters[kCntEntries + 1] = 0;
    counters[kCntWords] = 0;
    counters[kCntWords + 1] = 0;
    counters[kCntPWordsLast] = 0;
    counters[kCntPWordsLast + 1] = 0;
    counters[kCntSearchNext] = 0;
}

__global__ void k_init_atom_groups(int n, spgnb_atom_group* nl, int* temp, int max_nb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        nl[i].atom_numbers = 0;
        nl[i].ghost_numbers = 0;
        nl[i].atom_serial = temp + (size_t)i * max_nb;
    }
}

// --------------------------------------------------------------- host side

void grid_dims(const spgnb_ltmatrix3& cell, float cutoff, float skin, int dims[3], float* gl)
{
    const float g = 0.5f * (cutoff + skin);
    dims[0] = (int)floorf(cell.a11 / g);
    dims[1] = (int)floorf(cell.a22 / g);
    dims[2] = (int)floorf(cell.a33 / g);
    *gl = g;
}

// The reference's stencil rule (Find_Neighor_Grids_Device), evaluated per
// cell by enumerating the offsets instead of the O(G^2) scan.  A cell's
// candidates are the cells B with B in stencil(A) (flag 1) or A in
// stencil(B) (flag 2), grouped into runs of consecutive cell ids with equal
// flags: {first | flags << 28, last + 1}.  Cell ids count from the system's
// first cell; start gets G + 1 entries.
int build_runs(const SysHost& sh, std::vector<int>& start, std::vector<int2>& runs)
{
    start.assign(1, 0);
    runs.clear();
    const int Nx = sh.dims[0], Ny = sh.dims[1], Nz = sh.dims[2];
    const int G = Nx * Ny * Nz;
    const float gl = sh.gl;
    const spgnb_ltmatrix3& c = sh.cell;
    const int dxy = (int)(c.a21 / gl), dxz = (int)(c.a31 / gl), dyz = (int)(c.a32 / gl);
    std::vector<std::vector<int>> fwd(G);
    std::vector<int> mark(G, -1);
    for (int g = 0; g < G; g++)
    {
        const int gx = g / (Ny * Nz), gy = (g / Nz) % Ny, gz = g % Nz;
        for (int k = 0; k < 27; k++)
        {
            const int dx = k / 9 - 1, dy = (k % 9) / 3 - 1, dz = k % 3 - 1;
            const int cx = (dy * c.a21 + dz * c.a31 == 0) ? -2 : -3;
            const int cy = (dz * c.a32 == 0) ? -2 : -3;
            const int sx = gx + dx * Nx + dy * dxy + dz * dxz, sy = gy + dy * Ny + dz * dyz, sz = gz + dz * Nz;
            for (int tx = cx; tx <= 2; tx++)
                for (int ty = cy; ty <= 2; ty++)
                    for (int tz = -2; tz <= 2; tz++)
                    {
                        const int jx = sx - tx, jy = sy - ty, jz = sz - tz;
                        if (jx < 0 || jx >= Nx || jy < 0 || jy >= Ny || jz < 0 || jz >= Nz) continue;
                        const int j = (jx * Ny + jy) * Nz + jz;
                        if (mark[j] != g)
                        {
                            mark[j] = g;
                            fwd[g].push_back(j);
                        }
                    }
        }
        if ((int)fwd[g].size() > kMaxStencil)
            return fail(SPGNB_E_UNSUPPORTED, "stencil of %zu cells exceeds the reference's %d", fwd[g].size(),
                        kMaxStencil);
    }
    std::vector<std::vector<int>> rev(G);
    for (int g = 0; g < G; g++)
        for (int j : fwd[g]) rev[j].push_back(g);
    std::vector<int> flag(G, 0);
    std::vector<int> touched;
    for (int g = 0; g < G; g++)
    {
        touched.clear();
        for (int j : fwd[g])
        {
            if (!flag[j]) touched.push_back(j);
            flag[j] |= 1;
        }
        for (int j : rev[g])
        {
            if (!flag[j]) touched.push_back(j);
            flag[j] |= 2;
        }
        std::sort(touched.begin(), touched.end());
        for (size_t i = 0; i < touched.size();)
        {
            size_t e = i + 1;
            while (e < touched.size() && touched[e] == touched[e - 1] + 1 && flag[touched[e]] == flag[touched[i]]) e++;
            runs.push_back(make_int2(touched[i] | (flag[touched[i]] << 28), touched[e - 1] + 1));
            i = e;
        }
        for (int j : touched) flag[j] = 0;
        start.push_back((int)runs.size());
    }
    return SPGNB_OK;
}

int fill_int(int* p, long long n, int v, cudaStream_t s)
{
    if (n <= 0) return SPGNB_OK;
    const long long blocks = std::min<long long>((n + 255) / 256, 4096);
    k_fill_int<<<(int)blocks, 256, 0, s>>>(p, n, v);
    SPGNB_CHECK_LAUNCH("k_fill_int");
    return SPGNB_OK;
}

__global__ void k_sys_flags(int id, int live_value, int* live, int* need, int* prune, int* ncl)
{
    live[id] = live_value;
    need[id] = 0;
    prune[id] = 0;
    ncl[id] = 0;
}

void free_nl(spgnb_nl* nl)
{
    dfree(nl->d_sys);
    dfree(nl->d_atom_sys);
    dfree(nl->d_cell_sys);
    dfree(nl->d_run_start);
    dfree(nl->d_runs);
    dfree(nl->d_cell_count);
    dfree(nl->d_cell_cursor);
    dfree(nl->d_cell_cl);
    dfree(nl->d_live);
    dfree(nl->d_need);
    dfree(nl->d_prune);
    dfree(nl->d_ncl);
    dfree(nl->d_atom_cell);
    dfree(nl->d_atom_shift);
    dfree(nl->d_tmp_atoms);
    dfree(nl->d_wrapped);
    dfree(nl->d_atom_slot);
    dfree(nl->d_slot_atom);
    dfree(nl->d_slot_x0);
    dfree(nl->d_slot_gid);
    dfree(nl->d_slot_d0);
    dfree(nl->d_slot_ex);
    dfree(nl->d_slot_count);
    dfree(nl->d_cl_cell);
    dfree(nl->d_cl_sys);
    dfree(nl->d_cl_u);
    dfree(nl->d_cl_q);
    dfree(nl->d_cl_c);
    dfree(nl->d_tcount);
    dfree(nl->d_tab);
    dfree(nl->d_tmask);
    dfree(nl->d_pwords);
    dfree(nl->d_pcount);
    dfree(nl->d_facc);
    dfree(nl->d_oacc);
    dfree(nl->d_pref);
    dfree(nl->d_counters);
    dfree(nl->d_nl);
    dfree(nl->d_temp);
    dfree(nl->d_rev);
    dfree(nl->d_rev_count);
}

// The reverse index of the tables (clusters_cap x table_cap element indices).
int alloc_rev(spgnb_nl* nl)
{
    int st;
    dfree(nl->d_rev);
    dfree(nl->d_rev_count);
    nl->rev_built = false;
    const size_t n = (size_t)nl->clusters_cap * nl->table_cap;
    if (n >= (size_t)0x7fffffff)
        return fail(SPGNB_E_UNSUPPORTED, "neighbour list: %zu table elements exceed the reverse index's int range", n);
    if ((st = dalloc(&nl->d_rev, n))) return st;
    return dalloc(&nl->d_rev_count, nl->clusters_cap);
}

int alloc_tables(spgnb_nl* nl)
{
    int st;
    dfree(nl->d_tab);
    dfree(nl->d_tmask);
    const size_t n = (size_t)nl->clusters_cap * nl->table_cap;
    if ((st = dalloc(&nl->d_tab, n))) return st;
    if ((st = dalloc(&nl->d_tmask, n))) return st;
    // the reverse index follows the tables' size once it exists
    return nl->d_rev ? alloc_rev(nl) : SPGNB_OK;
}

// Makes the reverse index from the current tables (with need, only when the
// device's rebuild flag is set).
int build_rev(const spgnb_nl* nl, cudaStream_t s, const int* need)
{
    const int ccap = nl->clusters_cap;
    const size_t smem = sizeof(int) * kRevWarps * (size_t)nl->table_cap;
    if (smem > 227 * 1024)
        return fail(SPGNB_E_UNSUPPORTED, "neighbour list: %d table elements per cluster exceed the reverse index's "
                                         "sort", nl->table_cap);
    const int warp_blocks = std::max(1, std::min((ccap + kRevWarps - 1) / kRevWarps, num_sms() * 16));
    k_rev_clear<<<(ccap + 255) / 256, 256, 0, s>>>(ccap, nl->d_rev_count, need);
    SPGNB_CHECK_LAUNCH("k_rev_clear");
    k_rev_fill<<<warp_blocks, kRevWarps * 32, 0, s>>>(ccap, nl->table_cap, nl->d_tcount, nl->d_tab, nl->d_rev,
                                                      nl->d_rev_count, nl->d_counters, need);
    SPGNB_CHECK_LAUNCH("k_rev_fill");
    if (smem > 48 * 1024)
        SPGNB_CUDA(cudaFuncSetAttribute(k_rev_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_rev_sort<<<warp_blocks, kRevWarps * 32, smem, s>>>(ccap, nl->table_cap, nl->d_rev, nl->d_rev_count, need);
    SPGNB_CHECK_LAUNCH("k_rev_sort");
    nl->rev_built = true;
    return SPGNB_OK;
}

// The pruned lists: list_cap words per cluster.
int alloc_words(spgnb_nl* nl)
{
    dfree(nl->d_pwords);
    return dalloc(&nl->d_pwords, (size_t)nl->clusters_cap * nl->list_cap);
}

// Squared radius of the pruned lists for the pruning cutoff rc.
float prune_r2_of(float rc, float buffer)
{
    if (!(buffer > 0.0f)) return 3.0e38f;
    const float r = rc + buffer + 1e-3f;
    return r * r;
}

SysDesc make_desc(const SysHost& sh, float skin_permit)
{
    SysDesc d{};
    d.cell = make_cell(sh.cell);
    d.rcell = make_cell(sh.rcell);
    d.gl = sh.gl;
    d.cs2 = sh.cs2;
    d.list_radius = sqrtf(sh.cs2) * 1.0001f + 1e-3f;
    d.frac_norm[0] = sqrtf(d.rcell.a11 * d.rcell.a11 + d.rcell.a21 * d.rcell.a21 + d.rcell.a31 * d.rcell.a31);
    d.frac_norm[1] = sqrtf(d.rcell.a22 * d.rcell.a22 + d.rcell.a32 * d.rcell.a32);
    d.frac_norm[2] = fabsf(d.rcell.a33);
    d.Nx = sh.dims[0];
    d.Ny = sh.dims[1];
    d.Nz = sh.dims[2];
    d.cell_begin = sh.cell_begin;
    d.cl_begin = sh.cl_begin;
    d.cl_cap = sh.cl_cap;
    d.atom_begin = sh.atom_begin;
    d.atom_count = sh.atom_count;
    d.triclinic = sh.triclinic ? 1 : 0;
    const float permit = sh.skin * skin_permit;
    d.permit2 = permit * permit;
    // a cluster lies inside one grid cell (the last cell of a row is the
    // widest, up to the box edge), so its centre is within half a cell
    // diagonal of its atoms; every pair the search meets then has fractional
    // separation below (list radius + 4 half diagonals) * |rcell row|
    const float wx = fmaxf(sh.gl, sh.cell.a11 - (sh.dims[0] - 1) * sh.gl);
    const float wy = fmaxf(sh.gl, sh.cell.a22 - (sh.dims[1] - 1) * sh.gl);
    const float wz = fmaxf(sh.gl, sh.cell.a33 - (sh.dims[2] - 1) * sh.gl);
    const float hd = 0.5f * sqrtf(wx * wx + wy * wy + wz * wz) + 1e-3f;
    const float fmax_norm = fmaxf(d.frac_norm[0], fmaxf(d.frac_norm[1], d.frac_norm[2]));
    d.all_safe = (!sh.triclinic && (d.list_radius + 4.0f * hd) * fmax_norm < 0.45f) ? 1 : 0;
    d.prune_r2 = 3.0e38f;  // set by the caller
    const float q = 2.384185791015625e-07f;  // 2^-22, exact scaling
    d.qcell = Cell{d.cell.a11 * q, d.cell.a21 * q, d.cell.a22 * q, d.cell.a31 * q, d.cell.a32 * q, d.cell.a33 * q};
    return d;
}

// Arrays for the pool's capacities, every range parked.
int alloc_nl(spgnb_nl* nl)
{
    int st;
    const int n = nl->n_cap, G = nl->G, S = nl->S;
    if (((long long)nl->clusters_cap + 1) * kClusterSize > kMaxSlots)
        return fail(SPGNB_E_UNSUPPORTED, "neighbour list: %d clusters exceed the %d-slot limit of the lists",
                    nl->clusters_cap, kMaxSlots);
    const size_t slots = (size_t)nl->clusters_cap * kClusterSize;
    nl->sys.assign(S, SysHost{});
    nl->live.assign(S, 0);
    nl->free_ids.clear();
    for (int i = 0; i < S; i++) nl->free_ids.insert(i);
    nl->cell_pool.reset(G);
    nl->cl_pool.reset(nl->clusters_cap);
    nl->run_pool.reset(nl->runs_cap);
    nl->h_desc.assign(S + 1, SysDesc{});
    cudaStream_t s0 = nullptr;
    if ((st = dalloc(&nl->d_sys, S + 1))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_sys, 0, sizeof(SysDesc) * (S + 1)));
    if ((st = dalloc(&nl->d_atom_sys, n))) return st;
    if ((st = fill_int(nl->d_atom_sys, n, S, s0))) return st;
    if ((st = dalloc(&nl->d_cell_sys, G))) return st;
    if ((st = fill_int(nl->d_cell_sys, G, S, s0))) return st;
    if ((st = dalloc(&nl->d_run_start, G + 1))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_run_start, 0, sizeof(int) * (G + 1)));
    if ((st = dalloc(&nl->d_runs, nl->runs_cap))) return st;
    if ((st = dalloc(&nl->d_cell_count, G))) return st;
    if ((st = dalloc(&nl->d_cell_cursor, G))) return st;
    if ((st = dalloc(&nl->d_cell_cl, G))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_cell_cl, 0, sizeof(int2) * G));
    SPGNB_CUDA(cudaMemset(nl->d_cell_count, 0, sizeof(int) * G));
    SPGNB_CUDA(cudaMemset(nl->d_cell_cursor, 0, sizeof(int) * G));
    if ((st = dalloc(&nl->d_live, S + 1))) return st;
    if ((st = dalloc(&nl->d_need, S + 1))) return st;
    if ((st = dalloc(&nl->d_prune, S + 1))) return st;
    if ((st = dalloc(&nl->d_ncl, S + 1))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_live, 0, sizeof(int) * (S + 1)));
    SPGNB_CUDA(cudaMemset(nl->d_need, 0, sizeof(int) * (S + 1)));
    SPGNB_CUDA(cudaMemset(nl->d_prune, 0, sizeof(int) * (S + 1)));
    SPGNB_CUDA(cudaMemset(nl->d_ncl, 0, sizeof(int) * (S + 1)));
    if ((st = dalloc(&nl->d_atom_cell, n))) return st;
    if ((st = dalloc(&nl->d_atom_shift, n))) return st;
    if ((st = dalloc(&nl->d_wrapped, n))) return st;
    if ((st = dalloc(&nl->d_atom_slot, n))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_atom_slot, 0xff, sizeof(int) * n));
    if ((st = dalloc(&nl->d_tmp_atoms, slots))) return st;
    if ((st = dalloc(&nl->d_slot_atom, slots))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_slot_atom, 0xff, sizeof(int) * slots));
    if ((st = dalloc(&nl->d_slot_x0, slots))) return st;
    if ((st = dalloc(&nl->d_slot_gid, slots))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_slot_gid, 0xff, sizeof(int) * slots));
    if ((st = dalloc(&nl->d_slot_d0, slots))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_slot_d0, 0, sizeof(float4) * slots));
    if ((st = dalloc(&nl->d_slot_ex, slots))) return st;
    if ((st = dalloc(&nl->d_slot_count, slots))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_slot_count, 0, sizeof(int) * slots));
    if ((st = dalloc(&nl->d_pcount, slots))) return st;
    if ((st = dalloc(&nl->d_facc, 3 * (size_t)slots))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_facc, 0, sizeof(long long) * 3 * (size_t)slots));
    if ((st = dalloc(&nl->d_oacc, 8 * (size_t)slots))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_oacc, 0, sizeof(long long) * 8 * (size_t)slots));
    if ((st = dalloc(&nl->d_pref, slots))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_pcount, 0, sizeof(int) * slots));
    if ((st = dalloc(&nl->d_cl_cell, nl->clusters_cap))) return st;
    if ((st = dalloc(&nl->d_cl_sys, nl->clusters_cap))) return st;
    if ((st = fill_int(nl->d_cl_sys, nl->clusters_cap, S, s0))) return st;
    if ((st = dalloc(&nl->d_cl_u, nl->clusters_cap))) return st;
    // one more: the null cluster of the padding slot (centre 0)
    if ((st = dalloc(&nl->d_cl_q, nl->clusters_cap + 1))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_cl_q, 0, sizeof(int4) * (nl->clusters_cap + 1)));
    if ((st = dalloc(&nl->d_cl_c, nl->clusters_cap))) return st;
    if ((st = dalloc(&nl->d_tcount, nl->clusters_cap))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_tcount, 0, sizeof(int) * nl->clusters_cap));
    if ((st = dalloc(&nl->d_counters, kCntSize))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_counters, 0, sizeof(int) * kCntSize));
    if ((st = alloc_tables(nl))) return st;
    if ((st = alloc_words(nl))) return st;
    // the reference-layout export reads each atom's partners on both sides,
    // the lower ones through the reverse index
    if (nl->opt.export_atom_groups && (st = alloc_rev(nl))) return st;
    if (nl->opt.export_atom_groups)
    {
        if ((st = dalloc(&nl->d_nl, n))) return st;
        if ((st = dalloc(&nl->d_temp, (size_t)n * nl->opt.max_neighbor_numbers))) return st;
        k_init_atom_groups<<<(n + 255) / 256, 256>>>(n, nl->d_nl, nl->d_temp, nl->opt.max_neighbor_numbers);
        SPGNB_CHECK_LAUNCH("k_init_atom_groups");
    }
    SPGNB_CUDA(cudaDeviceSynchronize());
    return SPGNB_OK;
}

int table_cap_for(double per_cluster) { return std::max((int)(per_cluster * 1.3) + 64, 128); }

void resolve_options(const spgnb_nl_options* opt, spgnb_nl_options* o)
{
    if (opt)
        *o = *opt;
    else
        spgnb_nl_default_options(o);
    if (o->max_neighbor_numbers <= 0) o->max_neighbor_numbers = 1200;
    if (!(o->prune_buffer >= 0.0f)) o->prune_buffer = 0.0f;
}

}  // namespace

int list_cap_for(double per_cluster) { return (((int)(per_cluster * 1.3) + 31) & ~31) + 64; }

void nl_capacity_for(double atoms_per_A3, double atom_count, float cutoff, float skin, float prune_buffer,
                     double* table_per_cluster, double* words_per_cluster)
{
    // neighbour clusters within rc + skin + 6 A of an 8-atom cluster; pruned
    // partners of a cluster (any of its atoms within rc + buffer) within
    // rc + buffer + 1 A of a sphere holding the cluster (radius 2.5 A)
    const double R = cutoff + skin + 6.0;
    *table_per_cluster = std::min(4.18879 * R * R * R * atoms_per_A3, atom_count) / kClusterSize;
    const double buf = prune_buffer > 0.0f ? prune_buffer + 1.0 : skin;
    const double Rl = cutoff + buf + 2.5;
    *words_per_cluster = std::min(4.18879 * Rl * Rl * Rl * atoms_per_A3, atom_count);
}

int nl_init_system(SysHost& sh, int atom_count, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, float cutoff,
                   float skin, int index)
{
    if (atom_count <= 0 || !(cutoff > 0.0f) || !(skin >= 0.0f) ||
        !(cell.a11 > 0.0f && cell.a22 > 0.0f && cell.a33 > 0.0f))
        return fail(SPGNB_E_ARG, "neighbour list: system %d has bad atoms/cutoff/skin/cell", index);
    sh = SysHost{};
    sh.atom_count = atom_count;
    sh.cell = cell;
    sh.rcell = rcell;
    sh.cutoff = cutoff;
    sh.skin = skin;
    sh.triclinic = cell.a21 != 0.0f || cell.a31 != 0.0f || cell.a32 != 0.0f;
    grid_dims(cell, cutoff, skin, sh.dims, &sh.gl);
    sh.cs2 = sh.gl * sh.gl * 4.0f;
    if (sh.dims[0] <= 2 || sh.dims[1] <= 2 || sh.dims[2] <= 2)
        return fail(SPGNB_E_ARG,
                    "NEIGHBOR_LIST: the box is too small (system %d: grid %dx%dx%d, need >= 3 per dimension)", index,
                    sh.dims[0], sh.dims[1], sh.dims[2]);
    return SPGNB_OK;
}

int nl_system_runs(const SysHost& sh, std::vector<int>& run_start, std::vector<int2>& runs)
{
    return build_runs(sh, run_start, runs);
}

int nl_create_pool(const NLPoolSpec& spec, const spgnb_nl_options* opt, spgnb_nl** out)
{
    *out = nullptr;
    if (spec.systems <= 0 || spec.atoms <= 0 || spec.cells <= 0 || spec.clusters <= 0 || spec.runs <= 0 ||
        spec.table_cap <= 0 || spec.list_cap <= 0)
        return fail(SPGNB_E_ARG, "neighbour list: empty pool capacities");
    if (spec.atoms > (1 << 28) || spec.cells >= (1 << 28))
        return fail(SPGNB_E_UNSUPPORTED, "neighbour list: %d atoms / %d cells exceed the 2^28 limit", spec.atoms,
                    spec.cells);
    spgnb_nl* nl = new spgnb_nl();
    resolve_options(opt, &nl->opt);
    nl->S = spec.systems;
    nl->n_cap = spec.atoms;
    nl->G = spec.cells;
    nl->clusters_cap = spec.clusters;
    nl->runs_cap = spec.runs;
    nl->table_cap = nl->opt.max_entries_per_cluster > 0 ? nl->opt.max_entries_per_cluster : spec.table_cap;
    nl->list_cap = spec.list_cap;
    nl->prune_rc = spec.prune_rc;
    const int st = alloc_nl(nl);
    if (st)
    {
        free_nl(nl);
        delete nl;
        return st;
    }
    *out = nl;
    return SPGNB_OK;
}

int Uploader::put(void* dst, const void* src, size_t bytes, cudaStream_t s)
{
    if (bytes == 0) return SPGNB_OK;
    const void* from = src;
    if (st)
    {
        if (st->used + bytes > st->cap) return fail(SPGNB_E_STATE, "upload staging buffer too small");
        memcpy(st->p + st->used, src, bytes);
        from = st->p + st->used;
        st->used += (bytes + 15) & ~(size_t)15;
    }
    SPGNB_CUDA(cudaMemcpyAsync(dst, from, bytes, cudaMemcpyHostToDevice, s));
    return SPGNB_OK;
}

size_t nl_admit_upload_bytes(const SysHost& sh, size_t n_runs)
{
    return sizeof(SysDesc) + 16 + n_runs * sizeof(int2) + 16 + (size_t)(sh.cells() + 1) * sizeof(int) + 16;
}

int nl_admit(spgnb_nl* nl, SysHost sh, const std::vector<int>* run_start, const std::vector<int2>* runs,
             cudaStream_t s, int* id, Uploader up)
{
    int st;
    std::vector<int> start_own;
    std::vector<int2> runs_own;
    if (!run_start || !runs)
    {
        if ((st = build_runs(sh, start_own, runs_own))) return st;
        run_start = &start_own;
        runs = &runs_own;
    }
    const int G = sh.cells();
    if ((int)run_start->size() != G + 1) return fail(SPGNB_E_ARG, "nl_admit: run table of the wrong size");
    if (sh.atom_begin < 0 || (long long)sh.atom_begin + sh.atom_count > nl->n_cap)
        return fail(SPGNB_E_ARG, "nl_admit: atoms outside the pool");
    const long long cl_cap = sh.atom_count / kClusterSize + G + 1;
    if (cl_cap * kClusterSize > kMaxSystemSlots)
        return fail(SPGNB_E_UNSUPPORTED, "neighbour list: a system of %d atoms in %d cells exceeds the %d slots of one "
                                         "system's lists", sh.atom_count, G, kMaxSystemSlots);
    if (nl->free_ids.empty()) return SPGNB_E_OOM;
    const long long cb = nl->cell_pool.alloc(G + 1);
    if (cb < 0) return SPGNB_E_OOM;
    const long long clb = nl->cl_pool.alloc(cl_cap);
    if (clb < 0)
    {
        nl->cell_pool.release(cb, G + 1);
        return SPGNB_E_OOM;
    }
    const long long nr = (long long)runs->size();
    const long long rb = nl->run_pool.alloc(nr);
    if (rb < 0)
    {
        nl->cl_pool.release(clb, cl_cap);
        nl->cell_pool.release(cb, G + 1);
        return SPGNB_E_OOM;
    }
    const int sid = *nl->free_ids.begin();
    nl->free_ids.erase(nl->free_ids.begin());
    sh.cell_begin = (int)cb;
    sh.cl_begin = (int)clb;
    sh.cl_cap = (int)cl_cap;
    sh.run_begin = rb;
    sh.run_count = nr;
    std::vector<int2> ra(nr);
    for (long long k = 0; k < nr; k++) ra[k] = make_int2((*runs)[k].x + (int)cb, (*runs)[k].y + (int)cb);
    std::vector<int> sa(G + 1);
    for (int g = 0; g <= G; g++) sa[g] = (*run_start)[g] + (int)rb;
    nl->h_desc[sid] = make_desc(sh, nl->opt.skin_permit);
    nl->h_desc[sid].prune_r2 = prune_r2_of(nl->prune_rc, nl->opt.prune_buffer);
    // recorded before the uploads, so a failing one can hand everything back
    nl->sys[sid] = sh;
    nl->live[sid] = 1;
    if ((st = up.put(nl->d_sys + sid, &nl->h_desc[sid], sizeof(SysDesc), s)) ||
        (st = up.put(nl->d_runs + rb, ra.data(), sizeof(int2) * nr, s)) ||
        (st = up.put(nl->d_run_start + cb, sa.data(), sizeof(int) * (G + 1), s)) ||
        (st = fill_int(nl->d_atom_sys + sh.atom_begin, sh.atom_count, sid, s)) ||
        (st = fill_int(nl->d_cell_sys + cb, G, sid, s)) || (st = fill_int(nl->d_cl_sys + clb, cl_cap, sid, s)))
    {
        nl_retire(nl, sid, s);
        return st;
    }
    k_sys_flags<<<1, 1, 0, s>>>(sid, 1, nl->d_live, nl->d_need, nl->d_prune, nl->d_ncl);
    SPGNB_CHECK_LAUNCH("k_sys_flags");
    nl->triclinic = nl->triclinic || sh.triclinic;
    *id = sid;
    return SPGNB_OK;
}

int nl_retire(spgnb_nl* nl, int id, cudaStream_t s)
{
    int st;
    if (id < 0 || id >= nl->S || !nl->live[id]) return fail(SPGNB_E_ARG, "nl_retire: system %d is not in the list", id);
    const SysHost sh = nl->sys[id];
    const int G = sh.cells();
    const size_t slot0 = (size_t)sh.cl_begin * kClusterSize, nslots = (size_t)sh.cl_cap * kClusterSize;
    if ((st = fill_int(nl->d_atom_sys + sh.atom_begin, sh.atom_count, nl->S, s))) return st;
    SPGNB_CUDA(cudaMemsetAsync(nl->d_atom_slot + sh.atom_begin, 0xff, sizeof(int) * sh.atom_count, s));
    if ((st = fill_int(nl->d_cell_sys + sh.cell_begin, G, nl->S, s))) return st;
    SPGNB_CUDA(cudaMemsetAsync(nl->d_cell_count + sh.cell_begin, 0, sizeof(int) * (G + 1), s));
    SPGNB_CUDA(cudaMemsetAsync(nl->d_cell_cursor + sh.cell_begin, 0, sizeof(int) * (G + 1), s));
    if ((st = fill_int(nl->d_cl_sys + sh.cl_begin, sh.cl_cap, nl->S, s))) return st;
    SPGNB_CUDA(cudaMemsetAsync(nl->d_slot_atom + slot0, 0xff, sizeof(int) * nslots, s));
    SPGNB_CUDA(cudaMemsetAsync(nl->d_slot_count + slot0, 0, sizeof(int) * nslots, s));
    SPGNB_CUDA(cudaMemsetAsync(nl->d_pcount + slot0, 0, sizeof(int) * nslots, s));
    SPGNB_CUDA(cudaMemsetAsync(nl->d_tcount + sh.cl_begin, 0, sizeof(int) * sh.cl_cap, s));
    k_sys_flags<<<1, 1, 0, s>>>(id, 0, nl->d_live, nl->d_need, nl->d_prune, nl->d_ncl);
    SPGNB_CHECK_LAUNCH("k_sys_flags");
    nl->cell_pool.release(sh.cell_begin, G + 1);
    nl->cl_pool.release(sh.cl_begin, sh.cl_cap);
    nl->run_pool.release(sh.run_begin, sh.run_count);
    nl->free_ids.insert(id);
    nl->live[id] = 0;
    nl->sys[id] = SysHost{};
    nl->h_desc[id] = SysDesc{};
    nl->triclinic = false;
    for (int k = 0; k < nl->S; k++) nl->triclinic = nl->triclinic || (nl->live[k] && nl->sys[k].triclinic);
    return SPGNB_OK;
}

int nl_prune_all(spgnb_nl* nl, cudaStream_t s)
{
    k_prune_live<<<(nl->S + 255) / 256, 256, 0, s>>>(nl->S, nl->d_live, nl->d_prune, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_prune_live");
    return SPGNB_OK;
}

size_t nl_device_bytes(const spgnb_nl* nl)
{
    const size_t n = nl->n_cap, G = nl->G, S = nl->S + 1, C = nl->clusters_cap, slots = C * kClusterSize;
    size_t b = 0;
    b += n * (4 + 4 + 4 + 16 + 4);                                   // atom system, cell, shift, wrapped, slot
    b += slots * (4 + 4 + 16 + 4 + 16 + 8 + 4 + 4 + 24 + 64 + 16);   // per-slot arrays (with the int64 staging)
    b += C * (size_t)nl->list_cap * 4;                               // pruned lists
    b += C * (4 + 4 + 16 + 16 + 16 + 4) + 16;                        // per-cluster arrays
    b += C * (size_t)nl->table_cap * (16 + 8);                       // neighbour tables
    b += G * (4 + 4 + 4 + 8 + 4) + 4 + (size_t)nl->runs_cap * 8;     // cells and runs
    b += S * (sizeof(SysDesc) + 16);
    if (nl->opt.export_atom_groups) b += n * sizeof(spgnb_atom_group) + n * (size_t)nl->opt.max_neighbor_numbers * 4;
    return b;
}

int nl_create_multi(int n_systems, const int* atom_counts, const spgnb_ltmatrix3* cells,
                    const spgnb_ltmatrix3* rcells, const float* cutoffs, const float* skins,
                    const spgnb_nl_options* opt, spgnb_nl** out)
{
    *out = nullptr;
    if (n_systems <= 0) return fail(SPGNB_E_ARG, "neighbour list: no systems");
    int st;
    spgnb_nl_options o;
    resolve_options(opt, &o);
    std::vector<SysHost> hs(n_systems);
    std::vector<std::vector<int>> starts(n_systems);
    std::vector<std::vector<int2>> runs(n_systems);
    long long atoms = 0, cellsum = 0, clsum = 0, runsum = 0;
    double per_cluster = 0, per_list = 0;
    float rcmax = 0;
    for (int s = 0; s < n_systems; s++)
    {
        if ((st = nl_init_system(hs[s], atom_counts[s], cells[s], rcells[s], cutoffs[s], skins[s], s))) return st;
        hs[s].atom_begin = (int)std::min<long long>(atoms, 0x7fffffff);
        atoms += atom_counts[s];
        if ((st = build_runs(hs[s], starts[s], runs[s]))) return st;
        const int G = hs[s].cells();
        cellsum += G + 1;
        clsum += atom_counts[s] / kClusterSize + G + 1;
        runsum += (long long)runs[s].size();
        const double vol = (double)cells[s].a11 * cells[s].a22 * cells[s].a33;
        double pc, pa;
        nl_capacity_for(atom_counts[s] / vol, atom_counts[s], cutoffs[s], skins[s], o.prune_buffer, &pc, &pa);
        per_cluster = std::max(per_cluster, pc);
        per_list = std::max(per_list, pa);
        rcmax = std::max(rcmax, cutoffs[s]);
    }
    if (atoms > (1LL << 28)) return fail(SPGNB_E_UNSUPPORTED, "neighbour list: %lld atoms exceed the 2^28 limit", atoms);
    if ((clsum + 1) * kClusterSize > kMaxSlots)
        return fail(SPGNB_E_UNSUPPORTED, "neighbour list: %lld atoms in %lld cells exceed the %d-slot limit of the lists",
                    atoms, cellsum, kMaxSlots);
    NLPoolSpec spec;
    spec.systems = n_systems;
    spec.atoms = (int)atoms;
    spec.cells = (int)cellsum;
    spec.clusters = (int)clsum;
    spec.runs = std::max(1LL, runsum);
    spec.table_cap = table_cap_for(per_cluster);
    spec.list_cap = list_cap_for(per_list);
    spec.prune_rc = rcmax;
    spgnb_nl* nl = nullptr;
    if ((st = nl_create_pool(spec, &o, &nl))) return st;
    cudaStream_t s0 = stream();
    for (int s = 0; s < n_systems; s++)
    {
        int id = -1;
        st = nl_admit(nl, hs[s], &starts[s], &runs[s], s0, &id);
        if (st || id != s)
        {
            free_nl(nl);
            delete nl;
            return st ? (st == SPGNB_E_OOM ? fail(st, "neighbour list: pool sizing error") : st)
                      : fail(SPGNB_E_STATE, "neighbour list: unexpected system id");
        }
    }
    cudaError_t e = cudaStreamSynchronize(s0);
    if (e != cudaSuccess)
    {
        free_nl(nl);
        delete nl;
        return cuda_fail(e, "nl_create_multi");
    }
    nl->cutoff = nl->sys[0].cutoff;
    nl->skin = nl->sys[0].skin;
    nl->grid_length = nl->sys[0].gl;
    nl->cs2 = nl->sys[0].cs2;
    nl->cell = nl->sys[0].cell;
    nl->rcell = nl->sys[0].rcell;
    memcpy(nl->dims, nl->sys[0].dims, sizeof(nl->dims));
    *out = nl;
    return SPGNB_OK;
}

// Queues one rebuild, or the device-side decision about one, on stream s.
// how: kBuildForced rebuilds every live system, kBuildSkin lets each
// system's skin check decide, kBuildInterval rebuilds a system when its step
// count (aux) reaches a multiple of `interval`, kBuildPreset rebuilds the
// systems flagged in aux.
int nl_queue_build(spgnb_nl* nl, int n, const float3* d_crd, const int* d_atom_local, const int* ex_start,
                   const int* ex_list, const int* ex_num, int how, cudaStream_t s, const int* d_aux, int interval,
                   const int* d_active)
{
    const int slots_cap = nl->clusters_cap * kClusterSize;
    const int sb = (nl->S + 255) / 256;
    if (how != kBuildSkin)
    {
        if ((how == kBuildInterval || how == kBuildPreset) && !d_aux)
            return fail(SPGNB_E_ARG, "nl_queue_build: per-system steps or flags missing");
        SPGNB_CUDA(cudaMemsetAsync(nl->d_counters + kCntNeed, 0, sizeof(int), s));
        if (how == kBuildForced)
            k_set_need<<<sb, 256, 0, s>>>(nl->S, nl->d_live, d_active, nl->d_need, nl->d_counters);
        else if (how == kBuildInterval)
            k_interval_need<<<sb, 256, 0, s>>>(nl->S, interval, d_aux, nl->d_live, d_active, nl->d_need,
                                               nl->d_counters);
        else
            k_need_preset<<<sb, 256, 0, s>>>(nl->S, d_aux, nl->d_live, nl->d_need, nl->d_counters);
        SPGNB_CHECK_LAUNCH("k_need");
    }
    else
    {
        SPGNB_CUDA(cudaMemsetAsync(nl->d_counters + kCntNeed, 0, sizeof(int), s));
        SPGNB_CUDA(cudaMemsetAsync(nl->d_need, 0, sizeof(int) * nl->S, s));
        k_check_refresh<<<(slots_cap + 255) / 256, 256, 0, s>>>(slots_cap, nl->d_slot_atom, nl->d_cl_sys, nl->d_sys,
                                                                  d_crd, nl->d_slot_x0, nl->d_need, nl->d_counters);
        SPGNB_CHECK_LAUNCH("k_check_refresh");
    }
    return nl_queue_build_body(nl, n, d_crd, d_atom_local, ex_start, ex_list, ex_num, s);
}

int nl_queue_build_body(spgnb_nl* nl, int n, const float3* d_crd, const int* d_atom_local, const int* ex_start,
                        const int* ex_list, const int* ex_num, cudaStream_t s)
{
    const int sms = num_sms();
    const int slots_cap = nl->clusters_cap * kClusterSize;
    const int ccap = nl->clusters_cap;
    k_reset_list_counters<<<1, 1, 0, s>>>(nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_reset_list_counters");
    k_bin<<<(n + 255) / 256, 256, 0, s>>>(n, d_crd, nl->d_atom_sys, nl->d_sys, nl->d_atom_cell, nl->d_atom_shift,
                                            nl->d_wrapped, nl->d_cell_count, nl->d_need, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_bin");
    k_scan_cells<<<nl->S, 1024, 0, s>>>(nl->d_sys, nl->d_cell_count, nl->d_cell_cl, nl->opt.max_atom_in_grid_numbers,
                                         nl->d_need, nl->d_ncl, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_scan_cells");
    k_scatter<<<(n + 255) / 256, 256, 0, s>>>(n, nl->d_atom_sys, nl->d_atom_cell, nl->d_cell_cl, nl->d_ncl, nl->d_sys,
                                                nl->d_cell_cursor, nl->d_tmp_atoms, nl->d_need, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_scatter");
    k_sort_cells<<<std::min(nl->G, sms * 16), 128, kMaxCellAtoms * sizeof(unsigned long long), s>>>(
        nl->G, nl->d_cell_sys, nl->d_sys, nl->d_cell_count, nl->d_cell_cl, nl->d_ncl, nl->d_tmp_atoms, nl->d_wrapped,
        nl->d_slot_atom, nl->d_cl_cell, nl->d_atom_slot, nl->d_need, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_sort_cells");
    k_cluster_props<<<(slots_cap + 255) / 256, 256, 0, s>>>(
        d_crd, nl->d_slot_atom, nl->d_atom_shift, d_atom_local, nl->d_cl_sys, nl->d_sys, nl->d_counters, nl->d_cl_u,
        nl->d_cl_q, nl->d_cl_c, nl->d_slot_x0, nl->d_slot_gid, nl->d_slot_d0, nl->d_slot_ex, ex_start, ex_list, ex_num,
        ccap, nl->d_need, nl->d_ncl, nl->d_tcount, nl->d_slot_count, nl->d_pcount);
    SPGNB_CHECK_LAUNCH("k_cluster_props");
    // one resident wave (five blocks per SM)
    const int search_blocks = std::max(1, std::min((ccap + kSearchWarps - 1) / kSearchWarps, sms * 5));
    k_search<<<search_blocks, kSearchWarps * 32, 0, s>>>(
        nl->d_sys, ccap, nl->table_cap, nl->d_need, nl->d_ncl, nl->d_run_start, nl->d_runs, nl->d_cell_cl,
        nl->d_cl_cell, nl->d_cl_sys, nl->d_cl_u, nl->d_cl_q, nl->d_cl_c, nl->d_slot_x0, nl->d_slot_d0, nl->d_slot_ex,
        ex_start, ex_list, ex_num, nl->d_tcount, nl->d_tab, nl->d_tmask, nl->d_slot_count, nl->d_counters,
        nl->d_counters + kCntNeed, 1, nl->d_slot_atom, nl->two_sided_atoms);
    SPGNB_CHECK_LAUNCH("k_search");
    nl->sym_built = false;
    nl->two_sided_built = nl->two_sided_atoms;
    nl->rev_built = false;
    nl->ex_start_last = ex_start;
    nl->ex_list_last = ex_list;
    nl->ex_num_last = ex_num;
    if (nl->opt.export_atom_groups)
    {
        int st = build_rev(nl, s, nl->d_counters + kCntNeed);
        if (st) return st;
        k_export_zero<<<(n + 255) / 256, 256, 0, s>>>(n, nl->d_nl, nl->d_counters);
        SPGNB_CHECK_LAUNCH("k_export_zero");
        k_export_lists<true><<<std::max(1, std::min((ccap + 3) / 4, sms * 16)), 128, 0, s>>>(
            ccap, nl->table_cap, nl->d_tcount, nl->d_tab, nl->d_tmask, nl->d_slot_atom, nl->d_slot_x0, nl->d_slot_gid,
            nullptr,
            Cell{}, Cell{}, -1.0f, nl->d_nl, nl->opt.max_neighbor_numbers, nl->d_counters + kCntOverflow, kOvfList,
            nl->d_counters + kCntNeed, nl->d_rev, nl->d_rev_count);
        SPGNB_CHECK_LAUNCH("k_export_lists");
    }
    const int fin = std::max(nl->G, nl->S);
    k_finish<<<(fin + 255) / 256, 256, 0, s>>>(nl->G, nl->S, nl->d_cell_sys, nl->d_need, nl->d_prune,
                                                  nl->d_cell_count, nl->d_cell_cursor, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_finish");
    nl->built = true;
    nl->local_atoms = n;
    nl->host_builds++;
    return SPGNB_OK;
}

// Makes the pruned lists cover pairs within rc (a force module whose cutoff
// exceeds the list's): the radius grows and a pruning is queued.
int nl_set_prune_rc(spgnb_nl* nl, float rc, cudaStream_t s)
{
    if (!(rc > nl->prune_rc)) return SPGNB_OK;
    nl->prune_rc = rc;
    for (int k = 0; k < nl->S; k++)
        if (nl->live[k]) nl->h_desc[k].prune_r2 = prune_r2_of(rc, nl->opt.prune_buffer);
    SPGNB_CUDA(cudaMemcpyAsync(nl->d_sys, nl->h_desc.data(), sizeof(SysDesc) * nl->S, cudaMemcpyHostToDevice, s));
    int st = nl_prune_all(nl, s);
    if (st) return st;
    SPGNB_CUDA(cudaStreamSynchronize(s));
    return SPGNB_OK;
}

// Regrows what overflowed (1.1x, as neighbor_list.cpp:896-941 does; the
// cluster tables 1.3x) and clears the flags; the caller forces the next build.
int nl_regrow(spgnb_nl* nl, int flags)
{
    int st;
    if (flags & kOvfGrid) nl->opt.max_atom_in_grid_numbers = (int)(nl->opt.max_atom_in_grid_numbers * 1.1) + 1;
    if (flags & kOvfList)
    {
        nl->opt.max_neighbor_numbers = (int)(nl->opt.max_neighbor_numbers * 1.1) + 1;
        dfree(nl->d_nl);
        dfree(nl->d_temp);
        if ((st = dalloc(&nl->d_nl, nl->n_cap))) return st;
        if ((st = dalloc(&nl->d_temp, (size_t)nl->n_cap * nl->opt.max_neighbor_numbers))) return st;
        k_init_atom_groups<<<(nl->n_cap + 255) / 256, 256, 0, stream()>>>(nl->n_cap, nl->d_nl, nl->d_temp,
                                                                         nl->opt.max_neighbor_numbers);
        SPGNB_CHECK_LAUNCH("k_init_atom_groups");
    }
    if (flags & kOvfPairs)
    {
        nl->table_cap = (int)(nl->table_cap * 1.3) + 8;
        if ((st = alloc_tables(nl))) return st;
    }
    if (flags & kOvfWords)
    {
        nl->list_cap = (((int)(nl->list_cap * 1.3)) + 31) & ~31;
        if ((st = alloc_words(nl))) return st;
    }
    SPGNB_CUDA(cudaMemsetAsync(nl->d_counters + kCntOverflow, 0, sizeof(int), stream()));
    nl->built = false;
    return SPGNB_OK;
}

}  // namespace spgnb

using namespace spgnb;

extern "C" {

void spgnb_nl_default_options(spgnb_nl_options* o)
{
    if (!o) return;
    o->max_neighbor_numbers = 1200;
    o->max_atom_in_grid_numbers = 150;
    o->max_ghost_in_grid_numbers = 150;
    o->refresh_interval = 0;
    o->skin_permit = 0.5f;
    o->check_overflow_interval = 150;
    o->throw_error_when_overflow = 0;
    o->export_atom_groups = 1;
    o->max_entries_per_cluster = 0;
    o->prune_buffer = 1.0f;
}

int spgnb_nl_create(int atom_numbers, float cutoff, float skin, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                    const spgnb_nl_options* opt, spgnb_nl** out)
{
    if (!out) return fail(SPGNB_E_ARG, "spgnb_nl_create: out is NULL");
    *out = nullptr;
    if (atom_numbers <= 0) return fail(SPGNB_E_ARG, "spgnb_nl_create: atom_numbers must be positive");
    if (!(cutoff > 0.0f) || !(skin >= 0.0f)) return fail(SPGNB_E_ARG, "spgnb_nl_create: bad cutoff/skin");
    if (!(cell.a11 > 0.0f && cell.a22 > 0.0f && cell.a33 > 0.0f))
        return fail(SPGNB_E_ARG, "spgnb_nl_create: cell diagonal must be positive");
    return nl_create_multi(1, &atom_numbers, &cell, &rcell, &cutoff, &skin, opt, out);
}

int spgnb_nl_update(spgnb_nl* nl, const int* d_atom_local, int local_atom_numbers, int ghost_numbers,
                    const spgnb_vector* d_crd, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, int step, int update,
                    const int* d_excluded_list_start, const int* d_excluded_list, const int* d_excluded_numbers)
{
    if (!nl) return fail(SPGNB_E_ARG, "spgnb_nl_update: nl is NULL");
    if (local_atom_numbers <= 0 && ghost_numbers <= 0) return SPGNB_OK;
    if (nl->S != 1) return fail(SPGNB_E_STATE, "spgnb_nl_update: the list holds several systems");
    if (ghost_numbers != 0)
        return fail(SPGNB_E_UNSUPPORTED, "spgnb_nl_update: ghost atoms (multi-rank domain decomposition) are not "
                                         "supported; run one rank per system");
    if (local_atom_numbers > nl->n_cap)
        return fail(SPGNB_E_ARG, "spgnb_nl_update: %d local atoms exceed the %d the list was created for",
                    local_atom_numbers, nl->n_cap);
    if (!d_atom_local || !d_crd || !d_excluded_list_start || !d_excluded_list || !d_excluded_numbers)
        return fail(SPGNB_E_ARG, "spgnb_nl_update: NULL device pointer");
    cudaStream_t s = stream();
    bool box_changed = false;
    if (memcmp(&cell, &nl->cell, sizeof(cell)) != 0)
    {
        // The reference re-initialises on a large box change (main.cpp:864-939);
        // here the grid follows the new box when its shape allows, and the
        // list is rebuilt (the stored centre differences belong to the old box).
        int dims[3];
        float gl;
        grid_dims(cell, nl->cutoff, nl->skin, dims, &gl);
        if (dims[0] != nl->dims[0] || dims[1] != nl->dims[1] || dims[2] != nl->dims[2])
            return fail(SPGNB_E_STATE, "spgnb_nl_update: the box changed the grid; recreate the list");
        SysHost& sh = nl->sys[0];
        sh.cell = cell;
        sh.rcell = rcell;
        sh.gl = gl;
        sh.cs2 = gl * gl * 4.0f;
        sh.triclinic = cell.a21 != 0.0f || cell.a31 != 0.0f || cell.a32 != 0.0f;
        nl->cell = cell;
        nl->rcell = rcell;
        nl->grid_length = gl;
        nl->cs2 = sh.cs2;
        nl->triclinic = sh.triclinic;
        nl->h_desc[0] = make_desc(sh, nl->opt.skin_permit);
        nl->h_desc[0].prune_r2 = prune_r2_of(nl->prune_rc, nl->opt.prune_buffer);
        SPGNB_CUDA(cudaMemcpyAsync(nl->d_sys, nl->h_desc.data(), sizeof(SysDesc), cudaMemcpyHostToDevice, s));
        box_changed = true;
    }
    const bool host_knows = update == SPGNB_FORCED_UPDATE || !nl->built || nl->opt.refresh_interval > 0 ||
                            local_atom_numbers != nl->local_atoms || box_changed;
    if (host_knows)
    {
        const bool rebuild = update == SPGNB_FORCED_UPDATE || !nl->built || local_atom_numbers != nl->local_atoms ||
                             box_changed || ((step + 1) % nl->opt.refresh_interval == 0);
        if (!rebuild) return SPGNB_OK;
    }
    return nl_queue_build(nl, local_atom_numbers, (const float3*)d_crd, d_atom_local, d_excluded_list_start,
                          d_excluded_list, d_excluded_numbers, host_knows ? kBuildForced : kBuildSkin, s, nullptr,
                          0);
}

int spgnb_nl_get_stats(spgnb_nl* nl, spgnb_nl_stats* out)
{
    if (!nl || !out) return fail(SPGNB_E_ARG, "spgnb_nl_get_stats: NULL argument");
    int h[kCntSize];
    SPGNB_CUDA(cudaMemcpyAsync(h, nl->d_counters, sizeof(h), cudaMemcpyDeviceToHost, stream()));
    SPGNB_CUDA(cudaStreamSynchronize(stream()));
    out->atom_numbers = nl->local_atoms;
    out->grid_numbers = nl->G;
    out->grid_dims[0] = nl->dims[0];
    out->grid_dims[1] = nl->dims[1];
    out->grid_dims[2] = nl->dims[2];
    std::vector<int> ncl(nl->S);
    SPGNB_CUDA(cudaMemcpy(ncl.data(), nl->d_ncl, sizeof(int) * nl->S, cudaMemcpyDeviceToHost));
    long long nclt = 0;
    for (int v : ncl) nclt += v;
    out->clusters = (int)nclt;
    long long e;
    memcpy(&e, &h[kCntEntries], sizeof(e));
    out->entries = e;
    out->work_items = (int)nclt;
    out->builds = h[kCntBuilds];
    out->overflow = h[kCntOverflow];
    memcpy(&out->full_list_words, &h[kCntWords], sizeof(long long));
    out->prunes = h[kCntPrunes];
    memcpy(&out->pruned_list_words, &h[kCntPWordsLast], sizeof(long long));
    out->device_bytes = (long long)nl_device_bytes(nl);
    return SPGNB_OK;
}

int spgnb_nl_check_overflow(spgnb_nl* nl, int steps, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                            int* reinitialized)
{
    (void)cell;
    (void)rcell;
    if (!nl) return fail(SPGNB_E_ARG, "spgnb_nl_check_overflow: nl is NULL");
    if (reinitialized) *reinitialized = 0;
    if (nl->opt.check_overflow_interval > 0 && (steps + 1) % nl->opt.check_overflow_interval != 0)
        return SPGNB_OK;
    int flags = 0;
    SPGNB_CUDA(cudaMemcpyAsync(&flags, nl->d_counters + kCntOverflow, sizeof(int), cudaMemcpyDeviceToHost,
                               stream()));
    SPGNB_CUDA(cudaStreamSynchronize(stream()));
    if (!flags) return SPGNB_OK;
    if (nl->opt.throw_error_when_overflow)
        return fail(SPGNB_E_OVERFLOW, "NEIGHBOR_LIST::Check_Overflow: overflow occurred in neighbor searching "
                                      "(flags 0x%x)",
                    flags);
    if (flags & kOvfCellHard)
        return fail(SPGNB_E_UNSUPPORTED, "NEIGHBOR_LIST: a grid cell holds more than %d atoms", kMaxCellAtoms);
    int st = nl_regrow(nl, flags);
    if (st) return st;
    if (reinitialized) *reinitialized = 1;
    return SPGNB_OK;
}

int spgnb_nl_atom_groups(spgnb_nl* nl, spgnb_atom_group** d_nl, int** d_temp)
{
    if (!nl) return fail(SPGNB_E_ARG, "spgnb_nl_atom_groups: nl is NULL");
    if (!nl->opt.export_atom_groups)
        return fail(SPGNB_E_STATE, "spgnb_nl_atom_groups: the list was created with export_atom_groups = 0");
    if (d_nl) *d_nl = nl->d_nl;
    if (d_temp) *d_temp = nl->d_temp;
    return SPGNB_OK;
}

int spgnb_nl_copy_atom_groups(spgnb_nl* nl, int* h_counts, int* h_lists, long long capacity, long long* total)
{
    if (!nl || !h_counts) return fail(SPGNB_E_ARG, "spgnb_nl_copy_atom_groups: NULL argument");
    if (!nl->opt.export_atom_groups || !nl->d_nl)
        return fail(SPGNB_E_STATE, "spgnb_nl_copy_atom_groups: the list was created with export_atom_groups = 0");
    const int n = nl->local_atoms;
    std::vector<spgnb_atom_group> h(n);
    SPGNB_CUDA(cudaMemcpyAsync(h.data(), nl->d_nl, sizeof(spgnb_atom_group) * n, cudaMemcpyDeviceToHost, stream()));
    SPGNB_CUDA(cudaStreamSynchronize(stream()));
    long long t = 0;
    for (int i = 0; i < n; i++)
    {
        h_counts[i] = h[i].atom_numbers;
        t += h[i].atom_numbers;
    }
    if (total) *total = t;
    if (h_lists && capacity >= t)
    {
        const int m = nl->opt.max_neighbor_numbers;
        std::vector<int> slab((size_t)n * m);
        SPGNB_CUDA(cudaMemcpy(slab.data(), nl->d_temp, sizeof(int) * slab.size(), cudaMemcpyDeviceToHost));
        long long off = 0;
        for (int i = 0; i < n; i++)
        {
            const int c = std::min(h[i].atom_numbers, m);
            memcpy(h_lists + off, slab.data() + (size_t)i * m, sizeof(int) * c);
            off += h[i].atom_numbers;
        }
    }
    return SPGNB_OK;
}

}  // extern "C"

namespace spgnb
{

// Re-runs the search of the last build (same clusters and build
// coordinates) with two-sided tables everywhere (flags null, half 0) or for
// the flagged atoms' clusters.
int research_last_build(const spgnb_nl* nl, cudaStream_t s, int half, const unsigned char* flags)
{
    k_sym_begin<<<1, 1, 0, s>>>(nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_sym_begin");
    const int ccap = nl->clusters_cap;
    const int search_blocks = std::max(1, std::min((ccap + kSearchWarps - 1) / kSearchWarps, num_sms() * 5));
    // every live system, whatever the last build flagged: a system's tables
    // are those of its own last build either way
    k_search<<<search_blocks, kSearchWarps * 32, 0, s>>>(
        nl->d_sys, ccap, nl->table_cap, nl->d_live, nl->d_ncl, nl->d_run_start, nl->d_runs, nl->d_cell_cl,
        nl->d_cl_cell, nl->d_cl_sys, nl->d_cl_u, nl->d_cl_q, nl->d_cl_c, nl->d_slot_x0, nl->d_slot_d0, nl->d_slot_ex,
        nl->ex_start_last, nl->ex_list_last, nl->ex_num_last, nl->d_tcount, nl->d_tab, nl->d_tmask, nl->d_slot_count,
        nl->d_counters, nullptr, half, nl->d_slot_atom, flags);
    SPGNB_CHECK_LAUNCH("k_search");
    nl->rev_built = false;  // the tables' elements moved
    return SPGNB_OK;
}

int nl_symmetrize(const spgnb_nl* nl, cudaStream_t s)
{
    if (!nl->built || nl->sym_built) return SPGNB_OK;
    const int st = research_last_build(nl, s, 0, nullptr);
    if (st) return st;
    nl->sym_built = true;
    nl->two_sided_built = nullptr;
    return SPGNB_OK;
}

int nl_two_sided_atoms(const spgnb_nl* nl, const unsigned char* d_flags, cudaStream_t s)
{
    nl->two_sided_atoms = d_flags;
    if (!nl->built || nl->sym_built || nl->two_sided_built == d_flags) return SPGNB_OK;
    const int st = research_last_build(nl, s, 1, d_flags);
    if (st) return st;
    nl->two_sided_built = d_flags;
    return SPGNB_OK;
}

}  // namespace spgnb

extern "C" {

int spgnb_nl_build_full(spgnb_nl* nl, int local_atom_numbers, const spgnb_vector* d_crd, spgnb_ltmatrix3 cell,
                        spgnb_ltmatrix3 rcell, float cutoff, spgnb_atom_group* d_full_nl, int max_neighbor_numbers,
                        int* d_overflow)
{
    if (!nl || !d_full_nl) return fail(SPGNB_E_ARG, "spgnb_nl_build_full: NULL argument");
    if (!nl->built) return fail(SPGNB_E_STATE, "spgnb_nl_build_full: the list was never built");
    if (local_atom_numbers != nl->local_atoms)
        return fail(SPGNB_E_ARG, "spgnb_nl_build_full: %d local atoms, the list was built for %d", local_atom_numbers,
                    nl->local_atoms);
    if (max_neighbor_numbers <= 0) return fail(SPGNB_E_ARG, "spgnb_nl_build_full: max_neighbor_numbers must be positive");
    if (cutoff > 0.0f && !d_crd) return fail(SPGNB_E_ARG, "spgnb_nl_build_full: a cutoff needs coordinates");
    if (!d_overflow) return fail(SPGNB_E_ARG, "spgnb_nl_build_full: NULL overflow flag");
    cudaStream_t s = stream();
    int st;
    // each atom's lower partners through the reverse index of the tables
    if (!nl->d_rev && (st = alloc_rev(nl))) return st;
    if (!nl->rev_built && (st = build_rev(nl, s, nullptr))) return st;
    const int n = local_atom_numbers;
    // atoms in no cluster with a table (none, normally) keep a zero count
    k_zero_groups<<<(n + 255) / 256, 256, 0, s>>>(n, d_full_nl);
    SPGNB_CHECK_LAUNCH("k_zero_groups");
    const int ccap = nl->clusters_cap;
    k_export_lists<false><<<std::max(1, std::min((ccap + 3) / 4, num_sms() * 16)), 128, 0, s>>>(
        ccap, nl->table_cap, nl->d_tcount, nl->d_tab, nl->d_tmask, nl->d_slot_atom, nl->d_slot_x0, nl->d_slot_gid,
        (const float3*)d_crd, make_cell(cell), make_cell(rcell), cutoff > 0.0f ? cutoff * cutoff : -1.0f, d_full_nl,
        max_neighbor_numbers, d_overflow, 1, nullptr, nl->d_rev, nl->d_rev_count);
    SPGNB_CHECK_LAUNCH("k_export_lists");
    return SPGNB_OK;
}

int spgnb_nl_destroy(spgnb_nl* nl)
{
    if (!nl) return SPGNB_OK;
    free_nl(nl);
    delete nl;
    return SPGNB_OK;
}

}  // extern "C"
