// Neighbour-list rebuild: NEIGHBOR_LIST::Initial / Update / Check_Overflow /
// Clear of SPONGE/neighbor_list/neighbor_list.cpp, rebuilt around 8-atom
// clusters.
//
// The listed set is the reference's, pair for pair: atoms are binned into the
// reference grid (cells of (rc+skin)/2, same wrap and clamp, :206-275), pairs
// are considered between a cell and its stencil (:5-49), and a pair (i, j)
// with atom_local[i] < atom_local[j] is listed when the FP32 expression
// Get_Periodic_Displacement(crd_i, crd_j)^2 (vector.hpp:322-327) is below
// 4*grid_length^2 (:367-372, :705) and j is not in i's exclusion list
// (:594-665).  Instead of per-atom arrays the result is stored as
// (i-cluster, j-cluster, 64-bit pair mask) entries that the pair kernel
// consumes; spgnb_nl_atom_groups exports the reference layout.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace spgnb
{
namespace
{

struct Grid
{
    int Nx, Ny, Nz, G;
    float gl, cs2;
    Cell cell, rcell;
};

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
// the dot product produces (see orc_pair_dr2, mode 1, in the oracle).
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

// Check_Refresh (neighbor_list.cpp:166-180): any atom moved more than
// skin*skin_permit since the last build.
__global__ void k_check_refresh(int n_slots, const int* __restrict__ slot_atom,
                                const float3* __restrict__ crd, const float4* __restrict__ x0, Cell cell,
                                Cell rcell, float permit2, int* counters)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    int total = counters[kCntClusters] * kClusterSize;
    bool move = false;
    if (s < n_slots && s < total)
    {
        int a = slot_atom[s];
        if (a >= 0)
        {
            float3 c = crd[a];
            float4 o = x0[s];
            float dx = c.x - o.x, dy = c.y - o.y, dz = c.z - o.z;
            float sx = floorf(dx * rcell.a11 + dy * rcell.a21 + dz * rcell.a31 + 0.5f);
            float sy = floorf(dy * rcell.a22 + dz * rcell.a32 + 0.5f);
            float sz = floorf(dz * rcell.a33 + 0.5f);
            dx -= sx * cell.a11 + sy * cell.a21 + sz * cell.a31;
            dy -= sy * cell.a22 + sz * cell.a32;
            dz -= sz * cell.a33;
            move = dx * dx + dy * dy + dz * dz > permit2;
        }
    }
    if (__any_sync(0xffffffffu, move) && (threadIdx.x & 31) == 0) atomicExch(&counters[kCntNeed], 1);
}

// Put_Atom_In_Grids (neighbor_list.cpp:206-275): brick wrap, cell index
// nx*Ny*Nz + ny*Nz + nz with clamping, per-cell count.
__global__ void k_bin(int n, const float3* __restrict__ crd, Grid g, int* __restrict__ atom_cell,
                      int* __restrict__ atom_shift, float4* __restrict__ wrapped, int* __restrict__ cell_count,
                      const int* __restrict__ counters)
{
    if (counters[kCntNeed] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 c = crd[i];
    float x = c.x, y = c.y, z = c.z;
    float k3 = floorf(__fdiv_rn(z, g.cell.a33));
    z = __fsub_rn(z, __fmul_rn(k3, g.cell.a33));
    y = __fsub_rn(y, __fmul_rn(k3, g.cell.a32));
    float k2 = floorf(__fdiv_rn(y, g.cell.a22));
    y = __fsub_rn(y, __fmul_rn(k2, g.cell.a22));
    x = __fsub_rn(x, __fadd_rn(__fmul_rn(k3, g.cell.a31), __fmul_rn(k2, g.cell.a21)));
    float k1 = floorf(__fdiv_rn(x, g.cell.a11));
    x = __fsub_rn(x, __fmul_rn(k1, g.cell.a11));
    int nx = (int)__fdiv_rn(x, g.gl);
    int ny = (int)__fdiv_rn(y, g.gl);
    int nz = (int)__fdiv_rn(z, g.gl);
    nx = nx < 0 ? 0 : (nx < g.Nx ? nx : g.Nx - 1);
    ny = ny < 0 ? 0 : (ny < g.Ny ? ny : g.Ny - 1);
    nz = nz < 0 ? 0 : (nz < g.Nz ? nz : g.Nz - 1);
    int cid = nx * g.Ny * g.Nz + ny * g.Nz + nz;
    atom_cell[i] = cid;
    atom_shift[i] = pack_shift((int)k1, (int)k2, (int)k3);
    wrapped[i] = make_float4(x, y, z, 0.0f);
    atomicAdd(&cell_count[cid], 1);
}

// Cluster counts per cell (ceil(count/8)) and their exclusive scan; one block.
__global__ void k_scan_cells(int G, const int* __restrict__ cell_count, int* __restrict__ cell_cl_start,
                             int max_atom_in_grid, int clusters_cap, int* counters)
{
    if (counters[kCntNeed] == 0) return;
    __shared__ int warp_sums[32];
    __shared__ int warp_max[32];
    const int T = blockDim.x;
    const int per = (G + T - 1) / T;
    const int lo = threadIdx.x * per;
    const int hi = min(G, lo + per);
    int sum = 0, mx = 0;
    for (int c = lo; c < hi; c++)
    {
        int cnt = cell_count[c];
        sum += (cnt + kClusterSize - 1) / kClusterSize;
        mx = max(mx, cnt);
    }
    // block exclusive scan of sum
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int v = sum;
    for (int o = 1; o < 32; o <<= 1)
    {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    int m = mx;
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 31) warp_sums[warp] = v;
    if (lane == 0) warp_max[warp] = m;
    __syncthreads();
    if (warp == 0)
    {
        int nw = T >> 5;
        int w = lane < nw ? warp_sums[lane] : 0;
        int wm = lane < nw ? warp_max[lane] : 0;
        for (int o = 1; o < 32; o <<= 1)
        {
            int t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        for (int o = 16; o > 0; o >>= 1) wm = max(wm, __shfl_xor_sync(0xffffffffu, wm, o));
        if (lane < nw) warp_sums[lane] = w;
        if (lane == 0) warp_max[0] = wm;
    }
    __syncthreads();
    int excl = v - sum + (warp > 0 ? warp_sums[warp - 1] : 0);
    for (int c = lo; c < hi; c++)
    {
        cell_cl_start[c] = excl;
        excl += (cell_count[c] + kClusterSize - 1) / kClusterSize;
    }
    if (threadIdx.x == T - 1)
    {
        int total = warp_sums[(T >> 5) - 1];
        cell_cl_start[G] = total;
        counters[kCntClusters] = min(total, clusters_cap);
        counters[kCntMaxCell] = warp_max[0];
        int flags = 0;
        if (warp_max[0] > max_atom_in_grid) flags |= kOvfGrid;
        if (total > clusters_cap) flags |= kOvfPairs;
        if (warp_max[0] > 2048) flags |= kOvfCellHard;
        if (flags) atomicOr(&counters[kCntOverflow], flags);
    }
}

__global__ void k_scatter(int n, const int* __restrict__ atom_cell, const int* __restrict__ cell_cl_start,
                          int* __restrict__ cell_cursor, int* __restrict__ tmp_atoms, int slots_cap,
                          const int* __restrict__ counters)
{
    if (counters[kCntNeed] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = atom_cell[i];
    int pos = atomicAdd(&cell_cursor[c], 1);
    int s = cell_cl_start[c] * kClusterSize + pos;
    if (s < slots_cap) tmp_atoms[s] = i;
}

__device__ __forceinline__ unsigned spread3(unsigned v)
{
    // 2-bit value -> bits 0 and 3
    return (v & 1u) | ((v & 2u) << 2);
}

// Deterministic in-cell order: by a 4x4x4 Morton sub-cell key, then by atom
// index, so clusters are spatially compact and the build reproducible.
__global__ void k_sort_cells(Grid g, const int* __restrict__ cell_count, const int* __restrict__ cell_cl_start,
                             const int* __restrict__ tmp_atoms, const float4* __restrict__ wrapped,
                             int* __restrict__ slot_atom, int* __restrict__ cl_cell, int* __restrict__ atom_slot,
                             int slots_cap, const int* __restrict__ counters)
{
    if (counters[kCntNeed] == 0) return;
    extern __shared__ unsigned long long keys[];
    for (int c = blockIdx.x; c < g.G; c += gridDim.x)
    {
        int n = min(cell_count[c], 2048);
        int cl0 = cell_cl_start[c], cl1 = cell_cl_start[c + 1];
        int base = cl0 * kClusterSize;
        int nslots = (cl1 - cl0) * kClusterSize;
        if (base + nslots > slots_cap) continue;
        int nz = c % g.Nz, ny = (c / g.Nz) % g.Ny, nx = c / (g.Ny * g.Nz);
        float inv = 4.0f / g.gl;
        for (int e = threadIdx.x; e < n; e += blockDim.x)
        {
            int a = tmp_atoms[base + e];
            float4 w = wrapped[a];
            int sx = min(3, max(0, (int)((w.x - nx * g.gl) * inv)));
            int sy = min(3, max(0, (int)((w.y - ny * g.gl) * inv)));
            int sz = min(3, max(0, (int)((w.z - nz * g.gl) * inv)));
            unsigned key = (spread3(sx) << 2) | (spread3(sy) << 1) | spread3(sz);
            keys[e] = ((unsigned long long)key << 32) | (unsigned)a;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nslots; e += blockDim.x)
        {
            if (e < n)
            {
                unsigned long long k = keys[e];
                int r = 0;
                for (int f = 0; f < n; f++) r += keys[f] < k;
                const int a = (int)(k & 0xffffffffu);
                slot_atom[base + r] = a;
                atom_slot[a] = base + r;
            }
            else
            {
                slot_atom[base + e] = -1;
            }
        }
        for (int k = cl0 + threadIdx.x; k < cl1; k += blockDim.x) cl_cell[k] = c;
        __syncthreads();
    }
}

// Per cluster: centre (double, bounding-box middle of the wrapped positions),
// radius, fractional fixed-point centre, per-slot offsets and build
// coordinates.  Eight lanes per cluster.
__global__ void k_cluster_props(const float3* __restrict__ crd, const int* __restrict__ slot_atom,
                                const int* __restrict__ atom_shift, const int* __restrict__ atom_local, Cell cell,
                                int* counters, uint4* __restrict__ cl_u, float4* __restrict__ cl_c,
                                float4* __restrict__ slot_x0, float4* __restrict__ slot_d0, int clusters_cap)
{
    if (counters[kCntNeed] == 0) return;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int k = t >> 3;
    int l8 = t & 7;
    int nc = counters[kCntClusters];
    bool live = k < nc && k < clusters_cap;
    int s = k * kClusterSize + l8;
    int a = live ? slot_atom[s] : -1;
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
    for (int d = 0; d < 3; d++) cen[d] = 0.5 * (lo[d] + hi[d]);
    // fractional centre; the double inverse of the float cell
    double c11 = cell.a11, c21 = cell.a21, c22 = cell.a22, c31 = cell.a31, c32 = cell.a32, c33 = cell.a33;
    double r33 = 1.0 / c33, r22 = 1.0 / c22, r11 = 1.0 / c11;
    double r32 = -c32 * r33 / c22;
    double r31 = (c32 * c21 * r33 - c31 * c22) / (c11 * c22 * c33);
    double r21 = -c21 * r22 / c11;
    double sfr[3] = {cen[0] * r11 + cen[1] * r21 + cen[2] * r31, cen[1] * r22 + cen[2] * r32, cen[2] * r33};
    unsigned u[3];
    double q[3];
    for (int d = 0; d < 3; d++)
    {
        double f = floor(sfr[d]);
        double frac = sfr[d] - f;
        double scaled = floor(frac * 4294967296.0);
        if (scaled >= 4294967296.0) scaled = 4294967295.0;
        u[d] = (unsigned)scaled;
        q[d] = scaled / 4294967296.0 + f;  // the quantised centre, unwrapped
    }
    double cq[3] = {q[0] * c11 + q[1] * c21 + q[2] * c31, q[1] * c22 + q[2] * c32, q[2] * c33};
    double r2 = 0;
    if (a >= 0)
    {
        double d0 = w[0] - cq[0], d1 = w[1] - cq[1], d2 = w[2] - cq[2];
        r2 = d0 * d0 + d1 * d1 + d2 * d2;
        slot_d0[s] = make_float4((float)d0, (float)d1, (float)d2, 0.0f);
        // raw build coordinates, w = the atom's global index (-1: padding)
        slot_x0[s] = make_float4(x.x, x.y, x.z, __int_as_float(atom_local[a]));
    }
    else if (live)
    {
        float p = kPadCoordinate + (float)s;
        slot_d0[s] = make_float4(p, p, p, 0.0f);
        slot_x0[s] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
    }
    for (int o = 1; o < 8; o <<= 1) r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, o));
    if (live && l8 == 0)
    {
        float rad = (float)(sqrt(r2) * (1.0 + 1e-6) + 1e-5);
        cl_u[k] = make_uint4(u[0], u[1], u[2], __float_as_uint(rad));
        cl_c[k] = make_float4((float)cq[0], (float)cq[1], (float)cq[2], rad);
    }
}

struct SearchParams
{
    Grid g;
    float list_radius;    // sqrt(cs2) with a margin, for the sphere prefilter
    float frac_norm[3];   // norms of the columns of rcell
    int triclinic;
    long long entries_cap;
    int items_cap;
    int clusters_cap;
};

__device__ __forceinline__ float3 frac_delta(uint4 ui, uint4 uj)
{
    const float s = 2.3283064365386963e-10f;  // 2^-32
    return make_float3((float)(int)(uj.x - ui.x) * s, (float)(int)(uj.y - ui.y) * s, (float)(int)(uj.z - ui.z) * s);
}

__device__ __forceinline__ float3 frac_to_cart(float3 f, const Cell& c)
{
    return make_float3(f.x * c.a11 + f.y * c.a21 + f.z * c.a31, f.y * c.a22 + f.z * c.a32, f.z * c.a33);
}

__device__ __forceinline__ bool excluded_pair(int glo, int ghi, const int* __restrict__ ex_start,
                                              const int* __restrict__ ex_list, const int* __restrict__ ex_num)
{
    int k = ex_num[glo];
    if (k <= 0) return false;
    const int* l = ex_list + ex_start[glo];
    if (ghi < l[0] || ghi > l[k - 1]) return false;
    for (int t = 0; t < k; t++)
        if (l[t] == ghi) return true;
    return false;
}

// Cluster-pair search, one warp per i-cluster.  For every stencil cell of the
// i-cluster's cell, every j-cluster (j >= i in cluster order) that survives a
// conservative sphere test gets its 64 pairs tested with the reference's
// expression; a non-zero mask becomes an entry.  Entries of one i-cluster are
// written in chunks of kChunk behind a work item.
constexpr int kSearchWarps = 4;

__global__ void __launch_bounds__(kSearchWarps * 32)
    k_search(SearchParams p, const int* __restrict__ cand_start, const int* __restrict__ cand,
             const int* __restrict__ cell_cl_start, const int* __restrict__ cl_cell, const uint4* __restrict__ cl_u,
             const float4* __restrict__ slot_x0, const int* __restrict__ ex_start, const int* __restrict__ ex_list, const int* __restrict__ ex_num,
             int4* __restrict__ ents, float4* __restrict__ ents_d, int4* __restrict__ items, int* counters)
{
    if (counters[kCntNeed] == 0) return;
    __shared__ int4 stage[kSearchWarps][kChunk];
    __shared__ float4 stage_d[kSearchWarps][kChunk];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int nc = counters[kCntClusters];
    const int total_warps = gridDim.x * kSearchWarps;
    unsigned long long* ent_counter = (unsigned long long*)&counters[kCntEntries];

    for (int ci = blockIdx.x * kSearchWarps + wib; ci < nc; ci += total_warps)
    {
        const int cellA = cl_cell[ci];
        const uint4 ui = cl_u[ci];
        const float ri = __uint_as_float(ui.w);
        // the two i-atoms this lane tests (rounds h = 0, 1)
        int ga[2];
        float3 xa[2];
        for (int h = 0; h < 2; h++)
        {
            const int a = h * 4 + (lane >> 3);
            const float4 x = slot_x0[ci * kClusterSize + a];
            ga[h] = __float_as_int(x.w);
            xa[h] = make_float3(x.x, x.y, x.z);
        }
        int staged = 0;
        auto flush = [&](int count) {
            // reserve space for `count` entries and one work item
            long long e0 = 0;
            int it = 0;
            if (lane == 0)
            {
                e0 = (long long)atomicAdd(ent_counter, (unsigned long long)count);
                it = atomicAdd(&counters[kCntItems], 1);
            }
            e0 = __shfl_sync(0xffffffffu, e0, 0);
            it = __shfl_sync(0xffffffffu, it, 0);
            const bool ok = (e0 + count <= p.entries_cap) && (it < p.items_cap);
            if (ok && lane < count)
            {
                ents[e0 + lane] = stage[wib][lane];
                ents_d[e0 + lane] = stage_d[wib][lane];
            }
            // an item slot that exists is always written, empty when its
            // entries did not fit, so readers never see a stale range
            if (lane == 0 && it < p.items_cap) items[it] = make_int4(ci, ok ? (int)e0 : 0, ok ? count : 0, 0);
            if (lane == 0 && !ok) atomicOr(&counters[kCntOverflow], kOvfPairs);
            __syncwarp();
        };

        const int k0 = cand_start[cellA], k1 = cand_start[cellA + 1];
        for (int k = k0; k < k1; k++)
        {
            const int cv = cand[k];
            const int cellB = cv & 0x0fffffff;
            const bool fwd = (cv >> 28) & 1;  // cellB in stencil(cellA)
            const bool rev = (cv >> 29) & 1;  // cellA in stencil(cellB)
            int b0 = max(cell_cl_start[cellB], ci);
            const int b1 = min(cell_cl_start[cellB + 1], nc);
            for (; b0 < b1; b0 += 32)
            {
                int cj = b0 + lane;
                bool ok = false;
                if (cj < b1)
                {
                    uint4 uj = cl_u[cj];
                    float rsum = ri + __uint_as_float(uj.w) + p.list_radius;
                    float3 f = frac_delta(ui, uj);
                    if (!p.triclinic)
                    {
                        float3 d = frac_to_cart(f, p.g.cell);
                        ok = d.x * d.x + d.y * d.y + d.z * d.z < rsum * rsum;
                    }
                    else
                    {
                        for (int im = 0; im < 27 && !ok; im++)
                        {
                            float3 fi = make_float3(f.x + (float)(im / 9 - 1), f.y + (float)((im / 3) % 3 - 1),
                                                    f.z + (float)(im % 3 - 1));
                            float3 d = frac_to_cart(fi, p.g.cell);
                            ok = d.x * d.x + d.y * d.y + d.z * d.z < rsum * rsum;
                        }
                    }
                }
                unsigned surv = __ballot_sync(0xffffffffu, ok);
                while (surv)
                {
                    const int src = __ffs(surv) - 1;
                    surv &= surv - 1;
                    const int cjs = b0 + src;
                    const int b = lane & 7;
                    const float4 xj = slot_x0[cjs * kClusterSize + b];
                    const int gb = __float_as_int(xj.w);
                    const float3 xb = make_float3(xj.x, xj.y, xj.z);
                    unsigned bits[2];
                    for (int h = 0; h < 2; h++)
                    {
                        const int a = h * 4 + (lane >> 3);
                        bool in = ga[h] >= 0 && gb >= 0 && (cjs != ci || b > a);
                        if (in)
                        {
                            const bool a_lo = ga[h] < gb;
                            in = a_lo ? fwd : rev;
                            if (in)
                            {
                                float d2 = a_lo ? ref_pair_dr2(xa[h], xb, p.g.cell, p.g.rcell)
                                                : ref_pair_dr2(xb, xa[h], p.g.cell, p.g.rcell);
                                in = d2 < p.g.cs2;
                                if (in)
                                    in = !(a_lo ? excluded_pair(ga[h], gb, ex_start, ex_list, ex_num)
                                                : excluded_pair(gb, ga[h], ex_start, ex_list, ex_num));
                            }
                        }
                        bits[h] = __ballot_sync(0xffffffffu, in);
                    }
                    if (bits[0] | bits[1])
                    {
                        // one image per entry is enough when every pair of the two
                        // spheres stays inside half a box in fractional terms
                        const uint4 uj = cl_u[cjs];
                        const float3 f = frac_delta(ui, uj);
                        const float rr = ri + __uint_as_float(uj.w);
                        bool safe = fabsf(f.x) + rr * p.frac_norm[0] < 0.49f &&
                                    fabsf(f.y) + rr * p.frac_norm[1] < 0.49f &&
                                    fabsf(f.z) + rr * p.frac_norm[2] < 0.49f;
                        if (lane == 0)
                        {
                            stage[wib][staged] =
                                make_int4(cjs, safe ? 0 : kEntPairImage, (int)bits[0], (int)bits[1]);
                            // centre difference from the quantised centres, in double
                            const double q = 2.3283064365386963e-10;
                            const double fx = (double)(int)(uj.x - ui.x) * q, fy = (double)(int)(uj.y - ui.y) * q,
                                         fz = (double)(int)(uj.z - ui.z) * q;
                            const Cell& c = p.g.cell;
                            stage_d[wib][staged] = make_float4(
                                (float)(fx * (double)c.a11 + fy * (double)c.a21 + fz * (double)c.a31),
                                (float)(fy * (double)c.a22 + fz * (double)c.a32), (float)(fz * (double)c.a33), 0.0f);
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
    }
}

// Reference-layout export: zero the counts, then scatter every listed pair
// to its owner (the lower atom_local index) as the reference stores it.
__global__ void k_export_zero(int n, spgnb_atom_group* __restrict__ nl, const int* __restrict__ counters)
{
    if (counters[kCntNeed] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        nl[i].atom_numbers = 0;
        nl[i].ghost_numbers = 0;
    }
}

__global__ void k_export(const int4* __restrict__ items, const int4* __restrict__ ents,
                         const int* __restrict__ slot_atom, const int* __restrict__ atom_local,
                         spgnb_atom_group* __restrict__ nl, int* __restrict__ temp, int max_nb, int* counters,
                         int items_cap)
{
    if (counters[kCntNeed] == 0) return;
    const int lane = threadIdx.x & 31;
    const int nitems = min(counters[kCntItems], items_cap);
    const int total_warps = gridDim.x * (blockDim.x >> 5);
    for (int it = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < nitems; it += total_warps)
    {
        int4 item = items[it];
        const int ci = item.x;
        for (int e = item.y; e < item.y + item.z; e++)
        {
            int4 en = ents[e];
            for (int h = 0; h < 2; h++)
            {
                unsigned m = (unsigned)(h ? en.w : en.z);
                if (!((m >> lane) & 1u)) continue;
                int a = h * 4 + (lane >> 3), b = lane & 7;
                int ia = slot_atom[ci * kClusterSize + a];
                int jb = slot_atom[en.x * kClusterSize + b];
                int owner = atom_local[ia] < atom_local[jb] ? ia : jb;
                int other = owner == ia ? jb : ia;
                int slot = atomicAdd(&nl[owner].atom_numbers, 1);
                if (slot < max_nb)
                    temp[(size_t)owner * max_nb + slot] = other;
                else
                    atomicOr(&counters[kCntOverflow], kOvfList);
            }
        }
    }
}

__global__ void k_finish(int G, int* __restrict__ cell_count, int* __restrict__ cell_cursor, int* counters)
{
    if (counters[kCntNeed] == 0) return;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < G)
    {
        cell_count[c] = 0;
        cell_cursor[c] = 0;
    }
    if (c == 0) counters[kCntBuilds] += 1;
}

__global__ void k_set_need(int* counters) { counters[kCntNeed] = 1; }

__global__ void k_reset_list_counters(int* counters)
{
    if (counters[kCntNeed] == 0) return;
    counters[kCntItems] = 0;
    counters[kCntEntries] = 0;
    counters[kCntEntries + 1] = 0;
}

__global__ void k_init_atom_groups(int n, spgnb_atom_group* nl, int* temp, int max_nb)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        nl[i].atom_numbers = 0;
        nl[i].ghost_numbers = 0;
        nl[i].atom_serial = temp + (size_t)i * max_nb;
    }
}

// --------------------------------------------------------------- host side

int grid_dims(const spgnb_ltmatrix3& cell, float cutoff, float skin, int dims[3], float* gl)
{
    float g = 0.5f * (cutoff + skin);
    dims[0] = (int)floorf(cell.a11 / g);
    dims[1] = (int)floorf(cell.a22 / g);
    dims[2] = (int)floorf(cell.a33 / g);
    *gl = g;
    return SPGNB_OK;
}

// The reference's stencil rule (Find_Neighor_Grids_Device), evaluated per
// cell by enumerating the offsets instead of the O(G^2) scan; forward and
// reverse stencils merged with flags (bit 28: B in stencil(A), bit 29: A in
// stencil(B)).
int build_candidates(spgnb_nl* nl, std::vector<int>& start, std::vector<int>& cand)
{
    const int Nx = nl->dims[0], Ny = nl->dims[1], Nz = nl->dims[2];
    const int G = nl->G;
    const float gl = nl->grid_length;
    const spgnb_ltmatrix3& c = nl->cell;
    int dxy = (int)(c.a21 / gl), dxz = (int)(c.a31 / gl), dyz = (int)(c.a32 / gl);
    std::vector<std::vector<int>> fwd(G);
    std::vector<int> mark(G, -1);
    for (int g = 0; g < G; g++)
    {
        int gx = g / (Ny * Nz), gy = (g / Nz) % Ny, gz = g % Nz;
        for (int k = 0; k < 27; k++)
        {
            int dx = k / 9 - 1, dy = (k % 9) / 3 - 1, dz = k % 3 - 1;
            int cx = (dy * c.a21 + dz * c.a31 == 0) ? -2 : -3;
            int cy = (dz * c.a32 == 0) ? -2 : -3;
            int sx = gx + dx * Nx + dy * dxy + dz * dxz, sy = gy + dy * Ny + dz * dyz, sz = gz + dz * Nz;
            for (int tx = cx; tx <= 2; tx++)
                for (int ty = cy; ty <= 2; ty++)
                    for (int tz = -2; tz <= 2; tz++)
                    {
                        int jx = sx - tx, jy = sy - ty, jz = sz - tz;
                        if (jx < 0 || jx >= Nx || jy < 0 || jy >= Ny || jz < 0 || jz >= Nz) continue;
                        int j = (jx * Ny + jy) * Nz + jz;
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
    start.assign(G + 1, 0);
    cand.clear();
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
        for (int j : touched)
        {
            cand.push_back(j | ((flag[j] & 1) << 28) | ((flag[j] & 2) << 28));
            flag[j] = 0;
        }
        start[g + 1] = (int)cand.size();
    }
    return SPGNB_OK;
}

void free_nl(spgnb_nl* nl)
{
    dfree(nl->d_cand_start);
    dfree(nl->d_cand);
    dfree(nl->d_cell_count);
    dfree(nl->d_cell_cursor);
    dfree(nl->d_cell_cl_start);
    dfree(nl->d_atom_cell);
    dfree(nl->d_atom_shift);
    dfree(nl->d_tmp_atoms);
    dfree(nl->d_slot_atom);
    dfree(nl->d_slot_x0);
    dfree(nl->d_slot_d0);
    dfree(nl->d_cl_cell);
    dfree(nl->d_cl_u);
    dfree(nl->d_cl_c);
    dfree(nl->d_ents);
    dfree(nl->d_ents_d);
    dfree(nl->d_items);
    dfree(nl->d_counters);
    dfree(nl->d_atom_slot);
    dfree(nl->d_nl);
    dfree(nl->d_temp);
    dfree(nl->d_wrapped);
}

int alloc_pair_list(spgnb_nl* nl)
{
    int st;
    dfree(nl->d_ents);
    dfree(nl->d_ents_d);
    dfree(nl->d_items);
    nl->entries_cap = (long long)nl->clusters_cap * nl->entries_per_cluster;
    nl->items_cap = (int)std::min<long long>(nl->entries_cap / kChunk + nl->clusters_cap + 1024, 0x7fffffffLL);
    if ((st = dalloc(&nl->d_ents, (size_t)nl->entries_cap))) return st;
    if ((st = dalloc(&nl->d_ents_d, (size_t)nl->entries_cap))) return st;
    if ((st = dalloc(&nl->d_items, (size_t)nl->items_cap))) return st;
    return SPGNB_OK;
}

int alloc_nl(spgnb_nl* nl)
{
    int st;
    const int n = nl->n_cap;
    const int G = nl->G;
    nl->clusters_cap = n / kClusterSize + G + 1;
    const size_t slots = (size_t)nl->clusters_cap * kClusterSize;
    std::vector<int> start, cand;
    if ((st = build_candidates(nl, start, cand))) return st;
    if ((st = dalloc(&nl->d_cand_start, G + 1))) return st;
    if ((st = dalloc(&nl->d_cand, cand.size()))) return st;
    SPGNB_CUDA(cudaMemcpy(nl->d_cand_start, start.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice));
    SPGNB_CUDA(cudaMemcpy(nl->d_cand, cand.data(), sizeof(int) * cand.size(), cudaMemcpyHostToDevice));
    if ((st = dalloc(&nl->d_cell_count, G))) return st;
    if ((st = dalloc(&nl->d_cell_cursor, G))) return st;
    if ((st = dalloc(&nl->d_cell_cl_start, G + 1))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_cell_count, 0, sizeof(int) * G));
    SPGNB_CUDA(cudaMemset(nl->d_cell_cursor, 0, sizeof(int) * G));
    if ((st = dalloc(&nl->d_atom_cell, n))) return st;
    if ((st = dalloc(&nl->d_atom_shift, n))) return st;
    if ((st = dalloc(&nl->d_wrapped, n))) return st;
    if ((st = dalloc(&nl->d_atom_slot, n))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_atom_slot, 0xff, sizeof(int) * n));
    if ((st = dalloc(&nl->d_tmp_atoms, slots))) return st;
    if ((st = dalloc(&nl->d_slot_atom, slots))) return st;
    if ((st = dalloc(&nl->d_slot_x0, slots))) return st;
    if ((st = dalloc(&nl->d_slot_d0, slots))) return st;
    if ((st = dalloc(&nl->d_cl_cell, nl->clusters_cap))) return st;
    if ((st = dalloc(&nl->d_cl_u, nl->clusters_cap))) return st;
    if ((st = dalloc(&nl->d_cl_c, nl->clusters_cap))) return st;
    if ((st = dalloc(&nl->d_counters, kCntSize))) return st;
    SPGNB_CUDA(cudaMemset(nl->d_counters, 0, sizeof(int) * kCntSize));
    if ((st = alloc_pair_list(nl))) return st;
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

int estimate_entries_per_cluster(const spgnb_nl* nl)
{
    if (nl->opt.max_entries_per_cluster > 0) return nl->opt.max_entries_per_cluster;
    double vol = (double)nl->cell.a11 * nl->cell.a22 * nl->cell.a33;
    double rho = nl->n_cap / vol;
    double R = nl->cutoff + nl->skin + 6.0;
    double per = 4.18879 * R * R * R * rho / kClusterSize;  // clusters within R
    int e = (int)(per * 0.5 * 2.0) + 64;                     // half list, 2x margin
    return std::max(e, 96);
}

}  // namespace
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
    spgnb_nl* nl = new spgnb_nl();
    if (opt)
        nl->opt = *opt;
    else
        spgnb_nl_default_options(&nl->opt);
    if (nl->opt.max_neighbor_numbers <= 0) nl->opt.max_neighbor_numbers = 1200;
    nl->n_cap = atom_numbers;
    nl->cutoff = cutoff;
    nl->skin = skin;
    nl->cell = cell;
    nl->rcell = rcell;
    nl->triclinic = cell.a21 != 0.0f || cell.a31 != 0.0f || cell.a32 != 0.0f;
    grid_dims(cell, cutoff, skin, nl->dims, &nl->grid_length);
    nl->cs2 = nl->grid_length * nl->grid_length * 4.0f;
    if (nl->dims[0] <= 2 || nl->dims[1] <= 2 || nl->dims[2] <= 2)
    {
        delete nl;
        return fail(SPGNB_E_ARG, "NEIGHBOR_LIST: the box is too small (grid %dx%dx%d, need >= 3 per dimension)",
                    (int)floorf(cell.a11 / (0.5f * (cutoff + skin))), (int)floorf(cell.a22 / (0.5f * (cutoff + skin))),
                    (int)floorf(cell.a33 / (0.5f * (cutoff + skin))));
    }
    nl->G = nl->dims[0] * nl->dims[1] * nl->dims[2];
    nl->entries_per_cluster = estimate_entries_per_cluster(nl);
    int st = alloc_nl(nl);
    if (st)
    {
        free_nl(nl);
        delete nl;
        return st;
    }
    *out = nl;
    return SPGNB_OK;
}

int spgnb_nl_update(spgnb_nl* nl, const int* d_atom_local, int local_atom_numbers, int ghost_numbers,
                    const spgnb_vector* d_crd, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, int step, int update,
                    const int* d_excluded_list_start, const int* d_excluded_list, const int* d_excluded_numbers)
{
    if (!nl) return fail(SPGNB_E_ARG, "spgnb_nl_update: nl is NULL");
    if (local_atom_numbers <= 0 && ghost_numbers <= 0) return SPGNB_OK;
    if (ghost_numbers != 0)
        return fail(SPGNB_E_UNSUPPORTED, "spgnb_nl_update: ghost atoms (multi-rank domain decomposition) are not "
                                         "supported; run one rank per system");
    if (local_atom_numbers > nl->n_cap)
        return fail(SPGNB_E_ARG, "spgnb_nl_update: %d local atoms exceed the %d the list was created for",
                    local_atom_numbers, nl->n_cap);
    if (!d_atom_local || !d_crd || !d_excluded_list_start || !d_excluded_list || !d_excluded_numbers)
        return fail(SPGNB_E_ARG, "spgnb_nl_update: NULL device pointer");
    if (memcmp(&cell, &nl->cell, sizeof(cell)) != 0)
    {
        // The reference re-initialises on a large box change (main.cpp:864-939);
        // here the grid follows the new box when its shape allows.
        int dims[3];
        float gl;
        grid_dims(cell, nl->cutoff, nl->skin, dims, &gl);
        if (dims[0] != nl->dims[0] || dims[1] != nl->dims[1] || dims[2] != nl->dims[2])
            return fail(SPGNB_E_STATE, "spgnb_nl_update: the box changed the grid; recreate the list");
        nl->cell = cell;
        nl->rcell = rcell;
        nl->grid_length = gl;
        nl->cs2 = gl * gl * 4.0f;
    }
    cudaStream_t s = stream();
    const Cell c = make_cell(cell), rc = make_cell(rcell);
    const bool host_knows = update == SPGNB_FORCED_UPDATE || !nl->built || nl->opt.refresh_interval > 0 ||
                            local_atom_numbers != nl->local_atoms;
    if (host_knows)
    {
        bool rebuild = update == SPGNB_FORCED_UPDATE || !nl->built || local_atom_numbers != nl->local_atoms ||
                       ((step + 1) % nl->opt.refresh_interval == 0);
        if (!rebuild) return SPGNB_OK;
        k_set_need<<<1, 1, 0, s>>>(nl->d_counters);
        SPGNB_CHECK_LAUNCH("k_set_need");
    }
    else
    {
        SPGNB_CUDA(cudaMemsetAsync(nl->d_counters + kCntNeed, 0, sizeof(int), s));
        float permit = nl->skin * nl->opt.skin_permit;
        int slots = nl->clusters_cap * kClusterSize;
        k_check_refresh<<<(slots + 255) / 256, 256, 0, s>>>(slots, nl->d_slot_atom, (const float3*)d_crd,
                                                              nl->d_slot_x0, c, rc, permit * permit,
                                                              nl->d_counters);
        SPGNB_CHECK_LAUNCH("k_check_refresh");
    }
    const int n = local_atom_numbers;
    Grid g{nl->dims[0], nl->dims[1], nl->dims[2], nl->G, nl->grid_length, nl->cs2, c, rc};
    k_reset_list_counters<<<1, 1, 0, s>>>(nl->d_counters);
    k_bin<<<(n + 255) / 256, 256, 0, s>>>(n, (const float3*)d_crd, g, nl->d_atom_cell, nl->d_atom_shift,
                                            nl->d_wrapped, nl->d_cell_count, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_bin");
    k_scan_cells<<<1, 1024, 0, s>>>(nl->G, nl->d_cell_count, nl->d_cell_cl_start,
                                     nl->opt.max_atom_in_grid_numbers, nl->clusters_cap, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_scan_cells");
    const int slots_cap = nl->clusters_cap * kClusterSize;
    k_scatter<<<(n + 255) / 256, 256, 0, s>>>(n, nl->d_atom_cell, nl->d_cell_cl_start, nl->d_cell_cursor,
                                                nl->d_tmp_atoms, slots_cap, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_scatter");
    int sort_blocks = std::min(nl->G, num_sms() * 16);
    k_sort_cells<<<sort_blocks, 128, 2048 * sizeof(unsigned long long), s>>>(
        g, nl->d_cell_count, nl->d_cell_cl_start, nl->d_tmp_atoms, nl->d_wrapped, nl->d_slot_atom,
        nl->d_cl_cell, nl->d_atom_slot, slots_cap, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_sort_cells");
    k_cluster_props<<<(slots_cap + 255) / 256, 256, 0, s>>>((const float3*)d_crd, nl->d_slot_atom,
                                                             nl->d_atom_shift, d_atom_local, c, nl->d_counters,
                                                             nl->d_cl_u,
                                                             nl->d_cl_c, nl->d_slot_x0, nl->d_slot_d0,
                                                             nl->clusters_cap);
    SPGNB_CHECK_LAUNCH("k_cluster_props");
    SearchParams sp;
    sp.g = g;
    sp.list_radius = sqrtf(nl->cs2) * 1.0001f + 1e-3f;
    sp.frac_norm[0] = sqrtf(rc.a11 * rc.a11 + rc.a21 * rc.a21 + rc.a31 * rc.a31);
    sp.frac_norm[1] = sqrtf(rc.a22 * rc.a22 + rc.a32 * rc.a32);
    sp.frac_norm[2] = fabsf(rc.a33);
    sp.triclinic = nl->triclinic ? 1 : 0;
    sp.entries_cap = nl->entries_cap;
    sp.items_cap = nl->items_cap;
    sp.clusters_cap = nl->clusters_cap;
    int search_blocks = std::min((nl->clusters_cap + kSearchWarps - 1) / kSearchWarps, num_sms() * 8);
    k_search<<<search_blocks, kSearchWarps * 32, 0, s>>>(
        sp, nl->d_cand_start, nl->d_cand, nl->d_cell_cl_start, nl->d_cl_cell, nl->d_cl_u, nl->d_slot_x0,
        d_excluded_list_start, d_excluded_list, d_excluded_numbers,
        nl->d_ents, nl->d_ents_d, nl->d_items, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_search");
    if (nl->opt.export_atom_groups)
    {
        k_export_zero<<<(n + 255) / 256, 256, 0, s>>>(n, nl->d_nl, nl->d_counters);
        SPGNB_CHECK_LAUNCH("k_export_zero");
        k_export<<<num_sms() * 8, 128, 0, s>>>(nl->d_items, nl->d_ents, nl->d_slot_atom, d_atom_local, nl->d_nl,
                                                nl->d_temp, nl->opt.max_neighbor_numbers, nl->d_counters,
                                                nl->items_cap);
        SPGNB_CHECK_LAUNCH("k_export");
    }
    k_finish<<<(nl->G + 255) / 256, 256, 0, s>>>(nl->G, nl->d_cell_count, nl->d_cell_cursor, nl->d_counters);
    SPGNB_CHECK_LAUNCH("k_finish");
    nl->built = true;
    nl->local_atoms = local_atom_numbers;
    nl->host_builds++;
    return SPGNB_OK;
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
    out->clusters = h[kCntClusters];
    long long e;
    memcpy(&e, &h[kCntEntries], sizeof(e));
    out->entries = e;
    out->work_items = h[kCntItems];
    out->builds = h[kCntBuilds];
    out->overflow = h[kCntOverflow];
    return SPGNB_OK;
}

int spgnb_nl_check_overflow(spgnb_nl* nl, int steps, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                            int* reinitialized)
{
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
    // Regrow by 1.1x as the reference does (neighbor_list.cpp:896-941) and
    // force a rebuild on the next update.
    if (flags & kOvfGrid) nl->opt.max_atom_in_grid_numbers = (int)(nl->opt.max_atom_in_grid_numbers * 1.1);
    if (flags & kOvfList)
    {
        nl->opt.max_neighbor_numbers = (int)(nl->opt.max_neighbor_numbers * 1.1);
        dfree(nl->d_nl);
        dfree(nl->d_temp);
        int st;
        if ((st = dalloc(&nl->d_nl, nl->n_cap))) return st;
        if ((st = dalloc(&nl->d_temp, (size_t)nl->n_cap * nl->opt.max_neighbor_numbers))) return st;
        k_init_atom_groups<<<(nl->n_cap + 255) / 256, 256, 0, stream()>>>(nl->n_cap, nl->d_nl, nl->d_temp,
                                                                         nl->opt.max_neighbor_numbers);
        SPGNB_CHECK_LAUNCH("k_init_atom_groups");
    }
    if (flags & kOvfPairs)
    {
        nl->entries_per_cluster = (int)(nl->entries_per_cluster * 1.1) + 8;
        int st = alloc_pair_list(nl);
        if (st) return st;
    }
    if (memcmp(&cell, &nl->cell, sizeof(cell)) != 0)
    {
        nl->cell = cell;
        nl->rcell = rcell;
    }
    SPGNB_CUDA(cudaMemsetAsync(nl->d_counters + kCntOverflow, 0, sizeof(int), stream()));
    nl->built = false;
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
            int c = std::min(h[i].atom_numbers, m);
            memcpy(h_lists + off, slab.data() + (size_t)i * m, sizeof(int) * c);
            off += h[i].atom_numbers;
        }
    }
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
