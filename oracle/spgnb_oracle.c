/*
 * spgnb oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of SPONGE's short-range nonbonded path, used by the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark as the
 * checker.  Nothing in the product links, loads or calls this file.
 *
 * Parity pins: the neighbour-set rule and the FP32 candidate test are checked
 * against outputs of the reference's own CPU build (oracle/_ref, built from
 * the reference sources by oracle/Makefile) stored as golden fixtures under
 * tests/golden/, and the FP64 pair sum against the same fixtures and the
 * GROMACS lj_sr energy the reference's comparison suite holds
 * (benchmarks/comparison/reference/gromacs/reference.json).
 *
 * Functions and the reference lines they restate:
 *   orc_beta            SPONGE/PM_force/PM_force.cpp:244-272 (Get_Beta)
 *   orc_grid_dims       SPONGE/neighbor_list/neighbor_list.cpp:58-67
 *   orc_stencil         SPONGE/neighbor_list/neighbor_list.cpp:5-49
 *   orc_cell_of         SPONGE/neighbor_list/neighbor_list.cpp:219-239
 *   orc_pair_dr2        SPONGE/utils/vector.hpp:322-327 + neighbor_list.cpp:367-372
 *   orc_nl_build        neighbor_list.cpp:279-492 (half rule, candidate radius
 *                       (rc+skin)^2 = 4*grid_length^2 from :705) and
 *                       neighbor_list.cpp:594-665 (exclusion removal)
 *   orc_pair_force_fp64 SPONGE/Lennard_Jones_force/Lennard_Jones_force.h:44-73
 *                       and Lennard_Jones_force.cpp:61-135 (sign, cutoff test,
 *                       virial, energy owner), evaluated in double
 *   orc_direct_sum_fp64 the same pair function over every pair within rc
 *                       (no neighbour list): the FP64 direct pair sum
 *   orc_long_range      Lennard_Jones_force.cpp:146-184,267-268,312-341
 *   orc_soft_core_fp64  SPONGE/Lennard_Jones_force/LJ_soft_core.cpp:198-414 and
 *                       LJ_soft_core.h:33-150 (the two-state pair, soft cores,
 *                       dH/dlambda), evaluated in double over every pair within rc
 *   orc_soft_long_range LJ_soft_core.cpp:83-181, :605-635
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_STENCIL 192

/* ---------------------------------------------------------------- beta */
float orc_beta(float cutoff, float tolerance)
{
    float beta = 0.0f, low, high, tempf;
    int ilow, ihigh;
    high = 1.0f;
    ihigh = 1;
    for (;;)
    {
        tempf = erfcf(high * cutoff) / cutoff;
        if (tempf <= tolerance) break;
        high *= 2;
        ihigh++;
    }
    ihigh += 50;
    low = 0.0f;
    for (ilow = 1; ilow < ihigh; ilow++)
    {
        beta = (low + high) / 2;
        tempf = erfcf(beta * cutoff) / cutoff;
        if (tempf >= tolerance)
            low = beta;
        else
            high = beta;
    }
    return beta;
}

/* ---------------------------------------------------------------- grid */
void orc_grid_dims(const float* cell, float cutoff, float skin, int* dims, float* grid_length)
{
    float gl = 0.5f * (cutoff + skin);
    dims[0] = (int)floorf(cell[0] / gl);
    dims[1] = (int)floorf(cell[2] / gl);
    dims[2] = (int)floorf(cell[5] / gl);
    *grid_length = gl;
}

/* Stencil of grid cell g: the cells j for which some periodic image offset
 * (i + shift_k - j) lies inside [cx,2]x[cy,2]x[-2,2]; each j listed once. */
int orc_stencil(int g, const int* dims, float grid_length, const float* cell, int* out)
{
    int Nx = dims[0], Ny = dims[1], Nz = dims[2];
    int NyNz = Ny * Nz;
    int gx = g / NyNz, gy = (g % NyNz) / Nz, gz = g % Nz;
    int dxy = (int)(cell[1] / grid_length);
    int dxz = (int)(cell[3] / grid_length);
    int dyz = (int)(cell[4] / grid_length);
    int G = Nx * Ny * Nz;
    char* seen = (char*)calloc((size_t)G, 1);
    int count = 0;
    for (int k = 0; k < 27; k++)
    {
        int dx = k / 9 - 1, dy = (k % 9) / 3 - 1, dz = k % 3 - 1;
        int cx = (dy * cell[1] + dz * cell[3] == 0) ? -2 : -3;
        int cy = (dz * cell[4] == 0) ? -2 : -3;
        int sx = gx + dx * Nx + dy * dxy + dz * dxz;
        int sy = gy + dy * Ny + dz * dyz;
        int sz = gz + dz * Nz;
        for (int tx = cx; tx <= 2; tx++)
            for (int ty = cy; ty <= 2; ty++)
                for (int tz = -2; tz <= 2; tz++)
                {
                    int jx = sx - tx, jy = sy - ty, jz = sz - tz;
                    if (jx < 0 || jx >= Nx || jy < 0 || jy >= Ny || jz < 0 || jz >= Nz) continue;
                    int j = jx * NyNz + jy * Nz + jz;
                    if (!seen[j])
                    {
                        seen[j] = 1;
                        if (count < ORC_MAX_STENCIL) out[count] = j;
                        count++;
                    }
                }
    }
    free(seen);
    /* ascending order, as the reference enumerates grid_j */
    int n = count < ORC_MAX_STENCIL ? count : ORC_MAX_STENCIL;
    for (int a = 1; a < n; a++)
    {
        int v = out[a], b = a - 1;
        while (b >= 0 && out[b] > v)
        {
            out[b + 1] = out[b];
            b--;
        }
        out[b + 1] = v;
    }
    return count;
}

int orc_cell_of(const float* crd3, const float* cell, const int* dims, float grid_length)
{
    float x = crd3[0], y = crd3[1], z = crd3[2];
    float k3 = floorf(z / cell[5]);
    z -= k3 * cell[5];
    y -= k3 * cell[4];
    float k2 = floorf(y / cell[2]);
    y -= k2 * cell[2];
    x -= k3 * cell[3] + k2 * cell[1];
    x -= floorf(x / cell[0]) * cell[0];
    int nx = (int)(x / grid_length);
    int ny = (int)(y / grid_length);
    int nz = (int)(z / grid_length);
    nx = nx < 0 ? 0 : (nx < dims[0] ? nx : dims[0] - 1);
    ny = ny < 0 ? 0 : (ny < dims[1] ? ny : dims[1] - 1);
    nz = nz < 0 ? 0 : (nz < dims[2] ? nz : dims[2] - 1);
    return nx * dims[1] * dims[2] + ny * dims[2] + nz;
}

/* FP32 squared minimum-image distance of a = crd_i, b = crd_j, in the
 * operation order of Get_Periodic_Displacement followed by the dot product.
 * mode 0: every multiply and add rounded separately (a host compiler with
 * contraction off).  mode 1: the fused multiply-adds a CUDA compiler forms
 * from the same expression: s = x*r11 + y*r21 + z*r31 -> fma(z,r31,fma(x,r11,y*r21)),
 * s.z + 0.5 -> fma(z,r33,0.5), n*cell products are exact, and
 * x*x + y*y + z*z -> fma(z,z,fma(x,x,y*y)). */
float orc_pair_dr2(const float* a, const float* b, const float* cell, const float* rc, int mode)
{
    float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    float sx, sy, sz;
    if (mode == 0)
    {
        sx = dx * rc[0] + dy * rc[1] + dz * rc[3];
        sy = dy * rc[2] + dz * rc[4];
        sz = dz * rc[5];
        sx = floorf(sx + 0.5f);
        sy = floorf(sy + 0.5f);
        sz = floorf(sz + 0.5f);
        float tx = sx * cell[0] + sy * cell[1] + sz * cell[3];
        float ty = sy * cell[2] + sz * cell[4];
        float tz = sz * cell[5];
        dx = dx - tx;
        dy = dy - ty;
        dz = dz - tz;
        return dx * dx + dy * dy + dz * dz;
    }
    sx = fmaf(dz, rc[3], fmaf(dx, rc[0], dy * rc[1]));
    sy = fmaf(dy, rc[2], dz * rc[4]);
    sx = floorf(sx + 0.5f);
    sy = floorf(sy + 0.5f);
    sz = floorf(fmaf(dz, rc[5], 0.5f));
    float tx = fmaf(sz, cell[3], fmaf(sx, cell[0], sy * cell[1]));
    float ty = fmaf(sy, cell[2], sz * cell[4]);
    dx = dx - tx;
    dy = dy - ty;
    dz = fmaf(-sz, cell[5], dz);
    return fmaf(dz, dz, fmaf(dx, dx, dy * dy));
}

static int excluded_upper(int lo, int hi, const int* es, const int* en, const int* el)
{
    int k = en[lo];
    if (k <= 0) return 0;
    const int* l = el + es[lo];
    if (hi < l[0] || hi > l[k - 1]) return 0;
    for (int t = 0; t < k; t++)
        if (l[t] == hi) return 1;
    return 0;
}

static int cmp_int(const void* a, const void* b)
{
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* Half neighbour list of the reference: owner i holds j with j > i (global
 * index == local index on one rank), FP32 dr2 < 4*gl^2, excluded pairs
 * removed.  counts[n] is always filled; the sorted lists go to out[] when
 * capacity suffices.  Returns the number of pairs, or -1 on a stencil
 * overflow, -2 on a box too small for the grid (fewer than 3 cells). */
long long orc_nl_build(int n, const float* crd, const float* cell, const float* rcell, float cutoff,
                       float skin, const int* excl_start, const int* excl_numbers, const int* excl_list,
                       int mode, int* counts, int* out, long long capacity)
{
    int dims[3];
    float gl;
    orc_grid_dims(cell, cutoff, skin, dims, &gl);
    if (dims[0] <= 2 || dims[1] <= 2 || dims[2] <= 2) return -2;
    float cs2 = gl * gl * 4.0f;
    int G = dims[0] * dims[1] * dims[2];
    int* cell_of = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* cstart = (int*)calloc((size_t)G + 1, sizeof(int));
    int* catoms = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++)
    {
        cell_of[i] = orc_cell_of(crd + 3 * i, cell, dims, gl);
        cstart[cell_of[i] + 1]++;
    }
    for (int g = 0; g < G; g++) cstart[g + 1] += cstart[g];
    {
        int* fill = (int*)malloc(sizeof(int) * (size_t)G);
        memcpy(fill, cstart, sizeof(int) * (size_t)G);
        for (int i = 0; i < n; i++) catoms[fill[cell_of[i]]++] = i;
        free(fill);
    }
    int overflow = 0;
    memset(counts, 0, sizeof(int) * (size_t)n);
    /* pass 1: counts */
#pragma omp parallel for schedule(dynamic) reduction(| : overflow)
    for (int g = 0; g < G; g++)
    {
        int st[ORC_MAX_STENCIL];
        int ns = orc_stencil(g, dims, gl, cell, st);
        if (ns > ORC_MAX_STENCIL)
        {
            overflow = 1;
            ns = ORC_MAX_STENCIL;
        }
        for (int a = cstart[g]; a < cstart[g + 1]; a++)
        {
            int i = catoms[a];
            int c = 0;
            for (int s = 0; s < ns; s++)
            {
                int h = st[s];
                for (int b = cstart[h]; b < cstart[h + 1]; b++)
                {
                    int j = catoms[b];
                    if (j <= i) continue;
                    if (orc_pair_dr2(crd + 3 * i, crd + 3 * j, cell, rcell, mode) < cs2 &&
                        !excluded_upper(i, j, excl_start, excl_numbers, excl_list))
                        c++;
                }
            }
            counts[i] = c;
        }
    }
    long long total = 0;
    for (int i = 0; i < n; i++) total += counts[i];
    if (out != NULL && capacity >= total && !overflow)
    {
        long long* off = (long long*)malloc(sizeof(long long) * (size_t)(n + 1));
        off[0] = 0;
        for (int i = 0; i < n; i++) off[i + 1] = off[i] + counts[i];
#pragma omp parallel for schedule(dynamic)
        for (int g = 0; g < G; g++)
        {
            int st[ORC_MAX_STENCIL];
            int ns = orc_stencil(g, dims, gl, cell, st);
            if (ns > ORC_MAX_STENCIL) ns = ORC_MAX_STENCIL;
            for (int a = cstart[g]; a < cstart[g + 1]; a++)
            {
                int i = catoms[a];
                long long w = off[i];
                for (int s = 0; s < ns; s++)
                {
                    int h = st[s];
                    for (int b = cstart[h]; b < cstart[h + 1]; b++)
                    {
                        int j = catoms[b];
                        if (j <= i) continue;
                        if (orc_pair_dr2(crd + 3 * i, crd + 3 * j, cell, rcell, mode) < cs2 &&
                            !excluded_upper(i, j, excl_start, excl_numbers, excl_list))
                            out[w++] = j;
                    }
                }
                qsort(out + off[i], (size_t)counts[i], sizeof(int), cmp_int);
            }
        }
        free(off);
    }
    free(cell_of);
    free(cstart);
    free(catoms);
    return overflow ? -1 : total;
}

/* ------------------------------------------------------ FP64 pair force */
static inline int lj_index(int a, int b)
{
    int hi = a > b ? a : b, lo = a > b ? b : a;
    return hi * (hi + 1) / 2 + lo;
}

typedef struct
{
    double e_lj, e_coul, vir[6];
    long long pairs_in_cutoff;
} orc_totals;

/* Accumulates the pair (i owner, j) in double.  dr = r_j - r_i with the
 * minimum image taken in double on the double inverse cell; the reference's
 * F/r = (B - A r^-6) r^-8 - q_i q_j r^-3 (erfc(beta r) + 2 beta r/sqrt(pi)
 * exp(-beta^2 r^2)); F_i += F/r dr; F_j -= F/r dr; the owner's virial gets
 * -(F/r) dr (x) dr in the symmetrised lower-triangular form, its energy
 * E_lj = (A/12 r^-6 - B/6) r^-6 and E_c = q_i q_j erfc(beta r)/r. */
static inline void pair_fp64(int i, int j, const float* crd, const float* charge, const int* type,
                             const float* A, const float* B, const double* cell, const double* ri,
                             double rc, double beta, double* frc, double* e_atom_lj, double* e_atom_c,
                             double* vir_atom, orc_totals* t)
{
    double dx = (double)crd[3 * j] - crd[3 * i];
    double dy = (double)crd[3 * j + 1] - crd[3 * i + 1];
    double dz = (double)crd[3 * j + 2] - crd[3 * i + 2];
    double sx = dx * ri[0] + dy * ri[1] + dz * ri[3];
    double sy = dy * ri[2] + dz * ri[4];
    double sz = dz * ri[5];
    sx = floor(sx + 0.5);
    sy = floor(sy + 0.5);
    sz = floor(sz + 0.5);
    dx -= sx * cell[0] + sy * cell[1] + sz * cell[3];
    dy -= sy * cell[2] + sz * cell[4];
    dz -= sz * cell[5];
    double r2 = dx * dx + dy * dy + dz * dz;
    double r = sqrt(r2);
    if (!(r < rc)) return;
    int p = lj_index(type[i], type[j]);
    double a = A[p], b = B[p];
    double r6 = 1.0 / (r2 * r2 * r2);
    double r8 = r6 / r2;
    double qq = (double)charge[i] * (double)charge[j];
    double br = beta * r;
    double erfcv = erfc(br);
    double fscal = (b - a * r6) * r8 - qq / (r2 * r) * (erfcv + 1.1283791670955126 * br * exp(-br * br));
    double fx = fscal * dx, fy = fscal * dy, fz = fscal * dz;
    frc[3 * i] += fx;
    frc[3 * i + 1] += fy;
    frc[3 * i + 2] += fz;
    frc[3 * j] -= fx;
    frc[3 * j + 1] -= fy;
    frc[3 * j + 2] -= fz;
    double elj = (a / 12.0 * r6 - b / 6.0) * r6;
    double ec = qq * erfcv / r;
    double v[6] = {-fx * dx, -(fx * dy + fy * dx), -fy * dy, -(fx * dz + fz * dx), -(fy * dz + fz * dy), -fz * dz};
    if (e_atom_lj) e_atom_lj[i] += elj;
    if (e_atom_c) e_atom_c[i] += ec;
    if (vir_atom)
        for (int k = 0; k < 6; k++) vir_atom[6 * i + k] += v[k];
    t->e_lj += elj;
    t->e_coul += ec;
    for (int k = 0; k < 6; k++) t->vir[k] += v[k];
    t->pairs_in_cutoff++;
}

static void cell_inverse_fp64(const float* cell, double* c, double* ri)
{
    for (int k = 0; k < 6; k++) c[k] = cell[k];
    ri[0] = 1.0 / c[0];
    ri[2] = 1.0 / c[2];
    ri[5] = 1.0 / c[5];
    ri[1] = -c[1] * ri[2] / c[0];
    ri[4] = -c[4] * ri[5] / c[2];
    ri[3] = (c[4] * c[1] * ri[5] - c[3] * c[2]) / (c[0] * c[2] * c[5]);
}

/* FP64 forces/energies over a given half list (CSR: counts + sorted lists).
 * Outputs are overwritten.  Returns the number of pairs inside rc. */
long long orc_pair_force_fp64(int n, const float* crd, const float* charge, const int* type, const float* A,
                              const float* B, const float* cell, float cutoff, float beta, const int* counts,
                              const int* list, double* frc, double* e_atom_lj, double* e_atom_c,
                              double* vir_atom, double* totals /* e_lj, e_coul, vir[6] */)
{
    double c[6], ri[6];
    cell_inverse_fp64(cell, c, ri);
    memset(frc, 0, sizeof(double) * 3 * (size_t)n);
    if (e_atom_lj) memset(e_atom_lj, 0, sizeof(double) * (size_t)n);
    if (e_atom_c) memset(e_atom_c, 0, sizeof(double) * (size_t)n);
    if (vir_atom) memset(vir_atom, 0, sizeof(double) * 6 * (size_t)n);
    orc_totals t;
    memset(&t, 0, sizeof(t));
    long long off = 0;
    for (int i = 0; i < n; i++)
    {
        for (int k = 0; k < counts[i]; k++)
            pair_fp64(i, list[off + k], crd, charge, type, A, B, c, ri, cutoff, beta, frc, e_atom_lj, e_atom_c,
                      vir_atom, &t);
        off += counts[i];
    }
    totals[0] = t.e_lj;
    totals[1] = t.e_coul;
    for (int k = 0; k < 6; k++) totals[2 + k] = t.vir[k];
    return t.pairs_in_cutoff;
}

/* Calls fn(i, j, ctx) for every pair i < j whose atoms sit in neighbouring
 * coarse cells (cells of at least rc in every fractional direction; every
 * cell when a dimension has fewer than 3), exclusions removed.  The caller
 * applies the distance test. */
typedef void (*orc_pair_fn)(int i, int j, void* ctx);

static void sweep_pairs(int n, const float* crd, const double* c, const double* ri, float cutoff,
                        const int* excl_start, const int* excl_numbers, const int* excl_list, orc_pair_fn fn,
                        void* ctx)
{
    double h[3] = {c[0], c[2], c[5]};
    int m[3];
    for (int d = 0; d < 3; d++)
    {
        m[d] = (int)floor(h[d] / cutoff);
        if (m[d] < 1) m[d] = 1;
    }
    int G = m[0] * m[1] * m[2];
    int* cell_of = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* cstart = (int*)calloc((size_t)G + 1, sizeof(int));
    int* catoms = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++)
    {
        double x = crd[3 * i], y = crd[3 * i + 1], z = crd[3 * i + 2];
        double s[3] = {x * ri[0] + y * ri[1] + z * ri[3], y * ri[2] + z * ri[4], z * ri[5]};
        int id[3];
        for (int d = 0; d < 3; d++)
        {
            double f = s[d] - floor(s[d]);
            id[d] = (int)(f * m[d]);
            if (id[d] >= m[d]) id[d] = m[d] - 1;
        }
        cell_of[i] = (id[0] * m[1] + id[1]) * m[2] + id[2];
        cstart[cell_of[i] + 1]++;
    }
    for (int g = 0; g < G; g++) cstart[g + 1] += cstart[g];
    {
        int* fill = (int*)malloc(sizeof(int) * (size_t)G);
        memcpy(fill, cstart, sizeof(int) * (size_t)G);
        for (int i = 0; i < n; i++) catoms[fill[cell_of[i]]++] = i;
        free(fill);
    }
    for (int i = 0; i < n; i++)
    {
        int g = cell_of[i];
        int gx = g / (m[1] * m[2]), gy = (g / m[2]) % m[1], gz = g % m[2];
        int rx = m[0] < 3 ? m[0] : 3, ry = m[1] < 3 ? m[1] : 3, rz = m[2] < 3 ? m[2] : 3;
        for (int ax = 0; ax < rx; ax++)
            for (int ay = 0; ay < ry; ay++)
                for (int az = 0; az < rz; az++)
                {
                    int hx = m[0] < 3 ? ax : (gx + ax - 1 + m[0]) % m[0];
                    int hy = m[1] < 3 ? ay : (gy + ay - 1 + m[1]) % m[1];
                    int hz = m[2] < 3 ? az : (gz + az - 1 + m[2]) % m[2];
                    int hcell = (hx * m[1] + hy) * m[2] + hz;
                    for (int b = cstart[hcell]; b < cstart[hcell + 1]; b++)
                    {
                        int j = catoms[b];
                        if (j <= i) continue;
                        if (excluded_upper(i, j, excl_start, excl_numbers, excl_list)) continue;
                        fn(i, j, ctx);
                    }
                }
    }
    free(cell_of);
    free(cstart);
    free(catoms);
}

typedef struct
{
    const float *crd, *charge, *A, *B;
    const int* type;
    const double *c, *ri;
    double rc, beta;
    double *frc, *e_atom_lj, *e_atom_c, *vir_atom;
    orc_totals t;
} plain_ctx;

static void plain_pair(int i, int j, void* ctx)
{
    plain_ctx* p = (plain_ctx*)ctx;
    pair_fp64(i, j, p->crd, p->charge, p->type, p->A, p->B, p->c, p->ri, p->rc, p->beta, p->frc, p->e_atom_lj,
              p->e_atom_c, p->vir_atom, &p->t);
}

/* FP64 direct pair sum: every pair with double minimum-image distance < rc,
 * exclusions removed, found by a cell sweep independent of the neighbour
 * list.  Same outputs as orc_pair_force_fp64. */
long long orc_direct_sum_fp64(int n, const float* crd, const float* charge, const int* type, const float* A,
                              const float* B, const float* cell, float cutoff, float beta, const int* excl_start,
                              const int* excl_numbers, const int* excl_list, double* frc, double* e_atom_lj,
                              double* e_atom_c, double* vir_atom, double* totals)
{
    double c[6], ri[6];
    cell_inverse_fp64(cell, c, ri);
    memset(frc, 0, sizeof(double) * 3 * (size_t)n);
    if (e_atom_lj) memset(e_atom_lj, 0, sizeof(double) * (size_t)n);
    if (e_atom_c) memset(e_atom_c, 0, sizeof(double) * (size_t)n);
    if (vir_atom) memset(vir_atom, 0, sizeof(double) * 6 * (size_t)n);
    plain_ctx p = {crd, charge, A, B, type, c, ri, cutoff, beta, frc, e_atom_lj, e_atom_c, vir_atom, {0}};
    sweep_pairs(n, crd, c, ri, cutoff, excl_start, excl_numbers, excl_list, plain_pair, &p);
    totals[0] = p.t.e_lj;
    totals[1] = p.t.e_coul;
    for (int k = 0; k < 6; k++) totals[2 + k] = p.t.vir[k];
    return p.t.pairs_in_cutoff;
}

/* FP64 forces on a subset of atoms: for each listed atom i, the force from
 * every partner j != i with double minimum-image distance < rc, exclusions
 * removed (either side of the upper-triangular CSR), by the same coarse-cell
 * sweep and the same pair function as pair_fp64 (Lennard_Jones_force.h:44-73,
 * vector.hpp:322-327).  For checking large boxes on a sample of atoms.
 * frc_sub gets 3 doubles per listed atom.  Returns the pairs counted. */
long long orc_direct_forces_subset_fp64(int n, const float* crd, const float* charge, const int* type,
                                        const float* A, const float* B, const float* cell, float cutoff, float beta,
                                        const int* excl_start, const int* excl_numbers, const int* excl_list,
                                        int n_sub, const int* sub, double* frc_sub)
{
    double c[6], ri[6];
    cell_inverse_fp64(cell, c, ri);
    double h[3] = {c[0], c[2], c[5]};
    int m[3];
    for (int d = 0; d < 3; d++)
    {
        m[d] = (int)floor(h[d] / cutoff);
        if (m[d] < 1) m[d] = 1;
    }
    int G = m[0] * m[1] * m[2];
    int* cell_of = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* cstart = (int*)calloc((size_t)G + 1, sizeof(int));
    int* catoms = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++)
    {
        double x = crd[3 * i], y = crd[3 * i + 1], z = crd[3 * i + 2];
        double sf[3] = {x * ri[0] + y * ri[1] + z * ri[3], y * ri[2] + z * ri[4], z * ri[5]};
        int id[3];
        for (int d = 0; d < 3; d++)
        {
            double f = sf[d] - floor(sf[d]);
            id[d] = (int)(f * m[d]);
            if (id[d] >= m[d]) id[d] = m[d] - 1;
        }
        cell_of[i] = (id[0] * m[1] + id[1]) * m[2] + id[2];
        cstart[cell_of[i] + 1]++;
    }
    for (int g = 0; g < G; g++) cstart[g + 1] += cstart[g];
    {
        int* fill = (int*)malloc(sizeof(int) * (size_t)G);
        memcpy(fill, cstart, sizeof(int) * (size_t)G);
        for (int i = 0; i < n; i++) catoms[fill[cell_of[i]]++] = i;
        free(fill);
    }
    long long pairs = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : pairs)
    for (int q = 0; q < n_sub; q++)
    {
        const int i = sub[q];
        double fx = 0, fy = 0, fz = 0;
        int g = cell_of[i];
        int gx = g / (m[1] * m[2]), gy = (g / m[2]) % m[1], gz = g % m[2];
        int rx = m[0] < 3 ? m[0] : 3, ry = m[1] < 3 ? m[1] : 3, rz = m[2] < 3 ? m[2] : 3;
        for (int ax = 0; ax < rx; ax++)
            for (int ay = 0; ay < ry; ay++)
                for (int az = 0; az < rz; az++)
                {
                    int hx = m[0] < 3 ? ax : (gx + ax - 1 + m[0]) % m[0];
                    int hy = m[1] < 3 ? ay : (gy + ay - 1 + m[1]) % m[1];
                    int hz = m[2] < 3 ? az : (gz + az - 1 + m[2]) % m[2];
                    int hcell = (hx * m[1] + hy) * m[2] + hz;
                    for (int b = cstart[hcell]; b < cstart[hcell + 1]; b++)
                    {
                        int j = catoms[b];
                        if (j == i) continue;
                        if (excluded_upper(i < j ? i : j, i < j ? j : i, excl_start, excl_numbers, excl_list)) continue;
                        double dx = (double)crd[3 * j] - crd[3 * i];
                        double dy = (double)crd[3 * j + 1] - crd[3 * i + 1];
                        double dz = (double)crd[3 * j + 2] - crd[3 * i + 2];
                        double sx = floor(dx * ri[0] + dy * ri[1] + dz * ri[3] + 0.5);
                        double sy = floor(dy * ri[2] + dz * ri[4] + 0.5);
                        double sz = floor(dz * ri[5] + 0.5);
                        dx -= sx * c[0] + sy * c[1] + sz * c[3];
                        dy -= sy * c[2] + sz * c[4];
                        dz -= sz * c[5];
                        double r2 = dx * dx + dy * dy + dz * dz;
                        double r = sqrt(r2);
                        if (!(r < cutoff)) continue;
                        int p = lj_index(type[i], type[j]);
                        double a = A[p], bb = B[p];
                        double r6 = 1.0 / (r2 * r2 * r2);
                        double r8 = r6 / r2;
                        double qq = (double)charge[i] * (double)charge[j];
                        double br = beta * r;
                        double fscal = (bb - a * r6) * r8 -
                                       qq / (r2 * r) * (erfc(br) + 1.1283791670955126 * br * exp(-br * br));
                        fx += fscal * dx;
                        fy += fscal * dy;
                        fz += fscal * dz;
                        pairs++;
                    }
                }
        frc_sub[3 * q] = fx;
        frc_sub[3 * q + 1] = fy;
        frc_sub[3 * q + 2] = fz;
    }
    free(cell_of);
    free(cstart);
    free(catoms);
    return pairs;
}

/* ------------------------------------------------- FP64 soft-core pair sum */
/* LJ_SOFT_CORE's pair (SPONGE/Lennard_Jones_force/LJ_soft_core.cpp:198-414,
 * pair functions LJ_soft_core.h:33-150) in double.  Owner i < j,
 * dr = r_j - r_i (minimum image in double), r < rc.  With l = lambda,
 * l' = 1 - l, the state tables AA/AB (state A) and BA/BB (state B):
 *   linear branch (BA*AA != 0 or BA + AA == 0):
 *     F/r = l' LJF(r; AA, AB) + l LJF(r; BA, BB) - CF(r),
 *     E_lj = l' LJE(r; AA, AB) + l LJE(r; BA, BB), E_c = q_i q_j erfc(beta r)/r,
 *     dH_lj = LJE(r; BA, BB) - LJE(r; AA, AB), dH_c = erfc(beta r) dq / r;
 *   soft-core branch: sigma_X = sigma^6 if the state's A or B is 0, else
 *     max(A/(2B), sigma_min^6); r_A^6 = r^6 + alpha l^p sigma_A,
 *     r_B^6 = r^6 + alpha l'^p sigma_B;
 *     F/r = l' r^4 (AB - AA r_A^-6) r_A^-12 + l r^4 (BB - BA r_B^-6) r_B^-12
 *           - [l' SCF(r_A) + l SCF(r_B)] r^4,  SCF(s) = q_i q_j (2/sqrt(pi) beta
 *           e^-(beta s)^2 + erfc(beta s)/s) s^-6,
 *     E_lj = l' LJE(r_A) + l LJE(r_B), E_c = l' CE(r_A) + l CE(r_B),
 *     dH_lj = LJE(r_B) - LJE(r_A) + D_A LJF(r_A) r_A^-4 sigma_A
 *             - D_B LJF(r_B) r_B^-4 sigma_B,
 *     dH_c = CE(r_B) - CE(r_A) + D_B CF(r_B) r_B^-4 sigma_B
 *            - D_A CF(r_A) r_A^-4 sigma_A + l dq erfc(beta r_B)/r_B
 *            + l' dq erfc(beta r_A)/r_A,
 *   with LJF(s; A, B) = (B - A s^-6) s^-8, LJE(s; A, B) = (A/12 s^-6 - B/6) s^-6,
 *   CF(s) = q_i q_j s^-3 (2/sqrt(pi) beta s e^-(beta s)^2 + erfc(beta s)),
 *   CE(s) = q_i q_j erfc(beta s)/s, dq = q_i^BA q_j + q_i q_j^BA,
 *   D_A = p alpha l' (l + FLT_MIN)^(p-1) / 6, D_B = p alpha l (l' + FLT_MIN)^(p-1) / 6.
 * Forces, owner energies and virial as pair_fp64; dh[0] += dH_lj, dh[1] += dH_c. */
typedef struct
{
    const float *crd, *charge, *charge_ba, *AA, *AB, *BA, *BB;
    const int *ta, *tb;
    const double *c, *ri;
    double rc, beta, l, l_, alp_a, alp_b, d_a, d_b, s6, s6min;
    double *frc, *e_atom_lj, *e_atom_c, *vir_atom, dh[2];
    orc_totals t;
} soft_ctx;

static double lje(double s, double a, double b)
{
    double s6 = pow(s, -6.0);
    return (a / 12.0 * s6 - b / 6.0) * s6;
}

static double ljf(double s, double a, double b) { return (b - a * pow(s, -6.0)) * pow(s, -8.0); }

static void soft_pair(int i, int j, void* ctx)
{
    soft_ctx* p = (soft_ctx*)ctx;
    const double* cell = p->c;
    const double* ri = p->ri;
    double dx = (double)p->crd[3 * j] - p->crd[3 * i];
    double dy = (double)p->crd[3 * j + 1] - p->crd[3 * i + 1];
    double dz = (double)p->crd[3 * j + 2] - p->crd[3 * i + 2];
    double sx = floor(dx * ri[0] + dy * ri[1] + dz * ri[3] + 0.5);
    double sy = floor(dy * ri[2] + dz * ri[4] + 0.5);
    double sz = floor(dz * ri[5] + 0.5);
    dx -= sx * cell[0] + sy * cell[1] + sz * cell[3];
    dy -= sy * cell[2] + sz * cell[4];
    dz -= sz * cell[5];
    double r2 = dx * dx + dy * dy + dz * dz;
    double r = sqrt(r2);
    if (!(r < p->rc)) return;
    int pa = lj_index(p->ta[i], p->ta[j]), pb = lj_index(p->tb[i], p->tb[j]);
    double AA = p->AA[pa], AB = p->AB[pa], BA = p->BA[pb], BB = p->BB[pb];
    double qq = (double)p->charge[i] * p->charge[j];
    double dq = p->charge_ba ? (double)p->charge_ba[i] * p->charge[j] + (double)p->charge[i] * p->charge_ba[j] : 0.0;
    double beta = p->beta, l = p->l, l_ = p->l_;
    double f, elj, ec, dlj, dc;
    if ((float)BA * (float)AA != 0.0f || BA + AA == 0.0)
    {
        double br = beta * r, erfc_r = erfc(br);
        double cf = qq / (r2 * r) * (br * 1.1283791670955126 * exp(-br * br) + erfc_r);
        f = l_ * ljf(r, AA, AB) + l * ljf(r, BA, BB) - cf;
        elj = l_ * lje(r, AA, AB) + l * lje(r, BA, BB);
        ec = qq * erfc_r / r;
        dlj = lje(r, BA, BB) - lje(r, AA, AB);
        dc = erfc_r * dq / r;
    }
    else
    {
        double sa = (AA == 0.0 || AB == 0.0) ? p->s6 : fmax(0.5 * AA / AB, p->s6min);
        double sb = (BA == 0.0 || BB == 0.0) ? p->s6 : fmax(0.5 * BA / BB, p->s6min);
        double r6 = r2 * r2 * r2, r4 = r2 * r2;
        double ra = pow(r6 + p->alp_a * sa, 1.0 / 6.0), rb = pow(r6 + p->alp_b * sb, 1.0 / 6.0);
        double bra = beta * ra, brb = beta * rb;
        double erfc_a = erfc(bra), erfc_b = erfc(brb), exp_a = exp(-bra * bra), exp_b = exp(-brb * brb);
        double scf_a = qq * (exp_a * 1.1283791670955126 * beta + erfc_a / ra) * pow(ra, -6.0);
        double scf_b = qq * (exp_b * 1.1283791670955126 * beta + erfc_b / rb) * pow(rb, -6.0);
        f = l_ * r4 * (AB - AA * pow(ra, -6.0)) * pow(ra, -12.0) + l * r4 * (BB - BA * pow(rb, -6.0)) * pow(rb, -12.0) -
            (l_ * scf_a + l * scf_b) * r4;
        double cea = qq * erfc_a / ra, ceb = qq * erfc_b / rb;
        elj = l_ * lje(ra, AA, AB) + l * lje(rb, BA, BB);
        ec = l_ * cea + l * ceb;
        dlj = lje(rb, BA, BB) - lje(ra, AA, AB) + p->d_a * ljf(ra, AA, AB) * pow(ra, -4.0) * sa -
              p->d_b * ljf(rb, BA, BB) * pow(rb, -4.0) * sb;
        double cf_a = qq * pow(ra, -3.0) * (bra * 1.1283791670955126 * exp_a + erfc_a);
        double cf_b = qq * pow(rb, -3.0) * (brb * 1.1283791670955126 * exp_b + erfc_b);
        dc = ceb - cea + p->d_b * cf_b * pow(rb, -4.0) * sb - p->d_a * cf_a * pow(ra, -4.0) * sa +
             l * dq * erfc_b / rb + l_ * dq * erfc_a / ra;
    }
    double fx = f * dx, fy = f * dy, fz = f * dz;
    p->frc[3 * i] += fx;
    p->frc[3 * i + 1] += fy;
    p->frc[3 * i + 2] += fz;
    p->frc[3 * j] -= fx;
    p->frc[3 * j + 1] -= fy;
    p->frc[3 * j + 2] -= fz;
    double v[6] = {-fx * dx, -(fx * dy + fy * dx), -fy * dy, -(fx * dz + fz * dx), -(fy * dz + fz * dy), -fz * dz};
    if (p->e_atom_lj) p->e_atom_lj[i] += elj;
    if (p->e_atom_c) p->e_atom_c[i] += ec;
    if (p->vir_atom)
        for (int k = 0; k < 6; k++) p->vir_atom[6 * i + k] += v[k];
    p->t.e_lj += elj;
    p->t.e_coul += ec;
    for (int k = 0; k < 6; k++) p->t.vir[k] += v[k];
    p->t.pairs_in_cutoff++;
    p->dh[0] += dlj;
    p->dh[1] += dc;
}

/* prm = {lambda, alpha, p, sigma, sigma_min}; charge_ba may be NULL (no
 * charge perturbation).  totals = {E_lj, E_c, virial[6], dH_lj, dH_c}.
 * Returns the number of pairs inside rc. */
long long orc_soft_core_fp64(int n, const float* crd, const float* charge, const float* charge_ba,
                             const int* type_a, const int* type_b, const float* AA, const float* AB,
                             const float* BA, const float* BB, const float* prm, const float* cell, float cutoff,
                             float beta, const int* excl_start, const int* excl_numbers, const int* excl_list,
                             double* frc, double* e_atom_lj, double* e_atom_c, double* vir_atom, double* totals)
{
    double c[6], ri[6];
    cell_inverse_fp64(cell, c, ri);
    memset(frc, 0, sizeof(double) * 3 * (size_t)n);
    if (e_atom_lj) memset(e_atom_lj, 0, sizeof(double) * (size_t)n);
    if (e_atom_c) memset(e_atom_c, 0, sizeof(double) * (size_t)n);
    if (vir_atom) memset(vir_atom, 0, sizeof(double) * 6 * (size_t)n);
    soft_ctx p;
    memset(&p, 0, sizeof(p));
    p.crd = crd;
    p.charge = charge;
    p.charge_ba = charge_ba;
    p.AA = AA;
    p.AB = AB;
    p.BA = BA;
    p.BB = BB;
    p.ta = type_a;
    p.tb = type_b;
    p.c = c;
    p.ri = ri;
    p.rc = cutoff;
    p.beta = beta;
    double lam = prm[0], alpha = prm[1], pw = prm[2];
    p.l = lam;
    p.l_ = 1.0 - lam;
    p.alp_a = alpha * pow(lam, pw);
    p.alp_b = alpha * pow(1.0 - lam, pw);
    p.d_a = pw * alpha * (1.0 - lam) * pow(lam + 1.1754943508222875e-38, pw - 1.0) / 6.0;
    p.d_b = pw * alpha * lam * pow(1.0 - lam + 1.1754943508222875e-38, pw - 1.0) / 6.0;
    p.s6 = pow(prm[3], 6.0);
    p.s6min = pow(prm[4], 6.0);
    p.frc = frc;
    p.e_atom_lj = e_atom_lj;
    p.e_atom_c = e_atom_c;
    p.vir_atom = vir_atom;
    sweep_pairs(n, crd, c, ri, cutoff, excl_start, excl_numbers, excl_list, soft_pair, &p);
    totals[0] = p.t.e_lj;
    totals[1] = p.t.e_coul;
    for (int k = 0; k < 6; k++) totals[2 + k] = p.t.vir[k];
    totals[8] = p.dh[0];
    totals[9] = p.dh[1];
    return p.t.pairs_in_cutoff;
}

/* LJ_SOFT_CORE's long-range factors (LJ_soft_core.cpp:83-181, :605-635):
 * sum over ordered atom pairs (i == j included) of (1 - l) AB + l BB and of
 * BB - AB, times -2/3 pi / rc^3 / 6. */
void orc_soft_long_range(int n, const int* type_a, const int* type_b, const float* AB, const float* BB, float lambda,
                         float cutoff, double* factor, double* factor_ti)
{
    double s = 0.0, st = 0.0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
        {
            double ab = AB[lj_index(type_a[i], type_a[j])], bb = BB[lj_index(type_b[i], type_b[j])];
            s += (1.0 - lambda) * ab + lambda * bb;
            st += bb - ab;
        }
    double k = -2.0 / 3.0 * 3.14159265358979323846 / cutoff / cutoff / cutoff / 6.0;
    *factor = s * k;
    *factor_ti = st * k;
}

/* Tail correction.  factor = -2/3 pi sum_{i,j} B(type_i,type_j) / rc^3 / 6,
 * the sum running over all ordered atom pairs, i == j included, evaluated
 * through a type histogram; E_long = factor / V, virial diagonal += 2 factor / V. */
double orc_long_range_factor(int n, const int* type, int n_types, const float* B, float cutoff)
{
    double* hist = (double*)calloc((size_t)n_types, sizeof(double));
    for (int i = 0; i < n; i++) hist[type[i]] += 1.0;
    double s = 0.0;
    for (int a = 0; a < n_types; a++)
        for (int b = 0; b < n_types; b++) s += hist[a] * hist[b] * (double)B[lj_index(a, b)];
    free(hist);
    return s * (-2.0 / 3.0 * 3.14159265358979323846 / cutoff / cutoff / cutoff / 6.0);
}
