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
    orc_totals t;
    memset(&t, 0, sizeof(t));
    /* coarse cells of at least rc in every fractional direction */
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
    /* neighbour cells: +-1 (or every cell when a dimension has < 3) */
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
                        pair_fp64(i, j, crd, charge, type, A, B, c, ri, cutoff, beta, frc, e_atom_lj, e_atom_c,
                                  vir_atom, &t);
                    }
                }
    }
    free(cell_of);
    free(cstart);
    free(catoms);
    totals[0] = t.e_lj;
    totals[1] = t.e_coul;
    for (int k = 0; k < 6; k++) totals[2 + k] = t.vir[k];
    return t.pairs_in_cutoff;
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
