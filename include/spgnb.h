/*
 * spgnb -- B200 short-range nonbonded engine for SPONGE (C ABI).
 *
 * The Lennard-Jones + PME direct-space pair force/energy/virial over a Verlet
 * neighbour list, and the cell-list neighbour-list rebuild that feeds it.  The
 * entry points mirror SPONGE's module API one call for one call:
 *
 *   NEIGHBOR_LIST               SPONGE/neighbor_list/neighbor_list.h:7-128
 *   LENNARD_JONES_INFORMATION   SPONGE/Lennard_Jones_force/Lennard_Jones_force.h:86-173
 *   SOLVENT_LENNARD_JONES       SPONGE/Lennard_Jones_force/solvent_LJ.h:9-43
 *   LJ_SOFT_CORE                SPONGE/Lennard_Jones_force/LJ_soft_core.h:162-276
 *
 * Conventions (same as the reference):
 *   - coordinates, charges, forces, energies and virials are DEVICE pointers
 *     owned by the caller; tables passed at creation are host pointers;
 *   - frc, atom_energy and atom_virial are accumulated into (+=); the module's
 *     own per-atom LJ energy and atom_direct_pme_energy are zeroed by the
 *     callee when energy is requested (Lennard_Jones_force.cpp:376-382);
 *   - charges are pre-scaled by 18.2223, LJ tables are the internal A = 12*A_file,
 *     B = 6*B_file in triangular order max*(max+1)/2 + min;
 *   - the cell is SPONGE's lower-triangular LTMatrix3 (row vectors), rcell its
 *     inverse; any triclinic cell SPONGE accepts is accepted.
 * Unlike the reference, every call returns a status instead of aborting the
 * process; spgnb_last_error() holds the message of the last failure.
 *
 * All work is issued on the stream set with spgnb_set_stream (default: the
 * legacy stream, as the reference) and no call synchronises the device except
 * those documented as reading results back.
 */
#ifndef SPGNB_H
#define SPGNB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Layout-compatible with VECTOR (SPONGE/utils/vector.hpp:30-34). */
typedef struct
{
    float x, y, z;
} spgnb_vector;

/* Layout-compatible with LTMatrix3 (SPONGE/utils/vector.hpp:256-258). */
typedef struct
{
    float a11, a21, a22, a31, a32, a33;
} spgnb_ltmatrix3;

/* Layout-compatible with ATOM_GROUP (SPONGE/common.h:175-180): one half
 * neighbour list per local atom, atom_serial pointing into one slab. */
typedef struct
{
    int atom_numbers;
    int ghost_numbers;
    int* atom_serial;
} spgnb_atom_group;

enum
{
    SPGNB_OK = 0,
    SPGNB_E_ARG = 1,         /* invalid argument (maps to spongeErrorValueErrorCommand) */
    SPGNB_E_OOM = 2,         /* device allocation failed (spongeErrorMallocFailed) */
    SPGNB_E_CUDA = 3,        /* CUDA runtime error */
    SPGNB_E_OVERFLOW = 4,    /* a fixed-capacity buffer overflowed (spongeErrorOverflow) */
    SPGNB_E_NONFINITE = 5,   /* non-finite force or energy (spongeErrorSimulationBreakDown) */
    SPGNB_E_STATE = 6,       /* call out of order (e.g. force before the first list build) */
    SPGNB_E_TIMEOUT = 7,     /* a bounded device-side wait gave up */
    SPGNB_E_UNSUPPORTED = 8  /* configuration outside what this build implements */
};

const char* spgnb_version(void);
const char* spgnb_status_string(int status);
/* Message of the last failing call on this host thread. */
const char* spgnb_last_error(void);
/* Stream for all later launches issued by this host thread (a cudaStream_t). */
int spgnb_set_stream(void* cuda_stream);
/* Ewald beta from the direct-space tolerance: erfc(beta*rc)/rc == tol.
 * Replaces Get_Beta, SPONGE/PM_force/PM_force.cpp:244-272. */
float spgnb_get_beta(float cutoff, float tolerance);

/* ----------------------------------------------------------- NEIGHBOR_LIST */
typedef struct spgnb_nl spgnb_nl;

/* The [neighbor_list] control keys of NEIGHBOR_LIST::Initial
 * (neighbor_list.cpp:747-799, :134-160). */
typedef struct
{
    int max_neighbor_numbers;      /* neighbor_list_max_neighbor_numbers, 1200 */
    int max_atom_in_grid_numbers;  /* neighbor_list_max_atom_in_grid_numbers, 150 */
    int max_ghost_in_grid_numbers; /* neighbor_list_max_ghost_in_grid_numbers, 150 */
    int refresh_interval;          /* neighbor_list_refresh_interval, 0 = skin trigger */
    float skin_permit;             /* neighbor_list_skin_permit, 0.5 */
    int check_overflow_interval;   /* neighbor_list_check_overflow_interval, 150 */
    int throw_error_when_overflow; /* neighbor_list_throw_error_when_overflow, 0 */
    int export_atom_groups;        /* keep the ATOM_GROUP list (d_nl/d_temp) current, 1 */
    int max_entries_per_cluster;   /* capacity of the internal cluster-pair list per
                                      8-atom cluster; 0 = sized from the density */
    float prune_buffer;            /* the force call evaluates a pruned copy of the list
                                      holding the pairs within cutoff + prune_buffer (A),
                                      re-pruned on the device whenever an atom has moved
                                      more than prune_buffer/2 since the last pruning, so
                                      no pair within the cutoff is ever left out; 0 = off,
                                      1.0 by default (no reference counterpart: the
                                      reference evaluates the whole list each step) */
} spgnb_nl_options;

void spgnb_nl_default_options(spgnb_nl_options* opt);

/* NEIGHBOR_LIST::Initial (neighbor_list.h:17-18, neighbor_list.cpp:729-832).
 * Grid cells of (cutoff+skin)/2, at least 3 per box dimension. */
int spgnb_nl_create(int atom_numbers, float cutoff, float skin, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                    const spgnb_nl_options* opt, spgnb_nl** out);

enum
{
    SPGNB_CONDITIONAL_UPDATE = 0,
    SPGNB_FORCED_UPDATE = 1
};

/* NEIGHBOR_LIST::Update (neighbor_list.h:19-23, neighbor_list.cpp:834-885).
 * Rebuilds when update == FORCED, or refresh_interval > 0 and
 * (step+1) % refresh_interval == 0, or refresh_interval <= 0 and some atom
 * moved more than skin*skin_permit since the last build (decided on the
 * device, no host synchronisation).  The list holds every pair with
 * atom_local[j] > atom_local[i] whose FP32 minimum-image distance^2 is below
 * (cutoff+skin)^2, excluded pairs removed -- the reference's set, pair for
 * pair.  One rank: ghost_numbers must be 0. */
int spgnb_nl_update(spgnb_nl* nl, const int* d_atom_local, int local_atom_numbers, int ghost_numbers,
                    const spgnb_vector* d_crd, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, int step, int update,
                    const int* d_excluded_list_start, const int* d_excluded_list,
                    const int* d_excluded_numbers);

/* NEIGHBOR_LIST::Check_Overflow (neighbor_list.h:24-25, neighbor_list.cpp:887-965).
 * On steps where (steps+1) % check_overflow_interval == 0 reads the overflow
 * flags (synchronises); on overflow grows the buffers by 1.1x and sets
 * *reinitialized (or returns SPGNB_E_OVERFLOW when throw_error_when_overflow). */
int spgnb_nl_check_overflow(spgnb_nl* nl, int steps, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                            int* reinitialized);

/* The reference-layout list (NEIGHBOR_LIST::d_nl / d_temp, neighbor_list.cpp:764-773)
 * for other consumers: d_nl[i].atom_serial points at d_temp + i*max_neighbor_numbers.
 * Kept current on each rebuild when export_atom_groups is set. */
int spgnb_nl_atom_groups(spgnb_nl* nl, spgnb_atom_group** d_nl, int** d_temp);

/* Host copy of the reference-layout list (the reference keeps h_nl for the
 * same purpose): counts[local_atom_numbers] always, each atom's entries
 * back to back in lists[] when capacity (in ints) suffices.  Returns the
 * number of entries through *total.  Synchronises. */
int spgnb_nl_copy_atom_groups(spgnb_nl* nl, int* h_counts, int* h_lists, long long capacity, long long* total);

typedef struct
{
    int atom_numbers;
    int grid_numbers;
    int grid_dims[3];
    int clusters;           /* 8-atom clusters of the last build */
    long long entries;      /* cluster pairs with at least one listed pair */
    int work_items;
    long long builds;       /* rebuilds performed so far */
    int overflow;           /* bit 0 list, 1 grid, 2 cluster-pair list */
    long long full_list_words;  /* listed partners summed over atoms (each pair twice) */
    long long prunes;       /* prunings performed so far */
    long long pruned_list_words; /* partners in the pruned lists of the last pruning */
    long long device_bytes; /* device memory the list's arrays hold (capacities, not use) */
} spgnb_nl_stats;

/* Reads counters back (synchronises the stream). */
int spgnb_nl_get_stats(spgnb_nl* nl, spgnb_nl_stats* out);

/* NEIGHBOR_LIST::Clear (neighbor_list.h:26, neighbor_list.cpp:967-981). */
/* FULL_NEIGHBOR_LIST::Build_From_Half / Build_From_Half_With_Cutoff
 * (full_neighbor_list.cpp:27-147), called where NEIGHBOR_LIST::Update calls
 * them (neighbor_list.cpp:871-882): every pair of the current list in both
 * atoms' lists, written into the caller's ATOM_GROUP array (atom_serial
 * pointers set by the caller, max_neighbor_numbers entries each).  cutoff > 0
 * keeps the pairs within it at d_crd (the reference passes cutoff_full +
 * skin).  A list longer than max_neighbor_numbers gets its full count and
 * sets *d_overflow to 1.  Lists come in a fixed order (no atomics). */
int spgnb_nl_build_full(spgnb_nl* nl, int local_atom_numbers, const spgnb_vector* d_crd, spgnb_ltmatrix3 cell,
                        spgnb_ltmatrix3 rcell, float cutoff, spgnb_atom_group* d_full_nl, int max_neighbor_numbers,
                        int* d_overflow);

int spgnb_nl_destroy(spgnb_nl* nl);

/* ----------------------------------------------- LENNARD_JONES_INFORMATION */
typedef struct spgnb_lj spgnb_lj;

/* LENNARD_JONES_INFORMATION::Initial (Lennard_Jones_force.h:117-118,
 * Lennard_Jones_force.cpp:186-283): per-atom types and the internal pair
 * tables (host pointers).  Also evaluates the long-range factor
 * -2/3 pi sum_ij B_ij / rc^3 / 6 (Total_C6_Get, :146-184, :267-268) through a
 * type histogram instead of the O(N^2) double loop, same value. */
int spgnb_lj_create(int atom_numbers, int atom_type_numbers, const int* h_atom_type, const float* h_pair_A,
                    const float* h_pair_B, float cutoff, spgnb_lj** out);

/* LENNARD_JONES_INFORMATION::Get_Local (Lennard_Jones_force.h:134-135). */
int spgnb_lj_get_local(spgnb_lj* lj, const int* d_atom_local, int local_atom_numbers, int ghost_numbers);

/* LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial
 * (Lennard_Jones_force.h:138-144, Lennard_Jones_force.cpp:359-417) over the
 * spgnb neighbour list.  Per pair inside the cutoff:
 *   F/r = (B - A r^-6) r^-8 - q_i q_j r^-3 (erfc(beta r) + 2 beta r/sqrt(pi) e^-(beta r)^2),
 *   frc_i += F/r dr, frc_j -= F/r dr, dr = r_j - r_i.
 * Forces accumulate in int64 fixed point (2^-32 kcal/mol/A), so the result
 * does not depend on summation order.  The pair energy and virial go to the
 * pair's owner (the lower atom_local index, or for water sites when
 * solvent_numbers > 0 the residue's first atom, as solvent_LJ.cpp:124-143
 * does); totals are also reduced exactly and read with spgnb_lj_totals.
 * All pairs are evaluated in this call, water included: the solvent module's
 * call becomes a no-op (spgnb_solvent_pme_direct_force). */
int spgnb_lj_pme_direct_force(spgnb_lj* lj, int atom_numbers, int local_atom_numbers, int solvent_numbers,
                              int ghost_numbers, const spgnb_vector* d_crd, const float* d_charge,
                              spgnb_vector* d_frc, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                              const spgnb_nl* nl, float pme_beta, int need_atom_energy, float* d_atom_energy,
                              int need_virial, spgnb_ltmatrix3* d_atom_virial, float* d_atom_direct_pme_energy);

/* The same call over a reference-layout list produced by anyone (the exact
 * signature of the reference method): atoms [0, local_atom_numbers -
 * solvent_numbers) own their lists, the water tail is left to the solvent
 * module, exactly as the reference splits the work. */
int spgnb_lj_pme_direct_force_atom_groups(spgnb_lj* lj, int atom_numbers, int local_atom_numbers,
                                          int solvent_numbers, int ghost_numbers, const spgnb_vector* d_crd,
                                          const float* d_charge, spgnb_vector* d_frc, spgnb_ltmatrix3 cell,
                                          spgnb_ltmatrix3 rcell, const spgnb_atom_group* d_nl, float pme_beta,
                                          int need_atom_energy, float* d_atom_energy, int need_virial,
                                          spgnb_ltmatrix3* d_atom_virial, float* d_atom_direct_pme_energy);

/* LENNARD_JONES_INFORMATION::Long_Range_Correction (Lennard_Jones_force.h:168-170,
 * Lennard_Jones_force.cpp:320-341): adds 2*factor/V to the virial diagonal and
 * factor/V to the potential, element 0 only. */
int spgnb_lj_long_range_correction(spgnb_lj* lj, int need_pressure, spgnb_ltmatrix3* d_virial,
                                   int need_potential, float* d_potential, float volume);

/* Step_Print (Lennard_Jones_force.cpp:419-433): LJ_short, LJ_long, LJ of the
 * last energy step, plus the direct-space Coulomb energy.  Synchronises. */
int spgnb_lj_energies(spgnb_lj* lj, double* lj_short, double* lj_long, double* lj_total, double* direct_coulomb);

/* FP64 totals of the last force call: {E_lj, E_coulomb_direct, virial a11,
 * a21, a22, a31, a32, a33} (symmetrised off-diagonals, as the per-atom
 * virial).  Energy totals need need_atom_energy, the virial need_virial.
 * Synchronises. */
int spgnb_lj_totals(spgnb_lj* lj, double out[8]);

/* Long-range factor computed at creation (host value). */
double spgnb_lj_long_range_factor(const spgnb_lj* lj);

/* The module's per-atom LJ energy array (LENNARD_JONES_INFORMATION::
 * d_LJ_energy_atom, Lennard_Jones_force.h:111), filled on energy steps. */
int spgnb_lj_atom_lj_energy(spgnb_lj* lj, float** d_atom_lj_energy);

/* Writes n packed {x, y, z, LJ type, charge} records, the VECTOR_LJ layout of
 * Lennard_Jones_force.h:13-17 that other modules read as
 * crd_with_LJ_parameters_local (Copy_Crd_And_Charge_To_New_Crd, :17-27). */
int spgnb_lj_export_vector_lj(spgnb_lj* lj, const spgnb_vector* d_crd, const float* d_charge, void* d_vector_lj,
                              int n);

/* The PME excluded-pair correction, Particle_Mesh::PME_Excluded_Force_With_Atom_Energy
 * (PM_force.cpp:918-997): for every excluded pair (the exclusion CSR, upper
 * triangular) the smooth part q_i q_j erf(beta r)/r that reciprocal space
 * counted is taken back out.  Forces are added to d_frc (int64 fixed-point
 * accumulation, the same in any order), the per-atom energy to
 * d_atom_energy when need_energy, the per-atom virial to d_atom_virial when
 * it is not NULL.  The total of the last call: spgnb_lj_pme_excluded_energy
 * (synchronises). */
int spgnb_lj_pme_excluded_force(spgnb_lj* lj, int atom_numbers, const spgnb_vector* d_crd, spgnb_ltmatrix3 cell,
                                spgnb_ltmatrix3 rcell, const float* d_charge, float pme_beta,
                                const int* d_excluded_list_start, const int* d_excluded_list,
                                const int* d_excluded_numbers, spgnb_vector* d_frc, int need_energy,
                                float* d_atom_energy, spgnb_ltmatrix3* d_atom_virial);
int spgnb_lj_pme_excluded_energy(spgnb_lj* lj, double* energy);

/* The same correction fused into this module's pair pass: after this call
 * every spgnb_lj_pme_direct_force also applies PME_Excluded_Force_With_Atom_Energy
 * (PM_force.cpp:918-997) for these exclusions, in the pair kernel's warps
 * (each atom walks its excluded partners on both sides after its list), so
 * the caller drops its separate excluded-correction call.  Outputs as
 * spgnb_lj_pme_excluded_force: forces (+=), the correction's per-atom energy
 * (+= d_atom_energy) and per-atom virial (+= d_atom_virial) when the force
 * call asks for per-atom outputs, its energy total (spgnb_lj_pme_excluded_energy)
 * on energy calls.  The exclusion CSR (upper triangular, the indices of
 * d_crd) is read once here (synchronises) and turned into a symmetric one;
 * call again after it changes.  NULL lists switch the fused correction off. */
int spgnb_lj_fuse_pme_excluded(spgnb_lj* lj, int atom_numbers, const int* d_excluded_list_start,
                               const int* d_excluded_list, const int* d_excluded_numbers, int excluded_total);

int spgnb_lj_destroy(spgnb_lj* lj);

/* ------------------------------------------------------------ LJ_SOFT_CORE */
/* Alchemical (FEP) LJ + PME direct space with soft cores, LJ_SOFT_CORE
 * (LJ_soft_core.h:162-276, LJ_soft_core.cpp:198-436).  Every atom has a
 * state-A and a state-B LJ type, each state its own triangular pair tables
 * (AA, AB: state A's r^-12 and r^-6 coefficients; BA, BB: state B's).  Per
 * pair inside the cutoff (dr = r_j - r_i, lambda' = 1 - lambda):
 *   - when BA*AA != 0 or BA + AA == 0, the states are mixed linearly:
 *       F/r = lambda' LJ(r; AA, AB) + lambda LJ(r; BA, BB) - Coulomb(r);
 *   - otherwise (one state has no r^-12 term) each state is evaluated at its
 *     soft-core distance r_X = (r^6 + alpha lambda_X^p sigma_X)^(1/6),
 *     lambda_A = lambda, lambda_B = lambda', sigma_X = sigma^6 when the
 *     state's A or B is zero, else max(A / (2 B), sigma_min^6).
 * B200 layout: atoms whose pairs can differ between the states (a minimal
 * vertex cover of the pair-type combinations that differ, found at creation)
 * are the "perturbed" atoms.  The regular pruned-list pair kernel evaluates
 * every pair with the perturbed atoms given a null LJ type and no charge; a
 * warp per perturbed atom then walks the atom's cluster-table neighbours and
 * adds its pairs with the formula above, in int64 fixed point. */
typedef struct spgnb_lj_soft spgnb_lj_soft;

/* LJ_SOFT_CORE::Initial's parameters (LJ_soft_core.cpp:464-531):
 * lambda_lj, soft_core_alpha, soft_core_powfer, soft_core_sigma,
 * soft_core_sigma_min. */
typedef struct
{
    float lambda;     /* required */
    float alpha;      /* default 0.5 */
    float p;          /* default 1.0 */
    float sigma;      /* default 3.0 */
    float sigma_min;  /* default 0.0 */
} spgnb_soft_core_params;

void spgnb_lj_soft_default_params(spgnb_soft_core_params* prm);

/* LJ_SOFT_CORE::Initial (LJ_soft_core.cpp:438-641) from host arrays: per-atom
 * state-A / state-B types and the four triangular pair tables (index
 * hi*(hi+1)/2 + lo).  Also the long-range factors of Total_C6_Get and
 * Total_C6_B_A_Get (:83-181, :605-635), through a histogram of (type A, type
 * B) combinations instead of the O(N^2) loop.  At most 127 state-A types. */
int spgnb_lj_soft_create(int atom_numbers, int atom_type_numbers_A, int atom_type_numbers_B,
                         const int* h_atom_LJ_type_A, const int* h_atom_LJ_type_B, const float* h_LJ_AA,
                         const float* h_LJ_AB, const float* h_LJ_BA, const float* h_LJ_BB,
                         const spgnb_soft_core_params* prm, float cutoff, spgnb_lj_soft** out);

/* LJ_SOFT_CORE::Get_Local (LJ_soft_core.cpp:905-919).  Reads d_atom_local
 * back once (synchronises) to list the perturbed local atoms. */
int spgnb_lj_soft_get_local(spgnb_lj_soft* lj, const int* d_atom_local, int local_atom_numbers, int ghost_numbers);

/* LJ_SOFT_CORE::LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial
 * (LJ_soft_core.cpp:721-784) over the spgnb list, every pair of the system
 * (water included; no solvent-module call follows).  Same outputs and owner
 * rule as spgnb_lj_pme_direct_force; the module's per-atom LJ energy array
 * (spgnb_lj_soft_atom_lj_energy) is d_LJ_energy_atom. */
int spgnb_lj_soft_pme_direct_force(spgnb_lj_soft* lj, int atom_numbers, int local_atom_numbers,
                                   int solvent_numbers, int ghost_numbers, const spgnb_vector* d_crd,
                                   const float* d_charge, spgnb_vector* d_frc, spgnb_ltmatrix3 cell,
                                   spgnb_ltmatrix3 rcell, const spgnb_nl* nl, float pme_beta, int need_atom_energy,
                                   float* d_atom_energy, int need_virial, spgnb_ltmatrix3* d_atom_virial,
                                   float* d_atom_direct_pme_energy);

/* LJ_SOFT_CORE::Get_Partial_H_Partial_Lambda_With_Columb_Direct
 * (LJ_soft_core.cpp:786-846): dH/dlambda of the LJ part plus the long-range
 * term long_range_factor_TI / (a11 a22 a33) to *dh_dlambda, and, when
 * charge_perturbated, the direct-space Coulomb part to *dh_dlambda_direct
 * (d_charge_B_A = q_B - q_A per local atom; NULL when not perturbed).  Sums
 * are int64 fixed point.  Synchronises. */
int spgnb_lj_soft_partial_h_partial_lambda(spgnb_lj_soft* lj, int solvent_numbers, const spgnb_vector* d_crd,
                                           spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, const float* d_charge,
                                           const spgnb_nl* nl, const float* d_charge_B_A, float pme_beta,
                                           int charge_perturbated, double* dh_dlambda, double* dh_dlambda_direct);

/* LJ_SOFT_CORE::Long_Range_Correction (LJ_soft_core.cpp:872-889). */
int spgnb_lj_soft_long_range_correction(spgnb_lj_soft* lj, int need_pressure, spgnb_ltmatrix3* d_virial,
                                        int need_potential, float* d_potential, float volume);

/* Step_Print (LJ_soft_core.cpp:848-862): LJ_soft_short, LJ_soft_long,
 * LJ_soft, plus the direct-space Coulomb energy.  Synchronises. */
int spgnb_lj_soft_energies(spgnb_lj_soft* lj, double* lj_short, double* lj_long, double* lj_total,
                           double* direct_coulomb);

/* FP64 totals of the last force call, as spgnb_lj_totals. */
int spgnb_lj_soft_totals(spgnb_lj_soft* lj, double out[8]);

/* The long-range factors (long_range_factor, long_range_factor_TI). */
int spgnb_lj_soft_long_range_factors(const spgnb_lj_soft* lj, double* factor, double* factor_ti);

/* The module's per-atom LJ energy array (d_LJ_energy_atom). */
int spgnb_lj_soft_atom_lj_energy(spgnb_lj_soft* lj, float** d_atom_lj_energy);

/* The perturbed atoms (global indices, ascending): *count always, the
 * indices when capacity suffices. */
int spgnb_lj_soft_perturbed_atoms(const spgnb_lj_soft* lj, int* count, int* h_atoms, int capacity);

int spgnb_lj_soft_destroy(spgnb_lj_soft* lj);

/* --------------------------------------------------- SOLVENT_LENNARD_JONES */
typedef struct spgnb_solvent spgnb_solvent;

/* SOLVENT_LENNARD_JONES::Initial (solvent_LJ.h:23-25, solvent_LJ.cpp:148-247)
 * for a trailing run of water_points-site residues (3 or 4). */
int spgnb_solvent_create(spgnb_lj* lj, int water_points, spgnb_solvent** out);

/* SOLVENT_LENNARD_JONES::Get_Local (solvent_LJ.h:41-42, solvent_LJ.cpp:433-482):
 * counts the trailing water residues from residue lengths and masses (device
 * pointers) and returns the solvent atom count (synchronises, as the reference). */
int spgnb_solvent_get_local(spgnb_solvent* s, int local_res_numbers, const int* d_res_len, int atom_numbers,
                            const float* d_mass, int* local_solvent_numbers);

/* SOLVENT_LENNARD_JONES::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial
 * (solvent_LJ.h:26-32, solvent_LJ.cpp:255-431) over a reference-layout list:
 * water residues from d_res_start[solvent_start_local..residue_numbers), all
 * sites against the first site's list.  Over an spgnb list (nl != NULL) the
 * water pairs were already evaluated by spgnb_lj_pme_direct_force and this
 * call returns immediately. */
int spgnb_solvent_pme_direct_force(spgnb_solvent* s, int atom_numbers, int residue_numbers,
                                   const int* d_res_start, const spgnb_vector* d_crd, const float* d_charge,
                                   spgnb_vector* d_frc, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                                   const spgnb_nl* nl, const spgnb_atom_group* d_nl, float pme_beta,
                                   int need_atom_energy, float* d_atom_energy, int need_virial,
                                   spgnb_ltmatrix3* d_atom_virial, float* d_atom_direct_pme_energy);

/* The same module next to LJ_SOFT_CORE (an alchemical run has no plain LJ
 * module; solvent_LJ.cpp:310-349 takes the waters with the soft-core
 * module's state-A table): over an spgnb list the soft-core force call
 * evaluates the water pairs and this module's call returns at once. */
int spgnb_solvent_create_soft(spgnb_lj_soft* lj, int water_points, spgnb_solvent** out);

int spgnb_solvent_destroy(spgnb_solvent* s);

/* ------------------------------------------------ no-allocation force call */
/* No counterpart in the reference.  The force of
 * spgnb_lj_pme_direct_force_atom_groups (forces only, accumulated into d_frc)
 * for callers that cannot allocate device memory where they need the force:
 * a plugin hook inside the MD step (cudaMalloc would synchronise the device
 * and stall the work already queued) or a process whose device memory is
 * fixed in advance by an admission budget.  It creates nothing and allocates
 * nothing: its scratch is a fixed array inside the library (about 2.6 MB,
 * held by every GPU that loads the library until the process exits).
 * Limits: at most 65,536 local atoms and 64 LJ types (larger inputs return
 * SPGNB_E_ARG).  Inputs: per-local-atom LJ types (values in
 * [0, atom_type_numbers)), the triangular pair tables A = 12*A_file and
 * B = 6*B_file on the device, coordinates, charges, the reference-layout
 * list; owners are atoms [0, local_atom_numbers - solvent_numbers) as in the
 * reference's LJ call.  Like spgnb_lj_pme_direct_force, it takes one rank's
 * atoms only: ghost_numbers != 0 returns SPGNB_E_UNSUPPORTED.  A list entry
 * outside [0, local_atom_numbers) or a type outside [0, atom_type_numbers) is
 * a caller error: such an entry is skipped (a type is clamped into the
 * table), nothing is read out of bounds, and the forces of those pairs are
 * missing.  The pair evaluation adds each partner's force with one int64
 * atomic per pair and component: correct, but slower than the cluster-list
 * path.  All calls share the one scratch array and each call
 * clears what must start at zero; calls whose kernels overlap on the GPU race
 * on it, so serialise them.  The first call on a device looks up the array's
 * device address with that device current; make it before capturing any
 * stream on that device. */
int spgnb_lj_pme_direct_force_noalloc(int local_atom_numbers, int solvent_numbers, int ghost_numbers,
                                      int atom_type_numbers,
                                      const int* d_atom_type, const float* d_pair_A, const float* d_pair_B,
                                      const spgnb_vector* d_crd, const float* d_charge, spgnb_vector* d_frc,
                                      spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell, const spgnb_atom_group* d_nl,
                                      float cutoff, float pme_beta);

/* ----------------------------------------------------------------- BATCH */
/* Many independent periodic systems stepped together (no reference
 * counterpart: the reference runs one system per process).  Every system
 * keeps its own box, cutoff, skin, Ewald beta, exclusions and rigid waters,
 * and either the batch's LJ type table or one of its own (as each SPONGE
 * process reads its own LJ_in_file, Lennard_Jones_force.cpp:186-231).  One
 * step = one kernel for leap-frog (kick with F(t), drift), SETTLE for the
 * rigid waters, a Berendsen thermostat when on (the velocity scale from the
 * previous step's kinetic energy), the slot records of the force pass and
 * the rebuild decision (refresh interval, or the skin trigger of
 * NEIGHBOR_LIST::Update, per system); the list build and the pruning when
 * some system needs them; the LJ and PME direct-space forces of all systems
 * in one kernel.  Steps are replayed from captured CUDA graphs.  A system's
 * results do not depend on the other systems in the batch. */
typedef struct spgnb_batch spgnb_batch;

typedef struct
{
    int atom_numbers;
    float cutoff;                  /* LJ/PME direct-space cutoff (A) */
    float skin;                    /* neighbour-list skin (A) */
    float pme_beta;                /* Ewald beta (1/A) */
    spgnb_ltmatrix3 cell, rcell;   /* orthorhombic or triclinic box */
    const float* h_crd;            /* 3N, A */
    const float* h_vel;            /* 3N, A/ps, or NULL for zero */
    const float* h_charge;         /* N, scaled by the reference's charge factor */
    const float* h_mass;           /* N, g/mol (0 = fixed atom) */
    const int* h_atom_type;        /* N, index into the batch's type table */
    const int* h_excluded_start;   /* N, this system's exclusion CSR (local indices, j > i) */
    const int* h_excluded_numbers; /* N */
    const int* h_excluded_list;    /* excluded_total entries */
    int excluded_total;
    int water_begin;               /* rigid 3-site waters O,H,H from this local atom */
    int water_numbers;             /* how many */
    int atom_type_numbers;         /* > 0: this system's own LJ type table below, h_atom_type indexes it;
                                      0: the batch's table (h_pair_A / h_pair_B ignored) */
    const float* h_pair_A;         /* its pair_A / pair_B, the reference's triangular layout (x12 / x6) */
    const float* h_pair_B;
} spgnb_batch_system;

typedef struct
{
    float dt;                      /* ps, 0.002 by default */
    float water_doh, water_dhh;    /* rigid water geometry (A): 0.9572, 1.5139 */
    float skin_permit;             /* rebuild at skin * skin_permit displacement, 0.5 */
    float prune_buffer;            /* as spgnb_nl_options.prune_buffer, 1.0 */
    int steps_per_graph;           /* steps per captured graph, 10 */
    int use_graphs;                /* 1 = replay captured graphs, 0 = launch each step */
    float thermostat_tau;          /* Berendsen coupling time (ps) per system, 0 = off */
    float temperature;             /* its target (K), 300 */
    int refresh_interval;          /* > 0: rebuild every system's list every this many steps
                                      (neighbor_list_refresh_interval); 0: per-system skin trigger */
} spgnb_batch_options;

void spgnb_batch_default_options(spgnb_batch_options* opt);

/* Copies the systems to the device and builds their lists.  The batch's
 * type table (atom_type_numbers types, pair_A / pair_B in the reference's
 * triangular layout, already x12 / x6) serves every system that brings none
 * of its own; at most 128 types per table. */
int spgnb_batch_create(int n_systems, const spgnb_batch_system* systems, int atom_type_numbers,
                       const float* h_pair_A, const float* h_pair_B, const spgnb_batch_options* opt,
                       spgnb_batch** out);
/* Advances every system by `steps` steps; when energy_interval > 0, energies
 * and virials are evaluated on steps whose count is a multiple of it (the
 * last ones are kept).  Returns without synchronising. */
int spgnb_batch_run(spgnb_batch* b, int steps, int energy_interval);
/* Per system id, 9 doubles: LJ short-range, LJ long-range correction, PME
 * direct-space Coulomb (kcal/mol), virial a11 a21 a22 a31 a32 a33 of the
 * last energy evaluation.  Synchronises. */
int spgnb_batch_energies(spgnb_batch* b, double* out);
/* Coordinates, velocities and forces of system `sys` (3N floats each, NULL
 * to skip).  Synchronises. */
int spgnb_batch_download(spgnb_batch* b, int sys, float* h_crd, float* h_vel, float* h_frc);
/* Changes the per-system Berendsen thermostat (tau 0 = off) for later steps. */
int spgnb_batch_set_thermostat(spgnb_batch* b, float tau, float temperature);
/* Reads the overflow flags (synchronises); on overflow regrows the buffers,
 * rebuilds every list and sets *regrown. */
int spgnb_batch_check_overflow(spgnb_batch* b, int* regrown);
/* Steps done, list rebuilds (all systems), prunings, overflow flags. */
int spgnb_batch_stats(spgnb_batch* b, long long* steps, long long* rebuilds, long long* prunings, int* overflow);
/* Picks the launch configuration with the fastest step for this batch by
 * timing a few steps of each candidate, one setting after the other (the
 * systems advance meanwhile): the prune buffer (up to the one the lists were
 * sized for), the force kernel's resident blocks per SM, the pruning
 * kernel's blocks per SM and the steps per captured graph.  Results are the
 * same for every choice; only the time differs. */
int spgnb_batch_autotune(spgnb_batch* b, int steps_per_candidate, float* chosen_buffer);
typedef struct
{
    float prune_buffer;         /* A */
    int pair_blocks_per_sm;     /* force kernel, 0 = as many as are resident */
    int prune_blocks_per_sm;    /* pruning kernel */
    int steps_per_graph;
    float ms_per_step;          /* of the chosen configuration, 0 before any tuning */
} spgnb_batch_tuning;
/* The launch configuration in use (chosen by spgnb_batch_autotune). */
int spgnb_batch_get_tuning(spgnb_batch* b, spgnb_batch_tuning* in_use);
/* Applies a launch configuration (one saved from an earlier tuning, say);
 * the prune buffer at most the one the lists were sized for.  ms_per_step
 * is ignored. */
int spgnb_batch_set_tuning(spgnb_batch* b, const spgnb_batch_tuning* tuning);
/* Kernel launches of a replayed step: those every step runs (the step
 * kernel and the pair kernel), and those of the list build and the pruning
 * that follows it, the bodies of conditional graph nodes, which run only on
 * steps where some system rebuilds (the pruning alone, one kernel, on steps
 * where some system prunes). */
int spgnb_batch_launch_counts(spgnb_batch* b, int* per_step, int* per_rebuild);
/* The batch's CUDA stream (a cudaStream_t), for events around its work. */
void* spgnb_batch_stream(spgnb_batch* b);
int spgnb_batch_destroy(spgnb_batch* b);

/* ------------------------------------------------------ POOL (serving) */
/* A batch created empty with fixed capacities, into which systems are
 * admitted and from which they are retired while the others keep running
 * (continuous batching).  Every system owns ranges of the pool's arrays, so
 * admitting or retiring one changes nothing for the others: a system's
 * trajectory is bitwise the same alone and in any mix.  A system admitted
 * with a step count stops (its state frozen) after that many steps. */
typedef struct
{
    int max_systems;            /* system ids [0, max_systems) */
    int max_atoms;              /* 0: as many as hbm_budget_bytes allows */
    long long max_excluded;     /* exclusion entries; 0: 2 per atom */
    int max_waters;             /* 0: max_atoms / 3 */
    float max_cutoff;           /* largest cutoff admitted (list sizes), 12 */
    float min_cutoff;           /* smallest (cells per atom), 8 */
    float skin;                 /* 2 */
    float density;              /* atoms per A^3 of the systems admitted, 0.1003 */
    double hbm_budget_bytes;    /* device memory for the pool when max_atoms is 0 */
    int max_types;              /* most LJ types of an admitted system's own table; 0: the pool's table's */
    double type_table_bytes;    /* device memory for admitted systems' own tables (16 B x types^3 each),
                                   64 MiB */
} spgnb_batch_pool_options;

void spgnb_batch_pool_default_options(spgnb_batch_pool_options* opt);
int spgnb_batch_create_pool(const spgnb_batch_pool_options* pool, int atom_type_numbers, const float* h_pair_A,
                            const float* h_pair_B, const spgnb_batch_options* opt, spgnb_batch** out);
/* Copies a system in (stream-ordered after the work already queued) and
 * gives it an id; `steps` > 0 = the system stops after that many steps, 0 =
 * runs until retired.  Its lists, forces and energies at step 0 are made
 * before the next run.  SPGNB_E_OOM: no room now (nothing changed); a table
 * of its own with more than max_types types: SPGNB_E_UNSUPPORTED. */
int spgnb_batch_admit(spgnb_batch* b, const spgnb_batch_system* sys, int steps, int* id);
/* Returns a system's ranges to the pool (its results must have been read). */
int spgnb_batch_retire(spgnb_batch* b, int id);
/* Evaluates forces, energies and virial now for the listed systems only. */
int spgnb_batch_evaluate(spgnb_batch* b, const int* ids, int n);
/* Per system id (max_systems entries, NULL to skip): steps done and steps
 * left (-1 = unlimited; a retired id reads 0 and 0).  Synchronises. */
int spgnb_batch_progress(spgnb_batch* b, int* steps_done, int* steps_left);
/* Capacity: system ids, atoms in the pool and free now, device bytes held. */
int spgnb_batch_capacity(spgnb_batch* b, int* max_systems, long long* max_atoms, long long* free_atoms,
                         double* device_bytes);

/* ------------------------------------------------------------ diagnostics */
/* Measurement hooks for benchmarks and profiling only: no SPONGE module calls
 * these and nothing on the force path depends on them. */
/* Kernel launches issued by the library so far (all threads). */
unsigned long long spgnb_launch_count(void);
/* CUDA events (cudaEvent_t, or NULL to stop) recorded around every later
 * cluster-pair force kernel launched from this host thread. */
int spgnb_debug_set_pair_events(void* start_event, void* stop_event);
/* Listed pairs of the last build and those inside `cutoff` at d_crd
 * (synchronises; the inputs of the algorithmic work count). */
int spgnb_nl_count_pairs(spgnb_nl* nl, const spgnb_vector* d_crd, spgnb_ltmatrix3 cell, spgnb_ltmatrix3 rcell,
                         float cutoff, long long* listed, long long* in_cutoff);
/* FP32 fused-multiply-add throughput of this device in TFLOP/s (best of
 * `repeats` timed launches of independent FMA chains). */
int spgnb_probe_fp32_fma_tflops(int repeats, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* SPGNB_H */
