// Reference harness -- TEST INFRASTRUCTURE ONLY.
//
// Plain C entry points over the reference's own module classes
// (NEIGHBOR_LIST, LENNARD_JONES_INFORMATION, SOLVENT_LENNARD_JONES,
// LJ_SOFT_CORE), compiled
// from the reference sources where they lie (oracle/Makefile).  The CPU build
// generates golden fixtures and is the timed CPU baseline; the CUDA build runs
// the reference's own kernels on a B200 for the reference-kernel parity check
// and the speed comparison.  The product never loads this library.
//
// The call sequence mirrors SPONGE/main.cpp: Main_Refresh_Local_State
// (FORCED_UPDATE, :571; lj.Get_Local, :581) and Main_Calculate_Force
// (CONDITIONAL_UPDATE, :307-311; LJ, :371-377; solvent LJ, :387-392).
#include <fcntl.h>
#include <unistd.h>

#include <chrono>
#include <vector>

#include "Lennard_Jones_force/LJ_soft_core.h"
#include "Lennard_Jones_force/Lennard_Jones_force.h"
#include "Lennard_Jones_force/solvent_LJ.h"
#include "common.h"
#include "control.h"
#include "neighbor_list/neighbor_list.h"
#include "xponge/xponge.h"
#ifdef REF_HARNESS_PME
#include "PM_force/PM_force.h"
#endif
#ifdef REF_HARNESS_MD
#include "MD_core/MD_core.h"
#include "MD_core/nve.hpp"
#include "constrain/constrain.h"
#include "constrain/settle.h"
#endif

CONTROLLER controller;
namespace Xponge
{
System system;
}

namespace
{
struct Quiet
{
    int saved = -1;
    Quiet()
    {
        fflush(stdout);
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        if (devnull >= 0)
        {
            dup2(devnull, 1);
            close(devnull);
        }
    }
    ~Quiet()
    {
        fflush(stdout);
        if (saved >= 0)
        {
            dup2(saved, 1);
            close(saved);
        }
    }
};

struct State
{
    int n = 0;
    int max_neighbor = 1200;
    float cutoff = 10.0f, skin = 2.0f;
    LTMatrix3 cell, rcell;
    NEIGHBOR_LIST* nl = nullptr;
    LENNARD_JONES_INFORMATION* lj = nullptr;
    SOLVENT_LENNARD_JONES* slj = nullptr;
    LJ_SOFT_CORE* lj_soft = nullptr;
    int* d_atom_local = nullptr;
    VECTOR* d_crd = nullptr;
    float* d_charge = nullptr;
    VECTOR* d_frc = nullptr;
    float* d_energy = nullptr;
    LTMatrix3* d_virial = nullptr;
    float* d_direct = nullptr;
    int *d_excl_start = nullptr, *d_excl_list = nullptr, *d_excl_num = nullptr;
    int* d_res_start = nullptr;
    float* d_charge_ba = nullptr;
    int res_numbers = 0;
    int solvent_atoms = 0;
} S;

template <typename T>
T* dev_alloc(size_t count)
{
    void* p = nullptr;
    Device_Malloc_Safely(&p, sizeof(T) * (count > 0 ? count : 1));
    return (T*)p;
}

template <typename T>
void to_dev(T* dst, const T* src, size_t count)
{
    if (count) deviceMemcpy(dst, src, sizeof(T) * count, deviceMemcpyHostToDevice);
}

template <typename T>
void to_host(T* dst, const T* src, size_t count)
{
    if (count) deviceMemcpy(dst, src, sizeof(T) * count, deviceMemcpyDeviceToHost);
}

LTMatrix3 ltm(const float* m) { return LTMatrix3(m[0], m[1], m[2], m[3], m[4], m[5]); }

void sync_device()
{
#ifdef USE_GPU
    cudaDeviceSynchronize();
#endif
}
}  // namespace

extern "C" {

int ref_is_gpu()
{
#ifdef USE_GPU
    return 1;
#else
    return 0;
#endif
}

void ref_set_threads(int threads)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
}

// Sets one control key (e.g. neighbor_list_max_atom_in_grid_numbers) for the
// modules the next ref_init creates; an empty value removes it.
void ref_set_key(const char* key, const char* value)
{
    if (value && value[0])
        controller.commands[key] = value;
    else
        controller.commands.erase(key);
}

// NEIGHBOR_LIST::Initial + LENNARD_JONES_INFORMATION::Initial + Get_Local
// (identity atom_local, one rank, no ghosts).  refresh_interval <= 0 selects
// the skin-triggered rebuild.
int ref_init(int n, int n_types, const int* types, const float* pair_A, const float* pair_B, float cutoff,
             float skin, const float* cell, const float* rcell, int max_neighbor, int refresh_interval,
             const int* excl_start, const int* excl_numbers, const int* excl_list, int n_excl)
{
    Quiet q;
    S.n = n;
    S.cutoff = cutoff;
    S.skin = skin;
    S.cell = ltm(cell);
    S.rcell = ltm(rcell);
    S.max_neighbor = max_neighbor;
    controller.commands["neighbor_list_max_neighbor_numbers"] = std::to_string(max_neighbor);
    if (refresh_interval > 0)
        controller.commands["neighbor_list_refresh_interval"] = std::to_string(refresh_interval);
    else
        controller.commands.erase("neighbor_list_refresh_interval");

    auto& lj = Xponge::system.classical_force_field.lj;
    int p = n_types * (n_types + 1) / 2;
    lj.atom_type.assign(types, types + n);
    lj.pair_A.assign(pair_A, pair_A + p);
    lj.pair_B.assign(pair_B, pair_B + p);
    lj.atom_type_numbers = n_types;

    S.nl = new NEIGHBOR_LIST();
    S.nl->Initial(&controller, n, cutoff, skin, S.cell, S.rcell);
    S.lj = new LENNARD_JONES_INFORMATION();
    S.lj->Initial(&controller, cutoff, NULL);

    std::vector<int> ident(n);
    for (int i = 0; i < n; i++) ident[i] = i;
    S.d_atom_local = dev_alloc<int>(n);
    to_dev(S.d_atom_local, ident.data(), n);
    S.d_crd = dev_alloc<VECTOR>(n);
    S.d_charge = dev_alloc<float>(n);
    S.d_frc = dev_alloc<VECTOR>(n);
    S.d_energy = dev_alloc<float>(n);
    S.d_virial = dev_alloc<LTMatrix3>(n);
    S.d_direct = dev_alloc<float>(n);
    S.d_excl_start = dev_alloc<int>(n);
    S.d_excl_num = dev_alloc<int>(n);
    S.d_excl_list = dev_alloc<int>(n_excl);
    to_dev(S.d_excl_start, excl_start, n);
    to_dev(S.d_excl_num, excl_numbers, n);
    to_dev(S.d_excl_list, excl_list, n_excl);
    S.lj->Get_Local(S.d_atom_local, n, 0);
    sync_device();
    return 0;
}

double ref_long_range_factor() { return S.lj ? (double)S.lj->long_range_factor : 0.0; }

// NEIGHBOR_LIST::Update with the step counter and the forced flag.
int ref_nl_update(const float* crd, int step, int forced)
{
    to_dev(S.d_crd, (const VECTOR*)crd, S.n);
    S.nl->Update(S.d_atom_local, S.n, 0, S.d_crd, S.cell, S.rcell, step,
                 forced ? NEIGHBOR_LIST::FORCED_UPDATE : NEIGHBOR_LIST::CONDITIONAL_UPDATE, S.d_excl_start,
                 S.d_excl_list, S.d_excl_num);
    sync_device();
    return 0;
}

// Copies the half list out: counts[n] always, lists when capacity suffices.
// Returns the total number of entries.
long long ref_nl_get(int* counts, int* lists, long long capacity, int* overflow_flags)
{
    std::vector<ATOM_GROUP> h(S.n);
    to_host(h.data(), S.nl->d_nl, S.n);
    long long total = 0;
    for (int i = 0; i < S.n; i++)
    {
        counts[i] = h[i].atom_numbers;
        total += h[i].atom_numbers;
    }
    if (lists && capacity >= total)
    {
        long long off = 0;
        for (int i = 0; i < S.n; i++)
        {
            int c = h[i].atom_numbers < S.max_neighbor ? h[i].atom_numbers : S.max_neighbor;
            to_host(lists + off, h[i].atom_serial, c);
            off += h[i].atom_numbers;
        }
    }
    if (overflow_flags)
    {
        overflow_flags[0] = overflow_flags[1] = 0;
        if (S.nl->d_neighbor_list_overflow) to_host(&overflow_flags[0], S.nl->d_neighbor_list_overflow, 1);
        if (S.nl->d_neighbor_grid_overflow) to_host(&overflow_flags[1], S.nl->d_neighbor_grid_overflow, 1);
    }
    return total;
}

// The water-residue module, configured the way SOLVENT_LENNARD_JONES::Initial
// and Get_Local leave it for a trailing run of 3- or 4-site waters
// (solvent_LJ.cpp:186-228, :469-482).  GPU build only: the reference disables
// the module on CPU builds (solvent_LJ.cpp:183-185).
int ref_enable_solvent(int res_numbers, const int* res_start, int first_water_residue, int solvent_atoms,
                       int water_points)
{
#if defined(USE_GPU) && !defined(REF_HARNESS_SHIM)
    S.lj_soft = new LJ_SOFT_CORE();
    S.slj = new SOLVENT_LENNARD_JONES();
    S.slj->lj_info = S.lj;
    S.slj->lj_soft_info = S.lj_soft;
    S.slj->water_points = water_points;
    S.slj->solvent_numbers = solvent_atoms;
    S.slj->solvent_start = first_water_residue;
    S.slj->solvent_start_local = first_water_residue;
    S.slj->local_solvent_numbers = solvent_atoms;
    S.slj->is_initialized = 1;
    S.res_numbers = res_numbers;
    S.d_res_start = dev_alloc<int>(res_numbers);
    to_dev(S.d_res_start, res_start, res_numbers);
    S.solvent_atoms = solvent_atoms;
    return 0;
#else
    (void)res_numbers;
    (void)res_start;
    (void)first_water_residue;
    (void)solvent_atoms;
    (void)water_points;
    return -1;
#endif
}

// One force evaluation.  Outputs are overwritten: the harness zeroes the
// accumulated arrays the way MD_core / DD do before the call.
int ref_force(const float* crd, const float* charge, float beta, int need_energy, int need_virial, float* frc,
              float* atom_energy, float* atom_virial, float* atom_direct, float* atom_lj)
{
    to_dev(S.d_crd, (const VECTOR*)crd, S.n);
    to_dev(S.d_charge, charge, S.n);
    deviceMemset(S.d_frc, 0, sizeof(VECTOR) * S.n);
    deviceMemset(S.d_energy, 0, sizeof(float) * S.n);
    deviceMemset(S.d_virial, 0, sizeof(LTMatrix3) * S.n);
    deviceMemset(S.d_direct, 0, sizeof(float) * S.n);
    int solvent = S.slj ? S.slj->local_solvent_numbers : 0;
    S.lj->LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(S.n, S.n, solvent, 0, S.d_crd, S.d_charge, S.d_frc,
                                                           S.cell, S.rcell, S.nl->d_nl, beta, need_energy,
                                                           S.d_energy, need_virial, S.d_virial, S.d_direct);
    if (S.slj)
        S.slj->LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(S.n, S.res_numbers, S.d_res_start, S.d_crd,
                                                                S.d_charge, S.d_frc, S.cell, S.rcell, S.nl->d_nl,
                                                                beta, need_energy, S.d_energy, need_virial,
                                                                S.d_virial, S.d_direct);
    sync_device();
    to_host((VECTOR*)frc, S.d_frc, S.n);
    if (atom_energy) to_host(atom_energy, S.d_energy, S.n);
    if (atom_virial) to_host((LTMatrix3*)atom_virial, S.d_virial, S.n);
    if (atom_direct) to_host(atom_direct, S.d_direct, S.n);
    if (atom_lj) to_host(atom_lj, S.lj->d_LJ_energy_atom, S.n);
    return 0;
}

// Timed loop of the path the way Main_Calculate_Force runs it: per step a
// conditional neighbour-list update then the LJ + PME-direct force (and the
// solvent module when enabled).  Coordinates and charges are uploaded once;
// the returned seconds cover only the loop.
double ref_time_steps(const float* crd, const float* charge, float beta, int first_step, int steps,
                      int need_energy, int need_virial)
{
    to_dev(S.d_crd, (const VECTOR*)crd, S.n);
    to_dev(S.d_charge, charge, S.n);
    int solvent = S.slj ? S.slj->local_solvent_numbers : 0;
    sync_device();
    auto t0 = std::chrono::steady_clock::now();
    {
        Quiet q;
        for (int s = first_step; s < first_step + steps; s++)
        {
            S.nl->Update(S.d_atom_local, S.n, 0, S.d_crd, S.cell, S.rcell, s, NEIGHBOR_LIST::CONDITIONAL_UPDATE,
                         S.d_excl_start, S.d_excl_list, S.d_excl_num);
            S.lj->LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
                S.n, S.n, solvent, 0, S.d_crd, S.d_charge, S.d_frc, S.cell, S.rcell, S.nl->d_nl, beta,
                need_energy, S.d_energy, need_virial, S.d_virial, S.d_direct);
            if (S.slj)
                S.slj->LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
                    S.n, S.res_numbers, S.d_res_start, S.d_crd, S.d_charge, S.d_frc, S.cell, S.rcell, S.nl->d_nl,
                    beta, need_energy, S.d_energy, need_virial, S.d_virial, S.d_direct);
        }
        sync_device();
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Times the two parts separately: a forced rebuild and a force-only step.
double ref_time_rebuild(const float* crd, int reps)
{
    to_dev(S.d_crd, (const VECTOR*)crd, S.n);
    sync_device();
    auto t0 = std::chrono::steady_clock::now();
    {
        Quiet q;
        for (int r = 0; r < reps; r++)
            S.nl->Update(S.d_atom_local, S.n, 0, S.d_crd, S.cell, S.rcell, 0, NEIGHBOR_LIST::FORCED_UPDATE,
                         S.d_excl_start, S.d_excl_list, S.d_excl_num);
        sync_device();
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count() / (reps > 0 ? reps : 1);
}

// LJ_SOFT_CORE::Initial (LJ_soft_core.cpp:438-641) from arrays given the way
// Xponge hands them over (Xponge::LJSoftCore, xponge/ir/forcefield.h:82-94),
// the control keys set from prm = {lambda_lj, soft_core_alpha,
// soft_core_powfer, soft_core_sigma, soft_core_sigma_min}, then Get_Local
// with the identity map.  ref_init must have run first (it owns the list).
int ref_soft_init(int n, int nA, int nB, const int* type_a, const int* type_b, const float* AA, const float* AB,
                  const float* BA, const float* BB, const float* prm, float cutoff)
{
    Quiet q;
    auto& ls = Xponge::system.classical_force_field.lj_soft_core;
    ls.atom_numbers = n;
    ls.atom_type_numbers_A = nA;
    ls.atom_type_numbers_B = nB;
    const int pa = nA * (nA + 1) / 2, pb = nB * (nB + 1) / 2;
    ls.LJ_AA.assign(AA, AA + pa);
    ls.LJ_AB.assign(AB, AB + pa);
    ls.LJ_BA.assign(BA, BA + pb);
    ls.LJ_BB.assign(BB, BB + pb);
    ls.atom_LJ_type_A.assign(type_a, type_a + n);
    ls.atom_LJ_type_B.assign(type_b, type_b + n);
    ls.subsystem_division.clear();
    const char* keys[5] = {"lambda_lj", "soft_core_alpha", "soft_core_powfer", "soft_core_sigma",
                           "soft_core_sigma_min"};
    for (int k = 0; k < 5; k++)
    {
        char buf[64];
        snprintf(buf, sizeof buf, "%.9g", prm[k]);
        controller.commands[keys[k]] = buf;
    }
    delete S.lj_soft;
    S.lj_soft = new LJ_SOFT_CORE();
    if (S.slj) S.slj->lj_soft_info = S.lj_soft;
    S.lj_soft->Initial(&controller, cutoff, NULL);
    if (!S.lj_soft->is_initialized) return -1;
    S.lj_soft->Get_Local(S.d_atom_local, n, 0);
#ifdef USE_GPU
    if (S.slj)
    {
        // An alchemical run has no plain LJ module (the system carries
        // LJ_soft_core only), so the solvent module takes its soft-core
        // branch (solvent_LJ.cpp:310-349), which reads the soft_to_hard_crd
        // buffer SOLVENT_LENNARD_JONES::Initial allocates when LJ_SOFT_CORE
        // is on (:220-225).
        S.lj->is_initialized = 0;
        S.slj->soft_to_hard_crd = dev_alloc<VECTOR_LJ>(n);
    }
#endif
    if (S.d_charge_ba) Free_Single_Device_Pointer((void**)&S.d_charge_ba);
    S.d_charge_ba = dev_alloc<float>(n);
    sync_device();
    return 0;
}

void ref_soft_long_range(double* factor, double* factor_ti)
{
    *factor = S.lj_soft ? (double)S.lj_soft->long_range_factor : 0.0;
    *factor_ti = S.lj_soft ? (double)S.lj_soft->long_range_factor_TI : 0.0;
}

// The soft-core force the way Main_Calculate_Force runs it in an alchemical
// run (main.cpp:379-392): LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial
// for the atoms before the water tail, then the solvent module for the waters
// when it is enabled (without it every atom owns its half list).  Outputs
// zeroed first as ref_force does.
static void soft_step(float beta, int need_energy, int need_virial)
{
    const int solvent = S.slj ? S.slj->local_solvent_numbers : 0;
    S.lj_soft->LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
        S.n, S.n, solvent, 0, S.d_crd, S.d_charge, S.d_frc, S.cell, S.rcell, S.nl->d_nl, beta, need_energy,
        S.d_energy, need_virial, S.d_virial, S.d_direct);
    if (S.slj)
        S.slj->LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(S.n, S.res_numbers, S.d_res_start, S.d_crd,
                                                                S.d_charge, S.d_frc, S.cell, S.rcell, S.nl->d_nl,
                                                                beta, need_energy, S.d_energy, need_virial,
                                                                S.d_virial, S.d_direct);
}

int ref_soft_force(const float* crd, const float* charge, float beta, int need_energy, int need_virial, float* frc,
                   float* atom_energy, float* atom_virial, float* atom_direct, float* atom_lj)
{
    to_dev(S.d_crd, (const VECTOR*)crd, S.n);
    to_dev(S.d_charge, charge, S.n);
    deviceMemset(S.d_frc, 0, sizeof(VECTOR) * S.n);
    deviceMemset(S.d_energy, 0, sizeof(float) * S.n);
    deviceMemset(S.d_virial, 0, sizeof(LTMatrix3) * S.n);
    deviceMemset(S.d_direct, 0, sizeof(float) * S.n);
    soft_step(beta, need_energy, need_virial);
    sync_device();
    to_host((VECTOR*)frc, S.d_frc, S.n);
    if (atom_energy) to_host(atom_energy, S.d_energy, S.n);
    if (atom_virial) to_host((LTMatrix3*)atom_virial, S.d_virial, S.n);
    if (atom_direct) to_host(atom_direct, S.d_direct, S.n);
    if (atom_lj) to_host(atom_lj, S.lj_soft->d_LJ_energy_atom, S.n);
    return 0;
}

// Get_Partial_H_Partial_Lambda_With_Columb_Direct (LJ_soft_core.cpp:786-846).
// Its kernel reads coordinates, charges and charge_BA from
// crd_with_LJ_parameters_local, but the method copies them into
// crd_with_parameters (:790-797): the local buffer keeps the coordinates and
// charges of the last force call and a charge_BA field nothing writes.  The
// harness writes the given crd, charge and charge_BA into the local buffer
// first, so the reference evaluates its formula at this state.  Returns the
// method's value (LJ part + long-range term); *direct = the direct-space
// Coulomb part it leaves in h_sigma_of_dH_dlambda_direct.
double ref_soft_dhdl(const float* crd, const float* charge, const float* charge_ba, float beta,
                     int charge_perturbated, double* direct)
{
    std::vector<VECTOR_LJ_SOFT_TYPE> h(S.n);
    to_host(h.data(), S.lj_soft->crd_with_LJ_parameters_local, S.n);
    for (int i = 0; i < S.n; i++)
    {
        h[i].crd = ((const VECTOR*)crd)[i];
        h[i].charge = charge[i];
        h[i].charge_BA = charge_ba ? charge_ba[i] : 0.0f;
    }
    to_dev(S.lj_soft->crd_with_LJ_parameters_local, h.data(), S.n);
    std::vector<float> cba(S.n, 0.0f);
    if (charge_ba) cba.assign(charge_ba, charge_ba + S.n);
    to_dev(S.d_charge_ba, cba.data(), S.n);
    to_dev(S.d_crd, (const VECTOR*)crd, S.n);
    to_dev(S.d_charge, charge, S.n);
    float r;
    {
        Quiet q;
        r = S.lj_soft->Get_Partial_H_Partial_Lambda_With_Columb_Direct(0, S.d_crd, S.cell, S.rcell, S.d_charge,
                                                                       S.nl->d_nl, S.d_charge_ba, beta,
                                                                       charge_perturbated);
    }
    if (direct) *direct = charge_perturbated ? (double)*S.lj_soft->h_sigma_of_dH_dlambda_direct : 0.0;
    return (double)r;
}

// Timed loop of the soft-core path: per step a conditional list update and
// soft_step.
double ref_soft_time_steps(const float* crd, const float* charge, float beta, int first_step, int steps,
                           int need_energy, int need_virial)
{
    to_dev(S.d_crd, (const VECTOR*)crd, S.n);
    to_dev(S.d_charge, charge, S.n);
    sync_device();
    auto t0 = std::chrono::steady_clock::now();
    {
        Quiet q;
        for (int s = first_step; s < first_step + steps; s++)
        {
            S.nl->Update(S.d_atom_local, S.n, 0, S.d_crd, S.cell, S.rcell, s, NEIGHBOR_LIST::CONDITIONAL_UPDATE,
                         S.d_excl_start, S.d_excl_list, S.d_excl_num);
            soft_step(beta, need_energy, need_virial);
        }
        sync_device();
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

void ref_clear()
{
    Quiet q;
    if (S.nl)
    {
        S.nl->Clear();
        delete S.nl;
        S.nl = nullptr;
    }
    delete S.lj;
    S.lj = nullptr;
    delete S.slj;
    S.slj = nullptr;
    delete S.lj_soft;
    S.lj_soft = nullptr;
    if (S.d_charge_ba) Free_Single_Device_Pointer((void**)&S.d_charge_ba);
    S.d_charge_ba = nullptr;
}

#ifdef REF_HARNESS_PME
// Particle_Mesh::PME_Excluded_Force_With_Atom_Energy (PM_force.cpp:918-1002),
// the reference's own kernel, on the system of the last ref_init: the
// method needs only the members set here (its reciprocal-space set-up is not
// run).  Outputs (overwritten): forces n x 3, per-atom energy n, per-atom
// virial n x 6; returns the correction's energy (sum of its per-atom record).
double ref_pme_excluded(const float* crd, const float* charge, float beta, int need_energy, float* frc,
                        float* atom_energy, float* atom_virial)
{
    static Particle_Mesh* pm = nullptr;
    if (!pm) pm = new Particle_Mesh();
    pm->is_initialized = 1;
    pm->calculate_excluded_part = true;
    pm->atom_numbers = S.n;
    pm->beta = beta;
    static float* d_corr = nullptr;
    static int corr_n = 0;
    if (corr_n < S.n)
    {
        if (d_corr) cudaFree(d_corr);
        d_corr = dev_alloc<float>(S.n);
        corr_n = S.n;
    }
    pm->d_correction_atom_energy = d_corr;
    to_dev(S.d_crd, (const VECTOR*)crd, S.n);
    to_dev(S.d_charge, charge, S.n);
    cudaMemset(S.d_frc, 0, sizeof(VECTOR) * S.n);
    cudaMemset(S.d_energy, 0, sizeof(float) * S.n);
    cudaMemset(S.d_virial, 0, sizeof(LTMatrix3) * S.n);
    cudaMemset(d_corr, 0, sizeof(float) * S.n);
    pm->PME_Excluded_Force_With_Atom_Energy(S.d_crd, S.cell, S.rcell, S.d_charge, S.d_excl_start, S.d_excl_list,
                                            S.d_excl_num, S.d_frc, need_energy, S.d_energy, S.d_virial);
    sync_device();
    to_host((VECTOR*)frc, S.d_frc, S.n);
    to_host(atom_energy, S.d_energy, S.n);
    to_host((LTMatrix3*)atom_virial, S.d_virial, S.n);
    std::vector<float> corr(S.n);
    to_host(corr.data(), d_corr, S.n);
    double e = 0;
    for (float v : corr) e += v;
    return e;
}
#endif

#ifdef REF_HARNESS_MD
namespace
{
struct MdState
{
    CONSTRAIN* con = nullptr;
    SETTLE* settle = nullptr;
    VECTOR* d_vel = nullptr;
    float* d_mass = nullptr;
    float* d_inv_mass = nullptr;
    int* d_local_id = nullptr;
    char* d_local_label = nullptr;
    float dt = 0.002f;
} M;
}  // namespace

// Rigid 3-site waters (O, H, H at water_first + 3k) constrained by the
// reference's SETTLE as SPONGE sets it up (settle.cpp:342-570) from the
// constraint pairs CONSTRAIN holds -- O-H, O-H, H-H with the reduced masses
// as constrain_k, x and v factors 1 (NVE leap-frog) -- on the system of the
// last ref_init, with a time step of dt_ps picoseconds.  Returns the number of
// SETTLE triangles.
int ref_md_init(const float* mass, int water_first, int n_waters, float d_oh, float d_hh, float dt_ps)
{
    Quiet q;
    // SPONGE's internal time unit (MD_core.cpp:133)
    const float dt = dt_ps * CONSTANT_TIME_CONVERTION;
    M.dt = dt;
    M.con = new CONSTRAIN();
    CONSTRAIN& c = *M.con;
    strcpy(c.module_name, "constrain");
    c.atom_numbers = S.n;
    c.dt = dt;
    c.dt_inverse = 1.0f / dt;
    c.v_factor = 1.0f;
    c.x_factor = 1.0f;
    c.constrain_pair_numbers = 3 * n_waters;
    Malloc_Safely((void**)&c.h_constrain_pair, sizeof(CONSTRAIN_PAIR) * (c.constrain_pair_numbers + 1));
    auto pair = [&](int k, int i, int j, float r) {
        CONSTRAIN_PAIR p;
        p.atom_i_serial = i;
        p.atom_j_serial = j;
        p.constant_r = r;
        p.constrain_k = mass[i] * mass[j] / (mass[i] + mass[j]);
        c.h_constrain_pair[k] = p;
    };
    for (int w = 0; w < n_waters; w++)
    {
        const int o = water_first + 3 * w;
        pair(3 * w, o, o + 1, d_oh);
        pair(3 * w + 1, o, o + 2, d_oh);
        pair(3 * w + 2, o + 1, o + 2, d_hh);
    }
    std::vector<float> h_mass(mass, mass + S.n);
    M.settle = new SETTLE();
    M.settle->Initial(&controller, M.con, h_mass.data());
    std::vector<int> id(S.n);
    for (int i = 0; i < S.n; i++) id[i] = i;
    std::vector<char> label(S.n, 1);
    std::vector<float> inv(S.n);
    for (int i = 0; i < S.n; i++) inv[i] = mass[i] > 0 ? 1.0f / mass[i] : 0.0f;
    M.d_local_id = dev_alloc<int>(S.n);
    M.d_local_label = dev_alloc<char>(S.n);
    M.d_vel = dev_alloc<VECTOR>(S.n);
    M.d_mass = dev_alloc<float>(S.n);
    M.d_inv_mass = dev_alloc<float>(S.n);
    to_dev(M.d_local_id, id.data(), S.n);
    to_dev(M.d_local_label, label.data(), S.n);
    to_dev(M.d_mass, h_mass.data(), S.n);
    to_dev(M.d_inv_mass, inv.data(), S.n);
    M.settle->Get_Local(M.d_local_id, M.d_local_label, S.n);
    sync_device();
    return M.settle->is_initialized ? M.settle->num_triangle_local : -1;
}

// `steps` NVE steps in Main_Iteration's order (main.cpp:622-710), each after
// Main_Calculate_Force's part of this path (main.cpp:307-397): the list
// update, the LJ (+ solvent) force with per-atom energies, then
// SETTLE::Remember_Last_Coordinates, the reference's leap-frog kernel
// (MD_core/nve.hpp) and SETTLE::Do_SETTLE.  energies[2 s] gets the LJ energy
// and energies[2 s + 1] the direct Coulomb energy at the positions of step s
// (before its integration); crd and vel are updated in place.
void ref_md_run(float* crd, float* vel, const float* charge, float beta, int first_step, int steps,
                double* energies)
{
    to_dev(S.d_crd, (const VECTOR*)crd, S.n);
    to_dev(S.d_charge, charge, S.n);
    to_dev(M.d_vel, (const VECTOR*)vel, S.n);
    int solvent = S.slj ? S.slj->local_solvent_numbers : 0;
    std::vector<float> e(S.n), d(S.n);
    {
        Quiet q;
        for (int s = first_step; s < first_step + steps; s++)
        {
            S.nl->Update(S.d_atom_local, S.n, 0, S.d_crd, S.cell, S.rcell, s, NEIGHBOR_LIST::CONDITIONAL_UPDATE,
                         S.d_excl_start, S.d_excl_list, S.d_excl_num);
            cudaMemset(S.d_frc, 0, sizeof(VECTOR) * S.n);
            cudaMemset(S.d_energy, 0, sizeof(float) * S.n);
            cudaMemset(S.d_virial, 0, sizeof(LTMatrix3) * S.n);
            S.lj->LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(S.n, S.n, solvent, 0, S.d_crd, S.d_charge, S.d_frc,
                                                                  S.cell, S.rcell, S.nl->d_nl, beta, 1, S.d_energy,
                                                                  0, S.d_virial, S.d_direct);
            if (S.slj)
                S.slj->LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
                    S.n, S.res_numbers, S.d_res_start, S.d_crd, S.d_charge, S.d_frc, S.cell, S.rcell, S.nl->d_nl,
                    beta, 1, S.d_energy, 0, S.d_virial, S.d_direct);
            to_host(e.data(), S.d_energy, S.n);
            to_host(d.data(), S.d_direct, S.n);
            double et = 0, ed = 0;
            for (int i = 0; i < S.n; i++)
            {
                et += e[i];
                ed += d[i];
            }
            energies[2 * (s - first_step)] = et - ed;
            energies[2 * (s - first_step) + 1] = ed;
            M.settle->Remember_Last_Coordinates(S.d_crd, S.cell, S.rcell);
            MD_Iteration_Leap_Frog<<<(S.n + 127) / 128, 128>>>(S.n, M.d_vel, S.d_crd, S.d_frc, M.d_inv_mass, M.dt);
            M.settle->Do_SETTLE(M.d_mass, S.d_crd, S.cell, S.rcell, M.d_vel, 0, nullptr);
        }
        sync_device();
    }
    to_host((VECTOR*)crd, S.d_crd, S.n);
    to_host((VECTOR*)vel, M.d_vel, S.n);
}
#endif

}  // extern "C"
