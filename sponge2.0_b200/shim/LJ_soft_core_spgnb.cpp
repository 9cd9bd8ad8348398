// Drop-in replacement for SPONGE/Lennard_Jones_force/LJ_soft_core.cpp.
//
// Keeps SPONGE's LJ_SOFT_CORE struct and the fields other modules read
// (types and tables with their host copies, lambda and the soft-core
// parameters, d_LJ_energy_atom, the long-range factors, the dH/dlambda
// results, crd_with_LJ_parameters_local) and evaluates the force and
// dH/dlambda over libspgnb's soft-core module (spgnb_lj_soft_*), which needs
// the list to be an spgnb list.  Over that list every pair of the system,
// water included, is evaluated by the force call: the solvent module's call
// returns at once.
#include <float.h>

#include <map>
#include <mutex>
#include <string>

#include "Lennard_Jones_force/LJ_soft_core.h"
#include "spgnb_shim.h"
#include "xponge/load/native/lj_soft.hpp"
#include "xponge/xponge.h"

using spgnb_shim::ltm;
using spgnb_shim::raise;

namespace
{
std::mutex g_mu;
std::map<const LJ_SOFT_CORE*, spgnb_lj_soft*>& handles()
{
    static std::map<const LJ_SOFT_CORE*, spgnb_lj_soft*> m;
    return m;
}
spgnb_lj_soft* handle_of(const LJ_SOFT_CORE* self)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = handles().find(self);
    return it == handles().end() ? nullptr : it->second;
}
float control_float(CONTROLLER* controller, const char* key, float fallback, const char* what)
{
    if (controller->Command_Exist(key))
    {
        const float v = atof(controller->Command(key));
        controller->printf("    FEP %s: %f\n", what, v);
        return v;
    }
    controller->printf("    FEP %s is set to default value %f\n", what, fallback);
    return fallback;
}
}  // namespace

spgnb_lj_soft* spgnb_shim::lj_soft_of(const void* lj_soft_core)
{
    return handle_of((const LJ_SOFT_CORE*)lj_soft_core);
}

// The packing kernels LJ_soft_core.h declares for other modules.
__global__ void Copy_LJ_Type_And_Mask_To_New_Crd(const int atom_numbers, VECTOR_LJ_SOFT_TYPE* new_crd,
                                                 const int* LJ_type_A, const int* LJ_type_B, const int* mask)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers)
    {
        new_crd[i].LJ_type = LJ_type_A[i];
        new_crd[i].LJ_type_B = LJ_type_B[i];
        new_crd[i].mask = mask[i];
    }
}

__global__ void Copy_Crd_And_Charge_To_New_Crd(const int atom_numbers, const VECTOR* crd,
                                               VECTOR_LJ_SOFT_TYPE* new_crd, const float* charge)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers)
    {
        new_crd[i].crd = crd[i];
        new_crd[i].charge = charge[i];
    }
}

__global__ void Copy_Crd_And_Charge_To_New_Crd(const int atom_numbers, const VECTOR* crd,
                                               VECTOR_LJ_SOFT_TYPE* new_crd, const float* charge,
                                               const float* charge_BA)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers)
    {
        new_crd[i].crd = crd[i];
        new_crd[i].charge = charge[i];
        new_crd[i].charge_BA = charge_BA[i];
    }
}

__global__ void Copy_Crd_To_New_Crd(const int atom_numbers, const VECTOR* crd, VECTOR_LJ_SOFT_TYPE* new_crd)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers) new_crd[i].crd = crd[i];
}

void LJ_SOFT_CORE::LJ_Soft_Core_Malloc()
{
    Malloc_Safely((void**)&h_LJ_energy_atom, sizeof(float) * atom_numbers);
    Malloc_Safely((void**)&h_atom_LJ_type_A, sizeof(int) * atom_numbers);
    Malloc_Safely((void**)&h_atom_LJ_type_B, sizeof(int) * atom_numbers);
    Malloc_Safely((void**)&h_LJ_AA, sizeof(float) * pair_type_numbers_A);
    Malloc_Safely((void**)&h_LJ_AB, sizeof(float) * pair_type_numbers_A);
    Malloc_Safely((void**)&h_LJ_BA, sizeof(float) * pair_type_numbers_B);
    Malloc_Safely((void**)&h_LJ_BB, sizeof(float) * pair_type_numbers_B);
    Malloc_Safely((void**)&h_subsys_division, sizeof(int) * atom_numbers);
    Malloc_Safely((void**)&h_sigma_of_dH_dlambda_lj, sizeof(float));
    Malloc_Safely((void**)&h_sigma_of_dH_dlambda_direct, sizeof(float));
    h_sigma_of_dH_dlambda_lj[0] = 0.0f;
    h_sigma_of_dH_dlambda_direct[0] = 0.0f;
}

void LJ_SOFT_CORE::Parameter_Host_To_Device()
{
    Device_Malloc_And_Copy_Safely((void**)&d_LJ_AA, h_LJ_AA, sizeof(float) * pair_type_numbers_A);
    Device_Malloc_And_Copy_Safely((void**)&d_LJ_AB, h_LJ_AB, sizeof(float) * pair_type_numbers_A);
    Device_Malloc_And_Copy_Safely((void**)&d_LJ_BA, h_LJ_BA, sizeof(float) * pair_type_numbers_B);
    Device_Malloc_And_Copy_Safely((void**)&d_LJ_BB, h_LJ_BB, sizeof(float) * pair_type_numbers_B);
    Device_Malloc_And_Copy_Safely((void**)&d_atom_LJ_type_A, h_atom_LJ_type_A, sizeof(int) * atom_numbers);
    Device_Malloc_And_Copy_Safely((void**)&d_atom_LJ_type_B, h_atom_LJ_type_B, sizeof(int) * atom_numbers);
    Device_Malloc_And_Copy_Safely((void**)&d_subsys_division, h_subsys_division, sizeof(int) * atom_numbers);
    Device_Malloc_Safely((void**)&crd_with_LJ_parameters_local, sizeof(VECTOR_LJ_SOFT_TYPE) * atom_numbers);
}

void LJ_SOFT_CORE::Initial(CONTROLLER* controller, float cutoff, char* module_name)
{
    strcpy(this->module_name, module_name == NULL ? "LJ_soft_core" : module_name);
    controller->printf("START INITIALIZING FEP SOFT CORE FOR LJ AND COULOMB (spgnb):\n");
    const Xponge::LJSoftCore* src = NULL;
    Xponge::LJSoftCore local_lj_soft;
    if (module_name == NULL)
        src = &Xponge::system.classical_force_field.lj_soft_core;
    else if (controller->Command_Exist(this->module_name, "in_file"))
    {
        Xponge::Native_Load_LJ_Soft_Core(&local_lj_soft, controller, this->module_name);
        src = &local_lj_soft;
    }
    if (src != NULL && src->atom_numbers > 0)
    {
        if (!controller->Command_Exist("lambda_lj"))
            controller->Throw_SPONGE_Error(spongeErrorMissingCommand, "LJ_SOFT_CORE::Initial",
                                           "Reason:\n\t'lambda_lj' is required for the calculation of "
                                           "LJ_soft_core\n");
        lambda = atof(controller->Command("lambda_lj"));
        controller->printf("    FEP lj lambda: %f\n", lambda);
        alpha = control_float(controller, "soft_core_alpha", 0.5f, "soft core alpha");
        p = control_float(controller, "soft_core_powfer", 1.0f, "soft core powfer");
        sigma = control_float(controller, "soft_core_sigma", 3.0f, "soft core sigma");
        sigma_min = control_float(controller, "soft_core_sigma_min", 0.0f, "soft core sigma min");
        atom_numbers = src->atom_numbers;
        atom_type_numbers_A = src->atom_type_numbers_A;
        atom_type_numbers_B = src->atom_type_numbers_B;
        pair_type_numbers_A = atom_type_numbers_A * (atom_type_numbers_A + 1) / 2;
        pair_type_numbers_B = atom_type_numbers_B * (atom_type_numbers_B + 1) / 2;
        LJ_Soft_Core_Malloc();
        for (int i = 0; i < pair_type_numbers_A; i++)
        {
            h_LJ_AA[i] = src->LJ_AA[i];
            h_LJ_AB[i] = src->LJ_AB[i];
        }
        for (int i = 0; i < pair_type_numbers_B; i++)
        {
            h_LJ_BA[i] = src->LJ_BA[i];
            h_LJ_BB[i] = src->LJ_BB[i];
        }
        for (int i = 0; i < atom_numbers; i++)
        {
            h_atom_LJ_type_A[i] = src->atom_LJ_type_A[i];
            h_atom_LJ_type_B[i] = src->atom_LJ_type_B[i];
            h_subsys_division[i] = src->subsystem_division.empty() ? 0 : src->subsystem_division[i];
        }
        Parameter_Host_To_Device();
        alpha_lambda_p = alpha * powf(lambda, p);
        alpha_lambda_p_ = alpha * powf(1 - lambda, p);
        sigma_6 = powf(sigma, 6);
        sigma_6_min = powf(sigma_min, 6);
        alpha_lambda_p_1 = alpha * powf(lambda, p - 1);
        alpha_lambda_p_1_ = alpha * powf(1.0 - lambda, p - 1);
        spgnb_soft_core_params prm;
        prm.lambda = lambda;
        prm.alpha = alpha;
        prm.p = p;
        prm.sigma = sigma;
        prm.sigma_min = sigma_min;
        spgnb_lj_soft* h = nullptr;
        raise(controller,
              spgnb_lj_soft_create(atom_numbers, atom_type_numbers_A, atom_type_numbers_B, h_atom_LJ_type_A,
                                   h_atom_LJ_type_B, h_LJ_AA, h_LJ_AB, h_LJ_BA, h_LJ_BB, &prm, cutoff, &h),
              "LJ_SOFT_CORE::Initial");
        raise(controller, spgnb_lj_soft_atom_lj_energy(h, &d_LJ_energy_atom), "LJ_SOFT_CORE::Initial");
        double f = 0, fti = 0;
        spgnb_lj_soft_long_range_factors(h, &f, &fti);
        long_range_factor = (float)f;
        long_range_factor_TI = (float)fti;
        int n_pert = 0;
        spgnb_lj_soft_perturbed_atoms(h, &n_pert, nullptr, 0);
        {
            std::lock_guard<std::mutex> lk(g_mu);
            handles()[this] = h;
        }
        this->cutoff = cutoff;
        controller->printf("    atom_numbers is %d, %d of them perturbed\n", atom_numbers, n_pert);
        controller->printf("    atom_LJ_type_number_A is %d, atom_LJ_type_number_B is %d\n", atom_type_numbers_A,
                           atom_type_numbers_B);
        controller->printf("        long range correction factor is: %e\n", long_range_factor);
        is_initialized = 1;
    }
    if (is_initialized && !is_controller_printf_initialized)
    {
        controller->Step_Print_Initial("LJ_soft", "%.2f");
        controller->Step_Print_Initial("LJ_soft_short", "%.2f");
        controller->Step_Print_Initial("LJ_soft_long", "%.2f");
        is_controller_printf_initialized = 1;
    }
    controller->printf("END INITIALIZING LENNADR JONES SOFT CORE INFORMATION\n\n");
}

void LJ_SOFT_CORE::Get_Local(int* atom_local, int local_atom_numbers, int ghost_numbers)
{
    if (!is_initialized) return;
    this->local_atom_numbers = local_atom_numbers;
    this->ghost_numbers = ghost_numbers;
    raise(spgnb_shim::default_controller(),
          spgnb_lj_soft_get_local(handle_of(this), atom_local, local_atom_numbers, ghost_numbers),
          "LJ_SOFT_CORE::Get_Local");
}

void LJ_SOFT_CORE::LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
    const int atom_numbers, const int local_atom_numbers, const int solvent_numbers, const int ghost_numbers,
    const VECTOR* crd, const float* charge, VECTOR* frc, const LTMatrix3 cell, const LTMatrix3 rcell,
    const ATOM_GROUP* nl, const float pme_beta, const int need_atom_energy, float* atom_energy,
    const int need_virial, LTMatrix3* atom_lj_virial, float* atom_direct_pme_energy)
{
    if (!is_initialized) return;
    CONTROLLER* c = spgnb_shim::default_controller();
    spgnb_nl* list = spgnb_shim::list_of(nl);
    if (!list)
        c->Throw_SPONGE_Error(spongeErrorNotImplemented,
                              "LJ_SOFT_CORE::LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial",
                              "the soft-core module evaluates over an spgnb neighbour list only");
    raise(c,
          spgnb_lj_soft_pme_direct_force(handle_of(this), atom_numbers, local_atom_numbers, solvent_numbers,
                                         ghost_numbers, (const spgnb_vector*)crd, charge, (spgnb_vector*)frc,
                                         ltm(cell), ltm(rcell), list, pme_beta, need_atom_energy, atom_energy,
                                         need_virial, (spgnb_ltmatrix3*)atom_lj_virial, atom_direct_pme_energy),
          "LJ_SOFT_CORE::LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial");
}

float LJ_SOFT_CORE::Get_Partial_H_Partial_Lambda_With_Columb_Direct(
    const int solvent_numbers, const VECTOR* crd, const LTMatrix3 cell, const LTMatrix3 rcell, const float* charge,
    const ATOM_GROUP* nl, const float* charge_B_A, const float pme_beta, const int charge_perturbated)
{
    if (!is_initialized) return NAN;
    CONTROLLER* c = spgnb_shim::default_controller();
    spgnb_nl* list = spgnb_shim::list_of(nl);
    if (!list)
        c->Throw_SPONGE_Error(spongeErrorNotImplemented, "LJ_SOFT_CORE::Get_Partial_H_Partial_Lambda_With_Columb_Direct",
                              "the soft-core module evaluates over an spgnb neighbour list only");
    double lj = 0, direct = 0;
    raise(c,
          spgnb_lj_soft_partial_h_partial_lambda(handle_of(this), solvent_numbers, (const spgnb_vector*)crd,
                                                 ltm(cell), ltm(rcell), charge, list, charge_B_A, pme_beta,
                                                 charge_perturbated, &lj, &direct),
          "LJ_SOFT_CORE::Get_Partial_H_Partial_Lambda_With_Columb_Direct");
    const float tail = long_range_factor_TI / cell.a11 / cell.a22 / cell.a33;
    h_sigma_of_dH_dlambda_lj[0] = (float)(lj - (double)tail);
    if (charge_perturbated) h_sigma_of_dH_dlambda_direct[0] = (float)direct;
    return (float)lj;
}

void LJ_SOFT_CORE::Step_Print(CONTROLLER* controller)
{
    if (!is_initialized || CONTROLLER::MPI_rank >= CONTROLLER::PP_MPI_size) return;
    double s = 0, l = 0, t = 0, d = 0;
    raise(controller, spgnb_lj_soft_energies(handle_of(this), &s, &l, &t, &d), "LJ_SOFT_CORE::Step_Print");
    h_LJ_energy_sum = (float)s;
    controller->Step_Print("LJ_soft_short", h_LJ_energy_sum);
    controller->Step_Print("LJ_soft_long", h_LJ_long_energy);
    controller->Step_Print("LJ_soft", h_LJ_energy_sum + h_LJ_long_energy, true);
}

void LJ_SOFT_CORE::Long_Range_Correction(int need_pressure, LTMatrix3* d_virial, int need_potential,
                                         float* d_potential, const float volume)
{
    if (!is_initialized || CONTROLLER::PP_MPI_rank != 0) return;
    raise(spgnb_shim::default_controller(),
          spgnb_lj_soft_long_range_correction(handle_of(this), need_pressure, (spgnb_ltmatrix3*)d_virial,
                                              need_potential, d_potential, volume),
          "LJ_SOFT_CORE::Long_Range_Correction");
    if (need_potential) h_LJ_long_energy = long_range_factor / volume;
}
