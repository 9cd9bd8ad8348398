// Drop-in replacement for SPONGE/Lennard_Jones_force/Lennard_Jones_force.cpp.
//
// Keeps SPONGE's LENNARD_JONES_INFORMATION struct and the fields other modules
// read (d_LJ_A/d_LJ_B/d_atom_LJ_type and their host copies,
// crd_with_LJ_parameters_local, d_LJ_energy_atom, cutoff, atom_type_numbers,
// long_range_factor) and evaluates the force over libspgnb: the cluster-pair
// kernel when the list is an spgnb list, the reference-layout kernel for a
// list produced by anyone else.
#include <map>
#include <mutex>

#include "Lennard_Jones_force/Lennard_Jones_force.h"
#include "spgnb_shim.h"
#include "xponge/load/native/lj.hpp"
#include "xponge/xponge.h"

using spgnb_shim::ltm;
using spgnb_shim::raise;

namespace
{
std::mutex g_mu;
std::map<const LENNARD_JONES_INFORMATION*, spgnb_lj*>& handles()
{
    static std::map<const LENNARD_JONES_INFORMATION*, spgnb_lj*> m;
    return m;
}
spgnb_lj* handle_of(const LENNARD_JONES_INFORMATION* self)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = handles().find(self);
    return it == handles().end() ? nullptr : it->second;
}
}  // namespace

spgnb_lj* spgnb_shim::lj_of(const void* lj_information)
{
    return handle_of((const LENNARD_JONES_INFORMATION*)lj_information);
}

// The packing kernels other modules (soft core, SITS) launch themselves;
// declared by Lennard_Jones_force.h.
__global__ void Copy_LJ_Type_To_New_Crd(const int atom_numbers, VECTOR_LJ* new_crd, const int* LJ_type)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers) new_crd[i].LJ_type = LJ_type[i];
}

__global__ void Copy_Crd_And_Charge_To_New_Crd(const int atom_numbers, const VECTOR* crd, VECTOR_LJ* new_crd,
                                               const float* charge)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers)
    {
        new_crd[i].crd = crd[i];
        new_crd[i].charge = charge[i];
    }
}

__global__ void Copy_Crd_To_New_Crd(const int atom_numbers, const VECTOR* crd, VECTOR_LJ* new_crd)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers) new_crd[i].crd = crd[i];
}

void LENNARD_JONES_INFORMATION::LJ_Malloc()
{
    Malloc_Safely((void**)&h_atom_LJ_type, sizeof(int) * atom_numbers);
    Malloc_Safely((void**)&h_LJ_A, sizeof(float) * pair_type_numbers);
    Malloc_Safely((void**)&h_LJ_B, sizeof(float) * pair_type_numbers);
    Malloc_Safely((void**)&h_LJ_energy_atom, sizeof(float) * atom_numbers);
}

void LENNARD_JONES_INFORMATION::Parameter_Host_To_Device()
{
    Device_Malloc_And_Copy_Safely((void**)&d_atom_LJ_type, h_atom_LJ_type, sizeof(int) * atom_numbers);
    Device_Malloc_And_Copy_Safely((void**)&d_LJ_A, h_LJ_A, sizeof(float) * pair_type_numbers);
    Device_Malloc_And_Copy_Safely((void**)&d_LJ_B, h_LJ_B, sizeof(float) * pair_type_numbers);
    Device_Malloc_Safely((void**)&d_LJ_energy_sum, sizeof(float));
    Device_Malloc_Safely((void**)&crd_with_LJ_parameters_local, sizeof(VECTOR_LJ) * atom_numbers);
}

void LENNARD_JONES_INFORMATION::Initial(CONTROLLER* controller, float cutoff, const char* module_name)
{
    strcpy(this->module_name, module_name == NULL ? "LJ" : module_name);
    controller->printf("START INITIALIZING LENNADR JONES INFORMATION (spgnb):\n");
    const Xponge::LennardJones* src = NULL;
    Xponge::LennardJones local_lj;
    if (module_name == NULL)
        src = &Xponge::system.classical_force_field.lj;
    else if (controller->Command_Exist(this->module_name, "in_file"))
    {
        Xponge::Native_Load_LJ(&local_lj, controller, 0, this->module_name);
        src = &local_lj;
    }
    if (src != NULL)
    {
        atom_numbers = (int)src->atom_type.size();
        atom_type_numbers = src->atom_type_numbers;
    }
    if (atom_numbers > 0)
    {
        pair_type_numbers = atom_type_numbers * (atom_type_numbers + 1) / 2;
        LJ_Malloc();
        for (int i = 0; i < pair_type_numbers; i++)
        {
            h_LJ_A[i] = src->pair_A[i];
            h_LJ_B[i] = src->pair_B[i];
        }
        for (int i = 0; i < atom_numbers; i++) h_atom_LJ_type[i] = src->atom_type[i];
        Parameter_Host_To_Device();
        spgnb_lj* h = nullptr;
        raise(controller,
              spgnb_lj_create(atom_numbers, atom_type_numbers, h_atom_LJ_type, h_LJ_A, h_LJ_B, cutoff, &h),
              "LENNARD_JONES_INFORMATION::Initial");
        raise(controller, spgnb_lj_atom_lj_energy(h, &d_LJ_energy_atom), "LENNARD_JONES_INFORMATION::Initial");
        {
            std::lock_guard<std::mutex> lk(g_mu);
            handles()[this] = h;
        }
        this->cutoff = cutoff;
        long_range_factor = (float)spgnb_lj_long_range_factor(h);
        controller->printf("    atom_numbers is %d\n    atom_LJ_type_number is %d\n", atom_numbers,
                           atom_type_numbers);
        controller->printf("        long range correction factor is: %e\n", long_range_factor);
        is_initialized = 1;
    }
    if (is_initialized && !is_controller_printf_initialized)
    {
        controller->Step_Print_Initial("LJ_short", "%.2f");
        controller->Step_Print_Initial("LJ_long", "%.2f");
        controller->Step_Print_Initial("LJ", "%.2f");
        is_controller_printf_initialized = 1;
    }
    controller->printf("END INITIALIZING LENNADR JONES INFORMATION\n\n");
}

void LENNARD_JONES_INFORMATION::Get_Local(int* atom_local, int local_atom_numbers, int ghost_numbers)
{
    if (!is_initialized) return;
    this->local_atom_numbers = local_atom_numbers;
    this->ghost_numbers = ghost_numbers;
    raise(spgnb_shim::default_controller(),
          spgnb_lj_get_local(handle_of(this), atom_local, local_atom_numbers, ghost_numbers),
          "LENNARD_JONES_INFORMATION::Get_Local");
}

void LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
    const int atom_numbers, const int local_atom_numbers, const int solvent_numbers, const int ghost_numbers,
    const VECTOR* crd, const float* charge, VECTOR* frc, const LTMatrix3 cell, const LTMatrix3 rcell,
    const ATOM_GROUP* nl, const float pme_beta, const int need_atom_energy, float* atom_energy, const int need_virial,
    LTMatrix3* atom_virial, float* atom_direct_pme_energy)
{
    if (!is_initialized) return;
    spgnb_lj* h = handle_of(this);
    CONTROLLER* c = spgnb_shim::default_controller();
    // other modules read the packed records (soft core, SITS)
    raise(c, spgnb_lj_export_vector_lj(h, (const spgnb_vector*)crd, charge, crd_with_LJ_parameters_local,
                                       this->local_atom_numbers + this->ghost_numbers),
          "LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial");
    if (atom_numbers == 0 || local_atom_numbers == 0) return;
    spgnb_nl* list = spgnb_shim::list_of(nl);
    int st;
    if (list)
        st = spgnb_lj_pme_direct_force(h, atom_numbers, local_atom_numbers, solvent_numbers, ghost_numbers,
                                       (const spgnb_vector*)crd, charge, (spgnb_vector*)frc, ltm(cell), ltm(rcell),
                                       list, pme_beta, need_atom_energy, atom_energy, need_virial,
                                       (spgnb_ltmatrix3*)atom_virial, atom_direct_pme_energy);
    else
        st = spgnb_lj_pme_direct_force_atom_groups(
            h, atom_numbers, local_atom_numbers, solvent_numbers, ghost_numbers, (const spgnb_vector*)crd, charge,
            (spgnb_vector*)frc, ltm(cell), ltm(rcell), (const spgnb_atom_group*)nl, pme_beta, need_atom_energy,
            atom_energy, need_virial, (spgnb_ltmatrix3*)atom_virial, atom_direct_pme_energy);
    raise(c, st, "LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial");
}

void LENNARD_JONES_INFORMATION::Long_Range_Correction(int need_pressure, LTMatrix3* d_virial, int need_potential,
                                                      float* d_potential, const float volume)
{
    if (!is_initialized || CONTROLLER::PP_MPI_rank != 0) return;
    raise(spgnb_shim::default_controller(),
          spgnb_lj_long_range_correction(handle_of(this), need_pressure, (spgnb_ltmatrix3*)d_virial, need_potential,
                                         d_potential, volume),
          "LENNARD_JONES_INFORMATION::Long_Range_Correction");
    if (need_potential) h_LJ_long_energy = long_range_factor / volume;
}

void LENNARD_JONES_INFORMATION::Step_Print(CONTROLLER* controller)
{
    if (!is_initialized || CONTROLLER::MPI_rank >= CONTROLLER::PP_MPI_size) return;
    double s = 0, l = 0, t = 0, d = 0;
    raise(controller, spgnb_lj_energies(handle_of(this), &s, &l, &t, &d), "LENNARD_JONES_INFORMATION::Step_Print");
    h_LJ_energy_sum = (float)s;
    controller->Step_Print("LJ_short", h_LJ_energy_sum);
    controller->Step_Print("LJ_long", h_LJ_long_energy);
    controller->Step_Print("LJ", h_LJ_energy_sum + h_LJ_long_energy, true);
}
