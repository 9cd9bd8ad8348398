// Drop-in replacement for SPONGE/Lennard_Jones_force/solvent_LJ.cpp.
//
// Same enable rule and water detection as the reference module
// (solvent_LJ.cpp:148-247): a trailing run of 3- or 4-site residues with
// masses O 16 +- 0.1 and H 1.008 +- 0.001, on by default in NVT/NPT with at
// least 10 update groups, or by the solvent_LJ key.  Over an spgnb list the
// water pairs are evaluated by the LJ module's call and this call returns;
// over a reference-layout list it runs the water-residue kernel.
#include <map>
#include <mutex>

#include "Lennard_Jones_force/solvent_LJ.h"
#include "spgnb_shim.h"

using spgnb_shim::ltm;
using spgnb_shim::raise;

namespace
{
std::mutex g_mu;
std::map<const SOLVENT_LENNARD_JONES*, spgnb_solvent*>& handles()
{
    static std::map<const SOLVENT_LENNARD_JONES*, spgnb_solvent*> m;
    return m;
}
spgnb_solvent* handle_of(const SOLVENT_LENNARD_JONES* self)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = handles().find(self);
    return it == handles().end() ? nullptr : it->second;
}
}  // namespace

void SOLVENT_LENNARD_JONES::Initial(CONTROLLER* controller, LENNARD_JONES_INFORMATION* lj, LJ_SOFT_CORE* lj_soft,
                                    MD_INFORMATION* md_info, bool default_enable, const char* module_name)
{
    strcpy(this->module_name, module_name == NULL ? "solvent_LJ" : module_name);
    bool enable;
    if (!controller->Command_Exist(this->module_name))
        enable = default_enable && (md_info->ug.ug_numbers >= 10);
    else
        enable = controller->Get_Bool(this->module_name, "SOLVENT_LENNARD_JONES::Initial");
    if (enable) water_points = md_info->ug.ug[md_info->ug.ug_numbers - 1].atom_numbers;
    if (water_points != 3 && water_points != 4) enable = false;
    // an alchemical run has the soft-core module instead of the plain one
    // (solvent_LJ.cpp:310-349): the waters go with it
    const bool soft = !lj->is_initialized && lj_soft->is_initialized;
    if (enable)
    {
        lj_info = lj;
        lj_soft_info = lj_soft;
        solvent_numbers = 0;
        solvent_start = md_info->ug.ug_numbers;
        for (int i = md_info->ug.ug_numbers - 1; i >= 0; i -= 1)
        {
            int n = md_info->ug.ug[i].atom_numbers;
            float mo = md_info->h_mass[md_info->ug.ug[i].atom_serial[0]];
            float m1 = md_info->h_mass[md_info->ug.ug[i].atom_serial[1]];
            float m2 = md_info->h_mass[md_info->ug.ug[i].atom_serial[2]];
            if (n == water_points && mo > 15.9f && mo < 16.1f && m1 > 1.007f && m1 < 1.009f && m2 > 1.007f &&
                m2 < 1.009f)
            {
                solvent_numbers += n;
                solvent_start -= 1;
            }
            else
                break;
        }
        controller->printf("    the solvent is %d-point, %d atoms from residue #%d (spgnb)\n", water_points,
                           solvent_numbers, solvent_start);
        if (solvent_numbers > 0)
        {
            spgnb_solvent* h = nullptr;
            raise(controller,
                  soft ? spgnb_solvent_create_soft(spgnb_shim::lj_soft_of(lj_soft), water_points, &h)
                       : spgnb_solvent_create(spgnb_shim::lj_of(lj), water_points, &h),
                  "SOLVENT_LENNARD_JONES::Initial");
            std::lock_guard<std::mutex> lk(g_mu);
            handles()[this] = h;
            is_initialized = 1;
        }
    }
    if (!is_initialized)
    {
        solvent_numbers = 0;
        local_solvent_numbers = 0;
        controller->printf("SOLVENT LJ IS NOT INITIALIZED\n\n");
    }
}

void SOLVENT_LENNARD_JONES::Get_Local(const int res_numbers, const int* d_res_len, const int atom_numbers,
                                      float* local_mass)
{
    if (!is_initialized) return;
    spgnb_solvent* h = handle_of(this);
    raise(spgnb_shim::default_controller(),
          spgnb_solvent_get_local(h, res_numbers, d_res_len, atom_numbers, local_mass, &local_solvent_numbers),
          "SOLVENT_LENNARD_JONES::Get_Local");
    solvent_start_local = res_numbers - local_solvent_numbers / water_points;
}

void SOLVENT_LENNARD_JONES::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
    const int atom_numbers, const int residue_numbers, const int* d_res_start, const VECTOR* crd,
    const float* charge, VECTOR* frc, const LTMatrix3 cell, const LTMatrix3 rcell, const ATOM_GROUP* nl,
    const float pme_beta, const int need_atom_energy, float* atom_energy, const int need_virial,
    LTMatrix3* atom_lj_virial, float* atom_direct_pme_energy)
{
    if (!is_initialized) return;
    spgnb_nl* list = spgnb_shim::list_of(nl);
    raise(spgnb_shim::default_controller(),
          spgnb_solvent_pme_direct_force(handle_of(this), atom_numbers, residue_numbers, d_res_start,
                                         (const spgnb_vector*)crd, charge, (spgnb_vector*)frc, ltm(cell), ltm(rcell),
                                         list, list ? nullptr : (const spgnb_atom_group*)nl, pme_beta,
                                         need_atom_energy, atom_energy, need_virial,
                                         (spgnb_ltmatrix3*)atom_lj_virial, atom_direct_pme_energy),
          "SOLVENT_LENNARD_JONES::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial");
}
