// Drop-in replacement for SPONGE/neighbor_list/neighbor_list.cpp.
//
// Keeps SPONGE's NEIGHBOR_LIST struct (neighbor_list/neighbor_list.h) and its
// public data contract -- d_nl / h_nl / d_temp in the ATOM_GROUP layout, the
// overflow flags, max_neighbor_numbers, the full list for many-body modules --
// and implements the methods over libspgnb (spgnb_nl_*).  Link this file, the
// other two shim files and libspgnb.so instead of neighbor_list.cpp,
// Lennard_Jones_force.cpp and solvent_LJ.cpp.
#include <map>
#include <mutex>

#include "neighbor_list/neighbor_list.h"
#include "spgnb_shim.h"

extern CONTROLLER controller;

namespace spgnb_shim
{
namespace
{
std::mutex g_mu;
std::map<const void*, spgnb_nl*>& registry()
{
    static std::map<const void*, spgnb_nl*> m;
    return m;
}
std::map<const NEIGHBOR_LIST*, spgnb_nl*>& owners()
{
    static std::map<const NEIGHBOR_LIST*, spgnb_nl*> m;
    return m;
}
}  // namespace

spgnb_nl* list_of(const ATOM_GROUP* d_nl)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = registry().find((const void*)d_nl);
    return it == registry().end() ? nullptr : it->second;
}

CONTROLLER* default_controller() { return &::controller; }

}  // namespace spgnb_shim

using spgnb_shim::ltm;
using spgnb_shim::raise;

static int read_int(CONTROLLER* c, const char* key, int def)
{
    if (!c->Command_Exist("neighbor_list", key)) return def;
    c->Check_Int("neighbor_list", key, "NEIGHBOR_LIST::Initial");
    return atoi(c->Command("neighbor_list", key));
}

static void attach_exports(NEIGHBOR_LIST* self, spgnb_nl* h, CONTROLLER* controller)
{
    spgnb_atom_group* dnl = nullptr;
    int* dtemp = nullptr;
    raise(controller, spgnb_nl_atom_groups(h, &dnl, &dtemp), "NEIGHBOR_LIST::Initial");
    self->d_nl = (ATOM_GROUP*)dnl;
    self->d_temp = dtemp;
    free(self->h_nl);
    self->h_nl = NULL;
    Malloc_Safely((void**)&self->h_nl, sizeof(ATOM_GROUP) * self->atom_numbers);
    for (int i = 0; i < self->atom_numbers; i++)
    {
        self->h_nl[i].atom_numbers = 0;
        self->h_nl[i].ghost_numbers = 0;
        self->h_nl[i].atom_serial = dtemp + (size_t)self->max_neighbor_numbers * i;
    }
    std::lock_guard<std::mutex> lk(spgnb_shim::g_mu);
    spgnb_shim::registry()[(const void*)dnl] = h;
    spgnb_shim::owners()[self] = h;
}

void NEIGHBOR_LIST::Initial(CONTROLLER* controller, int atom_numbers, float cutoff, float skin, LTMatrix3 cell,
                            LTMatrix3 rcell)
{
    this->atom_numbers = atom_numbers;
    this->cutoff = cutoff;
    this->skin = skin;
    controller->printf("START INITIALIZING NEIGHBOR LIST (spgnb):\n");
    spgnb_nl_options o;
    spgnb_nl_default_options(&o);
    throw_error_when_overflow = 0;
    if (controller->Command_Exist("neighbor_list", "throw_error_when_overflow"))
        throw_error_when_overflow =
            controller->Get_Bool("neighbor_list", "throw_error_when_overflow", "NEIGHBOR_LIST::Initial");
    o.throw_error_when_overflow = throw_error_when_overflow;
    o.max_neighbor_numbers = max_neighbor_numbers = read_int(controller, "max_neighbor_numbers", 1200);
    o.check_overflow_interval = check_overflow_interval = read_int(controller, "check_overflow_interval", 150);
    o.max_atom_in_grid_numbers = max_atom_in_grid_numbers = read_int(controller, "max_atom_in_grid_numbers", 150);
    o.max_ghost_in_grid_numbers = max_ghost_in_grid_numbers =
        read_int(controller, "max_ghost_in_grid_numbers", 150);
    o.refresh_interval = updator.refresh_interval = read_int(controller, "refresh_interval", 0);
    updator.skin_permit = 0.5f;
    if (o.refresh_interval <= 0 && controller->Command_Exist("neighbor_list", "skin_permit"))
    {
        controller->Check_Float("neighbor_list", "skin_permit", "NEIGHBOR_LIST::Initial");
        updator.skin_permit = atof(controller->Command("neighbor_list", "skin_permit"));
    }
    o.skin_permit = updator.skin_permit;
    o.export_atom_groups = 1;
    // spgnb's own key: the margin of the pruned list the force kernel walks
    // (re-pruned when an atom has moved half of it); 0 turns pruning off
    if (controller->Command_Exist("neighbor_list", "prune_buffer"))
    {
        controller->Check_Float("neighbor_list", "prune_buffer", "NEIGHBOR_LIST::Initial");
        o.prune_buffer = atof(controller->Command("neighbor_list", "prune_buffer"));
    }
    controller->printf("    Max number of neighbors for one atom: %d\n", max_neighbor_numbers);
    controller->printf("    The interval to refresh the neighbor list: %d\n", o.refresh_interval);
    spgnb_nl* h = nullptr;
    raise(controller, spgnb_nl_create(atom_numbers, cutoff, skin, ltm(cell), ltm(rcell), &o, &h),
          "NEIGHBOR_LIST::Initial");
    attach_exports(this, h, controller);
    spgnb_nl_stats st;
    if (spgnb_nl_get_stats(h, &st) == SPGNB_OK)
    {
        grids.Nx = st.grid_dims[0];
        grids.Ny = st.grid_dims[1];
        grids.Nz = st.grid_dims[2];
        grids.grid_numbers = st.grid_numbers;
        controller->printf("        Nx: %d        Ny: %d        Nz: %d\n", grids.Nx, grids.Ny, grids.Nz);
    }
    updator.time_recorder = controller->Get_Time_Recorder("neighbor searching");
    is_initialized = 1;
    if (this->is_needed_full)
    {
        controller->printf("    Initializing full neighbor list...\n");
        full_neighbor_list.Initial(atom_numbers, max_neighbor_numbers);
    }
    controller->printf("END INITIALIZING NEIGHBOR LIST\n\n");
}

void NEIGHBOR_LIST::Update(int* atom_local, int local_atom_numbers, int ghost_numbers, VECTOR* crd,
                           LTMatrix3 cell, LTMatrix3 rcell, int step, int update, int* excluded_list_start,
                           int* excluded_list, int* excluded_numbers)
{
    if (!is_initialized) return;
    if (local_atom_numbers <= 0 && ghost_numbers <= 0) return;
    spgnb_nl* h = nullptr;
    {
        std::lock_guard<std::mutex> lk(spgnb_shim::g_mu);
        h = spgnb_shim::owners()[this];
    }
    updator.time_recorder->Start();
    raise(spgnb_shim::default_controller(),
          spgnb_nl_update(h, atom_local, local_atom_numbers, ghost_numbers, (const spgnb_vector*)crd, ltm(cell),
                          ltm(rcell), step, update, excluded_list_start, excluded_list, excluded_numbers),
          "NEIGHBOR_LIST::Update");
    if (this->is_needed_full && full_neighbor_list.is_initialized)
    {
        // FULL_NEIGHBOR_LIST::Build_From_Half[_With_Cutoff], from the cluster
        // tables into the full list's own arrays
        raise(spgnb_shim::default_controller(),
              spgnb_nl_build_full(h, local_atom_numbers, (const spgnb_vector*)crd, ltm(cell), ltm(rcell),
                                  this->cutoff_full > 0.0f ? this->cutoff_full + skin : 0.0f,
                                  (spgnb_atom_group*)full_neighbor_list.d_nl, full_neighbor_list.max_neighbor_numbers,
                                  full_neighbor_list.d_overflow),
              "FULL_NEIGHBOR_LIST::Build_From_Half");
    }
    updator.time_recorder->Stop();
}

void NEIGHBOR_LIST::Check_Overflow(CONTROLLER* controller, int steps, const LTMatrix3 cell, const LTMatrix3 rcell,
                                   LTMatrix3* cell0)
{
    if (!is_initialized) return;
    spgnb_nl* h = nullptr;
    {
        std::lock_guard<std::mutex> lk(spgnb_shim::g_mu);
        h = spgnb_shim::owners()[this];
    }
    int reinit = 0;
    raise(controller, spgnb_nl_check_overflow(h, steps, ltm(cell), ltm(rcell), &reinit),
          "NEIGHBOR_LIST::Check_Overflow");
    if (reinit)
    {
        controller->printf("Overflow occured in neighbor searching; buffers regrown.\n");
        spgnb_nl_options o;
        spgnb_nl_default_options(&o);
        spgnb_atom_group* dnl = nullptr;
        int* dtemp = nullptr;
        spgnb_nl_atom_groups(h, &dnl, &dtemp);
        {
            std::lock_guard<std::mutex> lk(spgnb_shim::g_mu);
            for (auto it = spgnb_shim::registry().begin(); it != spgnb_shim::registry().end();)
                it = (it->second == h) ? spgnb_shim::registry().erase(it) : std::next(it);
        }
        // max_neighbor_numbers may have grown; re-read through the stats-free path
        if (dtemp != d_temp) max_neighbor_numbers = (int)(max_neighbor_numbers * 1.1);
        attach_exports(this, h, controller);
        if (cell0) cell0[0] = cell;
    }
}

void NEIGHBOR_LIST::Clear()
{
    if (!is_initialized) return;
    spgnb_nl* h = nullptr;
    {
        std::lock_guard<std::mutex> lk(spgnb_shim::g_mu);
        h = spgnb_shim::owners()[this];
        spgnb_shim::owners().erase(this);
        spgnb_shim::registry().erase((const void*)d_nl);
    }
    spgnb_nl_destroy(h);
    free(h_nl);
    h_nl = NULL;
    d_nl = NULL;
    d_temp = NULL;
    full_neighbor_list.Clear();
    is_initialized = 0;
}
