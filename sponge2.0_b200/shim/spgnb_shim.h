// Shared helpers of the SPONGE drop-in shim (compiled inside a SPONGE tree,
// against SPONGE's own headers).
#pragma once

#include "common.h"
#include "control.h"
#include "spgnb.h"

namespace spgnb_shim
{

// Maps an spgnb status to SPONGE's error numbers (utils/control/error.hpp:4-27)
// and raises it the way every SPONGE module reports a failure.
inline void raise(CONTROLLER* controller, int status, const char* where)
{
    if (status == SPGNB_OK) return;
    int code = spongeErrorSimulationBreakDown;
    switch (status)
    {
        case SPGNB_E_ARG:
            code = spongeErrorValueErrorCommand;
            break;
        case SPGNB_E_OOM:
            code = spongeErrorMallocFailed;
            break;
        case SPGNB_E_OVERFLOW:
            code = spongeErrorOverflow;
            break;
        case SPGNB_E_STATE:
            code = spongeErrorConflictingCommand;
            break;
        case SPGNB_E_UNSUPPORTED:
            code = spongeErrorNotImplemented;
            break;
        default:
            break;
    }
    controller->Throw_SPONGE_Error(code, where, spgnb_last_error());
}

inline spgnb_ltmatrix3 ltm(const LTMatrix3& m)
{
    spgnb_ltmatrix3 r;
    r.a11 = m.a11;
    r.a21 = m.a21;
    r.a22 = m.a22;
    r.a31 = m.a31;
    r.a32 = m.a32;
    r.a33 = m.a33;
    return r;
}

// The spgnb list whose exported ATOM_GROUP array is `d_nl`, or NULL when the
// array comes from elsewhere (defined in neighbor_list_spgnb.cpp).
spgnb_nl* list_of(const ATOM_GROUP* d_nl);

// The controller the shim reports errors through when a method has none.
CONTROLLER* default_controller();

// The spgnb module behind a LENNARD_JONES_INFORMATION (defined in
// Lennard_Jones_force_spgnb.cpp), NULL before its Initial.
spgnb_lj* lj_of(const void* lj_information);

// The spgnb soft-core module behind an LJ_SOFT_CORE (defined in
// LJ_soft_core_spgnb.cpp), NULL before its Initial.
spgnb_lj_soft* lj_soft_of(const void* lj_soft_core);

}  // namespace spgnb_shim
