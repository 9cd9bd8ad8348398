"""SPONGE's module interface for the short-range nonbonded path, over libspgnb.

Same class names, method names, argument order and meaning as the reference
structs (``SPONGE/neighbor_list/neighbor_list.h:7-128``,
``SPONGE/Lennard_Jones_force/Lennard_Jones_force.h:86-173``,
``SPONGE/Lennard_Jones_force/solvent_LJ.h:9-43``,
``SPONGE/Lennard_Jones_force/LJ_soft_core.h:162-276``).  Device arrays are
``torch`` CUDA tensors (``crd``/``frc`` float32 (N,3), virials float32 (N,6));
control keys come from a dict shaped like ``CONTROLLER::commands``
(``"neighbor_list_refresh_interval"`` and so on, ``control.cpp:137-145``).
Errors raise :class:`SpgnbError` instead of aborting the process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import LTMatrix3, NLOptions, NLStats, SoftCoreParams, SpgnbError, check, lib


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise SpgnbError(1, "device arrays must be CUDA tensors")
    if not t.is_contiguous():
        raise SpgnbError(1, "device arrays must be contiguous")
    return t.data_ptr()


def _bind_stream():
    lib().spgnb_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))


def _controller_int(controller, key, default):
    v = (controller or {}).get(key)
    return default if v is None else int(v)


def _controller_float(controller, key, default):
    v = (controller or {}).get(key)
    return default if v is None else float(v)


def _controller_bool(controller, key, default):
    v = (controller or {}).get(key)
    if v is None:
        return default
    if isinstance(v, str):
        return v.strip().lower() in ("1", "true", "yes", "on")
    return bool(v)


class NEIGHBOR_LIST:
    CONDITIONAL_UPDATE = 0
    FORCED_UPDATE = 1

    def __init__(self):
        self.handle = None
        self.is_initialized = False

    def Initial(self, controller, atom_numbers, cutoff, skin, cell, rcell, export_atom_groups=True):
        """NEIGHBOR_LIST::Initial (neighbor_list.cpp:729-832)."""
        L = lib()
        opt = NLOptions()
        L.spgnb_nl_default_options(C.byref(opt))
        opt.max_neighbor_numbers = _controller_int(controller, "neighbor_list_max_neighbor_numbers", 1200)
        opt.max_atom_in_grid_numbers = _controller_int(controller, "neighbor_list_max_atom_in_grid_numbers", 150)
        opt.max_ghost_in_grid_numbers = _controller_int(controller, "neighbor_list_max_ghost_in_grid_numbers", 150)
        opt.refresh_interval = _controller_int(controller, "neighbor_list_refresh_interval", 0)
        opt.skin_permit = _controller_float(controller, "neighbor_list_skin_permit", 0.5)
        opt.check_overflow_interval = _controller_int(controller, "neighbor_list_check_overflow_interval", 150)
        opt.throw_error_when_overflow = int(_controller_bool(controller, "neighbor_list_throw_error_when_overflow",
                                                             False))
        opt.export_atom_groups = int(bool(export_atom_groups))
        opt.max_entries_per_cluster = _controller_int(controller, "neighbor_list_max_entries_per_cluster", 0)
        opt.prune_buffer = _controller_float(controller, "neighbor_list_prune_buffer", opt.prune_buffer)
        self.atom_numbers = int(atom_numbers)
        self.cutoff = float(cutoff)
        self.skin = float(skin)
        self.max_neighbor_numbers = opt.max_neighbor_numbers
        h = C.c_void_p()
        check(L.spgnb_nl_create(self.atom_numbers, self.cutoff, self.skin, LTMatrix3.of(cell), LTMatrix3.of(rcell),
                                C.byref(opt), C.byref(h)))
        self.handle = h
        self.is_initialized = True

    def Update(self, atom_local, local_atom_numbers, ghost_numbers, crd, cell, rcell, step, update,
               excluded_list_start=None, excluded_list=None, excluded_numbers=None):
        """NEIGHBOR_LIST::Update (neighbor_list.cpp:834-885)."""
        if not self.is_initialized:
            return
        _bind_stream()
        check(lib().spgnb_nl_update(self.handle, _ptr(atom_local), int(local_atom_numbers), int(ghost_numbers),
                                    _ptr(crd), LTMatrix3.of(cell), LTMatrix3.of(rcell), int(step), int(update),
                                    _ptr(excluded_list_start), _ptr(excluded_list), _ptr(excluded_numbers)))

    def Check_Overflow(self, controller, steps, cell, rcell, cell0=None):
        """NEIGHBOR_LIST::Check_Overflow (neighbor_list.cpp:887-965); True when re-initialised."""
        _bind_stream()
        r = C.c_int(0)
        check(lib().spgnb_nl_check_overflow(self.handle, int(steps), LTMatrix3.of(cell), LTMatrix3.of(rcell),
                                            C.byref(r)))
        if r.value and cell0 is not None:
            cell0[:] = cell
        return bool(r.value)

    @property
    def d_nl(self):
        """Device address of the ATOM_GROUP array (neighbor_list.h:43)."""
        p = C.c_void_p()
        t = C.c_void_p()
        check(lib().spgnb_nl_atom_groups(self.handle, C.byref(p), C.byref(t)))
        return p.value

    def host_atom_groups(self, sort=True):
        """(counts, lists) of the reference-layout list, lists sorted per atom."""
        _bind_stream()
        n = self.stats()["atom_numbers"]
        counts = np.zeros(n, np.int32)
        total = C.c_longlong(0)
        check(lib().spgnb_nl_copy_atom_groups(self.handle, counts.ctypes.data_as(C.c_void_p), None, 0,
                                              C.byref(total)))
        lists = np.zeros(max(total.value, 1), np.int32)
        check(lib().spgnb_nl_copy_atom_groups(self.handle, counts.ctypes.data_as(C.c_void_p),
                                              lists.ctypes.data_as(C.c_void_p), total.value, C.byref(total)))
        lists = lists[:total.value]
        if sort and total.value:
            owner = np.repeat(np.arange(n, dtype=np.int64), counts)
            order = np.lexsort((lists, owner))
            lists = lists[order]
        return counts, lists

    def stats(self):
        _bind_stream()
        s = NLStats()
        check(lib().spgnb_nl_get_stats(self.handle, C.byref(s)))
        return {"atom_numbers": s.atom_numbers, "grid_numbers": s.grid_numbers, "grid_dims": tuple(s.grid_dims),
                "clusters": s.clusters, "entries": s.entries, "work_items": s.work_items, "builds": s.builds,
                "overflow": s.overflow}

    def build_full(self, local_atom_numbers, crd, cell, rcell, cutoff_full, max_neighbor_numbers, out=None):
        """FULL_NEIGHBOR_LIST::Build_From_Half[_With_Cutoff] (full_neighbor_list.cpp:27-147):
        returns (counts, lists, overflow) device tensors, lists[i, :counts[i]]
        the partners of atom i; cutoff_full <= 0 keeps every listed pair.
        ``out`` = the (lists, groups, overflow) of an earlier call, reused."""
        _bind_stream()
        n, m = int(local_atom_numbers), int(max_neighbor_numbers)
        dev = crd.device
        if out is None:
            temp = torch.zeros((n, m), dtype=torch.int32, device=dev)
            groups = torch.zeros((n, 2), dtype=torch.int64, device=dev)  # {count, ghost}, atom_serial
            groups[:, 1] = temp.data_ptr() + 4 * m * torch.arange(n, dtype=torch.int64, device=dev)
            overflow = torch.zeros(1, dtype=torch.int32, device=dev)
        else:
            temp, groups, overflow = out
        self._full_out = (temp, groups, overflow)
        check(lib().spgnb_nl_build_full(self.handle, n, _ptr(crd), LTMatrix3.of(cell), LTMatrix3.of(rcell),
                                        float(cutoff_full), groups.data_ptr(), m, overflow.data_ptr()))
        counts = groups.view(torch.int32)[:, 0]
        return counts, temp, overflow

    def Clear(self):
        if self.handle is not None:
            lib().spgnb_nl_destroy(self.handle)
            self.handle = None
        self.is_initialized = False

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass


class LENNARD_JONES_INFORMATION:
    def __init__(self):
        self.handle = None
        self.is_initialized = False
        self.h_LJ_energy_sum = 0.0
        self.h_LJ_long_energy = 0.0

    def Initial(self, controller, cutoff, atom_type, pair_A, pair_B, atom_type_numbers, module_name=None):
        """LENNARD_JONES_INFORMATION::Initial (Lennard_Jones_force.cpp:186-283).

        The reference reads the tables from Xponge::system; here they are
        passed in the same internal convention (A*12, B*6, triangular order).
        """
        self.module_name = module_name or "LJ"
        atom_type = np.ascontiguousarray(atom_type, np.int32)
        pair_A = np.ascontiguousarray(pair_A, np.float32)
        pair_B = np.ascontiguousarray(pair_B, np.float32)
        self.atom_numbers = len(atom_type)
        self.atom_type_numbers = int(atom_type_numbers)
        self.cutoff = float(cutoff)
        h = C.c_void_p()
        check(lib().spgnb_lj_create(self.atom_numbers, self.atom_type_numbers, atom_type.ctypes.data_as(C.c_void_p),
                                    pair_A.ctypes.data_as(C.c_void_p), pair_B.ctypes.data_as(C.c_void_p),
                                    self.cutoff, C.byref(h)))
        self.handle = h
        self.long_range_factor = lib().spgnb_lj_long_range_factor(h)
        self.is_initialized = True

    def Get_Local(self, atom_local, local_atom_numbers, ghost_numbers):
        _bind_stream()
        check(lib().spgnb_lj_get_local(self.handle, _ptr(atom_local), int(local_atom_numbers), int(ghost_numbers)))

    def LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(self, atom_numbers, local_atom_numbers, solvent_numbers,
                                                         ghost_numbers, crd, charge, frc, cell, rcell, nl, pme_beta,
                                                         need_atom_energy, atom_energy, need_virial, atom_virial,
                                                         atom_direct_pme_energy):
        """Lennard_Jones_force.cpp:359-417.  ``nl`` is a NEIGHBOR_LIST (spgnb list)
        or the device address of a reference-layout ATOM_GROUP array."""
        _bind_stream()
        args = (self.handle, int(atom_numbers), int(local_atom_numbers), int(solvent_numbers), int(ghost_numbers),
                _ptr(crd), _ptr(charge), _ptr(frc), LTMatrix3.of(cell), LTMatrix3.of(rcell))
        tail = (float(pme_beta), int(need_atom_energy), _ptr(atom_energy), int(need_virial), _ptr(atom_virial),
                _ptr(atom_direct_pme_energy))
        if isinstance(nl, NEIGHBOR_LIST):
            check(lib().spgnb_lj_pme_direct_force(*args, nl.handle, *tail))
        else:
            check(lib().spgnb_lj_pme_direct_force_atom_groups(*args, int(nl), *tail))

    def Long_Range_Correction(self, need_pressure, d_virial, need_potential, d_potential, volume):
        _bind_stream()
        check(lib().spgnb_lj_long_range_correction(self.handle, int(need_pressure), _ptr(d_virial),
                                                   int(need_potential), _ptr(d_potential), float(volume)))

    def PME_Excluded_Force_With_Atom_Energy(self, atom_numbers, crd, cell, rcell, charge, pme_beta,
                                           excluded_list_start, excluded_list, excluded_numbers, frc,
                                           need_energy, atom_energy, atom_virial=None):
        """Particle_Mesh::PME_Excluded_Force_With_Atom_Energy (PM_force.cpp:918-997):
        the erf(beta r)/r part of every excluded pair taken back out of the
        forces (+=), per-atom energies (+=) and per-atom virials (+=)."""
        _bind_stream()
        check(lib().spgnb_lj_pme_excluded_force(self.handle, int(atom_numbers), _ptr(crd), LTMatrix3.of(cell),
                                                LTMatrix3.of(rcell), _ptr(charge), float(pme_beta),
                                                _ptr(excluded_list_start), _ptr(excluded_list),
                                                _ptr(excluded_numbers), _ptr(frc), int(need_energy),
                                                _ptr(atom_energy), _ptr(atom_virial)))

    def Fuse_PME_Excluded(self, atom_numbers, excluded_list_start, excluded_list, excluded_numbers,
                          excluded_total):
        """Applies the PME excluded-pair correction inside every later
        LJ_PME_Direct_Force_With_Atom_Energy_And_Virial call over an spgnb list
        (the separate PME_Excluded_Force_With_Atom_Energy call is then left
        out).  None lists switch it off."""
        _bind_stream()
        check(lib().spgnb_lj_fuse_pme_excluded(self.handle, int(atom_numbers), _ptr(excluded_list_start),
                                               _ptr(excluded_list), _ptr(excluded_numbers), int(excluded_total)))

    def excluded_energy(self):
        """FP64 total of the last excluded-pair correction."""
        _bind_stream()
        e = C.c_double()
        check(lib().spgnb_lj_pme_excluded_energy(self.handle, C.byref(e)))
        return e.value

    def totals(self):
        """FP64 totals of the last call: E_lj, E_coulomb_direct, virial (6)."""
        _bind_stream()
        out = (C.c_double * 8)()
        check(lib().spgnb_lj_totals(self.handle, out))
        return np.array(out[:], np.float64)

    def Step_Print(self, controller=None):
        """Lennard_Jones_force.cpp:419-433: LJ_short, LJ_long and LJ."""
        _bind_stream()
        s, l, t, d = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        check(lib().spgnb_lj_energies(self.handle, C.byref(s), C.byref(l), C.byref(t), C.byref(d)))
        self.h_LJ_energy_sum = s.value
        self.h_LJ_long_energy = l.value
        out = {"LJ_short": s.value, "LJ_long": l.value, "LJ": t.value}
        if controller is not None and hasattr(controller, "update"):
            controller.update({f"print_{k}": v for k, v in out.items()})
        return out

    def Clear(self):
        if self.handle is not None:
            lib().spgnb_lj_destroy(self.handle)
            self.handle = None
        self.is_initialized = False

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass


class SOLVENT_LENNARD_JONES:
    def __init__(self):
        self.handle = None
        self.is_initialized = False
        self.local_solvent_numbers = 0

    def Initial(self, controller, lj, water_points=3, default_enable=True, module_name=None):
        """SOLVENT_LENNARD_JONES::Initial (solvent_LJ.cpp:148-247).  Enabled by the
        ``solvent_LJ`` key when present, else by ``default_enable``."""
        key = module_name or "solvent_LJ"
        enable = _controller_bool(controller, key, default_enable)
        if not enable:
            return
        h = C.c_void_p()
        check(lib().spgnb_solvent_create(lj.handle, int(water_points), C.byref(h)))
        self.handle = h
        self.lj = lj
        self.water_points = int(water_points)
        self.is_initialized = True

    def Get_Local(self, res_numbers, d_res_len, atom_numbers, local_mass):
        if not self.is_initialized:
            return
        _bind_stream()
        out = C.c_int(0)
        check(lib().spgnb_solvent_get_local(self.handle, int(res_numbers), _ptr(d_res_len), int(atom_numbers),
                                            _ptr(local_mass), C.byref(out)))
        self.local_solvent_numbers = out.value

    def LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(self, atom_numbers, residue_numbers, d_res_start, crd,
                                                         charge, frc, cell, rcell, nl, pme_beta, need_atom_energy,
                                                         atom_energy, need_virial, atom_lj_virial,
                                                         atom_direct_pme_energy):
        if not self.is_initialized:
            return
        _bind_stream()
        spg = nl.handle if isinstance(nl, NEIGHBOR_LIST) else None
        groups = None if spg is not None else int(nl)
        check(lib().spgnb_solvent_pme_direct_force(self.handle, int(atom_numbers), int(residue_numbers),
                                                   _ptr(d_res_start), _ptr(crd), _ptr(charge), _ptr(frc),
                                                   LTMatrix3.of(cell), LTMatrix3.of(rcell), spg, groups,
                                                   float(pme_beta), int(need_atom_energy), _ptr(atom_energy),
                                                   int(need_virial), _ptr(atom_lj_virial),
                                                   _ptr(atom_direct_pme_energy)))

    def Clear(self):
        if self.handle is not None:
            lib().spgnb_solvent_destroy(self.handle)
            self.handle = None
        self.is_initialized = False


class LJ_SOFT_CORE:
    """Alchemical LJ + PME direct space with soft cores (LJ_soft_core.h:162-276)
    over the spgnb list: every pair of the system in one call, water included."""

    def __init__(self):
        self.handle = None
        self.is_initialized = False
        self.h_LJ_energy_sum = 0.0
        self.h_LJ_long_energy = 0.0
        self.h_sigma_of_dH_dlambda_direct = 0.0

    def Initial(self, controller, cutoff, atom_type_A, atom_type_B, LJ_AA, LJ_AB, LJ_BA, LJ_BB,
                atom_type_numbers_A, atom_type_numbers_B, module_name=None):
        """LJ_SOFT_CORE::Initial (LJ_soft_core.cpp:438-641).  ``lambda_lj`` is
        required; ``soft_core_alpha`` (0.5), ``soft_core_powfer`` (1.0),
        ``soft_core_sigma`` (3.0), ``soft_core_sigma_min`` (0.0) as the
        reference.  Tables in the internal convention (A*12, B*6, triangular)."""
        self.module_name = module_name or "LJ_soft_core"
        if (controller or {}).get("lambda_lj") is None:
            raise SpgnbError(1, "'lambda_lj' is required for the calculation of LJ_soft_core")
        prm = SoftCoreParams()
        lib().spgnb_lj_soft_default_params(C.byref(prm))
        prm.lambda_ = _controller_float(controller, "lambda_lj", 0.0)
        prm.alpha = _controller_float(controller, "soft_core_alpha", prm.alpha)
        prm.p = _controller_float(controller, "soft_core_powfer", prm.p)
        prm.sigma = _controller_float(controller, "soft_core_sigma", prm.sigma)
        prm.sigma_min = _controller_float(controller, "soft_core_sigma_min", prm.sigma_min)
        self.lambda_, self.alpha, self.p = prm.lambda_, prm.alpha, prm.p
        self.sigma, self.sigma_min = prm.sigma, prm.sigma_min
        ta = np.ascontiguousarray(atom_type_A, np.int32)
        tb = np.ascontiguousarray(atom_type_B, np.int32)
        arrs = [np.ascontiguousarray(a, np.float32) for a in (LJ_AA, LJ_AB, LJ_BA, LJ_BB)]
        self.atom_numbers = len(ta)
        self.cutoff = float(cutoff)
        h = C.c_void_p()
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        check(lib().spgnb_lj_soft_create(self.atom_numbers, int(atom_type_numbers_A), int(atom_type_numbers_B),
                                         ptr(ta), ptr(tb), *[ptr(a) for a in arrs], C.byref(prm), self.cutoff,
                                         C.byref(h)))
        self.handle = h
        f, fti = C.c_double(), C.c_double()
        check(lib().spgnb_lj_soft_long_range_factors(h, C.byref(f), C.byref(fti)))
        self.long_range_factor, self.long_range_factor_TI = f.value, fti.value
        self.is_initialized = True

    def Get_Local(self, atom_local, local_atom_numbers, ghost_numbers):
        """LJ_SOFT_CORE::Get_Local (LJ_soft_core.cpp:905-919)."""
        _bind_stream()
        check(lib().spgnb_lj_soft_get_local(self.handle, _ptr(atom_local), int(local_atom_numbers),
                                            int(ghost_numbers)))

    def LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(self, atom_numbers, local_atom_numbers,
                                                                   solvent_numbers, ghost_numbers, crd, charge, frc,
                                                                   cell, rcell, nl, pme_beta, need_atom_energy,
                                                                   atom_energy, need_virial, atom_lj_virial,
                                                                   atom_direct_pme_energy):
        """LJ_soft_core.cpp:721-784 over a NEIGHBOR_LIST."""
        if not self.is_initialized:
            return
        if not isinstance(nl, NEIGHBOR_LIST):
            raise SpgnbError(1, "the soft-core module evaluates over an spgnb NEIGHBOR_LIST")
        _bind_stream()
        check(lib().spgnb_lj_soft_pme_direct_force(self.handle, int(atom_numbers), int(local_atom_numbers),
                                                   int(solvent_numbers), int(ghost_numbers), _ptr(crd),
                                                   _ptr(charge), _ptr(frc), LTMatrix3.of(cell), LTMatrix3.of(rcell),
                                                   nl.handle, float(pme_beta), int(need_atom_energy),
                                                   _ptr(atom_energy), int(need_virial), _ptr(atom_lj_virial),
                                                   _ptr(atom_direct_pme_energy)))

    def Get_Partial_H_Partial_Lambda_With_Columb_Direct(self, solvent_numbers, crd, cell, rcell, charge, nl,
                                                        charge_B_A, pme_beta, charge_perturbated):
        """LJ_soft_core.cpp:786-846: dH/dlambda of LJ (+ the long-range term);
        the direct-space Coulomb part is left in h_sigma_of_dH_dlambda_direct."""
        if not self.is_initialized:
            return float("nan")
        _bind_stream()
        v, vd = C.c_double(), C.c_double()
        check(lib().spgnb_lj_soft_partial_h_partial_lambda(self.handle, int(solvent_numbers), _ptr(crd),
                                                           LTMatrix3.of(cell), LTMatrix3.of(rcell), _ptr(charge),
                                                           nl.handle, _ptr(charge_B_A), float(pme_beta),
                                                           int(charge_perturbated), C.byref(v), C.byref(vd)))
        self.h_sigma_of_dH_dlambda_direct = vd.value
        return v.value

    def Long_Range_Correction(self, need_pressure, d_virial, need_potential, d_potential, volume):
        _bind_stream()
        check(lib().spgnb_lj_soft_long_range_correction(self.handle, int(need_pressure), _ptr(d_virial),
                                                        int(need_potential), _ptr(d_potential), float(volume)))

    def totals(self):
        """FP64 totals of the last call: E_lj, E_coulomb_direct, virial (6)."""
        _bind_stream()
        out = (C.c_double * 8)()
        check(lib().spgnb_lj_soft_totals(self.handle, out))
        return np.array(out[:], np.float64)

    def perturbed_atoms(self):
        """Atoms whose pairs the two-state kernel evaluates (global indices)."""
        n = C.c_int()
        check(lib().spgnb_lj_soft_perturbed_atoms(self.handle, C.byref(n), None, 0))
        out = np.zeros(max(n.value, 1), np.int32)
        check(lib().spgnb_lj_soft_perturbed_atoms(self.handle, C.byref(n), out.ctypes.data_as(C.c_void_p), n.value))
        return out[:n.value]

    def Step_Print(self, controller=None):
        """LJ_soft_core.cpp:848-862: LJ_soft_short, LJ_soft_long and LJ_soft."""
        _bind_stream()
        s, l, t, d = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        check(lib().spgnb_lj_soft_energies(self.handle, C.byref(s), C.byref(l), C.byref(t), C.byref(d)))
        self.h_LJ_energy_sum = s.value
        self.h_LJ_long_energy = l.value
        out = {"LJ_soft_short": s.value, "LJ_soft_long": l.value, "LJ_soft": t.value}
        if controller is not None and hasattr(controller, "update"):
            controller.update({f"print_{k}": v for k, v in out.items()})
        return out

    def Clear(self):
        if self.handle is not None:
            lib().spgnb_lj_soft_destroy(self.handle)
            self.handle = None
        self.is_initialized = False

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass
