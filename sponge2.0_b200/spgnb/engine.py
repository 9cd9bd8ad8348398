"""The plain per-system path driven the way SPONGE's step loop drives it.

``PlainPath`` owns one system's device arrays and the three modules and runs
the hot-path part of ``Main_Calculate_Force`` (``SPONGE/main.cpp:307-397``):
conditional neighbour-list update, then the LJ + PME direct-space force (the
water pairs included), then the long-range correction.  ``SoftCorePath`` is
the same loop for a two-state (alchemical) system through LJ_SOFT_CORE, the
module ``main.cpp:379-385`` calls in place of the plain one.
"""
from __future__ import annotations

import numpy as np
import torch

from .modules import LENNARD_JONES_INFORMATION, LJ_SOFT_CORE, NEIGHBOR_LIST, SOLVENT_LENNARD_JONES


class PlainPath:
    def __init__(self, system, refresh_interval=20, export_atom_groups=False, solvent=True, device="cuda",
                 max_neighbor_numbers=1200):
        s = system
        self.system = s
        dev = torch.device(device)
        self.device = dev
        n = s.n
        self.n = n
        self.crd = torch.from_numpy(np.ascontiguousarray(s.crd)).to(dev)
        self.charge = torch.from_numpy(np.ascontiguousarray(s.charge)).to(dev)
        self.atom_local = torch.arange(n, dtype=torch.int32, device=dev)
        self.excl_start = torch.from_numpy(np.ascontiguousarray(s.excl_start, np.int32)).to(dev)
        self.excl_numbers = torch.from_numpy(np.ascontiguousarray(s.excl_numbers, np.int32)).to(dev)
        ex = s.excl_list if len(s.excl_list) else np.zeros(1, np.int32)
        self.excl_list = torch.from_numpy(np.ascontiguousarray(ex, np.int32)).to(dev)
        self.frc = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.atom_energy = torch.zeros(n, dtype=torch.float32, device=dev)
        self.atom_virial = torch.zeros((n, 6), dtype=torch.float32, device=dev)
        self.atom_direct = torch.zeros(n, dtype=torch.float32, device=dev)
        self.cell = s.cell
        self.rcell = s.rcell
        controller = {"neighbor_list_refresh_interval": refresh_interval,
                      "neighbor_list_max_neighbor_numbers": max_neighbor_numbers}
        self.nl = NEIGHBOR_LIST()
        self.nl.Initial(controller, n, s.cutoff, s.skin, s.cell, s.rcell, export_atom_groups=export_atom_groups)
        self.lj = LENNARD_JONES_INFORMATION()
        self.lj.Initial(controller, s.cutoff, s.atom_type, s.pair_A, s.pair_B, s.n_types)
        self.lj.Get_Local(self.atom_local, n, 0)
        self.solvent_numbers = 0
        self.solvent = SOLVENT_LENNARD_JONES()
        if solvent and s.n_waters > 0:
            self.solvent.Initial(controller, self.lj, s.water_points, default_enable=True)
            res_len = torch.from_numpy(np.ascontiguousarray(s.res_len, np.int32)).to(dev)
            mass = torch.from_numpy(np.ascontiguousarray(s.mass, np.float32)).to(dev)
            self.res_start = torch.from_numpy(np.ascontiguousarray(s.res_start, np.int32)).to(dev)
            self.solvent.Get_Local(len(s.res_len), res_len, n, mass)
            self.solvent_numbers = self.solvent.local_solvent_numbers
        self.update(0, forced=True)

    def update(self, step, forced=False, crd=None):
        self.nl.Update(self.atom_local, self.n, 0, self.crd if crd is None else crd, self.cell, self.rcell, step,
                       NEIGHBOR_LIST.FORCED_UPDATE if forced else NEIGHBOR_LIST.CONDITIONAL_UPDATE,
                       self.excl_start, self.excl_list, self.excl_numbers)

    def force(self, need_energy=False, need_virial=False, zero=True, crd=None, per_atom=True):
        if zero:
            self.frc.zero_()
            if need_energy:
                self.atom_energy.zero_()
            if need_virial:
                self.atom_virial.zero_()
        c = self.crd if crd is None else crd
        self.lj.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
            self.n, self.n, self.solvent_numbers, 0, c, self.charge, self.frc, self.cell, self.rcell, self.nl,
            self.system.beta, need_energy, self.atom_energy if per_atom else None, need_virial,
            self.atom_virial if per_atom else None, self.atom_direct if per_atom else None)
        if self.solvent.is_initialized:
            self.solvent.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
                self.n, len(self.system.res_len), self.res_start, c, self.charge, self.frc, self.cell, self.rcell,
                self.nl, self.system.beta, need_energy, self.atom_energy, need_virial, self.atom_virial,
                self.atom_direct)
        return self.frc

    def step(self, step, need_energy=False, need_virial=False, crd=None, per_atom=True):
        self.update(step, crd=crd)
        return self.force(need_energy, need_virial, crd=crd, per_atom=per_atom)


class SoftCorePath:
    """One two-state system (``spgnb.systems.FepSystem``) through
    NEIGHBOR_LIST + LJ_SOFT_CORE: every pair in one force call."""

    def __init__(self, fep, lam=None, refresh_interval=20, device="cuda", max_neighbor_numbers=1200):
        s = fep.system(lam)
        self.fep = fep
        self.system = s
        dev = torch.device(device)
        self.device = dev
        n = s.n
        self.n = n
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).to(dev)
        self.crd = t(s.crd, np.float32)
        self.charge = t(s.charge, np.float32)
        self.charge_ba = t(fep.charge_ba(), np.float32)
        self.atom_local = torch.arange(n, dtype=torch.int32, device=dev)
        self.excl_start = t(s.excl_start, np.int32)
        self.excl_numbers = t(s.excl_numbers, np.int32)
        self.excl_list = t(s.excl_list if len(s.excl_list) else np.zeros(1, np.int32), np.int32)
        self.frc = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.atom_energy = torch.zeros(n, dtype=torch.float32, device=dev)
        self.atom_virial = torch.zeros((n, 6), dtype=torch.float32, device=dev)
        self.atom_direct = torch.zeros(n, dtype=torch.float32, device=dev)
        self.cell = s.cell
        self.rcell = s.rcell
        controller = {"neighbor_list_refresh_interval": refresh_interval,
                      "neighbor_list_max_neighbor_numbers": max_neighbor_numbers}
        controller.update(fep.controller(lam))
        self.nl = NEIGHBOR_LIST()
        self.nl.Initial(controller, n, s.cutoff, s.skin, s.cell, s.rcell, export_atom_groups=False)
        self.lj = LJ_SOFT_CORE()
        self.lj.Initial(controller, s.cutoff, fep.type_a, fep.type_b, fep.AA, fep.AB, fep.BA, fep.BB,
                        fep.n_types_a, fep.n_types_b)
        self.lj.Get_Local(self.atom_local, n, 0)
        self.update(0, forced=True)

    def update(self, step, forced=False, crd=None):
        self.nl.Update(self.atom_local, self.n, 0, self.crd if crd is None else crd, self.cell, self.rcell, step,
                       NEIGHBOR_LIST.FORCED_UPDATE if forced else NEIGHBOR_LIST.CONDITIONAL_UPDATE,
                       self.excl_start, self.excl_list, self.excl_numbers)

    def force(self, need_energy=False, need_virial=False, zero=True, crd=None, per_atom=True):
        if zero:
            self.frc.zero_()
            if need_energy:
                self.atom_energy.zero_()
            if need_virial:
                self.atom_virial.zero_()
        c = self.crd if crd is None else crd
        self.lj.LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
            self.n, self.n, 0, 0, c, self.charge, self.frc, self.cell, self.rcell, self.nl, self.system.beta,
            need_energy, self.atom_energy if per_atom else None, need_virial,
            self.atom_virial if per_atom else None, self.atom_direct if per_atom else None)
        return self.frc

    def dhdl(self, charge_perturbated=True, crd=None):
        """(dH/dlambda of LJ with the long-range term, direct-space Coulomb part)."""
        c = self.crd if crd is None else crd
        v = self.lj.Get_Partial_H_Partial_Lambda_With_Columb_Direct(
            0, c, self.cell, self.rcell, self.charge, self.nl, self.charge_ba if charge_perturbated else None,
            self.system.beta, int(bool(charge_perturbated)))
        return v, self.lj.h_sigma_of_dH_dlambda_direct

    def step(self, step, need_energy=False, need_virial=False, crd=None, per_atom=True):
        self.update(step, crd=crd)
        return self.force(need_energy, need_virial, crd=crd, per_atom=per_atom)
