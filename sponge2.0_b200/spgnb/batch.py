"""Batched engine: many independent systems stepped together on one GPU.

``Batch`` wraps the ``spgnb_batch_*`` C ABI.  Every system keeps its own box,
cutoff, skin, Ewald beta, exclusions and rigid waters; all share one LJ type
table.  A step is leap-frog velocity Verlet with SETTLE, the per-system
skin-triggered neighbour-list update and one LJ + PME direct-space force
launch over all systems, replayed from captured CUDA graphs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import BatchOptions, BatchSystem, LTMatrix3, check, lib


def default_options(**kw):
    o = BatchOptions()
    lib().spgnb_batch_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Batch:
    """Systems from ``spgnb.systems`` (same ``pair_A``/``pair_B`` table)."""

    def __init__(self, systems, options=None, **kw):
        L = lib()
        self.systems = list(systems)
        s0 = self.systems[0]
        for s in self.systems[1:]:
            if s.n_types != s0.n_types or not np.array_equal(s.pair_A, s0.pair_A) or \
                    not np.array_equal(s.pair_B, s0.pair_B):
                raise ValueError("the systems of a batch share one LJ type table")
        self._keep = []
        arr = (BatchSystem * len(self.systems))()
        for k, s in enumerate(self.systems):
            crd = np.ascontiguousarray(s.crd, np.float32)
            vel = np.ascontiguousarray(s.vel if s.vel is not None else np.zeros_like(s.crd), np.float32)
            charge = np.ascontiguousarray(s.charge, np.float32)
            mass = np.ascontiguousarray(s.mass, np.float32)
            atype = np.ascontiguousarray(s.atom_type, np.int32)
            es = np.ascontiguousarray(s.excl_start, np.int32)
            en = np.ascontiguousarray(s.excl_numbers, np.int32)
            el = np.ascontiguousarray(s.excl_list if len(s.excl_list) else np.zeros(1, np.int32), np.int32)
            self._keep += [crd, vel, charge, mass, atype, es, en, el]
            y = arr[k]
            y.atom_numbers = s.n
            y.cutoff = s.cutoff
            y.skin = s.skin
            y.pme_beta = s.beta
            y.cell = LTMatrix3.of(s.cell)
            y.rcell = LTMatrix3.of(s.rcell)
            y.h_crd, y.h_vel, y.h_charge, y.h_mass = _ptr(crd), _ptr(vel), _ptr(charge), _ptr(mass)
            y.h_atom_type, y.h_excluded_start, y.h_excluded_numbers = _ptr(atype), _ptr(es), _ptr(en)
            y.h_excluded_list = _ptr(el)
            y.excluded_total = len(s.excl_list)
            y.water_begin = s.n_solute
            y.water_numbers = s.n_waters
        self.options = options if options is not None else default_options(**kw)
        pa = np.ascontiguousarray(s0.pair_A, np.float32)
        pb = np.ascontiguousarray(s0.pair_B, np.float32)
        self._keep += [pa, pb]
        h = C.c_void_p()
        check(L.spgnb_batch_create(len(self.systems), arr, s0.n_types, _ptr(pa), _ptr(pb),
                                   C.byref(self.options), C.byref(h)))
        self.handle = h
        self.atoms = sum(s.n for s in self.systems)

    def run(self, steps, energy_interval=0):
        check(lib().spgnb_batch_run(self.handle, int(steps), int(energy_interval)))

    def energies(self):
        """(S, 9): LJ short, LJ long, Coulomb direct, virial a11 a21 a22 a31 a32 a33."""
        out = np.zeros((len(self.systems), 9), np.float64)
        check(lib().spgnb_batch_energies(self.handle, _ptr(out)))
        return out

    def download(self, k):
        n = self.systems[k].n
        crd = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        frc = np.zeros((n, 3), np.float32)
        check(lib().spgnb_batch_download(self.handle, int(k), _ptr(crd), _ptr(vel), _ptr(frc)))
        return crd, vel, frc

    def stats(self):
        steps, builds, prunes = C.c_longlong(), C.c_longlong(), C.c_longlong()
        ovf = C.c_int()
        check(lib().spgnb_batch_stats(self.handle, C.byref(steps), C.byref(builds), C.byref(prunes), C.byref(ovf)))
        return {"steps": steps.value, "rebuilds": builds.value, "prunings": prunes.value, "overflow": ovf.value}

    def set_thermostat(self, tau, temperature=300.0):
        check(lib().spgnb_batch_set_thermostat(self.handle, float(tau), float(temperature)))

    def check_overflow(self):
        """True when buffers overflowed and were regrown (the lists rebuilt)."""
        r = C.c_int()
        check(lib().spgnb_batch_check_overflow(self.handle, C.byref(r)))
        return bool(r.value)

    def autotune(self, steps_per_candidate=20):
        best = C.c_float()
        check(lib().spgnb_batch_autotune(self.handle, int(steps_per_candidate), C.byref(best)))
        return best.value

    @property
    def stream_ptr(self):
        """The batch's cudaStream_t as an integer (torch.cuda.ExternalStream)."""
        return lib().spgnb_batch_stream(self.handle)

    def close(self):
        if getattr(self, "handle", None):
            lib().spgnb_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
