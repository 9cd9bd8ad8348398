"""Batched engine: many independent systems stepped together on one GPU.

``Batch`` wraps the ``spgnb_batch_*`` C ABI for a fixed set of systems and
``Pool`` for a pool into which systems are admitted and from which they are
retired while the others run (continuous batching).  Every system keeps its
own box, cutoff, skin, Ewald beta, exclusions and rigid waters, and its own
LJ type table where it differs from the batch's.  A step is leap-frog velocity Verlet with SETTLE, the
per-system skin-triggered neighbour-list update and one LJ + PME direct-space
force launch over all systems, replayed from captured CUDA graphs.  A
system's results are bitwise the same alone and in any mix.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import SPGNB_OK, BatchOptions, BatchSystem, BatchTuning, LTMatrix3, PoolOptions, SpgnbError, check, lib

SPGNB_E_OOM = 2


def default_options(**kw):
    o = BatchOptions()
    lib().spgnb_batch_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def pool_options(**kw):
    o = PoolOptions()
    lib().spgnb_batch_pool_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _fill(y, s, keep, own_table=False):
    """Fill a BatchSystem from a ``spgnb.systems`` system; arrays go to keep.
    With own_table the system carries its type table (else the batch's)."""
    if getattr(s, "water_points", 3) != 3:
        raise ValueError("the batched engine constrains 3-site waters (SETTLE) only")
    crd = np.ascontiguousarray(s.crd, np.float32)
    vel = np.ascontiguousarray(s.vel if s.vel is not None else np.zeros_like(s.crd), np.float32)
    charge = np.ascontiguousarray(s.charge, np.float32)
    mass = np.ascontiguousarray(s.mass, np.float32)
    atype = np.ascontiguousarray(s.atom_type, np.int32)
    es = np.ascontiguousarray(s.excl_start, np.int32)
    en = np.ascontiguousarray(s.excl_numbers, np.int32)
    el = np.ascontiguousarray(s.excl_list if len(s.excl_list) else np.zeros(1, np.int32), np.int32)
    keep += [crd, vel, charge, mass, atype, es, en, el]
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
    if own_table:
        pa = np.ascontiguousarray(s.pair_A, np.float32)
        pb = np.ascontiguousarray(s.pair_B, np.float32)
        keep += [pa, pb]
        y.atom_type_numbers = s.n_types
        y.h_pair_A, y.h_pair_B = _ptr(pa), _ptr(pb)


def _same_table(a, b):
    return a.n_types == b.n_types and np.array_equal(a.pair_A, b.pair_A) and np.array_equal(a.pair_B, b.pair_B)


class _Common:
    """Methods shared by Batch and Pool (``self.handle``, ``self.n_ids``)."""

    def run(self, steps, energy_interval=0):
        check(lib().spgnb_batch_run(self.handle, int(steps), int(energy_interval)))

    def energies(self):
        """(ids, 9): LJ short, LJ long, Coulomb direct, virial a11 a21 a22 a31 a32 a33."""
        out = np.zeros((self.n_ids, 9), np.float64)
        check(lib().spgnb_batch_energies(self.handle, _ptr(out)))
        return out

    def _download(self, k, n):
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
        """Picks the fastest launch configuration (the systems advance
        meanwhile); returns the chosen prune buffer, ``tuning()`` the rest."""
        best = C.c_float()
        check(lib().spgnb_batch_autotune(self.handle, int(steps_per_candidate), C.byref(best)))
        return best.value

    def tuning(self):
        t = BatchTuning()
        check(lib().spgnb_batch_get_tuning(self.handle, C.byref(t)))
        return {"prune_buffer": t.prune_buffer, "pair_blocks_per_sm": t.pair_blocks_per_sm,
                "prune_blocks_per_sm": t.prune_blocks_per_sm, "steps_per_graph": t.steps_per_graph,
                "ms_per_step": t.ms_per_step}

    def launch_counts(self):
        """(kernels every replayed step launches, kernels of a step's list build)."""
        a, b = C.c_int(), C.c_int()
        check(lib().spgnb_batch_launch_counts(self.handle, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_tuning(self, prune_buffer, pair_blocks_per_sm, prune_blocks_per_sm, steps_per_graph):
        t = BatchTuning(float(prune_buffer), int(pair_blocks_per_sm), int(prune_blocks_per_sm),
                        int(steps_per_graph), 0.0)
        check(lib().spgnb_batch_set_tuning(self.handle, C.byref(t)))

    def evaluate(self, ids):
        """Forces, energies and virial now for these systems only."""
        arr = np.ascontiguousarray(list(ids), np.int32)
        check(lib().spgnb_batch_evaluate(self.handle, _ptr(arr), len(arr)))

    def progress(self):
        """(steps done, steps left) per system id; -1 left = unlimited."""
        d = np.zeros(self.n_ids, np.int32)
        left = np.zeros(self.n_ids, np.int32)
        check(lib().spgnb_batch_progress(self.handle, _ptr(d), _ptr(left)))
        return d, left

    def capacity(self):
        ms, ma, fa, by = C.c_int(), C.c_longlong(), C.c_longlong(), C.c_double()
        check(lib().spgnb_batch_capacity(self.handle, C.byref(ms), C.byref(ma), C.byref(fa), C.byref(by)))
        return {"max_systems": ms.value, "max_atoms": ma.value, "free_atoms": fa.value, "device_bytes": by.value}

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


class Batch(_Common):
    """Systems from ``spgnb.systems``, ids 0..n-1.  The first system's type
    table is the batch's; a system whose table differs carries its own."""

    def __init__(self, systems, options=None, **kw):
        L = lib()
        self.systems = list(systems)
        s0 = self.systems[0]
        self._keep = []
        arr = (BatchSystem * len(self.systems))()
        for k, s in enumerate(self.systems):
            _fill(arr[k], s, self._keep, own_table=not _same_table(s, s0))
        self.options = options if options is not None else default_options(**kw)
        pa = np.ascontiguousarray(s0.pair_A, np.float32)
        pb = np.ascontiguousarray(s0.pair_B, np.float32)
        h = C.c_void_p()
        check(L.spgnb_batch_create(len(self.systems), arr, s0.n_types, _ptr(pa), _ptr(pb),
                                   C.byref(self.options), C.byref(h)))
        self._keep = []
        self.handle = h
        self.n_ids = len(self.systems)
        self.atoms = sum(s.n for s in self.systems)

    def download(self, k):
        return self._download(k, self.systems[k].n)


class Pool(_Common):
    """An empty pool whose type table is that of ``template``; an admitted
    system whose table differs carries its own (up to the pool options'
    ``max_types`` types).

    ``admit`` returns an id, or None when the pool has no room now."""

    def __init__(self, template, pool=None, options=None, **kw):
        L = lib()
        self.pool_options = pool if pool is not None else pool_options()
        self.options = options if options is not None else default_options(**kw)
        self.template = template
        pa = np.ascontiguousarray(template.pair_A, np.float32)
        pb = np.ascontiguousarray(template.pair_B, np.float32)
        h = C.c_void_p()
        check(L.spgnb_batch_create_pool(C.byref(self.pool_options), template.n_types, _ptr(pa), _ptr(pb),
                                        C.byref(self.options), C.byref(h)))
        self.handle = h
        self.n_ids = self.pool_options.max_systems
        self.members = {}

    def admit(self, system, steps=0):
        keep = []
        y = BatchSystem()
        _fill(y, system, keep, own_table=not _same_table(system, self.template))
        i = C.c_int(-1)
        st = lib().spgnb_batch_admit(self.handle, C.byref(y), int(steps), C.byref(i))
        if st == SPGNB_E_OOM:
            return None
        if st != SPGNB_OK:
            raise SpgnbError(st, lib().spgnb_last_error().decode())
        self.members[i.value] = system
        return i.value

    def retire(self, k):
        check(lib().spgnb_batch_retire(self.handle, int(k)))
        self.members.pop(k, None)

    def download(self, k):
        return self._download(k, self.members[k].n)
