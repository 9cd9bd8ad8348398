"""Python access to the oracle (TEST INFRASTRUCTURE ONLY).

``Oracle`` wraps ``libspgnb_oracle.so`` (the C restatement in
``spgnb_oracle.c``); ``Reference`` wraps ``_ref/libspgref_cpu.so`` or
``_ref/libspgref_cuda.so`` (the reference's own code, built from its sources
by ``oracle/Makefile``).  Only the tests, the smoke check and the benchmark's
CPU-baseline leg import this module, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(name):
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (make -C oracle)")
    return C.CDLL(path)


def _c32(a):
    return np.ascontiguousarray(a, np.float32)


def _ci32(a):
    return np.ascontiguousarray(a, np.int32)


class Oracle:
    def __init__(self):
        lib = _load("libspgnb_oracle.so")
        lib.orc_beta.restype = C.c_float
        lib.orc_beta.argtypes = [C.c_float, C.c_float]
        lib.orc_nl_build.restype = C.c_longlong
        lib.orc_nl_build.argtypes = [C.c_int, _f32p, _f32p, _f32p, C.c_float, C.c_float, _i32p, _i32p, _i32p,
                                     C.c_int, _i32p, C.c_void_p, C.c_longlong]
        lib.orc_pair_force_fp64.restype = C.c_longlong
        lib.orc_pair_force_fp64.argtypes = [C.c_int, _f32p, _f32p, _i32p, _f32p, _f32p, _f32p, C.c_float,
                                            C.c_float, _i32p, _i32p, _f64p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, _f64p]
        lib.orc_direct_sum_fp64.restype = C.c_longlong
        lib.orc_direct_sum_fp64.argtypes = [C.c_int, _f32p, _f32p, _i32p, _f32p, _f32p, _f32p, C.c_float,
                                            C.c_float, _i32p, _i32p, _i32p, _f64p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, _f64p]
        lib.orc_long_range_factor.restype = C.c_double
        lib.orc_long_range_factor.argtypes = [C.c_int, _i32p, C.c_int, _f32p, C.c_float]
        lib.orc_soft_core_fp64.restype = C.c_longlong
        lib.orc_soft_core_fp64.argtypes = [C.c_int, _f32p, _f32p, C.c_void_p, _i32p, _i32p, _f32p, _f32p, _f32p,
                                           _f32p, _f32p, _f32p, C.c_float, C.c_float, _i32p, _i32p, _i32p, _f64p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, _f64p]
        lib.orc_soft_long_range.restype = None
        lib.orc_soft_long_range.argtypes = [C.c_int, _i32p, _i32p, _f32p, _f32p, C.c_float, C.c_float,
                                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.orc_direct_forces_subset_fp64.restype = C.c_longlong
        lib.orc_direct_forces_subset_fp64.argtypes = [C.c_int, _f32p, _f32p, _i32p, _f32p, _f32p, _f32p, C.c_float,
                                                      C.c_float, _i32p, _i32p, _i32p, C.c_int, _i32p, _f64p]
        lib.orc_pair_dr2.restype = C.c_float
        lib.orc_pair_dr2.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int]
        self.lib = lib

    def beta(self, cutoff, tol=1e-5):
        return float(self.lib.orc_beta(cutoff, tol))

    def nl_build(self, s, crd=None, mode=1):
        """Reference half list as (counts[n], lists) with each list sorted."""
        crd = _c32(s.crd if crd is None else crd)
        n = s.n
        counts = np.zeros(n, np.int32)
        args = (n, crd, _c32(s.cell), _c32(s.rcell), s.cutoff, s.skin, _ci32(s.excl_start),
                _ci32(s.excl_numbers), _ci32(s.excl_list if len(s.excl_list) else np.zeros(1, np.int32)), mode)
        total = self.lib.orc_nl_build(*args, counts, None, 0)
        if total < 0:
            raise RuntimeError(f"oracle neighbour build failed ({total})")
        lists = np.zeros(max(int(total), 1), np.int32)
        total2 = self.lib.orc_nl_build(*args, counts, lists.ctypes.data_as(C.c_void_p), int(total))
        assert total2 == total
        return counts, lists[:total]

    def pair_force(self, s, counts, lists, crd=None, per_atom=True):
        crd = _c32(s.crd if crd is None else crd)
        n = s.n
        frc = np.zeros(3 * n, np.float64)
        elj = np.zeros(n, np.float64) if per_atom else None
        ec = np.zeros(n, np.float64) if per_atom else None
        vir = np.zeros(6 * n, np.float64) if per_atom else None
        tot = np.zeros(8, np.float64)
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        npairs = self.lib.orc_pair_force_fp64(n, crd, _c32(s.charge), _ci32(s.atom_type), _c32(s.pair_A),
                                              _c32(s.pair_B), _c32(s.cell), s.cutoff, s.beta, _ci32(counts),
                                              _ci32(lists if len(lists) else np.zeros(1, np.int32)), frc,
                                              ptr(elj), ptr(ec), ptr(vir), tot)
        return _result(frc, elj, ec, vir, tot, npairs)

    def direct_forces_subset(self, s, atoms, crd=None):
        """FP64 forces on the given atoms from all their partners within rc
        (exclusions removed): (len(atoms), 3)."""
        crd = _c32(s.crd if crd is None else crd)
        atoms = _ci32(atoms)
        out = np.zeros(3 * len(atoms), np.float64)
        self.lib.orc_direct_forces_subset_fp64(
            s.n, crd, _c32(s.charge), _ci32(s.atom_type), _c32(s.pair_A), _c32(s.pair_B), _c32(s.cell),
            s.cutoff, s.beta, _ci32(s.excl_start), _ci32(s.excl_numbers),
            _ci32(s.excl_list if len(s.excl_list) else np.zeros(1, np.int32)), len(atoms), atoms, out)
        return out.reshape(-1, 3)

    def direct_sum(self, s, crd=None, per_atom=False):
        crd = _c32(s.crd if crd is None else crd)
        n = s.n
        frc = np.zeros(3 * n, np.float64)
        elj = np.zeros(n, np.float64) if per_atom else None
        ec = np.zeros(n, np.float64) if per_atom else None
        vir = np.zeros(6 * n, np.float64) if per_atom else None
        tot = np.zeros(8, np.float64)
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        npairs = self.lib.orc_direct_sum_fp64(n, crd, _c32(s.charge), _ci32(s.atom_type), _c32(s.pair_A),
                                              _c32(s.pair_B), _c32(s.cell), s.cutoff, s.beta,
                                              _ci32(s.excl_start), _ci32(s.excl_numbers),
                                              _ci32(s.excl_list if len(s.excl_list) else np.zeros(1, np.int32)),
                                              frc, ptr(elj), ptr(ec), ptr(vir), tot)
        return _result(frc, elj, ec, vir, tot, npairs)

    @staticmethod
    def pme_excluded(s):
        """FP64 PME excluded-pair correction (PM_force.cpp:918-974): for each
        excluded pair i < j of the CSR, dr = min image(r_j - r_i) and
        F_i += -q_i q_j (2/sqrt(pi) x exp(-x^2) + erfc(x) - 1) / r^3 dr,
        F_j -= the same, E_i -= q_i q_j erf(x)/r (x = beta r), and
        W_i -= Get_Virial_From_Force_Dis(F, dr)."""
        from scipy.special import erf, erfc
        n = s.n
        crd = np.asarray(s.crd, np.float64)
        q = np.asarray(s.charge, np.float64)
        start, num = np.asarray(s.excl_start), np.asarray(s.excl_numbers)
        lst = np.asarray(s.excl_list)
        ii = np.repeat(np.arange(n), num)
        jj = np.concatenate([lst[start[k]:start[k] + num[k]] for k in range(n) if num[k] > 0]) if num.sum() else \
            np.zeros(0, int)
        a11, a21, a22, a31, a32, a33 = (float(v) for v in s.cell)
        r11, r21, r22, r31, r32, r33 = (float(v) for v in s.rcell)
        d = crd[jj] - crd[ii]
        sx = np.floor(d[:, 0] * r11 + d[:, 1] * r21 + d[:, 2] * r31 + 0.5)
        sy = np.floor(d[:, 1] * r22 + d[:, 2] * r32 + 0.5)
        sz = np.floor(d[:, 2] * r33 + 0.5)
        d[:, 0] -= sx * a11 + sy * a21 + sz * a31
        d[:, 1] -= sy * a22 + sz * a32
        d[:, 2] -= sz * a33
        r2 = (d * d).sum(1)
        r = np.sqrt(r2)
        x = s.beta * r
        qq = q[ii] * q[jj]
        fa = -qq * (x * 2.0 / np.sqrt(np.pi) * np.exp(-x * x) + erfc(x) - 1.0) / r2 / r
        g = fa[:, None] * d
        frc = np.zeros((n, 3))
        np.add.at(frc, ii, g)
        np.add.at(frc, jj, -g)
        e_atom = np.zeros(n)
        np.add.at(e_atom, ii, -qq * erf(x) / r)
        w = -np.stack([g[:, 0] * d[:, 0], g[:, 0] * d[:, 1] + g[:, 1] * d[:, 0], g[:, 1] * d[:, 1],
                       g[:, 0] * d[:, 2] + g[:, 2] * d[:, 0], g[:, 1] * d[:, 2] + g[:, 2] * d[:, 1],
                       g[:, 2] * d[:, 2]], 1)
        vir = np.zeros((n, 6))
        np.add.at(vir, ii, w)
        return {"frc": frc, "e_atom": e_atom, "energy": float(e_atom.sum()), "virial_atom": vir, "pairs": len(ii)}

    def long_range_factor(self, s):
        return float(self.lib.orc_long_range_factor(s.n, _ci32(s.atom_type), s.n_types, _c32(s.pair_B),
                                                    s.cutoff))

    def soft_core(self, f, lam=None, crd=None, charge_ba=True, per_atom=True):
        """FP64 two-state soft-core pair sum of an FepSystem (orc_soft_core_fp64):
        forces, owner energies and virial as direct_sum, plus dh_lj and dh_c
        (dH/dlambda of LJ and of the direct-space Coulomb term, pair part)."""
        s = f.base
        crd = _c32(s.crd if crd is None else crd)
        n = s.n
        q = _c32(f.charge(lam))
        qba = _c32(f.charge_ba()) if charge_ba else None
        frc = np.zeros(3 * n, np.float64)
        elj = np.zeros(n, np.float64) if per_atom else None
        ec = np.zeros(n, np.float64) if per_atom else None
        vir = np.zeros(6 * n, np.float64) if per_atom else None
        tot = np.zeros(10, np.float64)
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        npairs = self.lib.orc_soft_core_fp64(n, crd, q, ptr(qba), _ci32(f.type_a), _ci32(f.type_b), _c32(f.AA),
                                             _c32(f.AB), _c32(f.BA), _c32(f.BB), _c32(f.params(lam)), _c32(s.cell),
                                             s.cutoff, s.beta, _ci32(s.excl_start), _ci32(s.excl_numbers),
                                             _ci32(s.excl_list if len(s.excl_list) else np.zeros(1, np.int32)),
                                             frc, ptr(elj), ptr(ec), ptr(vir), tot)
        out = _result(frc, elj, ec, vir, tot[:8], npairs)
        out["dh_lj"] = float(tot[8])
        out["dh_c"] = float(tot[9])
        return out

    def soft_long_range(self, f, lam=None):
        """(factor, factor_TI) of LJ_SOFT_CORE's long-range correction."""
        a, b = C.c_double(), C.c_double()
        self.lib.orc_soft_long_range(f.base.n, _ci32(f.type_a), _ci32(f.type_b), _c32(f.AB), _c32(f.BB),
                                     float(f.lam if lam is None else lam), f.base.cutoff, C.byref(a), C.byref(b))
        return a.value, b.value


def _result(frc, elj, ec, vir, tot, npairs):
    return {
        "frc": frc.reshape(-1, 3),
        "e_lj_atom": elj,
        "e_coul_atom": ec,
        "virial_atom": None if vir is None else vir.reshape(-1, 6),
        "e_lj": float(tot[0]),
        "e_coul": float(tot[1]),
        "virial": tot[2:8].copy(),
        "pairs_in_cutoff": int(npairs),
    }


class Reference:
    """The reference's own implementation of the path (CPU or CUDA build)."""

    def __init__(self, gpu=False, shim=False):
        name = "libspgref_shim.so" if shim else ("libspgref_cuda.so" if gpu else "libspgref_cpu.so")
        lib = _load(os.path.join("_ref", name))
        lib.ref_init.argtypes = [C.c_int, C.c_int, _i32p, _f32p, _f32p, C.c_float, C.c_float, _f32p, _f32p,
                                 C.c_int, C.c_int, _i32p, _i32p, _i32p, C.c_int]
        lib.ref_nl_update.argtypes = [_f32p, C.c_int, C.c_int]
        lib.ref_nl_get.restype = C.c_longlong
        lib.ref_nl_get.argtypes = [_i32p, C.c_void_p, C.c_longlong, C.c_void_p]
        lib.ref_force.argtypes = [_f32p, _f32p, C.c_float, C.c_int, C.c_int, _f32p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]
        lib.ref_time_steps.restype = C.c_double
        lib.ref_time_steps.argtypes = [_f32p, _f32p, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.ref_time_rebuild.restype = C.c_double
        lib.ref_time_rebuild.argtypes = [_f32p, C.c_int]
        lib.ref_long_range_factor.restype = C.c_double
        lib.ref_enable_solvent.argtypes = [C.c_int, _i32p, C.c_int, C.c_int, C.c_int]
        lib.ref_set_threads.argtypes = [C.c_int]
        lib.ref_set_key.argtypes = [C.c_char_p, C.c_char_p]
        if hasattr(lib, "ref_pme_excluded"):
            lib.ref_pme_excluded.restype = C.c_double
            lib.ref_pme_excluded.argtypes = [_f32p, _f32p, C.c_float, C.c_int, _f32p, _f32p, _f32p]
        if hasattr(lib, "ref_md_init"):
            lib.ref_md_init.restype = C.c_int
            lib.ref_md_init.argtypes = [_f32p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float]
            lib.ref_md_run.restype = None
            lib.ref_md_run.argtypes = [_f32p, _f32p, _f32p, C.c_float, C.c_int, C.c_int, _f64p]
        if hasattr(lib, "ref_soft_init"):
            lib.ref_soft_init.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p,
                                          _f32p, C.c_float]
            lib.ref_soft_force.argtypes = [_f32p, _f32p, C.c_float, C.c_int, C.c_int, _f32p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p]
            lib.ref_soft_dhdl.restype = C.c_double
            lib.ref_soft_dhdl.argtypes = [_f32p, _f32p, C.c_void_p, C.c_float, C.c_int, C.POINTER(C.c_double)]
            lib.ref_soft_long_range.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
            lib.ref_soft_long_range.restype = None
            lib.ref_soft_time_steps.restype = C.c_double
            lib.ref_soft_time_steps.argtypes = [_f32p, _f32p, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int]
        self.lib = lib
        self.gpu = bool(lib.ref_is_gpu())
        self.shim = shim
        self.s = None

    def set_threads(self, t):
        self.lib.ref_set_threads(int(t))

    def set_key(self, key, value):
        """A control key for the modules of the next init() (value None removes it)."""
        self.lib.ref_set_key(key.encode(), b"" if value is None else str(value).encode())

    def init(self, s, max_neighbor=1200, refresh_interval=0, solvent=False):
        self.s = s
        ex = _ci32(s.excl_list if len(s.excl_list) else np.zeros(1, np.int32))
        self.lib.ref_init(s.n, s.n_types, _ci32(s.atom_type), _c32(s.pair_A), _c32(s.pair_B), s.cutoff, s.skin,
                          _c32(s.cell), _c32(s.rcell), max_neighbor, refresh_interval, _ci32(s.excl_start),
                          _ci32(s.excl_numbers), ex, len(s.excl_list))
        if solvent:
            first_res = len(s.res_start) - s.n_waters
            wp = getattr(s, "water_points", 3)
            rc = self.lib.ref_enable_solvent(len(s.res_start), _ci32(s.res_start), first_res, wp * s.n_waters, wp)
            if rc != 0 and not self.shim:
                raise RuntimeError("the solvent module exists only in the reference's GPU build")

    def nl_update(self, crd=None, step=0, forced=True):
        self.lib.ref_nl_update(_c32(self.s.crd if crd is None else crd), step, 1 if forced else 0)

    def nl_get(self, sort=True):
        n = self.s.n
        counts = np.zeros(n, np.int32)
        total = self.lib.ref_nl_get(counts, None, 0, None)
        lists = np.zeros(max(int(total), 1), np.int32)
        flags = np.zeros(2, np.int32)
        self.lib.ref_nl_get(counts, lists.ctypes.data_as(C.c_void_p), int(total), flags.ctypes.data_as(C.c_void_p))
        lists = lists[:total]
        if sort:
            off = 0
            for i in range(n):
                c = int(counts[i])
                lists[off:off + c].sort()
                off += c
        return counts, lists, flags

    def force(self, crd=None, need_energy=True, need_virial=True):
        s = self.s
        n = s.n
        frc = np.zeros(3 * n, np.float32)
        e = np.zeros(n, np.float32)
        v = np.zeros(6 * n, np.float32)
        d = np.zeros(n, np.float32)
        lj = np.zeros(n, np.float32)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        self.lib.ref_force(_c32(s.crd if crd is None else crd), _c32(s.charge), s.beta, int(need_energy),
                           int(need_virial), frc, p(e), p(v), p(d), p(lj))
        return {"frc": frc.reshape(-1, 3), "atom_energy": e, "atom_virial": v.reshape(-1, 6),
                "atom_direct": d, "atom_lj": lj}

    def time_steps(self, steps, first_step=0, need_energy=False, need_virial=False, crd=None):
        s = self.s
        return float(self.lib.ref_time_steps(_c32(s.crd if crd is None else crd), _c32(s.charge), s.beta,
                                             first_step, steps, int(need_energy), int(need_virial)))

    def pme_excluded(self, crd=None, need_energy=True):
        """The reference's PME excluded-pair correction (CUDA build only) on
        the system of the last init(): forces, per-atom energy and virial,
        and the correction's energy."""
        s = self.s
        n = s.n
        frc = np.zeros(3 * n, np.float32)
        ene = np.zeros(n, np.float32)
        vir = np.zeros(6 * n, np.float32)
        e = self.lib.ref_pme_excluded(_c32(s.crd if crd is None else crd), _c32(s.charge), s.beta, int(need_energy),
                                      frc, ene, vir)
        return {"frc": frc.reshape(-1, 3), "atom_energy": ene, "atom_virial": vir.reshape(-1, 6), "energy": float(e)}

    def md_init(self, dt=0.002, d_oh=0.9572, d_hh=1.5139):
        """The reference's SETTLE for the system's trailing 3-site waters
        (CUDA build only); returns the number of SETTLE triangles."""
        s = self.s
        first = s.n - 3 * s.n_waters
        return int(self.lib.ref_md_init(_c32(s.mass), first, s.n_waters, d_oh, d_hh, dt))

    def md_run(self, crd, vel, steps, first_step=0):
        """NVE steps of the reference's force path, leap-frog and SETTLE:
        (crd, vel) after them and (steps, 2) LJ / direct Coulomb energies at
        each step's starting positions."""
        crd = np.array(crd, np.float32, copy=True, order="C")
        vel = np.array(vel, np.float32, copy=True, order="C")
        e = np.zeros(2 * steps, np.float64)
        self.lib.ref_md_run(crd, vel, _c32(self.s.charge), self.s.beta, first_step, steps, e)
        return crd, vel, e.reshape(-1, 2)

    def time_rebuild(self, reps=1, crd=None):
        return float(self.lib.ref_time_rebuild(_c32(self.s.crd if crd is None else crd), reps))

    def long_range_factor(self):
        return float(self.lib.ref_long_range_factor())

    def soft_init(self, f, lam=None):
        """LJ_SOFT_CORE::Initial + Get_Local for an FepSystem (after init())."""
        self.fep = f
        self.fep_lam = f.lam if lam is None else lam
        rc = self.lib.ref_soft_init(f.base.n, f.n_types_a, f.n_types_b, _ci32(f.type_a), _ci32(f.type_b),
                                    _c32(f.AA), _c32(f.AB), _c32(f.BA), _c32(f.BB), _c32(f.params(lam)),
                                    f.base.cutoff)
        if rc != 0:
            raise RuntimeError("LJ_SOFT_CORE did not initialise")

    def soft_force(self, crd=None, need_energy=True, need_virial=True):
        s, f = self.s, self.fep
        n = s.n
        frc = np.zeros(3 * n, np.float32)
        e = np.zeros(n, np.float32)
        v = np.zeros(6 * n, np.float32)
        d = np.zeros(n, np.float32)
        lj = np.zeros(n, np.float32)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        self.lib.ref_soft_force(_c32(s.crd if crd is None else crd), _c32(f.charge(self.fep_lam)), s.beta,
                                int(need_energy), int(need_virial), frc, p(e), p(v), p(d), p(lj))
        return {"frc": frc.reshape(-1, 3), "atom_energy": e, "atom_virial": v.reshape(-1, 6),
                "atom_direct": d, "atom_lj": lj}

    def soft_dhdl(self, crd=None, charge_perturbated=True):
        """(dH/dlambda LJ incl. the long-range term, direct-space Coulomb part)."""
        s, f = self.s, self.fep
        qba = _c32(f.charge_ba())
        direct = C.c_double()
        v = self.lib.ref_soft_dhdl(_c32(s.crd if crd is None else crd), _c32(f.charge(self.fep_lam)),
                                   qba.ctypes.data_as(C.c_void_p), s.beta, int(charge_perturbated), C.byref(direct))
        return float(v), float(direct.value)

    def soft_long_range(self):
        a, b = C.c_double(), C.c_double()
        self.lib.ref_soft_long_range(C.byref(a), C.byref(b))
        return a.value, b.value

    def soft_time_steps(self, steps, first_step=0, need_energy=False, need_virial=False, crd=None):
        s, f = self.s, self.fep
        return float(self.lib.ref_soft_time_steps(_c32(s.crd if crd is None else crd), _c32(f.charge(self.fep_lam)),
                                                  s.beta, first_step, steps, int(need_energy), int(need_virial)))

    def clear(self):
        self.lib.ref_clear()
