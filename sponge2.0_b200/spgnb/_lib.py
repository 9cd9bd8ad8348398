"""ctypes binding of libspgnb.so (the C ABI declared in include/spgnb.h).

The shared library is built in-tree (``sponge2.0_b200/libspgnb.so``).  There
is no fallback: if it is missing or cannot be loaded, every entry point
raises.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libspgnb.so")

SPGNB_OK = 0
STATUS_NAMES = {0: "SPGNB_OK", 1: "SPGNB_E_ARG", 2: "SPGNB_E_OOM", 3: "SPGNB_E_CUDA", 4: "SPGNB_E_OVERFLOW",
                5: "SPGNB_E_NONFINITE", 6: "SPGNB_E_STATE", 7: "SPGNB_E_TIMEOUT", 8: "SPGNB_E_UNSUPPORTED"}

# every symbol include/spgnb.h declares
EXPORTED = [
    "spgnb_version", "spgnb_status_string", "spgnb_last_error", "spgnb_set_stream", "spgnb_get_beta",
    "spgnb_nl_default_options", "spgnb_nl_create", "spgnb_nl_update", "spgnb_nl_check_overflow",
    "spgnb_nl_atom_groups", "spgnb_nl_copy_atom_groups", "spgnb_nl_get_stats", "spgnb_nl_destroy",
    "spgnb_lj_create", "spgnb_lj_get_local", "spgnb_lj_pme_direct_force", "spgnb_lj_pme_direct_force_atom_groups",
    "spgnb_lj_long_range_correction", "spgnb_lj_energies", "spgnb_lj_totals", "spgnb_lj_long_range_factor",
    "spgnb_lj_destroy", "spgnb_lj_atom_lj_energy", "spgnb_lj_export_vector_lj",
    "spgnb_lj_pme_excluded_force", "spgnb_lj_pme_excluded_energy", "spgnb_lj_fuse_pme_excluded",
    "spgnb_nl_build_full",
    "spgnb_solvent_create", "spgnb_solvent_get_local", "spgnb_solvent_pme_direct_force", "spgnb_solvent_destroy",
    "spgnb_launch_count", "spgnb_debug_set_pair_events", "spgnb_nl_count_pairs", "spgnb_probe_fp32_fma_tflops",
    "spgnb_lj_pme_direct_force_noalloc",
    "spgnb_lj_soft_default_params", "spgnb_lj_soft_create", "spgnb_lj_soft_get_local",
    "spgnb_lj_soft_pme_direct_force", "spgnb_lj_soft_partial_h_partial_lambda",
    "spgnb_lj_soft_long_range_correction", "spgnb_lj_soft_energies", "spgnb_lj_soft_totals",
    "spgnb_lj_soft_long_range_factors", "spgnb_lj_soft_atom_lj_energy", "spgnb_lj_soft_perturbed_atoms",
    "spgnb_lj_soft_destroy", "spgnb_solvent_create_soft",
    "spgnb_batch_default_options", "spgnb_batch_create", "spgnb_batch_run", "spgnb_batch_energies",
    "spgnb_batch_download", "spgnb_batch_stats", "spgnb_batch_autotune", "spgnb_batch_get_tuning", "spgnb_batch_set_tuning",
    "spgnb_batch_launch_counts",
    "spgnb_batch_stream",
    "spgnb_batch_check_overflow", "spgnb_batch_set_thermostat",
    "spgnb_batch_destroy",
    "spgnb_batch_pool_default_options", "spgnb_batch_create_pool", "spgnb_batch_admit", "spgnb_batch_retire",
    "spgnb_batch_evaluate", "spgnb_batch_progress", "spgnb_batch_capacity",
]


class SpgnbError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class LTMatrix3(C.Structure):
    _fields_ = [("a11", C.c_float), ("a21", C.c_float), ("a22", C.c_float), ("a31", C.c_float),
                ("a32", C.c_float), ("a33", C.c_float)]

    @classmethod
    def of(cls, m):
        m = [float(v) for v in m]
        return cls(*m)


class NLOptions(C.Structure):
    _fields_ = [("max_neighbor_numbers", C.c_int), ("max_atom_in_grid_numbers", C.c_int),
                ("max_ghost_in_grid_numbers", C.c_int), ("refresh_interval", C.c_int),
                ("skin_permit", C.c_float), ("check_overflow_interval", C.c_int),
                ("throw_error_when_overflow", C.c_int), ("export_atom_groups", C.c_int),
                ("max_entries_per_cluster", C.c_int), ("prune_buffer", C.c_float)]


class BatchSystem(C.Structure):
    _fields_ = [("atom_numbers", C.c_int), ("cutoff", C.c_float), ("skin", C.c_float), ("pme_beta", C.c_float),
                ("cell", LTMatrix3), ("rcell", LTMatrix3), ("h_crd", C.c_void_p), ("h_vel", C.c_void_p),
                ("h_charge", C.c_void_p), ("h_mass", C.c_void_p), ("h_atom_type", C.c_void_p),
                ("h_excluded_start", C.c_void_p), ("h_excluded_numbers", C.c_void_p),
                ("h_excluded_list", C.c_void_p), ("excluded_total", C.c_int), ("water_begin", C.c_int),
                ("water_numbers", C.c_int), ("atom_type_numbers", C.c_int), ("h_pair_A", C.c_void_p),
                ("h_pair_B", C.c_void_p)]


class BatchOptions(C.Structure):
    _fields_ = [("dt", C.c_float), ("water_doh", C.c_float), ("water_dhh", C.c_float), ("skin_permit", C.c_float),
                ("prune_buffer", C.c_float), ("steps_per_graph", C.c_int), ("use_graphs", C.c_int),
                ("thermostat_tau", C.c_float), ("temperature", C.c_float), ("refresh_interval", C.c_int)]


class BatchTuning(C.Structure):
    _fields_ = [("prune_buffer", C.c_float), ("pair_blocks_per_sm", C.c_int), ("prune_blocks_per_sm", C.c_int),
                ("steps_per_graph", C.c_int), ("ms_per_step", C.c_float)]


class PoolOptions(C.Structure):
    _fields_ = [("max_systems", C.c_int), ("max_atoms", C.c_int), ("max_excluded", C.c_longlong),
                ("max_waters", C.c_int), ("max_cutoff", C.c_float), ("min_cutoff", C.c_float), ("skin", C.c_float),
                ("density", C.c_float), ("hbm_budget_bytes", C.c_double), ("max_types", C.c_int),
                ("type_table_bytes", C.c_double)]


class SoftCoreParams(C.Structure):
    _fields_ = [("lambda_", C.c_float), ("alpha", C.c_float), ("p", C.c_float), ("sigma", C.c_float),
                ("sigma_min", C.c_float)]


class NLStats(C.Structure):
    _fields_ = [("atom_numbers", C.c_int), ("grid_numbers", C.c_int), ("grid_dims", C.c_int * 3),
                ("clusters", C.c_int), ("entries", C.c_longlong), ("work_items", C.c_int),
                ("builds", C.c_longlong), ("overflow", C.c_int), ("full_list_words", C.c_longlong),
                ("prunes", C.c_longlong), ("pruned_list_words", C.c_longlong), ("device_bytes", C.c_longlong)]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SpgnbError(8, f"{LIB_PATH} is not built; run __graft_entry__.build() or make -C sponge2.0_b200/csrc")
    L = C.CDLL(LIB_PATH)
    vp, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
    M = LTMatrix3
    L.spgnb_version.restype = C.c_char_p
    L.spgnb_status_string.restype = C.c_char_p
    L.spgnb_status_string.argtypes = [i]
    L.spgnb_last_error.restype = C.c_char_p
    L.spgnb_set_stream.argtypes = [vp]
    L.spgnb_get_beta.restype = f
    L.spgnb_get_beta.argtypes = [f, f]
    L.spgnb_nl_default_options.argtypes = [C.POINTER(NLOptions)]
    L.spgnb_nl_default_options.restype = None
    L.spgnb_nl_create.argtypes = [i, f, f, M, M, C.POINTER(NLOptions), C.POINTER(vp)]
    L.spgnb_nl_update.argtypes = [vp, vp, i, i, vp, M, M, i, i, vp, vp, vp]
    L.spgnb_nl_check_overflow.argtypes = [vp, i, M, M, C.POINTER(i)]
    L.spgnb_nl_atom_groups.argtypes = [vp, C.POINTER(vp), C.POINTER(vp)]
    L.spgnb_nl_copy_atom_groups.argtypes = [vp, vp, vp, C.c_longlong, C.POINTER(C.c_longlong)]
    L.spgnb_nl_get_stats.argtypes = [vp, C.POINTER(NLStats)]
    L.spgnb_nl_destroy.argtypes = [vp]
    L.spgnb_nl_build_full.argtypes = [vp, i, vp, M, M, f, vp, i, vp]
    L.spgnb_batch_default_options.argtypes = [C.POINTER(BatchOptions)]
    L.spgnb_batch_default_options.restype = None
    L.spgnb_batch_create.argtypes = [i, C.POINTER(BatchSystem), i, vp, vp, C.POINTER(BatchOptions), C.POINTER(vp)]
    L.spgnb_batch_run.argtypes = [vp, i, i]
    L.spgnb_batch_energies.argtypes = [vp, vp]
    L.spgnb_batch_download.argtypes = [vp, i, vp, vp, vp]
    L.spgnb_batch_stats.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                    C.POINTER(C.c_int)]
    L.spgnb_batch_autotune.argtypes = [vp, i, C.POINTER(C.c_float)]
    L.spgnb_batch_get_tuning.argtypes = [vp, C.POINTER(BatchTuning)]
    L.spgnb_batch_set_tuning.argtypes = [vp, C.POINTER(BatchTuning)]
    L.spgnb_batch_launch_counts.argtypes = [vp, C.POINTER(i), C.POINTER(i)]
    L.spgnb_batch_check_overflow.argtypes = [vp, C.POINTER(i)]
    L.spgnb_batch_set_thermostat.argtypes = [vp, f, f]
    L.spgnb_batch_stream.argtypes = [vp]
    L.spgnb_batch_stream.restype = vp
    L.spgnb_batch_destroy.argtypes = [vp]
    L.spgnb_batch_pool_default_options.argtypes = [C.POINTER(PoolOptions)]
    L.spgnb_batch_pool_default_options.restype = None
    L.spgnb_batch_create_pool.argtypes = [C.POINTER(PoolOptions), i, vp, vp, C.POINTER(BatchOptions), C.POINTER(vp)]
    L.spgnb_batch_admit.argtypes = [vp, C.POINTER(BatchSystem), i, C.POINTER(i)]
    L.spgnb_batch_retire.argtypes = [vp, i]
    L.spgnb_batch_evaluate.argtypes = [vp, vp, i]
    L.spgnb_batch_progress.argtypes = [vp, vp, vp]
    L.spgnb_batch_capacity.argtypes = [vp, C.POINTER(i), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                       C.POINTER(d)]
    L.spgnb_lj_create.argtypes = [i, i, vp, vp, vp, f, C.POINTER(vp)]
    L.spgnb_lj_get_local.argtypes = [vp, vp, i, i]
    L.spgnb_lj_pme_direct_force.argtypes = [vp, i, i, i, i, vp, vp, vp, M, M, vp, f, i, vp, i, vp, vp]
    L.spgnb_lj_pme_direct_force_atom_groups.argtypes = [vp, i, i, i, i, vp, vp, vp, M, M, vp, f, i, vp, i, vp, vp]
    L.spgnb_lj_long_range_correction.argtypes = [vp, i, vp, i, vp, f]
    L.spgnb_lj_energies.argtypes = [vp, C.POINTER(d), C.POINTER(d), C.POINTER(d), C.POINTER(d)]
    L.spgnb_lj_totals.argtypes = [vp, C.POINTER(d)]
    L.spgnb_lj_long_range_factor.restype = d
    L.spgnb_lj_long_range_factor.argtypes = [vp]
    L.spgnb_lj_destroy.argtypes = [vp]
    L.spgnb_lj_atom_lj_energy.argtypes = [vp, C.POINTER(vp)]
    L.spgnb_lj_export_vector_lj.argtypes = [vp, vp, vp, vp, i]
    L.spgnb_lj_pme_excluded_force.argtypes = [vp, i, vp, M, M, vp, f, vp, vp, vp, vp, i, vp, vp]
    L.spgnb_lj_pme_excluded_energy.argtypes = [vp, C.POINTER(d)]
    L.spgnb_lj_fuse_pme_excluded.argtypes = [vp, i, vp, vp, vp, i]
    L.spgnb_solvent_create.argtypes = [vp, i, C.POINTER(vp)]
    L.spgnb_solvent_get_local.argtypes = [vp, i, vp, i, vp, C.POINTER(i)]
    L.spgnb_solvent_pme_direct_force.argtypes = [vp, i, i, vp, vp, vp, vp, M, M, vp, vp, f, i, vp, i, vp, vp]
    L.spgnb_solvent_destroy.argtypes = [vp]
    L.spgnb_launch_count.restype = C.c_ulonglong
    L.spgnb_debug_set_pair_events.argtypes = [vp, vp]
    L.spgnb_nl_count_pairs.argtypes = [vp, vp, M, M, f, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    L.spgnb_probe_fp32_fma_tflops.argtypes = [i, C.POINTER(d)]
    L.spgnb_lj_pme_direct_force_noalloc.argtypes = [i, i, i, i, vp, vp, vp, vp, vp, vp, M, M, vp, f, f]
    SP = C.POINTER(SoftCoreParams)
    L.spgnb_lj_soft_default_params.argtypes = [SP]
    L.spgnb_lj_soft_default_params.restype = None
    L.spgnb_lj_soft_create.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp, SP, f, C.POINTER(vp)]
    L.spgnb_lj_soft_get_local.argtypes = [vp, vp, i, i]
    L.spgnb_lj_soft_pme_direct_force.argtypes = [vp, i, i, i, i, vp, vp, vp, M, M, vp, f, i, vp, i, vp, vp]
    L.spgnb_lj_soft_partial_h_partial_lambda.argtypes = [vp, i, vp, M, M, vp, vp, vp, f, i, C.POINTER(d),
                                                         C.POINTER(d)]
    L.spgnb_lj_soft_long_range_correction.argtypes = [vp, i, vp, i, vp, f]
    L.spgnb_lj_soft_energies.argtypes = [vp, C.POINTER(d), C.POINTER(d), C.POINTER(d), C.POINTER(d)]
    L.spgnb_lj_soft_totals.argtypes = [vp, C.POINTER(d)]
    L.spgnb_lj_soft_long_range_factors.argtypes = [vp, C.POINTER(d), C.POINTER(d)]
    L.spgnb_lj_soft_atom_lj_energy.argtypes = [vp, C.POINTER(vp)]
    L.spgnb_lj_soft_perturbed_atoms.argtypes = [vp, C.POINTER(i), vp, i]
    L.spgnb_lj_soft_destroy.argtypes = [vp]
    L.spgnb_solvent_create_soft.argtypes = [vp, i, C.POINTER(vp)]
    _lib = L
    return L


def check(status):
    if status != SPGNB_OK:
        raise SpgnbError(status, lib().spgnb_last_error().decode())
    return status


def version():
    return lib().spgnb_version().decode()
