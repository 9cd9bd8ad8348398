"""The oracle against the golden fixtures produced by the reference's own CPU
build (tests/golden/make_golden.py): identical neighbour lists, FP64 forces
and energies within FP32 error of the reference, and the GROMACS lj_sr pin
of the reference's comparison suite."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT, rel_rms

GOLDEN = os.path.join(ROOT, "tests", "golden")
META = json.load(open(os.path.join(GOLDEN, "golden.json")))
CASES = sorted(META)


def load_case(name):
    from spgnb import systems as S
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    m = META[name]
    s = S.System(crd=z["crd"], charge=z["charge"], atom_type=z["atom_type"], pair_A=z["pair_A"],
                 pair_B=z["pair_B"], n_types=m["n_types"], excl_start=z["excl_start"],
                 excl_numbers=z["excl_numbers"], excl_list=z["excl_list"], mass=z["mass"],
                 res_start=z["res_start"], res_len=z["res_len"], cell=z["cell"], rcell=z["rcell"],
                 cutoff=m["cutoff"], skin=m["skin"], beta=m["beta"], n_solute=m["n_solute"], name=name)
    return s, z, m


def digest(counts, lists):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(counts, np.int32).tobytes())
    h.update(np.ascontiguousarray(lists, np.int32).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", CASES)
def test_oracle_neighbor_list_equals_reference(oracle, name):
    s, z, m = load_case(name)
    counts, lists = oracle.nl_build(s, mode=0)
    assert np.array_equal(counts, z["ref_counts"])
    assert digest(counts, lists) == m["list_sha256"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_fp64_forces_and_energies(oracle, name):
    s, z, m = load_case(name)
    counts, lists = oracle.nl_build(s, mode=0)
    r = oracle.pair_force(s, counts, lists)
    # the reference computes in FP32: agree to FP32 accumulation error
    assert rel_rms(z["ref_frc"], r["frc"]) < 1e-5
    scale = abs(r["e_lj"]) + abs(r["e_coul"])
    assert abs(r["e_lj"] - m["ref_lj_energy"]) < 1e-5 * scale
    assert abs(r["e_coul"] - m["ref_direct_energy"]) < 1e-5 * scale
    vs = np.abs(r["virial"]).max()
    assert np.abs(r["virial"] - z["ref_virial_sum"]).max() < 1e-5 * vs


ORTHO = [c for c in CASES if not c.startswith("triclinic")]


@pytest.mark.parametrize("name", ORTHO)
def test_direct_sum_equals_list_sum_at_build(oracle, name):
    """Orthorhombic cells: at build time the list sum is the direct pair sum,
    the list misses no pair inside the cutoff."""
    s, z, m = load_case(name)
    counts, lists = oracle.nl_build(s, mode=0)
    a = oracle.pair_force(s, counts, lists, per_atom=False)
    b = oracle.direct_sum(s)
    assert a["pairs_in_cutoff"] == b["pairs_in_cutoff"]
    assert rel_rms(a["frc"], b["frc"]) < 1e-12


def test_reference_stencil_misses_pairs_in_skewed_cells(oracle):
    """A property of the reference, reproduced on purpose: for a cell whose
    a21 spans more than two grid cells, the stencil rule of
    neighbor_list.cpp:18-43 leaves out some pairs inside the cutoff.  The
    golden list (the reference's own) has them missing too, so parity for
    triclinic cells is taken against the FP64 sum over the reference list."""
    s, z, m = load_case("triclinic_5500")
    counts, lists = oracle.nl_build(s, mode=0)
    a = oracle.pair_force(s, counts, lists, per_atom=False)
    b = oracle.direct_sum(s)
    missing = b["pairs_in_cutoff"] - a["pairs_in_cutoff"]
    assert 0 < missing < 1e-3 * b["pairs_in_cutoff"]


@pytest.mark.parametrize("name", CASES)
def test_long_range_factor(oracle, name):
    s, z, m = load_case(name)
    f = oracle.long_range_factor(s)
    assert abs(f - m["ref_long_range_factor"]) <= 1e-6 * abs(f)


def test_gromacs_lj_sr_pin(oracle):
    """The alanine-dipeptide/TIP3P input of the reference's GROMACS suite:
    LJ short-range energy within that suite's 25 kcal/mol of GROMACS."""
    s, z, m = load_case("ala_tip3p")
    counts, lists = oracle.nl_build(s, mode=0)
    r = oracle.pair_force(s, counts, lists, per_atom=False)
    assert abs(r["e_lj"] - m["gromacs_lj_sr"]) <= m["gromacs_lj_sr_tolerance"]


def test_contraction_modes_agree_on_fixtures(oracle):
    """The FP32 candidate test with and without fused multiply-adds selects
    the same pairs on these inputs (the GPU build uses the fused order)."""
    for name in CASES:
        s, z, m = load_case(name)
        c0, l0 = oracle.nl_build(s, mode=0)
        c1, l1 = oracle.nl_build(s, mode=1)
        assert np.array_equal(c0, c1) and np.array_equal(l0, l1), name


def test_planted_mistake_is_caught(oracle):
    """A one-ulp change of the candidate radius in the oracle (planted on the
    CPU) changes the list, so the list comparisons above have teeth."""
    s, z, m = load_case("water_1944")
    counts, lists = oracle.nl_build(s, mode=0)
    s2 = load_case("water_1944")[0]
    s2.skin = float(np.nextafter(np.float32(s.skin), np.float32(0)))
    c2, l2 = oracle.nl_build(s2, mode=0)
    assert c2.sum() <= counts.sum()
