"""CPU checks of the soft-core oracle: the FP64 restatement against the golden
fixtures from the reference's own CPU build of LJ_SOFT_CORE
(tests/golden/make_golden_soft.py), dH/dlambda against finite differences of
the energy, and the two-state sum reducing to the one-state sum when the
states agree."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, rel_rms

GOLDEN = os.path.join(ROOT, "tests", "golden")
META = json.load(open(os.path.join(GOLDEN, "soft_core.json")))
CASES = sorted(META)


def load_soft(name):
    from spgnb import systems as S
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    m = META[name]
    base = S.System(crd=z["crd"], charge=z["charge"], atom_type=z["type_a"], pair_A=z["AA"], pair_B=z["AB"],
                    n_types=m["n_types_a"], excl_start=z["excl_start"], excl_numbers=z["excl_numbers"],
                    excl_list=z["excl_list"], mass=z["mass"], res_start=z["res_start"], res_len=z["res_len"],
                    cell=z["cell"], rcell=z["rcell"], cutoff=m["cutoff"], skin=m["skin"], beta=m["beta"],
                    n_solute=m["n_solute"], name=name)
    prm = z["params"]
    f = S.FepSystem(base=base, type_a=z["type_a"], type_b=z["type_b"], n_types_a=m["n_types_a"],
                    n_types_b=m["n_types_b"], AA=z["AA"], AB=z["AB"], BA=z["BA"], BB=z["BB"],
                    charge_a=z["charge_a"], charge_b=z["charge_b"], lam=float(prm[0]), alpha=float(prm[1]),
                    p=float(prm[2]), sigma=float(prm[3]), sigma_min=float(prm[4]), changed=z["changed"])
    assert np.array_equal(f.charge(), z["charge"])
    return f, z, m


@pytest.mark.parametrize("name", CASES)
def test_soft_oracle_matches_reference_cpu_build(oracle, name):
    f, z, m = load_soft(name)
    r = oracle.soft_core(f)
    # the reference computes in FP32 over its own list: agree to FP32 error
    assert rel_rms(z["ref_frc"], r["frc"]) < 1e-5
    scale = abs(r["e_lj"]) + abs(r["e_coul"])
    assert abs(r["e_lj"] - m["ref_lj_energy"]) < 1e-5 * scale
    assert abs(r["e_coul"] - m["ref_direct_energy"]) < 1e-5 * scale
    assert np.abs(r["virial"] - z["ref_virial_sum"]).max() < 1e-5 * np.abs(r["virial"]).max()
    # per-atom energies go to the lower-index atom of each pair, as the reference's half list
    e_ref = z["ref_atom_lj"].astype(np.float64)
    assert np.abs(r["e_lj_atom"] - e_ref).max() < 1e-4 * np.abs(e_ref).max()
    lr, lr_ti = oracle.soft_long_range(f)
    assert abs(lr - m["ref_long_range_factor"]) < 1e-6 * abs(lr)
    assert abs(lr_ti - m["ref_long_range_factor_ti"]) < 1e-6 * abs(lr_ti)
    # Get_Partial_H_Partial_Lambda_With_Columb_Direct = pair sum + factor_TI / V (float)
    vol = float(np.float32(z["cell"][0]) * np.float32(z["cell"][2]) * np.float32(z["cell"][5]))
    dh = r["dh_lj"] + lr_ti / vol
    assert abs(dh - m["ref_dhdl_lj"]) < 2e-5 * (abs(dh) + 10.0)
    assert abs(r["dh_c"] - m["ref_dhdl_direct"]) < 2e-5 * (abs(r["dh_c"]) + 10.0)


@pytest.mark.parametrize("name", CASES)
def test_soft_dhdl_is_the_lambda_derivative(oracle, name):
    """dH/dlambda (LJ and direct Coulomb, charges linear in lambda) against a
    central difference of the oracle's energies, with the float32 steps."""
    f, z, m = load_soft(name)
    lam = f.lam
    r = oracle.soft_core(f, per_atom=False)
    h = 1e-3
    up = oracle.soft_core(f, lam=lam + h, per_atom=False)
    dn = oracle.soft_core(f, lam=lam - h, per_atom=False)
    step = float(np.float32(lam + h)) - float(np.float32(lam - h))
    fd_lj = (up["e_lj"] - dn["e_lj"]) / step
    fd_c = (up["e_coul"] - dn["e_coul"]) / step
    assert abs(fd_lj - r["dh_lj"]) < 1e-4 * (abs(r["dh_lj"]) + 10.0)
    assert abs(fd_c - r["dh_c"]) < 1e-4 * (abs(r["dh_c"]) + 10.0)


def test_soft_sum_reduces_to_plain_sum_when_states_agree(oracle):
    from spgnb import systems as S
    b = S.water_system(700, 28.5, 31, n_solute=80, cutoff=8.0, skin=2.0)
    f = S.fep_system(b, n_perturbed=12, seed=3, kinds=("mutate",), permute_b=True, bond_perturbed=False)
    # undo the mutation: state B = state A under B's own numbering
    unchanged = np.setdiff1d(np.arange(b.n), f.changed)
    tb_of_ta = {}
    for ta, tb in zip(f.type_a[unchanged], f.type_b[unchanged]):
        assert tb_of_ta.setdefault(int(ta), int(tb)) == int(tb)
    same = S.FepSystem(base=f.base, type_a=f.type_a,
                       type_b=np.array([tb_of_ta.get(int(t), 0) for t in f.type_a], np.int32),
                       n_types_a=f.n_types_a, n_types_b=f.n_types_b, AA=f.AA, AB=f.AB, BA=f.BA, BB=f.BB,
                       charge_a=f.charge_a, charge_b=f.charge_a, lam=0.37)
    assert np.array_equal(same.type_b[unchanged], f.type_b[unchanged])
    r = oracle.soft_core(same)
    p = oracle.direct_sum(b)
    assert r["pairs_in_cutoff"] == p["pairs_in_cutoff"]
    assert rel_rms(r["frc"], p["frc"]) < 1e-12
    assert abs(r["e_lj"] - p["e_lj"]) < 1e-9 * abs(p["e_lj"])
    assert abs(r["dh_lj"]) < 1e-9 and abs(r["dh_c"]) < 1e-9
