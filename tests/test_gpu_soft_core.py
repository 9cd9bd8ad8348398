"""LJ_SOFT_CORE (alchemical LJ + PME direct space with soft cores,
LJ_soft_core.cpp:198-436) on the GPU through the C ABI: forces, energies,
virials and dH/dlambda against the FP64 oracle (itself pinned to the
reference's CPU build by tests/test_soft_core_cpu.py), against the
reference's own CUDA kernels on the same inputs, at lambda end points and
other soft-core parameters, and reducing to the plain module when the two
states agree."""
import os

import numpy as np
import pytest

from conftest import ROOT, rel_rms
from test_soft_core_cpu import CASES, load_soft

pytestmark = pytest.mark.gpu

FORCE_REL_RMS_TOL = 1e-5
ENERGY_REL_TOL = 1e-5
REF_CUDA = os.path.join(ROOT, "oracle", "_ref", "libspgref_cuda.so")


def _check_vs_oracle(p, f, ref, what):
    frc = p.frc.cpu().numpy()
    err = rel_rms(frc, ref["frc"])
    assert err <= FORCE_REL_RMS_TOL, f"{what}: force rel RMS {err:.3e}"
    tot = p.lj.totals()
    scale = abs(ref["e_lj"]) + abs(ref["e_coul"])
    assert abs(tot[0] - ref["e_lj"]) <= ENERGY_REL_TOL * scale + 1e-3, (what, tot[0], ref["e_lj"])
    assert abs(tot[1] - ref["e_coul"]) <= ENERGY_REL_TOL * scale + 1e-3, (what, tot[1], ref["e_coul"])
    vs = np.abs(ref["virial"]).max()
    assert np.abs(tot[2:] - ref["virial"]).max() <= ENERGY_REL_TOL * vs, what


@pytest.mark.parametrize("name", CASES)
def test_soft_core_force_energy_virial_vs_fp64(torch_cuda, oracle, name):
    from spgnb.engine import SoftCorePath
    f, z, m = load_soft(name)
    p = SoftCorePath(f, device="cuda:0")
    assert np.array_equal(np.sort(p.lj.perturbed_atoms()), np.sort(f.changed))
    p.force(need_energy=True, need_virial=True)
    ref = oracle.soft_core(f)
    _check_vs_oracle(p, f, ref, name)
    # per-atom outputs: energy and virial of each pair with its lower-index atom
    ene = p.atom_energy.cpu().numpy().astype(np.float64)
    e_ref = ref["e_lj_atom"] + ref["e_coul_atom"]
    assert np.abs(ene - e_ref).max() <= 1e-4 * np.abs(e_ref).max()
    direct = p.atom_direct.cpu().numpy().astype(np.float64)
    assert np.abs(direct - ref["e_coul_atom"]).max() <= 1e-4 * np.abs(ref["e_coul_atom"]).max()
    vir = p.atom_virial.cpu().numpy().astype(np.float64)
    assert np.abs(vir - ref["virial_atom"]).max() <= 1e-4 * np.abs(ref["virial_atom"]).max()
    # force-only and energy-only calls give the same forces within FP32 rounding
    p.force()
    assert rel_rms(p.frc.cpu().numpy(), ref["frc"]) <= FORCE_REL_RMS_TOL


@pytest.mark.parametrize("name", CASES)
def test_soft_core_dhdl_vs_fp64(torch_cuda, oracle, name):
    from spgnb.engine import SoftCorePath
    f, z, m = load_soft(name)
    p = SoftCorePath(f, device="cuda:0")
    ref = oracle.soft_core(f, per_atom=False)
    _, lr_ti = oracle.soft_long_range(f)
    vol = float(np.float32(z["cell"][0]) * np.float32(z["cell"][2]) * np.float32(z["cell"][5]))
    want = ref["dh_lj"] + lr_ti / vol
    v, vd = p.dhdl(charge_perturbated=True)
    assert abs(v - want) <= 1e-5 * (abs(want) + 10.0), (v, want)
    assert abs(vd - ref["dh_c"]) <= 1e-5 * (abs(ref["dh_c"]) + 10.0), (vd, ref["dh_c"])
    v2, vd2 = p.dhdl(charge_perturbated=False)
    assert v2 == v and vd2 == 0.0
    # the reference's own value (its CPU build, golden)
    assert abs(v - m["ref_dhdl_lj"]) <= 2e-5 * (abs(v) + 10.0)
    assert abs(vd - m["ref_dhdl_direct"]) <= 2e-5 * (abs(vd) + 10.0)


@pytest.mark.parametrize("lam,alpha,p_pow,sigma,sigma_min", [
    (0.0, 0.5, 1.0, 3.0, 0.0), (1.0, 0.5, 1.0, 3.0, 0.0), (0.25, 0.7, 2.0, 2.5, 1.5), (0.9, 0.3, 1.0, 3.5, 0.0)])
def test_soft_core_parameters_vs_fp64(torch_cuda, oracle, lam, alpha, p_pow, sigma, sigma_min):
    from spgnb import systems as S
    from spgnb.engine import SoftCorePath
    b = S.water_system(800, 30.0, 41, n_solute=140, cutoff=9.0, skin=2.0, name="soft-params")
    f = S.fep_system(b, n_perturbed=30, seed=5, lam=lam, alpha=alpha, p=p_pow, sigma=sigma, sigma_min=sigma_min)
    p = SoftCorePath(f, device="cuda:0")
    p.force(need_energy=True, need_virial=True)
    ref = oracle.soft_core(f)
    _check_vs_oracle(p, f, ref, f"lambda={lam}")
    v, vd = p.dhdl(charge_perturbated=True)
    _, lr_ti = oracle.soft_long_range(f)
    want = ref["dh_lj"] + lr_ti / b.volume
    assert abs(v - want) <= 1e-5 * (abs(want) + 10.0)
    assert abs(vd - ref["dh_c"]) <= 1e-5 * (abs(ref["dh_c"]) + 10.0)


def test_soft_core_reduces_to_the_plain_module(torch_cuda):
    """States that agree: no perturbed atom, and the soft module gives the
    plain LJ module's forces and totals up to the order of FP32 additions."""
    from spgnb import systems as S
    from spgnb.engine import PlainPath, SoftCorePath
    b = S.water_system(900, 31.0, 43, n_solute=100, cutoff=9.0, skin=2.0)
    f = S.fep_system(b, n_perturbed=10, seed=3, kinds=("mutate",), bond_perturbed=False)
    unchanged = np.setdiff1d(np.arange(b.n), f.changed)
    tb_of_ta = {int(a): int(t) for a, t in zip(f.type_a[unchanged], f.type_b[unchanged])}
    same = S.FepSystem(base=b, type_a=f.type_a, type_b=np.array([tb_of_ta[int(t)] for t in f.type_a], np.int32),
                       n_types_a=f.n_types_a, n_types_b=f.n_types_b, AA=f.AA, AB=f.AB, BA=f.BA, BB=f.BB,
                       charge_a=f.charge_a, charge_b=f.charge_a, lam=0.4)
    p = SoftCorePath(same, device="cuda:0")
    assert len(p.lj.perturbed_atoms()) == 0
    q = PlainPath(b, device="cuda:0", solvent=False)
    a = p.force(need_energy=True, need_virial=True).cpu().numpy()
    c = q.force(need_energy=True, need_virial=True).cpu().numpy()
    assert rel_rms(a, c) <= 1e-6
    tp, tq = p.lj.totals(), q.lj.totals()
    assert np.abs(tp - tq).max() <= 1e-6 * np.abs(tq).max()
    v, vd = p.dhdl(charge_perturbated=True)
    assert vd == 0.0


def test_soft_core_large_box_vs_fp64(torch_cuda, oracle):
    """The 96,000-atom mixed box with a 40-atom perturbed ligand."""
    from spgnb import systems as S
    from spgnb.engine import SoftCorePath
    f = S.fep_system(S.mixed_box_96k(), n_perturbed=40, seed=11, lam=0.6)
    p = SoftCorePath(f, device="cuda:0")
    p.force(need_energy=True, need_virial=True, per_atom=False)
    ref = oracle.soft_core(f, per_atom=False)
    _check_vs_oracle(p, f, ref, "mixed-96k")


@pytest.mark.skipif(not os.path.exists(REF_CUDA), reason="reference CUDA harness not built")
@pytest.mark.parametrize("solvent", [False, True])
@pytest.mark.parametrize("name", CASES)
def test_soft_core_vs_reference_cuda_kernels(torch_cuda, name, solvent):
    """The reference's own Lennard_Jones_And_Direct_Coulomb_Soft_Core_CUDA on the
    same inputs (its list, its kernels, FP32), alone or with the solvent
    module taking the waters as in an alchemical run: forces and energies
    agree to FP32 accumulation error."""
    import oracle as O
    from spgnb.engine import SoftCorePath
    f, z, m = load_soft(name)
    s = f.system()
    ref = O.Reference(gpu=True)
    ref.init(s, solvent=solvent)
    ref.nl_update(forced=True)
    ref.soft_init(f)
    r = ref.soft_force(need_energy=True, need_virial=True)
    dh, dh_c = ref.soft_dhdl(charge_perturbated=True)
    ref.clear()
    p = SoftCorePath(f, device="cuda:0")
    p.force(need_energy=True, need_virial=True)
    frc = p.frc.cpu().numpy()
    assert rel_rms(frc, r["frc"]) <= FORCE_REL_RMS_TOL
    tot = p.lj.totals()
    e_lj, e_c = r["atom_lj"].astype(np.float64).sum(), r["atom_direct"].astype(np.float64).sum()
    scale = abs(e_lj) + abs(e_c)
    assert abs(tot[0] - e_lj) <= ENERGY_REL_TOL * scale
    assert abs(tot[1] - e_c) <= ENERGY_REL_TOL * scale
    v, vd = p.dhdl(charge_perturbated=True)
    assert abs(v - dh) <= 2e-5 * (abs(v) + 10.0)
    assert abs(vd - dh_c) <= 2e-5 * (abs(vd) + 10.0)


REF_SHIM = os.path.join(ROOT, "oracle", "_ref", "libspgref_shim.so")


@pytest.mark.skipif(not os.path.exists(REF_SHIM), reason="drop-in harness not built")
@pytest.mark.parametrize("name", CASES)
def test_soft_core_through_sponge_module_api(torch_cuda, oracle, name):
    """SPONGE's own LJ_SOFT_CORE class, built with the drop-in shim over
    libspgnb (sponge2.0_b200/shim/LJ_soft_core_spgnb.cpp), driven by the same
    C++ harness as the reference: Initial from Xponge's arrays, Get_Local,
    the force and dH/dlambda, against the FP64 oracle."""
    import oracle as O
    f, z, m = load_soft(name)
    ref = O.Reference(shim=True)
    ref.init(f.system())
    ref.nl_update(forced=True)
    ref.soft_init(f)
    r = ref.soft_force(need_energy=True, need_virial=True)
    dh, dh_c = ref.soft_dhdl(charge_perturbated=True)
    lr, lr_ti = ref.soft_long_range()
    ref.clear()
    o = oracle.soft_core(f)
    assert rel_rms(r["frc"], o["frc"]) <= FORCE_REL_RMS_TOL
    scale = abs(o["e_lj"]) + abs(o["e_coul"])
    assert abs(r["atom_lj"].astype(np.float64).sum() - o["e_lj"]) <= ENERGY_REL_TOL * scale
    assert abs(r["atom_direct"].astype(np.float64).sum() - o["e_coul"]) <= ENERGY_REL_TOL * scale
    olr, olr_ti = oracle.soft_long_range(f)
    assert abs(lr - olr) <= 1e-6 * abs(olr) and abs(lr_ti - olr_ti) <= 1e-6 * abs(olr_ti)
    want = o["dh_lj"] + olr_ti / f.base.volume
    assert abs(dh - want) <= 2e-5 * (abs(want) + 10.0)
    assert abs(dh_c - o["dh_c"]) <= 2e-5 * (abs(o["dh_c"]) + 10.0)
