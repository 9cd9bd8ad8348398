"""4-site water (the 4-point variant of SOLVENT_LENNARD_JONES, solvent_LJ.cpp:25-145
with WAT_POINTS = 4): waters O, H, H, M with the charge on the massless site
M.  The pruned-list path and the reference-layout path (LJ module for the
solutes + 4-point solvent module for the waters) against the FP64 direct pair
sum, and against the reference's own CUDA kernels on the same inputs."""
import os

import numpy as np
import pytest

from conftest import ROOT, rel_rms

pytestmark = pytest.mark.gpu

FORCE_REL_RMS_TOL = 1e-5
ENERGY_REL_TOL = 1e-5


def _system(n_solute=0):
    from spgnb import systems as S
    return S.water_system(800, 29.0, 31, n_solute=n_solute, cutoff=8.0, skin=2.0, water_points=4, name="tip4p-3200")


@pytest.mark.parametrize("n_solute", [0, 150])
def test_water4_pruned_list_path_vs_fp64(torch_cuda, oracle, n_solute):
    from spgnb.engine import PlainPath
    s = _system(n_solute)
    p = PlainPath(s, device="cuda:0")
    frc = p.force(need_energy=True, need_virial=True).cpu().numpy()
    ref = oracle.direct_sum(s)
    err = rel_rms(frc, ref["frc"])
    assert err <= FORCE_REL_RMS_TOL, f"force rel RMS {err:.3e}"
    tot = p.lj.totals()
    assert abs(tot[0] - ref["e_lj"]) <= ENERGY_REL_TOL * abs(ref["e_lj"]) + 1e-3
    assert abs(tot[1] - ref["e_coul"]) <= ENERGY_REL_TOL * (abs(ref["e_lj"]) + abs(ref["e_coul"])) + 1e-3


@pytest.mark.parametrize("n_solute", [0, 150])
def test_water4_solvent_module_vs_fp64(torch_cuda, oracle, n_solute):
    torch = torch_cuda
    from spgnb.engine import PlainPath
    s = _system(n_solute)
    p = PlainPath(s, export_atom_groups=True, device="cuda:0")
    assert p.solvent.water_points == 4 and p.solvent_numbers == 4 * s.n_waters
    frc = torch.zeros_like(p.frc)
    p.lj.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(p.n, p.n, p.solvent_numbers, 0, p.crd, p.charge, frc,
                                                         s.cell, s.rcell, p.nl.d_nl, s.beta, 1, p.atom_energy, 1,
                                                         p.atom_virial, p.atom_direct)
    p.solvent.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(p.n, len(s.res_len), p.res_start, p.crd, p.charge,
                                                              frc, s.cell, s.rcell, p.nl.d_nl, s.beta, 1,
                                                              p.atom_energy, 1, p.atom_virial, p.atom_direct)
    ref = oracle.direct_sum(s)
    err = rel_rms(frc.cpu().numpy(), ref["frc"])
    assert err <= FORCE_REL_RMS_TOL, f"force rel RMS {err:.3e}"


REF_CUDA = os.path.join(ROOT, "oracle", "_ref", "libspgref_cuda.so")


@pytest.mark.skipif(not os.path.exists(REF_CUDA), reason="reference CUDA harness not built")
def test_water4_matches_reference_gpu_kernels(torch_cuda, oracle):
    import oracle as O
    from spgnb.engine import PlainPath
    s = _system(150)
    ref = O.Reference(gpu=True)
    ref.init(s, refresh_interval=20, solvent=True)
    ref.nl_update(forced=True)
    rc, rl, _ = ref.nl_get()
    p = PlainPath(s, export_atom_groups=True, device="cuda:0")
    counts, lists = p.nl.host_atom_groups()
    assert np.array_equal(counts, rc) and np.array_equal(lists, rl)
    r = ref.force()
    ours = p.force(need_energy=True, need_virial=True).cpu().numpy()
    fp64 = oracle.direct_sum(s)["frc"]
    e_ours, e_ref, e_diff = rel_rms(ours, fp64), rel_rms(r["frc"], fp64), rel_rms(ours, r["frc"])
    assert e_ours <= FORCE_REL_RMS_TOL
    assert e_diff <= FORCE_REL_RMS_TOL or (e_ref > FORCE_REL_RMS_TOL - e_ours and e_ours < e_ref), \
        (e_ours, e_ref, e_diff)
    ref.clear()
