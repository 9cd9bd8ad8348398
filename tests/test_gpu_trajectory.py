"""Config 0 as dynamics beside the reference's own integrator.

The 6,480-atom water box (2,160 rigid TIP3P-geometry waters, rc 10 A, skin
2 A, list rebuilt every 20 steps) stepped NVE at 2 fs from the same positions
and Maxwell velocities (300 K, seeded) by

* this library's batched engine with one system: leap-frog kick/drift,
  SETTLE for the waters, the list check/update and the cluster-pair force,
  all on the device;
* the reference's own CUDA code built from its sources: NEIGHBOR_LIST and the
  LJ and solvent modules for the force (main.cpp:307-397), then
  SETTLE::Remember_Last_Coordinates, the leap-frog kernel of MD_core/nve.hpp
  and SETTLE::Do_SETTLE (constrain/settle.cpp) in Main_Iteration's order
  (main.cpp:622-710).

Compared: the LJ and direct Coulomb energies at every step, the positions and
velocities after the run, and the rigid geometry.  A second test follows the
reference's own trajectory for 1,000 steps and compares the two force paths on
its states every 10 steps.  The two integrate the same
equations in FP32 with different summation orders, so they drift apart
slowly; the bounds are set well above that drift and far below any error in
the forces, the constraints or the step order.
"""
import os

import numpy as np
import pytest

from conftest import ROOT, rel_rms

pytestmark = pytest.mark.gpu

REF_CUDA = os.path.join(ROOT, "oracle", "_ref", "libspgref_cuda.so")
STEPS = 100
ENERGY_REL_TOL = 2e-3   # per-step energies over the run, relative to the terms' size
POS_RMS_TOL = 0.1       # A, positions after the run
VEL_RMS_REL_TOL = 0.2   # velocities after the run, relative to their RMS


def _rigid_errors(crd, s):
    first = s.n - 3 * s.n_waters
    o = crd[first::3][: s.n_waters].astype(np.float64)
    h1 = crd[first + 1::3][: s.n_waters].astype(np.float64)
    h2 = crd[first + 2::3][: s.n_waters].astype(np.float64)
    d1 = np.linalg.norm(h1 - o, axis=1)
    d2 = np.linalg.norm(h2 - o, axis=1)
    dh = np.linalg.norm(h2 - h1, axis=1)
    return max(np.abs(d1 - 0.9572).max(), np.abs(d2 - 0.9572).max()), np.abs(dh - 1.5139).max()


def _diffs(crd, vel, r_crd, r_vel, s):
    d = crd.astype(np.float64) - r_crd
    L = np.array([s.cell[0], s.cell[2], s.cell[5]], np.float64)
    d -= L * np.round(d / L)
    pos = float(np.sqrt((d * d).sum(1).mean()))
    vr = float(np.sqrt(((vel - r_vel) ** 2).sum(1).mean()) / np.sqrt((r_vel ** 2).sum(1).mean()))
    return pos, vr


@pytest.mark.skipif(not os.path.exists(REF_CUDA), reason="reference CUDA harness not built")
def test_water6480_nve_trajectory_vs_reference(torch_cuda, oracle):
    import oracle as O
    from spgnb import systems as S
    from spgnb.batch import Batch
    s = S.water_box_6480()
    # checkpoints: the differences must start at rounding level after one
    # step (same integrator, constraints and forces) and grow only as the
    # dynamics amplify rounding
    marks = (1, 10, STEPS)
    ref = O.Reference(gpu=True)
    ref.init(s, refresh_interval=20, solvent=True)
    ref.nl_update(forced=True)
    assert ref.md_init(dt=0.002) == s.n_waters
    r_states, r_e, r_crd, r_vel, done = {}, [], s.crd, s.vel, 0
    for m in marks:
        r_crd, r_vel, e = ref.md_run(r_crd, r_vel, m - done, first_step=done)
        r_e.append(e)
        r_states[m] = (r_crd, r_vel)
        done = m
    r_e = np.concatenate(r_e)
    ref.clear()

    b = Batch([s], refresh_interval=20, thermostat_tau=0.0)
    ours = [b.energies()[0]]
    states = {}
    for k in range(1, STEPS + 1):
        b.run(1, 1)
        if k < STEPS:
            ours.append(b.energies()[0])
        if k in marks:
            crd, vel, _ = b.download(0)
            states[k] = (crd, vel)
    b.close()
    ours = np.array(ours)
    e_lj, e_c = ours[:, 0], ours[:, 2]
    # energies relative to the size of the terms (the direct Coulomb sum
    # cancels strongly), as in the parity tests
    scale = np.abs(r_e[:, 0]) + np.abs(r_e[:, 1])
    lj_err = np.abs(e_lj - r_e[:, 0]) / scale
    c_err = np.abs(e_c - r_e[:, 1]) / scale
    fp = oracle.direct_sum(s)
    fp_scale = abs(fp["e_lj"]) + abs(fp["e_coul"])
    step0 = {"ours_lj": abs(e_lj[0] - fp["e_lj"]) / fp_scale, "ours_coul": abs(e_c[0] - fp["e_coul"]) / fp_scale,
             "ref_lj": abs(r_e[0, 0] - fp["e_lj"]) / fp_scale, "ref_coul": abs(r_e[0, 1] - fp["e_coul"]) / fp_scale}
    diffs = {m: _diffs(*states[m], *r_states[m], s) for m in marks}
    crd = states[STEPS][0]
    bond_ours, hh_ours = _rigid_errors(crd, s)
    bond_ref, hh_ref = _rigid_errors(r_states[STEPS][0], s)
    print({"case": "water-6480 NVE", "steps": STEPS, "step0_vs_fp64": step0,
           "energy_rel_at": {m: (float(lj_err[m - 1]), float(c_err[m - 1])) for m in marks},
           "pos_rms_A_and_vel_rel_at": diffs, "bond_err_ours": bond_ours, "bond_err_ref": bond_ref})
    # step 0 is the same positions: ours within 1e-5 of FP64, and of the
    # reference within both sides' error
    assert step0["ours_lj"] <= 1e-5 and step0["ours_coul"] <= 1e-5
    assert lj_err[0] <= max(1e-5, 2 * step0["ref_lj"]) and c_err[0] <= max(1e-5, 2 * step0["ref_coul"])
    # one step: rounding level
    assert diffs[1][0] <= 1e-5 and diffs[1][1] <= 1e-4
    # ten steps: still far below any physical difference
    assert diffs[10][0] <= 1e-4 and diffs[10][1] <= 1e-3
    # the run: the amplified rounding of a hot, strained start
    assert lj_err.max() <= ENERGY_REL_TOL and c_err.max() <= ENERGY_REL_TOL
    assert diffs[STEPS][0] <= POS_RMS_TOL and diffs[STEPS][1] <= VEL_RMS_REL_TOL
    # both keep the waters rigid to FP32 precision
    assert bond_ours <= 1e-4 and hh_ours <= 1e-4
    assert bond_ref <= 1e-4 and hh_ref <= 1e-4


@pytest.mark.skipif(not os.path.exists(REF_CUDA), reason="reference CUDA harness not built")
def test_water6480_force_energy_virial_along_1000_reference_steps(torch_cuda, oracle):
    """1,000 NVE steps of the reference's own force path, leap-frog and
    SETTLE from the Maxwell start; every 10 steps this library and the
    reference's kernels evaluate forces, energies and virial on the
    reference's state (each with a list built there): forces within 1e-5
    relative RMS of each other, the totals within 1e-5 of the terms' size,
    and every 20th state against the FP64 pair sum."""
    import copy
    import torch
    import oracle as O
    from spgnb import systems as S
    from spgnb.engine import PlainPath
    s = S.water_box_6480()
    ref = O.Reference(gpu=True)
    ref.init(s, refresh_interval=20, solvent=True)
    ref.nl_update(forced=True)
    assert ref.md_init(dt=0.002) == s.n_waters
    p = PlainPath(s, refresh_interval=20)
    crd, vel = s.crd, s.vel
    worst = {"force": 0.0, "e": 0.0, "virial": 0.0, "fp64": 0.0}
    for k in range(100):
        crd, vel, _ = ref.md_run(crd, vel, 10, first_step=10 * k)
        ref.nl_update(crd, step=10 * (k + 1), forced=True)
        r = ref.force(crd)
        p.crd.copy_(torch.from_numpy(np.ascontiguousarray(crd, np.float32)))
        p.update(0, forced=True)
        f = p.force(need_energy=True, need_virial=True).cpu().numpy()
        tot = p.lj.totals()
        e_lj, e_c = float(r["atom_lj"].astype(np.float64).sum()), float(r["atom_direct"].astype(np.float64).sum())
        vir = r["atom_virial"].astype(np.float64).sum(0)
        scale = abs(e_lj) + abs(e_c)
        worst["force"] = max(worst["force"], rel_rms(f, r["frc"]))
        worst["e"] = max(worst["e"], abs(tot[0] - e_lj) / scale, abs(tot[1] - e_c) / scale)
        worst["virial"] = max(worst["virial"], float(np.abs(tot[2:] - vir).max() / np.abs(vir).max()))
        if k % 20 == 19:
            st = copy.copy(s)
            st.crd = np.ascontiguousarray(crd, np.float32)
            worst["fp64"] = max(worst["fp64"], rel_rms(f, oracle.direct_sum(st)["frc"]))
    ref.clear()
    print({"case": "water-6480 along 1000 reference steps", **worst})
    assert worst["force"] <= 1e-5 and worst["fp64"] <= 1e-5
    assert worst["e"] <= 1e-5 and worst["virial"] <= 1e-5
    # the states stayed physical: rigid waters
    bond, hh = _rigid_errors(crd, s)
    assert bond <= 1e-4 and hh <= 1e-4
