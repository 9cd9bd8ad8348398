"""The reference's own CUDA kernels timed beside this library on the same GPU
and the same 96,000-atom box, both driven by the same C++ harness loop
(oracle/ref_harness.cpp) through SPONGE's own module classes: once built from
the reference's sources, once built with the drop-in shim over libspgnb.
Paths: the plain LJ + PME direct path (list update + LJ + solvent modules,
Main_Calculate_Force) and the alchemical path (list update + LJ_SOFT_CORE +
the solvent module) with a 40-atom perturbed ligand.  Both sides rebuild the
list every 20 steps; each path is timed with energy and virial (per-atom
arrays) every step and with forces only, SPONGE's step between energy
outputs.  Prints one JSON line per path (run with -s); fails when force-only
steps are not at least 1.5x the reference kernels' speed, or energy steps
not at least 1.1x."""
import json
import os

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

REF_CUDA = os.path.join(ROOT, "oracle", "_ref", "libspgref_cuda.so")
REF_SHIM = os.path.join(ROOT, "oracle", "_ref", "libspgref_shim.so")
# steps per timed loop; a launch-list capture of this test under a profiler
# sets fewer, and then only prints (serialised launches time nothing)
STEPS = int(os.environ.get("SPGNB_SPEED_STEPS", "300"))
UNDER_PROFILER = "SPGNB_SPEED_STEPS" in os.environ
REFRESH = 20


def _timed(fn):
    """fn() inside the NVTX range 'timed', so that a launch list of this
    test (ncu --nvtx --nvtx-include timed/) holds the timed steps only."""
    import torch
    torch.cuda.nvtx.range_push("timed")
    try:
        return fn()
    finally:
        torch.cuda.nvtx.range_pop()


def _harness_times(shim, s, f):
    """{(path, energy and virial?): seconds for STEPS steps}."""
    import oracle as O
    out = {}
    ref = O.Reference(gpu=not shim, shim=shim)
    ref.init(s, refresh_interval=REFRESH, solvent=True)
    ref.nl_update(forced=True)
    for ev in (True, False):
        ref.time_steps(10, need_energy=ev, need_virial=ev)
        out[("plain", ev)] = _timed(lambda: ref.time_steps(STEPS, first_step=10, need_energy=ev, need_virial=ev))
    ref.clear()
    ref.init(f.system(), refresh_interval=REFRESH, solvent=True)
    ref.nl_update(forced=True)
    ref.soft_init(f)
    for ev in (True, False):
        ref.soft_time_steps(10, need_energy=ev, need_virial=ev)
        out[("soft_core", ev)] = _timed(
            lambda: ref.soft_time_steps(STEPS, first_step=10, need_energy=ev, need_virial=ev))
    ref.clear()
    return out


@pytest.mark.skipif(not (os.path.exists(REF_CUDA) and os.path.exists(REF_SHIM)),
                    reason="reference CUDA harness or drop-in harness not built")
def test_plain_and_soft_core_paths_vs_reference_kernels(torch_cuda):
    from spgnb import systems as S
    s = S.mixed_box_96k()
    f = S.fep_system(s, n_perturbed=40, seed=11, lam=0.6)
    theirs = _harness_times(False, s, f)
    ours = _harness_times(True, s, f)
    speedup = {}
    for key in ours:
        name, ev = key
        line = {"path": name, "energy_virial_every_step": ev, "atoms": s.n, "steps": STEPS,
                "ours_ms_per_step": ours[key] * 1e3 / STEPS, "reference_ms_per_step": theirs[key] * 1e3 / STEPS,
                "speedup": theirs[key] / ours[key]}
        speedup[key] = line["speedup"]
        print(json.dumps(line))
    if UNDER_PROFILER:
        return
    for (name, ev), v in speedup.items():
        # measured 1.93x (force-only, SPONGE's step between energy outputs)
        # and 1.26x (per-atom energy and virial every step); the floors leave
        # room for host-clock loops on a shared box
        assert v >= (1.1 if ev else 1.5), (name, ev, v)
