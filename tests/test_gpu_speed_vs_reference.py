"""The reference's own CUDA kernels timed beside this library on the same GPU
and the same 96,000-atom box, both driven by the same C++ harness loop
(oracle/ref_harness.cpp) through SPONGE's own module classes: once built from
the reference's sources, once built with the drop-in shim over libspgnb.
Paths: the plain LJ + PME direct path (list update + LJ + solvent modules,
Main_Calculate_Force) and the alchemical path (list update + LJ_SOFT_CORE +
the solvent module) with a 40-atom perturbed ligand.  Both sides rebuild the
list every 20 steps and compute energy and virial every step.  Prints one
JSON line per path (run with -s); fails only if this library is clearly
slower than the reference kernels."""
import json
import os

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

REF_CUDA = os.path.join(ROOT, "oracle", "_ref", "libspgref_cuda.so")
REF_SHIM = os.path.join(ROOT, "oracle", "_ref", "libspgref_shim.so")
STEPS = 300
REFRESH = 20


def _harness_times(shim, s, f):
    import oracle as O
    ref = O.Reference(gpu=not shim, shim=shim)
    ref.init(s, refresh_interval=REFRESH, solvent=True)
    ref.nl_update(forced=True)
    ref.time_steps(10, need_energy=True, need_virial=True)
    t_plain = ref.time_steps(STEPS, first_step=10, need_energy=True, need_virial=True)
    ref.clear()
    ref.init(f.system(), refresh_interval=REFRESH, solvent=True)
    ref.nl_update(forced=True)
    ref.soft_init(f)
    ref.soft_time_steps(10, need_energy=True, need_virial=True)
    t_soft = ref.soft_time_steps(STEPS, first_step=10, need_energy=True, need_virial=True)
    ref.clear()
    return t_plain, t_soft


@pytest.mark.skipif(not (os.path.exists(REF_CUDA) and os.path.exists(REF_SHIM)),
                    reason="reference CUDA harness or drop-in harness not built")
def test_plain_and_soft_core_paths_vs_reference_kernels(torch_cuda):
    from spgnb import systems as S
    s = S.mixed_box_96k()
    f = S.fep_system(s, n_perturbed=40, seed=11, lam=0.6)
    theirs = _harness_times(False, s, f)
    ours = _harness_times(True, s, f)
    out = {}
    for k, name in enumerate(("plain", "soft_core")):
        out[name] = {"atoms": s.n, "steps": STEPS, "ours_atom_steps_per_s": s.n * STEPS / ours[k],
                     "reference_kernels_atom_steps_per_s": s.n * STEPS / theirs[k],
                     "ours_ms_per_step": ours[k] * 1e3 / STEPS, "reference_ms_per_step": theirs[k] * 1e3 / STEPS,
                     "speedup": theirs[k] / ours[k]}
        print(json.dumps({"path": name, **out[name]}))
    assert out["plain"]["speedup"] > 0.8
    assert out["soft_core"]["speedup"] > 0.8
