"""The reference's own CUDA kernels timed beside this library on the same GPU
and the same 96,000-atom box: the plain LJ + PME direct path (list update +
LJ kernel + solvent kernel, Main_Calculate_Force) and the soft-core path (list
update + Lennard_Jones_And_Direct_Coulomb_Soft_Core_CUDA for the solute + the
solvent kernel for the waters) with a 40-atom perturbed ligand.  Both sides
rebuild every 20 steps and compute energy and virial every step.  Prints one
JSON line per path (run with -s to see them); fails only if this library is
clearly slower than the reference."""
import json
import os

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

REF_CUDA = os.path.join(ROOT, "oracle", "_ref", "libspgref_cuda.so")
STEPS = 200
REFRESH = 20


def _ours(step_fn, torch, steps=STEPS):
    for k in range(5):
        step_fn(k)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for k in range(steps):
        step_fn(5 + k)
    b.record()
    b.synchronize()
    return a.elapsed_time(b) * 1e-3


@pytest.mark.skipif(not os.path.exists(REF_CUDA), reason="reference CUDA harness not built")
def test_plain_and_soft_core_paths_vs_reference_kernels(torch_cuda):
    import oracle as O
    from spgnb import systems as S
    from spgnb.engine import PlainPath, SoftCorePath
    torch = torch_cuda
    s = S.mixed_box_96k()
    f = S.fep_system(s, n_perturbed=40, seed=11, lam=0.6)

    ref = O.Reference(gpu=True)
    ref.init(s, refresh_interval=REFRESH, solvent=True)
    ref.nl_update(forced=True)
    ref.time_steps(5, need_energy=True, need_virial=True)
    t_ref_plain = ref.time_steps(STEPS, first_step=5, need_energy=True, need_virial=True)
    ref.clear()
    ref = O.Reference(gpu=True)
    ref.init(f.system(), refresh_interval=REFRESH, solvent=True)
    ref.nl_update(forced=True)
    ref.soft_init(f)
    ref.soft_time_steps(5, need_energy=True, need_virial=True)
    t_ref_soft = ref.soft_time_steps(STEPS, first_step=5, need_energy=True, need_virial=True)
    ref.clear()

    p = PlainPath(s, refresh_interval=REFRESH, device="cuda:0")
    t_plain = _ours(lambda k: p.step(k, need_energy=True, need_virial=True, per_atom=True), torch)
    del p
    q = SoftCorePath(f, refresh_interval=REFRESH, device="cuda:0")
    t_soft = _ours(lambda k: q.step(k, need_energy=True, need_virial=True, per_atom=True), torch)
    del q

    out = {}
    for name, ours, theirs in (("plain", t_plain, t_ref_plain), ("soft_core", t_soft, t_ref_soft)):
        out[name] = {"atoms": s.n, "steps": STEPS, "ours_atom_steps_per_s": s.n * STEPS / ours,
                     "reference_kernels_atom_steps_per_s": s.n * STEPS / theirs,
                     "ours_ms_per_step": ours * 1e3 / STEPS, "reference_ms_per_step": theirs * 1e3 / STEPS,
                     "speedup": theirs / ours}
        print(json.dumps({"path": name, **out[name]}))
    assert out["plain"]["speedup"] > 0.8
    assert out["soft_core"]["speedup"] > 0.8
