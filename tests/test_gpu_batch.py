"""Batched engine on the GPU: forces against the FP64 oracle, results that do
not depend on the batch, graph replay equal to step-by-step launches, rigid
waters kept rigid."""
import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu

FORCE_REL_RMS_TOL = 1e-5
ENERGY_REL_TOL = 1e-5


def _small_batch(k=3, seed=11):
    from spgnb import systems as S
    return S.batch_systems(k, seed=seed, n_min=1500, n_max=4000)


def test_batch_initial_forces_vs_fp64(torch_cuda, oracle):
    from spgnb.batch import Batch
    systems = _small_batch()
    b = Batch(systems)
    for k, s in enumerate(systems):
        _, _, frc = b.download(k)
        ref = oracle.direct_sum(s)
        err = rel_rms(frc, ref["frc"])
        assert err <= FORCE_REL_RMS_TOL, f"system {k}: force rel RMS {err:.3e}"
    e = b.energies()
    for k, s in enumerate(systems):
        ref = oracle.direct_sum(s)
        # FP32 pair terms summed exactly: the error scales with the terms' size
        scale = abs(ref["e_lj"]) + abs(ref["e_coul"])
        assert abs(e[k, 0] - ref["e_lj"]) <= ENERGY_REL_TOL * abs(ref["e_lj"]) + 1e-3
        assert abs(e[k, 2] - ref["e_coul"]) <= ENERGY_REL_TOL * scale + 1e-3
        vir_scale = np.abs(ref["virial"]).max()
        assert np.abs(e[k, 3:] - ref["virial"]).max() <= ENERGY_REL_TOL * vir_scale + 1e-3
        assert abs(e[k, 1] - oracle.long_range_factor(s) / s.volume) <= 1e-6 * abs(e[k, 1]) + 1e-9
    b.close()


def test_batch_result_same_alone_and_in_the_mix(torch_cuda):
    from spgnb.batch import Batch
    systems = _small_batch(3, seed=12)
    mix = Batch(systems)
    mix.run(40, energy_interval=10)
    e_mix = mix.energies()
    for k, s in enumerate(systems):
        alone = Batch([s])
        alone.run(40, energy_interval=10)
        a = alone.download(0)
        m = mix.download(k)
        for x, y, what in zip(a, m, ("crd", "vel", "frc")):
            assert np.array_equal(x, y), f"system {k}: {what} differs alone vs in the batch"
        assert np.array_equal(alone.energies()[0], e_mix[k])
        alone.close()
    mix.close()


def test_graph_replay_equals_step_launches(torch_cuda):
    from spgnb.batch import Batch
    systems = _small_batch(2, seed=13)
    g = Batch(systems, use_graphs=1, steps_per_graph=5)
    d = Batch(systems, use_graphs=0)
    g.run(20, energy_interval=5)
    d.run(20, energy_interval=5)
    for k in range(len(systems)):
        for x, y in zip(g.download(k), d.download(k)):
            assert np.array_equal(x, y)
    assert np.array_equal(g.energies(), d.energies())
    g.close()
    d.close()


def test_rigid_waters_stay_rigid(torch_cuda):
    from spgnb.batch import Batch
    systems = _small_batch(2, seed=14)
    b = Batch(systems)
    b.run(200)
    for k, s in enumerate(systems):
        crd, vel, frc = b.download(k)
        assert np.isfinite(crd).all() and np.isfinite(vel).all() and np.isfinite(frc).all()
        o = s.n_solute + 3 * np.arange(s.n_waters)
        doh1 = np.linalg.norm(crd[o + 1] - crd[o], axis=1)
        doh2 = np.linalg.norm(crd[o + 2] - crd[o], axis=1)
        dhh = np.linalg.norm(crd[o + 2] - crd[o + 1], axis=1)
        assert np.abs(doh1 - 0.9572).max() < 2e-4
        assert np.abs(doh2 - 0.9572).max() < 2e-4
        assert np.abs(dhh - 1.5139).max() < 3e-4
    st = b.stats()
    assert st["overflow"] == 0 and st["steps"] == 200
    b.close()


def test_launch_configuration_changes_no_result(torch_cuda):
    """The autotuner's knobs other than the prune buffer (the force and
    pruning kernels' grids, the steps per graph) change no bit of the
    results.  Applying a tuning re-prunes the lists, and the list words'
    order decides the FP32 partial sums, so both batches apply one at the
    same step."""
    from spgnb.batch import Batch
    systems = _small_batch(2, seed=15)
    a = Batch(systems, steps_per_graph=10)
    b = Batch(systems, steps_per_graph=10)
    buf = a.tuning()["prune_buffer"]
    a.set_tuning(buf, 0, 5, 10)
    b.set_tuning(buf, 2, 3, 5)
    assert b.tuning()["pair_blocks_per_sm"] == 2 and b.tuning()["steps_per_graph"] == 5
    a.run(30, energy_interval=10)
    b.run(30, energy_interval=10)
    for k in range(len(systems)):
        for x, y in zip(a.download(k), b.download(k)):
            assert np.array_equal(x, y)
    assert np.array_equal(a.energies(), b.energies())
    a.close()
    b.close()


def test_autotune_picks_among_candidates(torch_cuda):
    from spgnb.batch import Batch
    b = Batch(_small_batch(2, seed=16), prune_buffer=1.6)
    buf = b.autotune(5)
    t = b.tuning()
    assert buf == t["prune_buffer"] and 0.4 <= buf <= 1.6
    assert t["pair_blocks_per_sm"] in (0, 2, 3) and t["prune_blocks_per_sm"] in (3, 5, 8)
    assert t["steps_per_graph"] in (5, 10, 20) and t["ms_per_step"] > 0
    b.run(20)
    st = b.stats()
    assert st["overflow"] == 0
    b.close()
