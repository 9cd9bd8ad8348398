"""Systems with type tables of their own in one batch and in a pool.

Each SPONGE process reads its own LJ_in_file (Lennard_Jones_force.cpp:186-231),
so systems batched together may each have a different table.  A batch of
systems with 22, 9 and 30 types (the first table the batch's, the others
carried by their systems) must give every system the forces, energies,
virial and long-range term of the FP64 oracle on its own table, the same
results alone and in the mix, and a pool must admit a system with a table of
its own up to its max_types and refuse one above.
"""
import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu

FORCE_REL_RMS_TOL = 1e-5
ENERGY_REL_TOL = 1e-5
SPGNB_E_UNSUPPORTED = 8


def _mixed_tables():
    from spgnb import systems as S
    shared = S.batch_systems(2, seed=21, n_min=1500, n_max=3000)
    own9 = S.water_system(700, 29.0, 31, n_solute=150, cutoff=10.0, n_solute_types=7, name="own-9")
    own30 = S.water_system(900, 31.0, 32, n_solute=260, cutoff=8.0, n_solute_types=28, name="own-30")
    systems = [shared[0], own9, shared[1], own30]
    assert [s.n_types for s in systems] == [22, 9, 22, 30]
    return systems


def _check_vs_fp64(oracle, k, s, frc, e):
    ref = oracle.direct_sum(s)
    err = rel_rms(frc, ref["frc"])
    assert err <= FORCE_REL_RMS_TOL, f"system {k} ({s.n_types} types): force rel RMS {err:.3e}"
    scale = abs(ref["e_lj"]) + abs(ref["e_coul"])
    assert abs(e[0] - ref["e_lj"]) <= ENERGY_REL_TOL * abs(ref["e_lj"]) + 1e-3, k
    assert abs(e[2] - ref["e_coul"]) <= ENERGY_REL_TOL * scale + 1e-3, k
    assert np.abs(e[3:] - ref["virial"]).max() <= ENERGY_REL_TOL * np.abs(ref["virial"]).max() + 1e-3, k
    assert abs(e[1] - oracle.long_range_factor(s) / s.volume) <= 1e-6 * abs(e[1]) + 1e-9, k


def test_batch_with_tables_of_their_own_vs_fp64(torch_cuda, oracle):
    from spgnb.batch import Batch
    systems = _mixed_tables()
    b = Batch(systems)
    e = b.energies()
    for k, s in enumerate(systems):
        _, _, frc = b.download(k)
        _check_vs_fp64(oracle, k, s, frc, e[k])
    b.close()


def test_tables_of_their_own_same_alone_and_in_the_mix(torch_cuda):
    from spgnb.batch import Batch
    systems = _mixed_tables()
    mix = Batch(systems, thermostat_tau=0.05)
    mix.run(30, energy_interval=10)
    e_mix = mix.energies()
    for k in (1, 3):
        alone = Batch([systems[k]], thermostat_tau=0.05)
        alone.run(30, energy_interval=10)
        for x, y, what in zip(alone.download(0), mix.download(k), ("crd", "vel", "frc")):
            assert np.array_equal(x, y), f"system {k}: {what} differs alone vs in the batch"
        assert np.array_equal(alone.energies()[0], e_mix[k])
        alone.close()
    mix.close()


def test_pool_admits_tables_up_to_max_types(torch_cuda, oracle):
    from spgnb._lib import SpgnbError
    from spgnb.batch import Pool, pool_options
    systems = _mixed_tables()
    pool = Pool(systems[0], pool=pool_options(max_systems=8, max_atoms=1 << 16, max_types=30))
    ids = [pool.admit(s) for s in systems]
    assert None not in ids
    pool.evaluate(ids)
    e = pool.energies()
    for k, s in zip(ids, systems):
        _, _, frc = pool.download(k)
        _check_vs_fp64(oracle, k, s, frc, e[k])
    # the retired system's table room is reused
    pool.retire(ids[3])
    again = pool.admit(systems[3])
    assert again is not None
    pool.close()
    # a pool sized for its own table's 22 types refuses a 30-type system
    small = Pool(systems[0], pool=pool_options(max_systems=4, max_atoms=1 << 15))
    with pytest.raises(SpgnbError) as exc:
        small.admit(systems[3])
    assert exc.value.status == SPGNB_E_UNSUPPORTED
    assert small.admit(systems[1]) is not None
    small.close()
