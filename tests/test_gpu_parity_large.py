"""Parity at the large configurations: the ~1.0M-atom water box (rc 12 A) and
the full 256-system batch (1,500-24,000 atoms, rc 8/10/12 A).

The 1M box: the exported reference-layout list equals the oracle's
reference-rule list atom for atom (counts, and an order-independent hash of
each atom's partners), and the forces of a fixed random sample of 10,000
atoms are within 1e-5 relative RMS of their FP64 sums over all partners, in
the per-atom energy/virial mode and the force-only mode; the energy totals
match the FP64 pair sum.  The batch: the initial forces of sampled systems
(every cutoff value among them) against FP64, no overflow, finite energies.
"""
import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu

FORCE_REL_RMS_TOL = 1e-5
ENERGY_REL_TOL = 1e-5


def _set_hash(counts, lists):
    """Per-atom order-independent hash of the atom's partner list."""
    j = lists.astype(np.uint64)
    h = (j * np.uint64(0x9E3779B97F4A7C15)) ^ ((j * np.uint64(0xC2B2AE3D27D4EB4F)) >> np.uint64(29))
    cs = np.concatenate([np.zeros(1, np.uint64), np.cumsum(h, dtype=np.uint64)])
    off = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    return cs[off[1:]] - cs[off[:-1]]


def test_water1m_list_and_sampled_forces(torch_cuda, oracle):
    import torch
    from spgnb import systems as S
    from spgnb.engine import PlainPath
    s = S.water_box_1m()
    # at rc + skin = 14 A the lowest-index atoms hold nearly full lists (about
    # 1,150-1,250 partners): above SPONGE's default max_neighbor_numbers of
    # 1,200, which would overflow there in the reference too
    p = PlainPath(s, export_atom_groups=True, max_neighbor_numbers=2000)
    counts, lists = p.nl.host_atom_groups(sort=False)
    oc, ol = oracle.nl_build(s, mode=1)
    assert counts.sum() == oc.sum(), (counts.sum(), oc.sum())
    assert np.array_equal(counts, oc)
    assert np.array_equal(_set_hash(counts, lists), _set_hash(oc, ol))
    del lists, ol
    # no list overflow; the grid flag (bit 1) is set: the reference's grid
    # gives each row's last cell the remainder of the box (12.3 A of 215.3),
    # whose corner cells exceed its 150-atom buckets
    assert p.nl.stats()["overflow"] & 1 == 0
    rng = np.random.default_rng(2024)
    sample = np.sort(rng.choice(s.n, 10000, replace=False)).astype(np.int32)
    ref = oracle.direct_forces_subset(s, sample)
    for ev in (True, False):
        frc = p.force(need_energy=ev, need_virial=ev).cpu().numpy()[sample]
        err = rel_rms(frc, ref)
        print({"case": "water-1m", "energy_virial": ev, "sample_force_rel_rms": err})
        assert err <= FORCE_REL_RMS_TOL, (ev, err)
    # totals of the per-atom mode against the FP64 sum over the oracle's list
    # (each pair once, the reference rule)
    p.force(need_energy=True, need_virial=True)
    tot = p.lj.totals()
    fp = oracle.pair_force(s, oc, oracle.nl_build(s, mode=1)[1], per_atom=False)
    assert abs(tot[0] - fp["e_lj"]) <= ENERGY_REL_TOL * abs(fp["e_lj"]) + 1e-2
    assert abs(tot[1] - fp["e_coul"]) <= ENERGY_REL_TOL * (abs(fp["e_lj"]) + abs(fp["e_coul"])) + 1e-2
    vir_scale = np.abs(fp["virial"]).max()
    assert np.abs(tot[2:] - fp["virial"]).max() <= ENERGY_REL_TOL * vir_scale + 1e-2
    torch.cuda.synchronize()


def test_batch256_sampled_systems_vs_fp64(torch_cuda, oracle):
    from spgnb import systems as S
    from spgnb.batch import Batch
    systems = S.batch_systems(256)
    b = Batch(systems)
    st = b.stats()
    assert st["overflow"] == 0, st
    # eight systems spread over the size range, plus the first of every cutoff
    order = np.argsort([s.n for s in systems])
    picks = set(int(order[k]) for k in np.linspace(0, len(systems) - 1, 8).astype(int))
    for rc in sorted(set(float(s.cutoff) for s in systems)):
        picks.add(next(k for k, s in enumerate(systems) if float(s.cutoff) == rc))
    cutoffs = set()
    for k in sorted(picks):
        s = systems[k]
        _, _, frc = b.download(k)
        ref = oracle.direct_sum(s)
        err = rel_rms(frc, ref["frc"])
        print({"case": "batch256", "system": k, "atoms": s.n, "cutoff": s.cutoff, "force_rel_rms": err})
        assert err <= FORCE_REL_RMS_TOL, (k, s.n, s.cutoff, err)
        cutoffs.add(float(s.cutoff))
    assert cutoffs == set(float(s.cutoff) for s in systems)
    b.run(20, energy_interval=10)
    assert np.isfinite(b.energies()).all()
    assert b.stats()["overflow"] == 0
    b.close()
