"""Full neighbour list (FULL_NEIGHBOR_LIST::Build_From_Half[_With_Cutoff],
full_neighbor_list.cpp:27-147) built from the cluster tables on the GPU:
every pair of the reference's half list in both atoms' lists (and, with a
cutoff, exactly the pairs within it at the current coordinates), in the
same order on every call."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _half_pairs(oracle, s):
    counts, lists = oracle.nl_build(s, mode=1)
    owner = np.repeat(np.arange(s.n), counts)
    return owner, np.asarray(lists)


def _sets(n, a, b):
    out = [set() for _ in range(n)]
    for i, j in zip(a, b):
        out[i].add(int(j))
        out[j].add(int(i))
    return out


@pytest.mark.parametrize("name,cutoff_full", [("water-1944", 0.0), ("water-1944", 6.0), ("triclinic", 7.0)])
def test_full_list_matches_reference_rule(torch_cuda, oracle, name, cutoff_full):
    from spgnb import systems as S
    from spgnb.engine import PlainPath
    s = {"water-1944": lambda: S.water_system(648, 26.9, 21, cutoff=8.0, skin=2.0),
         "triclinic": lambda: S.water_system(1000, (33.0, 33.0, 33.0), 23, cutoff=8.0, skin=2.0,
                                             angles=(80.0, 95.0, 105.0))}[name]()
    p = PlainPath(s, export_atom_groups=True, device="cuda:0")
    runs = []
    for _ in range(2):
        counts, temp, ovf = p.nl.build_full(s.n, p.crd, s.cell, s.rcell, cutoff_full, 1200)
        runs.append((counts.cpu().numpy(), temp.cpu().numpy(), int(ovf.item())))
    (counts, temp, ovf), (counts2, temp2, _) = runs
    assert ovf == 0
    assert np.array_equal(counts, counts2) and np.array_equal(temp, temp2), "not the same order twice"
    a, b = _half_pairs(oracle, s)
    ambiguous = set()
    if cutoff_full > 0:
        crd = np.asarray(s.crd, np.float64)
        c = [float(v) for v in s.cell]
        r = [float(v) for v in s.rcell]
        d = crd[a] - crd[b]
        sx = np.floor(d[:, 0] * r[0] + d[:, 1] * r[1] + d[:, 2] * r[3] + 0.5)
        sy = np.floor(d[:, 1] * r[2] + d[:, 2] * r[4] + 0.5)
        sz = np.floor(d[:, 2] * r[5] + 0.5)
        d[:, 0] -= sx * c[0] + sy * c[1] + sz * c[3]
        d[:, 1] -= sy * c[2] + sz * c[4]
        d[:, 2] -= sz * c[5]
        d2 = (d * d).sum(1)
        cut2 = cutoff_full * cutoff_full
        # pairs within FP32 rounding of the cutoff may go either way
        amb = np.abs(d2 - cut2) < 1e-5 * cut2
        ambiguous = {(int(i), int(j)) for i, j in zip(a[amb], b[amb])} | {(int(j), int(i)) for i, j in zip(a[amb], b[amb])}
        keep = d2 <= cut2
        a, b = a[keep], b[keep]
    want = _sets(s.n, a, b)
    for i in range(s.n):
        got = set(temp[i, :counts[i]].tolist())
        assert len(got) == counts[i], f"atom {i}: repeated partners"
        diff = {(i, j) for j in got ^ want[i]}
        assert diff <= ambiguous, f"atom {i}: {sorted(diff)[:5]}"


def test_full_list_same_from_one_and_two_sided_tables(torch_cuda):
    """Each atom's upper partners come from its own cluster's table, its lower
    ones through the reverse index of the tables; the full list must come out
    bitwise the same whether the tables are one-sided (a plain build),
    two-sided for the perturbed atoms' clusters (after a soft-core force
    call) or two-sided everywhere (after dH/dlambda), and hold every pair in
    both atoms' lists once."""
    from spgnb import systems as S
    from spgnb.engine import SoftCorePath
    f = S.fep_system(S.water_system(1000, 31.0, 41, n_solute=100, cutoff=8.0, skin=2.0), n_perturbed=24)
    p = SoftCorePath(f, device="cuda:0")
    s = p.system

    def full():
        counts, temp, ovf = p.nl.build_full(s.n, p.crd, s.cell, s.rcell, 0.0, 1200)
        assert int(ovf.item()) == 0
        return counts.cpu().numpy().copy(), temp.cpu().numpy().copy()

    one = full()
    p.force(need_energy=True, need_virial=True)
    part = full()
    p.dhdl(charge_perturbated=True)
    every = full()
    for what, x in (("perturbed atoms' clusters two-sided", part), ("every cluster two-sided", every)):
        assert np.array_equal(one[0], x[0]) and np.array_equal(one[1], x[1]), what
    counts, temp = one
    pairs = {(i, int(j)) for i in range(s.n) for j in temp[i, :counts[i]]}
    assert len(pairs) == int(counts.sum()), "a partner listed twice"
    assert all((j, i) in pairs for (i, j) in pairs), "a pair in one atom's list only"
