"""Pool of systems on the GPU (continuous batching): systems admitted and
retired while others run give bitwise the results they get alone; the pool
refuses what does not fit and takes it once room frees up."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(k, seed):
    from spgnb import systems as S
    return S.batch_systems(k, seed=seed, n_min=1500, n_max=4000)


def _alone(system, steps, **kw):
    from spgnb.batch import Batch
    b = Batch([system], **kw)
    b.run(steps)
    b.evaluate([0])
    crd, vel, frc = b.download(0)
    e = b.energies()[0].copy()
    b.close()
    return crd, vel, frc, e


def _assert_same(got, ref, what):
    for x, y, name in zip(got, ref, ("crd", "vel", "frc", "energies")):
        assert np.array_equal(x, y), f"{what}: {name} differs alone vs in the pool"


@pytest.mark.parametrize("tau", [0.0, 0.05])
def test_pool_same_alone_and_in_the_mix(torch_cuda, tau):
    """Systems join and leave a running pool; each ends bitwise where it ends
    alone (with the per-system thermostat on too: its sums are fixed point)."""
    from spgnb.batch import Pool, pool_options
    systems = _systems(4, seed=21)
    steps = [60, 40, 30, 20]
    pool = Pool(systems[0], pool_options(max_systems=8, max_atoms=40000), thermostat_tau=tau)
    ids = {0: pool.admit(systems[0], steps[0]), 1: pool.admit(systems[1], steps[1])}
    pool.run(20)
    ids[2] = pool.admit(systems[2], steps[2])       # joins two running systems
    pool.run(20)
    done, left = pool.progress()
    assert left[ids[1]] == 0 and done[ids[1]] == 40 and done[ids[0]] == 40 and done[ids[2]] == 20
    results = {}
    pool.evaluate([ids[1]])
    results[1] = (*pool.download(ids[1]), pool.energies()[ids[1]].copy())
    pool.retire(ids[1])                              # leaves while the others run
    ids[3] = pool.admit(systems[3], steps[3])       # takes the freed room
    pool.run(20)
    done, left = pool.progress()
    for k in (0, 2, 3):
        assert left[ids[k]] == 0 and done[ids[k]] == steps[k], (k, done[ids[k]], left[ids[k]])
    pool.evaluate([ids[0], ids[2], ids[3]])
    e = pool.energies()
    for k in (0, 2, 3):
        results[k] = (*pool.download(ids[k]), e[ids[k]].copy())
    assert pool.stats()["overflow"] == 0
    pool.close()
    for k in range(4):
        _assert_same(results[k], _alone(systems[k], steps[k], thermostat_tau=tau), f"system {k}")


def test_pool_refuses_then_admits(torch_cuda):
    from spgnb.batch import Pool, pool_options
    systems = _systems(3, seed=22)
    pool = Pool(systems[0], pool_options(max_systems=2, max_atoms=16384))
    a = pool.admit(systems[0], 10)
    b = pool.admit(systems[1], 10)
    assert a is not None and b is not None
    assert pool.admit(systems[2], 10) is None        # no free system id
    pool.run(10)
    _, left = pool.progress()
    assert left[a] == 0 and left[b] == 0
    pool.retire(a)
    c = pool.admit(systems[2], 10)
    assert c == a                                    # the lowest free id
    pool.run(10)
    d, left = pool.progress()
    assert d[c] == 10 and left[c] == 0
    cap = pool.capacity()
    assert cap["free_atoms"] == cap["max_atoms"] - systems[1].n - systems[2].n
    pool.close()


def test_pool_budget_sizes_the_pool(torch_cuda):
    from spgnb.batch import Pool, pool_options
    systems = _systems(1, seed=23)
    budget = 1.5e9
    pool = Pool(systems[0], pool_options(max_systems=64, hbm_budget_bytes=budget))
    cap = pool.capacity()
    assert 0 < cap["device_bytes"] <= budget
    assert cap["max_atoms"] >= 50000
    pool.close()


def test_server_results_same_alone(torch_cuda):
    from spgnb import systems as S
    from spgnb.batch import Pool, pool_options
    from spgnb.serve import Server
    reqs = S.request_stream(duration_s=5.0, rate_per_s=6.0, seed=31, n_min=1500, n_max=5000,
                            steps_min=20, steps_max=60)[:5]
    reqs = [S.Request(r.rid, 0.0, r.n_atoms, r.steps, r.seed) for r in reqs]
    systems = {r.rid: S.request_system(r) for r in reqs}
    template = systems[reqs[0].rid]
    # two at a time: the later requests wait and join while others run
    pool = Pool(template, pool_options(max_systems=2, max_atoms=32768))
    srv = Server(pool, lambda r: systems[r.rid], chunk_steps=10, keep_results=True)
    rep = srv.run(reqs)
    assert rep["finished"] == len(reqs) and rep["rejected"] == 0
    assert rep["atom_steps"] == sum(systems[r.rid].n * r.steps for r in reqs)
    pool.close()
    for seg in srv.finished:
        r = seg.request
        got = (seg.result["crd"], seg.result["vel"], seg.result["frc"], seg.result["energies"])
        _assert_same(got, _alone(systems[r.rid], r.steps), f"request {r.rid}")
