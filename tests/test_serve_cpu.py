"""The serving loop's scheduling on the CPU, against a fake pool: FIFO
admission under the pool's capacity and the resident-atom cap, backfill,
segments leaving at exactly their step counts, latency bookkeeping."""
from types import SimpleNamespace

import numpy as np

from spgnb.serve import Server, percentile


class FakePool:
    """Capacity in system ids and atoms; each run advances every live system
    by up to k steps, then it stops at its count, as the device pool does."""

    def __init__(self, max_systems, max_atoms):
        self.max_systems, self.max_atoms = max_systems, max_atoms
        self.live = {}
        self.log = []

    def admit(self, system, steps):
        used = sum(s.n for s, _, _ in self.live.values())
        if len(self.live) >= self.max_systems or used + system.n > self.max_atoms:
            return None
        pid = min(set(range(self.max_systems)) - set(self.live))
        self.live[pid] = [system, 0, steps]
        self.log.append(("admit", system.name, pid))
        return pid

    def run(self, k):
        for v in self.live.values():
            v[1] = min(v[1] + k, v[2])

    def progress(self):
        d = np.zeros(self.max_systems, np.int32)
        left = np.zeros(self.max_systems, np.int32)
        for pid, (s, done, steps) in self.live.items():
            d[pid], left[pid] = done, steps - done
        return d, left

    def evaluate(self, ids):
        self.log.append(("evaluate", tuple(ids)))

    def energies(self):
        return np.zeros((self.max_systems, 9))

    def download(self, pid):
        n = self.live[pid][0].n
        return np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))

    def retire(self, pid):
        self.log.append(("retire", self.live[pid][0].name, pid))
        del self.live[pid]


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.001
        return self.t

    def sleep(self, dt):
        self.t += dt


def _req(rid, arrival, n, steps):
    return SimpleNamespace(rid=rid, arrival_s=arrival, n_atoms=n, steps=steps, seed=rid)


def _make(r):
    return SimpleNamespace(n=r.n_atoms, name=f"r{r.rid}")


def test_fifo_admission_and_exact_step_counts():
    pool = FakePool(max_systems=2, max_atoms=10_000)
    clock = FakeClock()
    reqs = [_req(0, 0.0, 3000, 25), _req(1, 0.0, 3000, 10), _req(2, 0.0, 3000, 30)]
    srv = Server(pool, _make, chunk_steps=10, clock=clock, sleep=clock.sleep)
    rep = srv.run(reqs)
    assert rep["finished"] == 3 and rep["queued_at_end"] == 0
    # every segment ran exactly its steps
    assert rep["atom_steps"] == sum(r.n_atoms * r.steps for r in reqs)
    admits = [e for e in pool.log if e[0] == "admit"]
    assert [a[1] for a in admits] == ["r0", "r1", "r2"]
    # r2 waited for a free id: it took r1's (the first to finish)
    assert admits[2][2] == admits[1][2]
    assert rep["max_resident_segments"] == 2
    fin = {s.request.rid: s for s in srv.finished}
    assert fin[2].queueing_s > 0 and fin[0].queueing_s < fin[2].queueing_s
    assert all(s.latency_s >= s.queueing_s for s in srv.finished)


def test_backfill_and_resident_atom_cap():
    pool = FakePool(max_systems=8, max_atoms=10_000)
    clock = FakeClock()
    reqs = [_req(0, 0.0, 6000, 20), _req(1, 0.0, 6000, 20), _req(2, 0.0, 2000, 20)]
    srv = Server(pool, _make, chunk_steps=10, clock=clock, sleep=clock.sleep, lookahead=4)
    srv.run(reqs)
    admits = [e[1] for e in pool.log if e[0] == "admit"]
    # r1 does not fit beside r0, r2 does: it goes ahead of r1
    assert admits[:2] == ["r0", "r2"] and admits[2] == "r1"
    pool = FakePool(max_systems=8, max_atoms=100_000)
    srv = Server(pool, _make, chunk_steps=10, clock=clock, sleep=clock.sleep, max_resident_atoms=7000)
    rep = srv.run([_req(k, 0.0, 3000, 20) for k in range(5)])
    assert rep["max_resident_atoms"] <= 7000 and rep["finished"] == 5


def test_too_large_for_the_empty_pool_is_rejected():
    pool = FakePool(max_systems=4, max_atoms=5000)
    clock = FakeClock()
    srv = Server(pool, _make, chunk_steps=10, clock=clock, sleep=clock.sleep)
    rep = srv.run([_req(0, 0.0, 9000, 20), _req(1, 0.0, 1000, 20)])
    assert rep["rejected"] == 1 and rep["finished"] == 1


def test_arrivals_wait_for_their_time_and_duration_stops():
    pool = FakePool(max_systems=4, max_atoms=100_000)
    clock = FakeClock()
    reqs = [_req(0, 0.5, 1000, 10), _req(1, 5.0, 1000, 10)]
    srv = Server(pool, _make, chunk_steps=10, clock=clock, sleep=clock.sleep)
    rep = srv.run(reqs, duration_s=2.0, drain=False)
    assert rep["finished"] == 1
    assert srv.finished[0].admitted_s >= 0.5
    assert srv.unserved == 1


def test_percentile():
    assert percentile([1.0, 2.0, 3.0], 50) == 2.0
    assert percentile([], 50) is None
