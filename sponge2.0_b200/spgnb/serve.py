"""Serving: MD segments admitted into a ``Pool`` as they arrive.

Continuous batching: requests wait in a FIFO queue until the pool has a free
system id and free ranges for their atoms, cells, clusters, exclusions and
waters (the pool's capacities come from its device-memory budget); admitted
segments run together, every step one launch sequence over all of them, and
a segment leaves the pool when its own step count is reached.  Admission and
retirement happen while a chunk of ``chunk_steps`` steps (one captured
graph) runs: admitted systems' uploads queue behind it and they start with
the next chunk; a segment that reaches its count inside a chunk is frozen on
the device until the chunk ends, so it runs exactly its steps.  A segment's
result is bitwise the one it gets alone.

The loop only needs ``admit`` / ``run`` / ``progress`` / ``evaluate`` /
``energies`` / ``download`` / ``retire`` from the pool, so it runs against a
fake pool on the CPU as well.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Segment:
    request: object            # spgnb.systems.Request: rid, arrival_s, n_atoms, steps, seed
    system: object = None      # made when the segment is first offered to the pool
    pool_id: int = -1
    admitted_s: float = None
    finished_s: float = None
    done_steps: int = 0
    result: dict = field(default=None, repr=False)

    @property
    def latency_s(self):
        return None if self.finished_s is None else self.finished_s - self.request.arrival_s

    @property
    def queueing_s(self):
        return None if self.admitted_s is None else self.admitted_s - self.request.arrival_s


def percentile(values, q):
    return float(np.percentile(np.asarray(values, np.float64), q)) if len(values) else None


class Server:
    """Runs a request stream against a pool.

    make_system(request) -> system; max_resident_atoms (0 = no limit) caps the
    atoms on the device besides the pool's own capacity; lookahead = how many
    queued requests past one that does not fit may be tried (backfill)."""

    def __init__(self, pool, make_system, chunk_steps=10, max_resident_atoms=0, lookahead=16,
                 keep_results=False, clock=time.perf_counter, sleep=time.sleep):
        self.pool = pool
        self.make_system = make_system
        self.chunk_steps = int(chunk_steps)
        self.max_resident_atoms = int(max_resident_atoms)
        self.lookahead = int(lookahead)
        self.keep_results = keep_results
        self.clock = clock
        self.sleep = sleep
        self.queue = []
        self.resident = {}       # pool id -> Segment
        self.finished = []
        self.atom_steps = 0
        self.resident_atoms = 0
        self.max_resident = 0
        self.max_resident_atoms_seen = 0
        self.chunks = 0
        self.rejected = []
        self.prefetch = 4
        self._t = {"make": 0.0, "admit": 0.0, "wait": 0.0, "results": 0.0}

    def _admit(self, now):
        tried = 0
        k = 0
        while k < len(self.queue) and tried <= self.lookahead:
            seg = self.queue[k]
            n = seg.request.n_atoms
            if self.max_resident_atoms and self.resident and self.resident_atoms + n > self.max_resident_atoms:
                tried += 1
                k += 1
                continue
            self._make(seg)
            t = self.clock()
            pid = self.pool.admit(seg.system, seg.request.steps)
            self._t["admit"] += self.clock() - t
            if pid is None:
                if not self.resident:
                    # too large for the empty pool: it can never run
                    self.rejected.append(seg)
                    self.queue.pop(k)
                    continue
                tried += 1
                k += 1
                continue
            seg.pool_id = pid
            seg.admitted_s = now
            seg.done_steps = 0
            self.resident[pid] = seg
            self.resident_atoms += seg.system.n
            self.queue.pop(k)
        self.max_resident = max(self.max_resident, len(self.resident))
        self.max_resident_atoms_seen = max(self.max_resident_atoms_seen, self.resident_atoms)

    def _make(self, seg):
        if seg.system is None:
            t = self.clock()
            seg.system = self.make_system(seg.request)
            self._t["make"] += self.clock() - t

    def host_times(self):
        """Host seconds spent making systems, admitting them (uploads),
        waiting for the device, and reading results."""
        return dict(self._t)

    def _collect(self, now):
        t = self.clock()
        done, left = self.pool.progress()
        self._t["wait"] += self.clock() - t
        finished = []
        for pid, seg in self.resident.items():
            d = int(done[pid])
            self.atom_steps += (d - seg.done_steps) * seg.system.n
            seg.done_steps = d
            if left[pid] == 0:
                finished.append(pid)
        if not finished:
            return
        t = self.clock()
        self.pool.evaluate(finished)
        energies = self.pool.energies()
        for pid in finished:
            seg = self.resident.pop(pid)
            if self.keep_results:
                crd, vel, frc = self.pool.download(pid)
                seg.result = {"crd": crd, "vel": vel, "frc": frc, "energies": energies[pid].copy()}
            self.pool.retire(pid)
            self.resident_atoms -= seg.system.n
            seg.finished_s = now
            seg.system = None if not self.keep_results else seg.system
            self.finished.append(seg)
        self._t["results"] += self.clock() - t

    def run(self, requests, duration_s=None, drain=True):
        """Serves requests (sorted by arrival) until duration_s has passed
        (then stops, unless drain) or everything has finished."""
        pending = sorted(requests, key=lambda r: r.arrival_s)
        nxt = 0
        t0 = self.clock()
        self.t_start = t0
        while True:
            now = self.clock() - t0
            while nxt < len(pending) and pending[nxt].arrival_s <= now:
                self.queue.append(Segment(pending[nxt]))
                nxt += 1
            over = duration_s is not None and now >= duration_s
            if over and not drain:
                break
            admitting = not over or drain
            if not self.resident:
                if admitting:
                    self._admit(now)
                if not self.resident:
                    if self.queue and not over:
                        continue
                    if nxt >= len(pending) or over:
                        break
                    wait = pending[nxt].arrival_s - now
                    if duration_s is not None:
                        wait = min(wait, duration_s - now)
                    if wait > 0:
                        self.sleep(wait)
                    continue
            self.pool.run(self.chunk_steps)
            self.chunks += 1
            # while the chunk runs: admit what fits (its uploads queue behind
            # the chunk; it starts with the next one) and make the systems of
            # the next requests in line
            if admitting:
                now = self.clock() - t0
                while nxt < len(pending) and pending[nxt].arrival_s <= now:
                    self.queue.append(Segment(pending[nxt]))
                    nxt += 1
                self._admit(now)
            for seg in self.queue[:self.prefetch]:
                self._make(seg)
            self._collect(self.clock() - t0)
        self.elapsed_s = self.clock() - t0
        self.unserved = len(self.queue) + (len(pending) - nxt)
        return self.report()

    def report(self):
        lat = [s.latency_s for s in self.finished]
        que = [s.queueing_s for s in self.finished]
        el = getattr(self, "elapsed_s", None) or 1e-30
        return {
            "finished": len(self.finished),
            "rejected": len(self.rejected),
            "resident_at_end": len(self.resident),
            "queued_at_end": len(self.queue),
            "latency_p50_s": percentile(lat, 50),
            "latency_p99_s": percentile(lat, 99),
            "queueing_p50_s": percentile(que, 50),
            "queueing_p99_s": percentile(que, 99),
            "atom_steps": self.atom_steps,
            "atom_steps_per_s": self.atom_steps / el,
            "elapsed_s": el,
            "chunks": self.chunks,
            "max_resident_segments": self.max_resident,
            "max_resident_atoms": self.max_resident_atoms_seen,
        }
