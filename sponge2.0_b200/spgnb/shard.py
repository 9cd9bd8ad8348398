"""Multi-GPU plumbing of the batched and served workloads.

Independent systems need no collective per step: each rank runs its own
systems (batched) or its own request stream (served), and the host merges
the per-rank figures once at the end.  torch.distributed carries only that
merge (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations


def pair_work(system):
    """Estimated pair work of a system: atoms x cutoff^3 (density is the same
    for every system of these workloads)."""
    return system.n * system.cutoff ** 3


def shard_systems(systems, world, rank):
    """Greedy bin packing of independent systems over ranks by estimated
    pair work, largest first; rank r takes bin r (indices, ascending)."""
    order = sorted(range(len(systems)), key=lambda k: (-pair_work(systems[k]), k))
    loads = [0.0] * world
    bins = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (loads[q], q))
        bins[r].append(k)
        loads[r] += pair_work(systems[k])
    return sorted(bins[rank])


def merge_served(reports):
    """One served report from the ranks' reports: segment latencies pooled
    for the percentiles, work summed, the job time the slowest rank's."""
    import numpy as np
    lat = [x for r in reports for x in r["latencies_s"]]
    que = [x for r in reports for x in r["queueing_s"]]
    pct = (lambda v, q: float(np.percentile(v, q)) if v else None)
    return {
        "finished": sum(r["finished"] for r in reports),
        "atom_steps": sum(r["atom_steps"] for r in reports),
        "elapsed_s": max(r["elapsed_s"] for r in reports),
        "latency_p50_s": pct(lat, 50), "latency_p99_s": pct(lat, 99),
        "queueing_p50_s": pct(que, 50), "queueing_p99_s": pct(que, 99),
    }


def gather(obj, dist=None):
    """All ranks' objects on every rank (a list in rank order); the object
    alone without a process group."""
    if dist is None or not dist.is_initialized():
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
