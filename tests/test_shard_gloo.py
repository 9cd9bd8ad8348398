"""Multi-rank plumbing of the batched and served workloads on two gloo ranks
(CPU): the system shards partition the batch with balanced pair work, the
served figures merge across ranks, and the benchmark's own cross-rank
reduction (slowest rank's time, summed work) runs over the real 256-system
batch."""
import json
import os
import socket
import subprocess
import sys
import textwrap

from conftest import ROOT

CHILD = textwrap.dedent("""
    import json, os, sys
    from types import SimpleNamespace
    sys.path.insert(0, os.path.join(os.environ["SPGNB_ROOT"], "sponge2.0_b200"))
    import datetime
    import numpy as np
    import torch.distributed as dist
    from spgnb.shard import gather, merge_served, pair_work, shard_systems
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rank, world = dist.get_rank(), dist.get_world_size()
    rng = np.random.default_rng(4)
    systems = [SimpleNamespace(n=int(np.exp(rng.uniform(np.log(1500), np.log(24000)))),
                               cutoff=float(rng.choice([8.0, 10.0, 12.0]))) for _ in range(256)]
    mine = shard_systems(systems, world, rank)
    load = sum(pair_work(systems[k]) for k in mine)
    rep = {"latencies_s": [1.0 + rank, 2.0 + rank], "queueing_s": [0.5], "finished": 2,
           "atom_steps": 1000 * (rank + 1), "elapsed_s": 10.0 + rank}
    shards = gather({"mine": mine, "load": load}, dist)
    merged = merge_served(gather(rep, dist))
    if rank == 0:
        with open(os.environ["SPGNB_OUT"], "w") as f:
            json.dump({"shards": shards, "merged": merged}, f)
    dist.barrier()
    dist.destroy_process_group()
""")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_and_merge(tmp_path):
    out = tmp_path / "out.json"
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                   SPGNB_ROOT=ROOT, SPGNB_OUT=str(out), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env))
    codes = [p.wait(timeout=120) for p in procs]
    assert codes == [0, 0]
    d = json.loads(out.read_text())
    a, b = d["shards"][0]["mine"], d["shards"][1]["mine"]
    assert sorted(a + b) == list(range(256)) and not set(a) & set(b)
    la, lb = d["shards"][0]["load"], d["shards"][1]["load"]
    assert abs(la - lb) / max(la, lb) < 0.01
    m = d["merged"]
    assert m["finished"] == 4 and m["atom_steps"] == 3000 and m["elapsed_s"] == 11.0
    assert m["latency_p50_s"] == 2.0 and m["latency_p99_s"] > 2.9  # pooled [1, 2, 2, 3]


CHILD_BATCH = textwrap.dedent("""
    import json, os, sys
    root = os.environ["SPGNB_ROOT"]
    sys.path.insert(0, os.path.join(root, "sponge2.0_b200"))
    sys.path.insert(0, root)
    import datetime
    import torch.distributed as dist
    import bench
    from spgnb import systems as S
    from spgnb.shard import gather, pair_work, shard_systems
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rank, world = dist.get_rank(), dist.get_world_size()
    systems = S.batch_systems(256)
    mine = shard_systems(systems, world, rank)
    atoms = sum(systems[k].n for k in mine)
    # stand-in device times of this rank's timed region and plain sample
    ms, plain_ms = 100.0 + 7.0 * rank, 50.0 - rank
    (ms_all, plain_all), (atoms_all, plain_as) = bench.rank_reduce([ms, plain_ms], [atoms, 3 * atoms], dist, "cpu")
    (only_max,), none = bench.rank_reduce([ms], [], dist, "cpu")
    info = gather({"mine": mine, "atoms": atoms, "load": sum(pair_work(systems[k]) for k in mine),
                   "ms_all": ms_all, "plain_all": plain_all, "atoms_all": atoms_all, "plain_as": plain_as,
                   "only_max": only_max, "none": none}, dist)
    if rank == 0:
        with open(os.environ["SPGNB_OUT"], "w") as f:
            json.dump({"ranks": info, "total_atoms": sum(s.n for s in systems)}, f)
    dist.barrier()
    dist.destroy_process_group()
""")


def test_two_gloo_ranks_batch_shards_and_timing_reduction(tmp_path):
    """The 256-system batch of the batched workload split over two ranks by
    the bench's own sharding, and its cross-rank reduction: the timed region
    is the slowest rank's, the work the sum over ranks, identical on every
    rank."""
    out = tmp_path / "out.json"
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                   SPGNB_ROOT=ROOT, SPGNB_OUT=str(out), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD_BATCH], env=env))
    codes = [p.wait(timeout=180) for p in procs]
    assert codes == [0, 0]
    d = json.loads(out.read_text())
    r0, r1 = d["ranks"]
    assert sorted(r0["mine"] + r1["mine"]) == list(range(256)) and not set(r0["mine"]) & set(r1["mine"])
    assert r0["atoms"] + r1["atoms"] == d["total_atoms"]
    assert abs(r0["load"] - r1["load"]) / max(r0["load"], r1["load"]) < 0.01
    for r in (r0, r1):
        assert r["ms_all"] == 107.0 and r["plain_all"] == 50.0 and r["only_max"] == 107.0
        assert r["atoms_all"] == d["total_atoms"] and r["plain_as"] == 3 * d["total_atoms"]
        assert r["none"] == []
