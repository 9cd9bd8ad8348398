#!/usr/bin/env python
"""Benchmark of the short-range nonbonded path.

One step is what SPONGE's Main_Calculate_Force runs on this path
(SPONGE/main.cpp:307-397): the caller zeroes the force array, a conditional
neighbour-list update (a full rebuild every 20 steps), and the LJ + PME
direct-space force (LJ_PME_Direct_Force_With_Atom_Energy_And_Virial with
need_atom_energy = need_virial = 0: the step SPONGE runs between energy
outputs).  ``--terms fev`` times the energy step instead (per-atom energy and
virial, the caller also zeroes those arrays, plus the long-range
correction); each line reports the other kind beside the headline, and the
FP64-totals form of the energy step.

Workloads (seeded synthetic coordinates, static between steps; the rebuild
cadence is the reference's refresh_interval):
  mixed96k (default)  30,000 rigid-geometry waters + 6,000 LJ solute atoms of
                      20 types, 99 A box, cutoff 10 A, skin 2 A
  water1m             333,333 waters, 215 A box, cutoff 12 A, skin 2 A
  batched / served    256 independent systems / a Poisson stream of segments

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl spgnb|reference] [--workload W]

Metric: atom-steps/s (whole job, all ranks) and ns/day at dt = 2 fs.  Each
timed step is bracketed by CUDA events on the launching stream, with L2
flushed (a 512 MiB write) between steps outside the events; the job time is
the max over ranks.  N > 1 runs independent replicas, one per GPU
(one-rank-per-system sharding, no collective in the data path).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sponge2.0_b200"))

DT_PS = 0.002
REFRESH_INTERVAL = 20


def _mixed96k():
    from spgnb import systems as S
    return S.mixed_box_96k()


def _water1m():
    from spgnb import systems as S
    return S.water_box_1m()


def _water1m_cpu_sample():
    # the reference's CPU Initial is O(N^2) in the atoms (Total_C6_Get,
    # Lennard_Jones_force.cpp:146-184) and O(G^2) in the cells (the stencil
    # scan, neighbor_list.cpp:5-49): hours at 1M atoms.  Its CPU rate is
    # taken on a box of the same density, cutoff and skin, 36,000 waters.
    from spgnb import systems as S
    n_w = 36000
    return S.water_system(n_w, (n_w / 0.0334) ** (1.0 / 3.0), 3, cutoff=12.0, skin=2.0, name="water-108k")


# plain-path workloads: generator, name, the box the reference's CPU path is
# timed on (None: the workload's own)
PLAIN = {
    "mixed96k": (_mixed96k, "mixed-box-96k: 30000 waters + 6000 LJ solutes (20 types), 99 A cubic, rc 10 A, skin 2 A",
                 None),
    "water1m": (_water1m, "water-box-1m: 333333 waters (999999 atoms), 215 A cubic, rc 12 A, skin 2 A",
                _water1m_cpu_sample),
}


def cpu_sample_box(workload, s):
    """The box the reference's CPU path is timed on, and a note when it is not
    the workload's own."""
    gen = PLAIN[workload][2]
    if gen is None:
        return s, ""
    b = gen()
    return b, f" (a {b.n}-atom box of the same density, cutoff and skin: the reference's CPU set-up is O(N^2))"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["spgnb", "reference"], default="spgnb")
    p.add_argument("--terms", choices=["f", "fev", "totals"], default="f",
                   help="f: force only, the step SPONGE runs between energy outputs (default); fev: force + "
                        "per-atom energy + virial every step (the reference API's energy step); totals: force + "
                        "energy and virial as FP64 totals (the reference arm runs its energy step for it)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU baseline sample")
    p.add_argument("--profile", action="store_true",
                   help="profiling run for ncu: warm-up and --steps steps (inside the NVTX range 'timed'), no L2 "
                        "flush, no e2e, no baseline")
    p.add_argument("--profile-path", choices=["plain", "soft_core", "graph_resident"], default="plain",
                   help="with --profile: plain (the module API, default); soft_core (the same box with a 40-atom "
                        "perturbed ligand); graph_resident (the box as dynamics in captured graphs)")
    p.add_argument("--step-launches", action="store_true",
                   help="with --profile-path graph_resident: launch the kernels step by step instead of replaying "
                        "graphs (a profiler's per-kernel list cannot look inside graphs with conditional nodes)")
    p.add_argument("--workload", choices=["mixed96k", "water1m", "batched", "served"], default="mixed96k",
                   help="mixed96k: the plain path on the 96k box (default); water1m: the plain path on the "
                        "1M-atom water box, rc 12; batched: 256 systems, batched engine against the plain "
                        "per-system path; served: Poisson stream of MD segments into a pool")
    p.add_argument("--no-batched", action="store_true", help="mixed96k: leave out the batched sub-measurement")
    p.add_argument("--systems", type=int, default=256, help="batched: number of systems")
    p.add_argument("--serve-seconds", type=float, default=60.0, help="served: length of the request stream")
    p.add_argument("--rate", type=float, default=40.0, help="served: mean arrivals per second")
    p.add_argument("--max-resident-atoms", type=int, default=2_500_000,
                   help="served: atoms on the device at once (0 = as many as the HBM budget holds)")
    p.add_argument("--hbm-budget-gb", type=float, default=120.0, help="served: device memory of the pool")
    return p.parse_args()


def rank_reduce(maxes, sums, dist, device):
    """Across the ranks: the max of each value of `maxes` (device times) and
    the sum of each of `sums` (work done); as given on one rank (dist None).
    Every rank passes lists of the same lengths, so all take the same
    collectives in the same order."""
    maxes, sums = [float(x) for x in maxes], [float(x) for x in sums]
    if dist is None:
        return maxes, sums
    import torch
    if maxes:
        tm = torch.tensor(maxes, dtype=torch.float64, device=device)
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        maxes = tm.tolist()
    if sums:
        ts = torch.tensor(sums, dtype=torch.float64, device=device)
        dist.all_reduce(ts, op=dist.ReduceOp.SUM)
        sums = ts.tolist()
    return maxes, sums


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def plain_config(args, s, world):
    """The config dict both arms print for a plain-path workload."""
    wl = PLAIN[args.workload][1]
    return {"workload": wl, "atoms_per_gpu": s.n, "terms": args.terms, "refresh_interval": REFRESH_INTERVAL,
            "l2": "flushed between steps (512 MiB write)",
            "parallelism": f"replicas x{world}" if world > 1 else "single system"}


def cpu_reference_rate(system, terms, budget_s, threads=None):
    """The reference's own CPU implementation of the path (oracle/_ref, built
    from its sources) timed on this host, on a bounded sample: one forced
    rebuild, and force steps between rebuilds; atom-steps/s with the rebuild
    amortised over refresh_interval steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ref = O.Reference(gpu=False)
    threads = threads or os.cpu_count() or 1
    ref.set_threads(threads)
    ref.init(system, refresh_interval=REFRESH_INTERVAL)
    ref.nl_update(forced=True)
    fe = terms != "f"
    t_build = ref.time_rebuild(1)
    probe = ref.time_steps(1, first_step=0, need_energy=fe, need_virial=fe)
    steps = max(1, min(REFRESH_INTERVAL - 2, int(max(0.0, budget_s - t_build) / max(probe, 1e-6))))
    t = ref.time_steps(steps, first_step=1, need_energy=fe, need_virial=fe)
    ref.clear()
    per_step = t / steps + t_build / REFRESH_INTERVAL
    return system.n / per_step, threads, steps, t + t_build, per_step


def reference_cuda_times(s, W, K):
    """The reference's own CUDA kernels (oracle/_ref/libspgref_cuda.so, built
    unchanged from its sources for sm_100a) on this GPU: SPONGE's classes
    driven by the harness loop (NEIGHBOR_LIST::Update, then the LJ and solvent
    modules), per step, host clock around K steps after W warm-up steps; the
    same step indices as the other arm, list rebuilt every 20 steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    out = {}
    ref = O.Reference(gpu=True)
    ref.init(s, refresh_interval=REFRESH_INTERVAL, solvent=True)
    ref.nl_update(forced=True)
    for name, ev in (("per_atom_energy_virial", True), ("force_only", False)):
        ref.time_steps(W, first_step=0, need_energy=ev, need_virial=ev)
        t = ref.time_steps(K, first_step=W, need_energy=ev, need_virial=ev)
        out[name] = {"ms_per_step": 1e3 * t / K, "atom_steps_per_s": s.n * K / t}
    ref.clear()
    out["how"] = ("reference CUDA build of NEIGHBOR_LIST + LENNARD_JONES_INFORMATION + SOLVENT_LENNARD_JONES "
                  "(SPONGE/main.cpp:307-397 order), harness loop, host clock, no L2 flush")
    return out


def run_reference_arm(args, world, rank):
    """The reference's CPU implementation of the path on this host's cores, on
    the other arm's workload, step indices, steps and warm-up; rank 0 only.
    Beside it, when a GPU is present, the reference's own CUDA kernels on the
    same workload (reference_cuda)."""
    from spgnb import systems as S
    if rank != 0:
        return
    s = PLAIN[args.workload][0]()
    cs, note = cpu_sample_box(args.workload, s)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ref = O.Reference(gpu=False)
    threads = os.cpu_count() or 1
    ref.set_threads(threads)
    fe = args.terms != "f"
    ref.init(cs, refresh_interval=REFRESH_INTERVAL)
    ref.nl_update(forced=True)
    W, K = args.warmup, args.steps
    if W > 0:
        ref.time_steps(W, first_step=0, need_energy=fe, need_virial=fe)
    t = ref.time_steps(K, first_step=W, need_energy=fe, need_virial=fe)
    ref.clear()
    rate = cs.n * K / t
    rebuilds = sum(1 for k in range(W, W + K) if (k + 1) % REFRESH_INTERVAL == 0)
    line = {"metric": "atom-steps/s", "value": rate, "unit": "atom-steps/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": 1e3 * t / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "ns_per_day": K * 86.4 * DT_PS / t,
            "config": plain_config(args, s, args.gpus),
            "cpu_baseline": {"value": rate, "unit": "atom-steps/s", "cores": threads, "kind": "reference",
                             "sample": f"steps {W}..{W + K - 1} of the box ({rebuilds} rebuilds), after {W} warm-up "
                                       f"steps, {'per-atom energy + virial' if fe else 'forces only'}{note}"},
            "e2e": {"value": rate, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    try:
        import torch
        if torch.cuda.is_available() and os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libspgref_cuda.so")):
            line["reference_cuda"] = reference_cuda_times(s, W, K)
    except Exception as exc:  # reported beside the CPU figure, not required
        line["reference_cuda"] = {"unavailable": str(exc)}
    print(json.dumps(line), flush=True)


def batched_measure(systems_all, K, W, world, rank, local, dist, k_plain=None):
    """Config 3: independent systems (log-uniform 1,500-24,000 atoms, 0-15 %
    solute, rc from {8, 10, 12}, skin 2) stepped by the batched engine
    (leap-frog + SETTLE + per-system list updates + one force launch, graph
    replay), against the plain per-system path: the same kernels for one
    system at a time, launched step by step.  Returns the figures of rank 0's
    line (max time and summed atoms over ranks)."""
    import copy
    import torch
    from spgnb._lib import lib
    from spgnb.batch import Batch
    from spgnb.shard import shard_systems
    mine = [systems_all[k] for k in shard_systems(systems_all, world, rank)]
    L = lib()

    def timed(b, steps, energy_interval=0):
        st = torch.cuda.ExternalStream(b.stream_ptr)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        b.run(steps, energy_interval)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    opts = dict(refresh_interval=REFRESH_INTERVAL, thermostat_tau=0.1, temperature=300.0)
    # the synthetic boxes start strained: relax them with a strongly coupled
    # thermostat first (not timed), then production coupling; lists sized for
    # a 1.6 A prune buffer, the largest the autotuner tries
    B = Batch(mine, **dict(opts, thermostat_tau=0.002, prune_buffer=1.6))
    B.run(200)
    B.check_overflow()
    B.set_thermostat(0.1, 300.0)
    tuned = B.autotune(10)
    tuning = B.tuning()
    B.run(W * tuning["steps_per_graph"])
    B.check_overflow()
    st0 = B.stats()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    if dist is not None:
        dist.barrier()
    launches0 = L.spgnb_launch_count()
    ms = timed(B, K, energy_interval=100)
    launches = L.spgnb_launch_count() - launches0
    clocks = sampler.stop()
    per_step, per_build = B.launch_counts()
    st = B.stats()
    atoms = sum(s.n for s in mine)
    e = B.energies()
    # plain per-system path from the same relaxed states: each system alone,
    # the same kernels launched step by step, a bounded sample of steps
    k_plain = k_plain or max(5, min(20, K // 5))
    plain_ms, plain_as = 0.0, 0
    for k, s in enumerate(mine):
        crd, vel, _ = B.download(k)
        s2 = copy.copy(s)
        s2.crd, s2.vel = crd, vel
        b = Batch([s2], use_graphs=0, **dict(opts, prune_buffer=tuned))
        b.run(W)
        plain_ms += timed(b, k_plain)
        plain_as += s.n * k_plain
        b.close()
    B.close()
    (ms, plain_ms), (atoms_all, plain_as_all) = rank_reduce([ms, plain_ms], [atoms, plain_as], dist, "cuda")
    value = atoms_all * K / (ms * 1e-3)
    plain = plain_as_all / (plain_ms * 1e-3)
    return {"value": value, "ms": ms, "K": K, "W": W, "systems": len(systems_all), "systems_per_gpu": len(mine),
            "atoms_all": int(sum(s.n for s in systems_all)), "atoms_per_gpu": atoms,
            "plain": plain, "k_plain": k_plain, "tuned": tuned, "tuning": tuning,
            "rebuilds": st["rebuilds"] - st0["rebuilds"], "prunings": st["prunings"] - st0["prunings"],
            "overflow": st["overflow"], "energies_finite": bool(np.isfinite(e).all()), "clocks": clocks,
            "launches": int(launches), "build_launches": per_build}


def batched_workload_name(m):
    return (f"batched: {m['systems']} systems, {m['atoms_all']} atoms, log-uniform 1500-24000, rc {{8,10,12}}, "
            "skin 2, leap-frog + SETTLE, 2 fs, Berendsen 300 K (tau 0.1 ps), lists rebuilt every 20 steps")


def run_batched(args, world, rank, local):
    import torch
    from spgnb import systems as S
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    m = batched_measure(S.batch_systems(args.systems), args.steps, max(3, args.warmup), world, rank, local, dist)
    if rank == 0:
        K = m["K"]
        line = {"metric": "atom-steps/s", "value": m["value"], "unit": "atom-steps/s", "n_gpus": world, "steps": K,
                "warmup": m["W"], "ms_per_step": m["ms"] / K, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": batched_workload_name(m), "systems_per_gpu": m["systems_per_gpu"],
                           "atoms_per_gpu": m["atoms_per_gpu"], "energy_interval": 100,
                           "prune_buffer_autotuned": m["tuned"], "autotuned": m["tuning"],
                           "l2": "inputs larger than L2",
                           "parallelism": f"systems sharded over {world} GPUs" if world > 1 else "single GPU"},
                "plain_per_system": {"value": m["plain"], "unit": "atom-steps/s",
                                     "how": f"each system alone from the same relaxed state, kernels launched step "
                                            f"by step, {m['k_plain']} steps each"},
                "batched_over_plain": m["value"] / m["plain"],
                "rebuilds": m["rebuilds"], "prunings": m["prunings"], "overflow": m["overflow"],
                "energies_finite": m["energies_finite"], "clocks": m["clocks"], "gpu_launches": m["launches"],
                "gpu_launches_per_step": m["launches"] / K,
                "build_launches_per_rebuild_step": m["build_launches"],
                "e2e": {"value": m["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                        "note": "state stays resident on the device between steps"}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_served(args, world, rank, local):
    """Config 4: Poisson arrivals (40/s) of MD segments, each a system made as
    in the batched workload with 1,000-50,000 atoms and 500-5,000 steps,
    admitted into a pool under the HBM budget as room frees up (continuous
    batching), state resident on the device.  Ranks serve independent
    streams (no collective in the data path)."""
    import torch
    from spgnb import systems as S
    from spgnb._lib import lib
    from spgnb.batch import Pool, pool_options
    from spgnb.serve import Server
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    L = lib()
    reqs = S.request_stream(duration_s=args.serve_seconds, rate_per_s=args.rate, seed=5 + 1000 * rank)
    warm = S.request_stream(duration_s=1.0, rate_per_s=8.0, seed=99 + rank, steps_min=40, steps_max=60)
    template = S.request_system(reqs[0])
    pool = Pool(template, pool_options(max_systems=1024, hbm_budget_bytes=args.hbm_budget_gb * 1e9),
                steps_per_graph=10, thermostat_tau=0.1, temperature=300.0)
    cap = pool.capacity()
    # warm-up: graph capture and first launches on a few short segments (not timed)
    Server(pool, S.request_system, chunk_steps=10).run([type(r)(r.rid, 0.0, r.n_atoms, r.steps, r.seed)
                                                       for r in warm[:max(3, args.warmup)]])
    torch.cuda.synchronize()
    st = torch.cuda.ExternalStream(pool.stream_ptr)
    sampler = ClockSampler(local)
    sampler.start()
    if dist is not None:
        dist.barrier()
    launches0 = L.spgnb_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    srv = Server(pool, S.request_system, chunk_steps=10, max_resident_atoms=args.max_resident_atoms)
    rep = srv.run(reqs, duration_s=args.serve_seconds, drain=False)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = L.spgnb_launch_count() - launches0
    clocks = sampler.stop()
    pst = pool.stats()
    lat = [x.latency_s for x in srv.finished]
    que = [x.queueing_s for x in srv.finished]
    admitted = [x for x in srv.finished] + list(srv.resident.values())
    h2d = sum(x.request.n_atoms * 40 for x in admitted)   # crd vel (12+12) charge mass type (12) exclusions (~4)
    d2h = sum(x.request.n_atoms * 36 + 72 for x in srv.finished)
    steps_chunks = max(1, srv.chunks * 10)
    from spgnb.shard import gather, merge_served
    mine = {"latencies_s": lat, "queueing_s": que, "finished": rep["finished"], "atom_steps": rep["atom_steps"],
            "elapsed_s": rep["elapsed_s"], "device_ms": ms}
    ranks = gather(mine, dist)
    merged = merge_served(ranks)
    ms = max(r["device_ms"] for r in ranks)
    wall, atom_steps = merged["elapsed_s"], float(merged["atom_steps"])
    if rank == 0:
        value = atom_steps / (ms * 1e-3)
        offered = world * sum(r.n_atoms * r.steps for r in reqs) / args.serve_seconds
        line = {"metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": world,
                "steps": steps_chunks, "warmup": max(3, args.warmup), "ms_per_step": ms / steps_chunks,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": f"served: Poisson {args.rate}/s for {args.serve_seconds:.0f} s, segments of "
                                       "1000-50000 atoms (log-uniform) x 500-5000 steps, systems as in the batched "
                                       "workload, leap-frog + SETTLE, 2 fs, Berendsen 300 K (tau 0.1 ps), "
                                       "skin-triggered lists",
                           "hbm_budget_gb": args.hbm_budget_gb, "pool_atoms": cap["max_atoms"],
                           "pool_device_gb": cap["device_bytes"] / 1e9, "max_resident_atoms": args.max_resident_atoms,
                           "chunk_steps": 10, "l2": "inputs larger than L2",
                           "parallelism": f"independent streams on {world} GPUs" if world > 1 else "single GPU"},
                "served": {"arrivals_per_gpu": len(reqs), "finished": merged["finished"], "rejected": rep["rejected"],
                           "resident_at_end": rep["resident_at_end"], "queued_at_end": rep["queued_at_end"],
                           "latency_p50_s": merged["latency_p50_s"], "latency_p99_s": merged["latency_p99_s"],
                           "queueing_p50_s": merged["queueing_p50_s"], "queueing_p99_s": merged["queueing_p99_s"],
                           "max_resident_segments": rep["max_resident_segments"],
                           "max_resident_atoms": rep["max_resident_atoms"],
                           "offered_atom_steps_per_s": offered, "wall_s": wall,
                           "wall_atom_steps_per_s": atom_steps / wall,
                           "rebuilds": pst["rebuilds"], "prunings": pst["prunings"], "overflow": pst["overflow"],
                           "host_s": srv.host_times()},
                "clocks": clocks, "gpu_launches": int(launches),
                "e2e": {"value": atom_steps / wall, "unit": "atom-steps/s",
                        "h2d_bytes_per_step": h2d / steps_chunks, "d2h_bytes_per_step": d2h / steps_chunks,
                        "note": "host clock over the serving loop: uploads of admitted systems, downloads of results"}}
        print(json.dumps(line), flush=True)
    pool.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.workload == "batched" and args.impl != "reference":
        run_batched(args, world, rank, local)
        return
    if args.workload == "served" and args.impl != "reference":
        run_served(args, world, rank, local)
        return
    if args.impl == "reference":
        # the reference arm is the reference's CPU path: rank 0 alone, no GPU work
        # besides the reference's own CUDA kernels timed beside it
        run_reference_arm(args, world, rank)
        return
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from spgnb._lib import lib
    from spgnb.engine import PlainPath
    import ctypes as C

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    s = PLAIN[args.workload][0]()
    main_box = args.workload == "mixed96k"
    if args.profile and args.profile_path != "plain":
        run_profile_path(args, s, dev)
        return
    L = lib()
    path = PlainPath(s, refresh_interval=REFRESH_INTERVAL, export_atom_groups=False, device=dev)
    stream = torch.cuda.current_stream()

    def step(k, terms):
        # Main_Calculate_Force's part of the path: the caller zeroes the force
        # (and on energy steps the per-atom arrays), then list update and the
        # LJ + PME direct force; an energy step adds per-atom energy and
        # virial and the tail correction.  "totals" is the energy step with
        # the FP64 totals in place of the per-atom arrays.
        fe = terms != "f"
        path.update(k)
        path.force(need_energy=fe, need_virial=fe, per_atom=terms == "fev")
        if terms == "fev":
            path.lj.Long_Range_Correction(1, path.atom_virial, 1, path.atom_energy, s.volume)

    W, K = args.warmup, args.steps
    for k in range(W):
        step(k, args.terms)
    torch.cuda.synchronize()
    if args.profile:
        torch.cuda.nvtx.range_push("timed")
        for k in range(K):
            step(W + k, args.terms)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        if rank == 0:
            print(json.dumps({"profile_run": True, "workload": args.workload, "steps": K, "warmup": W,
                              "atoms": s.n, "terms": args.terms}))
        if dist is not None:
            dist.destroy_process_group()
        return

    # algorithmic work of one pair-kernel launch (convention: 20 FLOP per
    # listed pair, 45 per pair inside rc, +22 with energy and virial)
    listed, inside = C.c_longlong(), C.c_longlong()
    L.spgnb_nl_count_pairs(path.nl.handle, C.c_void_p(path.crd.data_ptr()), _ltm(s.cell), _ltm(s.rcell),
                           s.cutoff, C.byref(listed), C.byref(inside))
    peak = C.c_double()
    L.spgnb_probe_fp32_fma_tflops(5, C.byref(peak))

    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    def timed_steps(terms, first, with_pair_events):
        """K steps, each bracketed by CUDA events on the stream, L2 flushed in
        between (outside the events); the pair kernel's own events too."""
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        for a, b in ev + pev:
            a.record()
            b.record()
        torch.cuda.synchronize()
        launches0 = L.spgnb_launch_count()
        for k in range(K):
            flush.fill_(k & 0xff)
            ev[k][0].record(stream)
            if with_pair_events:
                L.spgnb_debug_set_pair_events(C.c_void_p(pev[k][0].cuda_event), C.c_void_p(pev[k][1].cuda_event))
            step(first + k, terms)
            ev[k][1].record(stream)
        L.spgnb_debug_set_pair_events(None, None)
        torch.cuda.synchronize()
        launches = L.spgnb_launch_count() - launches0
        step_ms = [a.elapsed_time(b) for a, b in ev]
        pair_ms = [a.elapsed_time(b) for a, b in pev] if with_pair_events else []
        return step_ms, pair_ms, launches

    sampler = ClockSampler(local)
    sampler.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, pair_ms, launches = timed_steps(args.terms, W, True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = sum(step_ms)
    # the other step kind over the same step indices (the same rebuilds)
    other = "fev" if args.terms == "f" else "f"
    other_ms, other_pair_ms, _ = timed_steps(other, W, True)
    tot_ms, tot_pair_ms, _ = timed_steps("totals", W, True)

    # end to end through the module API with host buffers: pinned H2D of the
    # coordinates, the step, D2H of the forces and the energy/virial totals
    # (Step_Print's sums), every step
    crd_host = torch.from_numpy(s.crd.copy()).pin_memory()
    frc_host = torch.empty((s.n, 3), dtype=torch.float32).pin_memory()
    fe = args.terms != "f"
    e2e_ms = []
    for k in range(K):
        flush.fill_(k & 0xff)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        path.crd.copy_(crd_host, non_blocking=True)
        step(W + k, args.terms)
        frc_host.copy_(path.frc, non_blocking=True)
        if fe:
            path.lj.totals()
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e_total = sum(e2e_ms)

    extras = {}
    if main_box:
        extras = _main_box_extras(path, s, dev, stream, flush, world, rank, local, dist, args)

    (total_ms, e2e_total), _ = rank_reduce([total_ms, e2e_total], [], dist, dev)

    from spgnb._lib import NLStats
    st = NLStats()
    L.spgnb_nl_get_stats(path.nl.handle, C.byref(st))

    if rank == 0:
        atoms_steps = world * s.n * K
        value = atoms_steps / (total_ms * 1e-3)
        pair_avg_ms = sum(pair_ms) / len(pair_ms)
        flop_per_launch = 20.0 * listed.value + (45.0 + (22.0 if fe else 0.0)) * inside.value
        achieved = flop_per_launch / (pair_avg_ms * 1e-3) / 1e12
        prof = _profile_traffic(args.workload, args.terms)
        line = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "ns_per_day": K * 86.4 * DT_PS / (total_ms * 1e-3),
            "config": plain_config(args, s, world),
            "step": {"f": "list update + LJ/PME direct force (the step SPONGE runs between energy outputs)",
                     "fev": "list update + LJ/PME direct force with per-atom energy and virial + tail correction "
                            "(the reference API's energy step)",
                     "totals": "list update + LJ/PME direct force with FP64 energy and virial totals"}[args.terms],
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                         "frac": achieved / peak.value if peak.value else None,
                         "traffic": prof.get("bytes_per_launch"),
                         "kernel": "k_pair8", "kernel_ms": pair_avg_ms,
                         "flop_per_launch": flop_per_launch, "listed_pairs": listed.value,
                         "pairs_in_cutoff": inside.value,
                         "pruned_list_words": st.pruned_list_words, "prunings": st.prunes, "rebuilds": st.builds,
                         "peak_source": "measured FP32 FFMA throughput on this device (spgnb_probe_fp32_fma_tflops)",
                         "traffic_source": prof.get("source")},
            ("per_atom_energy_virial" if other == "fev" else "force_only"): {
                "ms_per_step": sum(other_ms) / K, "atom_steps_per_s": world * s.n * K / (sum(other_ms) * 1e-3),
                "pair_kernel_ms": sum(other_pair_ms) / K},
            "energy_virial_totals": {
                "ms_per_step": sum(tot_ms) / K, "atom_steps_per_s": world * s.n * K / (sum(tot_ms) * 1e-3),
                "pair_kernel_ms": sum(tot_pair_ms) / K,
                "how": "force + energy and virial reduced to FP64 totals on the device, no per-atom arrays"},
            "list_device_bytes": st.device_bytes,
            "reference_d_temp_bytes": 4 * 1200 * s.n,
            "clocks": clocks,
            "gpu_launches": int(launches),
            "e2e": {"value": world * s.n * K / (e2e_total * 1e-3), "unit": "atom-steps/s",
                    "h2d_bytes_per_step": s.n * 12, "d2h_bytes_per_step": s.n * 12 + (64 if fe else 0)},
        }
        line.update(extras)
        if world == 1 and not args.no_cpu_baseline:
            try:
                cs, note = cpu_sample_box(args.workload, s)
                rate, threads, steps, t, per = cpu_reference_rate(cs, args.terms, args.cpu_seconds)
                line["cpu_baseline"] = {"value": rate, "unit": "atom-steps/s", "cores": threads, "kind": "reference",
                                        "sample": f"one rebuild + {steps} force steps on the host ({t:.1f} s), the "
                                                  f"rebuild amortised over {REFRESH_INTERVAL} steps{note}"}
                rate1, _, steps1, t1, _ = cpu_reference_rate(cs, args.terms, args.cpu_seconds / 2, threads=1)
                line["cpu_baseline"]["single_core"] = {
                    "value": rate1, "cores": 1,
                    "sample": f"one rebuild + {steps1} force steps on one core ({t1:.1f} s)"}
            except Exception as exc:  # the baseline is reported, not required
                line["cpu_baseline"] = {"value": None, "unit": "atom-steps/s", "cores": 0, "kind": "reference",
                                        "sample": f"unavailable: {exc}"}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _main_box_extras(path, s, dev, stream, flush, world, rank, local, dist, args):
    """The 96k box's side measurements: the PME excluded-pair correction
    alone and fused, the full neighbour list, the alchemical path, the box as
    graph-resident dynamics, and the batched workload (config 3, all systems,
    fewer steps)."""
    import torch
    from spgnb import systems as S
    fe = args.terms != "f"
    out = {}
    # the PME excluded-pair correction (PM_force.cpp:918-997), timed on its own
    # (SPONGE runs it in the PME module)
    ex_frc = torch.zeros_like(path.frc)
    ex_ene = torch.zeros_like(path.atom_energy)
    ex_vir = torch.zeros_like(path.atom_virial)

    def excluded():
        path.lj.PME_Excluded_Force_With_Atom_Energy(s.n, path.crd, s.cell, s.rcell, path.charge, s.beta,
                                                    path.excl_start, path.excl_list, path.excl_numbers, ex_frc,
                                                    1, ex_ene, ex_vir)

    def mean_ms(fn, n=20):
        for _ in range(3):
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / n

    out["pme_excluded_correction_ms"] = mean_ms(excluded)
    # the same correction in the force call's finishing pass (spgnb_lj_fuse_pme_excluded)
    force_call = lambda: path.force(need_energy=fe, need_virial=fe, per_atom=True)
    plain_ms = mean_ms(force_call)
    path.lj.Fuse_PME_Excluded(s.n, path.excl_start, path.excl_list, path.excl_numbers, len(s.excl_list))
    fused_ms = mean_ms(force_call)
    path.lj.Fuse_PME_Excluded(s.n, None, None, None, 0)
    out["pme_excluded_fused"] = {"force_call_ms": plain_ms, "force_call_with_correction_ms": fused_ms,
                                 "extra_ms": fused_ms - plain_ms}
    # the full neighbour list for many-body modules (FULL_NEIGHBOR_LIST)
    for _ in range(2):
        path.nl.build_full(s.n, path.crd, s.cell, s.rcell, 0.0, 1200)
    full_out = path.nl._full_out
    out["full_neighbor_list_ms"] = mean_ms(
        lambda: path.nl.build_full(s.n, path.crd, s.cell, s.rcell, 0.0, 1200, out=full_out), 5)
    # the alchemical path on the same box: LJ_SOFT_CORE with a 40-atom perturbed
    # ligand (main.cpp:379-385), per step the list update and the soft-core
    # force; and one dH/dlambda evaluation (it reads back)
    out["soft_core"] = _time_soft_core(s, fe, dev, stream, flush)
    out["graph_resident"] = _time_graph_resident(s)
    if not args.no_batched:
        m = batched_measure(S.batch_systems(args.systems), 100, 3, world, rank, local, dist, k_plain=5)
        out["batched"] = {"workload": batched_workload_name(m), "steps": m["K"], "ms_per_step": m["ms"] / m["K"],
                          "atom_steps_per_s": m["value"], "plain_per_system_atom_steps_per_s": m["plain"],
                          "batched_over_plain": m["value"] / m["plain"],
                          "plain_how": f"each system alone from the same relaxed state, kernels launched step by "
                                       f"step, {m['k_plain']} steps each",
                          "gpu_launches_per_step": m["launches"] / m["K"],
                          "build_launches_per_rebuild_step": m["build_launches"],
                          "prune_buffer_autotuned": m["tuned"],
                          "autotuned": m["tuning"],
                          "rebuilds": m["rebuilds"], "prunings": m["prunings"], "overflow": m["overflow"],
                          "energies_finite": m["energies_finite"], "clocks": m["clocks"]}
    return out


def _time_soft_core(s, fe, dev, stream, flush, steps=50):
    import torch
    from spgnb import systems as S
    from spgnb.engine import SoftCorePath
    f = S.fep_system(s, n_perturbed=40, seed=11, lam=0.6)
    p = SoftCorePath(f, refresh_interval=REFRESH_INTERVAL, device=dev)
    for k in range(5):
        p.step(k, need_energy=fe, need_virial=fe, per_atom=False)
    torch.cuda.synchronize()
    ms = []
    for k in range(steps):
        flush.fill_(k & 0xff)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        p.step(5 + k, need_energy=fe, need_virial=fe, per_atom=False)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    import time
    p.dhdl(charge_perturbated=True)
    t0 = time.perf_counter()
    for _ in range(5):
        p.dhdl(charge_perturbated=True)
    dh_ms = (time.perf_counter() - t0) * 1e3 / 5
    return {"ligand_atoms": int(len(p.lj.perturbed_atoms())), "lambda": f.lam, "steps": steps,
            "ms_per_step": sum(ms) / steps, "atom_steps_per_s": s.n * steps / (sum(ms) * 1e-3),
            "dhdl_ms_host": dh_ms}


def _time_graph_resident(s, steps=400):
    """The same box as dynamics with the whole step on the device: leap-frog +
    SETTLE + the skin/interval list check + list update + force, replayed from
    captured CUDA graphs (the batched engine with one system); energies every
    100 steps.  The box is relaxed first (strongly coupled thermostat, not
    timed) and the prune buffer autotuned as in the batched workload."""
    import torch
    from spgnb.batch import Batch
    b = Batch([s], refresh_interval=REFRESH_INTERVAL, thermostat_tau=0.002, temperature=300.0, prune_buffer=1.6)
    b.run(200)
    b.check_overflow()
    b.set_thermostat(0.1, 300.0)
    tuned = b.autotune(10)
    tuning = b.tuning()
    b.run(3 * tuning["steps_per_graph"])
    st = torch.cuda.ExternalStream(b.stream_ptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    b.run(steps, 100)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    stats = b.stats()
    b.close()
    return {"steps": steps, "ms_per_step": ms / steps, "atom_steps_per_s": s.n * steps / (ms * 1e-3),
            "ns_per_day": steps * 86.4 * DT_PS / (ms * 1e-3), "rebuilds": stats["rebuilds"],
            "prunings": stats["prunings"], "overflow": stats["overflow"], "prune_buffer_autotuned": tuned,
            "autotuned": tuning,
            "how": "leap-frog + SETTLE + list check/update + force in captured CUDA graphs, 2 fs, "
                   "Berendsen 300 K, energies every 100 steps"}


def run_profile_path(args, s, dev):
    """--profile on one of the side paths: set up and warm up as the timed
    measurement does, then --steps steps inside the NVTX range 'timed' (an
    ncu launch list takes --nvtx --nvtx-include timed/)."""
    import torch
    from spgnb import systems as S
    fe = args.terms != "f"
    W, K = args.warmup, args.steps
    if args.profile_path == "soft_core":
        from spgnb.engine import SoftCorePath
        p = SoftCorePath(S.fep_system(s, n_perturbed=40, seed=11, lam=0.6), refresh_interval=REFRESH_INTERVAL,
                         device=dev)
        run = lambda first, n: [p.step(first + k, need_energy=fe, need_virial=fe, per_atom=args.terms == "fev")
                                for k in range(n)]
    elif args.profile_path == "graph_resident":
        from spgnb.batch import Batch
        b = Batch([s], refresh_interval=REFRESH_INTERVAL, thermostat_tau=0.002, temperature=300.0, prune_buffer=1.6)
        b.run(200)
        b.check_overflow()
        b.set_thermostat(0.1, 300.0)
        b.autotune(10)
        if args.step_launches:
            # the same relaxed state and prune buffer, launched step by step
            import copy
            t = b.tuning()
            s2 = copy.copy(s)
            s2.crd, s2.vel, _ = b.download(0)
            b.close()
            b = Batch([s2], refresh_interval=REFRESH_INTERVAL, thermostat_tau=0.1, temperature=300.0,
                      prune_buffer=t["prune_buffer"], use_graphs=0)
        run = lambda first, n: b.run(n, 100)
    run(0, W)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")
    run(W, K)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile_run": True, "path": args.profile_path, "workload": args.workload, "steps": K,
                      "warmup": W, "atoms": s.n, "terms": args.terms}))


def _ltm(m):
    from spgnb._lib import LTMatrix3
    return LTMatrix3.of(m)


def _profile_traffic(workload, terms):
    """DRAM bytes per pair-kernel launch from the committed ncu summary of
    this workload and step kind."""
    p = os.path.join(ROOT, "profiles", f"k_pair8_{workload}_{terms}.json")
    if not os.path.exists(p):
        return {}
    try:
        d = json.load(open(p))
        return {"bytes_per_launch": d.get("dram_bytes_per_launch"), "source": d.get("source")}
    except Exception:
        return {}


if __name__ == "__main__":
    main()
