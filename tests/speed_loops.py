"""The C++ harness loops of tests/test_gpu_speed_vs_reference.py as a script,
for timing one of them alone or under a profiler's launch list:

    python tests/speed_loops.py {shim|ref}_{plain|soft} [steps] [f]

shim = SPONGE's module classes built with the drop-in shim over libspgnb
(oracle/_ref/libspgref_shim.so); ref = built from the reference's sources
(oracle/_ref/libspgref_cuda.so).  The 96,000-atom mixed box, rebuild every 20
steps, energy and virial with per-atom arrays every step (forces only with a
trailing "f"); plain = list update
+ LJ + solvent modules, soft = list update + LJ_SOFT_CORE (40-atom perturbed
ligand) + solvent module.  Prints the wall-clock ms per step of the loop.

    python tests/speed_loops.py graph [steps]

runs the same box as dynamics through the batched engine with one system
(leap-frog + SETTLE + list check/update + force replayed from CUDA graphs,
prune margin autotuned), the timed steps inside the NVTX range "timed"."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "sponge2.0_b200"))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))


def main():
    import oracle as O
    from spgnb import systems as S
    which = sys.argv[1]
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else 30
    if which == "graph":
        graph_loop(steps)
        return
    lib, path = which.split("_")
    ev = not (len(sys.argv) > 3 and sys.argv[3] == "f")
    s = S.mixed_box_96k()
    ref = O.Reference(gpu=lib == "ref", shim=lib == "shim")
    if path == "soft":
        f = S.fep_system(s, n_perturbed=40, seed=11, lam=0.6)
        ref.init(f.system(), refresh_interval=20, solvent=True)
        ref.nl_update(forced=True)
        ref.soft_init(f)
        ref.soft_time_steps(10, need_energy=ev, need_virial=ev)
        t = ref.soft_time_steps(steps, first_step=10, need_energy=ev, need_virial=ev)
    else:
        ref.init(s, refresh_interval=20, solvent=True)
        ref.nl_update(forced=True)
        ref.time_steps(10, need_energy=ev, need_virial=ev)
        t = ref.time_steps(steps, first_step=10, need_energy=ev, need_virial=ev)
    ref.clear()
    print(json.dumps({"loop": which, "steps": steps, "energy_virial": ev, "ms_per_step": t * 1e3 / steps}))


def graph_loop(steps):
    import time
    import torch
    from spgnb import systems as S
    from spgnb.batch import Batch
    s = S.mixed_box_96k()
    b = Batch([s], refresh_interval=20, thermostat_tau=0.002, temperature=300.0, prune_buffer=1.6)
    b.run(200)
    b.check_overflow()
    b.set_thermostat(0.1, 300.0)
    tuned = b.autotune(10)
    b.run(3 * b.options.steps_per_graph)
    torch.cuda.synchronize()
    st0 = b.stats()
    torch.cuda.nvtx.range_push("timed")
    t0 = time.perf_counter()
    b.run(steps, 100)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    torch.cuda.nvtx.range_pop()
    st1 = b.stats()
    b.close()
    print(json.dumps({"loop": "graph", "steps": steps, "ms_per_step": t * 1e3 / steps, "prune_buffer": tuned,
                      "rebuilds": st1["rebuilds"] - st0["rebuilds"], "prunings": st1["prunings"] - st0["prunings"]}))


if __name__ == "__main__":
    main()
