"""The C++ harness loops of tests/test_gpu_speed_vs_reference.py as a script,
for timing one of them alone or under a profiler's launch list:

    python tests/speed_loops.py {shim|ref}_{plain|soft} [steps]

shim = SPONGE's module classes built with the drop-in shim over libspgnb
(oracle/_ref/libspgref_shim.so); ref = built from the reference's sources
(oracle/_ref/libspgref_cuda.so).  The 96,000-atom mixed box, rebuild every 20
steps, energy and virial with per-atom arrays every step; plain = list update
+ LJ + solvent modules, soft = list update + LJ_SOFT_CORE (40-atom perturbed
ligand) + solvent module.  Prints the wall-clock ms per step of the loop."""
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
    lib, path = which.split("_")
    s = S.mixed_box_96k()
    ref = O.Reference(gpu=lib == "ref", shim=lib == "shim")
    if path == "soft":
        f = S.fep_system(s, n_perturbed=40, seed=11, lam=0.6)
        ref.init(f.system(), refresh_interval=20, solvent=True)
        ref.nl_update(forced=True)
        ref.soft_init(f)
        ref.soft_time_steps(10, need_energy=True, need_virial=True)
        t = ref.soft_time_steps(steps, first_step=10, need_energy=True, need_virial=True)
    else:
        ref.init(s, refresh_interval=20, solvent=True)
        ref.nl_update(forced=True)
        ref.time_steps(10, need_energy=True, need_virial=True)
        t = ref.time_steps(steps, first_step=10, need_energy=True, need_virial=True)
    ref.clear()
    print(json.dumps({"loop": which, "steps": steps, "ms_per_step": t * 1e3 / steps}))


if __name__ == "__main__":
    main()
