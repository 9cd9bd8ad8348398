"""Regenerates the golden fixtures in this directory from the reference's own
CPU build of the path (oracle/_ref/libspgref_cpu.so, ``make -C oracle ref``).

Each fixture stores its inputs and what the reference produced for them:
the half-list neighbour counts per atom plus a SHA-256 of the sorted lists,
forces, LJ / direct-Coulomb energies, the virial sum and the long-range
factor.  The alanine-dipeptide case takes its inputs from the reference's
GROMACS comparison suite (benchmarks/comparison/reference/gromacs/
sponge_inputs/alanine_dipeptide_charmm_tip3p/iter0, cutoff 12 as that
suite's sponge.mdin) and also records that suite's GROMACS lj_sr energy.

Run in the build container (it reads the reference tree):
    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "sponge2.0_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

REF_TREE = "/root/reference"
GMX = os.path.join(REF_TREE, "benchmarks/comparison/reference/gromacs")


def list_digest(counts, lists):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(counts, np.int32).tobytes())
    h.update(np.ascontiguousarray(lists, np.int32).tobytes())
    return h.hexdigest()


def load_native_case(d, prefix="sys_flexible"):
    """Reads the native SPONGE text inputs the comparison suite ships."""
    from spgnb import systems as S

    def tokens(name):
        return open(os.path.join(d, f"{prefix}_{name}.txt")).read().split()

    t = tokens("coordinate")
    n = int(t[0])
    crd = np.array(t[1:1 + 3 * n], np.float32).reshape(n, 3)
    box = [float(v) for v in t[1 + 3 * n:1 + 3 * n + 6]]
    cell, rcell = S.cell_from_box(*box)
    t = tokens("LJ")
    n2, T = int(t[0]), int(t[1])
    assert n2 == n
    P = T * (T + 1) // 2
    A = (np.array(t[2:2 + P], np.float32) * np.float32(12.0)).astype(np.float32)
    B = (np.array(t[2 + P:2 + 2 * P], np.float32) * np.float32(6.0)).astype(np.float32)
    types = np.array(t[2 + 2 * P:2 + 2 * P + n], np.int32)
    t = tokens("charge")
    charge = np.array(t[1:1 + n], np.float32)
    t = tokens("exclude")
    pos = 2
    nums, lst = [], []
    for i in range(n):
        k = int(t[pos])
        nums.append(k)
        lst.extend(int(v) for v in t[pos + 1:pos + 1 + k])
        pos += 1 + k
    nums = np.array(nums, np.int32)
    start = np.zeros(n, np.int32)
    start[1:] = np.cumsum(nums)[:-1]
    t = tokens("mass")
    mass = np.array(t[1:1 + n], np.float32)
    cutoff = 12.0
    return S.System(crd=crd, charge=charge, atom_type=types, pair_A=A, pair_B=B, n_types=T, excl_start=start,
                    excl_numbers=nums, excl_list=np.array(lst, np.int32), mass=mass,
                    res_start=np.zeros(1, np.int32), res_len=np.array([n], np.int32), cell=cell, rcell=rcell,
                    cutoff=cutoff, skin=2.0, beta=S.get_beta(cutoff, 1e-5), name="ala-tip3p-iter0")


def cases():
    from spgnb import systems as S
    out = {
        "water_1944": S.water_system(648, 26.9, 21, cutoff=8.0, skin=2.0, name="water-1944"),
        "water_6480": S.water_box_6480(),
        "mixed_3000": S.water_system(2600, 44.8, 11, n_solute=400, cutoff=8.0, skin=2.0, name="mixed-3000"),
        "triclinic_5500": S.water_system(1800, (38.3, 39.6, 41.5), 12, n_solute=100, cutoff=8.0, skin=2.0,
                                         angles=(75.0, 80.0, 70.0), name="triclinic"),
    }
    out["ala_tip3p"] = load_native_case(os.path.join(GMX, "sponge_inputs/alanine_dipeptide_charmm_tip3p/iter0"))
    return out


def main():
    import oracle as O
    ref = O.Reference(gpu=False)
    meta = {}
    for name, s in cases().items():
        ref.init(s, refresh_interval=0)
        ref.nl_update(forced=True)
        counts, lists, flags = ref.nl_get()
        assert flags.sum() == 0, f"{name}: reference overflow flags {flags}"
        r = ref.force(need_energy=True, need_virial=True)
        arrays = dict(crd=s.crd, charge=s.charge, atom_type=s.atom_type, pair_A=s.pair_A, pair_B=s.pair_B,
                      excl_start=s.excl_start, excl_numbers=s.excl_numbers, excl_list=s.excl_list, mass=s.mass,
                      res_start=s.res_start, res_len=s.res_len, cell=s.cell, rcell=s.rcell,
                      ref_counts=counts, ref_frc=r["frc"], ref_atom_energy=r["atom_energy"],
                      ref_atom_lj=r["atom_lj"], ref_atom_direct=r["atom_direct"],
                      ref_virial_sum=r["atom_virial"].astype(np.float64).sum(0))
        info = {"n": s.n, "n_types": s.n_types, "cutoff": s.cutoff, "skin": s.skin, "beta": s.beta,
                "n_solute": s.n_solute, "pairs": int(counts.sum()), "list_sha256": list_digest(counts, lists),
                "ref_lj_energy": float(r["atom_lj"].astype(np.float64).sum()),
                "ref_direct_energy": float(r["atom_direct"].astype(np.float64).sum()),
                "ref_long_range_factor": ref.long_range_factor()}
        if name == "ala_tip3p":
            rj = json.load(open(os.path.join(GMX, "reference.json")))
            e = [x for x in rj["entries"] if x["case_name"] == "alanine_dipeptide_charmm_tip3p"
                 and x["iteration"] == 0][0]
            info["gromacs_lj_sr"] = float(e["lj_sr"])
            info["gromacs_lj_sr_tolerance"] = 25.0  # comp_alanine_dipeptide.py:111
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        meta[name] = info
        ref.clear()
        print(name, info["pairs"], info["ref_lj_energy"], info["ref_direct_energy"])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
