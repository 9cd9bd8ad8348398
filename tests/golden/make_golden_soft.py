"""Regenerates the soft-core golden fixtures (soft_*.npz, soft_core.json) from
the reference's own CPU build of LJ_SOFT_CORE (oracle/_ref/libspgref_cpu.so,
``make -C oracle ref``): LJ_SOFT_CORE::Initial + Get_Local, one
LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial over the
reference's own half list, and Get_Partial_H_Partial_Lambda_With_Columb_Direct
with and without charge perturbation.

Each fixture stores the two-state inputs (types, tables, state charges, the
charge at lambda, soft-core parameters, exclusions, cell) and what the
reference produced: forces, per-atom energies, the virial sum, dH/dlambda and
the long-range factors.

Run in the build container (it needs the reference build):
    python tests/golden/make_golden_soft.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "sponge2.0_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def cases():
    from spgnb import systems as S
    a = S.water_system(900, 31.0, 11, n_solute=120, cutoff=9.0, skin=2.0, name="soft-2820")
    b = S.water_system(1000, (33.0, 34.0, 35.0), 13, n_solute=160, cutoff=8.0, skin=2.0,
                       angles=(88.0, 86.0, 84.0), name="soft-triclinic-3160")
    return {
        "soft_2820": S.fep_system(a, n_perturbed=24, seed=7, lam=0.5),
        "soft_triclinic_3160": S.fep_system(b, n_perturbed=30, seed=9, lam=0.3, alpha=0.7, p=2.0, sigma=2.5,
                                            sigma_min=1.5),
    }


def main():
    import oracle as O
    ref = O.Reference(gpu=False)
    meta = {}
    for name, f in cases().items():
        s = f.system()
        ref.init(s, refresh_interval=0)
        ref.nl_update(forced=True)
        counts, lists, flags = ref.nl_get()
        assert flags.sum() == 0, f"{name}: reference overflow flags {flags}"
        ref.soft_init(f)
        r = ref.soft_force(need_energy=True, need_virial=True)
        dh_lj_q, dh_c = ref.soft_dhdl(charge_perturbated=True)
        dh_lj, _ = ref.soft_dhdl(charge_perturbated=False)
        lr, lr_ti = ref.soft_long_range()
        arrays = dict(crd=s.crd, charge=s.charge, charge_a=f.charge_a, charge_b=f.charge_b, type_a=f.type_a,
                      type_b=f.type_b, AA=f.AA, AB=f.AB, BA=f.BA, BB=f.BB, params=f.params(),
                      excl_start=s.excl_start, excl_numbers=s.excl_numbers, excl_list=s.excl_list, mass=s.mass,
                      res_start=s.res_start, res_len=s.res_len, cell=s.cell, rcell=s.rcell, changed=f.changed,
                      ref_counts=counts, ref_frc=r["frc"], ref_atom_energy=r["atom_energy"],
                      ref_atom_lj=r["atom_lj"], ref_atom_direct=r["atom_direct"],
                      ref_virial_sum=r["atom_virial"].astype(np.float64).sum(0))
        info = {"n": s.n, "n_types_a": f.n_types_a, "n_types_b": f.n_types_b, "cutoff": s.cutoff, "skin": s.skin,
                "beta": s.beta, "n_solute": s.n_solute, "pairs": int(counts.sum()),
                "ref_lj_energy": float(r["atom_lj"].astype(np.float64).sum()),
                "ref_direct_energy": float(r["atom_direct"].astype(np.float64).sum()),
                "ref_dhdl_lj": dh_lj, "ref_dhdl_lj_charge_run": dh_lj_q, "ref_dhdl_direct": dh_c,
                "ref_long_range_factor": lr, "ref_long_range_factor_ti": lr_ti}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        meta[name] = info
        ref.clear()
        print(name, info["pairs"], info["ref_lj_energy"], info["ref_direct_energy"], dh_lj, dh_c)
    with open(os.path.join(HERE, "soft_core.json"), "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
