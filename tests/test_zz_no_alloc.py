"""The no-allocation force entry point against the regular one and the oracle.

spgnb_lj_pme_direct_force_noalloc serves callers that cannot allocate device
memory where they need the force (a plugin hook inside the MD step, where
cudaMalloc would synchronise the device; a process with a fixed device-memory
budget).  Called twice in a row through the C ABI, it must reproduce the
forces of spgnb_lj_pme_direct_force_atom_groups on the same reference-layout
list, with and without a water tail left to the solvent module, and the FP64
pair sum of the oracle, within the force tolerance of the parity tests; and
it must refuse what its fixed scratch or its one-rank contract cannot hold.
This file is collected last so a stop-at-first-failure run has already run
every other test.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from conftest import rel_rms  # noqa: E402

pytestmark = pytest.mark.gpu

FORCE_REL_RMS_TOL = 1e-5
SPGNB_E_ARG, SPGNB_E_UNSUPPORTED = 1, 8


def test_noalloc_matches_regular_entry_point_and_oracle(oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spgnb import systems as S
    from spgnb._lib import LTMatrix3, lib
    from spgnb.engine import PlainPath

    s = S.water_system(2600, 44.8, 11, n_solute=400, cutoff=8.0, skin=2.0, name="noalloc")
    p = PlainPath(s, export_atom_groups=True, solvent=False)
    dev = p.crd.device
    n = s.n
    types = torch.from_numpy(np.ascontiguousarray(s.atom_type, np.int32)).to(dev)
    A = torch.from_numpy(np.ascontiguousarray(s.pair_A, np.float32)).to(dev)
    B = torch.from_numpy(np.ascontiguousarray(s.pair_B, np.float32)).to(dev)
    L = lib()
    L.spgnb_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))

    def regular(solvent):
        f = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        p.lj.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(n, n, solvent, 0, p.crd, p.charge, f, s.cell, s.rcell,
                                                             p.nl.d_nl, s.beta, 0, None, 0, None, None)
        torch.cuda.synchronize()
        return f.cpu().numpy()

    def noalloc(out, solvent=0, ghosts=0, n_types=s.n_types, atoms=n):
        return L.spgnb_lj_pme_direct_force_noalloc(atoms, solvent, ghosts, n_types, C.c_void_p(types.data_ptr()),
                                                   C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()),
                                                   C.c_void_p(p.crd.data_ptr()), C.c_void_p(p.charge.data_ptr()),
                                                   C.c_void_p(out.data_ptr()), LTMatrix3.of(s.cell),
                                                   LTMatrix3.of(s.rcell), C.c_void_p(p.nl.d_nl), s.cutoff, s.beta)

    fp64 = oracle.direct_sum(s)["frc"]
    # the water tail (3-site residues at the end) left out, as when the
    # solvent module evaluates it
    tail = 3 * 2600 // 2
    for solvent in (0, tail):
        ref = regular(solvent)
        for _ in range(2):
            f = torch.zeros((n, 3), dtype=torch.float32, device=dev)
            st = noalloc(f, solvent=solvent)
            assert st == 0, L.spgnb_last_error().decode()
            torch.cuda.synchronize()
            got = f.cpu().numpy()
            assert rel_rms(got, ref) <= FORCE_REL_RMS_TOL, (solvent, rel_rms(got, ref))
            if solvent == 0:
                assert rel_rms(got, fp64) <= FORCE_REL_RMS_TOL, rel_rms(got, fp64)
    f = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    # sizes beyond the fixed scratch, and ghost atoms, are refused before any work is queued
    st = noalloc(f, atoms=70000)
    assert st == SPGNB_E_ARG and "at most" in L.spgnb_last_error().decode()
    st = noalloc(f, n_types=65)
    assert st == SPGNB_E_ARG and "at most" in L.spgnb_last_error().decode()
    st = noalloc(f, ghosts=1)
    assert st == SPGNB_E_UNSUPPORTED and "ghost" in L.spgnb_last_error().decode()
    torch.cuda.synchronize()
    assert not f.abs().sum().item()
