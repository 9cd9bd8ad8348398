"""The no-allocation force entry point against the regular one.

spgnb_lj_pme_direct_force_noalloc serves callers that cannot allocate device
memory where they need the force (a plugin hook inside the MD step, where
cudaMalloc would synchronise the device; a process with a fixed device-memory
budget).  Called twice in a row through the C ABI, it must reproduce the
forces of spgnb_lj_pme_direct_force_atom_groups on the same reference-layout
list within the force tolerance of the parity tests.  This file is collected
last so a stop-at-first-failure run has already run every other test.
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


def test_noalloc_matches_regular_entry_point_twice():
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
    # regular entry point over the exported reference-layout list
    f_ref = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    p.lj.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(n, n, 0, 0, p.crd, p.charge, f_ref, s.cell, s.rcell,
                                                         p.nl.d_nl, s.beta, 0, None, 0, None, None)
    types = torch.from_numpy(np.ascontiguousarray(s.atom_type, np.int32)).to(dev)
    A = torch.from_numpy(np.ascontiguousarray(s.pair_A, np.float32)).to(dev)
    B = torch.from_numpy(np.ascontiguousarray(s.pair_B, np.float32)).to(dev)
    L = lib()
    L.spgnb_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))
    outs = []
    for _ in range(2):
        f = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        st = L.spgnb_lj_pme_direct_force_noalloc(n, 0, s.n_types, C.c_void_p(types.data_ptr()),
                                                 C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()),
                                                 C.c_void_p(p.crd.data_ptr()), C.c_void_p(p.charge.data_ptr()),
                                                 C.c_void_p(f.data_ptr()), LTMatrix3.of(s.cell),
                                                 LTMatrix3.of(s.rcell), C.c_void_p(p.nl.d_nl), s.cutoff, s.beta)
        assert st == 0, L.spgnb_last_error().decode()
        torch.cuda.synchronize()
        outs.append(f.cpu().numpy())
    ref = f_ref.cpu().numpy()
    for f in outs:
        assert rel_rms(f, ref) <= FORCE_REL_RMS_TOL
    # a size beyond the fixed scratch is refused before any work is queued
    st = L.spgnb_lj_pme_direct_force_noalloc(70000, 0, s.n_types, C.c_void_p(types.data_ptr()),
                                             C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()),
                                             C.c_void_p(p.crd.data_ptr()), C.c_void_p(p.charge.data_ptr()),
                                             C.c_void_p(f_ref.data_ptr()), LTMatrix3.of(s.cell),
                                             LTMatrix3.of(s.rcell), C.c_void_p(p.nl.d_nl), s.cutoff, s.beta)
    assert st == 1 and "at most" in L.spgnb_last_error().decode()
