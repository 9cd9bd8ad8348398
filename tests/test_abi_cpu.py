"""CPU checks of the C ABI: the library loads without a GPU, exports every
symbol include/spgnb.h declares, and its host-only entry points behave."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "spgnb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(spgnb_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from spgnb import _lib
    lib = _lib.lib()
    declared = _declared_functions()
    assert len(declared) >= 20
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    assert sorted(_lib.EXPORTED) == declared


def test_version_and_status_strings():
    from spgnb import _lib
    assert "sm_100a" in _lib.version()
    assert _lib.lib().spgnb_status_string(4).decode() == "buffer overflow"


@pytest.mark.parametrize("rc,expected", [(8.0, 0.348639), (10.0, 0.275106), (12.0, 0.226635)])
def test_get_beta_matches_reference_values(rc, expected, oracle):
    """Get_Beta (PM_force.cpp:244-272) at tolerance 1e-5."""
    from spgnb import _lib
    b = _lib.lib().spgnb_get_beta(rc, 1e-5)
    assert abs(b - expected) < 2e-6
    assert b == oracle.beta(rc, 1e-5)


def test_errors_are_reported_not_fatal():
    from spgnb import _lib
    L = _lib.lib()
    h = C.c_void_p()
    cell = _lib.LTMatrix3.of([10, 0, 10, 0, 0, 10])
    st = L.spgnb_nl_create(100, 10.0, 2.0, cell, cell, None, C.byref(h))
    assert st == 1  # the box is too small for the grid: SPGNB_E_ARG
    assert "too small" in L.spgnb_last_error().decode()
    st = L.spgnb_lj_create(0, 1, None, None, None, 10.0, C.byref(h))
    assert st == 1


def test_default_options_match_reference_keys():
    from spgnb import _lib
    o = _lib.NLOptions()
    _lib.lib().spgnb_nl_default_options(C.byref(o))
    assert o.max_neighbor_numbers == 1200
    assert o.max_atom_in_grid_numbers == 150
    assert o.refresh_interval == 0
    assert abs(o.skin_permit - 0.5) < 1e-7
    assert o.check_overflow_interval == 150
    assert o.throw_error_when_overflow == 0


def test_generator_shapes():
    from spgnb import systems as S
    s = S.water_box_6480()
    assert s.n == 6480 and s.n_waters == 2160
    assert np.isclose(s.charge.sum(), 0, atol=1e-3)
    assert s.excl_numbers.sum() == 3 * 2160
    assert abs(s.beta - 0.275106) < 2e-6
