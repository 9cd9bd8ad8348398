"""spgnb: B200 short-range nonbonded engine for SPONGE (host-side interface).

The package directory ``sponge2.0_b200`` holds the CUDA sources (``csrc/``),
the built ``libspgnb.so`` and this Python mirror of the reference's module
interface.  Import with ``sponge2.0_b200`` on ``sys.path``.
"""
from . import systems  # noqa: F401
from ._lib import SpgnbError, lib, version  # noqa: F401
