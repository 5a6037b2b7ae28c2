"""B200 (sm_100a) implementation of Sofia's nonbonded hot path.

The compute runs in ``libsofia_nb.so`` (hand-written CUDA behind the C ABI of
``include/sofia_nb.h``); this package only binds it and mirrors the
reference's subroutine interface.
"""
from ._lib import SofiaError, lib  # noqa: F401
