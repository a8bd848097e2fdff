"""drnum_b200 — B200 (sm_100a) implementation of DrNUM's per-patch explicit
finite-volume step (AUSM+ / Upwind2-van Albada / low-storage RK) behind a C
ABI (include/drnum_b200.h) and a host mirror of the reference's
patch/iterator/Runge-Kutta API (drnum_b200.api).
"""
from . import _lib  # noqa: F401

__all__ = ["_lib"]
