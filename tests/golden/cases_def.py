"""Definitions of the golden cases (shared by the generator and the tests).

Each case is a seeded input state, a spacing, a time step, a step count and
per-axis periodicity; the expected output comes from the reference library
itself (compiled FP64 from its own sources, one OpenMP thread).
"""
from __future__ import annotations

import numpy as np

from drnum_b200 import cases

ALPHA = cases.RK3_ALPHA


def build(name):
    """Returns dict(U0, h, dt, steps, periodic, active) for a case name."""
    if name == "rough_8":
        U = cases.random_state(8, 8, 8, seed=2, amp=0.05, mach=0.6)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.4), steps=2, periodic=(True, True, True), active=None)
    if name == "ragged_12x10x9":
        U = cases.random_state(12, 10, 9, seed=1, amp=0.01, mach=0.3)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=3, periodic=(True, True, True), active=None)
    if name == "vortex_16":
        U, h, dt = cases.periodic_box(16)
        return dict(U0=U, h=h, dt=dt, steps=5, periodic=(True, True, True), active=None)
    if name == "closed_10x7x12":
        U = cases.random_state(10, 7, 12, seed=3, amp=0.02, mach=0.5)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=3, periodic=(False, True, False), active=None)
    if name == "masked_9":
        U = cases.random_state(9, 9, 9, seed=4, amp=0.02, mach=0.3)
        h = 1.0 / 16
        rng = np.random.default_rng(5)
        act = (rng.random((9, 9, 9)) > 0.15).astype(np.uint8)
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=2, periodic=(True, False, True), active=act)
    if name == "thin_3x5x4":
        U = cases.random_state(3, 5, 4, seed=6, amp=0.02, mach=0.3)
        h = 1.0 / 16
        return dict(U0=U, h=h, dt=cases.cfl_dt(U, h, 0.5), steps=2, periodic=(False, False, False), active=None)
    if name == "cfg1_64_100":
        U, h, dt = cases.periodic_box(64)
        return dict(U0=U, h=h, dt=dt, steps=100, periodic=(True, True, True), active=None)
    raise KeyError(name)


# full-field fixtures (small); the 64^3 x 100 case stores a digest
FULL = ["rough_8", "ragged_12x10x9", "vortex_16", "closed_10x7x12", "masked_9", "thin_3x5x4"]
DIGEST = ["cfg1_64_100"]
