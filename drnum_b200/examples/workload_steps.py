"""Runs RK steps of one of the benchmark workloads (drnum_b200.workloads) in
FP32 bulk with a fixed tile shape and batched schedule, without a CUDA graph:
a small driver for profiling the batched stage kernels one launch at a time.

    python drnum_b200/examples/workload_steps.py NAME [SHAPE WAVES MIN_PLANES SCALE STEPS TABLES]

NAME: jet, sphere or tiled; SHAPE: tile shape of every patch (0: 8x32,
1: 16x16, 2: 16x32); WAVES, MIN_PLANES: DN_OPT_BATCH_WAVES and
DN_OPT_BATCH_MIN_PLANES (WAVES 0: one CTA per work item); SCALE: linear
scale of the workload (1 = full size); STEPS: RK steps (default 4);
TABLES: DN_OPT_DONOR_TABLES (0: interpolation patterns, 1: per-contribution
donor tables)."""
from __future__ import annotations

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))


def main(argv):
    from drnum_b200 import _lib, cases, workloads
    name = argv[0] if argv else "jet"
    shape, waves, min_planes = (int(x) for x in (argv[1:4] + ["2", "2", "8"][len(argv[1:4]):]))
    scale = float(argv[4]) if len(argv) > 4 else 1.0
    steps = int(argv[5]) if len(argv) > 5 else 4
    tables = int(argv[6]) if len(argv) > 6 else 0
    case = workloads.build(name, scale)
    _, objs = workloads.make_grid(case)
    it = workloads.make_iterator(objs, _lib.DN_FP32, 0)
    for q in range(len(objs)):
        it.setTile(q, shape)
    it.setOption(_lib.DN_OPT_BATCH_WAVES, waves)
    it.setOption(_lib.DN_OPT_BATCH_MIN_PLANES, min_planes)
    it.setOption(_lib.DN_OPT_DONOR_TABLES, tables)
    for _ in range(steps):
        it.rkStep(case["dt"], cases.RK3_ALPHA)
    it.sync()
    print(f"{name}: {steps} RK steps, {it.launchCount()} launches")
    it.close()


if __name__ == "__main__":
    main(sys.argv[1:])
