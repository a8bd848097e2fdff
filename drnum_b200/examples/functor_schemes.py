"""Runs the periodic vortex box through the generic flux-functor stage with
DrNUM's other Euler fluxes (VanLeer, Roe) and through the specialised AUSM+
kernel, FP64 on one GPU, and prints each one's throughput.

    python -m drnum_b200.examples.functor_schemes [n] [steps]
"""
import sys
import time

from drnum_b200 import _lib, cases
from drnum_b200.api import AusmPlus, B200CartesianIterator, CartesianPatch, Roe, VanLeer


def main(n=128, steps=5):
    U0, h, dt = cases.periodic_box(n)
    for name, op in [("AUSM+ (specialised kernel)", AusmPlus()), ("AUSM+ (functor stage)", AusmPlus(functor=True)),
                     ("VanLeer (functor stage)", VanLeer()), ("Roe (functor stage)", Roe())]:
        p = CartesianPatch(n, n, n, spacing=(h, h, h), periodic=(True, True, True))
        p.setField(0, U0)
        it = B200CartesianIterator(op, 0, _lib.DN_FP64)
        it.addPatch(p)
        it.updateDevice(fields=(0,))
        for _ in range(2):
            it.rkStep(dt, cases.RK3_ALPHA)
        it.sync()
        t = time.perf_counter()
        for _ in range(steps):
            it.rkStep(dt, cases.RK3_ALPHA)
        it.sync()
        s = (time.perf_counter() - t) / steps
        print(f"{name:28s} {n}^3: {s * 1e3:8.2f} ms per step, {n ** 3 * 3 / s / 1e6:7.0f} Mcell-updates/s per stage")
        it.close()


if __name__ == "__main__":
    main(*(int(a) for a in sys.argv[1:3]))
