"""Generate the golden fixtures in this directory from the reference's own
host integrator (oracle/_ref/libmiso_ref.so, built by `make -C oracle ref`
from the MISO headers).  Run here, where the reference sources exist:

    python tests/golden/make_golden.py

Each fixture stores, for one seeded case of miso_b200.problems, the time
step of every step and the interior of the 9 fields after the last step.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from miso_b200 import problems as P  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

CASES = {
    "ot24_s12": (lambda: P.orszag_tang(24), 12),
    "bw64x_s30": (lambda: P.brio_wu(64, axis=0, scale=[1.1, 0.9, 1.05, 0.95, 1.2, 0.85]), 30),
    "sod64z_s20": (lambda: P.sod(64, axis=2), 20),
    "turb8_s3": (lambda: P.turbulence(8, seed=3), 3),
    "blast12_s3": (lambda: P.blast(12, seed=2), 3),
}


def main():
    ref = Reference()
    for name, (make, nsteps) in CASES.items():
        prob = make()
        q = prob.q.copy()
        dts = ref.run(prob, q, nsteps)
        inner = q[(slice(None),) + prob.grid.interior]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), dt=dts, interior=inner,
                            nsteps=nsteps)
        print(name, inner.shape, dts[:3])


if __name__ == "__main__":
    main()
