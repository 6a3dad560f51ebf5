"""Generate tests/golden/blast384_sharp_reference.json: the reference's own
host integrator (oracle/_ref/libmiso_ref.so, built by `make -C oracle ref`
from the MISO headers) stepped on the magnetised blast of 384^3 cells with
the sharp pressure edge -- the blast configuration as stated, seed 0 --
recording after every step the time step, the FP64 sum and the minimum of
the internal energy over the interior.  The reference reaches non-finite
values at step 22.  One step takes about 4-5 minutes on one host core, so
the whole record about two hours; run it here, where the reference sources
exist:

    python tests/golden/make_blast384_record.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from miso_b200 import problems as P  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

STEPS = 22


def main():
    prob = P.blast(384, seed=0)
    g = prob.grid
    q = np.ascontiguousarray(prob.q.copy())
    ref = Reference()
    rec = []
    for s in range(STEPS):
        dts = ref.run(prob, q, 1, fill_first=(s == 0))
        ei = q[P.EI][g.interior]
        rec.append({"step": s + 1, "dt": float(dts[0]),
                    "sum_ei": float(np.sum(ei, dtype=np.float64)), "min_ei": float(ei.min())})
        print(json.dumps(rec[-1]), flush=True)
    with open(os.path.join(HERE, "blast384_sharp_reference.json"), "w") as f:
        json.dump({"case": "blast(384, seed=0), sharp edge, FP64 reference host integrator",
                   "steps": rec}, f, indent=1)


if __name__ == "__main__":
    main()
