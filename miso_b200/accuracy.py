"""Accuracy of the FP32 split-precision form against the FP64 form.

    python -m miso_b200.accuracy --problem turbulence --n 256 --steps 1000 --every 250

Both forms start from the same initial state and advance with the same time
steps: each step the FP64 form's CFL step (the reference's own cfl ->
update(dt) sequence, mhd_model_base.hpp:57-62) is handed to both, so the
difference measures the split form's arithmetic alone.  Every `--every`
steps the two states are compared over the interior -- relative L1 and
relative L-infinity of rho, of the gas pressure p = (gamma-1) rho ei and of
the magnetic field (all three components) -- and the drift of the FP64
monitors (total mass, momentum, energy) from their initial values is
reported for each form.  One JSON line per checkpoint.
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

from . import problems as P
from .integrator import Integrator

PROBLEMS = {
    "turbulence": lambda n, seed, smooth=0.0: P.turbulence(n, seed=seed),
    "blast": lambda n, seed, smooth=0.0: P.blast(n, seed=seed, smooth=smooth),
    "orszag_tang": lambda n, seed, smooth=0.0: P.orszag_tang(n),
    "brio_wu": lambda n, seed, smooth=0.0: P.brio_wu(n),
}


def _errors(a: np.ndarray, b: np.ndarray, gm: float) -> dict:
    """a: split state, b: FP64 state, both (9, ...) interior arrays."""
    def rel(x, y):
        d = np.abs(x - y)
        s = float(np.sum(np.abs(y)))
        m = float(np.max(np.abs(y)))
        return (float(np.sum(d)) / s if s else 0.0), (float(np.max(d)) / m if m else 0.0)

    pa = (gm - 1.0) * a[P.RO] * a[P.EI]
    pb = (gm - 1.0) * b[P.RO] * b[P.EI]
    out = {}
    for name, (x, y) in {"rho": (a[P.RO], b[P.RO]), "p": (pa, pb),
                         "B": (a[P.BX:P.BZ + 1], b[P.BX:P.BZ + 1])}.items():
        l1, linf = rel(x, y)
        out[f"l1_{name}"] = l1
        out[f"linf_{name}"] = linf
    return out


def _drift(m: dict, m0: dict) -> dict:
    scale = abs(m0["mass"]) or 1.0
    return {"mass": (m["mass"] - m0["mass"]) / scale,
            "mom": max(abs(m[k] - m0[k]) for k in ("mom_x", "mom_y", "mom_z")) / scale,
            "energy": (m["energy"] - m0["energy"]) / (abs(m0["energy"]) or 1.0)}


def compare(prob, steps: int, every: int, emit=print) -> dict:
    """Run `prob` in both forms for `steps` steps with the FP64 form's time
    steps; returns the last checkpoint's record."""
    gm = prob.config["eos"]["gm"]
    forms = {}
    for prec in ("fp64", "fp32_split"):
        integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision=prec)
        integ.upload(prob.q)
        integ.apply_boundary_condition()
        forms[prec] = integ
    m0 = {k: v.monitors() for k, v in forms.items()}
    inner = (slice(None),) + prob.grid.interior
    rec = {}
    t = 0.0
    from . import _lib
    for s in range(1, steps + 1):
        try:
            dt = forms["fp64"].cfl()
        except _lib.MisoError as exc:
            # the FP64 form (the reference's arithmetic) met a non-positive
            # density or internal energy: record where, and stop
            q = forms["fp64"].download()[inner]
            rec = {"problem": prob.name, "failed_at_step": s, "time": t, "form": "fp64",
                   "error": str(exc), "min_rho": float(q[P.RO].min()),
                   "min_ei": float(q[P.EI].min())}
            emit(json.dumps(rec))
            break
        forms["fp64"].update(dt)
        forms["fp32_split"].update(dt)
        t += dt
        if s % every == 0 or s == steps:
            a = forms["fp32_split"].download()[inner]
            b = forms["fp64"].download()[inner]
            rec = {"problem": prob.name, "steps": s, "time": t, **_errors(a, b, gm),
                   "drift_fp64": _drift(forms["fp64"].monitors(), m0["fp64"]),
                   "drift_split": _drift(forms["fp32_split"].monitors(), m0["fp32_split"])}
            emit(json.dumps(rec))
    for v in forms.values():
        v.close()
    return rec


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--problem", choices=sorted(PROBLEMS), default="turbulence")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--every", type=int, default=250)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--smooth", type=float, default=0.0,
                    help="blast: width in cells of the tanh edge of the sphere (0 = step)")
    args = ap.parse_args(argv)
    prob = PROBLEMS[args.problem](args.n, args.seed, args.smooth)
    compare(prob, args.steps, args.every, emit=lambda s: print(s, flush=True))
    return 0


if __name__ == "__main__":
    sys.exit(main())
