"""Run configuration with the reference's keys and defaults.

The keys are the ones the reference's integrator reads from its YAML
configuration (miso/include/miso/config.hpp:74-120 merges
config_defaults.hpp:3-33 under the user file):

* ``mhd.cfl_number`` (default 0.5)
* ``mhd.artificial_viscosity.{ep, fh, cs_fac, ca_fac, vv_fac}`` (defaults 1.0)
* ``eos.gm``
* ``domain.periodic.{x, y, z}``

A configuration is a plain nested ``dict``; :func:`merge_defaults` fills the
missing keys the way ``merge_yaml`` does (config.hpp:39-61).
"""
from __future__ import annotations

import copy

DEFAULTS = {
    "mhd": {
        "cfl_number": 0.5,
        "artificial_viscosity": {"ep": 1.0, "fh": 1.0, "cs_fac": 1.0, "ca_fac": 1.0,
                                 "vv_fac": 1.0},
    },
    "domain": {"periodic": {"x": False, "y": False, "z": False}},
}


def merge_defaults(target: dict | None, defaults: dict = DEFAULTS) -> dict:
    """Recursively add every default key absent from ``target``."""
    out = copy.deepcopy(target) if isinstance(target, dict) else {}
    for key, dval in defaults.items():
        if isinstance(dval, dict):
            out[key] = merge_defaults(out.get(key), dval)
        elif key not in out or out[key] is None:
            out[key] = dval
    return out


def make_config(gm: float, periodic=(False, False, False), cfl_number: float | None = None,
                **av) -> dict:
    """Build a configuration dict; ``av`` may set ep, fh, cs_fac, ca_fac, vv_fac."""
    cfg = {"eos": {"gm": float(gm)},
           "domain": {"periodic": {"x": bool(periodic[0]), "y": bool(periodic[1]),
                                   "z": bool(periodic[2])}},
           "mhd": {"artificial_viscosity": {k: float(v) for k, v in av.items()}}}
    if cfl_number is not None:
        cfg["mhd"]["cfl_number"] = float(cfl_number)
    bad = set(av) - {"ep", "fh", "cs_fac", "ca_fac", "vv_fac"}
    if bad:
        raise KeyError(f"unknown artificial_viscosity keys: {sorted(bad)}")
    return merge_defaults(cfg)
