"""Exact solution of the 1-D Riemann problem for an ideal gas.

Used to restate the reference's shock-tube accuracy test
(miso/tests/serial/test_hd1d_shock_tube.cpp:21-82: relative L1 of density and
velocity against the exact Sod solution below 5e-2).  Written from the
textbook method -- the star-region pressure solves
f_L(p) + f_R(p) + (u_R - u_L) = 0 by Newton iteration, with the shock
(Rankine-Hugoniot) or rarefaction (isentropic) branch for each side, and the
self-similar solution is then sampled at x/t (E. F. Toro, Riemann Solvers
and Numerical Methods for Fluid Dynamics, ch. 4).
"""
from __future__ import annotations

import math

import numpy as np


def _f(p, rho, pk, c, g):
    if p > pk:  # shock
        a = 2.0 / ((g + 1.0) * rho)
        b = (g - 1.0) / (g + 1.0) * pk
        q = math.sqrt(a / (p + b))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (b + p))
    # rarefaction
    r = (p / pk) ** ((g - 1.0) / (2.0 * g))
    return 2.0 * c / (g - 1.0) * (r - 1.0), 1.0 / (rho * c) * (p / pk) ** (-(g + 1.0) / (2.0 * g))


def star_state(rl, ul, pl, rr, ur, pr, g):
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = max(1e-8, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p_new = max(1e-10, p - dp)
        if abs(p_new - p) < 1e-14 * (p_new + p):
            p = p_new
            break
        p = p_new
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(x, t, x0, rl, ul, pl, rr, ur, pr, g):
    """Density, velocity and pressure at positions x, time t > 0."""
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    out_r = np.empty_like(x, dtype=float)
    out_u = np.empty_like(out_r)
    out_p = np.empty_like(out_r)
    gm = (g - 1.0) / (g + 1.0)
    for n, xx in enumerate(x):
        s = (xx - x0) / t
        if s <= us:  # left of the contact
            if ps > pl:  # left shock
                sl = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= sl:
                    r, u, p = rl, ul, pl
                else:
                    r = rl * (ps / pl + gm) / (gm * ps / pl + 1.0)
                    u, p = us, ps
            else:  # left rarefaction
                shl = ul - cl
                cml = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - cml
                if s <= shl:
                    r, u, p = rl, ul, pl
                elif s >= stl:
                    r, u, p = rl * (ps / pl) ** (1.0 / g), us, ps
                else:
                    u = 2.0 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                    c = 2.0 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                    r = rl * (c / cl) ** (2.0 / (g - 1))
                    p = pl * (c / cl) ** (2.0 * g / (g - 1))
        else:  # right of the contact
            if ps > pr:  # right shock
                sr = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= sr:
                    r, u, p = rr, ur, pr
                else:
                    r = rr * (ps / pr + gm) / (gm * ps / pr + 1.0)
                    u, p = us, ps
            else:  # right rarefaction
                shr = ur + cr
                cmr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + cmr
                if s >= shr:
                    r, u, p = rr, ur, pr
                elif s <= str_:
                    r, u, p = rr * (ps / pr) ** (1.0 / g), us, ps
                else:
                    u = 2.0 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                    c = 2.0 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                    r = rr * (c / cr) ** (2.0 / (g - 1))
                    p = pr * (c / cr) ** (2.0 * g / (g - 1))
        out_r[n], out_u[n], out_p[n] = r, u, p
    return out_r, out_u, out_p
