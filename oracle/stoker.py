"""Stoker's analytic solution of the wet dam break -- TEST INFRASTRUCTURE ONLY.

The reference checks its schemes against the SWASHES 1.03.00 wet dam-break
solution (reference/swashes_1_nx=*.csv, used by ConvergenceShock1D.ipynb
cells 5-16: L = 10 m, dam at x = 5 m, h = 0.005 m left, 0.001 m right,
t = 6 s).  This module restates the published Stoker solution that SWASHES
evaluates: a left rarefaction fan, a constant middle state and a right-moving
shock.  The middle depth h_m solves

    2 (sqrt(g h_l) - sqrt(g h_m)) = (h_m - h_r) sqrt(g (h_m + h_r) / (2 h_m h_r)),

the Riemann invariant across the fan equated with the Rankine-Hugoniot
velocity behind the shock; the shock moves at S = h_m u_m / (h_m - h_r).
tests/test_oracle.py pins this function against the SWASHES CSVs.
"""

from __future__ import annotations

import numpy as np


def middle_state(h_l, h_r, g=9.81):
    def f(hm):
        return 2.0 * (np.sqrt(g * h_l) - np.sqrt(g * hm)) - (hm - h_r) * np.sqrt(g * (hm + h_r) / (2.0 * hm * h_r))

    lo, hi = h_r, h_l
    for _ in range(200):  # bisection: f(h_r) > 0 > f(h_l)
        mid = 0.5 * (lo + hi)
        if f(mid) > 0.0:
            lo = mid
        else:
            hi = mid
    h_m = 0.5 * (lo + hi)
    u_m = 2.0 * (np.sqrt(g * h_l) - np.sqrt(g * h_m))
    return h_m, u_m


def stoker(x, t, x0=5.0, h_l=0.005, h_r=0.001, g=9.81):
    """Depth h and velocity u of the wet dam break at positions x and time t > 0."""
    x = np.asarray(x, dtype=np.float64)
    h_m, u_m = middle_state(h_l, h_r, g)
    c_l = np.sqrt(g * h_l)
    c_m = np.sqrt(g * h_m)
    S = h_m * u_m / (h_m - h_r)
    xi = (x - x0) / t
    h = np.empty_like(x)
    u = np.empty_like(x)
    left = xi <= -c_l
    fan = (xi > -c_l) & (xi <= u_m - c_m)
    mid = (xi > u_m - c_m) & (xi <= S)
    right = xi > S
    h[left], u[left] = h_l, 0.0
    h[fan] = (2.0 * c_l - xi[fan]) ** 2 / (9.0 * g)
    u[fan] = 2.0 / 3.0 * (c_l + xi[fan])
    h[mid], u[mid] = h_m, u_m
    h[right], u[right] = h_r, 0.0
    return h, u
