"""Where the discrete drag objective is smooth in a sphere coordinate.

A step's drag (calc_pres_visc_drag, boundary_condition.F90:1481-1645) and
reversal forcing (calc_inner_reversal_forcing, :1104-1479) interpolate
trilinearly at points that move with the sphere centre: the surface points
xc + R*b, the inner and outer reversal points xc + (R -+ dr)*b, and, for the
pressure, each of them shifted by -1/2 in x.  The interpolation weights are
linear inside a grid cell, so the step is smooth in a coordinate of xc as
long as no such point crosses a cell face (an integer coordinate) -- there
the gradient jumps -- and as long as no grid node enters or leaves the
sphere (the solid mask of grid_nodes_insphere, dependent_functions.F90:
783-963), which changes the step itself.  smooth_interval returns the
offsets of the nearest such event on either side, so that a finite
difference of J can be taken inside one smooth piece.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

SMALL = float(np.float32(1.0e-35))   # the mask's tolerance, SMALL_NUMBER


def smooth_interval(xc_m: np.ndarray, d: int, bnd: np.ndarray, radbdy: float, dr: float) -> Tuple[float, float]:
    """(lo, hi) with lo <= 0 <= hi: moving coordinate d of sphere centre
    xc_m (grid units) by any t with lo < t < hi crosses no cell face with a
    stencil point and changes no node of the solid mask.  bnd: (nbnd, 3)
    unit directions of the surface points (Solver.get_surface_points)."""
    c = float(xc_m[d])
    lo, hi = -math.inf, math.inf
    for r, shifts in ((radbdy, (0.0, 0.5)), (radbdy - dr, (0.0, 0.5)), (radbdy + dr, (0.0,))):
        v0 = c + bnd[:, d] * r
        for s in shifts if d == 0 else (0.0,):
            v = v0 - s
            f = np.floor(v)
            hi = min(hi, float(np.min(f + 1.0 - v)))
            lo = max(lo, -float(np.min(v - f)))
    # grid nodes within reach of the sphere surface: membership |node - xc| <= R
    R = radbdy + SMALL
    ax = [np.arange(math.ceil(float(xc_m[k]) - R) - 1, math.floor(float(xc_m[k]) + R) + 2) for k in range(3)]
    g = np.stack(np.meshgrid(*ax, indexing="ij"), -1).reshape(-1, 3).astype(float)
    a = g[:, d] - c
    o = [k for k in range(3) if k != d]
    q = (g[:, o[0]] - float(xc_m[o[0]])) ** 2 + (g[:, o[1]] - float(xc_m[o[1]])) ** 2
    ok = q <= R * R
    s = np.sqrt(R * R - q[ok])
    ev = np.concatenate([a[ok] - s, a[ok] + s])
    if np.any(ev > 0):
        hi = min(hi, float(ev[ev > 0].min()))
    if np.any(ev < 0):
        lo = max(lo, float(ev[ev < 0].max()))
    if np.any(ev == 0):
        lo = hi = 0.0
    return lo, hi


def fd_step(xc_m: np.ndarray, d: int, bnd: np.ndarray, radbdy: float, dr: float, h_max: float,
            margin: float = 0.9) -> float:
    """The largest central-difference step <= h_max whose interval
    [c - h, c + h] lies inside one smooth piece (0 when an event sits at c)."""
    lo, hi = smooth_interval(xc_m, d, bnd, radbdy, dr)
    return min(h_max, margin * min(-lo, hi))
