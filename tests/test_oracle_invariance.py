"""Translation invariance of the oracle step on the periodic grid.

Moving every sphere by a whole number of cells (across the periodic
boundaries, so that surface points, reversal points, their interpolation
stencils and the spreading reach over the edges) must move the whole
solution by the same number of cells: the set-up (geom_init.F90:44-242,
dependent_functions.F90:783-1051) places everything relative to the
centres and wraps indices periodically, and the spectral and x-line
solves do not see the shift.  The fields agree to rounding and the drag
history to rounding, step by step.

One part of the reference is not translation invariant and the oracle
keeps it: check_external_pt (dependent_functions.F90:966-1051) wraps an
outer reversal point into the box and measures its distance to a
neighbour's centre as stored, without the neighbour's periodic image, so a
point that lies inside a neighbour across a boundary stays active.  The
invariance cases therefore keep every reversal point clear of the other
spheres, and a close-packed array shows the departure.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle_ctypes as oc  # noqa: E402
from pureibm_ps2d_fd1d_b200 import config  # noqa: E402


def _run(prm, xc, nsteps):
    parts = config.Particles(xc)
    s = oc.OracleSolver(config.make_params(prm), parts.struct)
    try:
        reps = [s.step() for _ in range(nsteps)]
        u = s.get_state()["u"]
        real = np.stack([oc.ff2cr(np.transpose(u[c, :, :, :s.nx], (2, 0, 1)), s.my) for c in range(3)])
        return real, reps          # real: (3, x, z, y)
    finally:
        s.close()


def _shifted(xc, shift, n):
    """Centres moved by whole cells, wrapped into [1, n + 1) (grid units,
    node i at coordinate i)."""
    return (np.asarray(xc, dtype=np.float64) + np.asarray(shift, dtype=np.float64) - 1.0) % n + 1.0


def _cases():
    prm1, xc1 = config.single_sphere(my=32, dia_cells=8.0, re=5.0)
    prm3, _ = config.single_sphere(my=32, dia_cells=6.0, re=10.0)
    # three spheres far apart (centre distances > 19 cells), off-node by
    # dyadic fractions so that the shifted centres are exact; the shift puts
    # the first one on the corner of the box
    xc3 = np.array([[6.25, 6.75, 6.125], [20.5, 10.375, 24.875], [12.625, 26.25, 16.5]])
    return [("single_sphere", prm1, xc1, (14, 13, 15)),
            ("three_spheres", prm3, xc3, (27, 29, 28))]


@pytest.mark.parametrize("name,prm,xc,shift", _cases(), ids=lambda v: v if isinstance(v, str) else "")
def test_whole_cell_shift_shifts_the_solution(name, prm, xc, shift):
    n = int(prm["my"])
    r0, rep0 = _run(prm, xc, 8)
    r1, rep1 = _run(prm, _shifted(xc, shift, n), 8)
    # x, y, z shifts act on axes 1 (x), 3 (y) and 2 (z) of (comp, x, z, y)
    expect = np.roll(r0, shift=(shift[0], shift[2], shift[1]), axis=(1, 2, 3))
    assert np.abs(r1 - expect).max() <= 1e-13 * np.abs(r0).max()
    for a, b in zip(rep0, rep1):
        assert a["dt"] == b["dt"]
        assert b["norm_drag"] == pytest.approx(a["norm_drag"], rel=1e-12)
        assert b["nrpr_active_total"] == a["nrpr_active_total"]


def test_three_spheres_keep_every_reversal_point():
    """The invariance case above is clear of check_external_pt: every outer
    reversal point of every sphere is active, shifted or not."""
    _, prm, xc, shift = _cases()[1]
    for centres in (xc, _shifted(xc, shift, int(prm["my"]))):
        parts = config.Particles(centres)
        s = oc.OracleSolver(config.make_params(prm), parts.struct)
        try:
            rep = s.step()
            assert rep["nrpr_active_total"] == s.nbnd * s.nbody
            assert s.get_if_rev().all()
        finally:
            s.close()


def test_close_pairs_across_a_boundary_are_checked_without_the_periodic_image():
    """A close-packed random array (outer reversal points inside
    neighbours): shifting it moves pairs onto and off the boundaries, and
    the number of points check_external_pt deactivates changes, as in the
    reference."""
    prm, xc = config.random_array(my=32, dia_cells=6.0, phi=0.06, re=20.0, seed=5, mc_moves=50)
    _, rep0 = _run(prm, xc, 1)
    _, rep1 = _run(prm, _shifted(xc, (7, 20, 11), 32), 1)
    assert rep0[0]["nrpr_active_total"] != rep1[0]["nrpr_active_total"]
