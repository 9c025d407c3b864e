"""Physics sanity of the whole step on the CUDA engine: the Stokes-limit drag
of a simple cubic array of fixed spheres against Hasimoto's periodic-array
result, F / (3 pi mu d U_s) = 1 / (1 - 1.7601 c + c^3 - 1.5593 c^6 +
3.9799 c^8 - 3.0734 c^10), c = phi^(1/3) (Hasimoto 1959 with the
Sangani-Acrivos 1982 terms), U_s the superficial velocity.

One sphere of 16 cells in a 64^3 box (phi = 0.0082, K = 1.530), Re = 0.05,
mean flow held by the mpg controller (SET_MPG = F), so norm_drag is exactly
that ratio.  The direct-forcing step imposes the no-slip condition at the
reversal points while the forces act on the solid nodes, so the steady state
carries a slip error of order dt: the time step is set through VFL, the
reference's number of steps per viscous time at Re < 1 (initialize_flo.F90:
603), and the drag must approach K from below as dt shrinks, to within the
spatial error of d/dx = 16 (measured: 0.95 K with dt = 0.0017 dx/U, 0.967 K with
dt = 0.0005 dx/U, i.e. VFL 1600)."""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config

pytestmark = pytest.mark.gpu


def hasimoto(phi):
    c = phi ** (1.0 / 3.0)
    return 1.0 / (1.0 - 1.7601 * c + c ** 3 - 1.5593 * c ** 6 + 3.9799 * c ** 8 - 3.0734 * c ** 10)


def steady_drag(vfl, my=64, d=16.0, max_steps=40000):
    prm, xc = config.single_sphere(my=my, dia_cells=d, re=0.05, cfl=0.5)
    prm.update(vfl=vfl)
    s = pk.Solver(config.make_params(prm), xc)
    prev, n = None, 0
    while n < max_steps:
        nd = s.run(2000)["norm_drag"]
        n += 2000
        if prev is not None and abs(nd - prev) < 1e-7 * abs(nd):
            break
        prev = nd
    s.close()
    return nd


def test_stokes_drag_approaches_hasimoto_as_dt_shrinks():
    K = hasimoto(np.pi / 6.0 * (16.0 / 64.0) ** 3)
    coarse = steady_drag(480.0)
    fine = steady_drag(1600.0)
    assert coarse < fine < K
    assert fine > 0.95 * K, (fine, K)
    assert abs(fine - K) < abs(coarse - K)


def test_stokes_drag_at_higher_volume_fraction():
    """phi = 0.065 (d = 32 cells in 64^3, the Sangani-Acrivos series gives
    K = 2.842; Zick & Homsy's tabulated 2.81 at phi = 0.064): the engine's
    steady drag at a viscous number of 0.075 is within 3% below it
    (measured 2.762)."""
    K = hasimoto(np.pi / 6.0 * (32.0 / 64.0) ** 3)
    nd = steady_drag(12800.0, my=64, d=32.0)
    assert 0.95 * K < nd < K, (nd, K)
