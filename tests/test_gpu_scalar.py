"""Passive scalar (ISCALON = 1) of the CUDA engine against the CPU oracle.

The scalar step (scalstep) runs after every flow step; it is periodic in x up
to heat_ratio, forced at the inner reversal points, and solved per (ky,kz)
line with twisted-periodic corners.  Parity bar: relative difference <= 1e-10
in phi, the flow state, the per-sphere surface flux, heat_ratio and the
Nusselt number after the stated number of steps.
"""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc

TOL = 1e-10


def rel(a, b):
    d = np.max(np.abs(np.asarray(a) - np.asarray(b)))
    s = np.max(np.abs(np.asarray(b)))
    return d / s if s > 0 else d


def make_pair(prm, xc):
    P = config.make_params(prm)
    parts = config.Particles(xc)
    gpu = pk.Solver(P, xc)
    cpu = oc.OracleSolver(P, parts.struct)
    cpu._parts = parts
    return gpu, cpu


def compare(gpu, cpu):
    sg, sc = gpu.get_scalar(), oc.get_scalar(cpu)
    out = {"phif": rel(sg["phif"], sc["phif"]),
           "heat_ratio": abs(sg["heat_ratio"] - sc["heat_ratio"]) / abs(sc["heat_ratio"]),
           "nusselt": abs(sg["nusselt"] - sc["nusselt"]) / max(abs(sc["nusselt"]), 1e-300)}
    if gpu.nbody:
        out["flux_body"] = rel(sg["flux_body"], sc["flux_body"])
    fg, fc = gpu.get_state(), cpu.get_state()
    for k in ("u", "p"):
        out[k] = rel(fg[k], fc[k])
    bad = {k: v for k, v in out.items() if not v <= TOL}
    assert not bad, out
    return out


def scalar_params(prm, **kw):
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=0.0, phistream=1.0, initialize_zero=False)
    prm.update(kw)
    return prm


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["upwind", "center"])
def test_scalar_single_sphere_32(scheme):
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    gpu, cpu = make_pair(scalar_params(prm, discr_scheme=scheme), xc)
    for _ in range(10):
        rg, rc = gpu.step(), cpu.step()
    out = compare(gpu, cpu)
    assert rg["heat_ratio"] != 1.0 and np.isfinite(rg["nusselt"])
    assert abs(rg["nusselt"] - rc["nusselt"]) <= TOL * abs(rc["nusselt"])


@pytest.mark.gpu
def test_scalar_spheres_across_the_x_boundary_64():
    """Spheres straddling x = 1 and x = nx exercise the twice-evaluated
    reversal points of the last cell and every heat_ratio wrap."""
    prm, xc = config.random_array(my=64, dia_cells=12, nbody=6, seed=11, mc_moves=50)
    xc = np.asarray(xc, dtype=np.float64).copy()
    xc[0, 0] = 1.3
    xc[1, 0] = 64.6
    xc[1, 1] = xc[0, 1] + 32.0 if xc[0, 1] + 32.0 < 65 else xc[0, 1] - 32.0
    gpu, cpu = make_pair(scalar_params(prm), xc)
    for _ in range(30):
        gpu.step()
        cpu.step()
    compare(gpu, cpu)


@pytest.mark.gpu
def test_scalar_random_array_256_two_steps():
    """256^3 grid: the scalar's x-line solves run in 4-line tiles there."""
    prm, xc = config.random_array(my=256, dia_cells=20, nbody=6, seed=3, mc_moves=20)
    gpu, cpu = make_pair(scalar_params(prm), xc)
    for _ in range(2):
        gpu.step()
        cpu.step()
    compare(gpu, cpu)


@pytest.mark.gpu
def test_scalar_started_on_a_developed_flow():
    """The reference starts a scalar run on a converged flow (restart with
    ISCALON = 1, phi = 1); the flow state is carried over with set_state."""
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    prm.update(initialize_zero=True)
    flow = pk.Solver(config.make_params(prm), xc)
    flow.run(20)
    st = flow.get_state()
    prm_s = dict(prm)
    prm_s.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=0.0, phistream=1.0)
    gpu, cpu = make_pair(prm_s, xc)
    gpu.set_state(st)
    cpu.set_state(st)
    for _ in range(8):
        gpu.step()
        cpu.step()
    compare(gpu, cpu)
