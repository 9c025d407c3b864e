"""Full time steps of the CUDA engine against the CPU oracle.

Parity bar (floating point): relative difference <= 1e-10 in velocity,
pressure, nonlinear term and per-particle drag after the stated number of
steps; set-up integer data (active reversal points, solid mask) bit-exact.
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


def compare(gpu, cpu, tol=TOL):
    sg, sc = gpu.get_state(), cpu.get_state()
    out = {k: rel(sg[k], sc[k]) for k in ("u", "p", "nl")}
    out["umean"] = rel(sg["umean"], sc["umean"])
    out["mpg"] = rel(sg["mpg"], sc["mpg"])
    if gpu.nbody:
        pg, vg, fg, _, _ = gpu.get_particles()
        pc, vc, fc, _, _ = cpu.get_particles()
        out["pres"], out["visc"], out["force"] = rel(pg, pc), rel(vg, vc), rel(fg, fc)
    assert abs(sg["t"] - sc["t"]) <= tol * abs(sc["t"])
    bad = {k: v for k, v in out.items() if not v <= tol}
    assert not bad, out
    return out


@pytest.mark.gpu
def test_setup_geometry_bit_exact():
    prm, xc = config.random_array(my=64, dia_cells=12, nbody=12, seed=7, mc_moves=200)
    gpu, cpu = make_pair(prm, xc)
    assert gpu.nbnd == cpu.nbnd
    assert gpu.info.count_solid == cpu.info.count_solid
    assert np.array_equal(gpu.get_if_rev(), cpu.get_if_rev())
    assert np.array_equal(gpu.get_fluid_mask(), cpu.get_fluid_mask())
    assert gpu.info.dt == cpu.info.dt


@pytest.mark.gpu
@pytest.mark.parametrize("scheme,limiter", [("upwind", "none"), ("upwind", "minmod"), ("center", "none")])
def test_single_sphere_32_steps(scheme, limiter):
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    prm.update(discr_scheme=scheme, limiter=limiter)
    gpu, cpu = make_pair(prm, xc)
    for _ in range(10):
        rg, rc = gpu.step(), cpu.step()
    compare(gpu, cpu)
    assert abs(rg["divmax"]) < 1e-12


@pytest.mark.gpu
def test_single_sphere_64_100_steps():
    """Single fixed sphere, 64^3, d=16, Re=20, fluid at rest, 100 steps."""
    prm, xc = config.single_sphere(my=64, dia_cells=16, re=20.0)
    gpu, cpu = make_pair(prm, xc)
    for _ in range(100):
        gpu.step(); cpu.step()
    compare(gpu, cpu)


@pytest.mark.gpu
def test_random_array_64_10_spheres_100_steps():
    """Reduced random array: 64^3, 10 spheres of d=12, 100 steps."""
    prm, xc = config.random_array(my=64, dia_cells=12, nbody=10, re=50.0, seed=1234, mc_moves=1000)
    gpu, cpu = make_pair(prm, xc)
    for _ in range(100):
        gpu.step(); cpu.step()
    compare(gpu, cpu)


@pytest.mark.gpu
def test_graph_run_equals_step_loop_bitwise():
    prm, xc = config.random_array(my=32, dia_cells=8, nbody=4, seed=3, mc_moves=100)
    a = pk.Solver(config.make_params(prm), xc)
    b = pk.Solver(config.make_params(prm), xc)
    for _ in range(7):
        a.step()
    b.run(7)
    sa, sb = a.get_state(), b.get_state()
    for k in ("u", "p", "nl"):
        assert np.array_equal(sa[k], sb[k]), k


@pytest.mark.gpu
def test_state_round_trip_and_restart():
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    a = pk.Solver(config.make_params(prm), xc)
    a.run(5)
    st = a.get_state()
    b = pk.Solver(config.make_params(prm), xc)
    b.set_state(st)
    a.run(3); b.run(3)
    sa, sb = a.get_state(), b.get_state()
    for k in ("u", "p", "nl"):
        assert np.array_equal(sa[k], sb[k]), k


@pytest.mark.gpu
def test_deterministic_rerun():
    prm, xc = config.random_array(my=32, dia_cells=8, nbody=4, seed=5, mc_moves=100)
    outs = []
    for _ in range(2):
        s = pk.Solver(config.make_params(prm), xc)
        s.run(5)
        outs.append(s.get_state()["u"])
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.gpu
def test_random_array_256_two_steps():
    """256^3 grid (8-CTA plane clusters, 4-line x tiles), 6 spheres of d=20:
    two steps against the oracle."""
    prm, xc = config.random_array(my=256, dia_cells=20, nbody=6, seed=3, mc_moves=20)
    gpu, cpu = make_pair(prm, xc)
    for _ in range(2):
        gpu.step()
        cpu.step()
    compare(gpu, cpu)
