"""Parity on the configurations that bench.py times, against the CPU oracle.

* the 128^3 fixed random array of the headline number (100 spheres of
  d = 20, phi = 0.2, Re = 50, upwind): 100 steps on the step graphs that
  bench.py replays, with the autotuned x-line tile, and the same 100 steps
  launched one by one with the other tile width (bitwise equal);
* a 96^3 fixed array (27 spheres of d = 16, phi = 0.15): 100 steps;
* a moving array at 96^3 (300 spheres of d = 8, Maxwellian velocities,
  soft-sphere DEM with collisions): 100 steps, the DEM lists NEIGHBOURS / PN /
  PV and the solid mask compared after every step;
* the moving suspension with the passive scalar at 256^3 (1202 spheres of
  d = 20, phi = 0.3, rhos/rhof = 100, DEM restitution 0.9, Pr 0.7): 3 steps.

Parity bar: velocity, pressure, nonlinear term, per-particle pressure and
viscous drag and force, umean and mpg within 1e-10 relative; set-up and DEM
integer data (masks, reversal-point flags, contact lists) identical.  Sphere
positions and velocities of the moving runs follow from the drag, which the
device sums in another order than the oracle's serial loop, so they agree to
rounding level (the test bounds them by 1e-10 relative after 100 steps and
1e-12 after 3).
"""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc

pytestmark = pytest.mark.gpu

TOL = 1e-10
# the headline workload of bench.py (kept equal to bench.WORKLOAD)
BENCH_WORKLOAD = dict(my=128, dia_cells=20.0, phi=0.2, re=50.0, seed=1234, mc_moves=1000)


def rel(a, b):
    d = np.max(np.abs(np.asarray(a) - np.asarray(b)))
    s = np.max(np.abs(np.asarray(b)))
    return d / s if s > 0 else d


def _pair(prm, xc, vel=None):
    P = config.make_params(prm)
    parts = config.Particles(xc, vel)
    gpu = pk.Solver(P, xc, vel)
    cpu = oc.OracleSolver(P, parts.struct)
    cpu._parts = parts
    return gpu, cpu


def _compare_flow(gpu, cpu, tol=TOL):
    sg, sc = gpu.get_state(), cpu.get_state()
    out = {k: rel(sg[k], sc[k]) for k in ("u", "p", "nl", "umean", "mpg")}
    pg, vg, fg, _, _ = gpu.get_particles()
    pc, vc, fc, _, _ = cpu.get_particles()
    out.update(pres=rel(pg, pc), visc=rel(vg, vc), force=rel(fg, fc))
    assert abs(sg["t"] - sc["t"]) <= tol * abs(sc["t"])
    assert abs(sg["dt"] - sc["dt"]) <= tol * abs(sc["dt"])
    bad = {k: v for k, v in out.items() if not v <= tol}
    assert not bad, out
    return out


def _compare_dem(gpu, cpu, tol_pos):
    _, _, _, xg, vg = gpu.get_particles()
    _, _, _, xcpu, vcpu = cpu.get_particles()
    assert rel(xg, xcpu) <= tol_pos and rel(vg, vcpu) <= tol_pos, (rel(xg, xcpu), rel(vg, vcpu))
    cg, cc = gpu.get_contacts(), oc.get_contacts(cpu)
    for k in ("neighbours", "pn", "pv"):
        assert np.array_equal(cg[k], cc[k]), k
    assert np.array_equal(gpu.get_fluid_mask(), cpu.get_fluid_mask())
    assert np.array_equal(gpu.get_if_rev(), cpu.get_if_rev())
    return int(cg["pn"][0].sum())


def test_bench_workload_128_100_steps():
    """The benchmarked path: 128^3, 100 spheres of d = 20 (phi = 0.2), Re 50,
    fluid at rest, 100 steps.  Run A replays the step graphs (pibm_run, what
    bench.py times) with the tile the autotuner chose; run B steps one launch
    sequence at a time with the other x-line tile width.  Both must equal each
    other bitwise and the oracle within 1e-10."""
    prm, xc = config.random_array(**BENCH_WORKLOAD)
    assert xc.shape[0] == 100
    a, cpu = _pair(prm, xc)
    assert np.array_equal(a.get_if_rev(), cpu.get_if_rev())
    assert np.array_equal(a.get_fluid_mask(), cpu.get_fluid_mask())
    assert a.info.npts_active == cpu.info.npts_active
    tile = a.tuning()["lines_per_cta"]
    b = pk.Solver(config.make_params(prm), xc)
    b.set_tuning(8 if tile == 4 else 4)
    # first step: the set-up transient (fluid at rest, first dt)
    a.run(1)
    b.step()
    cpu.step()
    _compare_flow(a, cpu)
    a.run(99)
    for _ in range(99):
        b.step()
        cpu.step()
    out = _compare_flow(a, cpu)
    sa, sb = a.get_state(), b.get_state()
    for k in ("u", "p", "nl"):
        assert np.array_equal(sa[k], sb[k]), k
    print("128^3 bench workload, 100 steps, max rel diff:", out)


def test_random_array_96_100_steps():
    """96^3 fixed random array, 27 spheres of d = 16 (phi = 0.15), Re 50, 100 steps."""
    prm, xc = config.random_array(my=96, dia_cells=16.0, phi=0.15, re=50.0, seed=77, mc_moves=500)
    gpu, cpu = _pair(prm, xc)
    for _ in range(100):
        gpu.step()
        cpu.step()
    _compare_flow(gpu, cpu)


def test_moving_96_300_spheres_100_steps_lists_every_step():
    """Moving array at 96^3: 300 spheres of d = 8, Maxwellian velocities of
    spread 2 uchar, density ratio 100, soft-sphere DEM (e = 0.9), 100 steps.
    The contact lists, the solid mask and the active reversal points must be
    identical after every step."""
    prm, xc, vel = config.moving_array(my=96, dia_cells=8.0, nbody=300, seed=21, vel_spread=2.0)
    gpu, cpu = _pair(prm, xc, vel)
    contacts = 0
    for it in range(100):
        rg, rc = gpu.step(), cpu.step()
        assert rg["nrpr_active_total"] == rc["nrpr_active_total"], it
        contacts = max(contacts, _compare_dem(gpu, cpu, tol_pos=TOL))
    assert contacts > 0   # collisions happened
    _compare_flow(gpu, cpu)


def test_moving_suspension_256_scalar_3_steps():
    """The moving-suspension configuration of bench.py: 256^3, 1202 spheres of
    d = 20 (phi = 0.3), rhos/rhof = 100, Maxwellian velocities (0.1 uchar),
    soft-sphere DEM with restitution 0.9, passive scalar Pr 0.7 with the
    spheres at phisurf = 1 in a stream at 0; 3 steps."""
    prm, xc, vel = config.moving_array(my=256, dia_cells=20.0, nbody=1202, seed=2024, rhos=100.0, coeff_rest=0.9,
                                       vel_spread=0.1, mc_moves=1000)
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=1.0, phistream=0.0, initialize_zero=False)
    gpu, cpu = _pair(prm, xc, vel)
    for it in range(3):
        rg, rc = gpu.step(), cpu.step()
        assert rg["nrpr_active_total"] == rc["nrpr_active_total"], it
        _compare_dem(gpu, cpu, tol_pos=1e-12)
    _compare_flow(gpu, cpu)
    sg, sc = gpu.get_scalar(), oc.get_scalar(cpu)
    assert rel(sg["phif"], sc["phif"]) <= TOL
    assert rel(sg["flux_body"], sc["flux_body"]) <= TOL
    assert abs(rg["nusselt"] - rc["nusselt"]) <= TOL * abs(rc["nusselt"])
