"""Moving particles (IMOVE = 1) on the CUDA engine against the CPU oracle:
the soft-sphere DEM sub-steps, the per-step solid mask, reversal-point
activity and spreading map, and the flow they drive.

Parity bar: positions and velocities of the spheres within 1e-12 (relative
to the largest), the DEM neighbour and contact lists, the solid mask and the
active reversal points identical, the flow state within 1e-10 as for fixed
spheres.  The per-sphere drag that drives the DEM is summed in another order
on the device (rounding level), so positions are compared with a tolerance.
"""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc

TOL = 1e-10
TOL_POS = 1e-12


def rel(a, b):
    d = np.max(np.abs(np.asarray(a) - np.asarray(b)))
    s = np.max(np.abs(np.asarray(b)))
    return d / s if s > 0 else d


def make_pair(prm, xc, vel):
    P = config.make_params(prm)
    parts = config.Particles(xc, vel)
    gpu = pk.Solver(P, xc, vel)
    cpu = oc.OracleSolver(P, parts.struct)
    cpu._parts = parts
    return gpu, cpu


def compare(gpu, cpu, lists=True):
    _, _, _, xg, vg = gpu.get_particles()
    _, _, _, xcpu, vcpu = cpu.get_particles()
    out = {"xc": rel(xg, xcpu), "vel": rel(vg, vcpu)}
    assert out["xc"] <= TOL_POS and out["vel"] <= TOL_POS, out
    if lists:
        cg, cc = gpu.get_contacts(), oc.get_contacts(cpu)
        for k in ("neighbours", "pn", "pv"):
            assert np.array_equal(cg[k], cc[k]), k
    assert np.array_equal(gpu.get_fluid_mask(), cpu.get_fluid_mask())
    assert np.array_equal(gpu.get_if_rev(), cpu.get_if_rev())
    sg, sc = gpu.get_state(), cpu.get_state()
    for k in ("u", "p", "nl"):
        out[k] = rel(sg[k], sc[k])
        assert out[k] <= TOL, out
    return out


def _head_on(collision="softsphere", rhos=1000.0):
    prm, _ = config.single_sphere(my=32, dia_cells=8)
    prm.update(imove=1, collision_type=collision, rhos=rhos, rhof=1.0, coeff_rest=0.9, initialize_zero=True)
    xc = np.array([[10.0, 16.5, 16.5], [20.0, 16.5, 16.5]])
    vel = np.array([[0.5, 0.0, 0.0], [-0.5, 0.0, 0.0]])
    return prm, xc, vel


@pytest.mark.gpu
def test_head_on_collision_matches_oracle():
    prm, xc, vel = _head_on()
    gpu, cpu = make_pair(prm, xc, vel)
    compare(gpu, cpu)
    contact = False
    for it in range(24):
        rg, rc = gpu.step(), cpu.step()
        if it % 4 == 3:
            compare(gpu, cpu)
        contact |= gpu.get_contacts()["pn"][0, 0] > 0
        assert rg["nrpr_active_total"] == rc["nrpr_active_total"]
    assert contact
    compare(gpu, cpu)


@pytest.mark.gpu
def test_no_collision_translation_matches_oracle():
    prm, xc, vel = _head_on(collision="none")
    vel = vel * 0.2
    gpu, cpu = make_pair(prm, xc, vel)
    for _ in range(10):
        gpu.step(); cpu.step()
    compare(gpu, cpu, lists=False)


@pytest.mark.gpu
@pytest.mark.parametrize("my,dia,nbody,seed,spread", [(32, 6.0, 50, 4, 2.0), (64, 10.0, 60, 9, 1.5), (96, 8.0, 300, 21, 2.0)])
def test_moving_array_matches_oracle(my, dia, nbody, seed, spread):
    """A freely moving random array with Maxwellian velocities (several
    collisions, spheres crossing the periodic boundaries, reversal points
    switched off inside neighbours), 12 steps.  The DEM coarse grid has one
    cell per direction at 32^3 and 64^3 (serial search path) and seven at
    96^3 with d = 8 (the lane-per-cell search path)."""
    prm, xc, vel = config.moving_array(my=my, dia_cells=dia, nbody=nbody, seed=seed, vel_spread=spread)
    gpu, cpu = make_pair(prm, xc, vel)
    for _ in range(12):
        rg, rc = gpu.step(), cpu.step()
        assert rg["nrpr_active_total"] == rc["nrpr_active_total"]
    compare(gpu, cpu)


@pytest.mark.gpu
def test_moving_graph_replay_equals_steps():
    """pibm_run (captured graphs with the DEM sub-step loop) gives the same
    particles and flow as step-by-step launches."""
    prm, xc, vel = config.moving_array(my=32, dia_cells=6.0, nbody=50, seed=4, vel_spread=2.0)
    a = pk.Solver(config.make_params(prm), xc, vel)
    b = pk.Solver(config.make_params(prm), xc, vel)
    for _ in range(8):
        a.step()
    b.run(8)
    _, _, _, xa, va = a.get_particles()
    _, _, _, xb, vb = b.get_particles()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    assert np.array_equal(a.get_state()["u"], b.get_state()["u"])


@pytest.mark.gpu
def test_moving_with_passive_scalar_matches_oracle():
    """IMOVE = 1 with ISCALON = 1 (the freely evolving heated suspension): the
    scalar's reversal-point evaluations and spreading are rebuilt on the
    moved geometry every step; spheres cross the periodic x boundary."""
    prm, xc, vel = config.moving_array(my=32, dia_cells=6.0, nbody=50, seed=4, vel_spread=2.0)
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=0.0, phistream=1.0, initialize_zero=False)
    xc = xc.copy()
    xc[0, 0] = 1.2
    vel = vel.copy()
    vel[0, 0] = -abs(vel[0, 0]) - 0.1
    gpu, cpu = make_pair(prm, xc, vel)
    for _ in range(12):
        rg, rc = gpu.step(), cpu.step()
        assert rg["nrpr_active_total"] == rc["nrpr_active_total"]
    compare(gpu, cpu)
    sg, sc = gpu.get_scalar(), oc.get_scalar(cpu)
    assert rel(sg["phif"], sc["phif"]) <= TOL
    assert rel(sg["flux_body"], sc["flux_body"]) <= TOL
    assert abs(sg["heat_ratio"] - sc["heat_ratio"]) <= TOL * abs(sc["heat_ratio"])
    assert abs(rg["nusselt"] - rc["nusselt"]) <= TOL * abs(rc["nusselt"])
