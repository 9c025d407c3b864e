"""CPU oracle of the passive scalar: invariants that need no GPU."""
import numpy as np

from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc


def _run(prm, xc, steps):
    P = config.make_params(prm)
    parts = config.Particles(xc)
    s = oc.OracleSolver(P, parts.struct)
    s._parts = parts
    for _ in range(steps):
        rep = s.step()
    return s, rep


def test_uniform_scalar_in_uniform_flow_stays_uniform():
    """No spheres, uniform flow, phi = 1: the flux is constant, the diffusion
    and the forcing vanish, so phi stays 1 and heat_ratio stays 1."""
    prm, _ = config.single_sphere(my=32, dia_cells=8)
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=1.0, phistream=1.0, initialize_zero=False)
    s, rep = _run(prm, np.zeros((0, 3)), 5)
    sc = oc.get_scalar(s)
    phif = sc["phif"]
    assert abs(phif[0, 0, :].real - 1.0).max() < 1e-12
    phif[0, 0, :] = 0.0
    assert np.abs(phif).max() < 1e-12
    assert abs(sc["heat_ratio"] - 1.0) < 1e-12


def test_cold_sphere_heats_the_fluid_side_flux():
    """A sphere colder than the stream draws heat: positive surface flux of
    grad phi . n, a finite heat ratio and a Nusselt number of a few units at
    Re = 20, Pr = 0.7 (Ranz-Marshall gives about 4.4 for an isolated sphere)."""
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=0.0, phistream=1.0, initialize_zero=False)
    s, rep = _run(prm, xc, 30)
    sc = oc.get_scalar(s)
    assert sc["flux_body"][0] > 0.0
    assert np.isfinite(sc["heat_ratio"]) and 0.9 < sc["heat_ratio"] < 1.1
    assert 1.0 < rep["nusselt"] < 20.0


def test_scalar_wave_in_uniform_flow_decays_by_the_crank_nicolson_factor():
    """No spheres, uniform flow along x, phi = 1 + eps sin(ky y): the wave
    does not vary along the flow, so the x flux cancels and heat_ratio
    stays 1; the ky mode then only diffuses, with gamma = vis / Pr
    (scalar_init.F90:58-122), and each step multiplies it by the
    Crank-Nicolson factor (1 - gamma dt ky^2 / 2) / (1 + gamma dt ky^2 / 2)
    of the scalar's line solve (phistep, stepthescalar.F90:99-213)."""
    prm, _ = config.single_sphere(my=32, dia_cells=8)
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=1.0, phistream=1.0, initialize_zero=False)
    s, _ = _run(prm, np.zeros((0, 3)), 1)
    P = s.params
    m, eps = 2, 0.01
    phif = np.zeros_like(s.get_scalar()["phif"])
    phif[0, 0, :] = 1.0
    phif[0, m, :] = -0.5j * eps
    s.set_scalar(phif, np.zeros_like(phif), 1.0, 1.0)
    k = 2 * np.pi * m / (P.lybyd * P.dia_phys)
    gamma = P.vis / 0.7
    prev = phif[0, m, :]
    for _ in range(4):
        s.step()
        dt = s.get_state()["dt"]
        sc = s.get_scalar()
        g = (1 - 0.5 * gamma * dt * k * k) / (1 + 0.5 * gamma * dt * k * k)
        line = sc["phif"][0, m, :]
        assert np.abs(line - g * prev).max() <= 1e-13 * eps
        assert abs(sc["heat_ratio"] - 1.0) < 1e-12
        assert np.abs(sc["phif"][0, 0, :] - 1.0).max() < 1e-12
        rest = np.abs(sc["phif"]).copy()
        rest[0, 0, :] = 0
        rest[0, m, :] = 0
        assert rest.max() <= 1e-13 * eps
        prev = line
