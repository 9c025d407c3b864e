"""CPU oracle of moving particles (IMOVE = 1, soft-sphere DEM): physical
invariants and the bookkeeping of the contact and neighbour lists."""
import numpy as np

from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc


def _pair(coeff_rest=0.9, rhos=1000.0, collision="softsphere"):
    prm, _ = config.single_sphere(my=32, dia_cells=8)
    prm.update(imove=1, collision_type=collision, rhos=rhos, rhof=1.0, coeff_rest=coeff_rest, initialize_zero=True)
    xc = np.array([[10.0, 16.5, 16.5], [20.0, 16.5, 16.5]])
    vel = np.array([[0.5, 0.0, 0.0], [-0.5, 0.0, 0.0]])
    parts = config.Particles(xc, vel)
    s = oc.OracleSolver(config.make_params(prm), parts.struct)
    s._parts = parts
    return s


def test_head_on_collision_restitution_and_symmetry():
    """Two heavy spheres meet head on: they rebound with the restitution
    coefficient (the fluid barely slows spheres 1000 times denser), the motion
    stays mirror-symmetric, and the contact pair appears in PN only while the
    spheres overlap."""
    s = _pair()
    in_contact = False
    for _ in range(30):
        s.step()
        _, _, _, xc, vel = s.get_particles()
        c = oc.get_contacts(s)
        gap = xc[1, 0] - xc[0, 0] - 8.0
        if c["pn"][0, 0] > 0:
            in_contact = True
            assert c["pn"][1, 0] == 2 and c["pn"][1, 1] == 1
        assert abs(vel[0, 0] + vel[1, 0]) <= 1e-12 * abs(vel[0, 0])
        assert abs((xc[0, 0] - 15.0) + (xc[1, 0] - 15.0)) < 1e-11
    assert in_contact
    assert gap > 0 and c["pn"][0, 0] == 0
    ratio = -vel[0, 0] / 0.5
    assert 0.88 < ratio < 0.92, ratio


def test_elastic_collision_keeps_speed():
    """COEFF_REST = 1: no damping, the rebound speed equals the approach speed
    up to the fluid's drag on the way (heavier spheres lose less)."""
    out = []
    for rhos in (1000.0, 3000.0):
        s = _pair(coeff_rest=1.0, rhos=rhos)
        for _ in range(30):
            s.step()
        out.append(-s.get_particles()[4][0, 0] / 0.5)
    assert 0.99 < out[0] < out[1] < 1.0, out


def test_no_collision_translation():
    """COLLISION_TYPE = 'none': velocities are kept and each step moves the
    centres by vel*dt (grid units: vel*dt/dx)."""
    s = _pair(collision="none")
    _, _, _, x0, v0 = s.get_particles()
    t = 0.0
    for _ in range(5):
        rep = s.step()
        t += rep["dt"]
    _, _, _, x1, v1 = s.get_particles()
    dx = s.info.dx
    assert np.array_equal(v0, v1)
    assert np.allclose(x1 - x0, v0 * t / dx, rtol=0, atol=1e-10)


def test_neighbour_lists_are_symmetric_and_hold_self():
    prm, xc, vel = config.moving_array(my=32, dia_cells=6, nbody=20, seed=5)
    parts = config.Particles(xc, vel)
    s = oc.OracleSolver(config.make_params(prm), parts.struct)
    s._parts = parts
    for _ in range(3):
        s.step()
    c = oc.get_contacts(s)["neighbours"]
    n = xc.shape[0]
    sets = [set(c[1:1 + c[0, l], l].tolist()) for l in range(n)]
    for l in range(n):
        assert l + 1 in sets[l]
        for p in sets[l]:
            assert l + 1 in sets[p - 1]
