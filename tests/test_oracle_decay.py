"""Closed-form checks of the oracle step with no spheres: exact viscous
decay and advection (along x, y and z) of shear waves, the projection of a
random field, and the mean flow under a fixed mean pressure gradient.

With no spheres and the mean pressure gradient held at zero, a velocity
field with one component that does not vary along its own direction
(u_x(y, z), or u_y(x, z)) is an exact solution of the Navier-Stokes
equations: the conservative nonlinear term and the divergence vanish, the
pressure stays zero and each Fourier mode decays on its own.  The step's
Crank-Nicolson viscous solve (usteptime.F90:286-499, with coef(rks, 1:2)
from initialize_flo.F90:861-884) then multiplies the mode by

    g = (1 - c2 * nu * dt * lam) / (1 + c1 * nu * dt * lam)

per stage, lam = ky^2 + kz^2 + 4 sin^2(kx dx / 2) / dx^2 (spectral in y
and z, the three-point second difference in x).  These tests pin the
oracle's time integration, viscous line solves and projection against that
closed form, independently of the reference's outputs; the engine is held
to the oracle by the GPU parity tests.

With a uniform mean flow U along x (held by the zero mean pressure
gradient) the wave u_y = A sin(kx x) is also advected.  The conservative
nonlinear term is then linear, N = S a per mode, S = i U sin(kx dx) / dx
for the centred x flux and U (1 + i sin(kx dx) / 2)(1 - exp(-i kx dx)) / dx
(U > 0; mirrored for U < 0) for the upwind one without a limiter, and each
stage maps the mode amplitude a as

    a_k = ((1 - c2 nu dt lam) a_{k-1} - dt (c3 N(a_{k-1}) + c4 N(a_{k-2})))
          / (1 + c1 nu dt lam)

(coef(rks, 3:4) of the same table; the old nonlinear term of the first
stage is zero), which pins both flux forms, their sign and the AB2 / RK3
explicit coefficients.
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

MY = 32
LY = 4.0              # lybyd = 4 with d = 1
DX = LY / MY
NU = 0.05
AMP = 0.01
AB2_STAGES = [(0.5, 0.5)]
RK3_STAGES = [(4.0 / 15.0, 4.0 / 15.0), (1.0 / 15.0, 1.0 / 15.0), (1.0 / 6.0, 1.0 / 6.0)]


def _solver(scheme, rk3):
    prm = config.default_params()
    prm.update(my=MY, lybyd=LY, dbydx=MY / LY, re=1.0, vis=NU, cfl=0.2, cfl_max=0.5, discr_scheme=scheme,
               initialize_zero=True, dobnd=False, ramp_frac_steps=0, set_mpg=True, mpg=(0.0, 0.0, 0.0), rk3=rk3)
    parts = config.Particles(np.zeros((0, 3)))
    s = oc.OracleSolver(config.make_params(prm), parts.struct)
    s._parts = parts
    return s


def _wave(s, case):
    """Initial u (reference layout [comp][kz][ky][x]), the modes it occupies
    and their lam."""
    st = s.get_state()
    u = np.zeros_like(st["u"])
    x = np.arange(s.nx + 1) * DX                 # x_i = (i - 1) dx, i = 1..nx+1 (periodic image)
    if case == "ux_of_y":                        # u_x = A sin(2 pi 2 y / Ly): the (ky = 2, kz = 0) line
        m = 2
        u[0, 0, m, :] = -0.5j * AMP
        modes = [(0, 0, m)]
        lam = (2 * np.pi * m / LY) ** 2
    elif case == "ux_of_yz":                     # u_x = A sin(ky y + kz z), ky = 1, kz = 3 (ky > 0: the
                                                 # conjugate mode is implicit in the half spectrum)
        m, n = 1, 3
        u[0, n, m, :] = -0.5j * AMP
        modes = [(0, n, m)]
        lam = (2 * np.pi * m / LY) ** 2 + (2 * np.pi * n / LY) ** 2
    elif case == "uy_of_x":                      # u_y = A sin(kx x), kx = 3: the real (0, 0) line
        q = 3
        u[1, 0, 0, :] = AMP * np.sin(2 * np.pi * q * x / LY)
        modes = [(1, 0, 0)]
        lam = 4 * np.sin(np.pi * q / s.nx) ** 2 / DX ** 2
    elif case == "uy_of_xz":                     # u_y = A sin(kx x + kz z), kx = 5, kz = 2: a complex x line
        q, n = 5, 2
        e = -0.5j * AMP * np.exp(2j * np.pi * q * x / LY)
        u[1, n, 0, :] = e
        u[1, s.mz - n, 0, :] = np.conj(e)
        modes = [(1, n, 0), (1, s.mz - n, 0)]
        lam = 4 * np.sin(np.pi * q / s.nx) ** 2 / DX ** 2 + (2 * np.pi * n / LY) ** 2
    else:
        raise ValueError(case)
    st["u"] = u
    s.set_state(st)
    return modes, lam


@pytest.mark.parametrize("rk3", [False, True], ids=["ab2", "rk3"])
@pytest.mark.parametrize("scheme", ["upwind", "center"])
@pytest.mark.parametrize("case", ["ux_of_y", "ux_of_yz", "uy_of_x", "uy_of_xz"])
def test_shear_wave_decays_by_the_crank_nicolson_factor(case, scheme, rk3):
    s = _solver(scheme, rk3)
    try:
        modes, lam = _wave(s, case)
        prev = s.get_state()["u"]
        for _ in range(4):
            s.step()
            st = s.get_state()
            g = 1.0
            for c1, c2 in (RK3_STAGES if rk3 else AB2_STAGES):
                g *= (1 - c2 * NU * st["dt"] * lam) / (1 + c1 * NU * st["dt"] * lam)
            u = st["u"]
            for (c, k, j) in modes:
                line, line0 = u[c, k, j, :], prev[c, k, j, :]
                # relative to the line, with a floor at the initial amplitude's
                # rounding level for modes that decay by 10x per step
                tol = 1e-12 * np.abs(line0).max() + 1e-15 * AMP
                np.testing.assert_allclose(line, g * line0, rtol=0, atol=tol)
            rest = np.abs(u).copy()
            for (c, k, j) in modes:
                rest[c, k, j, :] = 0
            assert rest.max() <= 1e-14 * AMP
            assert np.abs(st["p"]).max() <= 1e-14 * AMP
            assert np.all(st["umean"] == 0)
            prev = u
    finally:
        s.close()


AB2_NL = [(1.5, -0.5)]
RK3_NL = [(8.0 / 15.0, 0.0), (5.0 / 12.0, -17.0 / 60.0), (3.0 / 4.0, -5.0 / 12.0)]


def _flux_symbol(scheme, U, theta):
    """Per-mode symbol of the x flux divergence of u_x * v for uniform u_x = U
    (form_nl, nl_allflow.F90:71-327): centred, F(i+1/2) - F(i-1/2) with
    F(i) = U v(i) over 2 dx; upwind without a limiter, the face states
    v(i) +- (v(i+1) - v(i-1)) / 4 with the Rusanov dissipation |U| / 2 times
    their jump, i.e. full upwinding of the centred-slope reconstruction."""
    if scheme == "center":
        return 1j * U * np.sin(theta) / DX
    if U > 0:
        return U * (1 + 0.5j * np.sin(theta)) * (1 - np.exp(-1j * theta)) / DX
    return U * (1 - 0.5j * np.sin(theta)) * (np.exp(1j * theta) - 1) / DX


@pytest.mark.parametrize("rk3", [False, True], ids=["ab2", "rk3"])
@pytest.mark.parametrize("scheme,U", [("center", 0.3), ("center", -0.3), ("upwind", 0.3), ("upwind", -0.3)])
def test_advected_wave_follows_the_flux_recurrence(scheme, U, rk3):
    s = _solver(scheme, rk3)
    try:
        q = 3
        kx = 2 * np.pi * q / LY
        st = s.get_state()
        u = np.zeros_like(st["u"])
        x = np.arange(s.nx + 1) * DX
        u[1, 0, 0, :] = AMP * np.sin(kx * x)
        st["u"] = u
        st["umean"] = np.array([U, 0.0, 0.0])
        s.set_state(st)
        lam = 4 * np.sin(kx * DX / 2) ** 2 / DX ** 2
        sym = _flux_symbol(scheme, U, kx * DX)
        phase = np.exp(1j * kx * x)

        def amp(line):                               # line = Re(a e^{i kx x}) up to rounding
            return 2 * np.sum(line[:-1] * np.conj(phase[:-1])) / s.nx

        a_old, a = 0.0, amp(s.get_state()["u"][1, 0, 0, :])
        for _ in range(4):
            for rks, ((c1, c2), (c3, c4)) in enumerate(zip(RK3_STAGES if rk3 else AB2_STAGES,
                                                           RK3_NL if rk3 else AB2_NL), start=1):
                if rk3:
                    s.step_rks(rks)
                else:
                    s.step()
                st = s.get_state()
                # the dt the stage used: RK3 computes the new dt at its last
                # stage and uses it there (the first step's stages 1-2 run at
                # the initial dt)
                dt = st["dt"]
                pred = ((1 - c2 * NU * dt * lam) * a - dt * (c3 * sym * a + c4 * sym * a_old)) / (1 + c1 * NU * dt * lam)
                line = st["u"][1, 0, 0, :]
                np.testing.assert_allclose(line, (pred * phase).real, rtol=0, atol=1e-14 * AMP)
                a_old, a = a, amp(line)
                rest = np.abs(st["u"]).copy()
                rest[1, 0, 0, :] = 0
                assert rest.max() <= 1e-14 * AMP
                assert np.abs(st["p"]).max() <= 1e-14 * AMP
                assert np.array_equal(st["umean"], [U, 0.0, 0.0])
    finally:
        s.close()


def _divergence(s, u):
    """The discrete divergence at the x faces i + 1/2 of every (ky, kz) line
    (check_divergence, poisson.F90:241-508): (u_x(i+1) - u_x(i)) / dx +
    i ky (u_y(i) + u_y(i+1)) / 2 + i kz (u_z(i) + u_z(i+1)) / 2."""
    ky = 2 * np.pi * np.arange(s.my2) / LY
    kz = 2 * np.pi * np.fft.fftfreq(s.mz, d=1.0 / s.mz) / LY
    wy, wz = 1j * ky[None, :, None], 1j * kz[:, None, None]
    ux, uy, uz = u[0], u[1], u[2]
    return ((ux[:, :, 1:] - ux[:, :, :-1]) / DX + 0.5 * wy * (uy[:, :, :-1] + uy[:, :, 1:])
            + 0.5 * wz * (uz[:, :, :-1] + uz[:, :, 1:]))


@pytest.mark.parametrize("rk3", [False, True], ids=["ab2", "rk3"])
@pytest.mark.parametrize("scheme", ["upwind", "center"])
def test_projection_removes_the_divergence_of_a_random_field(scheme, rk3):
    """A random, compressible initial field: after each step the discrete
    divergence, computed here from the returned state, is at rounding level
    (the pressure solve and divcorr project every line), and the step's
    reported divmax is that same quantity."""
    s = _solver(scheme, rk3)
    try:
        st = s.get_state()
        real = AMP * np.random.default_rng(3).standard_normal((3, s.nx, s.mz, s.my))
        u = np.zeros_like(st["u"])
        for c in range(3):
            u[c, :, :, :s.nx] = np.transpose(oc.ff2rc(real[c]), (1, 2, 0))   # x planes -> [kz][ky][x]
            u[c, :, :, s.nx] = u[c, :, :, 0]
        st["u"] = u
        s.set_state(st)
        d0 = np.abs(_divergence(s, u)).max()
        assert d0 > 1e-3
        for _ in range(3):
            rep = s.step()
            d = np.abs(_divergence(s, s.get_state()["u"])).max()
            assert d <= 1e-13 * d0
            assert rep["divmax"] == pytest.approx(d, rel=1e-12, abs=1e-30)
    finally:
        s.close()


@pytest.mark.parametrize("rk3", [False, True], ids=["ab2", "rk3"])
def test_fixed_mean_pressure_gradient_accelerates_the_mean_flow(rk3):
    """No spheres, fluid at rest, SET_MPG with mpg = (g, 0, 0): every stage
    adds -mpg * dt to the mean flow (steptheflow.F90:98, frmean = 0) and
    the fluctuation stays zero.  The reference applies that update in every
    velstep call with the full dt, so a three-stage RK3 step moves the mean
    by 3 g dt while t advances by dt; the restatement keeps it."""
    g = 0.02
    prm = config.default_params()
    prm.update(my=MY, lybyd=LY, dbydx=MY / LY, re=1.0, vis=NU, cfl=0.2, cfl_max=0.5, discr_scheme="upwind",
               initialize_zero=True, dobnd=False, ramp_frac_steps=0, set_mpg=True, mpg=(g, 0.0, 0.0), rk3=rk3)
    parts = config.Particles(np.zeros((0, 3)))
    s = oc.OracleSolver(config.make_params(prm), parts.struct)
    try:
        expect = 0.0
        for _ in range(4):
            for rks in range(1, 4 if rk3 else 2):
                if rk3:
                    s.step_rks(rks)
                else:
                    s.step()
                st = s.get_state()
                expect -= g * st["dt"]
                assert st["mpg"][0] == g
                assert np.abs(st["u"]).max() == 0.0 and np.abs(st["p"]).max() == 0.0
                assert st["umean"][0] == pytest.approx(expect, rel=1e-14)
                assert st["umean"][1] == 0.0 and st["umean"][2] == 0.0
        assert st["umean"][0] == pytest.approx(-g * st["t"] * (3 if rk3 else 1), rel=1e-13)
    finally:
        s.close()


@pytest.mark.parametrize("rk3", [False, True], ids=["ab2", "rk3"])
@pytest.mark.parametrize("direction", ["y", "z"])
def test_spectral_advection_of_a_shear_wave(direction, rk3):
    """Mean flow along y (u_z = A sin(ky y)) or z (u_x = A sin(kz z)): the
    nonlinear term is the spectral derivative of the product with the mean,
    S = i ky V (or i kz W) per mode (nonlinear, nl.F90:63-205), and the
    modes follow the same stage recurrence as the x-advected wave."""
    s = _solver("upwind", rk3)
    try:
        V, m = 0.25, 2
        st = s.get_state()
        u = np.zeros_like(st["u"])
        if direction == "y":
            st["umean"] = np.array([0.0, V, 0.0])
            u[2, 0, m, :] = -0.5j * AMP
            k = 2 * np.pi * m / LY
            modes = [((2, 0, m), 1j * k * V)]
        else:
            st["umean"] = np.array([0.0, 0.0, V])
            u[0, m, 0, :] = -0.5j * AMP
            u[0, s.mz - m, 0, :] = 0.5j * AMP
            k = 2 * np.pi * m / LY
            modes = [((0, m, 0), 1j * k * V), ((0, s.mz - m, 0), -1j * k * V)]
        st["u"] = u
        s.set_state(st)
        lam = k ** 2
        amp = {idx: (0.0, u[idx][0]) for idx, _ in modes}
        for _ in range(4):
            for rks, ((c1, c2), (c3, c4)) in enumerate(zip(RK3_STAGES if rk3 else AB2_STAGES,
                                                           RK3_NL if rk3 else AB2_NL), start=1):
                if rk3:
                    s.step_rks(rks)
                else:
                    s.step()
                st = s.get_state()
                dt = st["dt"]
                rest = np.abs(st["u"]).copy()
                for idx, sym in modes:
                    a_old, a = amp[idx]
                    pred = ((1 - c2 * NU * dt * lam) * a - dt * (c3 * sym * a + c4 * sym * a_old)) / (1 + c1 * NU * dt * lam)
                    line = st["u"][idx]
                    np.testing.assert_allclose(line, pred, rtol=0, atol=1e-14 * AMP)
                    amp[idx] = (a, line[0])
                    rest[idx] = 0
                assert rest.max() <= 1e-14 * AMP
                assert np.abs(st["p"]).max() <= 1e-14 * AMP
    finally:
        s.close()
