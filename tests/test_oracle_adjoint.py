"""CPU oracle of the discrete adjoint step: gradients of the time-averaged
summed drag J = (1/K) sum_n e . sum_m (pres_m + visc_m) with respect to the
sphere centres and the imposed mean pressure gradient, checked against
central finite differences of the oracle's forward step (fixed spheres,
SET_MPG, fixed dt; AB2, and RK3 with the drag of each step's last stage)."""
import numpy as np
import pytest

from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc

E = np.array([1.0, 0.3, -0.2])


def _solver(prm, xc, mpg=None):
    p = dict(prm)
    if mpg is not None:
        p["mpg"] = tuple(mpg)
    parts = config.Particles(xc)
    s = oc.OracleSolver(config.make_params(p), parts.struct)
    s._parts = parts
    return s


def _start(prm, xc, warm):
    s = _solver(prm, xc)
    st = s.get_state()
    st["umean"] = np.array(prm["umean0"])
    s.set_state(st)
    for _ in range(warm):
        s.step()
    return s.get_state()


def _J(prm, xc, st, K, mpg=None):
    s = _solver(prm, xc, mpg)
    st = dict(st)
    if mpg is not None:
        st["mpg"] = np.asarray(mpg, dtype=np.float64)
    s.set_state(st)
    J = 0.0
    for _ in range(K):
        r = s.step()
        J += float(np.dot(E, np.asarray(r["visc_total"]) - np.asarray(r["pres_total"])))
    return J / K


@pytest.mark.parametrize("scheme,limiter,K,rk3,frfl", [("upwind", "none", 4, False, False), ("center", "none", 3, False, False),
                                                      ("upwind", "minmod", 3, False, False), ("upwind", "none", 3, True, False),
                                                      ("upwind", "none", 3, False, True)])
def test_adjoint_matches_central_differences(scheme, limiter, K, rk3, frfl):
    prm, xc = config.adjoint_case(my=16, dia_cells=6.0, nbody=2, seed=5)
    prm.update(discr_scheme=scheme, limiter=limiter, rk3=rk3, include_frmeanfluid=frfl)
    st = _start(prm, xc, warm=6)
    s = _solver(prm, xc)
    s.set_state(st)
    out = s.adjoint(K, E)
    assert abs(out["J"] - _J(prm, xc, st, K)) <= 1e-13 * abs(out["J"])
    h = 1e-5
    for m, d in [(0, 0), (0, 1), (1, 2)]:
        xp, xm = xc.copy(), xc.copy()
        xp[m, d] += h
        xm[m, d] -= h
        fd = (_J(prm, xp, st, K) - _J(prm, xm, st, K)) / (2 * h)
        assert abs(out["g_xc"][m, d] - fd) <= 1e-6 * abs(fd), (m, d, out["g_xc"][m, d], fd)
    mpg0 = np.asarray(prm["mpg"], dtype=np.float64)
    for d in range(3):
        mp, mm = mpg0.copy(), mpg0.copy()
        mp[d] += 1e-6
        mm[d] -= 1e-6
        fd = (_J(prm, xc, st, K, mp) - _J(prm, xc, st, K, mm)) / 2e-6
        assert abs(out["g_mpg"][d] - fd) <= 1e-6 * max(abs(fd), 1e-3), (d, out["g_mpg"][d], fd)


def test_adjoint_initial_state_directional_derivative():
    """<lambda_u0, du> + <lambda_p0, dp> + <lambda_nl0, dnl> equals the
    directional derivative of J along a random state perturbation."""
    prm, xc = config.adjoint_case(my=16, dia_cells=6.0, nbody=2, seed=5)
    st = _start(prm, xc, warm=5)
    s = _solver(prm, xc)
    s.set_state(st)
    K = 3
    out = s.adjoint(K, E, state_grad=True)
    rng = np.random.default_rng(7)
    du = {k: (rng.standard_normal(st[k].shape) + 1j * rng.standard_normal(st[k].shape)) * 1e-3 for k in ("u", "nl", "p")}
    du["u"][..., -1] = du["u"][..., 0]      # image plane nx+1 = plane 1
    du["nl"][..., -1] = du["nl"][..., 0]
    pred = sum(np.sum((out[lk][..., :st["p"].shape[-1]].conj() * du[k][..., :st["p"].shape[-1]]).real)
               for lk, k in (("lu", "u"), ("lp", "p"), ("lnl", "nl")))
    eps = 1e-4
    def shifted(sg):
        s2 = dict(st)
        for k in ("u", "nl", "p"):
            s2[k] = st[k] + sg * eps * du[k]
        return _J(prm, xc, s2, K)
    fd = (shifted(1) - shifted(-1)) / (2 * eps)
    assert abs(pred - fd) <= 1e-6 * abs(fd), (pred, fd)
