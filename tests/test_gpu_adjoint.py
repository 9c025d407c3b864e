"""Discrete adjoint on the CUDA engine (pibm_adjoint_run): gradients of the
time-averaged summed drag J = (1/K) sum_n e . sum_m (pres_m + visc_m) with
respect to the sphere centres and the imposed mean pressure gradient.

Checked against the CPU oracle's adjoint on the same state (1e-8 relative:
the two differ only in summation order), against central finite differences
of the engine's own forward run (1e-6 relative, step 1e-6 diameters), and for
independence of the checkpoint interval."""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc

pytestmark = pytest.mark.gpu

E = np.array([1.0, 0.3, -0.2])


def _case(scheme="upwind", my=32, nbody=3, limiter="none", rk3=False, frfl=False):
    prm, xc = config.adjoint_case(my=my, dia_cells=8.0, nbody=nbody, seed=11, mc_moves=20)
    prm.update(discr_scheme=scheme, limiter=limiter, rk3=rk3, include_frmeanfluid=frfl)
    return prm, xc


def _start_state(prm, xc, warm):
    """The oracle's state after `warm` steps from a uniform mean flow."""
    parts = config.Particles(xc)
    s = oc.OracleSolver(config.make_params(prm), parts.struct)
    st = s.get_state()
    st["umean"] = np.array(prm["umean0"])
    s.set_state(st)
    for _ in range(warm):
        s.step()
    return s.get_state()


def _gpu(prm, xc, st, mpg=None):
    p = dict(prm)
    if mpg is not None:
        p["mpg"] = tuple(mpg)
    s = pk.Solver(config.make_params(p), xc)
    st = dict(st)
    if mpg is not None:
        st["mpg"] = np.asarray(mpg, dtype=np.float64)
    s.set_state(st)
    return s


def _gpu_J(prm, xc, st, K, mpg=None):
    s = _gpu(prm, xc, st, mpg)
    J = 0.0
    for _ in range(K):
        r = s.step(1)
        J += float(np.dot(E, np.asarray(r["visc_total"]) - np.asarray(r["pres_total"])))
    s.close()
    return J / K


@pytest.mark.parametrize("scheme,limiter,rk3,frfl", [("upwind", "none", False, False), ("center", "none", False, False),
                                                     ("upwind", "minmod", False, False), ("upwind", "none", True, False),
                                                     ("upwind", "none", False, True)])
def test_adjoint_matches_oracle_adjoint(scheme, limiter, rk3, frfl):
    prm, xc = _case(scheme, limiter=limiter, rk3=rk3, frfl=frfl)
    st = _start_state(prm, xc, warm=10)
    K = 6
    parts = config.Particles(xc)
    cpu = oc.OracleSolver(config.make_params(prm), parts.struct)
    cpu.set_state(st)
    ref = cpu.adjoint(K, E)
    gpu = _gpu(prm, xc, st)
    out = gpu.adjoint(K, E, checkpoint_every=4)
    assert abs(out["J"] - ref["J"]) <= 1e-10 * abs(ref["J"])
    scale = np.max(np.abs(ref["g_xc"]))
    assert np.max(np.abs(out["g_xc"] - ref["g_xc"])) <= 1e-8 * scale, (out["g_xc"], ref["g_xc"])
    assert np.max(np.abs(out["g_mpg"] - ref["g_mpg"])) <= 1e-8 * np.max(np.abs(ref["g_mpg"]))
    # the handle ends at the state after K steps, like the oracle
    sg, sc = gpu.get_state(), cpu.get_state()
    assert np.max(np.abs(sg["u"] - sc["u"])) <= 1e-10 * np.max(np.abs(sc["u"]))


def test_adjoint_matches_central_differences():
    prm, xc = _case("upwind")
    st = _start_state(prm, xc, warm=10)
    K = 8
    out = _gpu(prm, xc, st).adjoint(K, E, checkpoint_every=3)
    h = 1e-6 * 8.0
    for m, d in [(0, 0), (1, 1), (2, 2)]:
        xp, xm = xc.copy(), xc.copy()
        xp[m, d] += h
        xm[m, d] -= h
        fd = (_gpu_J(prm, xp, st, K) - _gpu_J(prm, xm, st, K)) / (2 * h)
        assert abs(out["g_xc"][m, d] - fd) <= 1e-6 * abs(fd) + 1e-9, (m, d, out["g_xc"][m, d], fd)
    mpg0 = np.asarray(prm["mpg"], dtype=np.float64)
    for d in range(3):
        mp, mm = mpg0.copy(), mpg0.copy()
        mp[d] += 1e-6
        mm[d] -= 1e-6
        fd = (_gpu_J(prm, xc, st, K, mp) - _gpu_J(prm, xc, st, K, mm)) / 2e-6
        assert abs(out["g_mpg"][d] - fd) <= 1e-6 * abs(fd) + 1e-9, (d, out["g_mpg"][d], fd)


@pytest.mark.parametrize("rk3", [False, True])
def test_adjoint_independent_of_checkpoint_interval(rk3):
    prm, xc = _case("upwind", rk3=rk3)
    st = _start_state(prm, xc, warm=4)
    K = 7
    outs = [_gpu(prm, xc, st).adjoint(K, E, checkpoint_every=ck) for ck in (1, 3, 7, 20, 0)]   # 0: from free memory
    for o in outs[1:]:
        assert o["J"] == outs[0]["J"]
        assert np.max(np.abs(o["g_xc"] - outs[0]["g_xc"])) <= 1e-12 * np.max(np.abs(outs[0]["g_xc"]))
        assert np.max(np.abs(o["g_mpg"] - outs[0]["g_mpg"])) <= 1e-12 * np.max(np.abs(outs[0]["g_mpg"]))


def test_adjoint_rejects_unsupported_runs():
    prm, xc = config.single_sphere(my=32, dia_cells=8)   # adaptive dt, mpg from ufmean_des
    s = pk.Solver(config.make_params(prm), xc)
    with pytest.raises(pk.PibmError):
        s.adjoint(2, E)


def test_torch_autograd_function_returns_the_adjoint_gradients():
    import torch
    from pureibm_ps2d_fd1d_b200.adjoint import drag_objective
    prm, xc = _case("upwind")
    st = _start_state(prm, xc, warm=4)
    K = 5
    ref = _gpu(prm, xc, st).adjoint(K, E, checkpoint_every=2)
    x = torch.tensor(xc, dtype=torch.float64, requires_grad=True)
    g = torch.tensor(prm["mpg"], dtype=torch.float64, requires_grad=True)
    J = drag_objective(x, g, prm, st, K, E, checkpoint_every=2)
    (2.0 * J).backward()
    assert abs(J.item() - ref["J"]) <= 1e-12 * abs(ref["J"])
    assert np.max(np.abs(x.grad.numpy() - 2.0 * ref["g_xc"])) <= 1e-12 * np.max(np.abs(ref["g_xc"]))
    assert np.max(np.abs(g.grad.numpy() - 2.0 * ref["g_mpg"])) <= 1e-12 * np.max(np.abs(ref["g_mpg"]))
    with torch.no_grad():
        J0 = drag_objective(x, g, prm, st, K, E)
    assert abs(J0.item() - ref["J"]) <= 1e-12 * abs(ref["J"])


@pytest.mark.parametrize("rk3", [False, True])
def test_host_driven_reverse_sweep_equals_adjoint_run(rk3):
    """pibm_adjoint_begin / _step / _end with the host's own copies of every
    state reproduce pibm_adjoint_run."""
    prm, xc = _case("upwind", rk3=rk3)
    st0 = _start_state(prm, xc, warm=4)
    K = 5
    ref = _gpu(prm, xc, st0).adjoint(K, E, checkpoint_every=2)
    s = _gpu(prm, xc, st0)
    states = []
    for _ in range(K):
        states.append(s.get_state())
        for rks in range(1, (3 if rk3 else 1) + 1):
            s.step(rks)
    s.adjoint_begin(K, E)
    for n in range(K - 1, -1, -1):
        s.set_state(states[n])
        s.adjoint_step()
    out = s.adjoint_end()
    assert np.max(np.abs(out["g_xc"] - ref["g_xc"])) <= 1e-12 * np.max(np.abs(ref["g_xc"]))
    assert np.max(np.abs(out["g_mpg"] - ref["g_mpg"])) <= 1e-12 * np.max(np.abs(ref["g_mpg"]))
    with pytest.raises(pk.PibmError):
        s.adjoint_step()   # every step was reversed


def test_adjoint_matches_oracle_at_64():
    prm, xc = config.adjoint_case(my=64, dia_cells=12.0, nbody=4, seed=2, mc_moves=20)
    parts = config.Particles(xc)
    cpu = oc.OracleSolver(config.make_params(prm), parts.struct)
    st = cpu.get_state()
    st["umean"] = np.array(prm["umean0"])
    cpu.set_state(st)
    for _ in range(3):
        cpu.step()
    st = cpu.get_state()
    K = 3
    ref = cpu.adjoint(K, E)
    out = _gpu(prm, xc, st).adjoint(K, E, checkpoint_every=2)
    assert abs(out["J"] - ref["J"]) <= 1e-10 * abs(ref["J"])
    assert np.max(np.abs(out["g_xc"] - ref["g_xc"])) <= 1e-8 * np.max(np.abs(ref["g_xc"]))
    assert np.max(np.abs(out["g_mpg"] - ref["g_mpg"])) <= 1e-8 * np.max(np.abs(ref["g_mpg"]))


def test_adjoint_matches_oracle_on_the_gradient_configuration():
    """The benchmarked gradient geometry (96^3, 30 spheres of d = 16, SET_MPG,
    fixed dt): engine adjoint = oracle adjoint over 2 steps."""
    prm, xc = config.adjoint_case()
    parts = config.Particles(xc)
    cpu = oc.OracleSolver(config.make_params(prm), parts.struct)
    st = cpu.get_state()
    st["umean"] = np.array(prm["umean0"])
    cpu.set_state(st)
    for _ in range(2):
        cpu.step()
    st = cpu.get_state()
    K = 2
    ref = cpu.adjoint(K, E)
    out = _gpu(prm, xc, st).adjoint(K, E, checkpoint_every=1)
    assert abs(out["J"] - ref["J"]) <= 1e-10 * abs(ref["J"])
    assert np.max(np.abs(out["g_xc"] - ref["g_xc"])) <= 1e-8 * np.max(np.abs(ref["g_xc"]))
    assert np.max(np.abs(out["g_mpg"] - ref["g_mpg"])) <= 1e-8 * np.max(np.abs(ref["g_mpg"]))


def test_adjoint_matches_oracle_at_256():
    """256^3: the adjoint x-line solves run in 4-line tiles there."""
    prm, xc = config.adjoint_case(my=256, dia_cells=20.0, nbody=6, seed=3, mc_moves=20)
    parts = config.Particles(xc)
    cpu = oc.OracleSolver(config.make_params(prm), parts.struct)
    st = cpu.get_state()
    st["umean"] = np.array(prm["umean0"])
    cpu.set_state(st)
    cpu.step()
    st = cpu.get_state()
    ref = cpu.adjoint(1, E)
    out = _gpu(prm, xc, st).adjoint(1, E, checkpoint_every=1)
    assert abs(out["J"] - ref["J"]) <= 1e-10 * abs(ref["J"])
    assert np.max(np.abs(out["g_xc"] - ref["g_xc"])) <= 1e-8 * np.max(np.abs(ref["g_xc"]))
    assert np.max(np.abs(out["g_mpg"] - ref["g_mpg"])) <= 1e-8 * np.max(np.abs(ref["g_mpg"]))


@pytest.mark.parametrize("my,nbody", [(128, 12), (256, 20)])
def test_adjoint_runs_at_large_grids(my, nbody):
    """The adjoint's other size instantiations: J equals the forward run's
    drag average and the gradients are finite and non-zero."""
    prm, xc = config.adjoint_case(my=my, dia_cells=20.0, nbody=nbody, seed=9, mc_moves=0)
    s = pk.Solver(config.make_params(prm), xc)
    st = s.get_state()
    st["umean"] = np.array(prm["umean0"])
    s.set_state(st)
    s.run(3)
    st = s.get_state()
    K = 2
    out = s.adjoint(K, E, checkpoint_every=1)
    assert abs(out["J"] - _gpu_J(prm, xc, st, K)) <= 1e-12 * abs(out["J"])
    assert np.all(np.isfinite(out["g_xc"])) and np.all(np.isfinite(out["g_mpg"]))
    assert np.max(np.abs(out["g_xc"])) > 0 and np.max(np.abs(out["g_mpg"])) > 0
