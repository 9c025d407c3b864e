"""Batched realizations (pibm_batch_*) against the same realizations run alone.

Every member's blocks run the device code of a single run's kernels, in the
same order, whether the member shares the launches of its grid-size group
(fixed spheres, no scalar) or steps as its own branch, so a member's state
after a batch run is bitwise equal to the same realization stepped on its own."""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config


def _members():
    return [(p, x) for p, x, _ in config.mis_ensemble(n=4, seed=5, grids=(32, 64), phi_range=(0.05, 0.2),
                                                       dia_range=(6, 10), re_range=(10.0, 50.0), mc_moves=50)]


@pytest.mark.gpu
def test_batch_members_match_single_runs_bitwise():
    members = _members()
    b = pk.Batch(members)
    b.run(3)
    b.members[1].step()        # members may also step on their own in between
    b.run(4)
    for q, (prm, xc) in enumerate(members):
        s = pk.Solver(prm, xc)
        s.run(3)
        if q == 1:
            s.step()
        s.run(4)
        want, got = s.get_state(), b.members[q].get_state()
        for k in ("u", "nl", "p"):
            np.testing.assert_array_equal(got[k], want[k])
        assert got["t"] == want["t"] and got["dt"] == want["dt"]
        s.close()
    b.close()


@pytest.mark.gpu
def test_batch_timing_advances_every_member():
    members = _members()
    b = pk.Batch(members)
    t_seq = b.time(2, sequential=True)
    t_bat = b.time(2, sequential=False)
    assert t_seq > 0 and t_bat > 0
    for q, (prm, xc) in enumerate(members):
        s = pk.Solver(prm, xc)
        s.run(4)
        np.testing.assert_array_equal(b.members[q].get_state()["u"], s.get_state()["u"])
        s.close()
    b.close()


def _mixed_members():
    """Groups of 32^3 and 64^3 realizations (upwind and centre schemes, a
    member without spheres), an RK3 pair, and a scalar member that steps as
    its own branch."""
    kw = dict(phi_range=(0.05, 0.2), dia_range=(6, 10), re_range=(10.0, 50.0), mc_moves=50)
    m32 = [(p, x) for p, x, _ in config.mis_ensemble(n=4, seed=11, grids=(32,), **kw)]
    m64 = [(p, x) for p, x, _ in config.mis_ensemble(n=2, seed=12, grids=(64,), **kw)]
    out = list(m32) + list(m64)
    p = dict(m32[1][0])
    p.update(discr_scheme="center")
    out[1] = (p, m32[1][1])
    out.append((dict(m32[0][0]), np.zeros((0, 3))))
    for q in (2, 3):
        p = dict(m32[q][0])
        p.update(rk3=True)
        out.append((p, m32[q][1]))
    p = dict(m32[0][0])
    p.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=1.0, phistream=0.0, initialize_zero=False)
    out.append((p, m32[0][1]))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("fused", [True, False])
def test_mixed_batch_matches_single_runs_bitwise(fused):
    members = _mixed_members()
    b = pk.Batch(members)
    if fused:
        b.run(3)
        b.members[4].step()     # a grouped member stepped alone flips its parity
        b.run(3)
    else:
        b.time(3, sequential=False, fused=False)
        b.members[4].step()
        b.time(3, sequential=False, fused=False)
    for q, (prm, xc) in enumerate(members):
        s = pk.Solver(prm, xc)
        s.run(3)
        if q == 4:
            s.step()
        s.run(3)
        want, got = s.get_state(), b.members[q].get_state()
        for k in ("u", "nl", "p"):
            np.testing.assert_array_equal(got[k], want[k], err_msg=f"member {q} {k}")
        assert got["t"] == want["t"] and got["dt"] == want["dt"]
        s.close()
    b.close()
