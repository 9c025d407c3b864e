"""Batched realizations (pibm_batch_*) against the same realizations run alone.

Every member's kernels are the ones a single run launches, in the same order,
so a member's state after a batch run is bitwise equal to the same realization
stepped on its own."""
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
