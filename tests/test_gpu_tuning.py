"""Autotuned x-line tile width (pibm_get_tuning / pibm_set_tuning): the
engine times 4 and 8 lines per CTA on the run's grid at creation, keeps the
faster, and the step's results do not depend on the choice.  Up to 128 the
4-line width is the persistent tensor-map kernel and the 8-line width the
staged one, so the comparison also checks that the two are bitwise equal."""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("my", [32, 64, 96, 128])
def test_tile_width_is_measured_and_does_not_change_results(my):
    prm, xc = config.random_array(my=my, dia_cells=8.0, phi=0.1, re=20.0, seed=3, mc_moves=10)
    a = pk.Solver(config.make_params(prm), xc)
    t = a.tuning()
    assert t["lines_per_cta"] in (4, 8)
    assert t["lines_ms"][4] > 0 and t["lines_ms"][8] > 0
    assert t["lines_ms"][t["lines_per_cta"]] == min(t["lines_ms"].values())   # the faster one is kept
    b = pk.Solver(config.make_params(prm), xc)
    a.set_tuning(4)
    b.set_tuning(8)
    a.run(5)
    b.run(5)
    sa, sb = a.get_state(), b.get_state()
    for k in ("u", "p", "nl"):
        assert np.array_equal(sa[k], sb[k]), k
    with pytest.raises(pk.PibmError):
        a.set_tuning(16)
