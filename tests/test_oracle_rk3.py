"""CPU oracle of the RK3 time integration (RK3 = T: three stages per step
with coef(rks, 1:4) of initialize_flo.F90:861-877, dt updated at the last
stage)."""
import numpy as np

from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc


def _run(rk3, steps):
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    prm.update(rk3=rk3)
    parts = config.Particles(xc)
    s = oc.OracleSolver(config.make_params(prm), parts.struct)
    s._parts = parts
    for _ in range(steps):
        rep = s.step()
    return s, rep


def test_rk3_step_advances_time_by_dt_and_stays_solenoidal():
    """The stage weights coef(rks,1)+coef(rks,2) sum to 1, so a step advances
    t by dt like AB2; the velocity stays divergence free and the mean flow
    develops like the AB2 run's."""
    s3, r3 = _run(True, 30)
    s2, r2 = _run(False, 30)
    assert abs(r3["t"] - r2["t"]) < 1e-12 * r2["t"]
    assert r3["divmax"] < 1e-12
    assert abs(r3["umean"][0] - r2["umean"][0]) < 0.02 * abs(r2["umean"][0])
    assert np.isfinite(r3["norm_drag"]) and r3["norm_drag"] > 0


def test_rk3_stages_equal_full_steps():
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    prm.update(rk3=True)
    parts = config.Particles(xc)
    a = oc.OracleSolver(config.make_params(prm), parts.struct)
    b = oc.OracleSolver(config.make_params(prm), parts.struct)
    for _ in range(3):
        a.step()
        for rks in (1, 2, 3):
            b.step_rks(rks)
    assert np.array_equal(a.get_state()["u"], b.get_state()["u"])
