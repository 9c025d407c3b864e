"""Restart files in the reference's unformatted format (restart_funcs.F90):
record layout round trip, the 1/2 set alternation, and resuming a run from
the files (CPU oracle here; the engine in test_gpu_restart.py)."""
import os

import numpy as np

from pureibm_ps2d_fd1d_b200 import config, restart
import oracle_ctypes as oc


def _oracle(prm, xc, vel=None):
    parts = config.Particles(xc, vel)
    s = oc.OracleSolver(config.make_params(prm), parts.struct)
    s._parts = parts
    return s


def _scalar_case():
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=0.0, phistream=1.0, initialize_zero=False)
    return prm, xc


def test_record_round_trip_and_set_alternation(tmp_path):
    prm, xc = _scalar_case()
    s = _oracle(prm, xc)
    for _ in range(3):
        s.step()
    d = str(tmp_path)
    assert restart.write_restart(s, d, "RUN") == 1
    assert restart.write_restart(s, d, "RUN") == 2
    assert not os.path.exists(os.path.join(d, "RUN_u_1.rst"))          # the other set is deleted
    assert open(os.path.join(d, "RUN_RESTART")).read().split()[0] == "2"
    data = restart.read_restart(d, "RUN", s.nx, s.my, s.mz, iscalon=True)
    st, sc = s.get_state(), s.get_scalar()
    for k in ("u", "nl", "p"):
        assert np.array_equal(data[k], st[k])
    assert np.array_equal(data["phif"], sc["phif"]) and np.array_equal(data["nlphif"], sc["nlphif"])
    assert data["t"] == st["t"] and data["dt"] == st["dt"] and data["cf"] == st["cf"]
    assert np.array_equal(data["umean"], st["umean"]) and np.array_equal(data["mpg"], st["mpg"])
    assert data["heat_ratio"] == sc["heat_ratio"] and data["heat_ratio_old"] == sc["heat_ratio_old"]
    assert np.array_equal(data["xc"], np.asarray(xc, dtype=np.float64))
    # the u file's records: 4-byte markers around (t, dt) first
    raw = open(os.path.join(d, "RUN_u_2.rst"), "rb").read()
    assert int.from_bytes(raw[:4], "little") == 16 and int.from_bytes(raw[20:24], "little") == 16


def test_resume_continues_bitwise(tmp_path):
    """A run resumed from its restart files steps to the same fields as the
    run that went on without stopping."""
    prm, xc = _scalar_case()
    a = _oracle(prm, xc)
    for _ in range(4):
        a.step()
    restart.write_restart(a, str(tmp_path), "RUN")
    b = restart.resume(prm, str(tmp_path), "RUN", solver_cls=lambda P, x, v: _oracle(prm, x, v))
    for _ in range(3):
        a.step()
        b.step()
    sa, sb = a.get_state(), b.get_state()
    for k in ("u", "nl", "p"):
        assert np.array_equal(sa[k], sb[k]), k
    assert np.array_equal(a.get_scalar()["phif"], b.get_scalar()["phif"])


def test_resume_moving_particles(tmp_path):
    """IMOVE = 1: the moved particles come from RUN_sphere_config_N.rst and
    usmean_des / ufmean_des from the u file, as read_unformatted does."""
    prm, xc, vel = config.moving_array(my=32, dia_cells=6.0, nbody=30, seed=4, vel_spread=1.0)
    a = _oracle(prm, xc, vel)
    for _ in range(3):
        a.step()
    restart.write_restart(a, str(tmp_path), "MOV")
    assert os.path.exists(os.path.join(str(tmp_path), "MOV_sphere_config_1.rst"))
    # the frame motion of the run, not its initial values, is in the file
    fv, fp = a.get_frame()
    assert np.any(fv != 0.0) and np.any(fp != 1.0)
    data = restart.read_restart(str(tmp_path), "MOV", a.nx, a.my, a.mz, imove=True)
    assert np.array_equal(data["frame_vel"], fv) and np.array_equal(data["frame_pos"], fp)
    b = restart.resume(prm, str(tmp_path), "MOV", solver_cls=lambda P, x, v: _oracle(prm, x, v))
    fvb, fpb = b.get_frame()
    assert np.array_equal(fvb, fv) and np.array_equal(fpb, fp)
    for _ in range(3):
        a.step()
        b.step()
    # the restart stores centres in grid units (xc = pos/dx + 1) and the DEM
    # restarts from pos = (xc - 1)*dx, so positions agree to rounding only
    xa, xb = a.get_particles()[3], b.get_particles()[3]
    assert np.abs(xa - xb).max() <= 1e-12 * np.abs(xa).max()
    ua, ub = a.get_state()["u"], b.get_state()["u"]
    assert np.abs(ua - ub).max() <= 1e-10 * np.abs(ua).max()
    fa, fb = a.get_frame(), b.get_frame()
    for k in range(2):
        assert np.abs(fa[k] - fb[k]).max() <= 1e-12 * max(np.abs(fa[k]).max(), 1.0)
