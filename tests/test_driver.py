"""The driver loop's per-step records: Fortran edit descriptors and the
columns of _norm_drag.dat, _drag_components.dat, _dt_history.dat."""
import os

import numpy as np

from pureibm_ps2d_fd1d_b200 import config, driver
import oracle_ctypes as oc


def test_fortran_e_and_g():
    assert driver.fortran_e(1.5) == "  0.150000000000E+01"
    assert driver.fortran_e(-2.5e-7) == " -0.250000000000E-06"
    assert driver.fortran_e(9.9999999999996) == "  0.100000000000E+02"
    assert driver.fortran_e(0.0) == "  0.000000000000E+00"
    assert driver.fortran_g(1.0) == "    1.0000000    "
    assert driver.fortran_g(0.5) == "   0.50000000    "
    assert driver.fortran_g(123.456) == "    123.45600    "
    assert driver.fortran_g(0.05).strip() == "0.50000000E-01"
    assert len(driver.fortran_g(3.0e9)) == 17 and driver.fortran_g(3.0e9).strip() == "0.30000000E+10"


def test_records_of_a_short_run(tmp_path):
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    parts = config.Particles(xc)
    s = oc.OracleSolver(config.make_params(prm), parts.struct)
    s._parts = parts
    run = driver.Run(config.make_params(prm), run_name="RUN", directory=str(tmp_path), tend=1.0, solver=s)
    rep = run.advance(3)
    nd = np.loadtxt(os.path.join(str(tmp_path), "RUN_norm_drag.dat"), converters=None)
    assert nd.shape == (3, 11)
    assert abs(nd[-1, 3] - rep["norm_drag"]) <= 1e-11 * abs(rep["norm_drag"])
    assert abs(nd[-1, 1] - rep["t"] / run.t_vis) <= 1e-11 * abs(nd[-1, 1])
    dc = np.loadtxt(os.path.join(str(tmp_path), "RUN_drag_components.dat"))
    assert dc.shape == (3, 6) and abs(dc[-1, 2] - rep["total_drag"]) <= 1e-11 * abs(rep["total_drag"])
    lines = open(os.path.join(str(tmp_path), "RUN_dt_history.dat")).read().splitlines()
    assert lines[0].split() == ["ISTEP", "DT", "#STEPS", "REQD", "CFL"]
    last = [float(v) for v in lines[-1].split()]
    assert last[0] == 3.0 and abs(last[1] - rep["dt"]) <= 1e-7 * rep["dt"]
