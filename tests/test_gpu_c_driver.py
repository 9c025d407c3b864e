"""The C host driver (pibm_main, gcc against include/pibm.h, linked to
libpibm.so) on the GPU: its four record files equal, byte for byte, those of
the Python driver (driver.Run) run on the same floparam.in and
sphr_center.inp; and a run with the reference's default DOBND = T is refused
by the library with PIBM_ERR_ARG instead of running another algorithm."""
import os
import subprocess

import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import build, config, driver
from test_c_driver import FLOPARAM

pytestmark = pytest.mark.gpu

RECORDS = ("norm_drag", "norm_drag_chem", "drag_components", "dt_history")


def _write_case(d, floparam, xc_grid, dbydx):
    with open(os.path.join(d, "RUN_floparam.in"), "w") as fh:
        fh.write(floparam)
    config.write_sphr_center(os.path.join(d, "RUN_sphr_center.inp"), xc_grid, dbydx)


@pytest.mark.parametrize("variant", ["ab2", "rk3_center"])
def test_c_driver_records_equal_python_driver(tmp_path, variant):
    exe = build.build_main()
    text = FLOPARAM
    if variant == "rk3_center":
        text = text.replace("RK3 = F", "RK3 = T").replace("'upwind'", "'center'").replace(
            "FLO_ANG = 0.d0, 90.d0, 90.d0", "FLO_ANG = 0.d0, 60.d0, 90.d0")
    _, xc = config.random_array(my=32, dia_cells=8, nbody=3, seed=11, mc_moves=50)
    cdir, pdir = tmp_path / "c", tmp_path / "py"
    cdir.mkdir()
    pdir.mkdir()
    _write_case(str(cdir), text, xc, 8.0)
    _write_case(str(pdir), text, xc, 8.0)
    nsteps = 6
    r = subprocess.run([exe, "RUN", str(nsteps)], cwd=str(cdir), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    prm = config.read_floparam(str(pdir / "RUN_floparam.in"))
    xin = config.read_sphr_center(str(pdir / "RUN_sphr_center.inp"), prm["dbydx"])
    run = driver.Run(prm, xin, run_name="RUN", directory=str(pdir), tend=prm["tend"])
    run.advance(nsteps)
    for name in RECORDS:
        a = open(cdir / f"RUN_{name}.dat", "rb").read()
        b = open(pdir / f"RUN_{name}.dat", "rb").read()
        assert a == b, (name, a[:400], b[:400])
    rows = np.loadtxt(str(cdir / "RUN_norm_drag.dat"))
    assert rows.shape == (nsteps, 11) and np.all(np.isfinite(rows))


def test_dobnd_default_is_refused(tmp_path):
    exe = build.build_main()
    text = FLOPARAM.replace("DOBND = F, ", "")          # the reference's default DOBND = T
    _, xc = config.random_array(my=32, dia_cells=8, nbody=3, seed=11, mc_moves=50)
    _write_case(str(tmp_path), text, xc, 8.0)
    r = subprocess.run([exe, "RUN", "2"], cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
    assert r.returncode == 1 and "DOBND" in r.stderr, (r.returncode, r.stderr)
    prm = config.read_floparam(str(tmp_path / "RUN_floparam.in"))
    with pytest.raises(RuntimeError, match="DOBND"):
        pk.Solver(config.make_params(prm), xc)
