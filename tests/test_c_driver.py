"""The C host driver (pureibm_ps2d_fd1d_b200/csrc/pibm_main.c) in its
library-free modes, against the Python reader and record writer:

* namelist files parse to the same pibm_params in C and in Python
  (config.read_floparam + config.make_params), and both refuse unknown
  variables, groups out of read_nmls's order and unsupported COLLISION_TYPEs;
* the C Ew.d / Gw.d editing equals driver.fortran_e / fortran_g on many
  values (the records are compared byte for byte on the GPU).
"""
import os
import subprocess

import numpy as np
import pytest

from pureibm_ps2d_fd1d_b200 import build, config, driver

FLOPARAM = """ &FLOANDGRID
 MY = 32, TEND = 5.0,
 VIS = 0.012, RE = 20.0 ,
 CFL = 0.1d0, CFL_MAX = 0.5D0, RAMP_FRAC_STEPS = 0,
 FLO_ANG = 0.d0, 90.d0, 90.d0
 /
 &PART_PROPT
 NBODY = 3, LYBYD = 4.0, DBYDX = 8.0, DIA_PHYS = 1.D0,
 INPUT_TYPE = 'default', DISCR_SCHEME = 'upwind',   ! the x-flux scheme
 COLLISION_TYPE = 'softsphere'
 /
 &FLAGS
 IMOVE = 0, ISCALON = 0, ADAPTIVE = T, RK3 = F,
 DORPR = T, DOBND = F, INCLUDE_FRMEANFLUID = F, SET_UMEAN = F, INITIALIZE_ZERO = T
 /
 &FILES
 SAVEITNS = 10
 /
 &PSD
 PSD_TYPE = 'discrete'
 /
 &GCG
 COEFF_REST = 0.9
 /
 &POSTLIST
 NBINS = 50
 /
"""


@pytest.fixture(scope="module")
def main_exe():
    if not os.path.exists(build.LIB):
        pytest.skip("libpibm.so is not built")
    return build.build_main()


def _c_params(exe, path):
    out = subprocess.run([exe, "--print-params", path], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return {k: v for k, v in (line.split() for line in out.stdout.splitlines())}


def _py_params(path):
    p = config.make_params(config.read_floparam(path))
    d = {}
    for name, _ in p._fields_:
        if name == "reserved":
            continue
        v = getattr(p, name)
        if name in ("flo_ang", "mpg"):
            for k in range(3):
                d[f"{name}{k}"] = v[k]
        else:
            d[name] = v
    return d


def _same(c, py):
    for k, v in py.items():
        cv = c[k]
        if isinstance(v, float):
            assert float(cv) == v, (k, cv, v)
        else:
            assert int(cv) == int(v), (k, cv, v)


def test_namelist_parse_matches_python(main_exe, tmp_path):
    variants = [
        FLOPARAM,
        FLOPARAM.replace("RK3 = F", "RK3 = .TRUE.").replace("FLO_ANG = 0.d0, 90.d0, 90.d0", "FLO_ANG(2) = 45.0"),
        FLOPARAM.replace("MY = 32,", "MY = 64, MPG = 2*-1.5d-3,").replace("DOBND = F", "DOBND = T"),
        FLOPARAM.replace("ISCALON = 0", "ISCALON = 1").replace(" &POSTLIST",
                         " &SCAL_PROPT\n PR_OR_SC_NU = 0.7D0, PHISURF = 1.0, PHISTREAM = 0.0\n /\n &POSTLIST"),
        FLOPARAM.replace("&GCG", "&MAT\n HHAT = 2.0\n /\n &GCG"),          # a group nobody reads is skipped
    ]
    for i, text in enumerate(variants):
        path = tmp_path / f"v{i}_floparam.in"
        path.write_text(text)
        py = _py_params(str(path))
        _same(_c_params(main_exe, str(path)), py)
    # the values the variants set
    p = config.make_params(config.read_floparam(str(tmp_path / "v1_floparam.in")))
    assert p.rk3 == 1 and tuple(p.flo_ang) == (0.0, 45.0, 90.0)
    p = config.make_params(config.read_floparam(str(tmp_path / "v2_floparam.in")))
    assert p.dobnd == 1 and tuple(p.mpg) == (-1.5e-3, -1.5e-3, 0.0)


def test_bad_inputs_are_refused(main_exe, tmp_path):
    bad = {
        "unknown": FLOPARAM.replace("MY = 32,", "MY = 32, NOSUCHKEY = 1,"),
        "order": FLOPARAM.replace(" &FLAGS", " &XX").replace(" &FLOANDGRID", " &FLAGS\n IMOVE = 0\n /\n &FLOANDGRID"),
        "collision": FLOPARAM.replace("'softsphere'", "'hardball'"),
        "missing": FLOPARAM.split(" &POSTLIST")[0],
    }
    for name, text in bad.items():
        path = tmp_path / f"{name}_floparam.in"
        path.write_text(text)
        r = subprocess.run([main_exe, "--print-params", str(path)], capture_output=True, text=True)
        assert r.returncode != 0, name
        with pytest.raises(ValueError):
            config.make_params(config.read_floparam(str(path)))


def test_edit_descriptors_match_python(main_exe):
    rng = np.random.default_rng(5)
    vals = list(rng.standard_normal(200) * 10.0 ** rng.integers(-12, 12, 200))
    vals += [0.0, -0.0, 1.0, 0.1, 0.09999999999, 99999999.5, 1e8, 12345678.9, 1e-120, -3.3e150, 0.5, 9.99999995]
    args = [repr(float(v)) for v in vals]
    out = subprocess.run([main_exe, "--format", *args], capture_output=True, text=True, check=True).stdout.splitlines()
    assert len(out) == len(vals)
    for v, line in zip(vals, out):
        e, g, _ = line.split("|")
        assert e == driver.fortran_e(float(v)), (v, e, driver.fortran_e(float(v)))
        assert g == driver.fortran_g(float(v)), (v, g, driver.fortran_g(float(v)))
