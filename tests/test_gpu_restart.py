"""The engine's restart in the reference's file format: a run resumed from
the files it wrote continues bitwise like the run that did not stop, the
engine reads the oracle's files (and the other way round), with the passive
scalar."""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config, restart
import oracle_ctypes as oc


def _case():
    prm, xc = config.random_array(my=32, dia_cells=8, nbody=3, seed=5, mc_moves=20)
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=0.0, phistream=1.0, initialize_zero=False)
    return prm, xc


@pytest.mark.gpu
def test_engine_resume_is_bitwise(tmp_path):
    prm, xc = _case()
    a = pk.Solver(config.make_params(prm), xc)
    a.run(5)
    restart.write_restart(a, str(tmp_path), "RUN")
    b = restart.resume(prm, str(tmp_path), "RUN")
    a.run(4)
    b.run(4)
    sa, sb = a.get_state(), b.get_state()
    for k in ("u", "nl", "p"):
        assert np.array_equal(sa[k], sb[k]), k
    assert np.array_equal(a.get_scalar()["phif"], b.get_scalar()["phif"])


@pytest.mark.gpu
def test_engine_resumes_oracle_files(tmp_path):
    """Files written from the oracle's state resume on the engine, which
    then tracks the oracle within the parity bar."""
    prm, xc = _case()
    parts = config.Particles(xc)
    cpu = oc.OracleSolver(config.make_params(prm), parts.struct)
    cpu._parts = parts
    for _ in range(5):
        cpu.step()
    restart.write_restart(cpu, str(tmp_path), "RUN")
    gpu = restart.resume(prm, str(tmp_path), "RUN")
    for _ in range(5):
        gpu.step()
        cpu.step()
    sg, sc = gpu.get_state(), cpu.get_state()
    for k in ("u", "p"):
        d = np.abs(sg[k] - sc[k]).max() / np.abs(sc[k]).max()
        assert d <= 1e-10, (k, d)
    d = np.abs(gpu.get_scalar()["phif"] - cpu.get_scalar()["phif"]).max()
    assert d <= 1e-10
