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


@pytest.mark.gpu
def test_moving_run_resumes_on_engine_and_oracle(tmp_path):
    """IMOVE = 1: the engine writes the moved particles and its frame motion
    (frame_vel, frame_pos), and the engine and the oracle resumed from those
    files track each other within the parity bar: positions and frame motion
    to 1e-12, the flow to 1e-10, identical contact lists."""
    prm, xc, vel = config.moving_array(my=64, dia_cells=8.0, nbody=60, seed=9, vel_spread=1.5)
    a = pk.Solver(config.make_params(prm), xc, vel)
    for _ in range(8):
        a.step()
    restart.write_restart(a, str(tmp_path), "MOV")
    fv, fp = a.get_frame()
    assert np.any(fv != 0.0)
    data = restart.read_restart(str(tmp_path), "MOV", a.nx, a.my, a.mz, imove=True)
    assert np.array_equal(data["frame_vel"], fv) and np.array_equal(data["frame_pos"], fp)
    gpu = restart.resume(prm, str(tmp_path), "MOV")
    assert all(np.array_equal(x, y) for x, y in zip(gpu.get_frame(), (fv, fp)))

    def oracle(P, x, v):
        parts = config.Particles(x, v)
        s = oc.OracleSolver(P, parts.struct)
        s._parts = parts
        return s

    cpu = restart.resume(prm, str(tmp_path), "MOV", solver_cls=oracle)
    for _ in range(8):
        gpu.step()
        cpu.step()
    xg, xo = gpu.get_particles()[3], cpu.get_particles()[3]
    assert np.abs(xg - xo).max() <= 1e-12 * np.abs(xo).max()
    for g, o in zip(gpu.get_frame(), cpu.get_frame()):
        assert np.abs(g - o).max() <= 1e-12 * max(np.abs(o).max(), 1.0)
    cg, cc = gpu.get_contacts(), oc.get_contacts(cpu)
    for k in ("neighbours", "pn", "pv"):
        assert np.array_equal(cg[k], cc[k]), k
    sg, so = gpu.get_state(), cpu.get_state()
    for k in ("u", "p"):
        d = np.abs(sg[k] - so[k]).max() / np.abs(so[k]).max()
        assert d <= 1e-10, (k, d)

