"""RK3 time integration (RK3 = T) on the CUDA engine against the CPU oracle:
stage by stage through pibm_step(rks) and full steps replayed from the step
graphs (three stages each).  Parity bar as for AB2: 1e-10 relative."""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc

TOL = 1e-10


def rel(a, b):
    d = np.max(np.abs(np.asarray(a) - np.asarray(b)))
    s = np.max(np.abs(np.asarray(b)))
    return d / s if s > 0 else d


def make_pair(prm, xc, vel=None):
    P = config.make_params(prm)
    parts = config.Particles(xc, vel)
    gpu = pk.Solver(P, xc, vel)
    cpu = oc.OracleSolver(P, parts.struct)
    cpu._parts = parts
    return gpu, cpu


def compare(gpu, cpu):
    sg, sc = gpu.get_state(), cpu.get_state()
    out = {k: rel(sg[k], sc[k]) for k in ("u", "p", "nl")}
    pg, vg, fg, _, _ = gpu.get_particles()
    pc, vc, fc, _, _ = cpu.get_particles()
    out["pres"], out["visc"], out["force"] = rel(pg, pc), rel(vg, vc), rel(fg, fc)
    assert abs(sg["t"] - sc["t"]) <= TOL * abs(sc["t"])
    bad = {k: v for k, v in out.items() if not v <= TOL}
    assert not bad, out
    return out


@pytest.mark.gpu
def test_rk3_single_sphere_stage_by_stage():
    prm, xc = config.single_sphere(my=32, dia_cells=8)
    prm.update(rk3=True)
    gpu, cpu = make_pair(prm, xc)
    for _ in range(8):
        for rks in (1, 2, 3):
            rg, rc = gpu.step(rks), cpu.step_rks(rks)
            assert abs(rg["dt"] - rc["dt"]) <= 1e-15 * rc["dt"]
        compare(gpu, cpu)
    with pytest.raises(RuntimeError):
        gpu.step(2)   # stages run in order


@pytest.mark.gpu
def test_rk3_array_with_scalar_graph_replay():
    """10-sphere array at 64^3 with the passive scalar: pibm_run replays
    three stages per step from the graphs."""
    prm, xc = config.random_array(my=64, dia_cells=12, nbody=10, seed=7, mc_moves=100)
    prm.update(rk3=True, iscalon=1, pr_or_sc_nu=0.7, phisurf=0.0, phistream=1.0, initialize_zero=False)
    gpu, cpu = make_pair(prm, xc)
    gpu.run(6)
    for _ in range(6):
        cpu.step()
    compare(gpu, cpu)
    sg, sc = gpu.get_scalar(), oc.get_scalar(cpu)
    assert rel(sg["phif"], sc["phif"]) <= TOL
