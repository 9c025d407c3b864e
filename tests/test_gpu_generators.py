"""INPUT_TYPE = 'random' end to end on the GPU: a configuration generated
from the run's seed file (generators.py) steps on the engine within the
parity bar of the oracle."""
import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk
from pureibm_ps2d_fd1d_b200 import config
import oracle_ctypes as oc
from test_generators import _write_random_run

pytestmark = pytest.mark.gpu


def test_random_input_runs_on_engine(tmp_path):
    d = str(tmp_path)
    _write_random_run(d)
    prm, xc = config.load_run(d, "RUN")
    P = config.make_params(prm)
    parts = config.Particles(xc)
    gpu = pk.Solver(P, xc)
    cpu = oc.OracleSolver(P, parts.struct)
    cpu._parts = parts
    for _ in range(5):
        gpu.step()
        cpu.step()
    sg, sc = gpu.get_state(), cpu.get_state()
    for k in ("u", "p"):
        assert np.abs(sg[k] - sc[k]).max() <= 1e-10 * np.abs(sc[k]).max(), k
