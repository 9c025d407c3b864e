"""pibm_ff2cr_noalloc: the allocation-free ff2cr on device buffers.

Callers that keep spectral planes on the GPU inside their own memory pool
cannot use pibm_ff2cr, which allocates and frees device buffers per call
(cudaFree waits for the whole device).  The allocation-free entry point keeps
its twiddle tables in a static device array written by the first call on each
device.  This file is named so that it is collected last: it must pass both
alone in a fresh process (where its first call does the set-up) and after
every other test has run.  Floating point: relative error <= 1e-13 against
the allocating entry point.
"""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk

TOL = 1e-13


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def _spectral_planes(rng, npl, n):
    a = rng.standard_normal((npl, n, n // 2 + 1)) + 1j * rng.standard_normal((npl, n, n // 2 + 1))
    return a.astype(np.complex128)


@pytest.mark.gpu
def test_noalloc_ff2cr_matches_allocating_entry_point():
    import torch

    lib = pk.load_library()
    rng = np.random.default_rng(2024)
    # two calls in a row at the largest size, then every other size and back
    for n in (128, 128, 32, 64, 96, 128):
        npl = 3
        a = _spectral_planes(rng, npl, n)
        want = pk.ff2cr(a, n)
        d_a = torch.from_numpy(a.view(np.float64).copy()).cuda()
        d_b = torch.full((npl, n, n), float("nan"), dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rc = lib.pibm_ff2cr_noalloc(n, n, npl, C.c_void_p(d_a.data_ptr()), C.c_void_p(d_b.data_ptr()),
                                    C.c_void_p(stream))
        assert rc == 0, lib.pibm_last_error().decode()
        torch.cuda.synchronize()
        got = d_b.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel(got, want) < TOL


@pytest.mark.gpu
def test_noalloc_ff2cr_rejects_sizes_beyond_the_static_scratch():
    import torch

    lib = pk.load_library()
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(d.data_ptr())
    rc = lib.pibm_ff2cr_noalloc(256, 256, 1, p, p, None)
    assert rc == pk.abi.PIBM_ERR_ARG
    assert "128" in lib.pibm_last_error().decode()
    rc = lib.pibm_ff2cr_noalloc(48, 48, 1, p, p, None)
    assert rc == pk.abi.PIBM_ERR_ARG


# Runs in a child process with no torch: device buffers come from the CUDA
# runtime the library is linked against, so a cudaDeviceReset between calls
# invalidates nothing but this process's own context.
_RESET_CHILD = textwrap.dedent("""
    import ctypes as C, sys
    import numpy as np
    sys.path.insert(0, sys.argv[1])
    import pureibm_ps2d_fd1d_b200 as pk
    lib = pk.load_library()
    rt = C.CDLL("libcudart.so.12")
    rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    rt.cudaFree.argtypes = [C.c_void_p]
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    n, npl = 64, 2
    rng = np.random.default_rng(5)
    worst = 0.0
    for rnd in range(2):
        a = rng.standard_normal((npl, n, n // 2 + 1)) + 1j * rng.standard_normal((npl, n, n // 2 + 1))
        want = pk.ff2cr(a, n)
        da, db = C.c_void_p(), C.c_void_p()
        assert rt.cudaMalloc(C.byref(da), a.nbytes) == 0
        assert rt.cudaMalloc(C.byref(db), want.nbytes) == 0
        assert rt.cudaMemcpy(da, a.ctypes.data, a.nbytes, 1) == 0
        rc = lib.pibm_ff2cr_noalloc(n, n, npl, da, db, None)
        assert rc == 0, lib.pibm_last_error().decode()
        got = np.empty_like(want)
        assert rt.cudaMemcpy(got.ctypes.data, db, want.nbytes, 2) == 0
        worst = max(worst, float(np.max(np.abs(got - want)) / np.max(np.abs(want))))
        rt.cudaFree(da)
        rt.cudaFree(db)
        if rnd == 0:
            assert rt.cudaDeviceReset() == 0
    print("worst", worst)
    assert worst < 1e-13, worst
""")


@pytest.mark.gpu
def test_noalloc_ff2cr_after_device_reset():
    """A device reset between two calls: the second call finds a new device
    context (whose copy of the static table starts zeroed) and writes the
    table again instead of reading zeros."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _RESET_CHILD, root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
