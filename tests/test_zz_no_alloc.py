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
    # two calls in a row at the largest size, then a size change and back
    for n in (128, 128, 64, 96, 128):
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
