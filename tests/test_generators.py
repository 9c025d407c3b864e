"""The reference's random configurations (INPUT_TYPE = 'random'):
the Rn library's streams, the starting lattice and the generated runs
(generators.py)."""
import math
import os

import numpy as np
import pytest

from pureibm_ps2d_fd1d_b200 import config, generators as G

F4 = np.float32


def test_vrand_integer_stream_is_randu():
    """i <- 65539 i in 32-bit integers with the negative values moved up by
    2**31 (the reference's form) is 65539 i mod 2**31: from seed 1 the
    published RANDU sequence, and every triple obeys x2 = 6 x1 - 9 x0 mod 2**31."""
    def fortran_step(i):
        v = (i * 65539) & 0xFFFFFFFF
        v = v - (1 << 32) if v >= (1 << 31) else v          # 32-bit wrap of i*65539
        return v + 2147483647 + 1 if v < 0 else v
    seq, i = [], 1
    for _ in range(5):
        i = G.Rn.next_int(i)
        seq.append(i)
    assert seq == [65539, 393225, 1769499, 7077969, 26542323]
    i = 987654321
    xs = []
    for _ in range(2000):
        j = G.Rn.next_int(i)
        assert j == fortran_step(i)
        xs.append(j)
        i = j
    for a, b, c in zip(xs, xs[1:], xs[2:]):
        assert c == (6 * b - 9 * a) % 2147483648


def test_vrand_shuffle_store():
    """First call: 98 values x = real(i)*0.46566127e-9 in single precision fill
    the store, k = int(store(98)*97 + 1); every draw returns store(k) and
    refills that slot from the stream (Rn/vrand.f:47-71)."""
    rn = G.Rn()
    rn.ransed(1)
    out = rn.vrand(3)
    i, store = 1, []
    for _ in range(98):
        i = (i * 65539) % 2147483648
        store.append(F4(F4(i) * F4(0.46566127e-9)))
    k = int(F4(F4(store[97] * F4(97)) + F4(1)))
    want = []
    for _ in range(3):
        want.append(store[k - 1])
        i = (i * 65539) % 2147483648
        store[k - 1] = F4(F4(i) * F4(0.46566127e-9))
        k = int(F4(F4(store[k - 1] * F4(97)) + F4(1)))
    assert [float(v) for v in out] == [float(v) for v in want]
    assert rn.ix == i
    # the store survives a new seed (SAVE): a second seed continues with it
    rn.ransed(7)
    a = rn.vrand(4)
    assert np.all((a > 0) & (a < 1))


def test_rann2_table_erff_and_standardisation():
    rn = G.Rn()
    rn.ransed(20240601)
    x = rn.rann2(500, 3)
    tab = rn.tab
    assert np.all(np.diff(tab) > 0) and tab[100] == 0.0
    assert np.array_equal(tab, -tab[::-1])
    for v in np.linspace(-3, 3, 61):
        assert abs(float(G.Rn.erff(F4(v))) - math.erf(v)) < 5e-7
    # ranstd: sample mean 0 and variance 1 per component, to single precision
    assert np.all(np.abs(x.mean(axis=0)) < 1e-6)
    assert np.all(np.abs(x.astype(float).var(axis=0) - 1.0) < 1e-5)
    # ranjn with a diagonal covariance scales the standard normals
    rn2 = G.Rn()
    rn2.ransed(20240601)
    v = rn2.ranjn(500, np.zeros(3), np.diag([4.0, 4.0, 4.0]))
    assert np.allclose(v.astype(float), 2.0 * x.astype(float), rtol=0, atol=1e-5)


def test_getnewseed_rewrites_the_seed_file(tmp_path):
    path = str(tmp_path / "RUN_seed.d")
    open(path, "w").write("12345678\n")
    rn = G.Rn()
    s1 = rn.getnewseed(path)
    assert 10000000 <= s1 <= 99999999
    assert int(open(path).read()) == s1                 # the first seed of a fresh array is written back
    s2 = rn.getnewseed(path)
    assert s2 != s1 and int(open(path).read()) == s1    # later draws leave the file alone
    open(path, "w").write("12345678\n")
    assert G.Rn().getnewseed(path) == s1                # deterministic in the file's seed


def test_gener_lattice_mod_by_hand():
    """Box 5 diameters, 20 spheres: nx = nz = ceil((5 - 1.05)/1.05) = 4 per
    row, 16 per layer at y = 0.525, the next 4 at y = 1.575."""
    xc = G.gener_lattice_mod(20, (5.0, 5.0, 5.0), 1.0)
    for n in range(20):
        layer, r = divmod(n, 16)
        k, i = divmod(r, 4)
        assert np.allclose(xc[n], (0.5 + i * 1.05, 0.525 + layer * 1.05, 0.5 + k * 1.05), rtol=0, atol=1e-12)


def _write_random_run(d, phiavg=0.2):
    text = """ &FLOANDGRID
 VIS = 0.012, RE = 20.0, CFL = 0.1, CFL_MAX = 0.5, RAMP_FRAC_STEPS = 0
 /
 &PART_PROPT
 LYBYD = 4.0, DBYDX = 16.0, DIA_PHYS = 1.0, INPUT_TYPE = 'random', DISCR_SCHEME = 'upwind'
 /
 &FLAGS
 DOBND = F, INITIALIZE_ZERO = T
 /
 &FILES
 /
 &PSD
 PSD_TYPE = 'discrete', PHIAVG = %s, NPHASES = 1
 /
 &GCG
 PVEL_VAR = 1.0
 /
 &POSTLIST
 /
""" % phiavg
    open(os.path.join(d, "RUN_floparam.in"), "w").write(text)
    open(os.path.join(d, "RUN_seed.d"), "w").write("20231107\n")


def test_random_input_generates_a_valid_configuration(tmp_path):
    d = str(tmp_path)
    _write_random_run(d)
    prm, xc = config.load_run(d, "RUN")
    assert prm["my"] == 64 and xc.shape == (int(0.2 * 6 * 64 / math.pi), 3)
    rad = 0.5 * prm["my"] / prm["lybyd"]
    L = float(prm["my"])
    assert np.all((xc >= 1.0) & (xc < L + 1.0))
    dd = xc[:, None, :] - xc[None, :, :]
    dd -= L * np.round(dd / L)
    r = np.sqrt((dd ** 2).sum(-1)) + np.eye(len(xc)) * 1e9
    assert r.min() >= 2.0 * rad
    # the same seed file gives the same configuration; the file moves on
    assert int(open(os.path.join(d, "RUN_seed.d")).read()) != 20231107
    open(os.path.join(d, "RUN_seed.d"), "w").write("20231107\n")
    _, xc2 = config.load_run(d, "RUN")
    assert np.array_equal(xc, xc2)
    P = config.make_params(prm)
    assert P.my == 64 and P.dobnd == 0


def test_random_input_taller_lattice_is_refused(tmp_path):
    d = str(tmp_path)
    _write_random_run(d, phiavg=0.45)
    with pytest.raises(ValueError, match="taller than the box"):
        config.load_run(d, "RUN")
