"""Seeded multiple-independent-simulation ensemble generator (host side)."""
import numpy as np

from pureibm_ps2d_fd1d_b200 import config


def _min_dist(pts, L):
    d = pts[:, None, :] - pts[None, :, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d ** 2).sum(-1))
    np.fill_diagonal(r, np.inf)
    return r.min() if len(pts) > 1 else np.inf


def test_ensemble_is_seeded_and_overlap_free():
    a = config.mis_ensemble(n=6, seed=7)
    b = config.mis_ensemble(n=6, seed=7)
    for (pa, xa, fa), (pb, xb, fb) in zip(a, b):
        assert pa == pb and fa == fb
        np.testing.assert_array_equal(xa, xb)
    for prm, xc, phi in a:
        L, d = prm["my"], prm["dbydx"]
        assert prm["my"] in (64, 96, 128)
        assert 12 <= d <= 20 and 10.0 <= prm["re"] <= 100.0
        assert np.all((xc >= 1.0) & (xc < 1.0 + L))
        assert _min_dist(xc, L) >= d - 1e-9
        assert 0.0 < phi <= 0.4 + 1e-9
        assert abs(phi - len(xc) * np.pi / 6 * d ** 3 / L ** 3) < 1e-12


def test_dense_members_use_the_lattice_start():
    ens = config.mis_ensemble(n=4, seed=11, grids=(64,), phi_range=(0.38, 0.4), dia_range=(12, 12))
    for prm, xc, phi in ens:
        assert phi > 0.3
        assert _min_dist(xc, prm["my"]) >= prm["dbydx"] - 1e-9


def test_fcc_subset_capacity():
    rng = np.random.default_rng(0)
    assert config.fcc_subset(33, 64.0, 20.0, rng) is None       # 2x2x2 cells hold 32 sites
    pts = config.fcc_subset(32, 64.0, 20.0, rng)
    assert pts.shape == (32, 3) and _min_dist(pts, 64.0) >= 20.0 * np.sqrt(2.0) / np.sqrt(2.0) - 1e-9
