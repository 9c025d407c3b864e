"""kinks.smooth_interval: the offsets of the nearest stencil-cell crossing or
mask change of a sphere coordinate, checked against a brute-force scan of the
step's geometry (the floors of every stencil point coordinate and the set of
solid nodes) on a fine grid of offsets."""
import math

import numpy as np

from pureibm_ps2d_fd1d_b200 import kinks


def _state(xc_m, bnd, R, dr):
    pts = []
    for r in (R, R - dr, R + dr):
        v = xc_m[None, :] + bnd * r
        pts.append(np.floor(v))
        if r != R + dr:
            w = v.copy()
            w[:, 0] -= 0.5
            pts.append(np.floor(w))
    Rs = R + kinks.SMALL
    ax = [np.arange(math.ceil(xc_m[k] - Rs) - 1, math.floor(xc_m[k] + Rs) + 2) for k in range(3)]
    g = np.stack(np.meshgrid(*ax, indexing="ij"), -1).reshape(-1, 3).astype(float)
    inside = np.sqrt(((g - xc_m) ** 2).sum(-1)) - R <= kinks.SMALL
    return np.concatenate([p.ravel() for p in pts]), {tuple(x) for x in g[inside]}


def test_smooth_interval_matches_a_scan():
    rng = np.random.default_rng(3)
    b = rng.standard_normal((60, 3))
    bnd = b / np.linalg.norm(b, axis=1, keepdims=True)
    R, dr = 4.0, 1.0
    for trial in range(6):
        xc_m = np.array([20.0, 20.0, 20.0]) + rng.uniform(0, 1, 3)
        d = trial % 3
        lo, hi = kinks.smooth_interval(xc_m, d, bnd, R, dr)
        assert lo <= 0.0 <= hi and hi - lo < 1.0
        base = _state(xc_m, bnd, R, dr)
        for t in np.linspace(lo, hi, 41)[1:-1]:
            x = xc_m.copy()
            x[d] += t
            s = _state(x, bnd, R, dr)
            assert np.array_equal(s[0], base[0]) and s[1] == base[1], (trial, t)
        for edge in (lo, hi):
            x = xc_m.copy()
            x[d] += edge + (1e-9 if edge > 0 else -1e-9)
            s = _state(x, bnd, R, dr)
            assert not (np.array_equal(s[0], base[0]) and s[1] == base[1]), (trial, edge)
    # a stencil point on a cell face: no smooth piece
    xc_m = np.array([20.0 - R, 20.3, 20.7])
    assert kinks.fd_step(xc_m, 0, np.array([[1.0, 0.0, 0.0]]), R, dr, 1e-3) == 0.0
