"""The reference's random particle configurations (INPUT_TYPE = 'random').

Restated here, host-side:

* the random-number stream of the reference's ``Rn`` library:
  ``vrand`` (Rn/vrand.f:1-80: the multiplicative congruential integer stream
  i <- 65539*i mod 2**31, single-precision conversion, a 97-entry shuffle
  store kept across calls), ``ranu2`` (Rn/ranu2.f: vectors drawn from it),
  ``ransed`` (Rn/ransed.f: the seed), ``rann2`` (Rn/rann2.f: standard normals
  by table inversion of the Abramowitz-Stegun 7.1.26 error function, with
  ``ranstd`` standardisation, Rn/ranstd.f), ``ranjn`` (Rn/ranjn.f:
  joint-normal vectors through a Cholesky factor), and ``getnewseed`` /
  ``uni_dist`` / ``jn_dist`` (SRC/SHARED_MODULES/randomno.F90:45-167: a
  400-entry seed array drawn from the seed in ``RUN_NAME_seed.d``, which is
  rewritten with the next seed).  The library works in single precision
  (REAL*4, as Rn/rn_opt_gfortran compiles it); so does this restatement,
  with numpy float32 arithmetic.  float32 exp / log / sqrt are numpy's, so a
  table entry of rann2 can differ from a compiled library's in the last bit.
  The reference passes REAL(8) arrays to these REAL*4 routines
  (randomno.F90:63-86, 100-119, 136); the restatement gives them the REAL*4
  arrays they declare.
* ``gener_lattice_mod`` (SRC/FLO/dependent_functions.F90:1551-1646): the
  starting lattice, exactly.
* ``generate_psd_config`` for one phase of PSD_TYPE = 'discrete'
  (SRC/FLO/initialize_flo.F90:2729-3133) and ``gener_config_random``
  (:3137-3413): particle count, box, grid, the buffered diameter, the lattice
  and its rescaling in y, the final scaling to grid units with the overlap
  check of ``scale_to_grid_units`` (dependent_functions.F90:1812-1942).
  The reference then shakes the lattice with its soft-sphere DEM (gravity
  settling with shrinking walls when the lattice is taller than the box,
  then an elastic shake with Maxwellian velocities for ten mean free times;
  ``des_time_march``).  That stage is chaotic -- no two machines reproduce it
  -- and is replaced here by hard-sphere Monte Carlo moves drawn from the
  same vrand stream, which relax the lattice to an equilibrium hard-sphere
  configuration of the same volume fraction.
"""
from __future__ import annotations

import math
import os
from typing import Dict, Optional, Tuple

import numpy as np

F4 = np.float32


# ---------------------------------------------------------------------------
# Rn library
# ---------------------------------------------------------------------------
class Rn:
    """State of the reference's random-number library: the seed ix
    (common /rancom/), vrand's shuffle store and rann2's table (both SAVEd,
    set up on their first call), and randomno's seed array."""

    NSTORE = 97
    C = F4(0.46566127e-9)

    def __init__(self):
        self.ix = 0
        self.store: Optional[np.ndarray] = None
        self.k = 0
        self.tab: Optional[np.ndarray] = None
        self.seedarray: Optional[np.ndarray] = None
        self.count = 0

    # vrand (Rn/vrand.f) -----------------------------------------------------
    @staticmethod
    def next_int(i: int) -> int:
        """i*65539 in 32-bit arithmetic, negative results moved up by 2**31:
        i*65539 mod 2**31 (Rn/vrand.f:52-53, 66-67)."""
        return (i * 65539) % 2147483648

    def _k_of(self, s: np.float32) -> int:
        return int(F4(F4(s * F4(self.NSTORE)) + F4(1.0)))

    def vrand(self, n: int) -> np.ndarray:
        if self.ix == 0:
            raise ValueError("error in vrand - seed = 0.")
        i = self.ix
        if self.store is None:
            self.store = np.zeros(self.NSTORE + 1, dtype=F4)
            for j in range(self.NSTORE + 1):
                i = self.next_int(i)
                self.store[j] = F4(F4(i) * self.C)
            self.k = self._k_of(self.store[self.NSTORE])
        out = np.empty(n, dtype=F4)
        for j in range(n):
            out[j] = self.store[self.k - 1]
            i = self.next_int(i)
            self.store[self.k - 1] = F4(F4(i) * self.C)
            self.k = self._k_of(self.store[self.k - 1])
        self.ix = i
        return out

    def ransed(self, seed: int):
        """ransed(-1, lu, seed, 1): ix = seed (Rn/ransed.f:15-20)."""
        self.ix = int(seed)

    def ranu2(self, nj: int, nk: int = 1) -> np.ndarray:
        """x(j, k), j fastest: nj*nk numbers of vrand (Rn/ranu2.f)."""
        return self.vrand(nj * nk).reshape(nk, nj).T.copy()

    # rann2 (Rn/rann2.f) -----------------------------------------------------
    @staticmethod
    def erff(x: np.float32) -> np.float32:
        """Abramowitz and Stegun 7.1.26 in single precision (Rn/rann2.f:236-252)."""
        p, a1, a2, a3, a4, a5 = (F4(v) for v in (.3275911, .254829592, -.284496736, 1.421413741, -1.453152027, 1.061405429))
        t = F4(F4(1.0) / F4(F4(1.0) + F4(p * F4(abs(x)))))
        h = a5                       # q = t*(a1+t*(a2+t*(a3+t*(a4+t*a5)))), innermost first
        for a in (a4, a3, a2, a1):
            h = F4(a + F4(t * h))
        q = F4(t * h)
        e = F4(F4(1.0) - F4(q * np.exp(F4(-F4(x * x)))))
        return F4(-e) if x < 0 else e

    def _rann2_table(self):
        ntab = 201
        pi, rtpii, rti = F4(3.1415927), F4(0.3989423), F4(0.7071068)
        fdens = lambda xx: F4(rtpii * np.exp(F4(F4(-0.5) * F4(xx * xx))))
        fdist = lambda xx: F4(F4(0.5) * F4(F4(1.0) + self.erff(F4(rti * xx))))
        ntabm, ntabmm, ntsq = ntab - 1, ntab - 2, ntab * ntab
        dy = F4(F4(1.0) / F4(ntabm))
        p3 = F4(F4(F4(ntsq) * F4(5.800e-6)) - F4(F4(ntab) * F4(4.35160e-3)) - F4(1.7006542))
        p2 = F4(F4(F4(ntsq) * F4(6.035e-6)) - F4(F4(ntab) * F4(4.46257e-3)) - F4(1.8738435))
        p1 = F4(F4(F4(ntabm) * np.exp(F4(F4(-p2 * p2) / F4(2.0)))) / np.sqrt(F4(F4(2.0) * pi)))
        xmin = F4(F4(F4(F4(2.0) * pi) * p1) * p1 * F4(1.e-14))
        xmin = F4(-np.log(xmin))
        xmin = F4(-np.sqrt(xmin))
        xmax = F4(-xmin)
        tab = np.zeros(ntab, dtype=F4)
        tab[0], tab[1], tab[2] = xmin, p2, p3
        tab[ntab - 1], tab[ntabm - 1], tab[ntabmm - 1] = xmax, -p2, -p3
        y = F4(F4(2.0) * dy)
        xx = F4(tab[2] + F4(dy * F4(xmax - xmin)))
        ntabh = ntab // 2
        for i in range(4, ntabh + 1):
            y = F4(y + dy)
            xxmin, xxmax = tab[i - 2], xmax
            for _ in range(50):
                yy = fdist(xx)
                err = F4(yy - y)
                if abs(err) < F4(1.e-6):
                    break
                if err > 0:
                    xxmax = xx
                if err < 0:
                    xxmin = xx
                xx = F4(xx + F4(err / max(fdens(xx), F4(1.e-10))))
                if xx <= xxmin or xx >= xxmax:
                    xx = F4(F4(0.5) * F4(xxmin + xxmax))
            tab[i - 1] = xx
        for i in range(1, ntabh + 1):
            tab[ntab - i] = -tab[i - 1]
        tab[ntabh] = F4(0.0)
        self.tab = tab
        self.dtab = (tab[1:] - tab[:-1]).astype(F4)
        self.p1, self.ntabm, self.pi = p1, ntabm, pi

    def rann2(self, nj: int, nk: int = 1) -> np.ndarray:
        """Standard normal x(j, k) (Rn/rann2.f:103-155)."""
        if self.tab is None:
            self._rann2_table()
        x = self.ranu2(nj, nk)
        twopp = F4(F4(F4(2.0) * self.pi) * self.p1) * self.p1
        for k in range(nk):
            for j in range(nj):
                u = x[j, k]
                yv = F4(F4(u * F4(self.ntabm)) + F4(1.0))
                i = int(yv)
                if i == 1:
                    y1 = F4(twopp * u * u)
                    if y1 <= 0:
                        y1 = F4(1.e-20)
                    x[j, k] = F4(-np.sqrt(F4(-np.log(y1))))
                elif i == self.ntabm:
                    y1 = F4(F4(1.0) - u)
                    y1 = F4(twopp * y1 * y1)
                    x[j, k] = F4(np.sqrt(F4(-np.log(y1))))
                else:
                    f = F4(yv - F4(i))
                    x[j, k] = F4(self.tab[i - 1] + F4(f * self.dtab[i - 1]))
        if nj >= 5:
            for k in range(nk):
                x[:, k] = self.ranstd(x[:, k])
        return x

    @staticmethod
    def ranstd(x: np.ndarray) -> np.ndarray:
        """Sample mean 0 and variance 1 (Rn/ranstd.f)."""
        n = len(x)
        if n <= 1:
            return x
        s1, s2 = F4(0.0), F4(0.0)
        for v in x:
            s1 = F4(s1 + v)
            s2 = F4(s2 + F4(v * v))
        s1 = F4(s1 / F4(n))
        s2 = F4(s2 / F4(n))
        s2 = F4(F4(1.0) / np.sqrt(F4(s2 - F4(s1 * s1)))) if s2 > 0 else F4(1.0)
        s1 = F4(-s1 * s2)
        return np.array([F4(s1 + F4(s2 * v)) for v in x], dtype=F4)

    def ranjn(self, nj: int, mean, cov) -> np.ndarray:
        """Joint-normal vectors x(j, :) of mean xm and covariance cv through
        the Cholesky factor of cv (Rn/ranjn.f:55-128)."""
        n = len(mean)
        L = np.array(cov, dtype=F4).copy()
        L[0, 0] = np.sqrt(L[0, 0])
        for k in range(1, n):
            if L[0, 0] > 0:
                L[k, 0] = F4(L[k, 0] / L[0, 0])
            sumllt = F4(L[k, 0] * L[k, 0])
            for j in range(1, k):
                s = F4(0.0)
                for m in range(j):
                    s = F4(s + F4(L[j, m] * L[k, m]))
                if L[j, j] > 0:
                    L[k, j] = F4(F4(L[k, j] - s) / L[j, j])
                sumllt = F4(sumllt + F4(L[k, j] * L[k, j]))
            cvkk = F4(L[k, k] - sumllt)
            if cvkk < 0:
                raise ValueError("ranjn: matrix non-positive definite")
            L[k, k] = np.sqrt(cvkk)
        x = self.rann2(nj, n)
        for j in range(nj):
            for kk in range(n - 1, -1, -1):
                s = F4(0.0)
                for ll in range(kk + 1):
                    s = F4(s + F4(L[kk, ll] * x[j, ll]))
                x[j, kk] = F4(F4(mean[kk]) + s)
        return x

    # randomno.F90 -----------------------------------------------------------
    def getnewseed(self, seed_file: str) -> int:
        """Next seed value: on the first call (and after the seed array runs
        out) the array of 400 uniforms is drawn from the seed in the seed
        file, which is then rewritten with the value taken; entries below
        0.1 (fewer than 8 digits) are skipped (randomno.F90:120-167)."""
        n = 400
        self.count += 1
        change = False
        while True:
            if self.count > n or self.count < 1:
                self.count = 1
            if self.count == 1:
                change = True
                with open(seed_file) as fh:
                    self.ransed(int(fh.readline()[:8]))
                self.seedarray = self.ranu2(n)[:, 0]
            while True:
                sd = int(float(self.seedarray[self.count - 1]) * 100000000)
                if sd // 10000000 != 0:
                    if change:
                        with open(seed_file, "w") as fh:
                            fh.write("%8d\n" % sd)
                    return sd
                self.count += 1
                if self.count >= n:
                    break

    def uni_dist(self, n: int, seed_file: str) -> np.ndarray:
        self.ransed(self.getnewseed(seed_file))
        return self.ranu2(n)[:, 0]

    def jn_dist(self, nj: int, mean, cov, seed_file: str) -> np.ndarray:
        self.ransed(self.getnewseed(seed_file))
        return self.ranjn(nj, mean, cov)


# ---------------------------------------------------------------------------
# Configuration
# ---------------------------------------------------------------------------
def gener_lattice_mod(nbody: int, doml, dia1: float) -> np.ndarray:
    """Starting lattice (dependent_functions.F90:1551-1646): rows of spheres
    along x, layers along z, stacked in y at spacing 1.05*dia1 from dia1/2."""
    fac = 1.05
    dmax = dia1
    xc = np.zeros((nbody, 3))
    n = 1
    yp = dmax * fac / 2.0
    while n < nbody:
        # nz takes real(DOMLIN(3) - dmax*fac): single precision, as written
        nz = math.ceil(float(np.float32(doml[2] - dmax * fac)) / (dmax * fac))
        nx = math.ceil((doml[0] - dmax * fac) / (dmax * fac))
        done = False
        for k in range(1, nz + 1):
            zp = dmax * 0.5 + (k - 1) * dmax * fac
            for i in range(1, nx + 1):
                xp = dmax * 0.5 + (i - 1) * dmax * fac
                xc[n - 1] = (xp, yp, zp)
                if n == nbody:
                    done = True
                    break
                n += 1
            if done:
                break
        if done:
            break
        yp = yp + dmax * fac
    return xc


def psd_discrete_one_phase(prm: Dict) -> Dict:
    """generate_psd_config for PSD_TYPE = 'discrete', NPHASES = 1
    (initialize_flo.F90:2829-2880, 2937-2975): particle count, box, grid and
    the buffered diameter."""
    davg = float(prm.get("dia_phys", 1.0))
    lybyd = float(prm["lybyd"])
    phiavg = float(prm.get("phiavg", prm.get("vol_frac1", 0.2)))
    doml = np.array([lybyd * davg] * 3)
    nbody = int(phiavg * 6.0 * (lybyd ** 3.0) / math.pi)
    my = int(prm.get("my") or 0)
    if my <= 0:
        my = int((doml[1] / davg) * float(prm["dbydx"]))
        if my % 2:
            my += 1
    dx = doml[1] / float(my)
    min_part_sep = float(prm.get("min_part_sep", 0.0))
    percent_buf = (min_part_sep * dx / davg) * 100.0 + 1.0
    dia_inc = davg * (1.0 + percent_buf / 100.0)
    return dict(nbody=nbody, doml=doml, my=my, dx=dx, davg=davg, dia_inc=dia_inc, percent_buf=percent_buf,
                min_part_sep=min_part_sep, phiavg=phiavg)


def hs_shake(xc: np.ndarray, doml, dia: float, rn: Rn, sweeps: int, step: float) -> Tuple[np.ndarray, int]:
    """Hard-sphere Monte Carlo moves in the periodic box, trial displacements
    and the particle order drawn from the vrand stream (stand-in for the
    DEM shake, see the module notes).  Returns the positions and the number
    of accepted moves."""
    L = np.asarray(doml, dtype=float)
    x = xc.copy()
    n = x.shape[0]
    acc = 0
    d2 = dia * dia
    for _ in range(sweeps):
        u = rn.ranu2(n, 4).astype(float)
        for m in range(n):
            i = min(int(u[m, 0] * n), n - 1)
            trial = x[i] + step * (2.0 * u[m, 1:4] - 1.0)
            trial -= L * np.floor(trial / L)
            d = x - trial
            d -= L * np.round(d / L)
            r2 = np.einsum("ij,ij->i", d, d)
            r2[i] = np.inf
            if np.min(r2) >= d2:
                x[i] = trial
                acc += 1
    return x, acc


def scale_to_grid_units(xp_unit: np.ndarray, rad_unit: np.ndarray, my: int, mbox: int, percent_buf: float,
                        min_part_sep: float) -> Tuple[np.ndarray, np.ndarray]:
    """Positions in [0,1) of the box to grid units (x: *(mbox-1)+1, y, z:
    *my+1), radii unbuffered and in grid units, and every sphere closer than
    min_part_sep grid points to another removed (dependent_functions.F90:1812-1942)."""
    xp = xp_unit.copy()
    xp[:, 0] = xp[:, 0] * (mbox - 1) + 1.0
    xp[:, 1:] = xp[:, 1:] * my + 1
    rad = rad_unit / (1.0 + percent_buf * 1.0 / 100.0) * my
    n = xp.shape[0]
    rmax = np.array([(mbox - 1) / 2.0, my / 2.0, my / 2.0])
    L = np.array([mbox - 1, my, my], dtype=float)
    towrite = np.ones(n, dtype=bool)
    for i in range(n):
        for j in range(n):
            if i != j and towrite[j]:
                t = xp[i] - xp[j]
                big = np.abs(t) > rmax
                t = np.where(big, np.where(t < 0, t + L, t - L), t)
                r = math.sqrt(float(np.sum(t ** 2.0)))
                if r <= rad[i] + rad[j] + min_part_sep:
                    towrite[i] = False
    return xp[towrite], rad[towrite]


def gener_config_random(prm: Dict, seed_file: str, rn: Optional[Rn] = None, sweeps: int = 200) -> Dict:
    """A random configuration for one phase of PSD_TYPE = 'discrete'
    (generate_psd_config + gener_config_random, initialize_flo.F90:2729-3413;
    the DEM shake replaced as the module notes say).  Returns the run's MY,
    the centres (nbody, 3) in grid units (node i at x = i) and the radius."""
    rn = rn or Rn()
    g = psd_discrete_one_phase(prm)
    nbody, doml, dia = g["nbody"], g["doml"], g["dia_inc"]
    xc = gener_lattice_mod(nbody, doml, dia)
    ylength = xc[:, 1].max() + dia * 0.5
    if ylength < doml[1]:
        # the lattice fits: stretch it over the box height (:3294-3307)
        ymin = xc[:, 1].min() - dia * 0.5
        ymax = xc[:, 1].max() + dia * 0.5
        a = doml[1] / (ymax - ymin)
        b = -a * ymin
        xc[:, 1] = xc[:, 1] * a + b
    else:
        raise ValueError("the starting lattice is taller than the box (volume fraction %.3f): the reference settles it "
                         "under gravity with shrinking walls (des_time_march with SHRINK), which is not restated"
                         % g["phiavg"])
    # the shake: Maxwellian velocities of variance pvel_var drawn as the
    # reference draws them (init_particles_jn, collision_mod.F90:1761-1783),
    # then hard-sphere moves of a tenth of a diameter
    pvel_var = float(prm.get("pvel_var", 1.0))
    cov = np.diag([pvel_var / 3.0] * 3)
    vel = rn.jn_dist(nbody, np.zeros(3), cov, seed_file).astype(float)
    xc, acc = hs_shake(xc, doml, dia, rn, sweeps, 0.1 * dia)
    mbox = g["my"] + 1
    xg, rad = scale_to_grid_units(xc / doml, np.full(nbody, 0.5 * dia / doml[1]), g["my"], mbox, g["percent_buf"],
                                  g["min_part_sep"])
    return dict(my=g["my"], xc=xg, radbdy=rad, nbody_requested=nbody, velocities=vel, accepted_moves=acc,
                doml=doml, dia=g["davg"])


def load_random_run(prm: Dict, directory: str, run_name: str, **kw) -> Tuple[Dict, np.ndarray]:
    """INPUT_TYPE = 'random': the run's parameters with MY (and LYBYD, DBYDX)
    set and the generated centres, from RUN_NAME_seed.d in `directory` (which
    is rewritten with the next seed, as the reference does)."""
    seed_file = os.path.join(directory, "%s_seed.d" % run_name)
    out = gener_config_random(prm, seed_file, **kw)
    prm = dict(prm)
    prm["my"] = out["my"]
    prm["mz"] = out["my"]
    prm["dbydx"] = out["my"] / float(prm["lybyd"])
    return prm, out["xc"]
