"""The reference driver's time loop with its per-step records
(SRC/FLO/dtibm_main_scal_flo.F90:426-527; records of bcset,
boundary_condition.F90:849-870, and of the driver, :319-322, 460).

    run = Run(params, xc, vel, run_name="RUN", directory="out", tend=10.0)
    run.advance(200)        # 200 time steps (every rks stage), records appended

Files (rank-0 output of the reference, the same columns and Fortran edit
descriptors):

    RUN_norm_drag.dat        t/t_conv/(1-maxvolfrac), t/t_vis, t/t_diff,
                             norm_drag, norm_drag of the phase, usmean_act(1:3),
                             ufmean(1:3)/ucharmod                 (2x, e20.12)
    RUN_norm_drag_chem.dat   t/t_conv/(1-maxvolfrac), t/t_vis, t/t_diff,
                             norm_drag_chem, norm_drag_chem of the phase
    RUN_drag_components.dat  pres_drag, visc_drag, total_drag, total_drag_mpg,
                             norm_drag, |total_drag - total_drag_mpg|/(total_drag + SMALL)
    RUN_dt_history.dat       ISTEP, DT, #STEPS REQD, CFL       (2x, g17.8)

The records are written after the last stage of every step (rks = itrmax),
as the reference does.  Quantities not in the step report are formed here
from the per-particle forces and the run's constants with the reference's
expressions.  One phase (the 'default' input): the phase drag equals the
mixture drag up to the volume-fraction weighting.
"""
from __future__ import annotations

import math
import os
from typing import Optional

import numpy as np

SMALL_NUMBER = float(np.float32(1.0e-35))
LARGE_NUMBER = float(np.float32(1.0e32))


# ---------------------------------------------------------------------------
# Fortran edit descriptors Ew.d and Gw.d (list of the rules: F2008 10.7.2.3)
# ---------------------------------------------------------------------------
def fortran_e(x: float, w: int = 20, d: int = 12) -> str:
    """Ew.d: 0.ddd...E+ee (two-digit exponent, three when |exp| > 99)."""
    if x != x:
        return "NaN".rjust(w)
    if math.isinf(x):
        return ("-Infinity" if x < 0 else "Infinity").rjust(w)
    if x == 0.0:
        s = "0." + "0" * d + "E+00"
        return ("-" + s if math.copysign(1.0, x) < 0 else s).rjust(w)
    m, e = "{:.{p}e}".format(abs(x), p=d - 1).split("e")
    digits = m.replace(".", "")
    exp = int(e) + 1
    es = "E%+03d" % exp if abs(exp) <= 99 else "%+04d" % exp
    s = "0." + digits + es
    return (("-" if x < 0 else "") + s).rjust(w)


def fortran_g(x: float, w: int = 17, d: int = 8) -> str:
    """Gw.d: F editing with d significant digits and 4 trailing blanks when
    0.1 <= |x| < 10**d (after rounding), else Ew.d."""
    ax = abs(x)
    if x == x and not math.isinf(x) and ax != 0.0:
        r = float("{:.{p}e}".format(ax, p=d - 1))
        if 0.1 <= r < 10.0 ** d:
            k = int(math.floor(math.log10(r))) + 1        # digits before the point
            s = "{:.{p}f}".format(ax, p=d - k)
            return ((("-" if x < 0 else "") + s).rjust(w - 4)) + "    "
    if ax == 0.0 and x == x:
        return ("0." + "0" * (d - 1)).rjust(w - 4) + "    "
    return fortran_e(x, w, d)


def _line(values, fmt) -> str:
    return "".join("  " + fmt(float(v)) for v in values) + "\n"


class Run:
    """A solver stepped the way the reference's driver steps it, with the
    rank-0 records appended after every time step."""

    def __init__(self, params, xc=None, vel=None, run_name: str = "RUN", directory: str = ".",
                 tend: Optional[float] = None, solver=None):
        from . import Solver, config
        self.P = params if not isinstance(params, dict) else config.make_params(params)
        self.s = solver if solver is not None else Solver(self.P, xc, vel)
        self.itrmax = 3 if self.P.rk3 else 1
        self.run_name, self.directory = run_name, directory
        self.tend = tend
        self.iglobstep = 0
        os.makedirs(directory, exist_ok=True)
        P = self.P
        info = self.s.info
        # initflo constants (initialize_flo.F90:277-283, 550-627; scalar_init.F90:79)
        uchar = (P.re * P.vis) / P.dia_phys
        self.uchar = [uchar * math.cos(math.pi * a / 180.0) for a in P.flo_ang]
        self.ucharmod = math.sqrt(sum(u * u for u in self.uchar))
        self.char_length = P.dia_phys
        self.maxvolfrac0 = info.maxvolfrac
        umeanslip = self.ucharmod / (1.0 - self.maxvolfrac0)
        self.t_conv = self.char_length / (umeanslip * (1.0 - self.maxvolfrac0))
        self.t_vis = (self.char_length * self.char_length) / P.vis
        self.t_diff = ((self.char_length * self.char_length) / (P.vis / P.pr_or_sc_nu)) if P.iscalon else LARGE_NUMBER
        d1 = P.lybyd * P.dia_phys
        self.dx = d1 / P.my
        self.voldom = (P.my * self.dx) * d1 * d1
        self.nbody = self.s.nbody
        self._open("dt_history", "".join("  " + h.rjust(17) for h in ("ISTEP", "DT", "#STEPS REQD", "CFL")) + "\n")
        for name in ("norm_drag", "norm_drag_chem", "drag_components"):
            self._open(name, None)

    def _path(self, name):
        return os.path.join(self.directory, "%s_%s.dat" % (self.run_name, name))

    def _open(self, name, header):
        with open(self._path(name), "w") as fh:
            if header:
                fh.write(header)

    def _append(self, name, text):
        with open(self._path(name), "a") as fh:
            fh.write(text)

    def advance(self, nsteps: int = 1) -> dict:
        rep = None
        for _ in range(nsteps):
            stage = getattr(self.s, "step_rks", None) or self.s.step
            for rks in range(1, self.itrmax + 1):
                rep = stage(rks)
            self.iglobstep += 1
            self._records(rep)
        return rep

    def _records(self, rep: dict):
        P = self.P
        t, dt = rep["t"], rep["dt"]
        # bcset records (boundary_condition.F90:849-870), last stage of the step
        c12 = (1.0 / 6.0 + 1.0 / 6.0) if self.itrmax == 3 else (0.5 + 0.5)
        mvf = self.maxvolfrac0
        tcol = [t / self.t_conv / (1.0 - mvf), t / self.t_vis, t / self.t_diff]
        nd = rep["norm_drag"]
        usact = np.zeros(3)
        nd_chem = 0.0
        if self.nbody:
            pres, visc, force, xc, vel = self.s.get_particles()
            for d in range(3):
                acc = 0.0
                for m in range(self.nbody):
                    acc = acc + float(vel[m, d])
                usact[d] = acc / self.nbody
            fchem = c12 * (pres + visc)
            avg = np.array([sum(float(v) for v in fchem[:, d]) / self.nbody for d in range(3)])
            nd_chem = math.sqrt(avg[0] ** 2 + avg[1] ** 2 + avg[2] ** 2)
            nf = 3.0 * math.pi * P.vis * ((rep["mixmeanslipmod"] + SMALL_NUMBER) if P.set_mpg else self.ucharmod) * self.char_length
            nd_chem = nd_chem / nf
        self._append("norm_drag", _line(tcol + [nd, nd] + list(usact) + [u / self.ucharmod for u in rep["ufmean"]], fortran_e))
        self._append("norm_drag_chem", _line(tcol + [nd_chem, nd_chem], fortran_e))
        norm_factor = (3.0 * math.pi * P.vis * (rep["mixmeanslipmod"] + SMALL_NUMBER) * self.char_length) * self.nbody
        mpg = rep["mpg"]
        mpg_avg = math.sqrt(mpg[0] * mpg[0] + mpg[1] * mpg[1] + mpg[2] * mpg[2])
        tdm = mpg_avg * self.voldom / norm_factor if norm_factor > 0 else 0.0
        td = rep["total_drag"]
        self._append("drag_components", _line([rep["pres_drag"], rep["visc_drag"], td, tdm, nd,
                                               abs(td - tdm) / (td + SMALL_NUMBER)], fortran_e))
        # driver record (dtibm_main_scal_flo.F90:460)
        tend = self.tend if self.tend is not None else t
        self._append("dt_history", _line([float(self.iglobstep), dt, (tend - t) / dt + float(self.iglobstep),
                                          self.uchar[0] * dt / self.dx], fortran_g))
