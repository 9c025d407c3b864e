"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (liboracle.so).

Imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg, and only as the checker or the timed CPU baseline.  The product
(``pureibm_ps2d_fd1d_b200``) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from pureibm_ps2d_fd1d_b200.abi import (pibm_params, pibm_particles, pibm_state_view,
                                        pibm_step_report, pibm_info)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "CXX=g++"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        vp = C.c_void_p
        L.orc_create.argtypes = [P(pibm_params), P(pibm_particles), P(vp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_destroy.restype = None
        L.orc_info.argtypes = [vp, P(pibm_info)]
        L.orc_step.argtypes = [vp, P(pibm_step_report)]
        L.orc_step_rks.argtypes = [vp, C.c_int, P(pibm_step_report)]
        L.orc_get_state.argtypes = [vp, P(pibm_state_view)]
        L.orc_set_state.argtypes = [vp, P(pibm_state_view)]
        L.orc_get_particles.argtypes = [vp] + [P(C.c_double)] * 5
        L.orc_get_if_rev.argtypes = [vp, P(C.c_uint8)]
        L.orc_get_fluid_mask.argtypes = [vp, P(C.c_uint8)]
        L.orc_get_geometry.argtypes = [vp, P(C.c_double), P(C.c_double)]
        L.orc_get_field.argtypes = [vp, C.c_int, P(C.c_double)]
        L.orc_get_scalar.argtypes = [vp, P(C.c_double), P(C.c_double), P(C.c_double)]
        L.orc_get_contacts.argtypes = [vp, C.c_int, P(C.c_int32), P(C.c_int32), P(C.c_int32)]
        L.orc_get_scalar_nl.argtypes = [vp, P(C.c_double)]
        L.orc_set_scalar.argtypes = [vp, P(C.c_double), P(C.c_double), P(C.c_double)]
        L.orc_set_desired_means.argtypes = [vp, P(C.c_double), P(C.c_double)]
        L.orc_get_frame.argtypes = [vp, P(C.c_double), P(C.c_double)]
        L.orc_set_frame.argtypes = [vp, P(C.c_double), P(C.c_double)]
        L.orc_ff2rc.argtypes = [C.c_int, C.c_int, C.c_int, P(C.c_double), P(C.c_double)]
        L.orc_ff2cr.argtypes = [C.c_int, C.c_int, C.c_int, P(C.c_double), P(C.c_double)]
        L.orc_cyclic_solve.argtypes = [C.c_int] + [P(C.c_double)] * 7
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_threads.restype = None
        L.orc_last_error.restype = C.c_char_p
        L.orc_adjoint.argtypes = [vp, C.c_int] + [P(C.c_double)] * 8
        L.orc_sizeof.argtypes = [C.c_int]
        L.orc_sizeof.restype = C.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def ff2rc(a: np.ndarray) -> np.ndarray:
    """a: real (nplanes, mz, my) C-order -> complex (nplanes, mz, my2)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    npl, mz, my = a.shape
    b = np.zeros((npl, mz, my // 2 + 1), dtype=np.complex128)
    rc = lib().orc_ff2rc(my, mz, npl, _dp(a), b.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0
    return b


def ff2cr(a: np.ndarray, my: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128)
    npl, mz, my2 = a.shape
    b = np.zeros((npl, mz, my), dtype=np.float64)
    rc = lib().orc_ff2cr(my, mz, npl, a.ctypes.data_as(C.POINTER(C.c_double)), _dp(b))
    assert rc == 0
    return b


def cyclic_solve(a, b, c, rr, ri):
    n = len(a)
    a, b, c, rr, ri = [np.ascontiguousarray(v, dtype=np.float64) for v in (a, b, c, rr, ri)]
    outr = np.zeros(n); outi = np.zeros(n)
    rc = lib().orc_cyclic_solve(n, _dp(a), _dp(b), _dp(c), _dp(rr), _dp(ri), _dp(outr), _dp(outi))
    return rc, outr, outi


class OracleSolver:
    """CPU oracle with the same surface as pureibm_ps2d_fd1d_b200.Solver."""

    def __init__(self, params: pibm_params, particles: pibm_particles):
        self._keep = (params, particles)
        h = C.c_void_p()
        rc = lib().orc_create(C.byref(params), C.byref(particles), C.byref(h))
        if rc != 0:
            raise RuntimeError("orc_create failed: %s" % lib().orc_last_error().decode())
        self.h = h
        info = pibm_info()
        lib().orc_info(self.h, C.byref(info))
        self.info = info
        self.nx, self.my, self.mz, self.my2 = info.nx, info.my, info.mz, info.my2
        self.nbody, self.nbnd = info.nbody, info.nbnd

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self) -> dict:
        """One full time step (every rks stage)."""
        rep = pibm_step_report()
        rc = lib().orc_step(self.h, C.byref(rep))
        if rc != 0:
            raise RuntimeError("orc_step failed with code %d" % rc)
        self.last_report = rep.as_dict()
        return self.last_report

    @property
    def params(self):
        return self._keep[0]

    def get_scalar(self) -> dict:
        out = get_scalar(self)
        nl = np.zeros_like(out["phif"])
        if lib().orc_get_scalar_nl(self.h, nl.ctypes.data_as(C.POINTER(C.c_double))) != 0:
            raise RuntimeError("oracle has no scalar (ISCALON = 0)")
        out["nlphif"] = nl
        return out

    def set_desired_means(self, usmean_des, ufmean_des):
        a = np.ascontiguousarray(usmean_des, dtype=np.float64)
        b = np.ascontiguousarray(ufmean_des, dtype=np.float64)
        lib().orc_set_desired_means(self.h, _dp(a), _dp(b))

    def get_frame(self):
        fv, fp = np.zeros(3), np.zeros(3)
        lib().orc_get_frame(self.h, _dp(fv), _dp(fp))
        return fv, fp

    def set_frame(self, frame_vel, frame_pos):
        a = np.ascontiguousarray(frame_vel, dtype=np.float64)
        b = np.ascontiguousarray(frame_pos, dtype=np.float64)
        lib().orc_set_frame(self.h, _dp(a), _dp(b))

    def set_scalar(self, phif, nlphif, heat_ratio, heat_ratio_old):
        a = np.ascontiguousarray(phif, dtype=np.complex128)
        b = np.ascontiguousarray(nlphif, dtype=np.complex128)
        r = np.array([heat_ratio, heat_ratio_old], dtype=np.float64)
        if lib().orc_set_scalar(self.h, a.ctypes.data_as(C.POINTER(C.c_double)),
                                b.ctypes.data_as(C.POINTER(C.c_double)), _dp(r)) != 0:
            raise RuntimeError("oracle has no scalar (ISCALON = 0)")

    def step_rks(self, rks: int) -> dict:
        """One stage rks of the driver's loop."""
        rep = pibm_step_report()
        rc = lib().orc_step_rks(self.h, int(rks), C.byref(rep))
        if rc != 0:
            raise RuntimeError("orc_step_rks failed with code %d" % rc)
        return rep.as_dict()

    def get_state(self):
        nx, my2, mz = self.nx, self.my2, self.mz
        u = np.zeros((3, mz, my2, nx + 1), dtype=np.complex128)   # Fortran (nx+1,my2,mz,3) viewed C-order
        nl = np.zeros_like(u)
        p = np.zeros((mz, my2, nx), dtype=np.complex128)
        s = pibm_state_view()
        s.u = u.ctypes.data_as(C.POINTER(C.c_double))
        s.nl = nl.ctypes.data_as(C.POINTER(C.c_double))
        s.p = p.ctypes.data_as(C.POINTER(C.c_double))
        lib().orc_get_state(self.h, C.byref(s))
        return dict(u=u, nl=nl, p=p, umean=np.array(s.umean[:]), mpg=np.array(s.mpg[:]),
                    ufmean=np.array(s.ufmean[:]), t=s.t, dt=s.dt, cf=s.cf)

    def set_state(self, st):
        s = pibm_state_view()
        u = np.ascontiguousarray(st["u"], dtype=np.complex128)
        nl = np.ascontiguousarray(st["nl"], dtype=np.complex128)
        p = np.ascontiguousarray(st["p"], dtype=np.complex128)
        s.u = u.ctypes.data_as(C.POINTER(C.c_double))
        s.nl = nl.ctypes.data_as(C.POINTER(C.c_double))
        s.p = p.ctypes.data_as(C.POINTER(C.c_double))
        for d in range(3):
            s.umean[d] = st["umean"][d]; s.mpg[d] = st["mpg"][d]; s.ufmean[d] = st["ufmean"][d]
        s.t, s.dt, s.cf = st["t"], st["dt"], st["cf"]
        lib().orc_set_state(self.h, C.byref(s))

    def adjoint(self, nsteps: int, direction=(1.0, 0.0, 0.0), state_grad: bool = False):
        """K = nsteps AB2 steps from the current state and the discrete
        adjoint of J = (1/K) sum_n e . sum_m (pres_m + visc_m).  Returns
        dict(J, g_xc (nbody,3), g_mpg (3,)) and, with state_grad, lambda of the
        initial u, p, nl (state layout) and umean.  The solver ends at the state
        after K steps."""
        e = np.ascontiguousarray(direction, dtype=np.float64)
        J = C.c_double()
        g = np.zeros(3 * self.nbody)
        gm = np.zeros(3)
        st = self.get_state() if state_grad else None
        lu = np.zeros_like(st["u"]) if state_grad else None
        lp = np.zeros_like(st["p"]) if state_grad else None
        lnl = np.zeros_like(st["nl"]) if state_grad else None
        lum = np.zeros(3) if state_grad else None
        cp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
        rc = lib().orc_adjoint(self.h, int(nsteps), _dp(e), C.byref(J), _dp(g), _dp(gm), cp(lu), cp(lp), cp(lnl), cp(lum))
        if rc != 0:
            raise RuntimeError("orc_adjoint failed with code %d: %s" % (rc, lib().orc_last_error().decode()))
        out = dict(J=J.value, g_xc=g.reshape(3, self.nbody).T.copy(), g_mpg=gm)
        if state_grad:
            out.update(lu=lu, lp=lp, lnl=lnl, lumean=lum)
        return out

    def get_particles(self):
        n = self.nbody
        out = [np.zeros(3 * n) for _ in range(5)]
        lib().orc_get_particles(self.h, *[_dp(a) for a in out])
        return [a.reshape(3, n).T.copy() for a in out]   # pres, visc, force, xc, vel as (nbody,3)

    def get_if_rev(self):
        out = np.zeros(self.nbnd * self.nbody, dtype=np.uint8)
        lib().orc_get_if_rev(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out.reshape(self.nbody, self.nbnd)

    def get_fluid_mask(self):
        out = np.zeros(self.nx * self.my * self.mz, dtype=np.uint8)
        lib().orc_get_fluid_mask(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out.reshape(self.mz, self.my, self.nx)

    def get_geometry(self):
        b = np.zeros(3 * self.nbnd); c = np.zeros(3 * self.nbnd)
        lib().orc_get_geometry(self.h, _dp(b), _dp(c))
        return b.reshape(self.nbnd, 3), c.reshape(self.nbnd, 3)

    def get_field(self, which: int):
        nx, my, mz, my2 = self.nx, self.my, self.mz, self.my2
        if which in (0, 1, 2, 3, 4, 5):
            out = np.zeros((3, mz, my, nx + 1))
        elif which == 6:
            out = np.zeros((mz, my, nx))
        elif which == 7:
            out = np.zeros((3, mz, my, nx))
        elif which == 8:
            out = np.zeros((3, mz, my2, nx + 1), dtype=np.complex128)
        else:
            raise ValueError(which)
        lib().orc_get_field(self.h, which, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out


def get_scalar(solver) -> dict:
    """Scalar state of an OracleSolver: phif complex (mz, my2, nx+1) (the
    reference's (nx+1,my2,mz) array viewed in C order), per-sphere surface
    flux, heat_ratio, heat_ratio_old and the Nusselt number."""
    nx, my2, mz = solver.nx, solver.my2, solver.mz
    phif = np.zeros((mz, my2, nx + 1), dtype=np.complex128)
    flux = np.zeros(max(solver.nbody, 1))
    ratios = np.zeros(3)
    rc = lib().orc_get_scalar(solver.h, phif.ctypes.data_as(C.POINTER(C.c_double)), _dp(flux), _dp(ratios))
    if rc != 0:
        raise RuntimeError("oracle has no scalar (ISCALON = 0)")
    return dict(phif=phif, flux_body=flux[:solver.nbody], heat_ratio=ratios[0], heat_ratio_old=ratios[1],
                nusselt=ratios[2])


MAXNEIGHBORS = 37   # MN + 1 + NWALLS (collision_mod.F90:508)


def get_contacts(solver, maxn: int = MAXNEIGHBORS) -> dict:
    """DEM lists of an OracleSolver with moving particles, in the reference
    layout (nbody, maxn) read as arrays [column][particle]: column 0 the count,
    then 1-based particle numbers (-1 fill; PV: flags, 0 fill)."""
    n = solver.nbody
    out = {k: np.zeros((maxn, n), dtype=np.int32) for k in ("neighbours", "pn", "pv")}
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    rc = lib().orc_get_contacts(solver.h, maxn, ip(out["neighbours"]), ip(out["pn"]), ip(out["pv"]))
    if rc != 0:
        raise RuntimeError("oracle has no DEM lists (IMOVE = 0) or maxn too small")
    return out
