"""B200-native PUReIBM-PS2D-FD1D time-step engine (host side).

The engine itself is ``_lib/libpibm.so`` (CUDA, sm_100a), reached through the
C ABI of ``include/pibm.h``.  This package is the host-side mirror of the
reference's step boundary: ``Solver.step()`` is one iteration of the driver's
rks loop (SRC/FLO/dtibm_main_scal_flo.F90:426-527), i.e. compute_new_timestep
-> nonlinear -> bcset -> velstep, executed on the GPU.  There is no CPU
fallback: if the library cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import abi
from .abi import pibm_params, pibm_state_view, pibm_step_report, pibm_info, pibm_adjoint_report
from . import config

__all__ = ["Solver", "Batch", "load_library", "ff2rc", "ff2cr", "config", "abi", "PibmError"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libpibm.so")
_lib = None


class PibmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s (%d): %s" % (abi.ERROR_NAMES.get(code, "PIBM_ERR"), code, msg))
        self.code = code


def load_library():
    """Load the in-tree CUDA engine; raises if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libpibm.so not built (run python -m pureibm_ps2d_fd1d_b200.build): " + LIB_PATH)
        _lib = abi.bind(C.CDLL(LIB_PATH))
    return _lib


def _check(rc: int):
    if rc != 0:
        raise PibmError(rc, load_library().pibm_last_error().decode())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def ff2rc(a: np.ndarray) -> np.ndarray:
    """Reference ff2rc on the GPU: real (nplanes, mz, my) -> complex (nplanes, mz, my/2+1)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    npl, mz, my = a.shape
    b = np.zeros((npl, mz, my // 2 + 1), dtype=np.complex128)
    _check(load_library().pibm_ff2rc(my, mz, npl, _dp(a), b.ctypes.data_as(C.POINTER(C.c_double))))
    return b


def ff2cr(a: np.ndarray, my: int) -> np.ndarray:
    """Reference ff2cr on the GPU: complex (nplanes, mz, my/2+1) -> real (nplanes, mz, my)."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    npl, mz, _ = a.shape
    b = np.zeros((npl, mz, my), dtype=np.float64)
    _check(load_library().pibm_ff2cr(my, mz, npl, a.ctypes.data_as(C.POINTER(C.c_double)), _dp(b)))
    return b


class Solver:
    """One run on the current CUDA device (one handle of the C ABI)."""

    def __init__(self, params, xc: Optional[np.ndarray] = None, vel: Optional[np.ndarray] = None):
        lib = load_library()
        self.params = params if isinstance(params, pibm_params) else config.make_params(params)
        self.particles = config.Particles(np.zeros((0, 3)) if xc is None else xc, vel)
        h = C.c_void_p()
        _check(lib.pibm_create(C.byref(self.params), C.byref(self.particles.struct), C.byref(h)))
        self._owned = True
        self._attach(h)

    @classmethod
    def _member(cls, h, owner):
        """A view of a batch member's handle (owned and freed by the batch)."""
        s = cls.__new__(cls)
        s._owned = False
        s._owner = owner
        s._attach(h)
        return s

    def _attach(self, h):
        lib = load_library()
        self.h = h
        self.last_report = None
        info = pibm_info()
        _check(lib.pibm_info_get(self.h, C.byref(info)))
        self.info = info
        self.nx, self.my, self.mz, self.my2 = info.nx, info.my, info.mz, info.my2
        self.nbody, self.nbnd = info.nbody, info.nbnd

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", False):
                load_library().pibm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the step boundary ----------------------------------------------------
    def step(self, rks: int = 1) -> dict:
        """compute_new_timestep -> nonlinear -> bcset -> velstep (one rks iteration)."""
        rep = pibm_step_report()
        _check(load_library().pibm_step(self.h, rks, C.byref(rep)))
        self.last_report = rep.as_dict()
        return self.last_report

    def run(self, nsteps: int) -> dict:
        """nsteps steps replayed from CUDA graphs, diagnostics of the last one."""
        rep = pibm_step_report()
        _check(load_library().pibm_run(self.h, int(nsteps), C.byref(rep)))
        self.last_report = rep.as_dict()
        return self.last_report

    # -- state in the reference layout -------------------------------------------
    def get_state(self) -> dict:
        nx, my2, mz = self.nx, self.my2, self.mz
        u = np.zeros((3, mz, my2, nx + 1), dtype=np.complex128)
        nl = np.zeros_like(u)
        p = np.zeros((mz, my2, nx), dtype=np.complex128)
        s = pibm_state_view()
        s.u, s.nl, s.p = (a.ctypes.data_as(C.POINTER(C.c_double)) for a in (u, nl, p))
        _check(load_library().pibm_get_state(self.h, C.byref(s)))
        return dict(u=u, nl=nl, p=p, umean=np.array(s.umean[:]), mpg=np.array(s.mpg[:]),
                    ufmean=np.array(s.ufmean[:]), t=s.t, dt=s.dt, cf=s.cf)

    def set_state(self, st: dict):
        s = pibm_state_view()
        keep = []
        for name in ("u", "nl", "p"):
            if st.get(name) is not None:
                a = np.ascontiguousarray(st[name], dtype=np.complex128)
                keep.append(a)
                setattr(s, name, a.ctypes.data_as(C.POINTER(C.c_double)))
        for d in range(3):
            s.umean[d] = st["umean"][d]; s.mpg[d] = st["mpg"][d]; s.ufmean[d] = st.get("ufmean", np.zeros(3))[d]
        s.t, s.dt, s.cf = st["t"], st["dt"], st["cf"]
        _check(load_library().pibm_set_state(self.h, C.byref(s)))

    def get_particles(self):
        """pres, visc, force, xc, vel as (nbody, 3) arrays."""
        n = self.nbody
        out = [np.zeros(3 * n) for _ in range(5)]
        _check(load_library().pibm_get_particles(self.h, *[_dp(a) for a in out]))
        return [a.reshape(3, n).T.copy() for a in out]

    def get_contacts(self, maxn: int = 37) -> dict:
        """Moving particles: the DEM lists NEIGHBOURS, PN, PV in the reference
        layout (nbody, maxn), returned as arrays [column][particle] (column 0
        the count, then 1-based particle numbers; -1 / 0 fill)."""
        n = self.nbody
        out = {k: np.zeros((maxn, n), dtype=np.int32) for k in ("neighbours", "pn", "pv")}
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        _check(load_library().pibm_get_contacts(self.h, maxn, ip(out["neighbours"]), ip(out["pn"]), ip(out["pv"])))
        return out

    def get_scalar(self) -> dict:
        """Passive scalar: phif complex (mz, my2, nx+1) (the reference's
        (nx+1,my2,mz) array in C order), per-sphere surface flux, heat_ratio,
        heat_ratio_old and the Nusselt number."""
        nx, my2, mz = self.nx, self.my2, self.mz
        phif = np.zeros((mz, my2, nx + 1), dtype=np.complex128)
        flux = np.zeros(max(self.nbody, 1))
        ratios = np.zeros(3)
        _check(load_library().pibm_get_scalar(self.h, phif.ctypes.data_as(C.POINTER(C.c_double)), _dp(flux), _dp(ratios)))
        nlphif = np.zeros_like(phif)
        _check(load_library().pibm_get_scalar_nl(self.h, nlphif.ctypes.data_as(C.POINTER(C.c_double))))
        return dict(phif=phif, nlphif=nlphif, flux_body=flux[:self.nbody], heat_ratio=ratios[0],
                    heat_ratio_old=ratios[1], nusselt=ratios[2])

    def adjoint(self, nsteps: int, direction=(1.0, 0.0, 0.0), checkpoint_every: int = 20) -> dict:
        """nsteps steps from the current state and the discrete adjoint of
        J = (1/K) sum_n e . sum_m (pres_m + visc_m) (pibm_adjoint_run).
        Returns dict(J, g_xc (nbody,3), g_mpg (3,), forward_ms, reverse_ms)."""
        lib = load_library()
        e = np.ascontiguousarray(direction, dtype=np.float64)
        g = np.zeros(3 * self.nbody)
        gm = np.zeros(3)
        rep = pibm_adjoint_report()
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        _check(lib.pibm_adjoint_run(self.h, int(nsteps), int(checkpoint_every), dp(e), dp(g), dp(gm), C.byref(rep)))
        return dict(J=rep.J, g_xc=g.reshape(3, self.nbody).T.copy(), g_mpg=gm, forward_ms=rep.forward_ms,
                    reverse_ms=rep.reverse_ms, adjoint_kernels_per_step=rep.adjoint_kernels_per_step)

    def tuning(self) -> dict:
        """x-line tile width chosen by the autotuner and the candidates' times."""
        lt = C.c_int32()
        ms = np.zeros(2)
        _check(load_library().pibm_get_tuning(self.h, C.byref(lt), ms.ctypes.data_as(C.POINTER(C.c_double))))
        return dict(lines_per_cta=lt.value, lines_ms={4: ms[0], 8: ms[1]})

    def set_tuning(self, lines_per_cta: int):
        _check(load_library().pibm_set_tuning(self.h, int(lines_per_cta)))

    # host-driven reverse sweep (pibm_adjoint_begin / _step / _end)
    def adjoint_begin(self, nsteps: int, direction=(1.0, 0.0, 0.0)):
        e = np.ascontiguousarray(direction, dtype=np.float64)
        _check(load_library().pibm_adjoint_begin(self.h, int(nsteps), e.ctypes.data_as(C.POINTER(C.c_double))))

    def adjoint_step(self):
        """Reverse step n (n = K, K-1, ..., 1); the solver must hold the state before step n."""
        _check(load_library().pibm_adjoint_step(self.h))

    def adjoint_end(self) -> dict:
        g = np.zeros(3 * self.nbody)
        gm = np.zeros(3)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        _check(load_library().pibm_adjoint_end(self.h, dp(g), dp(gm)))
        return dict(g_xc=g.reshape(3, self.nbody).T.copy(), g_mpg=gm)

    def set_desired_means(self, usmean_des, ufmean_des):
        """usmean_des / ufmean_des of a restarted run."""
        a = np.ascontiguousarray(usmean_des, dtype=np.float64)
        b = np.ascontiguousarray(ufmean_des, dtype=np.float64)
        _check(load_library().pibm_set_desired_means(self.h, _dp(a), _dp(b)))

    def get_surface_points(self) -> np.ndarray:
        """(nbnd, 3) unit directions of the surface quadrature points."""
        out = np.zeros((self.info.nbnd, 3))
        _check(load_library().pibm_get_surface_points(self.h, _dp(out)))
        return out

    def get_frame(self):
        """frame_vel(3), frame_pos(3) of a moving-particle run (0 and 1 for fixed spheres)."""
        fv, fp = np.zeros(3), np.zeros(3)
        _check(load_library().pibm_get_frame(self.h, _dp(fv), _dp(fp)))
        return fv, fp

    def set_frame(self, frame_vel, frame_pos):
        """Frame motion of a restarted moving-particle run."""
        a = np.ascontiguousarray(frame_vel, dtype=np.float64)
        b = np.ascontiguousarray(frame_pos, dtype=np.float64)
        _check(load_library().pibm_set_frame(self.h, _dp(a), _dp(b)))

    def set_scalar(self, phif, nlphif, heat_ratio: float, heat_ratio_old: float):
        """Scalar restart: phif and the last step's nlphif as (mz, my2, nx+1)."""
        a = np.ascontiguousarray(phif, dtype=np.complex128)
        b = np.ascontiguousarray(nlphif, dtype=np.complex128)
        r = np.array([heat_ratio, heat_ratio_old], dtype=np.float64)
        _check(load_library().pibm_set_scalar(self.h, a.ctypes.data_as(C.POINTER(C.c_double)),
                                              b.ctypes.data_as(C.POINTER(C.c_double)), _dp(r)))

    def get_if_rev(self) -> np.ndarray:
        out = np.zeros(self.nbnd * self.nbody, dtype=np.uint8)
        _check(load_library().pibm_get_if_rev(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out.reshape(self.nbody, self.nbnd)

    def get_fluid_mask(self) -> np.ndarray:
        out = np.zeros(self.nx * self.my * self.mz, dtype=np.uint8)
        _check(load_library().pibm_get_fluid_mask(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out.reshape(self.mz, self.my, self.nx)


class Batch:
    """Independent realizations (e.g. a multiple-independent-simulation
    ensemble) stepped together: one CUDA graph launch per step; members of one
    grid size with fixed spheres share each kernel launch, the others run as
    concurrent branches (pibm_batch_*)."""

    def __init__(self, members):
        """members: list of (params, centres) pairs, as config.mis_ensemble makes them."""
        lib = load_library()
        n = len(members)
        if n == 0:
            raise ValueError("empty batch")
        self._params = (pibm_params * n)(*[p if isinstance(p, pibm_params) else config.make_params(p)
                                            for p, xc in members])
        self._parts = [config.Particles(np.asarray(xc)) for _, xc in members]
        parts = (abi.pibm_particles * n)(*[pp.struct for pp in self._parts])
        h = C.c_void_p()
        _check(lib.pibm_batch_create(n, self._params, parts, C.byref(h)))
        self.h = h
        self.members = [Solver._member(C.c_void_p(lib.pibm_batch_member(h, i)), self) for i in range(n)]

    def run(self, nsteps: int):
        _check(load_library().pibm_batch_run(self.h, int(nsteps)))

    def time(self, nsteps: int, sequential: bool, fused: bool = True) -> float:
        """Device milliseconds of nsteps steps of every member: the plain
        per-realization loop (sequential) or the batch graph, with members of
        one grid size sharing launches (fused) or each member its own branch."""
        ms = C.c_double()
        mode = 1 if sequential else (0 if fused else 2)
        _check(load_library().pibm_batch_time(self.h, int(nsteps), mode, C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            for m in self.members:
                m.h = None
            load_library().pibm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
