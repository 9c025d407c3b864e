"""Restart files in the reference's format (SRC/FLO/restart_funcs.F90:69-614).

The reference writes Fortran unformatted sequential files (one record per
WRITE: a 4-byte length marker, the data, the marker again) and alternates
between two sets, RUN_NAME_{u,nl,p,scal}_1.rst and _2.rst, recording the set
last written in the formatted file RUN_NAME_RESTART; RUN_NAME_sphere_config.rst
holds the particles (and, for moving particles, RUN_NAME_sphere_config_N.rst
the moved ones plus the frame motion frame_vel, frame_pos).  Writing a set
deletes the other one.  A moving run resumes like the reference's: from the
moved positions and velocities and the frame motion, its soft-sphere contact
lists rebuilt by the neighbour search of a new run (the reference keeps no
contact history in its restart files).

    write_restart(solver, directory, run_name)        # next set (1 or 2)
    data = read_restart(directory, run_name, solver)  # the set named in _RESTART
    apply_restart(solver, data)                       # pibm_set_state [+ scalar]
    s = resume(params, directory, run_name)           # a new Solver from the files

Only the serial layout (PARALLEL = 0) is read and written.  Quantities that
this engine does not keep are written with neutral values and listed in
NOT_KEPT; they are the reference's convergence histories and do not enter
the step.
"""
from __future__ import annotations

import os
import struct
from typing import Dict, Optional

import numpy as np

NERR_STEPS = 100   # nerr_steps (initialize_flo.F90)
NOT_KEPT = ("ferror_array (written as the last ferror followed by 1.0)",
            "grant_error, grant_old, grant_array (moving particles; written as 1.0, 0.0, 1.0)",
            "nu_error, nu_error_array (scalar; written as 1.0)")


# ---------------------------------------------------------------------------
# Fortran unformatted sequential records (gfortran: 4-byte markers; records
# above 2 GiB are split into subrecords whose leading marker is negative
# when another subrecord follows).
# ---------------------------------------------------------------------------
class RecordWriter:
    def __init__(self, path: str):
        self.fh = open(path, "wb")

    def write(self, *items):
        data = b"".join(np.ascontiguousarray(x).tobytes() if isinstance(x, np.ndarray) else x for x in items)
        if len(data) > 2 ** 31 - 1:
            raise ValueError("record above 2 GiB")
        n = struct.pack("<i", len(data))
        self.fh.write(n + data + n)

    def close(self):
        self.fh.close()


class RecordReader:
    def __init__(self, path: str):
        self.fh = open(path, "rb")

    def read(self) -> bytes:
        out = []
        while True:
            head = self.fh.read(4)
            if len(head) < 4:
                raise EOFError("unexpected end of restart file")
            m = struct.unpack("<i", head)[0]
            out.append(self.fh.read(abs(m)))
            self.fh.read(4)
            if m >= 0:
                return b"".join(out)

    def f64(self, n: Optional[int] = None):
        a = np.frombuffer(self.read(), dtype="<f8")
        return a if n is None else a[:n]

    def i32(self):
        return np.frombuffer(self.read(), dtype="<i4")

    def c128(self, shape):
        return np.frombuffer(self.read(), dtype="<c16").reshape(shape).copy()

    def close(self):
        self.fh.close()


def _f64(*v):
    return np.array(v, dtype="<f8")


def _i32(*v):
    return np.array(v, dtype="<i4")


def _path(directory, run_name, name, count=None):
    return os.path.join(directory, "%s_%s%s.rst" % (run_name, name, "" if count is None else "_%d" % count))


def _params(solver) -> dict:
    p = getattr(solver, "params", None) or solver._keep[0]
    return {f: getattr(p, f) for f, _ in p._fields_}


def _initial_velocities(solver, nbody):
    parts = getattr(solver, "particles", None) or getattr(solver, "_parts", None)
    vel = getattr(parts, "vel_f", None)
    return np.zeros((nbody, 3)) if vel is None else np.asarray(vel).reshape(3, nbody).T


def _desired_means(solver, p):
    """usmean_des and ufmean_des as initflo sets them (initialize_flo.F90:
    277-353): the serial mean of the initial particle velocities and
    uchar/(1 - maxvolfrac)."""
    nbody = solver.nbody
    vel0 = _initial_velocities(solver, nbody)
    usd = np.zeros(3)
    for d in range(3):
        acc = 0.0
        for m in range(nbody):
            acc = acc + float(vel0[m, d])
        usd[d] = acc / nbody if nbody else 0.0
    uchar = (p["re"] * p["vis"]) / p["dia_phys"]
    uc = np.array([uchar * np.cos(np.pi * a / 180.0) for a in p["flo_ang"]])
    return usd, uc / (1.0 - solver.info.maxvolfrac)


def _domain(p):
    """DOML(1:3) for the 'default' input (initialize_flo.F90:1562-1590)."""
    d1 = p["lybyd"] * p["dia_phys"]
    dx = d1 / p["my"]
    return np.array([p["my"] * dx, d1, d1])


def next_count(directory: str, run_name: str) -> int:
    """The set the next write goes to: 1 after 2 (or when none exists), else 2."""
    path = os.path.join(directory, run_name + "_RESTART")
    try:
        with open(path) as fh:
            last = int(fh.read().split()[0])
    except (OSError, ValueError, IndexError):
        return 1
    return 1 if last == 2 else 2


def write_restart(solver, directory: str, run_name: str, count: Optional[int] = None,
                  nerr_steps: int = NERR_STEPS) -> int:
    """Write the restart set `count` (default: the next one) from a Solver
    (or any object with the same get_state / get_particles / info surface)
    and delete the other set, as save_unformatted does.  Returns the set."""
    os.makedirs(directory, exist_ok=True)
    count = count or next_count(directory, run_name)
    p = _params(solver)
    st = solver.get_state()
    rep = getattr(solver, "last_report", None) or {}
    nbody = solver.nbody
    pres, visc, force, xc, vel = solver.get_particles() if nbody else [np.zeros((0, 3))] * 5
    rad = np.full(nbody, 0.5 * p["my"] / p["lybyd"])
    doml = _domain(p)
    imove = p["imove"] == 1
    # particles: RUN_NAME_sphere_config.rst (and the moved ones for IMOVE = 1)
    usd, ufd = _desired_means(solver, p)
    char_length = p["dia_phys"]
    for name in ("sphere_config", "sphere_config_%d" % count) if imove else ("sphere_config",):
        w = RecordWriter(os.path.join(directory, "%s_%s.rst" % (run_name, name)))
        w.write(_i32(nbody))
        w.write(_i32(1))                                   # nphases
        w.write(_i32(nbody))                               # npart of the phase
        w.write(_f64(p["dia_phys"]))                        # phase diameter
        w.write(_f64(*doml))
        if name != "sphere_config":
            w.write(_i32(1))                                # move_particles = .TRUE.
        w.write(_f64(char_length))
        w.write(np.asfortranarray(xc, dtype="<f8").ravel(order="F"))
        w.write(rad.astype("<f8"))
        w.write(np.asfortranarray(vel, dtype="<f8").ravel(order="F"))
        if name != "sphere_config":
            fv, fp = solver.get_frame()
            w.write(np.asarray(fv, dtype="<f8"))
            w.write(np.asarray(fp, dtype="<f8"))
        w.close()
    # u: scalars, convergence histories, the velocity field
    ferror = float(rep.get("ferror", 1.0))
    fold = float(rep.get("norm_drag", 0.0))
    w = RecordWriter(_path(directory, run_name, "u", count))
    w.write(_f64(st["t"], st["dt"]))
    w.write(_f64(*st["umean"]))
    w.write(_f64(*usd))
    w.write(_f64(*ufd))
    w.write(_f64(st["cf"]))
    w.write(_i32(nerr_steps))
    w.write(_f64(ferror, fold))
    hist = np.ones(nerr_steps)
    hist[0] = ferror
    w.write(hist.astype("<f8"))
    w.write(_f64(ferror, fold))                             # the phase's ferror, fold
    if imove:
        w.write(_f64(1.0, 0.0))
    w.write(hist.astype("<f8"))
    if imove:
        w.write(np.ones(nerr_steps, dtype="<f8"))
    w.write(st["u"].astype("<c16"))
    w.close()
    w = RecordWriter(_path(directory, run_name, "nl", count))
    w.write(st["nl"].astype("<c16"))
    w.close()
    w = RecordWriter(_path(directory, run_name, "p", count))
    w.write(_f64(*st["mpg"]))
    w.write(st["p"].astype("<c16"))
    w.close()
    if p["iscalon"]:
        sc = solver.get_scalar()
        w = RecordWriter(_path(directory, run_name, "scal", count))
        w.write(_f64(1.0, float(sc["nusselt"])))            # nu_error, nu_old
        w.write(np.ones(nerr_steps, dtype="<f8"))
        w.write(sc["phif"].astype("<c16"))
        w.write(sc["nlphif"].astype("<c16"))
        w.write(np.full(nbody, p["phisurf"], dtype="<f8"))  # phisurfall(1:nbody, 1)
        phirmean = float(np.mean(sc["phif"][0, 0, :-1].real))
        w.write(_f64(phirmean, sc["heat_ratio"], sc["heat_ratio_old"]))
        w.close()
    with open(os.path.join(directory, run_name + "_RESTART"), "w") as fh:
        fh.write(" %d\n" % count)
    other = 2 if count == 1 else 1
    for name in ("u", "nl", "p", "scal") + (("sphere_config",) if imove else ()):
        path = _path(directory, run_name, name, other)
        if os.path.exists(path):
            os.remove(path)
    return count


def read_restart(directory: str, run_name: str, nx: int, my: int, mz: int, imove: bool = False,
                 iscalon: bool = False, count: Optional[int] = None) -> Dict:
    """Read the restart set named in RUN_NAME_RESTART (or `count`): the
    particles, the scalars and fields of read_unformatted, in the
    reference's layouts (u (nx+1,my2,mz,3) as a C-order (3,mz,my2,nx+1)
    array, p (nx,my2,mz) as (mz,my2,nx))."""
    if count is None:
        with open(os.path.join(directory, run_name + "_RESTART")) as fh:
            count = int(fh.read().split()[0])
    my2 = my // 2 + 1
    out: Dict = {"count": count}
    name = "sphere_config_%d" % count if imove else "sphere_config"
    r = RecordReader(os.path.join(directory, "%s_%s.rst" % (run_name, name)))
    nbody = int(r.i32()[0])
    nph = int(r.i32()[0])
    out["npart"] = [int(r.i32()[0]) for _ in range(nph)]
    out["phase_dia"] = [float(r.f64()[0]) for _ in range(nph)]
    out["doml"] = r.f64(3)
    if imove:
        out["move_particles"] = bool(r.i32()[0])
    out["char_length"] = float(r.f64()[0])
    out["xc"] = r.f64(3 * nbody).reshape(3, nbody).T.copy()
    out["radbdy"] = r.f64(nbody).copy()
    out["velbdy"] = r.f64(3 * nbody).reshape(3, nbody).T.copy()
    if imove:
        out["frame_vel"] = r.f64(3).copy()
        out["frame_pos"] = r.f64(3).copy()
    out["nbody"] = nbody
    r.close()
    r = RecordReader(_path(directory, run_name, "u", count))
    out["t"], out["dt"] = (float(v) for v in r.f64(2))
    out["umean"] = r.f64(3).copy()
    out["usmean_des"] = r.f64(3).copy()
    out["ufmean_des"] = r.f64(3).copy()
    out["cf"] = float(r.f64()[0])
    nerr = int(r.i32()[0])
    out["ferror"], out["fold"] = (float(v) for v in r.f64(2))
    out["ferror_array"] = r.f64(nerr).copy()
    for _ in range(nph):
        r.read()
        if imove:
            r.read()
    for _ in range(nph):
        r.read()
        if imove:
            r.read()
    out["u"] = r.c128((3, mz, my2, nx + 1))
    r.close()
    r = RecordReader(_path(directory, run_name, "nl", count))
    out["nl"] = r.c128((3, mz, my2, nx + 1))
    r.close()
    r = RecordReader(_path(directory, run_name, "p", count))
    out["mpg"] = r.f64(3).copy()
    out["p"] = r.c128((mz, my2, nx))
    r.close()
    if iscalon:
        r = RecordReader(_path(directory, run_name, "scal", count))
        r.read()
        r.read()
        out["phif"] = r.c128((mz, my2, nx + 1))
        out["nlphif"] = r.c128((mz, my2, nx + 1))
        out["phisurfall"] = r.f64(nbody).copy()
        v = r.f64(3)
        out["phirmean"], out["heat_ratio"], out["heat_ratio_old"] = (float(x) for x in v)
        r.close()
    return out


def apply_restart(solver, data: Dict):
    """Load a read_restart() set into a solver created for the same run."""
    solver.set_state({"u": data["u"], "nl": data["nl"], "p": data["p"], "umean": data["umean"],
                      "mpg": data["mpg"], "t": data["t"], "dt": data["dt"], "cf": data["cf"],
                      "ufmean": np.zeros(3)})
    solver.set_desired_means(data["usmean_des"], data["ufmean_des"])
    if "frame_vel" in data:
        solver.set_frame(data["frame_vel"], data["frame_pos"])
    if "phif" in data:
        solver.set_scalar(data["phif"], data["nlphif"], data["heat_ratio"], data["heat_ratio_old"])


def resume(params, directory: str, run_name: str, solver_cls=None):
    """A new solver for `params` with the particles of the restart set (the
    moved ones for IMOVE = 1) and its state loaded."""
    from . import Solver, config
    solver_cls = solver_cls or Solver
    P = params if not isinstance(params, dict) else config.make_params(params)
    my = P.my
    data = read_restart(directory, run_name, my, my, P.mz or my, imove=P.imove == 1, iscalon=bool(P.iscalon))
    s = solver_cls(P, data["xc"], data["velbdy"])
    apply_restart(s, data)
    return s
