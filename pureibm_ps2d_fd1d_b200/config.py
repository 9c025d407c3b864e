"""Run configuration: the reference's input files and the seeded workloads.

* ``default_params`` restates ``set_default`` (SRC/FLO/initialize.F90:73-271)
  for the keys the step uses.
* ``read_floparam`` reads a ``RUN_NAME_floparam.in`` (Fortran namelists
  FLOANDGRID, PART_PROPT, FLAGS, ... read in ``read_nmls``,
  initialize.F90:274-359) into the same dictionary, with the reference's
  group order and variable lists enforced.
* ``read_sphr_center`` reads ``RUN_NAME_sphr_center.inp`` like the
  ``input_type='default'`` branch (initialize_flo.F90:1485-1590): line 1 is
  skipped, columns are x y z r in diameters, positions are scaled by DBYDX and
  the radius column is ignored.  The reference's first pass over that file
  never increments ``nbody`` (initialize_flo.F90:1494-1503), so the reference
  itself loads no sphere from it; this reader returns every row.
* ``single_sphere`` / ``random_array`` / ``moving_suspension`` build the
  seeded synthetic workloads (fixed sphere at the box centre; random
  sequential addition followed by hard-sphere Monte Carlo moves).
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import Dict, Optional

import numpy as np

from .abi import pibm_params, pibm_particles, PIBM_SCHEME_CENTER, PIBM_SCHEME_UPWIND, \
    PIBM_LIMITER_NONE, PIBM_LIMITER_MINMOD


def default_params() -> Dict:
    """Reference defaults (initialize.F90:73-271) for the keys the step reads."""
    return dict(
        my=0, mz=0, lybyd=None, dbydx=None, dia_phys=1.0,
        vis=0.012, re=100.0, cfl=0.5, cfl_max=None, vfl=1.0,
        dr=1.0, f1=1.6, f2=1.6, flo_ang=(0.0, 90.0, 90.0), mpg=(0.0, 0.0, 0.0),
        rhof=1.0, rhos=1.0, coeff_rest=1.0, ramp_frac_steps=20,
        discr_scheme="center", limiter="none",
        adaptive=True, set_mpg=False, set_umean=False, initialize_zero=False,
        dorpr=True, revernorm=1, include_frmeanfluid=False,
        imove=0, collision_type="none", iscalon=0,
        pr_or_sc_nu=0.7, phisurf=0.0, phistream=1.0,
        rk3=False, xperiodic=True, nlcons=True, aliasflag=0, dobnd=True,
        input_type="default",
    )


_BOOL = {".true.": True, "t": True, ".t.": True, "true": True,
         ".false.": False, "f": False, ".f.": False, "false": False}


def _parse_value(tok: str):
    tok = tok.strip().rstrip(",").strip()
    if not tok:
        return None
    if tok[0] in "'\"":
        return tok.strip("'\"")
    low = tok.lower()
    if low in _BOOL:
        return _BOOL[low]
    parts = [p for p in re.split(r"[,\s]+", tok) if p]
    vals = []
    for p in parts:
        pl = p.lower()
        if pl in _BOOL:
            vals.append(_BOOL[pl])
            continue
        try:
            if re.fullmatch(r"[+-]?\d+", p):
                vals.append(int(p))
            else:
                vals.append(float(pl.replace("d", "e")))
        except ValueError:
            vals.append(p)
    return vals[0] if len(vals) == 1 else tuple(vals)


# Namelist groups and their variables as the reference declares them
# (SRC/FLO/global_data.F90:300-336, SRC/SCALAR/scalar_data.F90:89-91).
NAMELISTS = {
    "floandgrid": ("mx mxf my mz tstart ramp_frac_steps tend nerr_steps wtime_maxhrs saveforres_time tol_ferror vis "
                   "re rhof cpf kf archno cfl cfl_max vfl foffset mbuffer mpg ret flo_ang tol_gran_error"),
    "part_propt": ("nbody dr f1 f2 tstartmove lybyd dbydx dia_phys rhos cps ks input_type discr_scheme limiter "
                   "vol_frac1 min_part_sep nphases collision_type vel_distrib nl_slope_factor"),
    "flags": ("aliasflag maxzeroflag revernorm imove iscalon irestart iscal_restart saveforrestart saveforres_time "
              "xperiodic adaptive set_umean set_mpg nlcons rk3 mean_vel_to_particles dorpr dobnd include_frmeanfluid "
              "impose_grav debug_check cage_simul fixed_moving gof_avg only_dem movingcv iturbon moving_from_fixed_bed "
              "from_post change_frame use_drag_law initialize_zero"),
    "files": "outputfile rstsave outformat saveitns minunitno maxunitno errfile rstread write_output write_snapshot",
    "psd": "psd_type nphases sigmabydavg phiavg equal_momentum",
    "gcg": "coeff_rest pvel_var min_colisions mis_hs",
    "bidisperse": "volfrac_rat red1 dia_ratio yalpha",
    "lubtest": "hbyd",
    "matinput": "hhat mis_mat ibordel matern_treshold",
    "riser": "volume_fraction widthbyd aspect_ratio",
    "scal_propt": "nspmx phistream setphimean phisurf sourcepresent lumped_cap pr_or_sc_nu zero_flow_in_solid dorpr_scal",
    "postlist": ("nmis nbins skip_num post_no_flow_mem_alloc rad_factor power sa_max_itr post_error post_small rad_ratio "
                 "func_rad_ratio cooling_rate temp_init sa_error objective_coef1 objective_coef2 igeometry isa sa_in_itr "
                 "rad_reduction_ratio icohesive nsmall_length lybyd_small cluster_part_min cluster_part_max rotated "
                 "include_nmis"),
}
NAMELISTS = {g: frozenset(v.split()) for g, v in NAMELISTS.items()}
# array variables among the keys the engine reads, and their lengths
_ARRAYS = {"flo_ang": 3, "mpg": 3}


def _read_order(prm: Dict):
    """The groups read_nmls reads, in its order (SRC/FLO/initialize.F90:287-328).
    A generator: which groups come after GCG depends on values read before."""
    for g in ("floandgrid", "part_propt", "flags", "files", "psd", "gcg"):
        yield g
    it = str(prm.get("input_type", "default")).strip().lower()
    if it == "lubtest":
        yield "lubtest"
        yield "bidisperse"
    if it == "random" and str(prm.get("psd_type", "")).strip().lower() == "bidisp":
        yield "bidisperse"
    if it == "mat":
        yield "matinput"
    if it == "risers":
        yield "riser"
    if int(prm.get("iscalon", 0) or 0) == 1:
        yield "scal_propt"
    yield "postlist"


def _namelist_groups(text: str):
    """(name, body, start, end) of every &NAME ... / group, comments removed."""
    text = re.sub(r"![^\n]*", "", text)
    out = []
    for m in re.finditer(r"[&$](\w+)(.*?)(?:^\s*/|/\s*$|[&$]end\b)", text, flags=re.S | re.M | re.I):
        out.append((m.group(1).lower(), m.group(2), m.start(), m.end()))
    return out


def _group_items(body: str):
    """KEY = value pairs of one group body; values may span commas and lines,
    a repeat count n*v expands to n copies, KEY(i) = v sets one element."""
    for m in re.finditer(r"(\w+)(\(\s*\d+\s*\))?\s*=\s*(.*?)(?=[\s,]+\w+(\(\s*\d+\s*\))?\s*=|\Z)", body, flags=re.S):
        raw = m.group(3).replace("\n", " ").strip().rstrip(",")
        raw = re.sub(r"(\d+)\*([^\s,]+)", lambda r: ", ".join([r.group(2)] * int(r.group(1))), raw)
        idx = int(m.group(2).strip("() \t")) if m.group(2) else None
        yield m.group(1).lower(), idx, _parse_value(raw)


def read_floparam(path: str) -> Dict:
    """Read a floparam.in the way read_nmls does (SRC/FLO/initialize.F90:274-359).

    The groups are read in the reference's order, each one searched for
    after the end of the previous one (a sequential namelist read skips any
    other group on its way, as gfortran does), so a group that sits before
    one read earlier is never seen: that, and a group missing altogether,
    raise ValueError like the reference's end-of-file stop.  A variable that
    the group does not declare raises ValueError (the reference's namelist
    read aborts on it).  Keys are case-insensitive; ``!`` starts a comment.
    SET_UMEAN = T implies SET_MPG (initialize.F90:292).
    """
    prm = default_params()
    text = open(path).read()
    groups = _namelist_groups(text)
    pos = 0
    for name in _read_order(prm):
        hit = next((g for g in groups if g[0] == name and g[2] >= pos), None)
        if hit is None:
            where = "before an earlier group" if any(g[0] == name for g in groups) else "missing"
            raise ValueError(f"{path}: namelist group &{name.upper()} is {where}; read_nmls reads "
                             "FLOANDGRID, PART_PROPT, FLAGS, FILES, PSD, GCG, [LUBTEST, BIDISPERSE, MATINPUT, "
                             "RISER, SCAL_PROPT,] POSTLIST in that order")
        for key, idx, val in _group_items(hit[1]):
            if key not in NAMELISTS[name]:
                raise ValueError(f"{path}: &{name.upper()} has no variable {key.upper()}")
            if key in _ARRAYS:
                # a namelist array assignment sets elements idx, idx+1, ...
                # (from 1 without a subscript); the others keep their values
                cur = list(prm.get(key)) if isinstance(prm.get(key), (tuple, list)) else [0.0] * _ARRAYS[key]
                vals = list(val) if isinstance(val, (tuple, list)) else [val]
                for k, v in enumerate(vals):
                    if (idx or 1) - 1 + k >= len(cur):
                        raise ValueError(f"{path}: too many values for {key.upper()}")
                    cur[(idx or 1) - 1 + k] = v
                val = tuple(cur)
            elif idx is not None:
                raise ValueError(f"{path}: {key.upper()} is not an array")
            prm[key] = val
        pos = hit[3]
    if prm.get("set_umean"):
        prm["set_mpg"] = True
    return prm


def load_run(directory: str, run_name: str = "") -> tuple:
    """A run's parameters and sphere centres (grid units) from its input
    files, as initflo reads them: RUN_NAME_floparam.in (floparam.in without a
    run name), then for INPUT_TYPE = 'default' the centres of
    RUN_NAME_sphr_center.inp, for INPUT_TYPE = 'random' a configuration
    generated from RUN_NAME_seed.d (generators.load_random_run; the seed file
    is rewritten with the next seed, as the reference does)."""
    pre = run_name + "_" if run_name else ""
    prm = read_floparam(os.path.join(directory, pre + "floparam.in"))
    itype = str(prm.get("input_type", "default")).strip().lower()
    if itype == "random":
        from . import generators
        return generators.load_random_run(prm, directory, run_name or "")
    if itype != "default":
        raise ValueError(f"INPUT_TYPE = '{itype}' is not supported ('default' or 'random')")
    dbydx = prm["dbydx"] if prm.get("dbydx") is not None else prm["my"] / float(prm["lybyd"])
    return prm, read_sphr_center(os.path.join(directory, pre + "sphr_center.inp"), dbydx)


def read_sphr_center(path: str, dbydx: float) -> np.ndarray:
    """Sphere centres (nbody,3) in grid units from a sphr_center.inp file."""
    rows = []
    with open(path) as fh:
        next(fh)
        for line in fh:
            f = line.split()
            if len(f) >= 3:
                rows.append([float(v.replace("d", "e").replace("D", "e")) for v in f[:3]])
    return np.asarray(rows, dtype=np.float64).reshape(-1, 3) * float(dbydx)


def write_sphr_center(path: str, xc_grid: np.ndarray, dbydx: float, radius_diam: float = 0.5):
    """Write centres (grid units) in the reference's sphr_center.inp format."""
    with open(path, "w") as fh:
        fh.write(" generated\n")
        for i, row in enumerate(np.asarray(xc_grid) / dbydx):
            fh.write("  %.10f  %.10f  %.10f  %.10f  %d\n" % (row[0], row[1], row[2], radius_diam, i + 1))


def make_params(prm: Dict) -> pibm_params:
    """Fill a pibm_params struct from a parameter dict."""
    p = pibm_params()
    my = int(prm["my"])
    p.my = my
    p.mz = int(prm.get("mz") or my)
    p.lybyd = float(prm["lybyd"])
    p.dbydx = float(prm["dbydx"] if prm.get("dbydx") is not None else my / float(prm["lybyd"]))
    p.dia_phys = float(prm.get("dia_phys", 1.0))
    p.vis = float(prm["vis"])
    p.re = float(prm["re"])
    p.cfl = float(prm["cfl"])
    p.cfl_max = float(prm["cfl_max"] if prm.get("cfl_max") is not None else prm["cfl"])
    p.vfl = float(prm.get("vfl", 1.0))
    p.dr = float(prm.get("dr", 1.0))
    p.f1 = float(prm.get("f1", 1.6))
    p.f2 = float(prm.get("f2", 1.6))
    for d in range(3):
        p.flo_ang[d] = float(prm["flo_ang"][d])
        p.mpg[d] = float(prm["mpg"][d]) if isinstance(prm["mpg"], (tuple, list)) else float(prm["mpg"])
    p.rhof = float(prm.get("rhof", 1.0))
    p.rhos = float(prm.get("rhos", 1.0))
    p.coeff_rest = float(prm.get("coeff_rest", 1.0))
    p.ramp_frac_steps = int(prm.get("ramp_frac_steps", 20))
    sch = str(prm.get("discr_scheme", "center")).strip().lower()
    if sch not in ("center", "upwind"):
        raise ValueError("DISCR_SCHEME must be 'center' or 'upwind'")
    p.discr_scheme = PIBM_SCHEME_UPWIND if sch == "upwind" else PIBM_SCHEME_CENTER
    p.limiter = PIBM_LIMITER_MINMOD if str(prm.get("limiter", "none")).lower() == "minmod" else PIBM_LIMITER_NONE
    p.adaptive = int(bool(prm.get("adaptive", True)))
    p.set_mpg = int(bool(prm.get("set_mpg", False)))
    p.initialize_zero = int(bool(prm.get("initialize_zero", False)))
    p.dorpr = int(bool(prm.get("dorpr", True)))
    p.revernorm = int(prm.get("revernorm", 1))
    p.include_frmeanfluid = int(bool(prm.get("include_frmeanfluid", False)))
    p.imove = int(prm.get("imove", 0))
    p.collision_softsphere = int(str(prm.get("collision_type", "none")).lower() == "softsphere")
    p.iscalon = int(prm.get("iscalon", 0))
    p.pr_or_sc_nu = float(prm.get("pr_or_sc_nu", 0.7))
    p.phisurf = float(prm.get("phisurf", 0.0))
    p.phistream = float(prm.get("phistream", 1.0))
    p.rk3 = int(bool(prm.get("rk3", False)))
    if not prm.get("xperiodic", True):
        raise ValueError("XPERIODIC=F is not supported (x-periodic only)")
    # options that select reference code this engine does not run: passed on so
    # that the library refuses them (pibm_create returns PIBM_ERR_ARG)
    p.dobnd = int(bool(prm.get("dobnd", True)))
    p.aliasflag = int(prm.get("aliasflag", 0) or 0)
    p.nlcons_false = int(not prm.get("nlcons", True))
    ctype = str(prm.get("collision_type", "none")).strip().lower()
    if ctype not in ("none", "softsphere", "eventdriven"):
        raise ValueError(f"COLLISION_TYPE = '{ctype}' is not a reference collision model")
    if p.imove == 1 and ctype == "eventdriven":
        raise ValueError("COLLISION_TYPE = 'eventdriven' is not supported (soft-sphere DEM or 'none')")
    return p


class Particles:
    """Owns the arrays behind a pibm_particles struct (Fortran (nbody,3) layout)."""

    def __init__(self, xc: np.ndarray, vel: Optional[np.ndarray] = None):
        xc = np.asarray(xc, dtype=np.float64).reshape(-1, 3)
        self.nbody = xc.shape[0]
        self.xc_f = np.asfortranarray(xc).ravel(order="F").copy()
        self.vel_f = None if vel is None else np.asfortranarray(np.asarray(vel, np.float64).reshape(-1, 3)).ravel(order="F").copy()
        self.struct = pibm_particles()
        self.struct.nbody = self.nbody
        self.struct.xc = self.xc_f.ctypes.data_as(C.POINTER(C.c_double)) if self.nbody else None
        self.struct.velbdy = self.vel_f.ctypes.data_as(C.POINTER(C.c_double)) if self.vel_f is not None else None


# --------------------------------------------------------------------------
# Seeded synthetic workloads
# --------------------------------------------------------------------------

def _min_image(d, L):
    return d - L * np.round(d / L)


def random_sequential_addition(n: int, L: float, dia: float, rng, origin=1.0, max_tries=2_000_000):
    """n non-overlapping spheres (centres in [origin, origin+L)^3, periodic)."""
    pts = np.zeros((0, 3))
    tries = 0
    while pts.shape[0] < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("random sequential addition did not converge")
        c = origin + rng.random(3) * L
        if pts.shape[0]:
            d = _min_image(pts - c, L)
            if np.min(np.einsum("ij,ij->i", d, d)) < dia * dia:
                continue
        pts = np.vstack([pts, c])
    return pts


def hard_sphere_mc(pts: np.ndarray, L: float, dia: float, rng, moves: int, step: float, origin=1.0):
    """Seeded hard-sphere Monte Carlo displacement moves (periodic box)."""
    pts = pts.copy()
    n = pts.shape[0]
    acc = 0
    for _ in range(moves):
        i = rng.integers(n)
        trial = pts[i] + (rng.random(3) * 2.0 - 1.0) * step
        trial = origin + np.mod(trial - origin, L)
        d = _min_image(np.delete(pts, i, axis=0) - trial, L)
        if n == 1 or np.min(np.einsum("ij,ij->i", d, d)) >= dia * dia:
            pts[i] = trial
            acc += 1
    return pts, acc


def single_sphere(my: int = 64, dia_cells: float = 16.0, re: float = 20.0, vis: float = 0.012,
                  cfl: float = 0.1, steps: int = 100):
    """One fixed sphere at the box centre, fluid at rest, mpg-driven flow."""
    prm = default_params()
    prm.update(my=my, lybyd=my / dia_cells, dbydx=dia_cells, re=re, vis=vis, cfl=cfl, cfl_max=0.5,
               discr_scheme="upwind", initialize_zero=True, dobnd=False, ramp_frac_steps=0)
    xc = np.array([[1.0 + my / 2.0, 1.0 + my / 2.0, 1.0 + my / 2.0]])
    return prm, xc


def random_array(my: int = 128, dia_cells: float = 20.0, phi: float = 0.2, re: float = 50.0,
                 seed: int = 1234, mc_moves: int = 1000, vis: float = 0.012, cfl: float = 0.1,
                 nbody: Optional[int] = None):
    """Fixed random sphere array: RSA then hard-sphere MC (step 0.1 d)."""
    prm = default_params()
    prm.update(my=my, lybyd=my / dia_cells, dbydx=dia_cells, re=re, vis=vis, cfl=cfl, cfl_max=0.5,
               discr_scheme="upwind", initialize_zero=True, dobnd=False, ramp_frac_steps=0)
    if nbody is None:
        nbody = int(round(phi * my ** 3 / (np.pi / 6.0 * dia_cells ** 3)))
    rng = np.random.default_rng(seed)
    pts = random_sequential_addition(nbody, float(my), dia_cells, rng)
    pts, _ = hard_sphere_mc(pts, float(my), dia_cells, rng, mc_moves, 0.1 * dia_cells)
    return prm, pts


def adjoint_case(my: int = 96, dia_cells: float = 16.0, nbody: int = 30, seed: int = 4242, re: float = 20.0,
                 vis: float = 0.012, cfl: float = 0.1, mc_moves: int = 200):
    """Fixed random sphere array for gradient (adjoint) runs: SET_MPG with an
    imposed mean pressure gradient, a fixed time step (ADAPTIVE = F) and the
    upwind x flux.  The run starts from a uniform mean flow umean0 = (uchar,
    0, 0) (returned as prm['umean0']); the imposed mpg is about the Stokes
    drag of the array per unit fluid volume, so the mean flow stays of order
    uchar.  96^3 with 30 spheres of 16 cells is phi = 0.073."""
    prm = default_params()
    uchar = re * vis / 1.0
    volume = (my / dia_cells) ** 3
    mpg_x = -nbody * 3.0 * np.pi * vis * uchar * 2.0 / volume
    prm.update(my=my, lybyd=my / dia_cells, dbydx=dia_cells, re=re, vis=vis, cfl=cfl, cfl_max=0.5,
               discr_scheme="upwind", initialize_zero=True, dobnd=False, ramp_frac_steps=0,
               set_mpg=True, adaptive=False, mpg=(mpg_x, 0.0, 0.0))
    prm["umean0"] = (uchar, 0.0, 0.0)
    rng = np.random.default_rng(seed)
    pts = random_sequential_addition(nbody, float(my), dia_cells, rng)
    if mc_moves:
        pts, _ = hard_sphere_mc(pts, float(my), dia_cells, rng, mc_moves, 0.1 * dia_cells)
    return prm, pts


def moving_array(my: int = 64, dia_cells: float = 12.0, nbody: int = 12, seed: int = 11, re: float = 20.0,
                 rhos: float = 100.0, coeff_rest: float = 0.9, vel_spread: float = 0.1, mc_moves: int = 200,
                 collision_type: str = "softsphere", vis: float = 0.012):
    """Freely moving spheres (IMOVE = 1): a random array as random_array and
    seeded Maxwellian particle velocities of standard deviation
    vel_spread * uchar per component, with zero mean (the VEL_DISTRIB =
    'maxwellian' set-up of a freely evolving suspension)."""
    prm, pts = random_array(my=my, dia_cells=dia_cells, re=re, seed=seed, mc_moves=mc_moves, vis=vis, nbody=nbody)
    prm.update(imove=1, collision_type=collision_type, rhos=rhos, rhof=1.0, coeff_rest=coeff_rest)
    rng = np.random.default_rng(seed + 1)
    uchar = re * vis / float(prm.get("dia_phys", 1.0))
    vel = rng.normal(0.0, vel_spread * uchar, size=(pts.shape[0], 3))
    vel -= vel.mean(axis=0, keepdims=True)
    return prm, pts, vel


def fcc_subset(n: int, L: float, dia: float, rng, origin=1.0):
    """n sphere centres on randomly chosen sites of the densest periodic FCC
    lattice of the box whose nearest-neighbour distance is >= dia.  Returns
    None when the lattice has fewer than n sites."""
    k = int(np.floor(L / (dia * np.sqrt(2.0)) + 1e-12))
    if k < 1 or 4 * k ** 3 < n:
        return None
    a = L / k
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    cells = np.stack(np.meshgrid(np.arange(k), np.arange(k), np.arange(k), indexing="ij"), -1).reshape(-1, 1, 3)
    sites = ((cells + base[None]) * a).reshape(-1, 3)
    pick = rng.choice(sites.shape[0], size=n, replace=False)
    return origin + sites[np.sort(pick)]


def mis_ensemble(n: int = 16, seed: int = 2024, grids=(64, 96, 128), phi_range=(0.1, 0.4),
                 dia_range=(12, 20), re_range=(10.0, 100.0), mc_moves: int = 200, vis: float = 0.012,
                 cfl: float = 0.1):
    """Seeded ensemble of independent fixed-sphere realizations (multiple
    independent simulations, MIS): per member a grid from `grids`, a volume
    fraction ~ U(phi_range), an integer diameter ~ U(dia_range) cells and a
    particle Reynolds number ~ U(re_range).  Positions: random sequential
    addition up to phi = 0.3; above it (beyond what RSA reaches reliably) a
    random subset of the densest fitting FCC lattice, capped at the lattice's
    capacity; then hard-sphere Monte Carlo moves (step 0.1 d).  Returns a list
    of (params dict, centres (nbody, 3) grid units, achieved phi)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        my = int(rng.choice(np.asarray(grids)))
        phi = float(rng.uniform(*phi_range))
        dia = float(rng.integers(dia_range[0], dia_range[1] + 1))
        re = float(rng.uniform(*re_range))
        prm = default_params()
        prm.update(my=my, lybyd=my / dia, dbydx=dia, re=re, vis=vis, cfl=cfl, cfl_max=0.5,
                   discr_scheme="upwind", initialize_zero=True, dobnd=False, ramp_frac_steps=0)
        vsph = np.pi / 6.0 * dia ** 3
        nb = max(1, int(round(phi * my ** 3 / vsph)))
        pts = None
        if phi <= 0.3:
            try:
                pts = random_sequential_addition(nb, float(my), dia, rng, max_tries=200_000)
            except RuntimeError:
                pts = None
        if pts is None:
            k = int(np.floor(my / (dia * np.sqrt(2.0)) + 1e-12))
            nb = min(nb, 4 * k ** 3)
            pts = fcc_subset(nb, float(my), dia, rng)
        pts, _ = hard_sphere_mc(pts, float(my), dia, rng, mc_moves, 0.1 * dia)
        out.append((prm, pts, pts.shape[0] * vsph / my ** 3))
    return out
