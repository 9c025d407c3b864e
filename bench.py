"""Benchmark: Mcell-steps/s (FP64) of the per-step Navier-Stokes + IBM hot path.

Workload (one GPU): fixed random sphere array, 128^3 grid, 100 spheres of
diameter 20 cells (volume fraction 0.2), Re = 50, upwind x-flux, positions from
seeded random sequential addition followed by 1000 hard-sphere Monte Carlo
moves.  A step is one rks iteration: compute_new_timestep -> nonlinear ->
bcset -> velstep.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs N independent replicas (the step has no in-realization exchange),
one process per GPU under torch.distributed.run; value = all ranks' cell-steps
over the max-over-ranks device time.  ``--impl reference`` times the CPU
restatement of the reference step on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s FP64 at 128³ φ=0.2"
UNIT = "Mcell-steps/s"
WORKLOAD = dict(my=128, dia_cells=20.0, phi=0.2, re=50.0, seed=1234, mc_moves=1000)
PEAK_FALLBACK_GBS = 6650.0

# Algorithmic bytes per launch of each plane/line kernel, in units of one
# complex spectral field F_c = nx*my2*mz*16 B and one real field F_r = nx*my*mz*8 B:
# compulsory reads + writes of whole fields by that kernel alone.
KERNEL_BYTES = {
    "k_a0": (4, 10),     # read u(3), p; write ubcp(3), pbcp, omega(3), grad p(3)
    "k_flux": (0, 6),    # read ubcp(3); write the x-flux differences Dx(3)
    "k_nl": (9, 9),      # read ubcp(3), Dx(3), u(3), onl(3); write nl(3), Q(3)
    "k_ff": (3, 3),      # read fr(3); write ff(3)
    "k_lines": (17, 0),  # read u(3), p, nl(3), onl(3), ff(3); write u(3), p
}


def max_over_ranks(x: float, dist, device: str) -> float:
    """Max of a per-rank time over all ranks (every rank calls this)."""
    if not dist:
        return float(x)
    import torch
    tt = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def aggregate_mcells(ncell: int, steps: int, world: int, t_ms: float) -> float:
    """Whole-job Mcell-steps/s: every rank steps its own replica of ncell cells."""
    return ncell * steps * world / (t_ms / 1e3) / 1e6


def _peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


def _workload():
    from pureibm_ps2d_fd1d_b200 import config
    prm, xc = config.random_array(**WORKLOAD)
    return prm, xc


def _config_dict(n_gpus, xc, prm):
    return {
        "workload": "fixed random sphere array 128^3, %d spheres d=20 (phi=0.2), Re=50, upwind, AB2" % len(xc),
        "grid": [prm["my"], prm["my"], prm["my"]],
        "nbody": int(len(xc)),
        "parallelism": "replicas%d" % n_gpus if n_gpus > 1 else "single",
        "l2": "working set ~0.45 GB per replica > 126 MB L2 (no flush needed)",
        "seed": WORKLOAD["seed"],
    }


def _smi_id(torch, dev: int) -> str:
    """nvidia-smi -i identifier of torch device `dev` (its UUID, which does not
    depend on CUDA_VISIBLE_DEVICES); the physical index when no UUID is known."""
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        if u:
            return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        pass
    vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    return vis[dev].strip() if dev < len(vis) else str(dev)


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = str(gpu_index)
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu, "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(prm, xc, steps=2, warmup=1, threads=None):
    """The oracle (CPU restatement of the reference step) on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_ctypes as oc
    from pureibm_ps2d_fd1d_b200 import config
    threads = threads or os.cpu_count() or 1
    oc.set_threads(threads)
    P = config.make_params(prm)
    parts = config.Particles(xc)
    s = oc.OracleSolver(P, parts.struct)
    for _ in range(warmup):
        s.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step()
    el = time.perf_counter() - t0
    ncell = s.nx * s.my * s.mz
    s.close()
    return {"value": ncell * steps / el / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d steps (after %d warm-up) of the same 128^3 workload, oracle on %d threads" % (steps, warmup, threads),
            "s_per_step": el / steps}


def with_scalar(steps: int = 20, warmup: int = 3):
    """The same 128^3 sphere array with the passive scalar on (Pr = 0.7, cold
    spheres phisurf = 0 in a stream phistream = 1, initial flow uniform so the
    first mixed mean is defined): flow + scalar step throughput, device-timed."""
    import ctypes as C
    import pureibm_ps2d_fd1d_b200 as pk
    from pureibm_ps2d_fd1d_b200 import config, abi
    prm, xc = _workload()
    prm = dict(prm)
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=0.0, phistream=1.0, initialize_zero=False)
    s = pk.Solver(config.make_params(prm), xc)
    s.run(warmup)
    lib = pk.load_library()
    rep = abi.pibm_step_report()
    total = C.c_double()
    phases = (C.c_double * abi.PIBM_NPHASE)()
    rc = lib.pibm_run_timed(s.h, steps, C.byref(rep), C.byref(total))
    if rc != 0:
        raise RuntimeError("pibm_run_timed (scalar) failed: %d %s" % (rc, lib.pibm_last_error().decode()))
    ptotal = C.c_double()
    rc = lib.pibm_run_profiled(s.h, steps, C.byref(rep), C.byref(ptotal), phases, abi.PIBM_NPHASE)
    if rc != 0:
        raise RuntimeError("pibm_run_profiled (scalar) failed: %d %s" % (rc, lib.pibm_last_error().decode()))
    ncell = s.nx * s.my * s.mz
    out = {"unit": UNIT, "value": ncell * steps / (total.value / 1e3) / 1e6, "ms_per_step": total.value / steps,
           "serial_ms_per_step": ptotal.value / steps,
           "scalar_ms_per_step_serial": phases[abi.PIBM_NPHASE - 1] / steps, "steps": steps,
           "heat_ratio": rep.heat_ratio, "nusselt": rep.nusselt,
           "config": "128^3 sphere array above + passive scalar (Pr 0.7, phisurf 0, phistream 1)"}
    s.close()
    return out


def moving_suspension(steps: int = 10, warmup: int = 3):
    """The moving-particle configuration with scalar transport: 256^3, 1202
    spheres of diameter 20 cells (phi = 0.3), density ratio 100, seeded
    Maxwellian velocities (spread 0.1 uchar), soft-sphere DEM with
    restitution 0.9, passive scalar Pr 0.7 with sphere surfaces at
    phisurf = 1 in a stream at 0.  Flow + DEM + geometry rebuild + scalar
    step throughput, device-timed on the step graphs, and the serial phase
    split."""
    import ctypes as C
    import pureibm_ps2d_fd1d_b200 as pk
    from pureibm_ps2d_fd1d_b200 import config, abi
    prm, xc, vel = config.moving_array(my=256, dia_cells=20.0, nbody=1202, seed=2024, rhos=100.0, coeff_rest=0.9,
                                       vel_spread=0.1, mc_moves=1000)
    prm.update(iscalon=1, pr_or_sc_nu=0.7, phisurf=1.0, phistream=0.0, initialize_zero=False)
    s = pk.Solver(config.make_params(prm), xc, vel)
    s.run(warmup)
    lib = pk.load_library()
    rep = abi.pibm_step_report()
    total = C.c_double()
    rc = lib.pibm_run_timed(s.h, steps, C.byref(rep), C.byref(total))
    if rc != 0:
        raise RuntimeError("pibm_run_timed (moving) failed: %d %s" % (rc, lib.pibm_last_error().decode()))
    phases = (C.c_double * abi.PIBM_NPHASE)()
    ptotal = C.c_double()
    rc = lib.pibm_run_profiled(s.h, 3, C.byref(rep), C.byref(ptotal), phases, abi.PIBM_NPHASE)
    if rc != 0:
        raise RuntimeError("pibm_run_profiled (moving) failed: %d %s" % (rc, lib.pibm_last_error().decode()))
    contacts = s.get_contacts()
    ncell = s.nx * s.my * s.mz
    out = {"unit": UNIT, "value": ncell * steps / (total.value / 1e3) / 1e6, "ms_per_step": total.value / steps,
           "steps": steps, "serial_phase_ms_per_step": {abi.PHASE_NAMES[q]: phases[q] / 3 for q in range(abi.PIBM_NPHASE)},
           "active_reversal_points": rep.nrpr_active_total, "contact_entries": int(contacts["pn"][0].sum()),
           "dt": rep.dt, "nusselt": rep.nusselt,
           "config": "256^3, 1202 moving spheres d=20 (phi 0.3), rhos/rhof 100, Maxwellian velocities, "
                     "soft-sphere DEM e=0.9, passive scalar Pr 0.7"}
    s.close()
    return out


def adjoint_gradient(nsteps: int = 200, checkpoint_every: int = 20, warm: int = 100, fd: bool = True):
    """The gradient configuration: 96^3, 30 fixed spheres of diameter 16 cells
    (phi = 0.073, seeded), Re 20, imposed mean pressure gradient (SET_MPG),
    fixed dt, upwind x flux.  After `warm` steps from a uniform mean flow, J =
    time average over `nsteps` steps of the summed drag along x and its
    gradient w.r.t. all 90 sphere coordinates and the 3 mpg components
    (pibm_adjoint_run, checkpoints every `checkpoint_every` steps).  Reported:
    the forward time of the same steps on the step graphs, the adjoint run's
    forward (with checkpoints) and reverse sweep, their ratios, and central
    finite differences of the engine's forward run against the adjoint
    gradient for all 93 parameters.  J is piecewise
    smooth in xc: a stencil point crossing a grid cell face is a kink of the
    trilinear interpolation and a node entering the solid mask a jump, so each
    coordinate's fourth-order difference (steps up to 5e-6 diameters) stays
    inside the smooth piece around it (kinks.smooth_interval); coordinates
    whose piece is narrower than 1e-8 diameters are listed as skipped."""
    import ctypes as C
    import numpy as np
    import pureibm_ps2d_fd1d_b200 as pk
    from pureibm_ps2d_fd1d_b200 import config, abi
    prm, xc = config.adjoint_case()
    e = np.array([1.0, 0.0, 0.0])
    s = pk.Solver(config.make_params(prm), xc)
    st = s.get_state()
    st["umean"] = np.array(prm["umean0"])
    s.set_state(st)
    s.run(warm)
    st = s.get_state()
    lib = pk.load_library()
    rep = abi.pibm_step_report()
    total = C.c_double()
    rc = lib.pibm_run_timed(s.h, nsteps, C.byref(rep), C.byref(total))
    if rc != 0:
        raise RuntimeError("pibm_run_timed (adjoint case) failed: %d %s" % (rc, lib.pibm_last_error().decode()))
    fwd_ms = total.value
    s.set_state(st)
    out = s.adjoint(nsteps, e, checkpoint_every)
    # the same gradient with the whole trajectory's fields kept in HBM
    # (segment length from free memory: no recomputation when it fits)
    s.set_state(st)
    out_all = s.adjoint(nsteps, e, 0)
    s.close()
    res = {"config": "96^3, 30 fixed spheres d=16 (phi 0.073), Re 20, SET_MPG, fixed dt, upwind; %d steps after %d, "
                     "checkpoints every %d" % (nsteps, warm, checkpoint_every),
           "objective": "J = mean over the steps of e . sum_m (pres_m + visc_m), e = x",
           "J": out["J"], "forward_ms": fwd_ms, "adjoint_forward_ms": out["forward_ms"], "reverse_ms": out["reverse_ms"],
           "reverse_over_forward": out["reverse_ms"] / fwd_ms,
           "gradient_over_forward": (out["forward_ms"] + out["reverse_ms"]) / fwd_ms,
           "forward_ms_per_step": fwd_ms / nsteps, "reverse_ms_per_step": out["reverse_ms"] / nsteps,
           "adjoint_kernels_per_step": out["adjoint_kernels_per_step"],
           "store_all": {"reverse_ms": out_all["reverse_ms"], "reverse_over_forward": out_all["reverse_ms"] / fwd_ms,
                         "gradient_over_forward": (out_all["forward_ms"] + out_all["reverse_ms"]) / fwd_ms,
                         "max_rel_diff_vs_checkpointed": float(np.max(np.abs(out_all["g_xc"] - out["g_xc"])) /
                                                              np.max(np.abs(out["g_xc"])))},
           "g_mpg": list(out["g_mpg"]), "g_xc_norm": float(np.linalg.norm(out["g_xc"]))}
    if fd:
        # central differences of the engine's forward run for every
        # parameter (90 coordinates and mpg_x), each step inside the piece of
        # the coordinate on which J is smooth (no stencil point crosses a
        # cell face, no mask node changes: kinks.smooth_interval)
        from pureibm_ps2d_fd1d_b200 import kinks
        t0 = pk.Solver(config.make_params(prm), xc)
        bnd, R = t0.get_surface_points(), t0.info.radbdy
        t0.close()

        def J_of(xcv, mpg=None):
            p = dict(prm)
            st2 = dict(st)
            if mpg is not None:
                p["mpg"] = tuple(mpg)
                st2["mpg"] = np.asarray(mpg, dtype=np.float64)
            t = pk.Solver(config.make_params(p), xcv)
            t.set_state(st2)
            J = 0.0
            for _ in range(nsteps):
                r = t.step(1)
                J += float(np.dot(e, np.asarray(r["visc_total"]) - np.asarray(r["pres_total"])))
            t.close()
            return J / nsteps
        dia = 16.0
        # fourth-order central differences, f' = (-J(2h) + 8J(h) - 8J(-h) + J(-2h))/(12h),
        # with [-2h, 2h] inside the smooth piece: its truncation error is
        # negligible at h of a few 1e-6 d, where the rounding noise of the
        # forward runs (about |J| 1e-14 / h) still is; second order where the
        # piece is narrower than 2e-7 d
        h_max, h_min = 5e-6 * dia, 1e-8 * dia
        gmax = float(np.max(np.abs(out["g_xc"])))
        checks, skipped = [], []
        for m in range(xc.shape[0]):
            for d in range(3):
                lo, hi = kinks.smooth_interval(xc[m], d, bnd, R, float(prm.get("dr", 1.0)))
                half = min(-lo, hi)
                h4 = min(h_max, 0.45 * half)
                order = 4 if h4 >= 1e-7 * dia else 2
                h = h4 if order == 4 else min(h_max, 0.9 * half)
                if h < h_min:
                    skipped.append({"param": "xc[%d,%d]" % (m, d), "smooth_half_width_diameters": half / dia})
                    continue

                def J_at(t):
                    x = xc.copy()
                    x[m, d] += t
                    return J_of(x)
                if order == 4:
                    f = (-J_at(2 * h) + 8 * J_at(h) - 8 * J_at(-h) + J_at(-2 * h)) / (12 * h)
                else:
                    f = (J_at(h) - J_at(-h)) / (2 * h)
                a_ = float(out["g_xc"][m, d])
                checks.append({"param": "xc[%d,%d]" % (m, d), "step_diameters": h / dia, "order": order, "adjoint": a_,
                               "fd": f, "rel_err": abs(a_ - f) / max(abs(f), 1e-300), "err_over_gmax": abs(a_ - f) / gmax})
        mp = np.array(prm["mpg"], dtype=np.float64)
        dm = 1e-6 * abs(mp[0])
        a, b = mp.copy(), mp.copy()
        a[0] += dm
        b[0] -= dm
        f = (J_of(xc, a) - J_of(xc, b)) / (2 * dm)
        checks.append({"param": "mpg[0]", "step_rel": 1e-6, "adjoint": float(out["g_mpg"][0]), "fd": f,
                       "rel_err": abs(out["g_mpg"][0] - f) / max(abs(f), 1e-300)})
        xcs = [c for c in checks if c["param"].startswith("xc")]
        big = [c for c in xcs if abs(c["fd"]) >= 1e-2 * gmax]
        big10 = [c for c in xcs if abs(c["fd"]) >= 1e-1 * gmax]
        res["fd_check"] = {
            "method": "fourth-order central differences inside the smooth piece of each coordinate (step <= 5e-6 d; "
                      "second order where the piece is narrower; skipped below 1e-8 d), mpg_x second order at 1e-6 relative",
            "parameters_checked": len(checks), "parameters_skipped": skipped,
            "max_rel_err": max(c["rel_err"] for c in checks),
            "max_rel_err_components_above_1pct_of_max": max(c["rel_err"] for c in big) if big else None,
            "max_rel_err_components_above_10pct_of_max": max(c["rel_err"] for c in big10) if big10 else None,
            "median_step_diameters": float(np.median([c["step_diameters"] for c in xcs])),
            "max_err_over_gmax": max(c["err_over_gmax"] for c in xcs),
            "mpg_rel_err": checks[-1]["rel_err"],
            "worst": sorted(checks, key=lambda c: -c["rel_err"])[:5]}
    return res


def single_sphere(steps: int = 100, warmup: int = 5):
    """The single-sphere configuration: 64^3, one fixed sphere of diameter 16
    cells at the box centre (phi = 0.008), Re 20, fluid at rest driven by the
    mean pressure gradient, upwind; `steps` device-timed graph steps."""
    import ctypes as C
    import pureibm_ps2d_fd1d_b200 as pk
    from pureibm_ps2d_fd1d_b200 import config, abi
    prm, xc = config.single_sphere(my=64, dia_cells=16.0, re=20.0)
    s = pk.Solver(config.make_params(prm), xc)
    s.run(warmup)
    lib = pk.load_library()
    rep = abi.pibm_step_report()
    total = C.c_double()
    rc = lib.pibm_run_timed(s.h, steps, C.byref(rep), C.byref(total))
    if rc != 0:
        raise RuntimeError("pibm_run_timed (single sphere) failed: %d %s" % (rc, lib.pibm_last_error().decode()))
    ncell = s.nx * s.my * s.mz
    out = {"unit": UNIT, "value": ncell * steps / (total.value / 1e3) / 1e6, "ms_per_step": total.value / steps,
           "steps": steps, "norm_drag": rep.norm_drag, "tuning": s.tuning()["lines_per_cta"],
           "config": "64^3, 1 sphere d=16 at the centre, Re 20, upwind"}
    s.close()
    return out


def _mis_times(ens, steps: int, warmup: int, api_loop: bool):
    """Device ms of `steps` steps of every member of ensemble `ens`: the plain
    per-realization loop (each member replaying its own step graphs, one after
    another), the batch graph with every member's step its own branch, and the
    batch graph in which members of one grid size share each kernel launch;
    with api_loop also the reference-style host loop (each member stepped in
    turn through pibm_step, its report read back every step), wall-timed."""
    import pureibm_ps2d_fd1d_b200 as pk
    b = pk.Batch([(p, x) for p, x, _ in ens])
    b.run(warmup)
    cells = sum(p["my"] ** 3 for p, _, _ in ens) * steps
    t_plain = b.time(steps, sequential=True)
    b.time(1, sequential=False, fused=False)
    t_branch = b.time(steps, sequential=False, fused=False)
    b.time(1, sequential=False)
    t_batch = b.time(steps, sequential=False)
    out = {"plain": cells / (t_plain / 1e3) / 1e6, "batched": cells / (t_batch / 1e3) / 1e6,
           "ratio": t_plain / t_batch,
           "branches": cells / (t_branch / 1e3) / 1e6, "ratio_branches": t_plain / t_branch,
           "ms_per_step": {"plain": t_plain / steps, "branches": t_branch / steps, "batched": t_batch / steps}}
    if api_loop:
        t0 = time.perf_counter()
        for _ in range(steps):
            for m in b.members:
                m.step(1)
        t_api = (time.perf_counter() - t0) * 1e3
        out.update({"step_api_loop": cells / (t_api / 1e3) / 1e6, "ratio_vs_step_api_loop": t_api / t_batch})
    b.close()
    return out


def batched_mis(steps: int = 10, warmup: int = 3, n: int = 16, seed: int = 2024, sweep: bool = False):
    """Batched multiple-independent-simulation throughput against the plain
    per-realization loop on the same GPU (_mis_times): 16 seeded realizations
    (grids from {64, 96, 128}^3, phi ~ U[0.1, 0.4], d ~ U{12..20} cells,
    Re ~ U[10, 100]), `steps` steps of every member each way, device-timed;
    and the same for two small-grid ensembles of 16 (all 32^3; 32^3 and 64^3
    mixed), where one member alone leaves most SMs idle; with sweep also
    one-size ensembles of each grid size (seed 7)."""
    from pureibm_ps2d_fd1d_b200 import config
    ens = config.mis_ensemble(n=n, seed=seed)
    out = {"unit": "Mcell-steps/s", **_mis_times(ens, steps, warmup, api_loop=True),
           "members": n, "steps": steps, "seed": seed,
           "grids": [p["my"] for p, _, _ in ens], "nbody": [len(x) for _, x, _ in ens],
           "phi": [round(f, 4) for _, _, f in ens]}
    for key, grids in (("small_grids_32", (32,)), ("small_grids_32_64", (32, 64))):
        e = config.mis_ensemble(n=16, seed=7, grids=grids)
        out[key] = {**_mis_times(e, steps, warmup, api_loop=False), "members": 16, "seed": 7,
                    "grids": [p["my"] for p, _, _ in e], "nbody": [len(x) for _, x, _ in e]}
    if sweep:
        for g, m in ((64, 8), (96, 8), (128, 4)):
            e = config.mis_ensemble(n=m, seed=7, grids=(g,))
            out[f"one_size_{g}"] = {**_mis_times(e, steps, warmup, api_loop=False), "members": m, "seed": 7,
                                    "nbody": [len(x) for _, x, _ in e]}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    prm, xc = _workload()
    threads = os.cpu_count() or 1
    steps = max(1, args.steps)
    cb = cpu_baseline(prm, xc, steps=steps, warmup=max(0, min(args.warmup, 1)), threads=threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": cb["s_per_step"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded sphere positions)", "config": _config_dict(1, xc, prm),
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_gpu(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import numpy as np
    import torch
    # one GPU per rank: LOCAL_RANK indexes the devices this job was given (any
    # CUDA_VISIBLE_DEVICES subset the launcher set is kept); the engine
    # creates its handle on the current device of this thread
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import pureibm_ps2d_fd1d_b200 as pk
    from pureibm_ps2d_fd1d_b200 import config, abi

    prm, xc = _workload()
    s = pk.Solver(config.make_params(prm), xc)
    if args.lines_per_cta:
        # pins the x-line width the creation-time autotuner chose (a profiler's
        # serialised launches can distort the tuner's whole-step timings)
        s.set_tuning(args.lines_per_cta)
    ncell = s.nx * s.my * s.mz
    # warm-up (graph path) then the timed region with per-phase events on the engine's stream
    s.run(max(args.warmup, 3))

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    import ctypes as C
    lib = pk.load_library()
    rep = abi.pibm_step_report()
    total = C.c_double()
    phases = (C.c_double * abi.PIBM_NPHASE)()
    barrier()
    # the timed region: the production path (one CUDA graph per step, drag/mpg on a side stream)
    with ClockSampler(_smi_id(torch, dev)) as clk:
        rc = lib.pibm_run_timed(s.h, args.steps, C.byref(rep), C.byref(total))
    barrier()
    if rc != 0:
        raise RuntimeError("pibm_run_timed failed: %d %s" % (rc, lib.pibm_last_error().decode()))
    t_ms = max_over_ranks(total.value, dist, "cuda")
    # per-phase breakdown (serial launches with events between phases; not the timed number)
    ptotal = C.c_double()
    rc = lib.pibm_run_profiled(s.h, args.steps, C.byref(rep), C.byref(ptotal), phases, abi.PIBM_NPHASE)
    if rc != 0:
        raise RuntimeError("pibm_run_profiled failed: %d %s" % (rc, lib.pibm_last_error().decode()))
    value = aggregate_mcells(ncell, args.steps, world, t_ms)
    phase_ms = {abi.PHASE_NAMES[q]: phases[q] / args.steps for q in range(abi.PIBM_NPHASE)}
    # per-kernel breakdown: the same launches, serial, a CUDA event pair on the
    # engine's stream around every kernel (pibm_kernel_times)
    kms = (C.c_double * abi.PIBM_NKERNEL)()
    ktotal = C.c_double()
    rc = lib.pibm_kernel_times(s.h, args.steps, C.byref(ktotal), kms, abi.PIBM_NKERNEL)
    if rc != 0:
        raise RuntimeError("pibm_kernel_times failed: %d %s" % (rc, lib.pibm_last_error().decode()))
    kernel_ms = {abi.KERNEL_NAMES[k]: kms[k] / args.steps for k in range(abi.PIBM_NKERNEL)}

    # end-to-end through the C ABI with host buffers: every step uploads the
    # state (u, nl, p in the reference layout) from pinned memory, steps, and
    # downloads it again.
    nx, my2, mz = s.nx, s.my2, s.mz
    shp_u, shp_p = (3, mz, my2, nx + 1), (mz, my2, nx)
    pin = lambda shp: torch.empty(tuple(shp) + (2,), dtype=torch.float64).pin_memory()
    hu, hnl, hp = pin(shp_u), pin(shp_u), pin(shp_p)
    view = abi.pibm_state_view()
    view.u = C.cast(hu.data_ptr(), C.POINTER(C.c_double))
    view.nl = C.cast(hnl.data_ptr(), C.POINTER(C.c_double))
    view.p = C.cast(hp.data_ptr(), C.POINTER(C.c_double))
    assert lib.pibm_get_state(s.h, C.byref(view)) == 0
    e2e_steps = max(1, min(args.steps, 10))
    for _ in range(2):   # untimed: first calls load the layout kernels and touch the pinned pages
        assert lib.pibm_set_state(s.h, C.byref(view)) == 0
        assert lib.pibm_step(s.h, 1, C.byref(rep)) == 0
        assert lib.pibm_get_state(s.h, C.byref(view)) == 0
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        assert lib.pibm_set_state(s.h, C.byref(view)) == 0
        assert lib.pibm_step(s.h, 1, C.byref(rep)) == 0
        assert lib.pibm_get_state(s.h, C.byref(view)) == 0
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    bytes_state = (hu.numel() + hnl.numel() + hp.numel()) * 8
    # the drop-in loop of a host driver that keeps the state on the device:
    # one synchronous pibm_step per step, its report read back to the host
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        assert lib.pibm_step(s.h, 1, C.byref(rep)) == 0
    barrier()
    res_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    peak, peak_kind = _peak_gbs()
    Fc = nx * my2 * mz * 16
    Fr = nx * s.my * mz * 8
    traffic_tab = {}
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as fh:
            traffic_tab = json.load(fh)
    except Exception:
        pass

    def kernel_roof(name):
        nc, nr = KERNEL_BYTES[name]
        alg = nc * Fc + nr * Fr
        ach = alg / (kernel_ms[name] / 1e3) / 1e9
        ent = traffic_tab.get(name) if isinstance(traffic_tab.get(name), dict) else None
        return {"bound": "hbm", "kernel": name, "achieved": ach, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": ach / peak, "ms_per_launch": kernel_ms[name],
                "algorithmic_bytes_per_launch": alg,
                "traffic": float(ent["bytes_per_launch_at_128"]) if ent else None}

    kernel_roofline = {k: kernel_roof(k) for k in KERNEL_BYTES}
    dominant = max(KERNEL_BYTES, key=lambda k: kernel_ms[k])
    b_alg_step = 30 * Fc
    info = s.info
    # FP64 arithmetic: the reference's transform count (31 plane FFTs per
    # x-plane, 2.5 n log2 n flops each for a real n-point plane) and the
    # count this engine executes (25 plane transforms per x-plane; five
    # circulant line solves per (ky,kz) line, each a forward and an inverse
    # complex x-FFT of 5 nx log2 nx flops), against the measured DFMA peak
    import math
    nplane = s.my * mz
    f_plane = 2.5 * nplane * math.log2(nplane)
    f_ref = 31 * nx * f_plane
    f_exec = 25 * nx * f_plane + (my2 * mz) * 5 * 2 * 5 * nx * math.log2(nx)
    fp_peak, fp_ms = C.c_double(), C.c_double()
    fp64 = None
    if lib.pibm_fp64_peak(C.byref(fp_peak), C.byref(fp_ms)) == 0:
        ach = f_exec / (t_ms / args.steps / 1e3) / 1e12
        fp64 = {"peak_tflops": fp_peak.value, "peak_kind": "measured (DFMA chains, pibm_fp64_peak)",
                "flops_per_step_reference_count": f_ref, "flops_per_step_executed": f_exec,
                "achieved_tflops": ach, "frac": ach / fp_peak.value}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded sphere positions, fluid initially at rest)",
        "config": _config_dict(world, xc, prm),
        "lines_per_cta": s.tuning()["lines_per_cta"],   # x-line width the run used (tuned or pinned)
        "roofline": kernel_roofline[dominant],
        "kernel_roofline": kernel_roofline,
        "step_roofline": {"algorithmic_bytes_per_step": b_alg_step,
                          "achieved_GBps": b_alg_step / (t_ms / args.steps / 1e3) / 1e9,
                          "frac": b_alg_step / (t_ms / args.steps / 1e3) / 1e9 / peak},
        "phase_ms_per_step": phase_ms,
        "kernel_ms_per_step": kernel_ms,
        "e2e": {"value": ncell * e2e_steps * world / e2e_s / 1e6, "unit": UNIT,
                "h2d_bytes_per_step": bytes_state, "d2h_bytes_per_step": bytes_state + C.sizeof(rep),
                "path": "pibm_set_state(pinned host) + pibm_step + pibm_get_state(pinned host) per step"},
        "e2e_resident_state": {"value": ncell * e2e_steps * world / res_s / 1e6, "unit": UNIT, "h2d_bytes_per_step": 0,
                               "d2h_bytes_per_step": C.sizeof(rep),
                               "path": "one synchronous pibm_step per step with its report read back; the state stays on the device"},
        "gpu_launches": int(info.kernels_per_step) * args.steps,
        "clocks": clk.summary(),
        "fp64": fp64,
        "active_reversal_points": int(info.npts_active),
        "maxvolfrac": info.maxvolfrac,
        "last_step": {"divmax": rep.divmax, "norm_drag": rep.norm_drag, "dt": rep.dt},
    }
    def section(key, fn):
        # a failing optional measurement is recorded, never allowed to drop the headline line
        try:
            line[key] = fn()
        except Exception as ex:   # noqa: BLE001
            line[key] = {"error": repr(ex)[:400]}
            print("bench: section %s failed: %r" % (key, ex), file=sys.stderr)

    if world == 1:
        if not args.no_mis:
            section("batched_mis", batched_mis)
            section("single_sphere", single_sphere)
        if not args.no_scalar:
            section("with_scalar", with_scalar)
        if not args.no_moving:
            section("moving_suspension", moving_suspension)
        if not args.no_adjoint:
            section("adjoint", adjoint_gradient)
        if not args.no_cpu_baseline:
            keys = ("value", "unit", "cores", "kind", "sample")
            # about 10-15 s of host work each: 20 steps on all threads, 4 on one
            section("cpu_baseline", lambda: {k: v for k, v in cpu_baseline(prm, xc, steps=20, warmup=1).items() if k in keys})
            # the reference's own serial semantics: the same oracle on one thread
            section("cpu_baseline_1thread",
                    lambda: {k: v for k, v in cpu_baseline(prm, xc, steps=4, warmup=1, threads=1).items() if k in keys})
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mis", action="store_true", help="skip the batched-realization measurement")
    ap.add_argument("--no-scalar", action="store_true", help="skip the flow + passive-scalar measurement")
    ap.add_argument("--no-moving", action="store_true", help="skip the moving-particle suspension measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (gradient) measurement")
    ap.add_argument("--lines-per-cta", type=int, default=0, choices=[0, 4, 8],
                    help="headline run: x-line tile width (4 = persistent kernel up to 128^3, 8 = staged); "
                         "0 keeps the autotuner's choice")
    ap.add_argument("--mis-only", action="store_true",
                    help="print only the batched-realization measurement (steps and warm-up from --steps/--warmup)")
    ap.add_argument("--mis-sweep", action="store_true",
                    help="with --mis-only: also one-size ensembles (sixteen 32^3, eight 64^3, eight 96^3, four 128^3)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.mis_only:
        print(json.dumps(batched_mis(steps=args.steps, warmup=args.warmup, sweep=args.mis_sweep)))
        return 0
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
