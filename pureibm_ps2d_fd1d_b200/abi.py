"""ctypes mirror of include/pibm.h (the engine's C ABI).

Every structure here has the same field order and types as the header; the
tests check the sizes against the compiled library.
"""
import ctypes as C

PIBM_OK = 0
PIBM_ERR_ARG = -1
PIBM_ERR_BLOWUP = -2
PIBM_ERR_PIVOT = -3
PIBM_ERR_NAN = -4
PIBM_ERR_DEM_MOVE = -5
PIBM_ERR_NEIGH_OVERFLOW = -6
PIBM_ERR_TIMEOUT = -7
PIBM_ERR_CUDA = -8
PIBM_ERR_NOMEM = -9
PIBM_ERR_SPREAD_OVERFLOW = -10

ERROR_NAMES = {
    PIBM_ERR_ARG: "PIBM_ERR_ARG",
    PIBM_ERR_BLOWUP: "PIBM_ERR_BLOWUP",
    PIBM_ERR_PIVOT: "PIBM_ERR_PIVOT",
    PIBM_ERR_NAN: "PIBM_ERR_NAN",
    PIBM_ERR_DEM_MOVE: "PIBM_ERR_DEM_MOVE",
    PIBM_ERR_NEIGH_OVERFLOW: "PIBM_ERR_NEIGH_OVERFLOW",
    PIBM_ERR_TIMEOUT: "PIBM_ERR_TIMEOUT",
    PIBM_ERR_CUDA: "PIBM_ERR_CUDA",
    PIBM_ERR_NOMEM: "PIBM_ERR_NOMEM",
    PIBM_ERR_SPREAD_OVERFLOW: "PIBM_ERR_SPREAD_OVERFLOW",
}

PIBM_SCHEME_CENTER = 0
PIBM_SCHEME_UPWIND = 1
PIBM_LIMITER_NONE = 0
PIBM_LIMITER_MINMOD = 1
PIBM_NPHASE = 7
PHASE_NAMES = ["a0_fields_to_real", "nonlinear", "drag_mpg", "reversal_spread", "forcing_fft", "x_lines", "scalar"]
# kernel slots of pibm_kernel_times (PIBM_K_*), in launch order
PIBM_NKERNEL = 12
KERNEL_NAMES = ["k_a0", "k_scal_a", "k_flux", "k_nl", "k_drag", "k_scal_b", "k_rev", "k_scal_c", "k_spread",
                "k_ff", "k_lines", "k_scal_d"]

_i32 = C.c_int32
_f64 = C.c_double


class pibm_params(C.Structure):
    _fields_ = [
        ("my", _i32), ("mz", _i32),
        ("lybyd", _f64), ("dbydx", _f64), ("dia_phys", _f64),
        ("vis", _f64), ("re", _f64), ("cfl", _f64), ("cfl_max", _f64), ("vfl", _f64),
        ("dr", _f64), ("f1", _f64), ("f2", _f64),
        ("flo_ang", _f64 * 3), ("mpg", _f64 * 3),
        ("rhof", _f64), ("rhos", _f64), ("coeff_rest", _f64),
        ("ramp_frac_steps", _i32), ("discr_scheme", _i32), ("limiter", _i32),
        ("adaptive", _i32), ("set_mpg", _i32), ("initialize_zero", _i32),
        ("dorpr", _i32), ("revernorm", _i32), ("include_frmeanfluid", _i32),
        ("imove", _i32), ("collision_softsphere", _i32), ("iscalon", _i32),
        ("pr_or_sc_nu", _f64), ("phisurf", _f64), ("phistream", _f64),
        ("rk3", _i32), ("dobnd", _i32), ("aliasflag", _i32), ("nlcons_false", _i32), ("reserved", _i32 * 4),
    ]


class pibm_particles(C.Structure):
    _fields_ = [("nbody", _i32), ("xc", C.POINTER(_f64)), ("velbdy", C.POINTER(_f64))]


class pibm_state_view(C.Structure):
    _fields_ = [
        ("u", C.POINTER(_f64)), ("nl", C.POINTER(_f64)), ("p", C.POINTER(_f64)),
        ("umean", _f64 * 3), ("mpg", _f64 * 3), ("ufmean", _f64 * 3),
        ("t", _f64), ("dt", _f64), ("cf", _f64),
    ]


class pibm_step_report(C.Structure):
    _fields_ = [
        ("dt", _f64), ("t", _f64), ("cf", _f64), ("umax", _f64), ("divmax", _f64),
        ("ufmean", _f64 * 3), ("usmean", _f64 * 3), ("umean", _f64 * 3),
        ("mpg", _f64 * 3), ("frmean", _f64 * 3),
        ("pres_total", _f64 * 3), ("visc_total", _f64 * 3),
        ("norm_drag", _f64), ("ferror", _f64),
        ("pres_drag", _f64), ("visc_drag", _f64), ("total_drag", _f64),
        ("mixmeanslipmod", _f64),
        ("nrpr_active_total", C.c_int64),
        ("heat_ratio", _f64), ("nusselt", _f64),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class pibm_info(C.Structure):
    _fields_ = [
        ("nx", _i32), ("my", _i32), ("mz", _i32), ("my2", _i32), ("nbody", _i32), ("nbnd", _i32),
        ("dx", _f64), ("dt", _f64), ("radbdy", _f64), ("maxvolfrac", _f64),
        ("count_solid", C.c_int64), ("count_fluid", C.c_int64),
        ("npts_active", _i32), ("kernels_per_step", _i32),
    ]


class pibm_adjoint_report(C.Structure):
    _fields_ = [
        ("J", _f64), ("forward_ms", _f64), ("reverse_ms", _f64),
        ("nsteps", _i32), ("checkpoint_every", _i32), ("adjoint_kernels_per_step", _i32), ("reserved", _i32),
    ]


# Exported symbols of libpibm (declared in include/pibm.h).
EXPORTED = [
    "pibm_create", "pibm_info_get", "pibm_set_state", "pibm_step", "pibm_run", "pibm_run_timed",
    "pibm_run_profiled", "pibm_kernel_times", "pibm_kernel_name", "pibm_get_state", "pibm_get_particles", "pibm_get_scalar", "pibm_get_if_rev",
    "pibm_get_fluid_mask", "pibm_get_contacts", "pibm_get_scalar_nl", "pibm_set_scalar",
    "pibm_set_desired_means", "pibm_adjoint_run", "pibm_adjoint_begin", "pibm_adjoint_step", "pibm_adjoint_end", "pibm_fp64_peak", "pibm_qdiv_check", "pibm_get_tuning", "pibm_set_tuning", "pibm_destroy", "pibm_last_error", "pibm_ff2rc", "pibm_ff2cr",
    "pibm_ff2cr_noalloc", "pibm_batch_create", "pibm_batch_run", "pibm_batch_time", "pibm_batch_member",
    "pibm_batch_destroy", "pibm_get_frame", "pibm_set_frame", "pibm_get_surface_points",
]


def bind(lib):
    """Attach argtypes/restypes for the pibm_* entry points."""
    P = C.POINTER
    vp = C.c_void_p
    lib.pibm_create.argtypes = [P(pibm_params), P(pibm_particles), P(vp)]
    lib.pibm_info_get.argtypes = [vp, P(pibm_info)]
    lib.pibm_set_state.argtypes = [vp, P(pibm_state_view)]
    lib.pibm_step.argtypes = [vp, C.c_int, P(pibm_step_report)]
    lib.pibm_run.argtypes = [vp, C.c_int, P(pibm_step_report)]
    lib.pibm_get_state.argtypes = [vp, P(pibm_state_view)]
    lib.pibm_run_timed.argtypes = [vp, C.c_int, P(pibm_step_report), P(_f64)]
    lib.pibm_run_profiled.argtypes = [vp, C.c_int, P(pibm_step_report), P(_f64), P(_f64), C.c_int]
    lib.pibm_kernel_times.argtypes = [vp, C.c_int, P(_f64), P(_f64), C.c_int]
    lib.pibm_kernel_name.argtypes = [C.c_int]
    lib.pibm_kernel_name.restype = C.c_char_p
    lib.pibm_get_particles.argtypes = [vp] + [P(_f64)] * 5
    lib.pibm_get_scalar.argtypes = [vp, P(_f64), P(_f64), P(_f64)]
    lib.pibm_get_if_rev.argtypes = [vp, P(C.c_uint8)]
    lib.pibm_get_fluid_mask.argtypes = [vp, P(C.c_uint8)]
    lib.pibm_get_contacts.argtypes = [vp, C.c_int32, P(C.c_int32), P(C.c_int32), P(C.c_int32)]
    lib.pibm_get_scalar_nl.argtypes = [vp, P(_f64)]
    lib.pibm_get_frame.argtypes = [vp, P(_f64), P(_f64)]
    lib.pibm_get_surface_points.argtypes = [vp, P(_f64)]
    lib.pibm_set_frame.argtypes = [vp, P(_f64), P(_f64)]
    lib.pibm_set_scalar.argtypes = [vp, P(_f64), P(_f64), P(_f64)]
    lib.pibm_set_desired_means.argtypes = [vp, P(_f64), P(_f64)]
    lib.pibm_adjoint_run.argtypes = [vp, C.c_int, C.c_int, P(_f64), P(_f64), P(_f64), P(pibm_adjoint_report)]
    lib.pibm_fp64_peak.argtypes = [P(_f64), P(_f64)]
    lib.pibm_qdiv_check.argtypes = [P(_f64), C.c_longlong, P(_f64), C.c_int, P(C.c_longlong)]
    lib.pibm_adjoint_begin.argtypes = [vp, C.c_int, P(_f64)]
    lib.pibm_adjoint_step.argtypes = [vp]
    lib.pibm_adjoint_end.argtypes = [vp, P(_f64), P(_f64)]
    lib.pibm_get_tuning.argtypes = [vp, P(C.c_int32), P(_f64)]
    lib.pibm_set_tuning.argtypes = [vp, C.c_int32]
    lib.pibm_destroy.argtypes = [vp]
    lib.pibm_destroy.restype = None
    lib.pibm_last_error.argtypes = []
    lib.pibm_last_error.restype = C.c_char_p
    for fn in (lib.pibm_ff2rc, lib.pibm_ff2cr):
        fn.argtypes = [C.c_int, C.c_int, C.c_int, P(_f64), P(_f64)]
    lib.pibm_ff2cr_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp]
    lib.pibm_batch_create.argtypes = [C.c_int, P(pibm_params), P(pibm_particles), P(vp)]
    lib.pibm_batch_run.argtypes = [vp, C.c_int]
    lib.pibm_batch_time.argtypes = [vp, C.c_int, C.c_int, P(C.c_double)]
    lib.pibm_batch_member.argtypes = [vp, C.c_int]
    lib.pibm_batch_member.restype = vp
    lib.pibm_batch_destroy.argtypes = [vp]
    lib.pibm_batch_destroy.restype = None
    for name in ("pibm_create", "pibm_info_get", "pibm_set_state", "pibm_step", "pibm_run", "pibm_run_timed", "pibm_run_profiled",
                 "pibm_kernel_times", "pibm_get_state", "pibm_get_particles", "pibm_get_scalar", "pibm_get_if_rev", "pibm_get_fluid_mask",
                 "pibm_get_contacts", "pibm_get_scalar_nl", "pibm_set_scalar", "pibm_set_desired_means",
                 "pibm_get_frame", "pibm_set_frame", "pibm_get_surface_points", "pibm_adjoint_run", "pibm_adjoint_begin", "pibm_adjoint_step", "pibm_adjoint_end", "pibm_fp64_peak", "pibm_qdiv_check", "pibm_get_tuning", "pibm_set_tuning", "pibm_ff2rc", "pibm_ff2cr", "pibm_ff2cr_noalloc", "pibm_batch_create", "pibm_batch_run", "pibm_batch_time"):
        getattr(lib, name).restype = C.c_int
    return lib
