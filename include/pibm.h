/*
 * pibm.h -- C ABI of the B200-native PUReIBM-PS2D-FD1D time-step engine.
 *
 * The reference has no FFI: its step boundary is the fixed call sequence
 * inside the driver's rks loop (SRC/FLO/dtibm_main_scal_flo.F90:426-527):
 *     compute_new_timestep(rks) -> nonlinear(rks) [-> bcset(rks)] -> velstep(sflag,rks)
 * and every datum moves through module globals (SRC/FLO/global_data.F90:53-338).
 * This header replaces that boundary with explicit handles.  All arrays that
 * cross it keep the reference's Fortran layout (column-major, x fastest):
 *     u, nl  : complex(8) u(nx+1, my2, mz, 3)   (plane nx+1 is the periodic image of plane 1)
 *     p      : complex(8) p(nx, my2, mz)
 *     xc, velbdy, pres, visc, force : real(8) (nbody, 3)
 * complex(8) is passed as interleaved (re, im) doubles.
 *
 * Return codes: 0 on success, negative PIBM_ERR_* otherwise (the reference
 * stops the program instead; see each code).  Calls are synchronous; one host
 * thread per handle.  Device memory is owned by the handle; host arrays are
 * only borrowed for the duration of a call.
 */
#ifndef PIBM_H
#define PIBM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes (reference stop conditions they replace). */
#define PIBM_OK                   0
#define PIBM_ERR_ARG            (-1)  /* bad argument / unsupported option                         */
#define PIBM_ERR_BLOWUP         (-2)  /* norm_drag > 1e6: boundary_condition.F90:874-884            */
#define PIBM_ERR_PIVOT          (-3)  /* zero pivot in Thomas: tridiagonal.F90:62,72-76             */
#define PIBM_ERR_NAN            (-4)  /* non-finite state detected                                  */
#define PIBM_ERR_DEM_MOVE       (-5)  /* particle moved >= radius in one DEM sub-step: collision_mod.F90:1421-1428 */
#define PIBM_ERR_NEIGH_OVERFLOW (-6)  /* neighbour list overflow: collision_mod.F90:845-848          */
#define PIBM_ERR_TIMEOUT        (-7)  /* a bounded device wait ran out                              */
#define PIBM_ERR_CUDA           (-8)  /* CUDA runtime error                                         */
#define PIBM_ERR_NOMEM          (-9)  /* allocation failed                                          */
#define PIBM_ERR_SPREAD_OVERFLOW (-10) /* more force contributions on one node than the spreading buckets hold */

/* x-flux discretisation (Part_propt DISCR_SCHEME, nl_allflow.F90:98-100,192-207). */
#define PIBM_SCHEME_CENTER 0
#define PIBM_SCHEME_UPWIND 1
/* MUSCL slope limiter (Part_propt LIMITER, nl_allflow.F90:178-207). */
#define PIBM_LIMITER_NONE   0
#define PIBM_LIMITER_MINMOD 1

/*
 * Parsed floparam.in values that define one run (namelists FLOANDGRID,
 * PART_PROPT, FLAGS; defaults in SRC/FLO/initialize.F90:73-271).
 * Grid: mx = my+1, nx = mx-1 = my, my2 = my/2+1 (initialize.F90:340-352);
 * mz = my unless given.  Only the serial x-periodic path is supported
 * (PARALLEL=0, XPERIODIC=T, NLCONS=T, AliasFlag=0, DOBND=F), AB2 or RK3;
 * pibm_create returns PIBM_ERR_ARG for the others (fields dobnd, aliasflag,
 * nlcons_false below).
 */
typedef struct pibm_params {
    int32_t my;              /* MY (even)                                      */
    int32_t mz;              /* MZ (0 -> my)                                   */
    double  lybyd;           /* LYBYD: box length / diameter                   */
    double  dbydx;           /* DBYDX: diameter / dx (used by Re<1 dt limit)   */
    double  dia_phys;        /* DIA_PHYS                                       */
    double  vis;             /* VIS                                            */
    double  re;              /* RE                                             */
    double  cfl;             /* CFL                                            */
    double  cfl_max;         /* CFL_MAX                                        */
    double  vfl;             /* VFL                                            */
    double  dr;              /* DR (reversal-point offset, grid units)         */
    double  f1, f2;          /* F1, F2 (surface point density)                 */
    double  flo_ang[3];      /* FLO_ANG (degrees)                              */
    double  mpg[3];          /* MPG (used when set_mpg)                        */
    double  rhof, rhos;      /* RHOF, RHOS                                     */
    double  coeff_rest;      /* COEFF_REST (DEM restitution)                   */
    int32_t ramp_frac_steps; /* RAMP_FRAC_STEPS (soft start of cf)             */
    int32_t discr_scheme;    /* PIBM_SCHEME_*                                  */
    int32_t limiter;         /* PIBM_LIMITER_*                                 */
    int32_t adaptive;        /* ADAPTIVE                                       */
    int32_t set_mpg;         /* SET_MPG (or SET_UMEAN)                         */
    int32_t initialize_zero; /* INITIALIZE_ZERO                                */
    int32_t dorpr;           /* DORPR                                          */
    int32_t revernorm;       /* REVERNORM                                      */
    int32_t include_frmeanfluid; /* INCLUDE_FRMEANFLUID                        */
    int32_t imove;           /* IMOVE (1 = moving particles, DEM)              */
    int32_t collision_softsphere; /* COLLISION_TYPE == 'softsphere'            */
    int32_t iscalon;         /* ISCALON (passive scalar)                       */
    double  pr_or_sc_nu;     /* PR_OR_SC_NU                                    */
    double  phisurf;         /* PHISURF                                        */
    double  phistream;       /* PHISTREAM                                      */
    int32_t rk3;             /* RK3: 3-stage Runge-Kutta (coef, itrmax = 3, initialize_flo.F90:861-877); 0 = AB2/CN */
    /* Flags of the reference that select code this engine does not run.  They
     * are part of the struct so that a host copies its namelist values in and
     * the engine refuses the run (PIBM_ERR_ARG) instead of silently running
     * another algorithm; 0 is the only accepted value of each. */
    int32_t dobnd;           /* DOBND (1 = T): surface-point forcing calc_bnd_forcing, boundary_condition.F90:615,902-1102 */
    int32_t aliasflag;       /* ALIASFLAG (1 = 2/3 dealiasing of the nonlinear term, nl.F90:146)                         */
    int32_t nlcons_false;    /* 1 when NLCONS = F (non-conservative pressure gradient, boundary_condition.F90:1831-1880) */
    int32_t reserved[4];
} pibm_params;

/* Particle list (the reference's sphr_center.inp after scaling by DBYDX:
 * initialize_flo.F90:1517-1520).  Positions are in grid units (node i sits at
 * x = i, i = 1..nx).  velbdy may be NULL (zero velocities). */
typedef struct pibm_particles {
    int32_t       nbody;
    const double *xc;        /* (nbody,3) column-major                        */
    const double *velbdy;    /* (nbody,3) column-major, or NULL               */
} pibm_particles;

/* Borrowed view of the evolving state (restart records of
 * restart_funcs.F90:265-306: t, dt, umean, cf, u, nl, mpg, p). */
typedef struct pibm_state_view {
    double *u;               /* complex (nx+1,my2,mz,3) interleaved           */
    double *nl;              /* complex (nx+1,my2,mz,3) interleaved           */
    double *p;               /* complex (nx,my2,mz) interleaved               */
    double  umean[3];
    double  mpg[3];
    double  ufmean[3];       /* previous-step fluid mean (for dufmeandt)      */
    double  t, dt, cf;
} pibm_state_view;

/* Per-step diagnostics (what the reference prints each step). */
typedef struct pibm_step_report {
    double dt, t, cf;
    double umax;             /* max |u| used for the CFL check                */
    double divmax;           /* check_divergence, steptheflow.F90:219-240     */
    double ufmean[3], usmean[3], umean[3];
    double mpg[3], frmean[3];
    double pres_total[3], visc_total[3];
    double norm_drag, ferror;
    double pres_drag, visc_drag, total_drag;
    double mixmeanslipmod;
    int64_t nrpr_active_total;
    double heat_ratio;       /* scalar: phi(x + Lx) = phi(x) / heat_ratio (1 without scalar) */
    double nusselt;          /* scalar: nusselt_avg(3) of bcsetscal, bc_scalar.F90:361-363 */
} pibm_step_report;

/* Static description of a handle's grid and geometry. */
typedef struct pibm_info {
    int32_t nx, my, mz, my2, nbody, nbnd;
    double  dx, dt, radbdy, maxvolfrac;
    int64_t count_solid, count_fluid;
    int32_t npts_active;       /* active reversal points over all spheres     */
    int32_t kernels_per_step;  /* kernels one step launches                   */
} pibm_info;

typedef struct pibm_handle pibm_handle;

/* initflo (initialize_flo.F90:61-1013) for input_type='default':
 * grid, wavenumbers, AB2 coefficients, surface points (quadgener,
 * geom_init.F90:44-242), solid mask (grid_nodes_insphere,
 * dependent_functions.F90:783-963), DEM neighbour search
 * (collision_mod.F90:807-1062) and active reversal points
 * (update_nrpr_array, dependent_functions.F90:966-1051), initial dt. */
int  pibm_create(const pibm_params *prm, const pibm_particles *parts, pibm_handle **out);
int  pibm_info_get(pibm_handle *h, pibm_info *info);
/* Copy a state in (reference layout); the real-space AB2 history is rebuilt. */
int  pibm_set_state(pibm_handle *h, const pibm_state_view *s);
/* One rks iteration of the driver loop (dtibm_main_scal_flo.F90:426-527):
 * compute_new_timestep(rks) -> nonlinear(rks) -> bcset(rks) -> velstep(rks). */
int  pibm_step(pibm_handle *h, int rks, pibm_step_report *rep);
/* nsteps steps without per-step host synchronisation (graph-launched). */
int  pibm_run(pibm_handle *h, int nsteps, pibm_step_report *last);
/* nsteps graph-launched steps (as pibm_run) timed with CUDA events recorded on
 * the handle's stream around the launches: *total_ms = device time. */
int  pibm_run_timed(pibm_handle *h, int nsteps, pibm_step_report *last, double *total_ms);
/* nsteps steps launched without graphs, timed with CUDA events recorded on
 * the handle's stream: *total_ms = first-to-last event time; phase_ms[q]
 * (q < nphase <= PIBM_NPHASE) = summed duration of phase q over the steps.
 * One host synchronisation at the end. */
#define PIBM_NPHASE 7   /* 0 u,p,omega,grad p -> real  1 nonlinear + IBM field  2 drag+mpg  3 reversal+spread  4 forcing FFT  5 x-lines  6 passive scalar */
int  pibm_run_profiled(pibm_handle *h, int nsteps, pibm_step_report *last,
                       double *total_ms, double *phase_ms, int nphase);
/* Kernel slots of one flow step, in launch order (the same launches as the
 * step graphs, run serially on the handle's stream).  Slots a step does not
 * launch (no spheres, no active reversal points) time as zero.  With moving
 * particles the DEM and geometry-rebuild kernels are not in any slot (the
 * spreading rebuild is in PIBM_K_SPREAD); with the passive scalar its
 * kernels run after PIBM_K_SCAL_D, outside every slot. */
#define PIBM_K_A0      0   /* fields to real space          compute_new_timestep, calc_pressure, compute_omega, calc_pgrad */
#define PIBM_K_SCAL_A  1   /* CFL dt, t, cf, means          compute_new_timestep tail                                    */
#define PIBM_K_FLUX    2   /* x-flux differences            form_nl                                                     */
#define PIBM_K_NL      3   /* nonlinear term + IBM field Q  nonlinear, calc_visc                                        */
#define PIBM_K_DRAG    4   /* surface quadrature            calc_pres_visc_drag                                         */
#define PIBM_K_SCAL_B  5   /* drag totals, mpg, force       compute_mpg_at_n                                            */
#define PIBM_K_REV     6   /* reversal-point forcing        calc_inner_reversal_forcing                                 */
#define PIBM_K_SCAL_C  7   /* frmean                        bcset                                                       */
#define PIBM_K_SPREAD  8   /* spreading onto solid nodes    calc_inner_reversal_forcing (spread loop)                   */
#define PIBM_K_FF      9   /* forcing r2c                   bcset                                                       */
#define PIBM_K_LINES  10   /* x-line solves                 velstep: pressure, ustep, divcorr                           */
#define PIBM_K_SCAL_D 11   /* umean update, status          velstep                                                     */
#define PIBM_NKERNEL  12
/* nsteps steps launched serially with a CUDA event pair around every kernel
 * slot: kernel_ms[k] (k < nkernel <= PIBM_NKERNEL) = summed device time of
 * slot k over the steps, *total_ms = first slot start to last slot end.  No
 * counterpart in the reference (its per-phase CPU timers print wall time,
 * dtibm_main_scal_flo.F90:552-566). */
int  pibm_kernel_times(pibm_handle *h, int nsteps, double *total_ms, double *kernel_ms, int nkernel);
/* Name of kernel slot k ("k_a0", ...), NULL outside [0, PIBM_NKERNEL). */
const char *pibm_kernel_name(int k);
int  pibm_get_state(pibm_handle *h, pibm_state_view *s);
/* pres, visc, force: (nbody,3) column-major, as global_data.F90:115-117;
 * xc, vel: positions (grid units) and velocities.  Any pointer may be NULL. */
int  pibm_get_particles(pibm_handle *h, double *pres, double *visc, double *force,
                        double *xc, double *vel);
/* Passive scalar (ISCALON = 1; scalstep, SRC/SCALAR/stepthescalar.F90:51-94):
 * phif complex (nx+1,my2,mz) interleaved in the reference layout (plane nx+1
 * is phif(1)/heat_ratio), flux_body (nbody) = sum over surface points of
 * grad phi . n (calc_bndrev_data), ratios[0..2] = heat_ratio,
 * heat_ratio_old, Nusselt number.  Any pointer may be NULL. */
int  pibm_get_scalar(pibm_handle *h, double *phif, double *flux_body, double *ratios);
/* Desired mean particle and fluid velocities of a restarted run (the u
 * restart file's usmean_des, ufmean_des: restart_funcs.F90:450-452). */
int  pibm_set_desired_means(pibm_handle *h, const double usmean_des[3], const double ufmean_des[3]);
/* The scalar's nonlinear term of the last step, nlphif complex (nx+1,my2,mz)
 * interleaved (plane nx+1 = nlphif(1)/heat_ratio of that step). */
int  pibm_get_scalar_nl(pibm_handle *h, double *nlphif);
/* Scalar restart (read_unformatted, restart_funcs.F90:560-590): phif and
 * nlphif complex (nx+1,my2,mz) interleaved, ratios[0..1] = heat_ratio,
 * heat_ratio_old.  Call after pibm_set_state. */
int  pibm_set_scalar(pibm_handle *h, const double *phif, const double *nlphif, const double *ratios);
/* Moving particles (IMOVE = 1): the DEM lists of the last step in the
 * reference layout NEIGHBOURS / PN / PV (nbody, maxn) column-major
 * (dem_mod.F90; collision_mod.F90:807-1062, soft_sphere_coll.F90:120-420):
 * column 1 holds the count (PV: 1), columns 2.. the 1-based particle numbers
 * (-1 after the last; PV: the contact flags, 0 after the last).  maxn = 37
 * (MAXNEIGHBORS = MN + 1 + NWALLS) always suffices; PIBM_ERR_ARG if a list
 * does not fit or the run has fixed particles.  Any pointer may be NULL. */
int  pibm_get_contacts(pibm_handle *h, int32_t maxn, int32_t *neigh, int32_t *pn, int32_t *pv);
/* Surface quadrature points (quadgener, geom_init.F90:44-242): bnd (nbnd, 3)
 * row-major, the unit direction of point l.  Sphere m's surface point l sits
 * at xc_m + radbdy*bnd_l and its inner and outer reversal points at
 * xc_m + (radbdy -+ dr)*bnd_l (grid units). */
int  pibm_get_surface_points(pibm_handle *h, double *bnd);
/* Frame motion of a moving-particle run (IMOVE = 1): frame_vel(3), frame_pos(3)
 * of the reference (updated in velstep, steptheflow.F90:99-103; written to
 * RUN_NAME_sphere_config_N.rst, restart_funcs.F90:253-254, and read back on
 * restart, initialize_flo.F90:1891-1898).  Fixed runs keep 0 and 1.
 * pibm_set_frame: at a step boundary; either pointer of get may be NULL. */
int  pibm_get_frame(pibm_handle *h, double frame_vel[3], double frame_pos[3]);
int  pibm_set_frame(pibm_handle *h, const double frame_vel[3], const double frame_pos[3]);
/* Active reversal-point flags (part_array(m)%if_rev), (nbnd, nbody) column-major. */
int  pibm_get_if_rev(pibm_handle *h, uint8_t *if_rev);
/* Solid mask fluid_atijk(1:nx,1:my,1:mz) as 0/1 bytes, x fastest. */
int  pibm_get_fluid_mask(pibm_handle *h, uint8_t *mask);
void pibm_destroy(pibm_handle *h);
const char *pibm_last_error(void);

/* ---- plane transforms (the reference's ff2rc / ff2cr,
 *      fftw_interface.F90:48-133), batched over nplanes planes ----
 * ff2rc: real (my,mz) -> complex (my2,mz), forward e^{-i}, scaled 1/(my*mz).
 * ff2cr: complex (my2,mz) -> real (my,mz), inverse e^{+i}, unscaled; the
 *        imaginary parts of the ky=0 and ky=Nyquist columns are ignored after
 *        the z transform (FFTW / numpy irfft2 semantics).
 * Host pointers; y fastest within a plane, planes contiguous. */
int  pibm_ff2rc(int my, int mz, int nplanes, const double *a, double *b);
int  pibm_ff2cr(int my, int mz, int nplanes, const double *a, double *b);

/* Allocation-free ff2cr on DEVICE buffers.  No counterpart in the reference
 * (its ff2cr works on host arrays through FFTW plans); it exists for callers
 * that keep their spectral fields on the GPU and cannot allocate per call:
 * pibm_ff2cr above allocates and frees three device buffers each time, and
 * cudaFree waits for the whole device, which stalls a host that runs other
 * streams, and cudaMalloc competes with a host whose device memory is already
 * carved into its own pool (a caching allocator, pre-registered buffers).
 * This entry point allocates nothing: the only data it needs besides a and b
 * is a twiddle table kept in a static device array of 320 complex doubles
 * (5 KiB per GPU, held until the process exits) that covers every supported
 * size, my = mz in {32, 64, 96, 128}; larger or other sizes are rejected with
 * PIBM_ERR_ARG.  Set-up: the FIRST call on each device looks up that array's
 * address, writes the whole table with a blocking copy and waits for it, so
 * make that first call before starting any stream capture.  A device reset
 * (cudaDeviceReset) gives the device a new context whose copy of the array
 * starts zeroed; the first call after it writes the table again (the cached
 * set-up is keyed on the context's unique id).  After the set-up the table is
 * only read, so nothing in it must start at zero and calls on different
 * streams share it safely.
 * d_a: nplanes * mz * (my/2+1) complex (interleaved doubles); d_b: nplanes *
 * mz * my doubles; both device pointers with the layout of pibm_ff2cr.  The
 * transform is enqueued on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and the call returns without waiting for it. */
int  pibm_ff2cr_noalloc(int my, int mz, int nplanes, const double *d_a, double *d_b, void *stream);

/* ---- discrete adjoint (no counterpart in the reference) ----
 * K = nsteps AB2 steps from the handle's current state, then the exact
 * discrete adjoint of the step sequence for the objective
 *     J = (1/K) sum_{n=1..K} e . sum_m (pres_m + visc_m),
 * the summed pressure + viscous surface force of calc_pres_visc_drag
 * (boundary_condition.F90:1481-1645) evaluated inside step n and projected on
 * e = direction[3].  Returns dJ/dxc in g_xc (nbody,3) column-major (grid
 * units, the layout of pibm_particles.xc) and dJ/dmpg in g_mpg[3].  The
 * forward trajectory is kept as checkpoints every checkpoint_every steps and
 * recomputed segment by segment in the reverse sweep (the last segment's
 * fields are kept by the forward pass itself); checkpoint_every <= 0 takes
 * as many steps per segment as 80% of the free device memory holds, i.e. no
 * recomputation when the whole run fits.  The handle ends at the state after
 * the K steps, as after pibm_run(h, K).
 * Supported runs: fixed spheres, AB2 or RK3 (with RK3 the objective reads
 * the drag of each step's last stage, the driver's record), SET_MPG (imposed
 * mean pressure gradient), ADAPTIVE = F (fixed dt), DORPR, no scalar;
 * otherwise PIBM_ERR_ARG.  The solid mask, the active reversal
 * points and the upwind branches are those of the forward run (the gradient
 * of the piecewise-smooth map on the trajectory's branch). */
typedef struct pibm_adjoint_report {
    double J;                 /* the objective */
    double forward_ms;        /* device time of the K forward steps with checkpoints */
    double reverse_ms;        /* device time of the reverse sweep: recomputation + adjoint steps */
    int32_t nsteps, checkpoint_every;
    int32_t adjoint_kernels_per_step;   /* own kernel launches per reverse step (without the recomputed forward step) */
    int32_t reserved;
} pibm_adjoint_report;
int  pibm_adjoint_run(pibm_handle *h, int nsteps, int checkpoint_every, const double direction[3],
                      double *g_xc, double g_mpg[3], pibm_adjoint_report *rep);
/* The same reverse sweep driven step by step by the host (which keeps its
 * own checkpoints): pibm_adjoint_begin zeroes the adjoint state for an
 * objective over nsteps steps; each pibm_adjoint_step reverses one step n =
 * nsteps, nsteps-1, ..., 1 in that order and expects the handle to hold the
 * state before step n (pibm_set_state of the host's copy, or the state its
 * recomputation left): it runs step n to form the step's fields, then the
 * adjoint of step n, and leaves the handle after step n; pibm_adjoint_end
 * returns dJ/dxc and dJ/dmpg.  Same run restrictions as pibm_adjoint_run. */
int  pibm_adjoint_begin(pibm_handle *h, int nsteps, const double direction[3]);
int  pibm_adjoint_step(pibm_handle *h);
int  pibm_adjoint_end(pibm_handle *h, double *g_xc, double g_mpg[3]);

/* ---- tile shapes (no counterpart in the reference) ----
 * pibm_create times the x-line solve kernel with 4 and 8 (ky,kz) lines per
 * CTA on the run's own grid, on scratch copies of the state (fixed
 * particles: 6 whole steps after 2; moving particles: 10 launches after a
 * warm-up, each behind the forcing transform that precedes it in the step),
 * and keeps the faster; up to 128 the 4-line width is a persistent kernel
 * fed by tensor-map copies.  Results do not depend on the choice.
 * pibm_get_tuning returns the width in use and the mean time per timed unit
 * (a step, or a forcing transform + line kernel pair) of each candidate
 * (ms[0]: 4, ms[1]: 8);
 * pibm_set_tuning overrides it (4 or 8) before the next pibm_run (the
 * handle's step graphs are recaptured; batch graphs are not). */
int  pibm_get_tuning(pibm_handle *h, int32_t *lines_per_cta, double lines_ms[2]);
int  pibm_set_tuning(pibm_handle *h, int32_t lines_per_cta);

/* ---- measurement (no counterpart in the reference) ----
 * FP64 arithmetic peak of the current device: chains of fused multiply-adds
 * on 8 CTAs of 256 threads per SM, best of 5 event-timed runs (about 0.5 s).
 * tflops = 2 * fma count / time; ms (optional) = the best run's time. */
int  pibm_fp64_peak(double *tflops, double *ms);
/* Check of the engine's reciprocal division (no counterpart in the
 * reference): for every pair (a[i], b[j]) the quotient that the kernels form
 * from b's reciprocal (a*y and one FMA correction, y = 1/b) is compared bit
 * for bit with a / b on the device; mismatches = the number that differ. */
int  pibm_qdiv_check(const double *a, long long n, const double *b, int nb, long long *mismatches);

/* ---- batched independent realizations (the MIS ensemble of
 *      sample_inputs/set_mis_3d, run as one graph-captured launch stream) ---- */
typedef struct pibm_batch pibm_batch;
int  pibm_batch_create(int n, const pibm_params *prm, const pibm_particles *parts, pibm_batch **out);
/* nsteps steps of every member: one CUDA graph launch per step.  Members
 * with fixed spheres and no scalar that share the grid size and the scheme
 * (AB2 or RK3) step through one launch per kernel, the members along
 * gridDim.z; the other members' steps are independent branches that the GPU
 * runs beside them.  Each member's results are bitwise those of stepping it
 * alone.  Members may also be stepped on their own between batch runs. */
int  pibm_batch_run(pibm_batch *b, int nsteps);
/* Device time (CUDA events on the batch stream) of nsteps steps of every
 * member: sequential == 1 runs the plain per-realization loop (member after
 * member, each replaying its own step graphs); sequential == 0 runs the batch
 * graph; sequential == 2 runs a batch graph in which every member's step is
 * its own branch (no shared launches).  *ms = elapsed milliseconds; members
 * advance nsteps steps either way. */
int  pibm_batch_time(pibm_batch *b, int nsteps, int sequential, double *ms);
pibm_handle *pibm_batch_member(pibm_batch *b, int i);
void pibm_batch_destroy(pibm_batch *b);

#ifdef __cplusplus
}
#endif
#endif /* PIBM_H */
