// engine.cuh -- device-side data structures of the time-step engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pibm {

// Per-run constants passed by value to every kernel.
struct Geo {
    int nx, my, mz, my2;
    int PS;             // complex elements per spectral plane (my2*mz)
    int RS;             // real elements per physical plane (my*mz)
    double dx, dx2, rdx2, dx3, vis, nrm;   // nrm = float(my*mz) as in ff2rc
    double c1, c2, c3, c4;   // coef(rks, 1:4) of the stage this Geo is launched for
    int scheme, limiter, include_frmeanfluid, revernorm, set_mpg, adaptive;
    int dt_update;      // this stage takes the new dt (rks == itrmax, dependent_functions.F90:1246-1250)
    double cfl_max, ramp_frac_time, ucharmod, char_length, voldom, maxvolfrac, mean_volfrac, rhof, rhos;
    long long count_fluid, ncell;
    int plane_ctas;     // CTAs per plane in the plane kernels
    int lines_lt;       // x-line tile width of k_lines (4 or 8; 0 = the size's default), set by the autotuner
    int flux_seg;       // planes per thread of k_flux (flux_segment)
    double ufmean_des[3], usmean_des[3], usmean_act[3];
    // particles (moving: the geometry arrays below are rebuilt on the device
    // every step and npts is the capacity nbody*nbnd; Scal::npts is the count)
    int nbody, nbnd, npts, moving;
    double rb, ri, ro, dr, da1, sphere_vol;
    // device arrays (read-only)
    const double2 *tw;          // e^{-2 pi i m/my}, m < my (my == mz)
    const double *ky, *kz, *w2; // wavenumbers
    const uint8_t *fluid;       // [i][k][j] 1 = fluid
    const double *xc;           // (nbody,3) column-major
    const double *vel;          // (nbody,3)
    const double *bnd, *cd;     // (3,nbnd)
    const int *pt_m, *pt_l;     // active reversal points
    const double *da2;          // per sphere
    const int *sp_node, *sp_ptr, *sp_ent;   // spreading map
    int sp_nnodes;
    // passive scalar (iscalon)
    int scal;
    double gamma_s, phisurf, phistream;
    int nsev;                        // scalar reversal-point evaluations
    const int *sev_m, *sev_l, *sev_c;
    const double *sev_x;
    const int *ssp_node, *ssp_ptr, *ssp_ent;
    int ssp_nnodes;
};

// Evolving scalars of a run (one struct in device memory).
struct Scal {
    double umean[3], mpg[3], frmean[3], frmeanfluid[3];
    double ufmean[3], ufmean_old[3], usmean[3], dufmeandt[3];
    double dt, t, cf, cforig, umax, mixmeanslipmod;
    double pres_total[3], visc_total[3];
    double norm_drag, ferror, fold, pres_drag, visc_drag, total_drag;
    double frame_accln[3];
    unsigned long long divmax_bits;
    int status;
    unsigned lines_done;   // persistent x-line kernel: blocks finished (0 between launches)
    long long nsteps;
    // passive scalar: phi(x + Lx) = phi(x) / heat_ratio
    double heat_ratio, heat_ratio_old, heat_ratio_new, flux_global, nusselt;
    // particle geometry of the current step (constant for fixed particles):
    // solid/fluid node counts, solid fraction, active reversal points, mean
    // particle velocity; frame motion of moving particles
    long long count_solid, count_fluid;
    double maxvolfrac;
    int npts;
    int dem_substeps;
    int nsev;
    unsigned lines_next;   // persistent x-line kernel: next tile ticket (0 between launches)
    double usmean_act[3], frame_vel[3], frame_pos[3];
};



// Moving particles (IMOVE = 1): soft-sphere DEM state and the scratch of the
// per-step geometry rebuild.  Particle indices are 0-based; list order is the
// reference's (collision_mod.F90 NEIGHBOURS / PN / PV).
struct Mov {
    int N, maxn, soft, max_factor;
    int cx, cy, cz, ncell;            // coarse grid nodes per direction; physical cells 2..c
    double dxc, dyc, dzc, LXs, LYs, LZs, XL, YL, ZL;
    double kn, eta_n, rad, pmass, pvol, rhof, dtsolid, max_radius;
    double *pos, *pos_old, *vel, *vel_old;    // [3*l + d], physical units
    int *pijk;                                 // [3*l + d]
    int *neigh, *ncnt;                         // NEIGHBOURS: [l*maxn + q], q < ncnt[l]
    int *pn, *pv, *pncnt;                      // contact lists at the start of a sub-step
    int *pn2, *pv2, *pncnt2;                   // contact lists written by the sub-step
    int *cstart, *clist;                       // particles per coarse cell, ascending
    int *factor;                               // [0] sub-steps of this flow step
    double *dts;                               // [0] sub-step size
    double *xc, *vel_ibm;                      // the step's xc (grid units) and velbdy, (nbody,3)
    uint8_t *fluid, *revflag;                  // solid mask; reversal-point activity [m*nbnd + l]
    int *nrpr, *ptoff, *pt_m, *pt_l;
    double *da2;
    int *spcnt, *spbuf;                        // spreading buckets: count and entries per node
    int kmax;                                  // bucket capacity per node
    // passive scalar with moving particles: reversal-point evaluations per
    // sphere and in total, and the scalar forcing's spreading buckets
    int *sev_cnt, *sev_off, *sev_m, *sev_l, *sev_c;
    double *sev_x;
    int *sspcnt, *sspbuf;
};

// Device buffers of one run.
// The flow step's buffers (what the step kernels read and write).
struct FlowBufs {
    double2 *u, *p, *nl[2], *ff;
    double *ubcp, *pbcp, *Q, *omega, *pgr, *fr, *Dx;
    double *part, *pres, *visc, *ptot, *force, *rec, *rz, *dpart, *blockpart;
    Scal *sc;
};

struct DevBufs : FlowBufs {
    // passive scalar: spectral phi, nlphi (two steps), ffphi over planes 1..nx;
    // real phi (planes 1..nx) and its c2r image plane nx+1; real nlphi of
    // the two steps, diffusion and gradient over planes 1..nx+1; forcing and
    // x-flux difference over planes 1..nx
    double2 *phif, *nls[2], *ffs;
    double *phr, *phimg, *nlr[2], *sdf, *gph, *sfr, *dsx;
    double *spart, *sctb, *sfd, *sdpart, *flux_body;
    Mov mov;   // moving particles (Geo::moving)
};

// One realization of a fused batch step (several runs of one grid size
// stepped by the same kernel launches, one launch per kernel with the runs
// along gridDim.z): its constants, its buffers, the nl buffer the step
// writes (nl[cur]; onl = nl[cur ^ 1]) and its reversal-forcing block count.
struct Member {
    Geo g;
    FlowBufs b;
    int cur;
    int nbk;
};

// The members of one fused launch, passed by value as a __grid_constant__
// kernel parameter (constant-bank loads indexed by blockIdx.z; 12.5 KB of the
// 32 KB parameter limit).  Larger groups are split into launches of kFuseMax.
constexpr int kFuseMax = 16;
struct MemberSet {
    Member m[kFuseMax];
};

// Planes one thread of k_flux marches through (a sliding window along x; a
// segment re-reads two planes on either side).  Short segments give grids up
// to 128^3 enough threads to keep loads in flight when the flux is on the
// step's critical path (k_flux 41 -> 35 us at 128^3); with the passive
// scalar's kernels running beside it the GPU is full, and long segments, which
// re-read less, give the shorter step.
inline int flux_segment(int n, bool scalar) { return (scalar || n >= 256) ? 32 : 8; }

// Launch extents of a fused batch step: runs in the group and the largest
// sphere count, reversal-forcing block count and spreading node count among
// them; the x-line tile width and the x-flux segment all of them use.
struct BatchShape {
    int nz, max_nbody, max_nbk, max_spn, lines_lt, flux_seg;
};

// Side streams of one run: the x flux and the nonlinear term need only the
// real fields of k_a0, so compute_new_timestep's scalars (k_scal_a), the drag
// quadrature and mpg run beside them on `side`, and the passive-scalar step,
// once those scalars are known, on `scal` (k_scal_a then runs first, on the
// main stream; with moving particles the scalar waits for the step's new
// geometry); without a scalar the frmean sums (k_scal_c) run on `side`
// beside the spreading.
struct StepStreams {
    cudaStream_t side = nullptr, scal = nullptr;
    cudaEvent_t fork = nullptr, drag_done = nullptr, scal_done = nullptr;
    cudaEvent_t geo_done = nullptr;   // moving particles: the step's geometry is rebuilt
    cudaEvent_t rev_done = nullptr, frmean_done = nullptr;   // k_scal_c beside k_spread
};

// Discrete adjoint of the AB2 step (fixed spheres, imposed mpg, fixed dt).
// Scalars of the reverse sweep in device memory.
struct AdjScal {
    double lumean[3];    // lambda of umean
    double lfrmean[3];   // lambda of frmean of the step being reversed
    double gmpg[3];      // dJ/dmpg
    double J;            // sum over the forward steps of e . (visc_total - pres_total)
    int status;          // PIBM_ERR_TIMEOUT / PIBM_ERR_PIVOT from an adjoint kernel
    int pad;
};
// Adjoint work arrays.  Spectral arrays are [comp][i][kz][ky] like u; real
// arrays [comp][i][transform-order plane] like ubcp.
struct AdjBufs {
    double2 *lu, *lp, *lnl;              // lambda of the state (u, p, nl) after the step being reversed
    double2 *lu2, *lp2;                  // lambda of the state before it (being formed)
    double2 *lnl_new, *lonl, *lff;       // lambda of the step's new nl, of its onl (-> lnl of the earlier state), of ff
    double2 *T;                          // 10 components: adjoint plane transforms of the real lambdas
    double *lfr, *lubcp, *lQ, *lpgr, *lpbcp, *lomega;   // real lambdas (3,3,3,3,1,3 components)
    double *W8;                          // 8 real components: products and x-flux lambdas of the nonlinear term
    double *gxc;                         // dJ/dxc (nbody,3) column-major
    AdjScal *as;
};

}  // namespace pibm
