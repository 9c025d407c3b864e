// kernels.cu -- sm_100a FP64 kernels of one AB2 time step.
//
// Data layout in HBM (chosen for the two sweep directions of the step):
//   spectral fields  double2 [comp][i][kz][ky]   (plane i contiguous, pitch my2)
//   physical fields  double  [comp][i][...]      (one plane = my*mz doubles in the
//                    order the plane transform leaves them: real_off(z, y))
// so every plane load/store is a straight contiguous copy, and for fixed i the
// (ky,kz) lines of a plane are contiguous (line-kernel loads are coalesced
// across consecutive lines).  The periodic image plane nx+1 of the reference
// is never stored; x indices wrap instead.
//
// Step pipeline (reference routines in brackets):
//   k_a0      10 c2r per plane: ubcp (+umean), pbcp, omega, grad p (without mpg);
//             fluid/solid means and max|u|       [compute_new_timestep, calc_pressure,
//                                                   compute_omega, calc_pgrad]
//   k_scal_a  CFL dt, t, cf (soft start), ufmean, mean slip   [compute_new_timestep]
//   k_nl      products + x flux, 9 r2c -> nl; 3 c2r -> Q = -c3 nl - c4 onl - c12 diffn
//                                                  [form_nl, nonlinear, calc_visc]
//   k_drag    per-sphere surface quadrature of p and omega     [calc_pres_visc_drag]
//   k_scal_b  pres/visc totals, mpg, per-sphere force, drag diagnostics   [compute_mpg_at_n, bcset]
//   k_rev     reversal-point force per active point            [calc_inner_reversal_forcing]
//   k_scal_c  frmean
//   k_spread  gather of point forces onto solid nodes in reference order
//   k_ff      fr - frmean -> ff (3 r2c)                        [bcset]
//   k_lines   pressure -> ustep -> divcorr per (ky,kz) line     [velstep]
//   k_scal_d  umean update, divergence, status                 [velstep]
// The IBM force needs -c3 nl - c4 onl - c12 diffn only at the inner reversal
// points; by linearity of the transform and of the interpolation it is formed
// once in spectral space (Q) instead of three separately interpolated fields.
#include <algorithm>

#include "step_common.cuh"
#include "line_solve.cuh"
#include "lines_pipe.cuh"
#include "../../include/pibm.h"

namespace pibm {

void enqueue_scalar(const Geo &g, DevBufs &b, int cur, cudaStream_t s);
int scalar_kernels_per_step(const Geo &g);
void enqueue_moving(const Geo &g, const Mov &m, Scal *sc, const double *pres, const double *visc, cudaStream_t s);
void enqueue_spread_dyn(const Geo &g, const Mov &m, const double *rec, const double *rz, double *fr, Scal *sc, cudaStream_t s);
int moving_kernels_per_step(const Mov &m);

// ============================================================================
// k_a0: 10 c2r per plane (dependent_functions.F90:1085-1122, 336-349;
// boundary_condition.F90:1648-1765, 1817-1896).  The x differences of omega and
// grad p are taken on the spectral planes before the transform (linear).
// part[i*12 + q]: q 0-2 fluid sums, 3-5 solid sums, 6-8 all sums, 9-11 max |u|.
// ============================================================================
template <int N>
__device__ __forceinline__ void b_a0(const Geo &g, const double2 *__restrict__ u, const double2 *__restrict__ p,
                                                   double *__restrict__ ubcp, double *__restrict__ pbcp,
                                                   double *__restrict__ omega, double *__restrict__ pgr,
                                                   Scal *__restrict__ sc, double *__restrict__ part) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RSP = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    __shared__ double scr[32 * 3];
    __shared__ uint64_t mb;
    if (threadIdx.x == 0) mbar_init(&mb, 1);
    load_tw<N>(tws, g);
    __syncthreads();
    grid_dep_wait();   // the twiddles above are set-up data; the fields come from earlier kernels
    const int i = blockIdx.x / L::C, rank = blockIdx.x % L::C, nx = g.nx;
    const int im = (i - 1 + nx) % nx, ip = (i + 1) % nx;
    const size_t roff = (size_t)rank * L::RL;
    const TwT tw{tws, N};
    const double tdx = 2.0 * g.dx, rtdx = 1.0 / tdx;   // divisor and reciprocal for qdiv
    const double2 *U0 = u + (size_t)i * PS, *U1 = u + ((size_t)nx + i) * PS, *U2 = u + ((size_t)2 * nx + i) * PS;
    const double2 *Pp = p + (size_t)i * PS;
    const size_t slot = ((size_t)i * L::C + rank) * 12;
    {
        const int t = blockIdx.y;
        if (t < 4) {
            // a plain copy of u_t or p: the CTA's MC columns of every kz row as N
            // bulk copies into the padded rows, all in flight at once; rank 0's
            // Nyquist column (slot MC) with plain loads beside them
            const double2 *src = t == 0 ? U0 : t == 1 ? U1 : t == 2 ? U2 : Pp;
            uint32_t phase = 0;
            if (threadIdx.x < 32)
                bulk_load_rows(buf, L::PZ * 16, src + rank * L::MC, (size_t)my2 * 16, L::MC * 16, N, &mb);
            if (rank == 0)
                for (int kz = threadIdx.x; kz < N; kz += L::T) buf[kz * L::PZ + L::MC] = src[kz * my2 + L::M];
            load_wait(&mb, phase, sc);
        } else {
            // omega and grad p: spectral differences formed from plain loads
#pragma unroll 4
            for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
                const int kz = e / L::PZ, jl = e - kz * L::PZ;
                if (jl == L::MC && rank != 0) continue;
                const int j = cl_col<N>(jl, rank), ge = kz * my2 + j;
                const double ky = g.ky[j], kzv = g.kz[kz];
                double2 f;
                if (t == 4) {   // wy*u3 - wz*u2
                    const double2 a = U2[ge], b = U1[ge];
                    f = make_double2(-ky * a.y - (-kzv * b.y), ky * a.x - kzv * b.x);
                } else if (t == 5) {   // wz*u1 - d(u3)/dx
                    const double2 a = U0[ge];
                    const double2 hp = u[((size_t)2 * nx + ip) * PS + ge], hm = u[((size_t)2 * nx + im) * PS + ge];
                    const double2 d = make_double2(qdiv(hp.x - hm.x, tdx, rtdx), qdiv(hp.y - hm.y, tdx, rtdx));
                    f = make_double2(-kzv * a.y - d.x, kzv * a.x - d.y);
                } else if (t == 6) {   // d(u2)/dx - wy*u1
                    const double2 a = U0[ge];
                    const double2 hp = u[((size_t)nx + ip) * PS + ge], hm = u[((size_t)nx + im) * PS + ge];
                    const double2 d = make_double2(qdiv(hp.x - hm.x, tdx, rtdx), qdiv(hp.y - hm.y, tdx, rtdx));
                    f = make_double2(d.x - (-ky * a.y), d.y - ky * a.x);
                } else if (t == 7) {
                    const double2 a = p[(size_t)ip * PS + ge], b = p[(size_t)im * PS + ge];
                    f = make_double2(qdiv(a.x - b.x, tdx, rtdx), qdiv(a.y - b.y, tdx, rtdx));
                } else if (t == 8) { const double2 a = Pp[ge]; f = make_double2(-a.y * ky, a.x * ky); }
                else { const double2 a = Pp[ge]; f = make_double2(-a.y * kzv, a.x * kzv); }
                buf[e] = f;
            }
        }
        __syncthreads();
        cl_c2r<N>(buf, tw, rank);
        if (t < 3) {
            // u + umean; fluid, solid and total sums and max |u| of this CTA's rows
            const double um = sc->umean[t];
            double *b = (double *)buf;
            const uint8_t *fl = g.fluid + (size_t)i * RSP + roff;
            double sf = 0.0, ss = 0.0, sa = 0.0, mx = kSmallD;
            for (int e = threadIdx.x; e < L::RL; e += L::T) {
                if (e % (N + 2) >= N) continue;
                const double v = b[e] + um;
                b[e] = v;
                if (fl[e]) sf += v; else ss += v;
                sa += v;
                mx = fmax(mx, fabs(v));
            }
            double v3[3] = {sf, ss, sa};
            block_reduce_k<3>(v3, scr);   // the three sums of block_sum's tree, two barriers
            mx = block_max(mx, scr);
            if (threadIdx.x == 0) { part[slot + t] = v3[0]; part[slot + 3 + t] = v3[1]; part[slot + 6 + t] = v3[2]; part[slot + 9 + t] = mx; }
        }
        double *dst = t < 3 ? ubcp + ((size_t)t * nx + i) * RSP
                    : t == 3 ? pbcp + (size_t)i * RSP
                    : (t < 7 ? omega + ((size_t)(t - 4) * nx + i) * RSP : pgr + ((size_t)(t - 7) * nx + i) * RSP);
        if (threadIdx.x == 0) { bulk_store(dst + roff, buf, L::RBYTES); bulk_wait_read(); }
    }
}
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_a0(Geo g, const double2 *__restrict__ u, const double2 *__restrict__ p,
                                                   double *__restrict__ ubcp, double *__restrict__ pbcp,
                                                   double *__restrict__ omega, double *__restrict__ pgr,
                                                   Scal *__restrict__ sc, double *__restrict__ part) { b_a0<N>(g, u, p, ubcp, pbcp, omega, pgr, sc, part); }

// compute_new_timestep's scalar tail (dependent_functions.F90:1137-1280).
__device__ __forceinline__ void b_scal_a(const Geo &g, Scal *sc, const double *part) {
    __shared__ double scr[32 * 3];
    __shared__ double red[6];
    if (block_failed(sc)) return;
    {
        double a[3] = {0.0, 0.0, 0.0}, m[3] = {kSmallD, kSmallD, kSmallD};
        for (int i = threadIdx.x; i < g.nx * g.plane_ctas; i += blockDim.x)
#pragma unroll
            for (int d = 0; d < 3; ++d) { a[d] += part[(size_t)i * 12 + d]; m[d] = fmax(m[d], part[(size_t)i * 12 + 9 + d]); }
        block_reduce_k<3>(a, scr);
        block_reduce_k<3, true>(m, scr);
        if (threadIdx.x == 0)
            for (int d = 0; d < 3; ++d) { red[d] = a[d]; red[3 + d] = m[d]; }
    }
    __shared__ double vmean[3], upmax;
    if (g.moving) {
        // particle speed limit (dependent_functions.F90:1156-1164) and the mean
        // particle velocity (:1185-1193): the maximum in any order, the sums
        // serial over the spheres as in the reference (one thread per component)
        const int NB = g.nbody;
        double um = kSmallD;
        for (int m = threadIdx.x; m < NB; m += blockDim.x) {
            double s2 = 0.0;
            for (int d = 0; d < 3; ++d) s2 = __dadd_rn(s2, __dmul_rn(g.vel[m + d * NB], g.vel[m + d * NB]));
            um = fmax(um, sqrt(s2));
        }
        um = block_max(um, scr);
        if (threadIdx.x < 3) {
            const double *v = g.vel + (size_t)threadIdx.x * NB;
            double a = 0.0;
#pragma unroll 8
            for (int m = 0; m < NB; ++m) a = a + v[m];
            vmean[threadIdx.x] = a / (double)NB;
        }
        if (threadIdx.x == 0) upmax = um;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double umax = fmax(fmax(red[3], red[4]), red[5]);
    sc->umax = umax;
    double dtnew = sc->dt;
    if (umax * sc->dt / g.dx > g.cfl_max) dtnew = g.cfl_max * g.dx / umax;
    if (g.moving) {
        // the new dt is taken from the fluid speed, as the reference writes it
        if (upmax * sc->dt / g.dx > g.cfl_max) dtnew = g.cfl_max * g.dx / umax;
        for (int d = 0; d < 3; ++d) sc->usmean_act[d] = vmean[d];
    }
    for (int d = 0; d < 3; ++d) {
        sc->ufmean_old[d] = sc->ufmean[d];
        sc->ufmean[d] = red[d] / (double)sc->count_fluid;
        sc->dufmeandt[d] = -sc->cf * (sc->ufmean[d] - sc->ufmean_old[d]);
    }
    double ms[3];
    for (int d = 0; d < 3; ++d) {
        sc->usmean[d] = g.nbody > 0 ? (g.mean_volfrac * sc->usmean_act[d]) / g.mean_volfrac : 0.0;
        ms[d] = (1.0 - sc->maxvolfrac) * (sc->usmean[d] - sc->ufmean[d]);
    }
    sc->mixmeanslipmod = sqrt(ms[0] * ms[0] + ms[1] * ms[1] + ms[2] * ms[2]);
    if (g.adaptive && g.dt_update) sc->dt = dtnew;
    sc->t = sc->t + sc->dt * (g.c1 + g.c2);
    const double tempt = g.ramp_frac_time * (double)(float)(g.nx) * g.dx / g.ucharmod;
    sc->cf = -1.0 / sc->dt;
    sc->cforig = sc->cf;
    if (sc->t < tempt) sc->cf = sc->cf * (sc->t / tempt);
    sc->divmax_bits = 0ull;
}
__global__ void __launch_bounds__(256) k_scal_a(Geo g, Scal *sc, const double *part) { b_scal_a(g, sc, part); }

// ============================================================================
// k_nl: nonlinear term -div(uu) of one plane (nl_allflow.F90:71-327, nl.F90:99-173).
// nl_c = -( (wy*F(u_a u_b) + wz*F(u_a' u_b')) + F(D_c) ),  D_c = x-flux difference.
// ============================================================================
__device__ __forceinline__ double slope_lim(double um1, double u0, double up1, double dx, int limiter) {
    double s = (up1 - um1) / (2.0 * dx);
    double phi = 1.0;
    if (limiter == PIBM_LIMITER_MINMOD) {
        phi = (u0 - um1) / (up1 - u0 + kSmallD);
        phi = phi <= 0.0 ? 0.0 : fmin(1.0, phi);
    }
    return s * phi * 1.0;
}
// slope_lim with the divisor 2 dx given with its reciprocal (qdiv)
__device__ __forceinline__ double slope_lim_q(double um1, double u0, double up1, double tdx, double rtdx, int limiter) {
    double s = qdiv(up1 - um1, tdx, rtdx);
    double phi = 1.0;
    if (limiter == PIBM_LIMITER_MINMOD) {
        phi = (u0 - um1) / (up1 - u0 + kSmallD);
        phi = phi <= 0.0 ? 0.0 : fmin(1.0, phi);
    }
    return s * phi * 1.0;
}

// x-flux difference D_c at plane i for node e of the plane (upwind: MUSCL
// states + Rusanov flux, nl_allflow.F90:139-294; center: nl_allflow.F90:97-124,298-310).
__device__ __forceinline__ double xflux_diff(const Geo &g, const double *__restrict__ ubcp, int i, int e, int c) {
    const int nx = g.nx;
    const size_t RS = g.RS;
    auto U = [&](int comp, int ii) -> double {
        ii = ii < 0 ? ii + nx : (ii >= nx ? ii - nx : ii);
        return __ldg(ubcp + ((size_t)comp * nx + ii) * RS + e);
    };
    const double dx = g.dx;
    if (g.scheme == PIBM_SCHEME_CENTER) {
        const double fp = U(0, i + 1) * U(c, i + 1), fm = U(0, i - 1) * U(c, i - 1);
        return (fp - fm) / (2.0 * dx);
    }
    // cells i-2 .. i+2 of component 0 (advecting velocity) and component c
    double a[5], b[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) { a[q] = U(0, i - 2 + q); b[q] = (c == 0) ? a[q] : U(c, i - 2 + q); }
    // slopes at cells i-1, i, i+1 (index 1..3 in the window)
    double sa[3], sb[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        sa[q] = slope_lim(a[q], a[q + 1], a[q + 2], dx, g.limiter);
        sb[q] = (c == 0) ? sa[q] : slope_lim(b[q], b[q + 1], b[q + 2], dx, g.limiter);
    }
    const double h = dx / 2.0;
    double F[2];
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        // interface between window cells (f+1) and (f+2): global interface m = i-1+f
        const double uminus = a[f + 1] + sa[f] * h;
        const double uplus = a[f + 2] - sa[f + 1] * h;
        const double Um = b[f + 1] + sb[f] * h;
        const double Up = b[f + 2] - sb[f + 1] * h;
        const double Am = 0.5 * uminus * Um, Ap = 0.5 * uplus * Up;
        const double ms = fmax(fabs(uminus), fabs(uplus));
        int m = i - 1 + f;
        m = m < 0 ? m + nx : m;
        // interface nx (m == nx-1 here, 0-based) receives the cell-1 contribution first
        const double s = (m == nx - 1) ? ((0.0 + Ap) + Am) : ((0.0 + Am) + Ap);
        F[f] = s - 0.5 * ms * (Up - Um);
    }
    return (F[1] - F[0]) / dx;
}

// ============================================================================
// k_flux: x-flux differences D_c(i) = (F_c(i) - F_c(i-1))/dx of the conservative
// nonlinear term for all nodes (nl_allflow.F90:121-310).  One thread owns one
// (y,z) node and a segment of SEG x-planes and streams along x with a rolling
// window, so every ubcp value is read once per segment (plus a 4-plane halo).
// Upwind: MUSCL states with optional minmod limiter and a Rusanov flux; the
// periodic interface between cells nx and 1 accumulates its two halves in the
// reference's order (cell 1's contribution first).  Center: (f(i+1)-f(i-1))/(2dx).
// ============================================================================
template <int N>
__device__ __forceinline__ void b_flux(const Geo &g, const double *__restrict__ ubcp, double *__restrict__ Dx,
                                              const Scal *__restrict__ sc) {
    constexpr int RSP = RP<N>::RSP;
    const int nx = g.nx, SEG = g.flux_seg, nseg = nx / SEG;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= RSP * nseg || sc->status) return;
    const int e = t % RSP, i0 = (t / RSP) * SEG;
    if (e % (N + 2) >= N) return;   // row padding
    const size_t CR = (size_t)nx * RSP;
    auto U = [&](int c, int ii) -> double {
        ii = ii < 0 ? ii + nx : (ii >= nx ? ii - nx : ii);
        return __ldg(ubcp + c * CR + (size_t)ii * RSP + e);
    };
    const double dx = g.dx, h = dx / 2.0;
    const double tdx = 2.0 * dx, rtdx = 1.0 / tdx, rdx = 1.0 / dx;   // divisors and reciprocals for qdiv
    if (g.scheme == PIBM_SCHEME_CENTER) {
        for (int i = i0; i < i0 + SEG; ++i) {
            const double ap = U(0, i + 1), am = U(0, i - 1);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double fp = ap * (c == 0 ? ap : U(c, i + 1)), fm = am * (c == 0 ? am : U(c, i - 1));
                Dx[c * CR + (size_t)i * RSP + e] = qdiv(fp - fm, tdx, rtdx);
            }
        }
        return;
    }
    const int lim = g.limiter;
    // window: w[c][k] = u_c(i-1+k), k = 0..3 ; slopes sl[c][0] = s(i), sl[c][1] = s(i+1)
    double w[3][4], sl[3][2], Fm[3];
    auto flux = [&](int c, int m, double a0, double a1, double sa0, double sa1, double b0, double b1, double sb0, double sb1) {
        const double uminus = a0 + sa0 * h, uplus = a1 - sa1 * h;
        const double Um = (c == 0) ? uminus : b0 + sb0 * h;
        const double Up = (c == 0) ? uplus : b1 - sb1 * h;
        const double Am = 0.5 * uminus * Um, Ap = 0.5 * uplus * Up;
        const double ms = fmax(fabs(uminus), fabs(uplus));
        const double s0 = (m == nx - 1) ? ((0.0 + Ap) + Am) : ((0.0 + Am) + Ap);
        return s0 - 0.5 * ms * (Up - Um);
    };
    // prologue: cells i0-2 .. i0+1
    double um2[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        um2[c] = U(c, i0 - 2);
        w[c][0] = U(c, i0 - 1); w[c][1] = U(c, i0); w[c][2] = U(c, i0 + 1);
    }
    double sprev[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        sprev[c] = slope_lim_q(um2[c], w[c][0], w[c][1], tdx, rtdx, lim);     // s(i0-1)
        sl[c][0] = slope_lim_q(w[c][0], w[c][1], w[c][2], tdx, rtdx, lim);     // s(i0)
    }
    {
        const int m = (i0 - 1 + nx) % nx;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            Fm[c] = flux(c, m, w[0][0], w[0][1], sprev[0], sl[0][0], w[c][0], w[c][1], sprev[c], sl[c][0]);
    }
    for (int i = i0; i < i0 + SEG; ++i) {
#pragma unroll
        for (int c = 0; c < 3; ++c) w[c][3] = U(c, i + 2);
#pragma unroll
        for (int c = 0; c < 3; ++c) sl[c][1] = slope_lim_q(w[c][1], w[c][2], w[c][3], tdx, rtdx, lim);   // s(i+1)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double F = flux(c, i, w[0][1], w[0][2], sl[0][0], sl[0][1], w[c][1], w[c][2], sl[c][0], sl[c][1]);
            Dx[c * CR + (size_t)i * RSP + e] = qdiv(F - Fm[c], dx, rdx);
            Fm[c] = F;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) { w[c][0] = w[c][1]; w[c][1] = w[c][2]; w[c][2] = w[c][3]; sl[c][0] = sl[c][1]; }
    }
}
// MB blocks per SM.  Flow alone: four (64 registers, 28 bytes spilled),
// 0.034 against 0.036 ms at three (74, no spills).  With a passive scalar on its side stream from the start of
// the step (fixed spheres) the pair k_flux<N, 3> + k_rev<N, 3> leaves room
// for the scalar's blocks: step 1.088 against 1.134 ms at 128^3, while either
// one alone gains under 0.01 ms.  A moving run forks its scalar later and
// keeps the flow's bounds (k_rev<N, 3> cost 0.085 ms per step at 256^3 there).
template <int N, int MB>
__global__ void __launch_bounds__(256, MB) k_flux(Geo g, const double *__restrict__ ubcp, double *__restrict__ Dx,
                                              const Scal *__restrict__ sc) { b_flux<N>(g, ubcp, Dx, sc); }

template <int N>
__device__ __forceinline__ void b_nl(const Geo &g, const double *__restrict__ ubcp, const double *__restrict__ Dx,
                                                   const double2 *__restrict__ u,
                                                   const double2 *__restrict__ onl, double2 *__restrict__ nl_new,
                                                   double *__restrict__ Q, Scal *__restrict__ sc) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RS = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    __shared__ uint64_t mb;
    if (threadIdx.x == 0) mbar_init(&mb, 1);
    load_tw<N>(tws, g);
    __syncthreads();
    grid_dep_wait();   // the twiddles above are set-up data; the fields come from earlier kernels
    uint32_t phase = 0;
    const int i = blockIdx.x / L::C, rank = blockIdx.x % L::C, nx = g.nx;
    const int im = (i - 1 + nx) % nx, ip = (i + 1) % nx;
    const size_t roff = (size_t)rank * L::RL;
    const TwT tw{tws, N};
    // real component n of this CTA's rows
    auto Uc = [&](int n) { return ubcp + ((size_t)n * nx + i) * RS + roff; };
    const double c12 = g.c1 + g.c2;
    {
        const int c = blockIdx.y;
        // nl_new of this plane accumulates i ky F(pa) + i kz F(pb) + F(D_c) in place
        double2 *dst = nl_new + ((size_t)c * nx + i) * PS;
        for (int q = 0; q < 3; ++q) {
            if (q < 2) {
                // product pairs of component c: wy term (u1 u2, u2 u2, u2 u3), wz term (c, 2);
                // the first factor's rows arrive by one bulk copy, the second by
                // 16-byte loads multiplied in place
                const int na = q == 0 ? (c == 0 ? 0 : 1) : c, nb = q == 0 ? (c == 2 ? 2 : 1) : 2;
                if (threadIdx.x == 0) {
                    fence_async_smem();
                    bulk_load(buf, Uc(na), L::RBYTES, &mb);
                }
                load_wait(&mb, phase, sc);
                double2 *b2 = buf;
                const double2 *B2 = (const double2 *)Uc(nb);
#pragma unroll 8
                for (int e = threadIdx.x; e < L::RL / 2; e += L::T) {
                    const double2 x = b2[e], y = B2[e];
                    b2[e] = make_double2(x.x * y.x, x.y * y.y);
                }
                __syncthreads();
            } else {
                if (threadIdx.x == 0) {
                    fence_async_smem();
                    bulk_load(buf, Dx + ((size_t)c * nx + i) * RS + roff, L::RBYTES, &mb);
                }
                load_wait(&mb, phase, sc);
            }
            cl_r2c<N>(buf, tw, rank);
            if (q < 2) {
#pragma unroll 4
                for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
                    const int kz = e / L::PZ, jl = e - kz * L::PZ;
                    if (jl == L::MC && rank != 0) continue;
                    const int ge = kz * my2 + cl_col<N>(jl, rank);
                    const double2 Xr = cl_unpack<N>(buf, kz, jl, rank);
                    const double2 X = r2c_norm<N>(Xr, g.nrm);
                    if (q == 0) { const double ky = g.ky[cl_col<N>(jl, rank)]; dst[ge] = make_double2(-ky * X.y, ky * X.x); }
                    else { const double kzv = g.kz[kz]; dst[ge] = cadd(dst[ge], make_double2(-kzv * X.y, kzv * X.x)); }
                }
                __syncthreads();
            }
        }
        // nl = -(...) (nl.F90:146-152); Q = -c3 nl - c4 onl - c12 diffn (calc_visc spectrum)
        const double2 *on = onl + ((size_t)c * nx + i) * PS;
        const double2 *uc = u + (size_t)c * nx * PS;
        // the nl value of element (kz, jl) and the transform input of Q there
        auto nl_q = [&](int kz, int jl) -> double2 {
            const int ge = kz * my2 + cl_col<N>(jl, rank);
            const double2 X = r2c_norm<N>(cl_unpack<N>(buf, kz, jl, rank), g.nrm);
            const double2 s = cadd(dst[ge], X);
            const double2 v = make_double2(-s.x, -s.y);
            dst[ge] = v;
            const double2 a = uc[(size_t)im * PS + ge], bb = uc[(size_t)i * PS + ge], cv = uc[(size_t)ip * PS + ge];
            double2 df = make_double2(g.rdx2 * ((a.x - 2.0 * bb.x) + cv.x), g.rdx2 * ((a.y - 2.0 * bb.y) + cv.y));
            const double w2 = g.w2[ge];
            df = make_double2((df.x - w2 * bb.x) * g.vis, (df.y - w2 * bb.y) * g.vis);
            const double2 o = on[ge];
            return make_double2((-g.c3 * v.x - g.c4 * o.x) - c12 * df.x, (-g.c3 * v.y - g.c4 * o.y) - c12 * df.y);
        };
        // Every element is read and rewritten by its own thread, except rank 0's
        // column 0, which cl_unpack also reads for ky = 0 and ky = M at the
        // mirrored kz: it is rewritten after a barrier.
#pragma unroll 2
        for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
            const int kz = e / L::PZ, jl = e - kz * L::PZ;
            if ((jl == L::MC && rank != 0) || (jl == 0 && rank == 0)) continue;
            buf[e] = nl_q(kz, jl);
        }
        if (rank == 0) {
            constexpr int K0 = (N + L::T - 1) / L::T;
            double2 q0[K0];
#pragma unroll
            for (int k = 0; k < K0; ++k) {
                const int kz = (int)threadIdx.x + k * L::T;
                if (kz < N) q0[k] = nl_q(kz, 0);
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < K0; ++k) {
                const int kz = (int)threadIdx.x + k * L::T;
                if (kz < N) buf[kz * L::PZ] = q0[k];
            }
        }
        __syncthreads();
        cl_c2r<N>(buf, tw, rank);
        if (threadIdx.x == 0) { bulk_store(Q + ((size_t)c * nx + i) * RS + roff, buf, L::RBYTES); bulk_wait_read(); }
    }
}
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_nl(Geo g, const double *__restrict__ ubcp, const double *__restrict__ Dx,
                                                   const double2 *__restrict__ u,
                                                   const double2 *__restrict__ onl, double2 *__restrict__ nl_new,
                                                   double *__restrict__ Q, Scal *__restrict__ sc) { b_nl<N>(g, ubcp, Dx, u, onl, nl_new, Q, sc); }

// ============================================================================
// k_drag: per-sphere pressure and viscous force from the surface quadrature
// (calc_pres_visc_drag, boundary_condition.F90:1481-1645).  One CTA per sphere.
// ============================================================================

template <int N>
__device__ __forceinline__ void b_drag(const Geo &g, const double *__restrict__ pbcp, const double *__restrict__ omega,
                                              double *__restrict__ dpart, const Scal *__restrict__ sc) {
    __shared__ double scr[32];
    const int m = blockIdx.x / kDragSplit, part = blockIdx.x % kDragSplit;
    const int NB = g.nbody;
    const double xcm[3] = {g.xc[m], g.xc[m + NB], g.xc[m + 2 * NB]};
    double sa[3] = {0, 0, 0}, sb[3] = {0, 0, 0};
    const size_t CR = (size_t)g.nx * RP<N>::RSP;
    const int chunk = (g.nbnd + kDragSplit - 1) / kDragSplit;
    const int l0 = part * chunk, l1 = min(g.nbnd, l0 + chunk);
    for (int l = l0 + threadIdx.x; l < l1; l += blockDim.x) {
        double xl[3], xpb[3], cdl[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) { xl[d] = __dadd_rn(xcm[d], __dmul_rn(g.bnd[3 * l + d], g.rb)); cdl[d] = g.cd[3 * l + d]; }
        xpb[0] = __dsub_rn(xl[0], 0.5); xpb[1] = xl[1]; xpb[2] = xl[2];
        Sten sp, sv;
        make_sten(g, xpb, sp);
        make_sten(g, xl, sv);
        const double pl = dot_ijk<N>(sp, pbcp);
        double vort[3];
#pragma unroll
        for (int n = 0; n < 3; ++n) vort[n] = interp_kji<N>(sv, omega + n * CR);
        double df[3];
        df[0] = vort[2] * cdl[1]; df[0] = df[0] - vort[1] * cdl[2];
        df[1] = vort[0] * cdl[2]; df[1] = df[1] - vort[2] * cdl[0];
        df[2] = vort[1] * cdl[0]; df[2] = df[2] - vort[0] * cdl[1];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sa[d] += pl * cdl[d] * g.da1;
            sb[d] += (-df[d]) * g.vis * g.da1;
        }
    }
    for (int d = 0; d < 3; ++d) {
        const double a = block_sum(sa[d], scr), b = block_sum(sb[d], scr);
        if (threadIdx.x == 0) { dpart[(size_t)blockIdx.x * 6 + d] = a; dpart[(size_t)blockIdx.x * 6 + 3 + d] = b; }
    }
}
template <int N>
__global__ void __launch_bounds__(256) k_drag(Geo g, const double *__restrict__ pbcp, const double *__restrict__ omega,
                                              double *__restrict__ dpart, const Scal *__restrict__ sc) { b_drag<N>(g, pbcp, omega, dpart, sc); }

// compute_mpg_at_n tail + bcset diagnostics (boundary_condition.F90:356-464, 701-884).
__device__ __forceinline__ void b_scal_b(const Geo &g, Scal *sc, double *pres, double *visc, double *ptot,
                                                double *force, const double *dpart) {
    __shared__ double scr[32 * 9];
    __shared__ double tot[12];
    if (block_failed(sc)) return;
    const int NB = g.nbody;
    // per-sphere sums of the k_drag partials (fixed order)
    for (int m = threadIdx.x; m < NB; m += blockDim.x) {
        double a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
        for (int q = 0; q < kDragSplit; ++q)
            for (int d = 0; d < 3; ++d) { a[d] += dpart[((size_t)m * kDragSplit + q) * 6 + d]; b[d] += dpart[((size_t)m * kDragSplit + q) * 6 + 3 + d]; }
        for (int d = 0; d < 3; ++d) { pres[m + d * NB] = -a[d]; ptot[m + d * NB] = a[d]; visc[m + d * NB] = b[d]; }
    }
    __syncthreads();
    {
        double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // ptot, visc, pres sums per component
        for (int m = threadIdx.x; m < NB; m += blockDim.x)
#pragma unroll
            for (int d = 0; d < 3; ++d) { v[d] += ptot[m + d * NB]; v[3 + d] += visc[m + d * NB]; v[6 + d] += pres[m + d * NB]; }
        block_reduce_k<9>(v, scr);
        if (threadIdx.x == 0)
            for (int q = 0; q < 9; ++q) tot[q] = v[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int d = 0; d < 3; ++d) { sc->pres_total[d] = tot[d]; sc->visc_total[d] = tot[3 + d]; }
        const double nf = (3.0 * 3.14159265358979323846 * g.vis * (sc->mixmeanslipmod + kSmallD) * g.char_length) * (double)NB;
        const double pa = sqrt(tot[6] * tot[6] + tot[7] * tot[7] + tot[8] * tot[8]);
        const double va = sqrt(tot[3] * tot[3] + tot[4] * tot[4] + tot[5] * tot[5]);
        sc->pres_drag = pa / nf / (1.0 - sc->maxvolfrac);
        sc->visc_drag = va / nf / (1.0 - sc->maxvolfrac);
        sc->total_drag = sc->pres_drag + sc->visc_drag;
        const double rhof = g.rhof, rhos = g.rhos, mvf = g.mean_volfrac;
        if (!g.set_mpg) {
            for (int d = 0; d < 3; ++d) {
                if (g.moving) {
                    // moving particles: mpg and the frame acceleration (:389-398)
                    double m = sc->cf * (g.ufmean_des[d] - sc->ufmean[d]) + sc->cf * (sc->usmean[d] - g.usmean_des[d]);
                    m = m + (sc->pres_total[d] - (sc->visc_total[d])) * (1.0 / (rhof * (1.0 - mvf)) + 1.0 / (mvf * rhos)) / g.voldom;
                    sc->mpg[d] = m / (1.0 / rhof - 1.0 / rhos);
                    sc->frame_accln[d] = -sc->mpg[d] / rhos - (sc->pres_total[d] - sc->visc_total[d]) / (mvf * rhos * g.voldom) +
                                         sc->cf * (g.usmean_des[d] - sc->usmean[d]);
                } else {
                    sc->mpg[d] = sc->cf * (g.ufmean_des[d] - sc->ufmean[d]) +
                                 (sc->pres_total[d] / g.voldom - (sc->visc_total[d]) / g.voldom) / (1.0 - sc->maxvolfrac);
                }
                if (g.include_frmeanfluid) sc->mpg[d] = sc->mpg[d] + sc->frmeanfluid[d];
            }
        } else if (g.moving) {
            for (int d = 0; d < 3; ++d)
                sc->frame_accln[d] = -sc->mpg[d] / rhos - (sc->pres_total[d] - sc->visc_total[d]) / (mvf * rhos * g.voldom) +
                                     sc->cf * (g.usmean_des[d] - sc->usmean[d]);
        }
    }
    __syncthreads();
    const double c12 = g.c1 + g.c2;
    const double mp[3] = {sc->mpg[0], sc->mpg[1], sc->mpg[2]};
    double fs[3] = {0, 0, 0};
    for (int m = threadIdx.x; m < NB; m += blockDim.x)
        for (int d = 0; d < 3; ++d) {
            const double f = c12 * (pres[m + d * NB] + visc[m + d * NB]) - c12 * mp[d] * g.sphere_vol;
            force[m + d * NB] = f;
            fs[d] += f;
        }
    block_reduce_k<3>(fs, scr);
    if (threadIdx.x == 0) {
        double avg[3];
        for (int d = 0; d < 3; ++d) avg[d] = (fs[d] / NB) * g.mean_volfrac / g.mean_volfrac;
        const double nd = sqrt(avg[0] * avg[0] + avg[1] * avg[1] + avg[2] * avg[2]);
        double nf = 3.0 * 3.14159265358979323846 * g.vis * g.ucharmod * g.char_length;
        if (g.set_mpg) nf = 3.0 * 3.14159265358979323846 * g.vis * (sc->mixmeanslipmod + kSmallD) * g.char_length;
        sc->norm_drag = nd / nf;
        sc->ferror = sc->norm_drag > 0.0 ? fabs(sc->norm_drag - sc->fold) / sc->norm_drag : 1.0;
        sc->fold = sc->norm_drag;
        if (sc->norm_drag > 1.0e6) sc->status = PIBM_ERR_BLOWUP;
    }
}
__global__ void __launch_bounds__(256) k_scal_b(Geo g, Scal *sc, double *pres, double *visc, double *ptot,
                                                double *force, const double *dpart) { b_scal_b(g, sc, pres, visc, ptot, force, dpart); }

// ============================================================================
// k_rev: direct forcing at the inner reversal points
// (calc_inner_reversal_forcing, boundary_condition.F90:1104-1479).
// rec[p*6 + 0..2] = force_tmp, rec[p*6 + 3..5] = force_dist, rz[p*3 + 0..2] =
// the inner point's offsets in its cell (the spreading forms each corner's
// weight*force_tmp/dx^3 from them, corner_contrib); blockpart = sums of
// tmppa/dx^3 over all corners (frmean) and over fluid corners (frmeanfluid).
// ============================================================================
__device__ __forceinline__ void inner_point(const Geo &g, int m, int l, double xli[3]) {
    const int NB = g.nbody;
#pragma unroll
    for (int d = 0; d < 3; ++d) xli[d] = __dadd_rn(g.xc[m + d * NB], __dmul_rn(g.bnd[3 * l + d], g.ri));
}

template <int N>
__device__ __forceinline__ void b_rev(const Geo &g, const double *__restrict__ ubcp, const double *__restrict__ pgr,
                                                const double *__restrict__ Q, const Scal *__restrict__ sc,
                                                double *__restrict__ rec, double *__restrict__ rz, double *__restrict__ blockpart) {
    __shared__ double scr[32 * 6];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    double fm[3] = {0, 0, 0}, ffl[3] = {0, 0, 0};
    if (p < sc->npts && !sc->status) {
        const int m = g.pt_m[p], l = g.pt_l[p], NB = g.nbody;
        const size_t CR = (size_t)g.nx * RP<N>::RSP;
        const double rdx3 = 1.0 / g.dx3;   // reciprocal for qdiv
        double xli[3], xlo[3], xpi[3], snorm[3];
        inner_point(g, m, l, xli);
        double rad = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            xlo[d] = __dadd_rn(g.xc[m + d * NB], __dmul_rn(g.bnd[3 * l + d], g.ro));
            const double a = __dmul_rn(g.bnd[3 * l + d], g.ri);
            rad = __dadd_rn(rad, __dmul_rn(a, a));
        }
        rad = sqrt(rad);
#pragma unroll
        for (int d = 0; d < 3; ++d) snorm[d] = __dmul_rn(g.bnd[3 * l + d], g.ri) / rad;
        xpi[0] = __dsub_rn(xli[0], 0.5); xpi[1] = xli[1]; xpi[2] = xli[2];
        Sten so, spi, si;
        make_sten(g, xlo, so);
        make_sten(g, xpi, spi);
        make_sten(g, xli, si);
        double ulo[3], ppll[3], uli[3], qll[3];
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            ulo[n] = interp_kji<N>(so, ubcp + n * CR);
            ppll[n] = interp_kji<N>(spi, pgr + n * CR, sc->mpg[n]);
            uli[n] = interp_kji<N>(si, ubcp + n * CR);
            qll[n] = dot_ijk<N>(si, Q + n * CR);
        }
        double linvel[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) linvel[d] = g.vel[m + d * NB];
        double unmag = 0.0, ubnmag = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) { unmag = unmag + snorm[d] * ulo[d]; ubnmag = ubnmag + snorm[d] * linvel[d]; }
        const double ro = g.ro, ri = g.ri, rb = g.rb;
        double ucar[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double unorm = snorm[d] * unmag, utang = ulo[d] - unorm;
            const double ubnorm = snorm[d] * ubnmag, ubtang = linvel[d] - ubnorm;
            double utangi = ubtang * (ro - ri) - utang * (rb - ri);
            utangi = utangi / (ro - rb);
            double unormi = 0.0;
            if (g.revernorm == 1) { unormi = ubnorm * (ro - ri) - unorm * (rb - ri); unormi = unormi / (ro - rb); }
            ucar[d] = utangi + unormi;
        }
        const double cf = sc->cf, c12 = g.c1 + g.c2, da2 = g.da2[m];
        double ft[3];
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            double f = cf * (-ucar[n] + uli[n]);
            f = f + qll[n];
            f = f + c12 * ppll[n];
            ft[n] = f * da2 * g.dr * g.dx;
        }
        int count_fl = 0;
        double force_fl[3] = {0, 0, 0};
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const bool fl = g.fluid[(size_t)si.ii[a] * RP<N>::RSP + real_off<N>(si.kk[c], si.jj[b])] != 0;
                    const double w = si.w(a, b, c);
#pragma unroll
                    for (int n = 0; n < 3; ++n) {
                        const double t = qdiv(w * ft[n], g.dx3, rdx3);
                        if (fl) { force_fl[n] = force_fl[n] + t; ffl[n] += t; }
                        fm[n] += t;
                    }
                    count_fl += fl ? 1 : 0;
                }
        const int count_so = 8 - count_fl;
        rz[(size_t)p * 3] = si.xv[1];
        rz[(size_t)p * 3 + 1] = si.yv[1];
        rz[(size_t)p * 3 + 2] = si.zv[1];
        double *r = rec + (size_t)p * 6;
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            r[n] = ft[n];
            r[3 + n] = count_so > 0 ? force_fl[n] / (double)count_so : 0.0;
        }
    }
    double v[6] = {fm[0], fm[1], fm[2], ffl[0], ffl[1], ffl[2]};
    block_reduce_k<6>(v, scr);
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) blockpart[(size_t)blockIdx.x * 6 + q] = v[q];
}
// MB blocks per SM.  Flow alone: two (128 registers), more gathers in flight
// per thread beat the occupancy of three blocks at 80 registers and 32 bytes
// spilled (0.069 against 0.076 ms at 128^3); three beside a passive scalar
// (k_flux above).
template <int N, int MB>
__global__ void __launch_bounds__(256, MB) k_rev(Geo g, const double *__restrict__ ubcp, const double *__restrict__ pgr,
                                                const double *__restrict__ Q, const Scal *__restrict__ sc,
                                                double *__restrict__ rec, double *__restrict__ rz, double *__restrict__ blockpart) { b_rev<N>(g, ubcp, pgr, Q, sc, rec, rz, blockpart); }

__device__ __forceinline__ void b_scal_c(const Geo &g, Scal *sc, const double *blockpart, int nblocks) {
    __shared__ double scr[32 * 6];
    if (block_failed(sc)) return;
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < 6; ++q) a[q] += blockpart[(size_t)b * 6 + q];
    block_reduce_k<6>(a, scr);
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) {
            if (q < 3) sc->frmean[q] = a[q] / (double)g.ncell;
            else sc->frmeanfluid[q - 3] = a[q] / (double)sc->count_fluid;
        }
}
__global__ void __launch_bounds__(256) k_scal_c(Geo g, Scal *sc, const double *blockpart, int nblocks) { b_scal_c(g, sc, blockpart, nblocks); }

// k_spread: fr at every forced node, accumulated over its (point, corner)
// contributions in the reference's (sphere, point) order
// (boundary_condition.F90:1425-1462).  sp_node holds physical offsets.
__device__ __forceinline__ void b_spread(const Geo &g, const double *__restrict__ rec, const double *__restrict__ rz,
                                                double *__restrict__ fr, const Scal *__restrict__ sc) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.sp_nnodes || sc->status) return;
    const int node = g.sp_node[q];
    const double rdx3 = 1.0 / g.dx3;
    double acc[3] = {0.0, 0.0, 0.0};
    const int e0 = g.sp_ptr[q], e1 = g.sp_ptr[q + 1];
#pragma unroll 4
    for (int e = e0; e < e1; ++e) {
        const int ent = __ldg(g.sp_ent + e);
        double t[3];
        corner_contrib(rz, rec, ent, g.dx3, rdx3, t);
        if (g.include_frmeanfluid) {
#pragma unroll
            for (int n = 0; n < 3; ++n) acc[n] = acc[n] + t[n];
        } else {
            const double *r = rec + (size_t)(ent >> 3) * 6 + 3;
#pragma unroll
            for (int n = 0; n < 3; ++n) acc[n] = (acc[n] + t[n]) + __ldg(r + n);
        }
    }
    const size_t CR = (size_t)g.nx * g.RS;
#pragma unroll
    for (int n = 0; n < 3; ++n) fr[n * CR + node] = acc[n];
}
__global__ void __launch_bounds__(256) k_spread(Geo g, const double *__restrict__ rec, const double *__restrict__ rz,
                                                double *__restrict__ fr, const Scal *__restrict__ sc) { b_spread(g, rec, rz, fr, sc); }

// k_ff: ff = r2c(fr - frmean) (boundary_condition.F90:678-700).
template <int N>
__device__ __forceinline__ void b_ff(const Geo &g, const double *__restrict__ fr, double2 *__restrict__ ff,
                                                   Scal *__restrict__ sc) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RSP = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    __shared__ uint64_t mb;
    if (threadIdx.x == 0) mbar_init(&mb, 1);
    load_tw<N>(tws, g);
    __syncthreads();
    grid_dep_wait();   // the twiddles above are set-up data; the fields come from earlier kernels
    uint32_t phase = 0;
    const int i = blockIdx.x / L::C, rank = blockIdx.x % L::C, nx = g.nx;
    const size_t roff = (size_t)rank * L::RL;
    const TwT tw{tws, N};
    {
        const int n = blockIdx.y;
        if (threadIdx.x == 0) {
            fence_async_smem();
            bulk_load(buf, fr + ((size_t)n * nx + i) * RSP + roff, L::RBYTES, &mb);
        }
        load_wait(&mb, phase, sc);
        const double fmn = sc->frmean[n];
        double *b = (double *)buf;
        for (int e = threadIdx.x; e < L::RL; e += L::T) b[e] = b[e] - fmn;
        __syncthreads();
        cl_r2c<N>(buf, tw, rank);
        double2 *dst = ff + ((size_t)n * nx + i) * PS;
#pragma unroll 4
        for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
            const int kz = e / L::PZ, jl = e - kz * L::PZ;
            if (jl == L::MC && rank != 0) continue;
            const double2 X = cl_unpack<N>(buf, kz, jl, rank);
            dst[kz * my2 + cl_col<N>(jl, rank)] = r2c_norm<N>(X, g.nrm);
        }
    }
}
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_ff(Geo g, const double *__restrict__ fr, double2 *__restrict__ ff,
                                                   Scal *__restrict__ sc) { b_ff<N>(g, fr, ff, sc); }

// ============================================================================
// k_lines: pressure -> ustep -> divcorr for a tile of LT (ky,kz) lines per CTA
// (poisson.F90:55-508, usteptime.F90:45-269, check_divergence
// steptheflow.F90:219-240).
//
// Every cyclic system of velstep has constant coefficients (a = c, b on every
// row, periodic coupling), i.e. it is a symmetric circulant matrix; the
// reference solves it with Thomas + Sherman-Morrison (tridiagonal.F90:90-150,
// usteptime.F90:344-349,457-468).  Here one warp solves one line exactly
// through its eigen-decomposition: forward FFT along x in registers
// (group_fft), division by N*lambda_m with lambda_m = b + 2a cos(2 pi m/N),
// and the exact inverse of the forward stages.  The (ky,kz) = (0,0) line is
// not circulant (nx-1 unknowns, p(nx) = 0: poisson.F90:127-142, 309-325) and
// keeps the reference's Thomas recursion.
// Tiles live in shared memory as [line][i]; global loads and stores run over
// consecutive lines (contiguous in the [i][k][j] layout).
// ============================================================================
template <int NX, int LT>
__device__ __forceinline__ void b_lines(const Geo &g, double2 *__restrict__ u, double2 *__restrict__ p,
                                                   const double2 *__restrict__ nl, const double2 *__restrict__ onl,
                                                   const double2 *__restrict__ ff, Scal *__restrict__ sc) {
    constexpr int R = NX / 32;
    constexpr int NP = lines_pitch<NX, LT>();
    extern __shared__ double2 sm[];
    double2 *tws = sm;
    double2 *RHS = tws + NX;
    double2 *P = RHS + LT * NP;
    double2 *U = P + LT * NP;                 // [comp][line][i]
    double *gam = (double *)(U + 3 * LT * NP);
    double2 *st = (double2 *)(gam + NX);      // cross-lane stage twiddles
    double *lcs = (double *)(st + 32);        // per-lane constants of the solves
    double2 *ltr = (double2 *)(lcs + NX);
    if (block_failed(sc)) return;
    for (int t = threadIdx.x; t < NX; t += blockDim.x) tws[t] = g.tw[t];
    fill_stage_table<32>(st, g.tw, NX);
    fill_line_tw<R>(lcs, ltr, g.tw);
    const int PS = g.PS, nx = NX;
    const int q0 = blockIdx.x * LT;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const double dx = g.dx, dx2 = g.dx2, dt = sc->dt, vis = g.vis;
    const double c1 = g.c1, c2 = g.c2, c3 = g.c3, c4 = g.c4;
    const double c12 = c1 + c2, rdx = 1.0 / dx, rdx2 = 1.0 / dx2, rc12 = 1.0 / c12;   // divisors and reciprocals for qdiv
    const LineTw<R> tw{{tws, NX, 1, st}, lcs, ltr};
    auto KY = [&](int q) { return g.ky[q % g.my2]; };
    auto KZ = [&](int q) { return g.kz[q / g.my2]; };
    auto G = [&](const double2 *f, int comp, int i, int q) -> double2 {
        i = i >= nx ? i - nx : (i < 0 ? i + nx : i);
        return f[((size_t)comp * nx + i) * PS + q];
    };
    bool ok = true;
    // ---------------- pressure: source (poisson.F90:97-116) and old p ----------------
    // Thread t holds (line t % LT, plane t / LT): for LT = 8 the plane i+1 of a lane
    // sits LT lanes higher in the same warp, except in the warp's last plane row.
    static_assert(LT == 8 || LT == 4, "tile width");
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT;
        const int q = min(q0 + line, PS - 1);   // clamped: every lane takes part in the shuffles
        const double ky = KY(q), kz = KZ(q);
        double2 x0[9], x1[9];   // nl, ff, onl (3 components each) at planes i and i+1
#pragma unroll
        for (int n = 0; n < 3; ++n) { x0[n] = G(nl, n, i, q); x0[3 + n] = G(ff, n, i, q); x0[6 + n] = G(onl, n, i, q); }
        const bool last_row = lane >= 32 - LT;
#pragma unroll
        for (int f = 0; f < 9; ++f) {
            x1[f].x = __shfl_down_sync(0xffffffffu, x0[f].x, LT);
            x1[f].y = __shfl_down_sync(0xffffffffu, x0[f].y, LT);
        }
        if (last_row) {
#pragma unroll
            for (int n = 0; n < 3; ++n) { x1[n] = G(nl, n, i + 1, q); x1[3 + n] = G(ff, n, i + 1, q); x1[6 + n] = G(onl, n, i + 1, q); }
        }
        if (q0 + line >= PS) continue;
        // pressure source, its terms in the reference's order: (nl, ff) per component, then onl
        double2 tt = make_double2(0.0, 0.0);
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            tt = cadd_rn(tt, psrc_term<true>(n, c3, x0[n], x1[n], ky, kz, dx, rdx));
            tt = cadd_rn(tt, psrc_term<false>(n, 1.0, x0[3 + n], x1[3 + n], ky, kz, dx, rdx));
        }
#pragma unroll
        for (int n = 0; n < 3; ++n) tt = cadd_rn(tt, psrc_term<true>(n, c4, x0[6 + n], x1[6 + n], ky, kz, dx, rdx));
        RHS[line * NP + i] = make_double2(qdiv(tt.x, c12, rc12), qdiv(tt.y, c12, rc12));
        P[line * NP + i] = p[(size_t)i * PS + q];
        // explicit part of the ustep right-hand sides, dt*(c3 nl + ff + c4 onl) per component
        // (usteptime.F90:291-297), kept in the velocity tiles until each component is solved
#pragma unroll
        for (int n = 0; n < 3; ++n)
            U[(n * LT + line) * NP + i] = cadd_rn(cadd_rn(cscale_rn(x0[n], dt * c3), cscale_rn(x0[3 + n], dt)), cscale_rn(x0[6 + n], dt * c4));
    }
    __syncthreads();
    const int qw = q0 + w;
    const bool wact = qw < PS;
    const double w2w = wact ? g.w2[qw] : 0.0;
    const LineCoef kw = line_coef(dt, vis, c1, c2, dx2, w2w);   // line qw's coefficients
    {
        double2 *row = RHS + w * NP;
        if (wact) {
            if (qw == 0) {
                if (lane == 0) ok = thomas_real(row, gam, kw.pa, kw.pb, kw.pc, NX - 1) && ok;
                __syncwarp();
            } else {
                circulant_solve<R>(row, kw.pa, kw.pb, tw, lane);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r;
                P[w * NP + i] = p_update(P[w * NP + i], row[i]);
            }
        }
    }
    __syncthreads();
    // ---------------- ustep per component (usteptime.F90:73-470) ----------------
    constexpr int EPT = (LT * NX) / (LT * 32);   // tile elements per thread
    for (int n = 0; n < 3; ++n) {
        // stage u_n of the tile, then form every right-hand side from the staged
        // neighbours before overwriting the tile with them
        for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
            const int line = t % LT, i = t / LT, q = q0 + line;
            RHS[line * NP + i] = q < PS ? G(u, n, i, q) : make_double2(0.0, 0.0);
        }
        __syncthreads();
        double2 rr[EPT];
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const int t = threadIdx.x + k * LT * 32;
            const int line = t % LT, i = t / LT, q = q0 + line;
            if (q >= PS) continue;
            const LineCoef kq = line_coef(dt, vis, c1, c2, dx2, g.w2[q]);
            const int im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
            rr[k] = ustep_rhs(n, kq, RHS[line * NP + i], RHS[line * NP + im], RHS[line * NP + ip], U[(n * LT + line) * NP + i],
                              P[line * NP + im], P[line * NP + i], i == 0, KY(q), KZ(q), dx, rdx, dx2, rdx2);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const int t = threadIdx.x + k * LT * 32;
            const int line = t % LT, i = t / LT, q = q0 + line;
            if (q < PS) RHS[line * NP + i] = rr[k];
        }
        __syncthreads();
        if (wact) {
            double2 *row = RHS + w * NP;
            circulant_solve<R>(row, kw.ua, kw.ub, tw, lane);
#pragma unroll
            for (int r = 0; r < R; ++r) U[(n * LT + w) * NP + lane + 32 * r] = row[lane + 32 * r];
        }
        __syncthreads();
    }
    // ---------------- divcorr (poisson.F90:241-508) ----------------
    const double alpc = kw.alp, ralpc = 1.0 / alpc;
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT, q = q0 + line;
        if (q >= PS) continue;
        const int ip = i == nx - 1 ? 0 : i + 1;
        const double2 *U1 = U + (0 * LT + line) * NP, *U2 = U + (1 * LT + line) * NP, *U3 = U + (2 * LT + line) * NP;
        const double2 tt = div_term(U1[i], U1[ip], U2[i], U2[ip], U3[i], U3[ip], KY(q), KZ(q), dx, rdx);
        RHS[line * NP + i] = make_double2(qdiv(tt.x, alpc, ralpc), qdiv(tt.y, alpc, ralpc));
    }
    __syncthreads();
    if (wact) {
        const double ky = KY(qw), kz = KZ(qw);
        double2 *row = RHS + w * NP;
        if (qw == 0) {
            if (lane == 0) ok = thomas_real(row, gam, kw.pa, kw.pb, kw.pc, NX - 1) && ok;
            __syncwarp();
        } else {
            circulant_solve<R>(row, kw.pa, kw.pb, tw, lane);
        }
        double2 *U1 = U + (0 * LT + w) * NP, *U2 = U + (1 * LT + w) * NP, *U3 = U + (2 * LT + w) * NP;
        double2 *Pw = P + w * NP;
        double2 nu1[R], nu2[R], nu3[R], np[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            const int im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
            divcorr_update(kw, row[i], row[im], row[ip], i == 0, U1[i], U2[i], U3[i], Pw[i], ky, kz, w2w, dx, rdx, dx2, rdx2, nu1[r],
                           nu2[r], nu3[r], np[r]);
        }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            U1[i] = nu1[r]; U2[i] = nu2[r]; U3[i] = nu3[r]; Pw[i] = np[r];
        }
        __syncwarp();
        // check_divergence for this line
        double dmax = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r, ip = i == nx - 1 ? 0 : i + 1;
            dmax = fmax(dmax, cabs_rn(div_term(U1[i], U1[ip], U2[i], U2[ip], U3[i], U3[ip], ky, kz, dx, rdx)));
        }
        for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
        if (lane == 0) atomicMax(&sc->divmax_bits, (unsigned long long)__double_as_longlong(dmax));
    }
    __syncthreads();
    // coalesced write-back of u and p
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT, q = q0 + line;
        if (q >= PS) continue;
#pragma unroll
        for (int n = 0; n < 3; ++n) u[((size_t)n * nx + i) * PS + q] = U[(n * LT + line) * NP + i];
        p[(size_t)i * PS + q] = P[line * NP + i];
    }
    if (!ok) atomicCAS(&sc->status, 0, PIBM_ERR_PIVOT);
}
template <int NX, int LT>
__global__ void __launch_bounds__(LT * 32) k_lines(Geo g, double2 *__restrict__ u, double2 *__restrict__ p,
                                                   const double2 *__restrict__ nl, const double2 *__restrict__ onl,
                                                   const double2 *__restrict__ ff, Scal *__restrict__ sc) { b_lines<NX, LT>(g, u, p, nl, onl, ff, sc); }

// x-line tile width (lines per CTA): 4 or 8, chosen per run by autotune_lines
// (a run that was not tuned takes the default below).
template <int NX> struct LinesCfg { static constexpr int LT = NX >= 256 ? 4 : 8; };
template <int NX>
static size_t lines_smem(int lt) {
    const int np = lt == 4 ? lines_pitch<NX, 4>() : lines_pitch<NX, 8>();
    return (size_t)(NX + 5 * lt * np + 32) * sizeof(double2) + NX * sizeof(double) + line_tw_bytes<NX / 32>();
}
// Tensor maps of the persistent x-line kernel (lines_pipe.cuh): a field of
// ncomp components [comp][i][PS complex] as FLOAT64 {2 PS, nx, ncomp}, box
// {8, N, 1} (4 lines x N planes), 64-byte swizzle.  The encoder comes from
// the driver through the runtime's entry-point query (no libcuda link).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *, const cuuint64_t *,
                                  const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}
static bool line_map(CUtensorMap *m, const void *base, int PS, int nx, int ncomp, int N) {
    const EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t dim[3] = {(cuuint64_t)2 * PS, (cuuint64_t)nx, (cuuint64_t)ncomp};
    const cuuint64_t stride[2] = {(cuuint64_t)PS * 16, (cuuint64_t)nx * PS * 16};
    const cuuint32_t box[3] = {8, (cuuint32_t)N, 1}, es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base), dim, stride, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
// SMs of the current device (cached per device).
static int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}
// The 4-line width runs the persistent tensor-map kernel on grids up to 128
// (three blocks of 72 KB per SM); at 256 a slab is 16 KB and the staged
// kernel is kept.  Both give bitwise the same results.
// launch_planes with programmatic dependent launch: the blocks may start
// (and run the prologue before their grid_dep_wait) while the previous kernel
// of the stream drains.
template <int N, typename... KArgs, typename... Args>
inline void launch_planes_pdl(void (*k)(KArgs...), int nplanes, int items, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nplanes * PL<N>::C), (unsigned)items, 1);
    cfg.blockDim = dim3(PL<N>::T, 1, 1);
    cfg.dynamicSmemBytes = plane_smem<N>();
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = PL<N>::C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    cudaLaunchKernelEx(&cfg, k, args...);
}

template <int N>
static void launch_lines(const Geo &g, DevBufs &b, double2 *u, double2 *p, int cur, Scal *sc, cudaStream_t s) {
    const int old = cur ^ 1;
    const int lt = g.lines_lt ? g.lines_lt : LinesCfg<N>::LT;
    if constexpr (N <= 128) {
        if (lt == 4 && g.PS % LPipe<N>::LT == 0) {
            LineMaps mp;
            if (line_map(&mp.u, u, g.PS, g.nx, 3, N) && line_map(&mp.p, p, g.PS, g.nx, 1, N) &&
                line_map(&mp.nl, b.nl[cur], g.PS, g.nx, 3, N) && line_map(&mp.onl, b.nl[old], g.PS, g.nx, 3, N) &&
                line_map(&mp.ff, b.ff, g.PS, g.nx, 3, N)) {
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)std::min(g.PS / LPipe<N>::LT, LPipe<N>::MINB * sm_count()), 1, 1);
                cfg.blockDim = dim3(LPipe<N>::T, 1, 1);
                cfg.dynamicSmemBytes = LPipe<N>::SMEM;
                cfg.stream = s;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                at[0].val.programmaticStreamSerializationAllowed = 1;   // prologue beside the previous kernel's tail
                cfg.attrs = at;
                cfg.numAttrs = 1;
                cudaLaunchKernelEx(&cfg, k_lines_pipe<N>, g, mp, sc);
                return;
            }
        }
    }
    if (lt == 4) k_lines<N, 4><<<(g.PS + 3) / 4, 4 * 32, lines_smem<N>(4), s>>>(g, u, p, b.nl[cur], b.nl[old], b.ff, sc);
    else k_lines<N, 8><<<(g.PS + 7) / 8, 8 * 32, lines_smem<N>(8), s>>>(g, u, p, b.nl[cur], b.nl[old], b.ff, sc);
}

// velstep tail: umean update (steptheflow.F90:99) and the NaN check.
__device__ __forceinline__ void b_scal_d(const Geo &g, Scal *sc) {
    if (threadIdx.x != 0 || sc->status) return;
    for (int d = 0; d < 3; ++d) sc->umean[d] = sc->umean[d] + (-sc->mpg[d] + sc->frmean[d] - sc->frame_accln[d]) * sc->dt;
    if (g.moving)
        for (int d = 0; d < 3; ++d) {   // steptheflow.F90:101-104
            sc->frame_vel[d] = sc->frame_vel[d] + sc->frame_accln[d] * sc->dt;
            sc->frame_pos[d] = sc->frame_pos[d] + sc->frame_vel[d] * sc->dt;
        }
    const double dm = __longlong_as_double((long long)sc->divmax_bits);
    if (!(dm == dm) || !(sc->umean[0] == sc->umean[0]) || !(sc->mpg[0] == sc->mpg[0])) sc->status = PIBM_ERR_NAN;
    sc->nsteps += 1;
}
__global__ void k_scal_d(Geo g, Scal *sc) { b_scal_d(g, sc); }

// ============================================================================
// Layout conversion between the reference's Fortran arrays and the device
// layout (get/set state): u(nx+1,my2,mz,ncomp) <-> [comp][i][kz][ky].
// Tiled 32x32 transpose through shared memory.
// ============================================================================
__global__ void k_f2d(const double2 *__restrict__ f, double2 *__restrict__ d, int nx, int nxf, int PS, int ncomp) {
    __shared__ double2 tile[32][33];
    const int comp = blockIdx.z;
    const int i0 = blockIdx.x * 32, e0 = blockIdx.y * 32;
    const double2 *fc = f + (size_t)comp * PS * nxf;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int e = e0 + r, i = i0 + threadIdx.x;
        if (e < PS && i < nx) tile[r][threadIdx.x] = fc[(size_t)e * nxf + i];
    }
    __syncthreads();
    double2 *dc = d + (size_t)comp * PS * nx;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, e = e0 + threadIdx.x;
        if (e < PS && i < nx) dc[(size_t)i * PS + e] = tile[threadIdx.x][r];
    }
}
__global__ void k_d2f(const double2 *__restrict__ d, double2 *__restrict__ f, int nx, int nxf, int PS, int ncomp) {
    __shared__ double2 tile[32][33];
    const int comp = blockIdx.z;
    const int i0 = blockIdx.x * 32, e0 = blockIdx.y * 32;
    const double2 *dc = d + (size_t)comp * PS * nx;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, e = e0 + threadIdx.x;
        if (e < PS && i < nxf) tile[r][threadIdx.x] = dc[(size_t)(i == nx ? 0 : i) * PS + e];
    }
    __syncthreads();
    double2 *fc = f + (size_t)comp * PS * nxf;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int e = e0 + r, i = i0 + threadIdx.x;
        if (e < PS && i < nxf) fc[(size_t)e * nxf + i] = tile[threadIdx.x][r];
    }
}

// Standalone batched plane transforms (pibm_ff2rc / pibm_ff2cr) on natural
// host layouts: real a[z*my + y], complex b[kz*my2 + ky].
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_ff2cr(Geo g, const double2 *__restrict__ a, double *__restrict__ b) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RS = N * N;
    double2 *buf = sm, *tws = sm + L::BUF;
    load_tw<N>(tws, g);
    const TwT tw{tws, N};
    const size_t q = blockIdx.x / L::C;
    const int rank = blockIdx.x % L::C;
    for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
        const int kz = e / L::PZ, jl = e - kz * L::PZ;
        if (jl == L::MC && rank != 0) continue;
        buf[e] = a[q * PS + kz * my2 + cl_col<N>(jl, rank)];
    }
    __syncthreads();
    cl_c2r<N>(buf, tw, rank);
    const double *rb = (const double *)buf;
    for (int e = threadIdx.x; e < L::NR * N; e += L::T) {
        const int r = e / N, y = e - r * N;
        const int z = zinv<N>(rank * L::NR + r);
        b[q * RS + (size_t)z * N + y] = rb[r * (N + 2) + 2 * yslot<N>(y >> 1) + (y & 1)];
    }
}
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_ff2rc(Geo g, const double *__restrict__ a, double2 *__restrict__ b) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RS = N * N;
    double2 *buf = sm, *tws = sm + L::BUF;
    load_tw<N>(tws, g);
    const TwT tw{tws, N};
    const size_t q = blockIdx.x / L::C;
    const int rank = blockIdx.x % L::C;
    double *rb = (double *)buf;
    for (int e = threadIdx.x; e < L::NR * N; e += L::T) {
        const int r = e / N, y = e - r * N;
        const int z = zinv<N>(rank * L::NR + r);
        rb[r * (N + 2) + 2 * yslot<N>(y >> 1) + (y & 1)] = a[q * RS + (size_t)z * N + y];
    }
    __syncthreads();
    cl_r2c<N>(buf, tw, rank);
    for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
        const int kz = e / L::PZ, jl = e - kz * L::PZ;
        if (jl == L::MC && rank != 0) continue;
        const double2 X = cl_unpack<N>(buf, kz, jl, rank);
        b[q * PS + kz * my2 + cl_col<N>(jl, rank)] = r2c_norm<N>(X, g.nrm);
    }
}

// ============================================================================
// Fused batch step: the kernels of one time step for every run of a batch
// that has the same grid size, one launch per kernel, the runs along
// gridDim.z.  Each run's blocks execute the
// same device code as its own launches, so its results are bitwise those of
// stepping it alone.  Launches are sized for the largest run of the group;
// blocks beyond a run's own extent return at once.  The Member array comes in
// the parameter space (MemberSet), so each run's constants are read through
// the constant cache, as a single run's Geo parameter is.
// ============================================================================
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) kb_a0(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    b_a0<N>(m.g, m.b.u, m.b.p, m.b.ubcp, m.b.pbcp, m.b.omega, m.b.pgr, m.b.sc, m.b.part);
}
__global__ void __launch_bounds__(256) kb_scal_a(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    b_scal_a(m.g, m.b.sc, m.b.part);
}
template <int N>
__global__ void __launch_bounds__(256, 4) kb_flux(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    b_flux<N>(m.g, m.b.ubcp, m.b.Dx, m.b.sc);
}
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) kb_nl(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    b_nl<N>(m.g, m.b.ubcp, m.b.Dx, m.b.u, m.b.nl[m.cur ^ 1], m.b.nl[m.cur], m.b.Q, m.b.sc);
}
template <int N>
__global__ void __launch_bounds__(256) kb_drag(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    if ((int)blockIdx.x >= m.g.nbody * kDragSplit) return;
    b_drag<N>(m.g, m.b.pbcp, m.b.omega, m.b.dpart, m.b.sc);
}
__global__ void __launch_bounds__(256) kb_scal_b(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    if (m.g.nbody == 0) return;
    b_scal_b(m.g, m.b.sc, m.b.pres, m.b.visc, m.b.ptot, m.b.force, m.b.dpart);
}
template <int N>
__global__ void __launch_bounds__(256, 2) kb_rev(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    if (m.g.nbody == 0 || m.g.npts == 0 || (int)blockIdx.x >= m.nbk) return;
    b_rev<N>(m.g, m.b.ubcp, m.b.pgr, m.b.Q, m.b.sc, m.b.rec, m.b.rz, m.b.blockpart);
}
__global__ void __launch_bounds__(256) kb_scal_c(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    if (m.g.nbody == 0 || m.g.npts == 0) return;
    b_scal_c(m.g, m.b.sc, m.b.blockpart, m.nbk);
}
__global__ void __launch_bounds__(256) kb_spread(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    if (m.g.nbody == 0 || m.g.npts == 0) return;
    b_spread(m.g, m.b.rec, m.b.rz, m.b.fr, m.b.sc);
}
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) kb_ff(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    if (m.g.nbody == 0) return;
    b_ff<N>(m.g, m.b.fr, m.b.ff, m.b.sc);
}
// CTAs per SM of the single-run x-line kernels at their register counts,
// kept as a bound here (the indexed parameter loads would raise the count).
template <int N, int LT> constexpr int kb_lines_minb() { return N <= 128 ? (LT == 4 ? 4 : 2) : (LT == 4 ? 2 : 1); }
template <int N, int LT>
__global__ void __launch_bounds__(LT * 32, kb_lines_minb<N, LT>()) kb_lines(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    b_lines<N, LT>(m.g, m.b.u, m.b.p, m.b.nl[m.cur], m.b.nl[m.cur ^ 1], m.b.ff, m.b.sc);
}
__global__ void kb_scal_d(const __grid_constant__ MemberSet ms) {
    const Member &m = ms.m[blockIdx.z];
    b_scal_d(m.g, m.b.sc);
}

// One fused step of nz runs of size N (ms.m[0..nz-1]): the step's scalars,
// the drag and mpg kernels on `side` beside the nonlinear term, and the
// frmean sums beside the spreading, as in a single run's graph.
template <int N>
static void enqueue_batch_step_t(const MemberSet &ms, const BatchShape &bs, cudaStream_t s, cudaStream_t side,
                                 cudaEvent_t fork, cudaEvent_t join) {
    const int nz = bs.nz;
    launch_planes_z<N>(kb_a0<N>, N, 10, nz, s, ms);
    const bool spheres = bs.max_nbody > 0;
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(side, fork, 0);
    kb_scal_a<<<dim3(1, 1, nz), 256, 0, side>>>(ms);
    if (spheres) {
        kb_drag<N><<<dim3(bs.max_nbody * kDragSplit, 1, nz), 256, 0, side>>>(ms);
        kb_scal_b<<<dim3(1, 1, nz), 256, 0, side>>>(ms);
    }
    cudaEventRecord(join, side);
    kb_flux<N><<<dim3((RP<N>::RSP * (N / bs.flux_seg) + 255) / 256, 1, nz), 256, 0, s>>>(ms);
    launch_planes_z<N>(kb_nl<N>, N, 3, nz, s, ms);
    cudaStreamWaitEvent(s, join, 0);
    if (spheres) {
        if (bs.max_nbk > 0) {
            kb_rev<N><<<dim3(bs.max_nbk, 1, nz), 256, 0, s>>>(ms);
            cudaEventRecord(fork, s);
            cudaStreamWaitEvent(side, fork, 0);
            kb_scal_c<<<dim3(1, 1, nz), 256, 0, side>>>(ms);
            cudaEventRecord(join, side);
            if (bs.max_spn > 0) kb_spread<<<dim3((bs.max_spn + 255) / 256, 1, nz), 256, 0, s>>>(ms);
            cudaStreamWaitEvent(s, join, 0);
        }
        launch_planes_z<N>(kb_ff<N>, N, 3, nz, s, ms);
    }
    const int PS = (N / 2 + 1) * N;
    if (bs.lines_lt == 4) kb_lines<N, 4><<<dim3((PS + 3) / 4, 1, nz), 4 * 32, lines_smem<N>(4), s>>>(ms);
    else kb_lines<N, 8><<<dim3((PS + 7) / 8, 1, nz), 8 * 32, lines_smem<N>(8), s>>>(ms);
    kb_scal_d<<<dim3(1, 1, nz), 32, 0, s>>>(ms);
}

void enqueue_batch_step(int n, const MemberSet &ms, const BatchShape &bs, cudaStream_t s, cudaStream_t side,
                        cudaEvent_t fork, cudaEvent_t join) {
    switch (n) {
        case 32: enqueue_batch_step_t<32>(ms, bs, s, side, fork, join); break;
        case 64: enqueue_batch_step_t<64>(ms, bs, s, side, fork, join); break;
        case 96: enqueue_batch_step_t<96>(ms, bs, s, side, fork, join); break;
        case 128: enqueue_batch_step_t<128>(ms, bs, s, side, fork, join); break;
        case 256: enqueue_batch_step_t<256>(ms, bs, s, side, fork, join); break;
    }
}
// Kernels one fused batch step launches.
int batch_kernels_per_step(const BatchShape &bs) {
    return 6 + (bs.max_nbody > 0 ? 3 + (bs.max_nbk > 0 ? 2 + (bs.max_spn > 0 ? 1 : 0) : 0) : 0);
}

// ============================================================================
// Host-side launch helpers
// ============================================================================
template <int N>
static cudaError_t set_attrs() {
    const int maxs = (int)plane_smem<N>();
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_a0<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_nl<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_ff<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_ff2cr<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_ff2rc<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_lines<N, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lines_smem<N>(4))) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_lines<N, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lines_smem<N>(8))) != cudaSuccess) return e;
    if constexpr (N <= 128)
        if ((e = cudaFuncSetAttribute(k_lines_pipe<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, LPipe<N>::SMEM)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(kb_a0<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(kb_nl<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(kb_ff<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(kb_lines<N, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lines_smem<N>(4))) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(kb_lines<N, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lines_smem<N>(8))) != cudaSuccess) return e;
    return cudaSuccess;
}

cudaError_t configure_kernels(int n) {
    switch (n) {
        case 32: return set_attrs<32>();
        case 64: return set_attrs<64>();
        case 96: return set_attrs<96>();
        case 128: return set_attrs<128>();
        case 256: return set_attrs<256>();
        default: return cudaErrorInvalidValue;
    }
}

bool supported_size(int n) { return n == 32 || n == 64 || n == 96 || n == 128 || n == 256; }

// CTAs that share one plane in the plane kernels (per-plane partial sums come in that many parts).
int plane_ctas(int n) {
    switch (n) {
        case 32: return PL<32>::C;
        case 64: return PL<64>::C;
        case 96: return PL<96>::C;
        case 128: return PL<128>::C;
        case 256: return PL<256>::C;
        default: return 1;
    }
}

// Physical offset of real node (z, y) in one plane (host side of real_off).
int real_offset(int n, int z, int y) {
    switch (n) {
        case 32: return real_off<32>(z, y);
        case 64: return real_off<64>(z, y);
        case 96: return real_off<96>(z, y);
        case 128: return real_off<128>(z, y);
        case 256: return real_off<256>(z, y);
        default: return -1;
    }
}

// Enqueue one full step on stream s.  cur = index of the nl buffer that
// receives this step's nonlinear term (the other holds the previous step's).
// ev (phase events, PIBM_NPHASE + 1) or kev (kernel events, 2 per kernel
// slot PIBM_K_*: before and after the slot's launch) select the serial,
// timed variant on one stream; without either, drag + mpg and the scalar
// step fork onto the side streams of ss.
template <int N>
static void enqueue_step_t(const Geo &g, DevBufs &b, int cur, cudaStream_t s, cudaEvent_t *ev, const StepStreams *ss,
                           cudaEvent_t *kev) {
    const int old = 1 - cur;
    auto mark = [&](int q) { if (ev) cudaEventRecord(ev[q], s); };
    auto kb = [&](int k) { if (kev) cudaEventRecord(kev[2 * k], s); };
    auto ke = [&](int k) { if (kev) cudaEventRecord(kev[2 * k + 1], s); };
    auto kskip = [&](int k) { kb(k); ke(k); };
    // forked: the step's scalars (k_scal_a), drag + mpg on ss->side and the scalar
    // step on ss->scal run beside the x flux and the nonlinear term, which read
    // only k_a0's real fields, and the frmean sums (k_scal_c) beside the
    // spreading; the timed variants keep one serial stream.  With a passive
    // scalar k_scal_a and k_scal_c stay on the main stream: the scalar's plane
    // kernels then start with the x flux and fill the GPU, and the flow's short
    // side kernels measured slower queued beside them.
    const bool fork = ss && !ev && !kev;
    const bool scal_first = g.scal && !g.moving;
    mark(0);
    kb(PIBM_K_A0);
    launch_planes_pdl<N>(k_a0<N>, g.nx, 10, s, g, (const double2 *)b.u, (const double2 *)b.p, b.ubcp, b.pbcp, b.omega, b.pgr, b.sc, b.part);
    ke(PIBM_K_A0);
    if (fork) {
        if (scal_first) k_scal_a<<<1, 256, 0, s>>>(g, b.sc, b.part);
        cudaEventRecord(ss->fork, s);
        cudaStreamWaitEvent(ss->side, ss->fork, 0);
        if (scal_first) {
            cudaStreamWaitEvent(ss->scal, ss->fork, 0);
            enqueue_scalar(g, b, cur, ss->scal);
            cudaEventRecord(ss->scal_done, ss->scal);
        } else {
            k_scal_a<<<1, 256, 0, ss->side>>>(g, b.sc, b.part);
        }
        if (g.nbody > 0) {
            k_drag<N><<<g.nbody * kDragSplit, 256, 0, ss->side>>>(g, b.pbcp, b.omega, b.dpart, b.sc);
            k_scal_b<<<1, 256, 0, ss->side>>>(g, b.sc, b.pres, b.visc, b.ptot, b.force, b.dpart);
        }
        cudaEventRecord(ss->drag_done, ss->side);
    } else {
        kb(PIBM_K_SCAL_A);
        k_scal_a<<<1, 256, 0, s>>>(g, b.sc, b.part);
        ke(PIBM_K_SCAL_A);
    }
    mark(1);
    kb(PIBM_K_FLUX);
    const int fgrid = (RP<N>::RSP * (g.nx / g.flux_seg) + 255) / 256;
    if (scal_first) k_flux<N, 3><<<fgrid, 256, 0, s>>>(g, b.ubcp, b.Dx, b.sc);
    else k_flux<N, 4><<<fgrid, 256, 0, s>>>(g, b.ubcp, b.Dx, b.sc);
    ke(PIBM_K_FLUX);
    kb(PIBM_K_NL);
    launch_planes_pdl<N>(k_nl<N>, g.nx, 3, s, g, (const double *)b.ubcp, (const double *)b.Dx, (const double2 *)b.u,
                         (const double2 *)b.nl[old], b.nl[cur], b.Q, b.sc);
    ke(PIBM_K_NL);
    mark(2);
    if (fork) cudaStreamWaitEvent(s, ss->drag_done, 0);
    if (g.nbody > 0) {
        if (!fork) {
            kb(PIBM_K_DRAG);
            k_drag<N><<<g.nbody * kDragSplit, 256, 0, s>>>(g, b.pbcp, b.omega, b.dpart, b.sc);
            ke(PIBM_K_DRAG);
            kb(PIBM_K_SCAL_B);
            k_scal_b<<<1, 256, 0, s>>>(g, b.sc, b.pres, b.visc, b.ptot, b.force, b.dpart);
            ke(PIBM_K_SCAL_B);
        }
        if (g.moving) {
            enqueue_moving(g, b.mov, b.sc, b.pres, b.visc, s);
            if (fork && g.scal) {   // the scalar step needs the new geometry
                cudaEventRecord(ss->geo_done, s);
                cudaStreamWaitEvent(ss->scal, ss->geo_done, 0);
                enqueue_scalar(g, b, cur, ss->scal);
                cudaEventRecord(ss->scal_done, ss->scal);
            }
        }
        mark(3);
        const int nbk = (g.npts + 255) / 256;
        if (g.npts > 0) {
            kb(PIBM_K_REV);
            if (scal_first) k_rev<N, 3><<<nbk, 256, 0, s>>>(g, b.ubcp, b.pgr, b.Q, b.sc, b.rec, b.rz, b.blockpart);
            else k_rev<N, 2><<<nbk, 256, 0, s>>>(g, b.ubcp, b.pgr, b.Q, b.sc, b.rec, b.rz, b.blockpart);
            ke(PIBM_K_REV);
            if (fork && !scal_first) {
                // frmean (read from k_ff on) beside the spreading, which does not read it
                cudaEventRecord(ss->rev_done, s);
                cudaStreamWaitEvent(ss->side, ss->rev_done, 0);
                k_scal_c<<<1, 256, 0, ss->side>>>(g, b.sc, b.blockpart, nbk);
                cudaEventRecord(ss->frmean_done, ss->side);
            } else {
                kb(PIBM_K_SCAL_C);
                k_scal_c<<<1, 256, 0, s>>>(g, b.sc, b.blockpart, nbk);
                ke(PIBM_K_SCAL_C);
            }
            kb(PIBM_K_SPREAD);
            if (g.moving) enqueue_spread_dyn(g, b.mov, b.rec, b.rz, b.fr, b.sc, s);
            else if (g.sp_nnodes > 0) k_spread<<<(g.sp_nnodes + 255) / 256, 256, 0, s>>>(g, b.rec, b.rz, b.fr, b.sc);
            ke(PIBM_K_SPREAD);
            if (fork && !scal_first) cudaStreamWaitEvent(s, ss->frmean_done, 0);
        } else {
            kskip(PIBM_K_REV); kskip(PIBM_K_SCAL_C); kskip(PIBM_K_SPREAD);
        }
        mark(4);
        kb(PIBM_K_FF);
        launch_planes_pdl<N>(k_ff<N>, g.nx, 3, s, g, (const double *)b.fr, b.ff, b.sc);
        ke(PIBM_K_FF);
    } else {
        mark(3); mark(4);
        kskip(PIBM_K_DRAG); kskip(PIBM_K_SCAL_B); kskip(PIBM_K_REV); kskip(PIBM_K_SCAL_C); kskip(PIBM_K_SPREAD);
        kskip(PIBM_K_FF);
    }
    mark(5);
    kb(PIBM_K_LINES);
    launch_lines<N>(g, b, b.u, b.p, cur, b.sc, s);
    ke(PIBM_K_LINES);
    kb(PIBM_K_SCAL_D);
    k_scal_d<<<1, 32, 0, s>>>(g, b.sc);
    ke(PIBM_K_SCAL_D);
    mark(6);
    if (g.scal) {
        if (fork) cudaStreamWaitEvent(s, ss->scal_done, 0);
        else enqueue_scalar(g, b, cur, s);
    }
    mark(7);
}

// Kernels launched per step (for launch accounting).
int kernels_per_step(const Geo &g, const Mov &m) {
    int n = 6;   // a0, scal_a, flux, nl, lines, scal_d
    if (g.nbody > 0) n += 3 + (g.npts > 0 ? 2 + (g.sp_nnodes > 0 || g.moving ? 1 : 0) : 0);
    if (g.moving) n += moving_kernels_per_step(m);
    return n + scalar_kernels_per_step(g);
}

void enqueue_step(const Geo &g, DevBufs &b, int cur, cudaStream_t s, cudaEvent_t *ev, const StepStreams *ss,
                  cudaEvent_t *kev) {
    switch (g.my) {
        case 32: enqueue_step_t<32>(g, b, cur, s, ev, ss, kev); break;
        case 64: enqueue_step_t<64>(g, b, cur, s, ev, ss, kev); break;
        case 96: enqueue_step_t<96>(g, b, cur, s, ev, ss, kev); break;
        case 128: enqueue_step_t<128>(g, b, cur, s, ev, ss, kev); break;
        case 256: enqueue_step_t<256>(g, b, cur, s, ev, ss, kev); break;
    }
}

template <int N>
static void enqueue_c2r_t(const Geo &g, const double2 *a, double *b, int nplanes, cudaStream_t s) {
    launch_planes<N>(k_ff2cr<N>, nplanes, 1, s, g, a, b);
}
void enqueue_c2r(const Geo &g, const double2 *a, double *b, int nplanes, cudaStream_t s) {
    switch (g.my) {
        case 32: enqueue_c2r_t<32>(g, a, b, nplanes, s); break;
        case 64: enqueue_c2r_t<64>(g, a, b, nplanes, s); break;
        case 96: enqueue_c2r_t<96>(g, a, b, nplanes, s); break;
        case 128: enqueue_c2r_t<128>(g, a, b, nplanes, s); break;
        case 256: enqueue_c2r_t<256>(g, a, b, nplanes, s); break;
    }
}
template <int N>
static void enqueue_r2c_t(const Geo &g, const double *a, double2 *b, int nplanes, cudaStream_t s) {
    launch_planes<N>(k_ff2rc<N>, nplanes, 1, s, g, a, b);
}
void enqueue_r2c(const Geo &g, const double *a, double2 *b, int nplanes, cudaStream_t s) {
    switch (g.my) {
        case 32: enqueue_r2c_t<32>(g, a, b, nplanes, s); break;
        case 64: enqueue_r2c_t<64>(g, a, b, nplanes, s); break;
        case 96: enqueue_r2c_t<96>(g, a, b, nplanes, s); break;
        case 128: enqueue_r2c_t<128>(g, a, b, nplanes, s); break;
        case 256: enqueue_r2c_t<256>(g, a, b, nplanes, s); break;
    }
}

// ---------------------------------------------------------------------------
// Autotuner of the x-line tile width: every candidate width runs on scratch
// copies of the state (the run's own state is not touched; results do not
// depend on the width): whole steps where the state is u, p, nl and the
// scalars, else the line kernel behind the forcing transform; two warm-up
// units, then `reps` units timed together; the fastest width is kept in
// g.lines_lt.  ms[k] = mean time per unit of candidate kLinesTiles[k].
// ---------------------------------------------------------------------------
extern const int kLinesTiles[2] = {4, 8};
template <int N>
static cudaError_t autotune_lines_t(Geo &g, DevBufs &b, int cur, cudaStream_t s, double ms[2]) {
    const size_t SC = (size_t)g.nx * g.PS;
    // Runs with fixed particles time complete steps on scratch copies of their
    // state (u, p, nl, the scalars and, with a passive scalar, its phi and
    // nonlinear terms): the line kernel's cost depends on what runs beside
    // and before it (the persistent kernel measured faster inside the step
    // and slower in isolation than the staged one).  Moving-particle runs,
    // whose state includes the particles, time the line kernel behind the
    // forcing transform that precedes it.
    const bool whole = !g.moving;
    const bool scal = whole && g.scal;
    const size_t NR1 = (size_t)(g.nx + 1) * g.RS;
    double2 *u = nullptr, *p = nullptr, *nl0 = nullptr, *nl1 = nullptr, *phif = nullptr, *ns0 = nullptr, *ns1 = nullptr;
    double *nr0 = nullptr, *nr1 = nullptr;
    Scal *sc = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&u, 3 * SC * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&p, SC * sizeof(double2));
    if (e == cudaSuccess && whole) e = cudaMalloc(&nl0, 3 * SC * sizeof(double2));
    if (e == cudaSuccess && whole) e = cudaMalloc(&nl1, 3 * SC * sizeof(double2));
    if (e == cudaSuccess && scal) e = cudaMalloc(&phif, SC * sizeof(double2));
    if (e == cudaSuccess && scal) e = cudaMalloc(&ns0, SC * sizeof(double2));
    if (e == cudaSuccess && scal) e = cudaMalloc(&ns1, SC * sizeof(double2));
    if (e == cudaSuccess && scal) e = cudaMalloc(&nr0, NR1 * sizeof(double));
    if (e == cudaSuccess && scal) e = cudaMalloc(&nr1, NR1 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&sc, sizeof(Scal));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const int reps = whole ? 6 : 10;
    double best = 1e30;
    int pick = 0;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        Geo gt = g;
        gt.lines_lt = kLinesTiles[k];
        cudaMemcpyAsync(u, b.u, 3 * SC * sizeof(double2), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(p, b.p, SC * sizeof(double2), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(sc, b.sc, sizeof(Scal), cudaMemcpyDeviceToDevice, s);
        DevBufs bt = b;
        if (whole) {
            cudaMemcpyAsync(nl0, b.nl[0], 3 * SC * sizeof(double2), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(nl1, b.nl[1], 3 * SC * sizeof(double2), cudaMemcpyDeviceToDevice, s);
            bt.u = u; bt.p = p; bt.nl[0] = nl0; bt.nl[1] = nl1; bt.sc = sc;
        }
        if (scal) {
            cudaMemcpyAsync(phif, b.phif, SC * sizeof(double2), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(ns0, b.nls[0], SC * sizeof(double2), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(ns1, b.nls[1], SC * sizeof(double2), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(nr0, b.nlr[0], NR1 * sizeof(double), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(nr1, b.nlr[1], NR1 * sizeof(double), cudaMemcpyDeviceToDevice, s);
            bt.phif = phif; bt.nls[0] = ns0; bt.nls[1] = ns1; bt.nlr[0] = nr0; bt.nlr[1] = nr1;
        }
        int c = cur;
        auto unit = [&]() {
            if (whole) {
                enqueue_step(gt, bt, c, s, nullptr, nullptr, nullptr);
                c ^= 1;
            } else {
                // the forcing transform writes only the work field ff, which the
                // step recomputes before its line kernel; runs without
                // particles have no forcing (fr is not allocated, ff stays zero)
                if (g.nbody > 0 && b.fr) launch_planes<N>(k_ff<N>, g.nx, 3, s, g, (const double *)b.fr, b.ff, sc);
                launch_lines<N>(gt, b, u, p, cur, sc, s);
            }
        };
        unit();   // warm-up
        unit();
        cudaEventRecord(e0, s);
        for (int r = 0; r < reps; ++r) unit();
        cudaEventRecord(e1, s);
        e = cudaEventSynchronize(e1);
        float t = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
        ms[k] = t / reps;
        if (ms[k] < best) { best = ms[k]; pick = k; }
    }
    // the scratch steps wrote the per-particle outputs: a run that has not
    // stepped reports zeros
    if (e == cudaSuccess && whole && g.nbody > 0) {
        for (double *f : {b.pres, b.visc, b.ptot, b.force})
            if (f) cudaMemsetAsync(f, 0, 3 * (size_t)g.nbody * sizeof(double), s);
        if (scal && b.flux_body) cudaMemsetAsync(b.flux_body, 0, (size_t)g.nbody * sizeof(double), s);
        e = cudaStreamSynchronize(s);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) g.lines_lt = kLinesTiles[pick];
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(u);
    cudaFree(p);
    cudaFree(nl0);
    cudaFree(nl1);
    cudaFree(phif);
    cudaFree(ns0);
    cudaFree(ns1);
    cudaFree(nr0);
    cudaFree(nr1);
    cudaFree(sc);
    return e;
}
cudaError_t autotune_lines(Geo &g, DevBufs &b, int cur, cudaStream_t s, double ms[2]) {
    switch (g.my) {
        case 32: return autotune_lines_t<32>(g, b, cur, s, ms);
        case 64: return autotune_lines_t<64>(g, b, cur, s, ms);
        case 96: return autotune_lines_t<96>(g, b, cur, s, ms);
        case 128: return autotune_lines_t<128>(g, b, cur, s, ms);
        case 256: return autotune_lines_t<256>(g, b, cur, s, ms);
    }
    return cudaErrorInvalidValue;
}

void enqueue_f2d(const double2 *f, double2 *d, int nx, int nxf, int PS, int ncomp, cudaStream_t s) {
    dim3 grid((nx + 31) / 32, (PS + 31) / 32, ncomp);
    k_f2d<<<grid, dim3(32, 8), 0, s>>>(f, d, nx, nxf, PS, ncomp);
}
void enqueue_d2f(const double2 *d, double2 *f, int nx, int nxf, int PS, int ncomp, cudaStream_t s) {
    dim3 grid((nxf + 31) / 32, (PS + 31) / 32, ncomp);
    k_d2f<<<grid, dim3(32, 8), 0, s>>>(d, f, nx, nxf, PS, ncomp);
}

}  // namespace pibm
