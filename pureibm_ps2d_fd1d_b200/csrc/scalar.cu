// scalar.cu -- sm_100a FP64 kernels of the passive-scalar step (ISCALON = 1,
// one species), enqueued after the flow step: scalstep,
// SRC/SCALAR/stepthescalar.F90:51-94.
//
// The scalar is periodic in x up to a factor, phi(x + Lx) = phi(x)/heat_ratio
// (fully developed heat transfer, SRC/SCALAR/nl_allphi.F90:256-330), so every
// x wrap multiplies by heat_ratio (or divides), and the plane nx+1 that the
// reference keeps as an image of plane 1 is formed where it is read.
//
// Step pipeline (reference routines in brackets):
//   k_sa     per plane and item: phi, diffn, grad phi (c2r); the image plane's
//            phi and its fluid sums of u*phi and u   [form_nlphi, calc_diffn,
//                                                     compute_phim_heat_ratio]
//   k_sheat  heat_ratio_new = 1 / mixed-mean phi of plane nx+1
//   k_sflux  x flux of u*phi (upwind MUSCL + Rusanov, or centred) and its
//            difference per node                       [form_nlphi]
//   k_snl    nlphi = -(i ky F(v phi) + i kz F(w phi) + F(D)), its c2r  [form_nlphi, nlphi_graduphi]
//   k_simg   c2r of nlphi(1)/heat_ratio (image plane)
//   k_sbnd   surface flux per sphere from grad phi       [calc_bndrev_data]
//   k_srev   forcing per reversal-point evaluation       [calc_inner_rev_data]
//   k_sspread  gather of the forcing onto solid nodes in reference order
//   k_sff    r2c of the forcing                          [bcsetscal]
//   k_slines per (ky,kz) line: Crank-Nicolson solve with twisted-periodic
//            corners                                      [phistep]
//   k_sfin   heat_ratio update, Nusselt number, status
#include "step_common.cuh"

namespace pibm {

// Spectral phi of plane i (1-based, 1..nx+1) at element ge: plane nx+1 is
// phif(1)/heat_ratio (the reference stores that image, stepthescalar.F90:210).
__device__ __forceinline__ double2 phi_at(const Geo &g, const double2 *__restrict__ phif, int i, int ge, double h) {
    if (i <= g.nx) return phif[(size_t)(i - 1) * g.PS + ge];
    const double2 v = phif[ge];
    return make_double2(v.x / h, v.y / h);
}

// ============================================================================
// k_sa: item t of plane p (p = nx is the image plane nx+1):
//   t = 0  phi = c2r(phif) -> phr (p = nx: -> phimg, and the fluid sums of
//          u*phi, u and the fluid count of that plane into spart)
//   t = 1  diffn = c2r(gamma*((phif(i-1) - 2 phif(i) + phif(i+1))/dx^2 - k^2 phif(i))) -> sdf
//   t = 2  d phi/dx (centred), t = 3, 4  i ky phif, i kz phif -> gph
// (nl_allphi.F90:96-114, 256-330; bc_scalar.F90:935-1033, serial branches)
// ============================================================================
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_sa(Geo g, const double2 *__restrict__ phif,
                                                              const double *__restrict__ ubcp, double *__restrict__ phr,
                                                              double *__restrict__ phimg, double *__restrict__ sdf,
                                                              double *__restrict__ gph, const Scal *__restrict__ sc,
                                                              double *__restrict__ spart) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, RSP = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    __shared__ double scr[32];
    load_tw<N>(tws, g);
    __syncthreads();
    const int p = blockIdx.x / L::C, rank = blockIdx.x % L::C, nx = g.nx, t = blockIdx.y;
    const int i = p + 1;   // reference plane index
    const size_t roff = (size_t)rank * L::RL;
    const TwT tw{tws, N};
    const double h = sc->heat_ratio, tdx = 2.0 * g.dx, rtdx = 1.0 / tdx;   // reciprocal for qdiv
#pragma unroll 4
    for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
        const int kz = e / L::PZ, jl = e - kz * L::PZ;
        if (jl == L::MC && rank != 0) continue;
        const int j = cl_col<N>(jl, rank), ge = kz * my2 + j;
        const double2 c = phi_at(g, phif, i, ge, h);
        double2 f;
        if (t == 0) {
            f = c;
        } else if (t == 1) {
            double2 a;
            if (i == 1) {
                const double2 pm = phi_at(g, phif, nx, ge, h), pp = phi_at(g, phif, 2, ge, h);
                a = make_double2((pm.x * h - 2.0 * c.x) + pp.x, (pm.y * h - 2.0 * c.y) + pp.y);
            } else if (i == nx || i == nx + 1) {
                const double2 pm = phi_at(g, phif, i - 1, ge, h), q = phi_at(g, phif, i == nx ? 1 : 2, ge, h);
                a = make_double2((pm.x - 2.0 * c.x) + q.x / h, (pm.y - 2.0 * c.y) + q.y / h);
            } else {
                const double2 pm = phi_at(g, phif, i - 1, ge, h), pp = phi_at(g, phif, i + 1, ge, h);
                a = make_double2((pm.x - 2.0 * c.x) + pp.x, (pm.y - 2.0 * c.y) + pp.y);
            }
            const double w2 = g.w2[ge];
            a = make_double2(g.rdx2 * a.x, g.rdx2 * a.y);
            a = make_double2(a.x - w2 * c.x, a.y - w2 * c.y);
            f = make_double2(a.x * g.gamma_s, a.y * g.gamma_s);
        } else if (t == 2) {
            if (i == 1) {
                const double2 pp = phi_at(g, phif, 2, ge, h), pm = phi_at(g, phif, nx, ge, h);
                f = make_double2(qdiv(pp.x - pm.x * h, tdx, rtdx), qdiv(pp.y - pm.y * h, tdx, rtdx));
            } else if (i == nx || i == nx + 1) {
                const double2 q = phi_at(g, phif, i == nx ? 1 : 2, ge, h), pm = phi_at(g, phif, i - 1, ge, h);
                f = make_double2(qdiv(q.x / h - pm.x, tdx, rtdx), qdiv(q.y / h - pm.y, tdx, rtdx));
            } else {
                const double2 pp = phi_at(g, phif, i + 1, ge, h), pm = phi_at(g, phif, i - 1, ge, h);
                f = make_double2(qdiv(pp.x - pm.x, tdx, rtdx), qdiv(pp.y - pm.y, tdx, rtdx));
            }
        } else {
            const double k = t == 3 ? g.ky[j] : g.kz[kz];
            f = make_double2(-c.y * k, c.x * k);
        }
        buf[e] = f;
    }
    __syncthreads();
    cl_c2r<N>(buf, tw, rank);
    double *dst;
    if (t == 0) {
        dst = p < nx ? phr + (size_t)p * RSP : phimg;
        if (p == nx) {
            // compute_phim_heat_ratio over plane nx+1 = image of plane 1 (fluid_atijk(mx) = fluid_atijk(1))
            const double *b = (const double *)buf;
            const double *u1 = ubcp + roff;
            const uint8_t *fl = g.fluid + roff;
            double sp = 0.0, su = 0.0, cnt = 0.0;
            for (int e = threadIdx.x; e < L::RL; e += L::T) {
                if (e % (N + 2) >= N || !fl[e]) continue;
                sp += u1[e] * b[e];
                su += u1[e];
                cnt += 1.0;
            }
            sp = block_sum(sp, scr);
            su = block_sum(su, scr);
            cnt = block_sum(cnt, scr);
            if (threadIdx.x == 0) { spart[rank * 3 + 0] = sp; spart[rank * 3 + 1] = su; spart[rank * 3 + 2] = cnt; }
        }
    } else if (t == 1) {
        dst = sdf + (size_t)p * RSP;
    } else {
        dst = gph + ((size_t)(t - 2) * (nx + 1) + p) * RSP;
    }
    if (threadIdx.x == 0) { bulk_store(dst + roff, buf, L::RBYTES); bulk_wait_read(); }
}

// heat_ratio_new = 1/phim(nx+1), phim = sum(u phi) / (um * count), um = sum(u)/count
// (nl_allphi.F90:280-301).
__global__ void k_sheat(Geo g, Scal *sc, const double *spart) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || sc->status) return;
    double sp = 0.0, su = 0.0, cnt = 0.0;
    for (int r = 0; r < g.plane_ctas; ++r) { sp += spart[r * 3 + 0]; su += spart[r * 3 + 1]; cnt += spart[r * 3 + 2]; }
    const double um = su / cnt;
    const double phim = sp / (um * cnt);
    sc->heat_ratio_new = 1.0 / phim;
}

// ============================================================================
// k_sflux: x-flux difference of u*phi at every node of planes 1..nx
// (form_nlphi, nl_allphi.F90:115-214, serial branch).  One thread per (y,z)
// node walks along x.  Upwind: MUSCL states with unlimited slopes and a
// Rusanov flux at interfaces 0..nx; the states across the periodic boundary
// carry heat_ratio.  Centred: (u phi)(i+1) - (u phi)(i-1) over 2 dx, with
// (u phi)(0) = (u phi)(nx) * heat_ratio.
// ============================================================================
template <int N>
__global__ void __launch_bounds__(256) k_sflux(Geo g, const double *__restrict__ ubcp, const double *__restrict__ phr,
                                               const double *__restrict__ phimg, double *__restrict__ dsx,
                                               const Scal *__restrict__ sc) {
    // one thread per (y,z) node and segment of SEG planes
    constexpr int RSP = RP<N>::RSP, SEG = kScalarFluxSeg;
    const int nx = g.nx, nseg = (nx + SEG - 1) / SEG;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int e = t % RSP, sg = t / RSP;
    if (sg >= nseg || (e % (N + 2)) >= N || sc->status) return;
    const int i0 = sg * SEG + 1, i1 = min(nx, (sg + 1) * SEG);
    const double h = sc->heat_ratio, dx = g.dx, hdx = dx / 2.0, tdx = 2.0 * dx;
    const double rtdx = 1.0 / tdx, rdx = 1.0 / dx;   // reciprocals for qdiv
    auto U = [&](int i) { return __ldg(ubcp + (size_t)(i <= nx ? i - 1 : i - 1 - nx) * RSP + e); };   // i in 1..nx+2
    auto PB = [&](int i) { return i <= nx ? __ldg(phr + (size_t)(i - 1) * RSP + e) : __ldg(phimg + e); };  // i in 1..nx+1
    if (g.scheme == PIBM_SCHEME_CENTER) {
        double fm = i0 == 1 ? (U(nx) * PB(nx)) * h : U(i0 - 1) * PB(i0 - 1);   // fdderiv(i0-1), fdderiv(0) = fdderiv(nx)*h
        double f0 = U(i0) * PB(i0);
        for (int i = i0; i <= i1; ++i) {
            const double fp = U(i + 1) * PB(i + 1);
            dsx[(size_t)(i - 1) * RSP + e] = qdiv(fp - fm, tdx, rtdx);
            fm = f0;
            f0 = fp;
        }
        return;
    }
    // slopes of cell c (1..nx): (pfp phi(c+1) - pfm phi(c-1)) / 2dx, pfm = heat_ratio at c = 1
    auto slope_phi = [&](int c) {
        return c == 1 ? qdiv(1.0 * PB(2) - h * PB(nx), tdx, rtdx) : qdiv(1.0 * PB(c + 1) - 1.0 * PB(c - 1), tdx, rtdx);
    };
    auto slope_u = [&](int c) { return qdiv(U(c + 1) - U(c == 1 ? nx : c - 1), tdx, rtdx); };
    auto flux = [](double up, double um, double Up, double Um) {
        const double ms = fmax(fabs(um), fabs(up));
        const double f = 0.5 * (up * Up) + 0.5 * (um * Um);
        return f - 0.5 * ms * (Up - Um);
    };
    // Rusanov flux at interface i (between cells i and i+1); 0 and nx are the periodic ends
    auto F = [&](int i) {
        if (i == 0) {
            const double sp0 = qdiv(PB(1) - PB(nx - 1) * h, tdx, rtdx), su0 = qdiv(U(1) - U(nx - 1), tdx, rtdx);
            return flux(U(1) - slope_u(1) * hdx, U(nx) + su0 * hdx, PB(1) - slope_phi(1) * hdx, PB(nx) * h + sp0 * hdx);
        }
        if (i == nx) {
            const double spm = qdiv(PB(2) / h - PB(nx), tdx, rtdx), sum = qdiv(U(2) - U(nx), tdx, rtdx);
            return flux(U(1) - sum * hdx, U(nx) + slope_u(nx) * hdx, PB(1) / h - spm * hdx, PB(nx) + slope_phi(nx) * hdx);
        }
        return flux(U(i + 1) - slope_u(i + 1) * hdx, U(i) + slope_u(i) * hdx, PB(i + 1) - slope_phi(i + 1) * hdx,
                    PB(i) + slope_phi(i) * hdx);
    };
    double Fm = F(i0 - 1);
    for (int i = i0; i <= i1; ++i) {
        const double Fi = F(i);
        dsx[(size_t)(i - 1) * RSP + e] = qdiv(Fi - Fm, dx, rdx);
        Fm = Fi;
    }
}

// ============================================================================
// k_snl: nlphi of plane p = -( i ky F(v phi) + i kz F(w phi) + F(D) ), written to
// the new nonlinear buffer, and its c2r (the real nonlinear term of the IBM)
// (form_nlphi, nl_allphi.F90:96-114, 190-236; nlphi_graduphi, nlphi.F90:116-128).
// ============================================================================
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_snl(Geo g, const double *__restrict__ ubcp,
                                                               const double *__restrict__ phr, const double *__restrict__ dsx,
                                                               double2 *__restrict__ nls, double *__restrict__ nlr,
                                                               Scal *__restrict__ sc) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RSP = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    __shared__ uint64_t mb;
    if (threadIdx.x == 0) mbar_init(&mb, 1);
    load_tw<N>(tws, g);
    __syncthreads();
    uint32_t phase = 0;
    const int p = blockIdx.x / L::C, rank = blockIdx.x % L::C, nx = g.nx;
    const size_t roff = (size_t)rank * L::RL;
    const TwT tw{tws, N};
    double2 *dst = nls + (size_t)p * PS;
    const double *PB = phr + (size_t)p * RSP + roff;
    for (int q = 0; q < 3; ++q) {
        if (q < 2) {
            const double *V = ubcp + ((size_t)(q + 1) * nx + p) * RSP + roff;
            double *b = (double *)buf;
#pragma unroll 4
            for (int e = threadIdx.x; e < L::RL; e += L::T) b[e] = V[e] * PB[e];
            __syncthreads();
        } else {
            if (threadIdx.x == 0) {
                fence_async_smem();
                bulk_load(buf, dsx + (size_t)p * RSP + roff, L::RBYTES, &mb);
            }
            load_wait(&mb, phase, sc);
        }
        cl_r2c<N>(buf, tw, rank);
#pragma unroll 4
        for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
            const int kz = e / L::PZ, jl = e - kz * L::PZ;
            if (jl == L::MC && rank != 0) continue;
            const int j = cl_col<N>(jl, rank), ge = kz * my2 + j;
            const double2 Xr = cl_unpack<N>(buf, kz, jl, rank);
            const double2 X = r2c_norm<N>(Xr, g.nrm);
            if (q == 0) { const double ky = g.ky[j]; dst[ge] = make_double2(-ky * X.y, ky * X.x); }
            else if (q == 1) { const double kzv = g.kz[kz]; dst[ge] = cadd(dst[ge], make_double2(-kzv * X.y, kzv * X.x)); }
            else { const double2 a = cadd(dst[ge], X); dst[ge] = make_double2(-a.x, -a.y); }
        }
        __syncthreads();
    }
    // c2r of the new nonlinear term (each thread re-reads the values it wrote)
#pragma unroll 4
    for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
        const int kz = e / L::PZ, jl = e - kz * L::PZ;
        if (jl == L::MC && rank != 0) continue;
        buf[e] = dst[kz * my2 + cl_col<N>(jl, rank)];
    }
    __syncthreads();
    cl_c2r<N>(buf, tw, rank);
    if (threadIdx.x == 0) { bulk_store(nlr + (size_t)p * RSP + roff, buf, L::RBYTES); bulk_wait_read(); }
}

// k_simg: real nonlinear term of the image plane nx+1 = c2r(nlphif(1)/heat_ratio)
// (nl_allphi.F90:219, nlphi.F90:116-128).
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_simg(Geo g, const double2 *__restrict__ nls,
                                                                double *__restrict__ nlr, const Scal *__restrict__ sc) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, RSP = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    load_tw<N>(tws, g);
    const int rank = blockIdx.x % L::C;
    const TwT tw{tws, N};
    const double h = sc->heat_ratio;
    for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
        const int kz = e / L::PZ, jl = e - kz * L::PZ;
        if (jl == L::MC && rank != 0) continue;
        const double2 v = nls[kz * my2 + cl_col<N>(jl, rank)];
        buf[e] = make_double2(v.x / h, v.y / h);
    }
    __syncthreads();
    cl_c2r<N>(buf, tw, rank);
    if (threadIdx.x == 0) { bulk_store(nlr + (size_t)g.nx * RSP + (size_t)rank * L::RL, buf, L::RBYTES); bulk_wait_read(); }
}

// k_sreal: c2r of spectral planes into the real-field layout of the step
// (transform order, RSP doubles per plane): restores the real nonlinear term
// of a restarted scalar (pibm_set_scalar).
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_sreal(Geo g, const double2 *__restrict__ src, double *__restrict__ dst) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RSP = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    load_tw<N>(tws, g);
    const int p = blockIdx.x / L::C, rank = blockIdx.x % L::C;
    const TwT tw{tws, N};
    for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
        const int kz = e / L::PZ, jl = e - kz * L::PZ;
        if (jl == L::MC && rank != 0) continue;
        buf[e] = src[(size_t)p * PS + kz * my2 + cl_col<N>(jl, rank)];
    }
    __syncthreads();
    cl_c2r<N>(buf, tw, rank);
    if (threadIdx.x == 0) { bulk_store(dst + (size_t)p * RSP + (size_t)rank * L::RL, buf, L::RBYTES); bulk_wait_read(); }
}

// ============================================================================
// Scalar interpolation (interpolate_phidata, SRC/SCALAR/bc_scalar.F90:1036-1153,
// serial): stencil [pc, pc+1] on raw x cells; a corner below plane 1 wraps by
// mxf-1 and carries heat_ratio (heat_ratio_old for the old nonlinear term),
// one beyond mxf wraps back and carries 1/heat_ratio.  Weights as the flow's
// (interp_threed with shape2).
// ============================================================================
struct SSten {
    int pc0;                 // raw x cell
    int jj[2], kk[2];        // wrapped, 0-based
    double xv[2], yv[2], zv[2];
    __device__ __forceinline__ double w(int a, int b, int c) const { return __dmul_rn(__dmul_rn(xv[a], yv[b]), zv[c]); }
};
__device__ __forceinline__ void make_ssten(const Geo &g, const double pos[3], const int pc[3], SSten &s) {
    const double zx = __dsub_rn(pos[0], (double)pc[0]);
    const double zy = __dsub_rn(pos[1], (double)pc[1]);
    const double zz = __dsub_rn(pos[2], (double)pc[2]);
    s.xv[0] = __dsub_rn(1.0, zx); s.xv[1] = zx;
    s.yv[0] = __dsub_rn(1.0, zy); s.yv[1] = zy;
    s.zv[0] = __dsub_rn(1.0, zz); s.zv[1] = zz;
    s.pc0 = pc[0];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        s.jj[q] = wrapi(pc[1] + q, g.my) - 1;
        s.kk[q] = wrapi(pc[2] + q, g.mz) - 1;
    }
}
// x corner a of the stencil: reference plane index (1..nx+1) and the wrap factors
__device__ __forceinline__ int sx_plane(const Geo &g, const SSten &s, int a, double h, double hold, double &pf, double &pfo) {
    int ii = s.pc0 + a;
    pf = 1.0; pfo = 1.0;
    if (ii < 1) { ii = (g.nx + 1) + ii - 1; pf = h; pfo = hold; }
    else if (ii > g.nx + 1) { ii = ii - (g.nx + 1) + 1; pf = 1.0 / h; }
    return ii;
}

// ============================================================================
// k_sbnd: surface flux of sphere m, sum over its surface points of
// (interpolated grad phi) . normal (calc_bndrev_data with DOBND = F,
// bc_scalar.F90:385-556).  kDragSplit CTAs per sphere, partial sums in order.
// ============================================================================
template <int N>
__global__ void __launch_bounds__(256) k_sbnd(Geo g, const double *__restrict__ gph, const Scal *__restrict__ sc,
                                              double *__restrict__ sdpart) {
    __shared__ double scr[32];
    const int m = blockIdx.x / kDragSplit, part = blockIdx.x % kDragSplit, NB = g.nbody, nx = g.nx;
    const int chunk = (g.nbnd + kDragSplit - 1) / kDragSplit;
    const int l0 = part * chunk, l1 = min(g.nbnd, l0 + chunk);
    const size_t CR = (size_t)(nx + 1) * RP<N>::RSP;
    const double h = sc->heat_ratio;
    double acc = 0.0;
    for (int l = l0 + threadIdx.x; l < l1; l += blockDim.x) {
        double xl[3];
        int is[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            xl[d] = __dadd_rn(g.xc[m + d * NB], __dmul_rn(g.bnd[3 * l + d], g.rb));
            is[d] = cell_of(xl[d]);
        }
        if (!(1 <= is[0] && is[0] <= nx)) {
            if (is[0] < 1) { xl[0] = __dsub_rn(__dadd_rn((double)(nx + 1), xl[0]), 1.0); is[0] = (nx + 1) + is[0] - 1; }
            else if (is[0] >= nx + 1) { xl[0] = __dsub_rn(xl[0], (double)nx); is[0] = is[0] - nx; }
        }
        SSten s;
        make_ssten(g, xl, is, s);
        double gb[3];
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            double r = 0.0;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                double pf, pfo;
                const int ii = sx_plane(g, s, a, h, h, pf, pfo);
                const double *G = gph + n * CR + (size_t)(ii - 1) * RP<N>::RSP;
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int c = 0; c < 2; ++c) r = r + (__ldg(G + real_off<N>(s.kk[c], s.jj[b])) * pf) * s.w(a, b, c);
            }
            gb[n] = r;
        }
        double d = 0.0;
#pragma unroll
        for (int n = 0; n < 3; ++n) d = d + gb[n] * g.bnd[3 * l + n];
        acc += d;
    }
    acc = block_sum(acc, scr);
    if (threadIdx.x == 0) sdpart[(size_t)m * kDragSplit + part] = acc;
}

// ============================================================================
// k_srev: forcing of one scalar reversal-point evaluation (calc_inner_rev_data,
// bc_scalar.F90:558-932, serial).  phi is interpolated at the outer point and
// at the inner point, the nonlinear and diffusion terms at the inner point;
// the evaluation's corner contributions w*t/dx^3 go to sctb, the share of the
// fluid corners per solid corner (force_fl / count_so) to sfd.
// ============================================================================
template <int N>
__device__ __forceinline__ double sval(const double *f, int plane, const SSten &s, int b, int c) {
    return __ldg(f + (size_t)plane * RP<N>::RSP + real_off<N>(s.kk[c], s.jj[b]));
}
template <int N>
// two blocks per SM (128 registers), as the flow's reversal forcing
__global__ void __launch_bounds__(256, 2) k_srev(Geo g, const double *__restrict__ phr, const double *__restrict__ nlr,
                                                 const double *__restrict__ onlr, const double *__restrict__ sdf,
                                                 const Scal *__restrict__ sc, double *__restrict__ sctb,
                                                 double *__restrict__ sfd) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= sc->nsev || sc->status) return;
    const int m = g.sev_m[e], l = g.sev_l[e], nx = g.nx;
    const double h = sc->heat_ratio, hold = sc->heat_ratio_old;
    double xli[3], xlo[3];
    int ci[3], co[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        xli[d] = g.sev_x[3 * e + d];
        ci[d] = g.sev_c[3 * e + d];
        xlo[d] = __dadd_rn(xli[d], __dmul_rn(g.bnd[3 * l + d], __dsub_rn(g.ro, g.ri)));
        co[d] = cell_of(xlo[d]);
    }
    SSten so, si;
    make_ssten(g, xlo, co, so);
    make_ssten(g, xli, ci, si);
    // phi at a corner: plane nx+1 holds phi(1)/heat_ratio (nl_allphi.F90:247)
    auto phi = [&](int ii, const SSten &s, int b, int c) {
        return ii <= nx ? sval<N>(phr, ii - 1, s, b, c) : sval<N>(phr, 0, s, b, c) / h;
    };
    double philo = 0.0, phili = 0.0, nll = 0.0, onll = 0.0, dfll = 0.0;
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                double pf, pfo;
                int ii = sx_plane(g, so, a, h, hold, pf, pfo);
                philo = philo + (phi(ii, so, b, c) * pf) * so.w(a, b, c);
                ii = sx_plane(g, si, a, h, hold, pf, pfo);
                phili = phili + (phi(ii, si, b, c) * pf) * si.w(a, b, c);
            }
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        double pf, pfo;
        const int ii = sx_plane(g, si, a, h, hold, pf, pfo);
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const double w = si.w(a, b, c);
                nll = nll + (sval<N>(nlr, ii - 1, si, b, c) * pf) * w;
                onll = onll + (sval<N>(onlr, ii - 1, si, b, c) * pfo) * w;
                dfll = dfll + (sval<N>(sdf, ii - 1, si, b, c) * pf) * w;
            }
    }
    const double ro = g.ro, ri = g.ri, rb = g.rb;
    philo = g.phisurf * (ro - ri) - philo * (rb - ri);
    philo = philo / (ro - rb);
    const double phil = sc->cf * (-philo + phili);
    double t = 0.0;
    t = t + phil;
    t = t - g.c3 * nll - g.c4 * onll;
    t = t - (g.c2 + g.c1) * dfll;
    t = t * g.da2[m] * 1.0 * g.dx;
    int count_fl = 0;
    double force_fl = 0.0;
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                int ii = si.pc0 + a;
                if (ii < 0) ii = (nx + 1) + ii - 1;
                const int mp = ii == 0 ? nx - 1 : (ii == nx + 1 ? 0 : ii - 1);   // fluid_atijk(0) = (nx), (nx+1) = (1)
                const bool fl = g.fluid[(size_t)mp * RP<N>::RSP + real_off<N>(si.kk[c], si.jj[b])] != 0;
                const double v = (si.w(a, b, c) * t) / g.dx3;
                if (fl) { count_fl += 1; force_fl = force_fl + v; }
                sctb[(size_t)e * 8 + a + 2 * b + 4 * c] = v;
            }
    const int count_so = 8 - count_fl;
    sfd[e] = count_so > 0 ? force_fl / (double)count_so : 0.0;
}

// Forcing of the nodes of planes 1..nx, contributions summed in reference order.
__global__ void __launch_bounds__(256) k_sspread(Geo g, const double *__restrict__ sctb, const double *__restrict__ sfd,
                                                 double *__restrict__ sfr, const Scal *__restrict__ sc) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.ssp_nnodes || sc->status) return;
    double v = 0.0;
    for (int k = g.ssp_ptr[q]; k < g.ssp_ptr[q + 1]; ++k) {
        const int en = g.ssp_ent[k];
        v = v + sctb[en];
        if (!g.include_frmeanfluid) v = v + sfd[en >> 3];
    }
    sfr[g.ssp_node[q]] = v;
}

// k_sff: ffphi = r2c(fr) over planes 1..nx (bcsetscal, bc_scalar.F90:323-349).
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_sff(Geo g, const double *__restrict__ sfr, double2 *__restrict__ ffs,
                                                               Scal *__restrict__ sc) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RSP = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    __shared__ uint64_t mb;
    if (threadIdx.x == 0) mbar_init(&mb, 1);
    load_tw<N>(tws, g);
    __syncthreads();
    uint32_t phase = 0;
    const int p = blockIdx.x / L::C, rank = blockIdx.x % L::C;
    const TwT tw{tws, N};
    if (threadIdx.x == 0) {
        fence_async_smem();
        bulk_load(buf, sfr + (size_t)p * RSP + (size_t)rank * L::RL, L::RBYTES, &mb);
    }
    load_wait(&mb, phase, sc);
    cl_r2c<N>(buf, tw, rank);
    double2 *dst = ffs + (size_t)p * PS;
#pragma unroll 4
    for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
        const int kz = e / L::PZ, jl = e - kz * L::PZ;
        if (jl == L::MC && rank != 0) continue;
        const double2 X = cl_unpack<N>(buf, kz, jl, rank);
        dst[kz * my2 + cl_col<N>(jl, rank)] = r2c_norm<N>(X, g.nrm);
    }
}

// ============================================================================
// k_slines: phistep per (ky,kz) line (stepthescalar.F90:99-213).  The system
//   a x(i-1) + b x(i) + c x(i+1) = r(i),  x(0) = H x(nx),  x(nx+1) = x(1)/H,
// H = heat_ratio_new, a = c (the reference's tridag3 + Sherman-Morrison with
// corners a*H and c/H) becomes circulant under x(i) = mu^i y(i), mu^nx = 1/H:
//   (a/mu) y(i-1) + b y(i) + (a mu) y(i+1) = r(i) mu^-i,  y periodic,
// and one warp solves it exactly through its eigenvalues
//   lambda_m = b + a (mu + 1/mu) cos(2 pi m/nx) + i a (mu - 1/mu) sin(2 pi m/nx)
// with a forward FFT in registers, a complex division and the exact inverse.
// LT lines per CTA; loads run over consecutive lines (coalesced).
// ============================================================================
template <int R>
__device__ __forceinline__ void twisted_solve(double2 *row, double a, double b, double mpl, double mmi,
                                              const double *pw, const double *ipw, const Tw &tw, int lane) {
    constexpr int N = R * 32;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        const double2 x = row[i];
        v[r] = make_double2(x.x * ipw[i], x.y * ipw[i]);
    }
    group_fft<R, 32>(v, lane, -1.0, tw);
    const int br = bitrev<32>(lane);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int m = r + R * br;
        const double2 e = tw.t[m * tw.stride];   // (cos, -sin)
        const double lr = (double)N * (b + a * mpl * e.x), li = (double)N * (a * mmi * (-e.y));
        const double den = lr * lr + li * li, rden = 1.0 / den;
        v[r] = make_double2(qdiv(v[r].x * lr + v[r].y * li, den, rden), qdiv(v[r].y * lr - v[r].x * li, den, rden));
    }
    // inverse stages: the lower lane of a pair first multiplies its own value
    // by conj w (the upper by 1), then both take pv + sgn v
#pragma unroll
    for (int h = 1; h < 32; h <<= 1) {
        const bool upper = (lane & h) == 0;
        const double sgn = upper ? 1.0 : -1.0;
        const double2 w = (upper || h == 1) ? make_double2(1.0, 0.0) : tw.stage(h, lane & (h - 1), +1.0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double2 m = h == 1 ? v[r] : cmul(v[r], w);   // the first stage's twiddle is 1
            const double2 pv = shfl_xor2(m, h, 32);
            v[r] = make_double2(__fma_rn(sgn, m.x, pv.x), __fma_rn(sgn, m.y, pv.y));
        }
    }
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw.get((lane * r) % N, +1.0));
    dft_inlane<R>(v, +1.0, tw);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        row[i] = make_double2(v[r].x * pw[i], v[r].y * pw[i]);
    }
    __syncwarp();
}

template <int NX, int LT>
__global__ void __launch_bounds__(LT * 32) k_slines(Geo g, double2 *__restrict__ phif, const double2 *__restrict__ nln,
                                                    const double2 *__restrict__ nlo, const double2 *__restrict__ ffs,
                                                    Scal *__restrict__ sc) {
    constexpr int R = NX / 32, NP = lines_pitch<NX, LT>();
    extern __shared__ double2 sm[];
    double2 *tws = sm;
    double2 *RHS = tws + NX;                       // [line][i], pitch NP
    double *pw = (double *)(RHS + LT * NP);        // mu^(i+1)
    double *ipw = pw + NX;                         // mu^-(i+1)
    double2 *st = (double2 *)(ipw + NX);           // cross-lane stage twiddles
    if (block_failed(sc)) return;
    fill_stage_table<32>(st, g.tw, NX);
    const int PS = g.PS, nx = NX;
    const double h = sc->heat_ratio, H = sc->heat_ratio_new;
    for (int t = threadIdx.x; t < NX; t += blockDim.x) {
        tws[t] = g.tw[t];
        const double lg = log(H) / (double)NX;
        pw[t] = exp(-(double)(t + 1) * lg);
        ipw[t] = exp((double)(t + 1) * lg);
    }
    const double mu = exp(-log(H) / (double)NX), imu = 1.0 / mu;
    const int q0 = blockIdx.x * LT;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const double dt = sc->dt, gm = g.gamma_s, dx2 = g.dx2, rdx2 = 1.0 / dx2;
    const double c1 = g.c1, c2 = g.c2, c3 = g.c3, c4 = g.c4;
    auto PF = [&](int i, int q) -> double2 {   // 1-based plane, nx+1 = phif(1)/heat_ratio_new of the last step
        if (i <= nx) return phif[(size_t)(i - 1) * PS + q];
        const double2 v = phif[q];
        return make_double2(v.x / h, v.y / h);
    };
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT + 1, q = q0 + line;
        if (q >= PS) continue;
        const double w2 = g.w2[q];
        const double2 pc = PF(i, q);
        const double fy = 1.0 - dt * c1 * gm * w2;
        double2 r = make_double2(pc.x * fy, pc.y * fy);
        const double2 nn = nln[(size_t)(i - 1) * PS + q], ff = ffs[(size_t)(i - 1) * PS + q], on = nlo[(size_t)(i - 1) * PS + q];
        r = make_double2(r.x + (dt * c3) * nn.x + dt * ff.x, r.y + (dt * c3) * nn.y + dt * ff.y);
        r = make_double2(r.x + (dt * c4) * on.x, r.y + (dt * c4) * on.y);
        const double k1 = dt * gm * c1;
        double2 lap;
        if (i >= 2) {
            const double2 pm = PF(i - 1, q), pp = PF(i + 1, q);
            lap = make_double2((pm.x + pp.x) - 2.0 * pc.x, (pm.y + pp.y) - 2.0 * pc.y);
        } else {
            const double2 pp = PF(2, q), pm = PF(nx, q);
            lap = make_double2((pp.x - 2.0 * pc.x) + pm.x * h, (pp.y - 2.0 * pc.y) + pm.y * h);
        }
        RHS[line * NP + (i - 1)] = make_double2(r.x + qdiv(k1 * lap.x, dx2, rdx2), r.y + qdiv(k1 * lap.y, dx2, rdx2));
    }
    __syncthreads();
    const int qw = q0 + w;
    if (qw < PS) {
        const double a = -(dt * gm * c2 / dx2);
        const double bd = 1.0 + dt * gm * c2 * (2.0 / dx2 + g.w2[qw]);
        const Tw tw{tws, NX, 1, st};
        twisted_solve<R>(RHS + w * NP, a, bd, mu + imu, mu - imu, pw, ipw, tw, lane);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT, q = q0 + line;
        if (q >= PS) continue;
        phif[(size_t)i * PS + q] = RHS[line * NP + i];
    }
}
template <int NX> struct SLinesCfg { static constexpr int LT = NX >= 256 ? 4 : 8; };
template <int NX>
static size_t slines_smem() {
    constexpr int LT = SLinesCfg<NX>::LT;
    return (size_t)(NX + LT * lines_pitch<NX, LT>() + 32) * sizeof(double2) + 2 * NX * sizeof(double);
}

// heat_ratio update, surface flux and Nusselt number (bcsetscal, bc_scalar.F90:186-190,
// 361-363; stepthescalar.F90:90-91), status.
__global__ void __launch_bounds__(256) k_sfin(Geo g, Scal *sc, const double *sdpart, double *flux_body) {
    if (block_failed(sc)) return;
    for (int m = threadIdx.x; m < g.nbody; m += blockDim.x) {
        double f = 0.0;
        for (int q = 0; q < kDragSplit; ++q) f += sdpart[(size_t)m * kDragSplit + q];
        flux_body[m] = f;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double da1 = g.da1;
    double fg = 0.0;
    for (int m = 0; m < g.nbody; ++m) fg = fg + flux_body[m] * da1;
    sc->flux_global = fg;
    sc->nusselt = -(fg * g.char_length * g.char_length) / (6.0 * g.voldom * sc->maxvolfrac * (g.phisurf - g.phistream));
    const double hn = sc->heat_ratio_new;
    if (!isfinite(hn) || !(hn > 0.0)) { atomicCAS(&sc->status, 0, PIBM_ERR_NAN); return; }
    sc->heat_ratio_old = sc->heat_ratio;
    sc->heat_ratio = hn;
}

// ============================================================================
// Host-side enqueue of the scalar step (after the flow step, same stream).
// ============================================================================
void enqueue_moving_scalar(const Geo &g, const Mov &m, Scal *sc, cudaStream_t s);
void enqueue_sspread_dyn(const Geo &g, const Mov &m, const double *sctb, const double *sfd, double *sfr, Scal *sc, cudaStream_t s);
int moving_scalar_kernels_per_step();

template <int N>
static void enqueue_scalar_t(const Geo &g, DevBufs &b, int cur, cudaStream_t s) {
    const int old = 1 - cur;
    launch_planes<N>(k_sa<N>, g.nx + 1, 5, s, g, (const double2 *)b.phif, (const double *)b.ubcp, b.phr, b.phimg,
                     b.sdf, b.gph, (const Scal *)b.sc, b.spart);
    k_sheat<<<1, 32, 0, s>>>(g, b.sc, b.spart);
    k_sflux<N><<<(RP<N>::RSP * ((g.nx + kScalarFluxSeg - 1) / kScalarFluxSeg) + 255) / 256, 256, 0, s>>>(g, b.ubcp, b.phr, b.phimg, b.dsx, b.sc);
    launch_planes<N>(k_snl<N>, g.nx, 1, s, g, (const double *)b.ubcp, (const double *)b.phr, (const double *)b.dsx,
                     b.nls[cur], b.nlr[cur], b.sc);
    launch_planes<N>(k_simg<N>, 1, 1, s, g, (const double2 *)b.nls[cur], b.nlr[cur], (const Scal *)b.sc);
    if (g.nbody > 0) k_sbnd<N><<<g.nbody * kDragSplit, 256, 0, s>>>(g, b.gph, b.sc, b.sdpart);
    if (g.moving) enqueue_moving_scalar(g, b.mov, b.sc, s);
    if (g.nsev > 0) {
        k_srev<N><<<(g.nsev + 255) / 256, 256, 0, s>>>(g, b.phr, b.nlr[cur], b.nlr[old], b.sdf, b.sc, b.sctb, b.sfd);
        if (g.moving) enqueue_sspread_dyn(g, b.mov, b.sctb, b.sfd, b.sfr, b.sc, s);
        else if (g.ssp_nnodes > 0) k_sspread<<<(g.ssp_nnodes + 255) / 256, 256, 0, s>>>(g, b.sctb, b.sfd, b.sfr, b.sc);
    }
    launch_planes<N>(k_sff<N>, g.nx, 1, s, g, (const double *)b.sfr, b.ffs, b.sc);
    constexpr int LT = SLinesCfg<N>::LT;
    k_slines<N, LT><<<(g.PS + LT - 1) / LT, LT * 32, slines_smem<N>(), s>>>(g, b.phif, b.nls[cur], b.nls[old], b.ffs, b.sc);
    k_sfin<<<1, 256, 0, s>>>(g, b.sc, b.sdpart, b.flux_body);
}

void enqueue_scalar(const Geo &g, DevBufs &b, int cur, cudaStream_t s) {
    switch (g.my) {
        case 32: enqueue_scalar_t<32>(g, b, cur, s); break;
        case 64: enqueue_scalar_t<64>(g, b, cur, s); break;
        case 96: enqueue_scalar_t<96>(g, b, cur, s); break;
        case 128: enqueue_scalar_t<128>(g, b, cur, s); break;
        case 256: enqueue_scalar_t<256>(g, b, cur, s); break;
    }
}

template <int N>
static void enqueue_scalar_c2r_t(const Geo &g, const double2 *src, double *dst, int nplanes, cudaStream_t s) {
    launch_planes<N>(k_sreal<N>, nplanes, 1, s, g, src, dst);
}
// c2r of nplanes spectral planes into the step's real layout.
void enqueue_scalar_c2r(const Geo &g, const double2 *src, double *dst, int nplanes, cudaStream_t s) {
    switch (g.my) {
        case 32: enqueue_scalar_c2r_t<32>(g, src, dst, nplanes, s); break;
        case 64: enqueue_scalar_c2r_t<64>(g, src, dst, nplanes, s); break;
        case 96: enqueue_scalar_c2r_t<96>(g, src, dst, nplanes, s); break;
        case 128: enqueue_scalar_c2r_t<128>(g, src, dst, nplanes, s); break;
        case 256: enqueue_scalar_c2r_t<256>(g, src, dst, nplanes, s); break;
    }
}

int scalar_kernels_per_step(const Geo &g) {
    if (!g.scal) return 0;
    int n = 8;   // sa, sheat, sflux, snl, simg, sff, slines, sfin
    if (g.nbody > 0) n += 1;
    if (g.nsev > 0) n += 1 + (g.ssp_nnodes > 0 || g.moving ? 1 : 0);
    if (g.moving) n += moving_scalar_kernels_per_step();
    return n;
}

template <int N>
static cudaError_t set_scalar_attrs() {
    const int maxs = (int)plane_smem<N>();
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_sa<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_snl<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_simg<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_sreal<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_sff<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_slines<N, SLinesCfg<N>::LT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)slines_smem<N>());
}

cudaError_t configure_scalar_kernels(int n) {
    switch (n) {
        case 32: return set_scalar_attrs<32>();
        case 64: return set_scalar_attrs<64>();
        case 96: return set_scalar_attrs<96>();
        case 128: return set_scalar_attrs<128>();
        case 256: return set_scalar_attrs<256>();
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace pibm
