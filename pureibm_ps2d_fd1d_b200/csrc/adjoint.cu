// adjoint.cu -- sm_100a FP64 kernels of the discrete adjoint of the AB2 step.
//
// The reference has no adjoint.  This is the exact transpose (on the forward
// trajectory) of the step that kernels.cu computes, for fixed spheres, an
// imposed mean pressure gradient (SET_MPG) and a fixed time step.  Objective:
//   J = (1/K) sum_{n=1..K} e . sum_m (pres_m + visc_m)
// (the summed surface force of calc_pres_visc_drag, boundary_condition.F90:
// 1481-1645, evaluated inside step n); gradients dJ/dxc and dJ/dmpg.
// The solid mask, the active reversal points, the fluid flags of the
// spreading stencils and the branches of the upwind flux are those of the
// forward run.
//
// Inner products: spectral arrays sum Re(a conj(b)) over the stored
// half-spectrum, real arrays the plain sum over nodes.  With them
//   c2r^T(r) = c_ky (my mz) r2c(r),   r2c^T(v) = c2r(v / c_ky) / (my mz),
// c_ky = 1 at ky = 0 and my/2, else 2; a complex factor a turns into conj(a);
// every x-line system of velstep is symmetric, so its solve is its own
// transpose; interpolation (trilinear gather) and spreading swap roles, and
// the weights' derivatives give the sphere-position gradient.
//
// One reverse step (enqueue_adjoint_step) reads step n's forward fields
// (ubcp, pbcp, omega, pgr, Q, the point forces rec and the step's Scal),
// stored while the segment holding step n was recomputed from its checkpoint:
//   k_adj_begin   umean update^T (steptheflow.F90:99)
//   k_adj_lines   velstep^T per (ky,kz) line: divcorr^T, ustep^T, pressure^T
//   k_adj_c2r     ff = r2c(fr - frmean) ^T  -> lambda fr;  k_adj_sum -> lambda frmean
//   k_adj_rev     reversal forcing + spreading ^T per active point (+ dJ/dxc, dJ/dmpg)
//   k_adj_drag    the objective's surface quadrature ^T (+ dJ/dxc)
//   k_adj_r2c     lambda Q -> spectral;  k_adj_q: Q = c2r(-c3 nl - c4 onl - c12 diffn) ^T
//   k_adj_c2r     nonlinear term's r2c ^T (5 products, 3 flux differences)
//   k_adj_flux    products and x flux ^T -> lambda ubcp;  k_adj_sum -> lambda umean
//   k_adj_r2c     lambda ubcp, omega, pbcp, pgr -> spectral;  k_adj_assemble -> lambda u, p
#include "step_common.cuh"
#include "line_solve.cuh"
#include "../../include/pibm.h"

namespace pibm {

__device__ __forceinline__ double cky(int j, int N) { return (j == 0 || j == N / 2) ? 1.0 : 2.0; }
// z * (i s) and z * conj(i s) for real s
__device__ __forceinline__ double2 mul_is(double2 z, double s) { return make_double2(-s * z.y, s * z.x); }
__device__ __forceinline__ double2 mul_cis(double2 z, double s) { return make_double2(s * z.y, -s * z.x); }
__device__ __forceinline__ double2 axpy2(double a, double2 x, double2 y) { return make_double2(a * x.x + y.x, a * x.y + y.y); }

// umean_n = umean_{n-1} + (-mpg + frmean - frame_accln) dt
__global__ void k_adj_begin(const Scal *sc, AdjScal *as) {
    if (threadIdx.x >= 3) return;
    const int d = threadIdx.x;
    as->lfrmean[d] = sc->dt * as->lumean[d];
    as->gmpg[d] -= sc->dt * as->lumean[d];
}

// J accumulation after each forward step: e . (visc_total - pres_total)
__global__ void k_adj_jacc(const Scal *sc, AdjScal *as, double e0, double e1, double e2) {
    if (threadIdx.x != 0) return;
    as->J += (e0 * (sc->visc_total[0] - sc->pres_total[0]) + e1 * (sc->visc_total[1] - sc->pres_total[1])) +
             e2 * (sc->visc_total[2] - sc->pres_total[2]);
}

// ============================================================================
// k_adj_lines: velstep^T for a tile of LT (ky,kz) lines (poisson.F90:55-508,
// usteptime.F90:286-499 transposed).  Tiles [line][i] in shared memory, one
// warp per line for the solves, like k_lines.
//   in : lu (3), lp, lnl (3)        lambda of u_n, p_n, nl_n
//   out: lu2 (3) = ustep^T part of lambda u_{n-1};  lp2 = 0 (p_{n-1} does not
//        reach the new state through velstep);  lnl_new = lnl + velstep^T part;
//        lonl, lff = velstep^T parts.
// ============================================================================
template <int NX, int LT>
__global__ void __launch_bounds__(LT * 32) k_adj_lines(Geo g, const double2 *__restrict__ lu, const double2 *__restrict__ lp,
                                                       const double2 *__restrict__ lnl, double2 *__restrict__ lu2,
                                                       double2 *__restrict__ lp2, double2 *__restrict__ lnl_new,
                                                       double2 *__restrict__ lonl, double2 *__restrict__ lff,
                                                       const Scal *__restrict__ sc, AdjScal *as) {
    constexpr int R = NX / 32;
    constexpr int NP = lines_pitch<NX, LT>();
    extern __shared__ double2 sm[];
    double2 *tws = sm;
    double2 *D = tws + NX;                 // lambda d, then lambda of the divcorr right-hand side
    double2 *P = D + LT * NP;              // lambda P, then lambda of the pressure right-hand side
    double2 *U = P + LT * NP;              // [comp][line][i]: lambda u_n -> lambda Us -> lambda r
    double *gam = (double *)(U + 3 * LT * NP);
    double2 *st = (double2 *)(gam + NX);
    double *lcs = (double *)(st + 32);        // per-lane constants of the solves
    double2 *ltr = (double2 *)(lcs + NX);
    for (int t = threadIdx.x; t < NX; t += blockDim.x) tws[t] = g.tw[t];
    fill_stage_table<32>(st, g.tw, NX);
    fill_line_tw<R>(lcs, ltr, g.tw);
    const int PS = g.PS, nx = NX;
    const int q0 = blockIdx.x * LT;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const double dx = g.dx, dx2 = g.dx2, dt = sc->dt, vis = g.vis, rdx2 = 1.0 / dx2;
    const double c1 = g.c1, c2 = g.c2, c3 = g.c3, c4 = g.c4;
    const double alp = (c1 + c2) * dt, c2dtv = (c2 * dt) * vis, gd = dt * vis * c1;
    const LineTw<R> tw{{tws, NX, 1, st}, lcs, ltr};
    auto KY = [&](int q) { return g.ky[q % g.my2]; };
    auto KZ = [&](int q) { return g.kz[q / g.my2]; };
    auto W = [&](int i) { return i < 0 ? i + nx : (i >= nx ? i - nx : i); };
    // ---- load lambda u_n, p_n ----
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT, q = q0 + line;
        const bool in = q < PS;
        for (int n = 0; n < 3; ++n) U[(n * LT + line) * NP + i] = in ? lu[((size_t)n * nx + i) * PS + q] : make_double2(0.0, 0.0);
        P[line * NP + i] = in ? lp[(size_t)i * PS + q] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    // ---- divcorr^T: lambda d ----
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT, q = min(q0 + line, PS - 1);
        const double ky = KY(q), kz = KZ(q), w2 = g.w2[q];
        const double2 *Pl = P + line * NP, *U0 = U + (0 * LT + line) * NP, *U1 = U + (1 * LT + line) * NP, *U2 = U + (2 * LT + line) * NP;
        const double2 pm = Pl[W(i - 1)], p0 = Pl[i], pp = Pl[W(i + 1)];
        double2 v = make_double2(p0.x - c2dtv * (qdiv((pm.x - 2.0 * p0.x) + pp.x, dx2, rdx2) - w2 * p0.x),
                                 p0.y - c2dtv * (qdiv((pm.y - 2.0 * p0.y) + pp.y, dx2, rdx2) - w2 * p0.y));
        const double2 a0 = U0[i], a1 = U0[W(i + 1)];
        v = make_double2(v.x - (alp / dx) * (a0.x - a1.x), v.y - (alp / dx) * (a0.y - a1.y));
        // conj(-alp wy / 2) = i alp ky / 2
        v = cadd(v, mul_is(cadd(U1[i], U1[W(i + 1)]), 0.5 * alp * ky));
        v = cadd(v, mul_is(cadd(U2[i], U2[W(i + 1)]), 0.5 * alp * kz));
        D[line * NP + i] = v;
    }
    __syncthreads();
    const int qw = q0 + w;
    const bool wact = qw < PS;
    const double w2w = wact ? g.w2[qw] : 0.0;
    bool ok = true;
    {
        const double a = 1.0 / dx2 - 0.25 * w2w, bd = -2.0 / dx2 - 0.5 * w2w, c = 1.0 / dx2 - 0.25 * w2w;
        double2 *row = D + w * NP;
        if (wact) {
            if (qw == 0) {
                if (lane == 0) ok = thomas_real(row, gam, a, bd, c, NX - 1) && ok;
                __syncwarp();
            } else {
                circulant_solve<R>(row, a, bd, tw, lane);
            }
        }
    }
    __syncthreads();
    // lambda Us = lambda u_n + (divergence right-hand side)^T lambda D
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT, q = min(q0 + line, PS - 1);
        const double ky = KY(q), kz = KZ(q);
        const double2 dm = D[line * NP + W(i - 1)], d0 = D[line * NP + i];
        double2 *U0 = U + (0 * LT + line) * NP, *U1 = U + (1 * LT + line) * NP, *U2 = U + (2 * LT + line) * NP;
        U0[i] = make_double2(U0[i].x + (dm.x - d0.x) / (dx * alp), U0[i].y + (dm.y - d0.y) / (dx * alp));
        // conj(0.5 wy / alp) = -i 0.5 ky / alp
        U1[i] = cadd(U1[i], mul_cis(cadd(d0, dm), 0.5 * ky / alp));
        U2[i] = cadd(U2[i], mul_cis(cadd(d0, dm), 0.5 * kz / alp));
    }
    __syncthreads();
    // ---- ustep^T: lambda r = A_u^-1 lambda Us per component ----
    if (wact) {
        const double a = -(1.0 * dt * vis * c2 / dx2);
        const double bd = 1.0 + dt * vis * c2 * (1.0 * 2.0 / dx2 + w2w);
        for (int n = 0; n < 3; ++n) circulant_solve<R>(U + (n * LT + w) * NP, a, bd, tw, lane);
    }
    __syncthreads();
    // lambda P += (grad P in the ustep right-hand sides)^T; lambda u_{n-1} (ustep part)
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT, q = q0 + line;
        const int qc = min(q, PS - 1);
        const double ky = KY(qc), kz = KZ(qc), w2 = g.w2[qc];
        const double fy = 1.0 - dt * vis * c1 * w2;
        const double2 *R0 = U + (0 * LT + line) * NP, *R1 = U + (1 * LT + line) * NP, *R2 = U + (2 * LT + line) * NP;
        const int ip = W(i + 1), im = W(i - 1);
        double2 v = P[line * NP + i];
        v = make_double2(v.x - (alp / dx) * (R0[i].x - R0[ip].x), v.y - (alp / dx) * (R0[i].y - R0[ip].y));
        // -conj(alp/2 wy) = i alp ky / 2
        v = cadd(v, mul_is(cadd(R1[i], R1[ip]), 0.5 * alp * ky));
        v = cadd(v, mul_is(cadd(R2[i], R2[ip]), 0.5 * alp * kz));
        P[line * NP + i] = v;
        if (q < PS) {
            const double2 *Rn[3] = {R0, R1, R2};
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                const double2 r0 = Rn[n][i], rm = Rn[n][im], rp = Rn[n][ip];
                lu2[((size_t)n * nx + i) * PS + q] = make_double2(fy * r0.x + qdiv(gd * ((rm.x + rp.x) - 2.0 * r0.x), dx2, rdx2),
                                                                 fy * r0.y + qdiv(gd * ((rm.y + rp.y) - 2.0 * r0.y), dx2, rdx2));
            }
        }
    }
    __syncthreads();
    // ---- pressure^T: lambda S = A_p^-1 lambda P / (c1 + c2) ----
    {
        const double a = 1.0 / dx2 - 0.25 * w2w, bd = -2.0 / dx2 - 0.5 * w2w, c = 1.0 / dx2 - 0.25 * w2w;
        double2 *row = P + w * NP;
        if (wact) {
            if (qw == 0) {
                if (lane == 0) ok = thomas_real(row, gam, a, bd, c, NX - 1) && ok;
                __syncwarp();
            } else {
                circulant_solve<R>(row, a, bd, tw, lane);
            }
        }
    }
    __syncthreads();
    // outputs: lambda nl_new, onl, ff (ustep + pressure parts), lambda p_{n-1} = 0
    for (int t = threadIdx.x; t < LT * NX; t += blockDim.x) {
        const int line = t % LT, i = t / LT, q = q0 + line;
        if (q >= PS) continue;
        const double ky = KY(q), kz = KZ(q);
        const double cs = 1.0 / (c1 + c2);
        const double2 s0 = cscale(P[line * NP + i], cs), sm = cscale(P[line * NP + W(i - 1)], cs);
        const double2 dif = csub(sm, s0), sum = cadd(s0, sm);
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const double2 r = U[(n * LT + line) * NP + i];
            double2 bnl, bff, bon;
            if (n == 0) { bnl = cscale(dif, c3 / dx); bff = cscale(dif, 1.0 / dx); bon = cscale(dif, c4 / dx); }
            else {
                const double k = n == 1 ? ky : kz;   // conj(a wy / 2) = -i a ky / 2
                bnl = mul_cis(sum, c3 * k / 2.0); bff = mul_cis(sum, k / 2.0); bon = mul_cis(sum, c4 * k / 2.0);
            }
            const size_t o = ((size_t)n * nx + i) * PS + q;
            lnl_new[o] = cadd(lnl[o], cadd(cscale(r, dt * c3), bnl));
            lff[o] = cadd(cscale(r, dt), bff);
            lonl[o] = cadd(cscale(r, dt * c4), bon);
        }
        lp2[(size_t)i * PS + q] = make_double2(0.0, 0.0);
    }
    if (!ok) atomicCAS(&as->status, 0, PIBM_ERR_PIVOT);
}

template <int NX>
static size_t adj_lines_smem() {
    constexpr int LT = NX >= 256 ? 4 : 8;
    return (size_t)(NX + 5 * LT * lines_pitch<NX, LT>() + 32) * sizeof(double2) + NX * sizeof(double) + line_tw_bytes<NX / 32>();
}

// ============================================================================
// k_adj_c2r: transposes of the step's r2c transforms, r2c^T(v) = c2r(v / c_ky) / (my mz).
//   mode 0: item n of src (3 components)            -> dst component n
//   mode 1: the nonlinear term nl_c = -(i ky F(p1_c) + i kz F(p2_c) + F(D_c))
//           with src = lambda nl_new and M = -lambda nl_new:
//           items 0..4: the products u0u1, u0u2, u1u1, u1u2, u2u2
//           (conj(i ky) M0, conj(i kz) M0, conj(i ky) M1, conj(i kz) M1 + conj(i ky) M2,
//           conj(i kz) M2), items 5..7: the x-flux differences D_c (M_c).
// ============================================================================
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_adj_c2r(Geo g, const double2 *__restrict__ src, double *__restrict__ dst,
                                                        int mode) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RSP = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    load_tw<N>(tws, g);
    const int i = blockIdx.x / L::C, rank = blockIdx.x % L::C, item = blockIdx.y, nx = g.nx;
    const TwT tw{tws, N};
    for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
        const int kz = e / L::PZ, jl = e - kz * L::PZ;
        if (jl == L::MC && rank != 0) continue;
        const int j = cl_col<N>(jl, rank), ge = kz * my2 + j;
        const double s = 1.0 / (cky(j, N) * g.nrm);
        double2 v;
        if (mode == 0) {
            v = src[((size_t)item * nx + i) * PS + ge];
        } else {
            auto M = [&](int n) { const double2 a = src[((size_t)n * nx + i) * PS + ge]; return make_double2(-a.x, -a.y); };
            const double ky = g.ky[j], kzv = g.kz[kz];
            switch (item) {
                case 0: v = mul_cis(M(0), ky); break;
                case 1: v = mul_cis(M(0), kzv); break;
                case 2: v = mul_cis(M(1), ky); break;
                case 3: v = cadd(mul_cis(M(1), kzv), mul_cis(M(2), ky)); break;
                case 4: v = mul_cis(M(2), kzv); break;
                default: v = M(item - 5); break;
            }
        }
        buf[e] = make_double2(v.x * s, v.y * s);
    }
    __syncthreads();
    cl_c2r<N>(buf, tw, rank);
    if (threadIdx.x == 0) { bulk_store(dst + ((size_t)item * nx + i) * RSP + (size_t)rank * L::RL, buf, L::RBYTES); bulk_wait_read(); }
}

// k_adj_r2c: transposes of the step's c2r transforms, c2r^T(r) = c_ky (my mz) r2c(r),
// over nplanes consecutive real planes (grid.x = nplanes * C).
template <int N>
__global__ void __launch_bounds__(PL<N>::T, PL<N>::MINB) k_adj_r2c(Geo g, const double *__restrict__ src, double2 *__restrict__ dst,
                                                        AdjScal *as) {
    using L = PL<N>;
    extern __shared__ double2 sm[];
    constexpr int my2 = N / 2 + 1, PS = my2 * N, RSP = RP<N>::RSP;
    double2 *buf = sm, *tws = sm + L::BUF;
    __shared__ uint64_t mb;
    if (threadIdx.x == 0) mbar_init(&mb, 1);
    load_tw<N>(tws, g);
    __syncthreads();
    const uint32_t phase = 0;
    const size_t pl = blockIdx.x / L::C;
    const int rank = blockIdx.x % L::C;
    const TwT tw{tws, N};
    if (threadIdx.x == 0) {
        fence_async_smem();
        bulk_load(buf, src + pl * RSP + (size_t)rank * L::RL, L::RBYTES, &mb);
    }
    if (!mbar_wait(&mb, phase)) atomicCAS(&as->status, 0, PIBM_ERR_TIMEOUT);
    __syncthreads();
    cl_r2c<N>(buf, tw, rank);
    for (int e = threadIdx.x; e < L::NOUT; e += L::T) {
        const int kz = e / L::PZ, jl = e - kz * L::PZ;
        if (jl == L::MC && rank != 0) continue;
        const int j = cl_col<N>(jl, rank);
        const double2 X = cl_unpack<N>(buf, kz, jl, rank);
        const double c = cky(j, N);
        dst[pl * PS + kz * my2 + j] = make_double2(X.x * c, X.y * c);
    }
}

// Sum over the nodes of component blockIdx.y of a real field (row padding
// excluded), times sign, added to out[blockIdx.y].
template <int N>
__global__ void __launch_bounds__(256) k_adj_sum(Geo g, const double *__restrict__ f, double *out, double sign) {
    __shared__ double scr[32];
    constexpr int RSP = RP<N>::RSP;
    const size_t CR = (size_t)g.nx * RSP;
    const double *fc = f + (size_t)blockIdx.y * CR;
    double a = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < CR; t += (size_t)gridDim.x * blockDim.x) {
        const int e = (int)(t % RSP);
        if (e % (N + 2) < N) a += fc[t];
    }
    a = block_sum(a, scr);
    if (threadIdx.x == 0) atomicAdd(out + blockIdx.y, sign * a);
}

// dJ/dxc accumulation: one atomic per warp when all its lanes belong to the
// same sphere (points are stored sphere by sphere), else one per lane.
__device__ __forceinline__ void add_gxc(double *gxc, int NB, int m, const double gpos[3]) {
    const unsigned full = 0xffffffffu;
    const int m0 = __shfl_sync(full, m, 0);
    if (__all_sync(full, m == m0)) {
        if (m0 < 0) return;
        double v[3] = {gpos[0], gpos[1], gpos[2]};
#pragma unroll
        for (int d = 0; d < 3; ++d)
            for (int o = 16; o > 0; o >>= 1) v[d] += __shfl_xor_sync(full, v[d], o);
        if ((threadIdx.x & 31) == 0)
            for (int d = 0; d < 3; ++d) atomicAdd(gxc + m0 + d * NB, v[d]);
    } else if (m >= 0) {
        for (int d = 0; d < 3; ++d) atomicAdd(gxc + m + d * NB, gpos[d]);
    }
}

// d w / d pos of a stencil corner (a, b, c): w = xv[a] yv[b] zv[c], xv = (1 - z, z).
__device__ __forceinline__ void sten_dw(const Sten &s, int a, int b, int c, double dw[3]) {
    const double da = a ? 1.0 : -1.0, db = b ? 1.0 : -1.0, dc = c ? 1.0 : -1.0;
    dw[0] = da * s.yv[b] * s.zv[c];
    dw[1] = s.xv[a] * db * s.zv[c];
    dw[2] = s.xv[a] * s.yv[b] * dc;
}

// adjoint of r = sum_corners w f: lf += w lr (atomic), gpos += (dw . f) lr; f may carry a constant shift
template <int N>
__device__ __forceinline__ void spread_adj(const Sten &s, const double *f, double fadd, double *lf, double lr, double gpos[3]) {
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const size_t node = (size_t)s.ii[a] * RP<N>::RSP + real_off<N>(s.kk[c], s.jj[b]);
                atomicAdd(lf + node, s.w(a, b, c) * lr);
                double dw[3];
                sten_dw(s, a, b, c, dw);
                const double fv = f[node] + fadd;
#pragma unroll
                for (int d = 0; d < 3; ++d) gpos[d] += dw[d] * fv * lr;
            }
}

// ============================================================================
// k_adj_rev: calc_inner_reversal_forcing^T (boundary_condition.F90:1104-1479)
// per active reversal point: spreading^T (solid corners, the fluid share
// redistributed over the solid corners, frmean), direct forcing^T, then the
// interpolations^T into lambda ubcp (outer and inner velocity), lambda Q
// (inner) and lambda pgr (inner pressure point); dJ/dxc from the weights of
// all four stencils, dJ/dmpg from the pressure-gradient interpolation.
// ============================================================================
template <int N>
__global__ void __launch_bounds__(256) k_adj_rev(Geo g, const double *__restrict__ ubcp, const double *__restrict__ pgr,
                                                 const double *__restrict__ Q, const double *__restrict__ rec,
                                                 const double *__restrict__ lfr, const Scal *__restrict__ sc, AdjScal *as,
                                                 double *lubcp, double *lQ, double *lpgr, double *gxc) {
    __shared__ double scr[32];
    constexpr int RSP = RP<N>::RSP;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int NB = g.nbody;
    const size_t CR = (size_t)g.nx * RSP;
    double gm[3] = {0, 0, 0}, gpos[3] = {0, 0, 0};
    int m = -1;
    if (p < sc->npts) {
        m = g.pt_m[p];
        const int l = g.pt_l[p];
        double xli[3], xlo[3], xpi[3], snorm[3], rad = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            xli[d] = __dadd_rn(g.xc[m + d * NB], __dmul_rn(g.bnd[3 * l + d], g.ri));
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
        double ft[3];
#pragma unroll
        for (int n = 0; n < 3; ++n) ft[n] = rec[(size_t)p * 6 + n];
        const double sfac = g.da2[m] * g.dr * g.dx;
        const double kap = -(g.rb - g.ri) / (g.ro - g.rb), kapn = g.revernorm == 1 ? kap : 0.0;
        const double rnc = 1.0 / (double)g.ncell;
        // spreading^T
        int count_fl = 0;
        double lsol[3] = {0, 0, 0};
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const size_t node = (size_t)si.ii[a] * RSP + real_off<N>(si.kk[c], si.jj[b]);
                    if (g.fluid[node]) count_fl += 1;
                    else for (int n = 0; n < 3; ++n) lsol[n] += lfr[n * CR + node];
                }
        const int count_so = 8 - count_fl;
        double lft[3] = {0, 0, 0};
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const size_t node = (size_t)si.ii[a] * RSP + real_off<N>(si.kk[c], si.jj[b]);
                    const bool isfl = g.fluid[node] != 0;
                    const double w = si.w(a, b, c);
                    double lw = 0.0;
#pragma unroll
                    for (int n = 0; n < 3; ++n) {
                        double gg = as->lfrmean[n] * rnc;
                        if (g.include_frmeanfluid || !isfl) gg += lfr[n * CR + node];   // INCLUDE_FRMEANFLUID: every corner keeps its share
                        else if (count_so > 0) gg += lsol[n] / (double)count_so;
                        lft[n] += w / g.dx3 * gg;
                        lw += ft[n] / g.dx3 * gg;
                    }
                    double dw[3];
                    sten_dw(si, a, b, c, dw);
#pragma unroll
                    for (int d = 0; d < 3; ++d) gpos[d] += dw[d] * lw;
                }
        // direct forcing^T: ft = sfac (cf (uli - ucar(ulo)) + qll + c12 ppll)
        const double cf = sc->cf, c12 = g.c1 + g.c2;
        double sn_l = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) sn_l += snorm[d] * lft[d];
        double wsum = 0.0;
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int a = 0; a < 2; ++a) wsum += spi.w(a, b, c);
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const double gq = lft[n] * sfac;
            const double lulo = -cf * sfac * (kap * (lft[n] - snorm[n] * sn_l) + kapn * snorm[n] * sn_l);
            const double luli = cf * gq, lppll = c12 * gq;
            gm[n] = lppll * wsum;
            spread_adj<N>(so, ubcp + n * CR, 0.0, lubcp + n * CR, lulo, gpos);
            spread_adj<N>(si, ubcp + n * CR, 0.0, lubcp + n * CR, luli, gpos);
            spread_adj<N>(si, Q + n * CR, 0.0, lQ + n * CR, gq, gpos);
            spread_adj<N>(spi, pgr + n * CR, sc->mpg[n], lpgr + n * CR, lppll, gpos);
        }
    }
    add_gxc(gxc, NB, m, gpos);
    for (int n = 0; n < 3; ++n) {
        const double a = block_sum(gm[n], scr);
        if (threadIdx.x == 0) atomicAdd(&as->gmpg[n], a);
    }
}

// ============================================================================
// k_adj_drag: the objective's share of step n, calc_pres_visc_drag^T
// (boundary_condition.F90:1481-1645): pres_m = -sum p(xl - 0.5 ex) cd da1,
// visc_m = vis da1 sum omega(xl) x cd; lambda pbcp, lambda omega and dJ/dxc.
// ============================================================================
template <int N>
__global__ void __launch_bounds__(256) k_adj_drag(Geo g, const double *__restrict__ pbcp, const double *__restrict__ omega,
                                                  double *lpbcp, double *lomega, double *gxc, double e0, double e1, double e2,
                                                  double wJ) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int NB = g.nbody;
    const size_t CR = (size_t)g.nx * RP<N>::RSP;
    double gpos[3] = {0, 0, 0};
    int m = -1;
    if (t < NB * g.nbnd) {
        m = t / g.nbnd;
        const int l = t - m * g.nbnd;
        double xl[3], xpb[3], cdl[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) { xl[d] = __dadd_rn(g.xc[m + d * NB], __dmul_rn(g.bnd[3 * l + d], g.rb)); cdl[d] = g.cd[3 * l + d]; }
        xpb[0] = __dsub_rn(xl[0], 0.5); xpb[1] = xl[1]; xpb[2] = xl[2];
        Sten sp, sv;
        make_sten(g, xpb, sp);
        make_sten(g, xl, sv);
        const double lpl = -wJ * g.da1 * ((e0 * cdl[0] + e1 * cdl[1]) + e2 * cdl[2]);
        const double cxe[3] = {cdl[1] * e2 - cdl[2] * e1, cdl[2] * e0 - cdl[0] * e2, cdl[0] * e1 - cdl[1] * e0};
        spread_adj<N>(sp, pbcp, 0.0, lpbcp, lpl, gpos);
#pragma unroll
        for (int n = 0; n < 3; ++n) spread_adj<N>(sv, omega + n * CR, 0.0, lomega + n * CR, wJ * g.vis * g.da1 * cxe[n], gpos);
    }
    add_gxc(gxc, NB, m, gpos);
}

// k_adj_q: Q = c2r(q), q_c = -c3 nl_new_c - c4 onl_c - c12 vis (d2x u_c / dx2 - w2 u_c)
// (k_nl, calc_visc boundary_condition.F90:1767-1815).  T = c2r^T(lambda Q).
__global__ void __launch_bounds__(256) k_adj_q(Geo g, const double2 *__restrict__ T, double2 *lnl_new, double2 *lonl, double2 *lu2) {
    const size_t PS = g.PS, nx = g.nx;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * nx * PS) return;
    const size_t q = t % PS, i = (t / PS) % nx, n = t / (PS * nx);
    const size_t im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
    const double2 v = T[t], vm = T[(n * nx + im) * PS + q], vp = T[(n * nx + ip) * PS + q];
    const double c12 = g.c1 + g.c2, w2 = g.w2[q];
    lnl_new[t] = axpy2(-g.c3, v, lnl_new[t]);
    lonl[t] = axpy2(-g.c4, v, lonl[t]);
    const double2 lap = make_double2(g.rdx2 * ((vm.x - 2.0 * v.x) + vp.x) - w2 * v.x, g.rdx2 * ((vm.y - 2.0 * v.y) + vp.y) - w2 * v.y);
    lu2[t] = axpy2(-c12 * g.vis, lap, lu2[t]);
}

// MUSCL slope of the forward flux (slope_lim) and its partials
// d s / d (u(i-1), u(i), u(i+1)).
// tdx = 2 dx with its reciprocal rtdx (qdiv).
__device__ __forceinline__ double slope_d(double um1, double u0, double up1, double tdx, double rtdx, int limiter, double ds[3]) {
    const double S = qdiv(up1 - um1, tdx, rtdx);
    double phi = 1.0, d0 = 0.0, d1 = 0.0, d2 = 0.0;
    if (limiter == PIBM_LIMITER_MINMOD) {
        const double num = u0 - um1, den = up1 - u0 + kSmallD;
        const double r = num / den;
        if (r <= 0.0) phi = 0.0;
        else if (r < 1.0) {
            phi = r;
            d0 = -1.0 / den;
            d1 = 1.0 / den + num / (den * den);
            d2 = -num / (den * den);
        }
    }
    ds[0] = qdiv(-phi, tdx, rtdx) + S * d0;
    ds[1] = S * d1;
    ds[2] = qdiv(phi, tdx, rtdx) + S * d2;
    return S * phi;
}

// ============================================================================
// k_adj_flux: products and x flux of the nonlinear term, transposed, into
// lambda ubcp (nl_allflow.F90:97-310 transposed).  W8 items 0..4 = lambda of
// the products u0u1, u0u2, u1u1, u1u2, u2u2; items 5..7 = lambda of the
// x-flux differences D_c.  Upwind: D_c(i) = (F(i) - F(i-1))/dx with F(m) the
// Rusanov flux at the face between cells m and m+1,
// F = (a A + b B - max(|a|,|b|) (B - A)) / 2, a, b the MUSCL states of u0 and
// A, B those of u_c; face m reads cells m-1 .. m+2.  One thread owns one
// (y,z) node and a segment of SEG cells and streams along x like k_flux:
// each face's partials are formed once and added to a rolling window of the
// four cells it reads; a cell is complete once the face after it is done.
// ============================================================================
constexpr int kAdjFluxSeg = 16;   // x cells per thread (divides every supported nx)
template <int N>
__global__ void __launch_bounds__(256) k_adj_flux(Geo g, const double *__restrict__ ubcp, const double *__restrict__ W8,
                                                  double *lubcp) {
    constexpr int RSP = RP<N>::RSP, SEG = kAdjFluxSeg;
    const int nx = g.nx, nseg = nx / SEG;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= RSP * nseg) return;
    const int e = t % RSP, i0 = (t / RSP) * SEG;
    if (e % (N + 2) >= N) return;
    const size_t CR = (size_t)nx * RSP;
    auto X = [&](int ii) { return ii < 0 ? ii + nx : (ii >= nx ? ii - nx : ii); };
    auto U = [&](int c, int ii) { return __ldg(ubcp + c * CR + (size_t)X(ii) * RSP + e); };
    auto LD = [&](int c, int ii) { return __ldg(W8 + (5 + c) * CR + (size_t)X(ii) * RSP + e); };
    const double dx = g.dx, h = dx / 2.0;
    const double tdx = 2.0 * dx, rtdx = 1.0 / tdx, rdx = 1.0 / dx;   // divisors and reciprocals for qdiv
    // pointwise part: the products, and the whole center-scheme flux
    auto pointwise = [&](int i, double lu[3]) {
        const size_t o = (size_t)i * RSP + e;
        const double u0 = U(0, i), u1 = U(1, i), u2 = U(2, i);
        const double P01 = W8[0 * CR + o], P02 = W8[1 * CR + o], P11 = W8[2 * CR + o], P12 = W8[3 * CR + o], P22 = W8[4 * CR + o];
        lu[0] = u1 * P01 + u2 * P02;
        lu[1] = (u0 * P01 + 2.0 * u1 * P11) + u2 * P12;
        lu[2] = (u0 * P02 + u1 * P12) + 2.0 * u2 * P22;
        if (g.scheme == PIBM_SCHEME_CENTER) {
            const double uc[3] = {u0, u1, u2};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double lf = qdiv(LD(c, i - 1) - LD(c, i + 1), tdx, rtdx);
                lu[0] += uc[c] * lf;
                lu[c] += u0 * lf;
            }
        }
    };
    if (g.scheme == PIBM_SCHEME_CENTER) {
        for (int i = i0; i < i0 + SEG; ++i) {
            double lu[3];
            pointwise(i, lu);
#pragma unroll
            for (int c = 0; c < 3; ++c) lubcp[c * CR + (size_t)i * RSP + e] += lu[c];
        }
        return;
    }
    const int lim = g.limiter;
    // window at face m: w[c][k] = u_c(m-1+k); sl/ds: slopes at cells m, m+1;
    // ld: lambda D at m, m+1; acc[c][k]: lambda u_c(m-1+k)
    double w[3][4], sl[3][2], ds[3][2][3], ld[3][2], acc[3][4];
    int m = i0 - 2;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int k = 0; k < 4; ++k) { w[c][k] = U(c, m - 1 + k); acc[c][k] = 0.0; }
        sl[c][0] = slope_d(w[c][0], w[c][1], w[c][2], tdx, rtdx, lim, ds[c][0]);
        sl[c][1] = slope_d(w[c][1], w[c][2], w[c][3], tdx, rtdx, lim, ds[c][1]);
        ld[c][0] = LD(c, m);
        ld[c][1] = LD(c, m + 1);
    }
    for (; m <= i0 + SEG; ++m) {
        const double a = w[0][1] + sl[0][0] * h, b = w[0][2] - sl[0][1] * h;
        const double M = fmax(fabs(a), fabs(b));
        const bool amax = !(fabs(a) < fabs(b));
        const double sa = a > 0.0 ? 1.0 : (a < 0.0 ? -1.0 : 0.0), sb = b > 0.0 ? 1.0 : (b < 0.0 ? -1.0 : 0.0);
        double la = 0.0, lb = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double lF = qdiv(ld[c][0] - ld[c][1], dx, rdx);
            const double A = w[c][1] + sl[c][0] * h, B = w[c][2] - sl[c][1] * h;
            const double pa = (0.5 * A - 0.5 * (B - A) * (amax ? sa : 0.0)) * lF;
            const double pb = (0.5 * B - 0.5 * (B - A) * (amax ? 0.0 : sb)) * lF;
            const double pA = (0.5 * a + 0.5 * M) * lF, pB = (0.5 * b - 0.5 * M) * lF;
            la += pa;
            lb += pb;
            // A = u_c(m) + h s_c(m), B = u_c(m+1) - h s_c(m+1)
            acc[c][1] += pA;
            acc[c][2] += pB;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                acc[c][q] += h * pA * ds[c][0][q];
                acc[c][q + 1] -= h * pB * ds[c][1][q];
            }
        }
        acc[0][1] += la;
        acc[0][2] += lb;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            acc[0][q] += h * la * ds[0][0][q];
            acc[0][q + 1] -= h * lb * ds[0][1][q];
        }
        // cell m-1 is complete
        const int ic = m - 1;
        if (ic >= i0 && ic < i0 + SEG) {
            double lu[3];
            pointwise(ic, lu);
#pragma unroll
            for (int c = 0; c < 3; ++c) lubcp[c * CR + (size_t)ic * RSP + e] += lu[c] + acc[c][0];
        }
        if (m == i0 + SEG) break;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            acc[c][0] = acc[c][1]; acc[c][1] = acc[c][2]; acc[c][2] = acc[c][3]; acc[c][3] = 0.0;
            w[c][0] = w[c][1]; w[c][1] = w[c][2]; w[c][2] = w[c][3]; w[c][3] = U(c, m + 3);
            sl[c][0] = sl[c][1];
            ds[c][0][0] = ds[c][1][0]; ds[c][0][1] = ds[c][1][1]; ds[c][0][2] = ds[c][1][2];
            sl[c][1] = slope_d(w[c][1], w[c][2], w[c][3], tdx, rtdx, lim, ds[c][1]);
            ld[c][0] = ld[c][1];
            ld[c][1] = LD(c, m + 2);
        }
    }
}

// k_adj_assemble: lambda u_{n-1}, p_{n-1} from T = c2r^T of lambda ubcp (0..2),
// omega (3..5), pbcp (6), pgr (7..9) (k_a0's ten transforms transposed):
// omega = (wy u2 - wz u1, wz u0 - dx u2, dx u1 - wy u0), pgr = (dx p, wy p, wz p),
// dx the central difference (f(i+1) - f(i-1)) / (2 dx).
__global__ void __launch_bounds__(256) k_adj_assemble(Geo g, const double2 *__restrict__ T, double2 *lu2, double2 *lp2) {
    const size_t PS = g.PS, nx = g.nx, SC = nx * PS;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= SC) return;
    const size_t q = t % PS, i = t / PS;
    const size_t im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
    const double ky = g.ky[q % g.my2], kz = g.kz[q / g.my2], tdx = 2.0 * g.dx, rtdx = 1.0 / tdx;
    auto C = [&](int c, size_t ii) { return T[c * SC + ii * PS + q]; };
    const double2 o0 = C(3, i), o1 = C(4, i), o2 = C(5, i);
    const double2 o1m = C(4, im), o1p = C(4, ip), o2m = C(5, im), o2p = C(5, ip);
    double2 a0 = cadd(C(0, i), cadd(mul_cis(o1, kz), mul_is(o2, ky)));
    double2 a1 = cadd(C(1, i), cadd(mul_is(o0, kz), make_double2(qdiv(o2m.x - o2p.x, tdx, rtdx), qdiv(o2m.y - o2p.y, tdx, rtdx))));
    double2 a2 = cadd(C(2, i), csub(mul_cis(o0, ky), make_double2(qdiv(o1m.x - o1p.x, tdx, rtdx), qdiv(o1m.y - o1p.y, tdx, rtdx))));
    lu2[t] = cadd(lu2[t], a0);
    lu2[SC + t] = cadd(lu2[SC + t], a1);
    lu2[2 * SC + t] = cadd(lu2[2 * SC + t], a2);
    const double2 gm = C(7, im), gp = C(7, ip);
    double2 pp = cadd(C(6, i), make_double2(qdiv(gm.x - gp.x, tdx, rtdx), qdiv(gm.y - gp.y, tdx, rtdx)));
    pp = cadd(pp, cadd(mul_cis(C(8, i), ky), mul_cis(C(9, i), kz)));
    lp2[t] = cadd(lp2[t], pp);
}

// ============================================================================
// Launch sequence of one reverse step (the order of the header comment).
// ============================================================================
template <int N>
static void enqueue_adjoint_step_t(const Geo &g, const DevBufs &b, const AdjBufs &a, const double e[3], double wJ, cudaStream_t s) {
    constexpr int LT = N >= 256 ? 4 : 8;
    const size_t CR = (size_t)g.nx * RP<N>::RSP, SC = (size_t)g.nx * g.PS;
    double *lfrmean = (double *)((char *)a.as + offsetof(AdjScal, lfrmean));
    double *lumean = (double *)((char *)a.as + offsetof(AdjScal, lumean));
    const int nsum = 2 * 148;
    k_adj_begin<<<1, 32, 0, s>>>(b.sc, a.as);
    k_adj_lines<N, LT><<<(g.PS + LT - 1) / LT, LT * 32, adj_lines_smem<N>(), s>>>(g, a.lu, a.lp, a.lnl, a.lu2, a.lp2, a.lnl_new,
                                                                                 a.lonl, a.lff, b.sc, a.as);
    launch_planes<N>(k_adj_c2r<N>, g.nx, 3, s, g, (const double2 *)a.lff, a.lfr, 0);
    k_adj_sum<N><<<dim3(nsum, 3), 256, 0, s>>>(g, a.lfr, lfrmean, -1.0);
    cudaMemsetAsync(a.lubcp, 0, 10 * CR * sizeof(double), s);   // lubcp, lomega, lpbcp, lpgr
    cudaMemsetAsync(a.lQ, 0, 3 * CR * sizeof(double), s);
    if (g.npts > 0)
        k_adj_rev<N><<<(g.npts + 255) / 256, 256, 0, s>>>(g, b.ubcp, b.pgr, b.Q, b.rec, a.lfr, b.sc, a.as, a.lubcp, a.lQ, a.lpgr, a.gxc);
    if (wJ != 0.0)   // RK3: only the step's last stage carries the objective
        k_adj_drag<N><<<(g.nbody * g.nbnd + 255) / 256, 256, 0, s>>>(g, b.pbcp, b.omega, a.lpbcp, a.lomega, a.gxc, e[0], e[1], e[2], wJ);
    launch_planes<N>(k_adj_r2c<N>, 3 * g.nx, 1, s, g, (const double *)a.lQ, a.T, a.as);
    k_adj_q<<<(unsigned)((3 * SC + 255) / 256), 256, 0, s>>>(g, a.T, a.lnl_new, a.lonl, a.lu2);
    launch_planes<N>(k_adj_c2r<N>, g.nx, 8, s, g, (const double2 *)a.lnl_new, a.W8, 1);
    k_adj_flux<N><<<(unsigned)((RP<N>::RSP * (g.nx / kAdjFluxSeg) + 255) / 256), 256, 0, s>>>(g, b.ubcp, a.W8, a.lubcp);
    k_adj_sum<N><<<dim3(nsum, 3), 256, 0, s>>>(g, a.lubcp, lumean, 1.0);
    launch_planes<N>(k_adj_r2c<N>, 10 * g.nx, 1, s, g, (const double *)a.lubcp, a.T, a.as);
    k_adj_assemble<<<(unsigned)((SC + 255) / 256), 256, 0, s>>>(g, a.T, a.lu2, a.lp2);
}

void enqueue_adjoint_step(const Geo &g, const DevBufs &b, const AdjBufs &a, const double e[3], double wJ, cudaStream_t s) {
    switch (g.my) {
        case 32: enqueue_adjoint_step_t<32>(g, b, a, e, wJ, s); break;
        case 64: enqueue_adjoint_step_t<64>(g, b, a, e, wJ, s); break;
        case 96: enqueue_adjoint_step_t<96>(g, b, a, e, wJ, s); break;
        case 128: enqueue_adjoint_step_t<128>(g, b, a, e, wJ, s); break;
        case 256: enqueue_adjoint_step_t<256>(g, b, a, e, wJ, s); break;
    }
}
int adjoint_kernels_per_step(const Geo &g) { return 13 + (g.npts > 0 ? 1 : 0); }

void enqueue_adjoint_jacc(const Scal *sc, AdjScal *as, const double e[3], cudaStream_t s) {
    k_adj_jacc<<<1, 32, 0, s>>>(sc, as, e[0], e[1], e[2]);
}

template <int N>
static cudaError_t set_adj_attrs() {
    const int maxs = (int)plane_smem<N>();
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_adj_c2r<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_adj_r2c<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs)) != cudaSuccess) return e;
    constexpr int LT = N >= 256 ? 4 : 8;
    return cudaFuncSetAttribute(k_adj_lines<N, LT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)adj_lines_smem<N>());
}
cudaError_t configure_adjoint_kernels(int n) {
    switch (n) {
        case 32: return set_adj_attrs<32>();
        case 64: return set_adj_attrs<64>();
        case 96: return set_adj_attrs<96>();
        case 128: return set_adj_attrs<128>();
        case 256: return set_adj_attrs<256>();
    }
    return cudaErrorInvalidValue;
}

}  // namespace pibm
