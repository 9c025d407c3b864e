// line_solve.cuh -- per-warp solves of the x-line systems of velstep.
//
// Every cyclic system of velstep has constant coefficients (a = c, b on every
// row, periodic coupling), i.e. it is a symmetric circulant matrix; the
// reference solves it with Thomas + Sherman-Morrison (tridiagonal.F90:90-150,
// usteptime.F90:344-349,457-468).  Here one warp solves one line exactly
// through its eigen-decomposition; the (ky,kz) = (0,0) pressure line is not
// circulant and keeps the reference's Thomas recursion.  Both matrices are
// symmetric, so the same solves serve the adjoint step.
#pragma once
#include "step_common.cuh"

namespace pibm {

// Per-lane constants of circulant_solve<R>, laid out [r][lane] so that a warp
// reads 32 consecutive entries (the table lookups they replace stride by
// R*bitrev(lane) and by r*lane, which alias shared-memory banks):
//   cs[r*32 + l]       = cos(2 pi m/N), m = r + R*bitrev(l)   (eigenvalue of mode m)
//   tr[(r-1)*32 + l]   = e^{-2 pi i (l r mod N)/N}, r = 1..R-1  (inter-stage twiddle)
// The entries are copies of the twiddle table's, so the solve's arithmetic is
// unchanged.
template <int R> struct LineTw {
    Tw tw;
    const double *cs;
    const double2 *tr;
};
template <int R> __host__ __device__ constexpr size_t line_tw_bytes() {
    return (size_t)R * 32 * sizeof(double) + (size_t)(R - 1) * 32 * sizeof(double2);
}
// Fill cs and tr from the global twiddle table t (e^{-2 pi i m/N}, m < N); block-wide, caller syncs.
template <int R> __device__ __forceinline__ void fill_line_tw(double *cs, double2 *tr, const double2 *t) {
    constexpr int N = R * 32;
    for (int e = threadIdx.x; e < R * 32; e += blockDim.x) {
        const int r = e / 32, l = e % 32;
        cs[e] = t[r + R * bitrev<32>(l)].x;
        if (r > 0) tr[e - 32] = t[(l * r) % N];
    }
}

// The solve on values held in registers: on entry v[r] = x[lane + 32 r], on
// exit the solution at the same places.
template <int R>
__device__ __forceinline__ void circulant_solve_reg(double2 (&v)[R], double a, double b, const LineTw<R> &lt, int lane) {
    constexpr int N = R * 32;
    const Tw &tw = lt.tw;
    // forward transform: group_fft<R, 32> with sign -1, its twiddles from the per-lane table
    dft_inlane<R>(v, -1.0, tw);
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], lt.tr[(r - 1) * 32 + lane]);
    // Each butterfly stage in one form for both lanes of a pair (no select of
    // two computed branches): the upper lane forms v + pv, the lower (pv - v) w,
    // i.e. t = pv + sgn v, then t times w' with w' = 1 on the upper lane.  The
    // last stage's twiddle is 1 on every lane: no multiply.
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
        const bool upper = (lane & h) == 0;
        const double sgn = upper ? 1.0 : -1.0;
        const double2 w = (upper || h == 1) ? make_double2(1.0, 0.0) : tw.stage(h, lane & (h - 1), -1.0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double2 pv = shfl_xor2(v[r], h, 32);
            const double2 t = make_double2(__fma_rn(sgn, v[r].x, pv.x), __fma_rn(sgn, v[r].y, pv.y));
            v[r] = h == 1 ? t : cmul(t, w);
        }
    }
    // lane holds modes m = r + R*bitrev(lane)
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const double lam = ((double)N) * (b + 2.0 * a * lt.cs[r * 32 + lane]), rlam = 1.0 / lam;
        v[r] = make_double2(qdiv(v[r].x, lam, rlam), qdiv(v[r].y, lam, rlam));
    }
    // exact inverse of the forward stages (unnormalised; 1/N folded into lam)
    // Inverse stages: the lower lane of a pair first multiplies its own value by
    // conj w (the upper by 1), then both take pv + sgn v: upper u + l conj w,
    // lower u - l conj w.
#pragma unroll
    for (int h = 1; h < 32; h <<= 1) {
        const bool upper = (lane & h) == 0;
        const double sgn = upper ? 1.0 : -1.0;
        const double2 w = (upper || h == 1) ? make_double2(1.0, 0.0) : tw.stage(h, lane & (h - 1), +1.0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double2 m = h == 1 ? v[r] : cmul(v[r], w);
            const double2 pv = shfl_xor2(m, h, 32);
            v[r] = make_double2(__fma_rn(sgn, m.x, pv.x), __fma_rn(sgn, m.y, pv.y));
        }
    }
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], cconj(lt.tr[(r - 1) * 32 + lane]));
    dft_inlane<R>(v, +1.0, tw);
}
// The solve on row[0..N-1] in shared memory (one warp, in place).
template <int R>
__device__ __forceinline__ void circulant_solve(double2 *row, double a, double b, const LineTw<R> &lt, int lane) {
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = row[lane + 32 * r];
    circulant_solve_reg<R>(v, a, b, lt, lane);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; ++r) row[lane + 32 * r] = v[r];
    __syncwarp();
}

// Pressure-source and explicit ustep terms of the x-line kernels with every
// rounding written out (no multiply-add contraction), so that a kernel which
// accumulates them one input field at a time forms bitwise the values of one
// that has every field at hand.
__device__ __forceinline__ double2 cadd_rn(double2 a, double2 b) { return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y)); }
__device__ __forceinline__ double2 cscale_rn(double2 a, double c) { return make_double2(__dmul_rn(c, a.x), __dmul_rn(c, a.y)); }
// Term of component n of one field (coefficient c when coef, none for ff) in
// the pressure source at plane i (poisson.F90:97-116): x0, x1 the field at
// planes i and i+1; n = 0: c (x1 - x0)/dx; n = 1, 2: c i k (x1 + x0)/2, k = ky, kz.
__device__ __forceinline__ double2 psrc_term_rt(int n, bool coef, double c, double2 x0, double2 x1, double ky, double kz, double dx,
                                                double rdx) {
    if (n == 0) {
        double2 d = make_double2(__dsub_rn(x1.x, x0.x), __dsub_rn(x1.y, x0.y));
        if (coef) d = cscale_rn(d, c);
        return make_double2(qdiv(d.x, dx, rdx), qdiv(d.y, dx, rdx));
    }
    const double k = n == 1 ? ky : kz;
    double2 d = make_double2(__dmul_rn(-k, __dadd_rn(x1.y, x0.y)), __dmul_rn(k, __dadd_rn(x1.x, x0.x)));
    if (coef) d = cscale_rn(d, c);
    return cscale_rn(d, 0.5);
}
template <bool kCoef>
__device__ __forceinline__ double2 psrc_term(int n, double c, double2 x0, double2 x1, double ky, double kz, double dx, double rdx) {
    return psrc_term_rt(n, kCoef, c, x0, x1, ky, kz, dx, rdx);
}
// Per-line coefficients of velstep's three systems and right-hand sides,
// every rounding written out (poisson.F90:118-161, usteptime.F90:73-300).
struct LineCoef {
    double pa, pb, pc;     // pressure and divcorr systems: a, b, c
    double ua, ub;         // ustep system: a (= c), b
    double fy, gd, alp;    // ustep right-hand side: 1 - dt vis c1 w2, dt vis c1, dt (c1 + c2)
    double c2dtv;          // divcorr pressure update: c2 dt vis
};
__device__ __forceinline__ LineCoef line_coef(double dt, double vis, double c1, double c2, double dx2, double w2) {
    LineCoef k;
    const double r1 = 1.0 / dx2, r2 = -2.0 / dx2, dtv = __dmul_rn(dt, vis);
    k.pa = __dsub_rn(r1, __dmul_rn(0.25, w2));
    k.pb = __dsub_rn(r2, __dmul_rn(0.5, w2));
    k.pc = k.pa;
    const double dvc2 = __dmul_rn(dtv, c2);
    k.ua = -(dvc2 / dx2);
    k.ub = __dadd_rn(1.0, __dmul_rn(dvc2, __dadd_rn(2.0 / dx2, w2)));
    k.gd = __dmul_rn(dtv, c1);
    k.fy = __dsub_rn(1.0, __dmul_rn(k.gd, w2));
    k.alp = __dmul_rn(dt, __dadd_rn(c1, c2));
    k.c2dtv = __dmul_rn(__dmul_rn(c2, dt), vis);
    return k;
}
// p + (phi - p): the pressure estimate of poisson.F90:163-175 with relaxation 1.
__device__ __forceinline__ double2 p_update(double2 po, double2 tp) {
    return make_double2(__dadd_rn(po.x, __dsub_rn(tp.x, po.x)), __dadd_rn(po.y, __dsub_rn(tp.y, po.y)));
}
// ustep right-hand side of component n at one plane (usteptime.F90:73-300):
// u fy + ex - alp grad_n p + gd lap(u)/dx^2, ex the explicit part, pm and p0
// the pressure at planes i-1 and i; the plane i = 0 forms the Laplacian as
// (u(i+1) - 2u) + u(i-1), the others as (u(i-1) + u(i+1)) - 2u.
__device__ __forceinline__ double2 ustep_rhs(int n, const LineCoef &k, double2 ui, double2 um, double2 up, double2 ex, double2 pm,
                                             double2 p0, bool i0, double ky, double kz, double dx, double rdx, double dx2,
                                             double rdx2) {
    double2 rv = make_double2(__dadd_rn(__dmul_rn(ui.x, k.fy), ex.x), __dadd_rn(__dmul_rn(ui.y, k.fy), ex.y));
    double2 gp;
    if (n == 0) {
        gp = make_double2(qdiv(__dmul_rn(k.alp, __dsub_rn(p0.x, pm.x)), dx, rdx), qdiv(__dmul_rn(k.alp, __dsub_rn(p0.y, pm.y)), dx, rdx));
    } else {
        const double ah = __dmul_rn(k.alp, 0.5), kk = n == 1 ? ky : kz;
        const double2 sp = make_double2(__dmul_rn(ah, __dadd_rn(pm.x, p0.x)), __dmul_rn(ah, __dadd_rn(pm.y, p0.y)));
        gp = make_double2(__dmul_rn(-kk, sp.y), __dmul_rn(kk, sp.x));
    }
    rv = make_double2(__dsub_rn(rv.x, gp.x), __dsub_rn(rv.y, gp.y));
    double2 lap;
    if (i0) lap = make_double2(__dadd_rn(__dsub_rn(up.x, __dmul_rn(2.0, ui.x)), um.x), __dadd_rn(__dsub_rn(up.y, __dmul_rn(2.0, ui.y)), um.y));
    else lap = make_double2(__dsub_rn(__dadd_rn(um.x, up.x), __dmul_rn(2.0, ui.x)), __dsub_rn(__dadd_rn(um.y, up.y), __dmul_rn(2.0, ui.y)));
    return make_double2(__dadd_rn(rv.x, qdiv(__dmul_rn(k.gd, lap.x), dx2, rdx2)), __dadd_rn(rv.y, qdiv(__dmul_rn(k.gd, lap.y), dx2, rdx2)));
}
// Divergence of u at plane i (poisson.F90:260-300, steptheflow.F90:219-240):
// (u1(i+1) - u1(i))/dx + i ky (u2(i) + u2(i+1))/2 + i kz (u3(i) + u3(i+1))/2.
__device__ __forceinline__ double2 div_term(double2 u1i, double2 u1p, double2 u2i, double2 u2p, double2 u3i, double2 u3p, double ky,
                                            double kz, double dx, double rdx) {
    double2 t = make_double2(qdiv(__dsub_rn(u1p.x, u1i.x), dx, rdx), qdiv(__dsub_rn(u1p.y, u1i.y), dx, rdx));
    const double2 sy = make_double2(__dmul_rn(__dadd_rn(u2i.x, u2p.x), 0.5), __dmul_rn(__dadd_rn(u2i.y, u2p.y), 0.5));
    const double2 sz = make_double2(__dmul_rn(__dadd_rn(u3i.x, u3p.x), 0.5), __dmul_rn(__dadd_rn(u3i.y, u3p.y), 0.5));
    t = make_double2(__dadd_rn(t.x, __dmul_rn(-ky, sy.y)), __dadd_rn(t.y, __dmul_rn(ky, sy.x)));
    return make_double2(__dadd_rn(t.x, __dmul_rn(-kz, sz.y)), __dadd_rn(t.y, __dmul_rn(kz, sz.x)));
}
__device__ __forceinline__ double cabs_rn(double2 t) { return __dsqrt_rn(__dadd_rn(__dmul_rn(t.x, t.x), __dmul_rn(t.y, t.y))); }
// divcorr's correction at plane i (poisson.F90:330-508): phi d0 at i, dm at
// i-1, dp at i+1; u -= alpc grad phi, p += phi - c2 dt vis lap(phi).
__device__ __forceinline__ void divcorr_update(const LineCoef &k, double2 d0, double2 dm, double2 dp, bool i0, double2 U1, double2 U2,
                                               double2 U3, double2 Pw, double ky, double kz, double w2, double dx, double rdx,
                                               double dx2, double rdx2, double2 &nu1, double2 &nu2, double2 &nu3, double2 &np) {
    const double alpc = k.alp;
    const double2 s = make_double2(__dadd_rn(dm.x, d0.x), __dadd_rn(dm.y, d0.y));
    double2 gy, gz;
    if (i0) {
        gy = make_double2(__dmul_rn(__dmul_rn(-ky, 0.0), 0.5), __dmul_rn(__dmul_rn(ky, alpc), 0.5));
        gz = make_double2(__dmul_rn(__dmul_rn(-kz, 0.0), 0.5), __dmul_rn(__dmul_rn(kz, alpc), 0.5));
    } else {
        const double ah = __dmul_rn(alpc, 0.5);
        gy = make_double2(__dmul_rn(-ky, 0.0), __dmul_rn(ky, ah));
        gz = make_double2(__dmul_rn(-kz, 0.0), __dmul_rn(kz, ah));
    }
    nu1 = make_double2(__dsub_rn(U1.x, qdiv(__dmul_rn(alpc, __dsub_rn(d0.x, dm.x)), dx, rdx)),
                       __dsub_rn(U1.y, qdiv(__dmul_rn(alpc, __dsub_rn(d0.y, dm.y)), dx, rdx)));
    nu2 = make_double2(__dsub_rn(U2.x, __dsub_rn(__dmul_rn(gy.x, s.x), __dmul_rn(gy.y, s.y))),
                       __dsub_rn(U2.y, __dadd_rn(__dmul_rn(gy.x, s.y), __dmul_rn(gy.y, s.x))));
    nu3 = make_double2(__dsub_rn(U3.x, __dsub_rn(__dmul_rn(gz.x, s.x), __dmul_rn(gz.y, s.y))),
                       __dsub_rn(U3.y, __dadd_rn(__dmul_rn(gz.x, s.y), __dmul_rn(gz.y, s.x))));
    const double2 lap = make_double2(__dsub_rn(qdiv(__dadd_rn(__dsub_rn(dm.x, __dmul_rn(2.0, d0.x)), dp.x), dx2, rdx2), __dmul_rn(w2, d0.x)),
                                     __dsub_rn(qdiv(__dadd_rn(__dsub_rn(dm.y, __dmul_rn(2.0, d0.y)), dp.y), dx2, rdx2), __dmul_rn(w2, d0.y)));
    np = make_double2(__dsub_rn(__dadd_rn(Pw.x, d0.x), __dmul_rn(k.c2dtv, lap.x)), __dsub_rn(__dadd_rn(Pw.y, d0.y), __dmul_rn(k.c2dtv, lap.y)));
}

// Thomas recursion (tridag, tridiagonal.F90:47-87) on the real parts of
// row[0..n-1]; constant a, b, c; result in row[].x, row[].y = 0, row[n] = 0.
__device__ __forceinline__ bool thomas_real(double2 *row, double *gam, double a, double b, double c, int n) {
    double bet = b;
    if (bet == 0.0) return false;
    double prev = row[0].x / bet;
    row[0] = make_double2(prev, 0.0);
    for (int j = 1; j < n; ++j) {
        gam[j] = c / bet;
        bet = b - a * gam[j];
        if (bet == 0.0) return false;
        prev = (row[j].x - a * prev) / bet;
        row[j] = make_double2(prev, 0.0);
    }
    for (int j = n - 2; j >= 0; --j) row[j].x = row[j].x - gam[j + 1] * row[j + 1].x;
    row[n] = make_double2(0.0, 0.0);
    return true;
}

}  // namespace pibm
