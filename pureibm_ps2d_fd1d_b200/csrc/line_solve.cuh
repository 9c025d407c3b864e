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

template <int R>
__device__ __forceinline__ void circulant_solve(double2 *row, double a, double b, const LineTw<R> &lt, int lane) {
    constexpr int N = R * 32;
    const Tw &tw = lt.tw;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = row[lane + 32 * r];
    // forward transform: group_fft<R, 32> with sign -1, its twiddles from the per-lane table
    dft_inlane<R>(v, -1.0, tw);
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], lt.tr[(r - 1) * 32 + lane]);
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
        const bool upper = (lane & h) == 0;
        const int q = lane & (h - 1);
        const double2 w = tw.stage(h, q, -1.0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            double2 pv = shfl_xor2(v[r], h, 32);
            v[r] = upper ? cadd(v[r], pv) : cmul(csub(pv, v[r]), w);
        }
    }
    // lane holds modes m = r + R*bitrev(lane)
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const double lam = ((double)N) * (b + 2.0 * a * lt.cs[r * 32 + lane]), rlam = 1.0 / lam;
        v[r] = make_double2(qdiv(v[r].x, lam, rlam), qdiv(v[r].y, lam, rlam));
    }
    // exact inverse of the forward stages (unnormalised; 1/N folded into lam)
#pragma unroll
    for (int h = 1; h < 32; h <<= 1) {
        const bool upper = (lane & h) == 0;
        const int q = lane & (h - 1);
        const double2 w = tw.stage(h, q, +1.0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double2 pv = shfl_xor2(v[r], h, 32);
            v[r] = upper ? cadd(v[r], cmul(pv, w)) : csub(pv, cmul(v[r], w));
        }
    }
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], cconj(lt.tr[(r - 1) * 32 + lane]));
    dft_inlane<R>(v, +1.0, tw);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; ++r) row[lane + 32 * r] = v[r];
    __syncwarp();
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
