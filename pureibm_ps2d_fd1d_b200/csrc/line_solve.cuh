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

template <int R>
__device__ __forceinline__ void circulant_solve(double2 *row, double a, double b, const Tw &tw, int lane) {
    constexpr int N = R * 32;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = row[lane + 32 * r];
    group_fft<R, 32>(v, lane, -1.0, tw);
    const int br = bitrev<32>(lane);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int m = r + R * br;
        const double lam = ((double)N) * (b + 2.0 * a * tw.t[m * tw.stride].x);
        v[r] = make_double2(v[r].x / lam, v[r].y / lam);
    }
    // exact inverse of group_fft's stages (unnormalised; 1/N folded into lam)
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
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw.get((lane * r) % N, +1.0));
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
