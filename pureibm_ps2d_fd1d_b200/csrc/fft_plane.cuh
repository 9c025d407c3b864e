// fft_plane.cuh -- FP64 2-D plane transforms for one y-z plane held in shared
// memory, with the conventions of the reference's ff2rc / ff2cr
// (SRC/FLO/fftw_interface.F90:48-133):
//   r2c: real (my,mz) -> complex (my2,mz), y halved, e^{-i}, scaled 1/(my*mz)
//   c2r: complex (my2,mz) -> real (my,mz), e^{+i}, unscaled; after the z pass
//        the imaginary parts of the ky=0 and ky=my/2 columns are ignored.
//
// Shared-memory plane layout: row k (z index) holds my2 complex slots; a real
// row of my doubles occupies the first my/2 complex slots of the same row, so
// a plane is transformed in place without a second buffer.
//
// Every 1-D transform is done by a group of L lanes (L = 32, or 16 for 48-
// point transforms) holding R = N/L elements each in registers:
//   N = R*L,  x[l + L*r]  ->  R-point DFT in-lane -> twiddle w_N^{l*k1}
//   -> L-point DIF across lanes with shfl_xor -> lane l holds X[k1 + R*bitrev(l)].
// Twiddles w_N^m come from tables computed on the host in extended precision.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pibm {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by s*i (s = +1 or -1)
__device__ __forceinline__ double2 cmuli(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }

__device__ __forceinline__ double2 shfl_xor2(double2 v, int m, int width) {
    v.x = __shfl_xor_sync(0xffffffffu, v.x, m, width);
    v.y = __shfl_xor_sync(0xffffffffu, v.y, m, width);
    return v;
}

template <int L> __device__ __forceinline__ int bitrev(int l) {
    int r = 0;
#pragma unroll
    for (int b = 1; b < L; b <<= 1) { r = (r << 1) | (l & 1); l >>= 1; }
    return r;
}

// Twiddle lookup: w_N^m with sign s (table holds e^{-2 pi i m / N}; s>0 takes the conjugate).
// st holds the twiddles of the cross-lane stages contiguously, st[h-1+q] =
// w_{2h}^q (h = 1, 2, ..., L/2): lanes of one stage read consecutive entries,
// so the reads are free of shared-memory bank conflicts.
struct Tw {
    const double2 *t;   // table of e^{-2 pi i m/(N*stride)}
    int N;              // transform length this view describes
    int stride;         // table step: w_N^m = t[m*stride]
    const double2 *st;  // stage table (see above)
    __device__ __forceinline__ double2 get(int m, double s) const {
        double2 w = t[m * stride];
        return s > 0 ? make_double2(w.x, -w.y) : w;
    }
    __device__ __forceinline__ double2 stage(int h, int q, double s) const {
        double2 w = st[h - 1 + q];
        return s > 0 ? make_double2(w.x, -w.y) : w;
    }
};
// Fill a stage table for L lanes from a table of N = L*R entries (block-wide, caller syncs).
template <int L>
__device__ __forceinline__ void fill_stage_table(double2 *st, const double2 *t, int N) {
    for (int e = threadIdx.x; e < L - 1; e += blockDim.x) {
        int h = 1;
        while (h - 1 + h <= e) h <<= 1;   // e in [h-1, 2h-1)
        const int q = e - (h - 1);
        st[e] = t[q * (N / (2 * h))];
    }
}

// In-lane R-point DFT (sign s) of v[0..R-1].
template <int R> __device__ __forceinline__ void dft_inlane(double2 (&v)[R], double s, const Tw &tw);

template <> __device__ __forceinline__ void dft_inlane<1>(double2 (&v)[1], double, const Tw &) {}
template <> __device__ __forceinline__ void dft_inlane<2>(double2 (&v)[2], double, const Tw &) {
    double2 a = v[0], b = v[1];
    v[0] = cadd(a, b); v[1] = csub(a, b);
}
template <> __device__ __forceinline__ void dft_inlane<3>(double2 (&v)[3], double s, const Tw &tw) {
    // w3 = e^{s 2 pi i/3} = (-1/2, s*sqrt(3)/2); take sqrt(3)/2 from the table
    const double h = -tw.get(tw.N / 3, -1.0).y;   // e^{-2 pi i/3}: -imag = +sin(2pi/3)
    double2 a0 = v[0], a1 = v[1], a2 = v[2];
    double2 t1 = cadd(a1, a2), t2 = csub(a1, a2);
    double2 c = make_double2(a0.x - 0.5 * t1.x, a0.y - 0.5 * t1.y);
    double2 jt2 = cmuli(t2, s * h);
    v[0] = cadd(a0, t1); v[1] = cadd(c, jt2); v[2] = csub(c, jt2);
}
template <> __device__ __forceinline__ void dft_inlane<4>(double2 (&v)[4], double s, const Tw &) {
    double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]), t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
    double2 jt3 = cmuli(t3, s);
    v[0] = cadd(t0, t2); v[1] = cadd(t1, jt3); v[2] = csub(t0, t2); v[3] = csub(t1, jt3);
}
template <> __device__ __forceinline__ void dft_inlane<8>(double2 (&v)[8], double s, const Tw &tw) {
    // radix-2 DIF first stage, then two radix-4 on even/odd outputs
    const double2 w8 = tw.get(tw.N / 8, s);
    double2 a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) { a[r] = cadd(v[r], v[r + 4]); b[r] = csub(v[r], v[r + 4]); }
    b[1] = cmul(b[1], w8);
    b[2] = cmuli(b[2], s);
    b[3] = cmul(cmuli(b[3], s), w8);
    dft_inlane<4>(a, s, tw);
    dft_inlane<4>(b, s, tw);
#pragma unroll
    for (int r = 0; r < 4; ++r) { v[2 * r] = a[r]; v[2 * r + 1] = b[r]; }
}

// One N = R*L point transform held by a lane group.  On entry v[r] = x[l + L*r];
// on exit v[r] = X[r + R*bitrev(l)].  tw must describe N (tw.N == N).
template <int R, int L>
__device__ __forceinline__ void group_fft(double2 (&v)[R], int l, double s, const Tw &tw) {
    constexpr int N = R * L;
    dft_inlane<R>(v, s, tw);
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw.get((l * r) % N, s));
    // each stage in one form for both lanes of a pair: the upper lane forms
    // v + pv, the lower (pv - v) w, i.e. t = pv + sgn v, then t w' (w' = 1 on
    // the upper lane)
#pragma unroll
    for (int h = L / 2; h >= 1; h >>= 1) {
        const bool upper = (l & h) == 0;
        const double sgn = upper ? 1.0 : -1.0;
        const double2 w = (upper || h == 1) ? make_double2(1.0, 0.0) : tw.stage(h, l & (h - 1), s);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double2 pv = shfl_xor2(v[r], h, L);
            const double2 t = make_double2(__fma_rn(sgn, v[r].x, pv.x), __fma_rn(sgn, v[r].y, pv.y));
            v[r] = h == 1 ? t : cmul(t, w);   // the last stage's twiddle is 1
        }
    }
}

}  // namespace pibm
