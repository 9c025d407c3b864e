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
struct Tw {
    const double2 *t;   // table of e^{-2 pi i m/(N*stride)}
    int N;              // transform length this view describes
    int stride;         // table step: w_N^m = t[m*stride]
    __device__ __forceinline__ double2 get(int m, double s) const {
        double2 w = t[m * stride];
        return s > 0 ? make_double2(w.x, -w.y) : w;
    }
};

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
#pragma unroll
    for (int h = L / 2; h >= 1; h >>= 1) {
        const bool upper = (l & h) == 0;
        const int q = l & (h - 1);
        const double2 w = tw.get(q * (N / (2 * h)), s);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            double2 pv = shfl_xor2(v[r], h, L);
            v[r] = upper ? cadd(v[r], pv) : cmul(csub(pv, v[r]), w);
        }
    }
}

// ---------------------------------------------------------------------------
// Plane transforms.  buf: mz rows x my2 complex slots (pitch my2).
// twz: table for N=mz; twy: table for N=my (the y half-length transform uses
// w_{my/2}^m = w_my^{2m}).  Called by all threads of the CTA; nwarps warps.
// ---------------------------------------------------------------------------
template <int RZ, int LZ>
__device__ __forceinline__ void z_pass(double2 *buf, int my2, int mz, double s, const Tw &twz) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    constexpr int G = 32 / LZ;       // columns per warp
    const int sub = lane / LZ, l = lane % LZ;
    for (int j0 = warp * G; j0 < my2; j0 += nwarps * G) {
        const int j = j0 + sub;
        const bool act = j < my2;
        double2 v[RZ];
#pragma unroll
        for (int r = 0; r < RZ; ++r) v[r] = act ? buf[(size_t)(l + LZ * r) * my2 + j] : make_double2(0.0, 0.0);
        group_fft<RZ, LZ>(v, l, s, twz);
        __syncwarp();
        const int br = bitrev<LZ>(l);
        if (act) {
#pragma unroll
            for (int r = 0; r < RZ; ++r) buf[(size_t)(r + RZ * br) * my2 + j] = v[r];
        }
        __syncwarp();
    }
}

// y direction complex-to-real on every row: X[0..M] (M = my/2) -> x[0..my-1]
// stored as complex pairs z[n] = x[2n] + i x[2n+1] in slots 0..M-1.
template <int RY, int LY>
__device__ __forceinline__ void y_c2r_pass(double2 *buf, int my2, int mz, const Tw &twy) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    constexpr int M = RY * LY;
    constexpr int G = 32 / LY;
    const int sub = lane / LY, l = lane % LY;
    for (int k0 = warp * G; k0 < mz; k0 += nwarps * G) {
        const int k = k0 + sub;
        const bool act = k < mz;
        double2 *row = buf + (size_t)(act ? k : 0) * my2;
        double2 v[RY];
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            const int n = l + LY * r;
            double2 xk = row[n], xm = row[M - n];
            if (n == 0) { xk.y = 0.0; xm.y = 0.0; }     // ignore Im of ky=0 and ky=M
            // Z[n] = (X[n] + conj X[M-n]) + i w+^n (X[n] - conj X[M-n]),  w+ = e^{+2 pi i/my}
            double2 e = make_double2(xk.x + xm.x, xk.y - xm.y);
            double2 d = make_double2(xk.x - xm.x, xk.y + xm.y);
            double2 od = cmul(d, twy.get(n, +1.0));
            v[r] = make_double2(e.x - od.y, e.y + od.x);
        }
        __syncwarp();
        group_fft<RY, LY>(v, l, +1.0, Tw{twy.t, M, 2 * twy.stride});   // w_M^m = w_my^{2m}
        const int br = bitrev<LY>(l);
        if (act) {
#pragma unroll
            for (int r = 0; r < RY; ++r) row[r + RY * br] = v[r];
        }
        __syncwarp();
    }
}

// y direction real-to-complex on every row: x (as pairs in slots 0..M-1) -> X[0..M].
template <int RY, int LY>
__device__ __forceinline__ void y_r2c_pass(double2 *buf, int my2, int mz, const Tw &twy) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    constexpr int M = RY * LY;
    constexpr int G = 32 / LY;
    const int sub = lane / LY, l = lane % LY;
    for (int k0 = warp * G; k0 < mz; k0 += nwarps * G) {
        const int k = k0 + sub;
        const bool act = k < mz;
        double2 *row = buf + (size_t)(act ? k : 0) * my2;
        double2 v[RY];
#pragma unroll
        for (int r = 0; r < RY; ++r) v[r] = row[l + LY * r];
        group_fft<RY, LY>(v, l, -1.0, Tw{twy.t, M, 2 * twy.stride});
        __syncwarp();
        const int br = bitrev<LY>(l);
        if (act) {
#pragma unroll
            for (int r = 0; r < RY; ++r) row[r + RY * br] = v[r];
        }
        __syncwarp();
        // post-process X[n] = (Z[n] + conj Z[M-n])/2 + w-^n (Z[n] - conj Z[M-n])/(2i), n = 0..M
        double2 out[RY];
        double2 nyq = make_double2(0.0, 0.0);
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            const int n = l + LY * r;
            double2 zk = row[n], zm = row[(M - n) % M];
            double2 e = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
            double2 o = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));   // (zk - conj zm)/(2i)
            double2 wo = cmul(twy.get(n, -1.0), o);
            out[r] = cadd(e, wo);
            if (n == 0) nyq = make_double2(zk.x - zk.y, 0.0);
        }
        __syncwarp();
        if (act) {
#pragma unroll
            for (int r = 0; r < RY; ++r) row[l + LY * r] = out[r];
            if (l == 0) row[M] = nyq;
        }
        __syncwarp();
    }
}

}  // namespace pibm
