// fft2d.cuh -- FP64 2-D plane transforms for one y-z plane held in shared
// memory, with the conventions of the reference's ff2rc / ff2cr
// (SRC/FLO/fftw_interface.F90:48-133):
//   r2c: real (my,mz) -> complex (my2,mz), y halved, e^{-i}, scaled 1/float(my*mz)
//   c2r: complex (my2,mz) -> real (my,mz), e^{+i}, unscaled; after the z pass
//        the imaginary parts of the ky=0 and ky=my/2 columns are ignored
//        (the real-to-complex reconstruction below forces them to zero).
//
// Layout: the plane is mz rows of `pitch` = my2 complex slots (pitch*16 B is
// 4 banks mod 32, so accesses that walk across rows or columns are
// conflict-free).  A real row of my values occupies the first my/2 slots as
// pairs (x[2m], x[2m+1]).
//
// 1-D transforms of length L = A*B are two in-place passes (four-step):
//   fft_v1: natural input; output slot B*k1+k2 holds X[k1 + A*k2]
//   fft_v2: input x[n1 + A*n2] at slot B*n1+n2; natural output
// Each thread owns whole A- or B-point sub-transforms in registers; the digit
// permutation perm(m) = B*(m % A) + m / A is absorbed into the loads/stores of
// the calling kernels, so no pass needs a second buffer.
// Twiddles come from one table of e^{-2 pi i m/N} (N = my = mz) computed on the
// host in extended precision.
#pragma once
#include <cuda_runtime.h>
#include "fft_plane.cuh"

namespace pibm {

// Twiddle view: w_L^m = e^{s 2 pi i m / L} read from a table of e^{-2 pi i m/N}.
struct TwT {
    const double2 *t;
    int N;
    __device__ __forceinline__ double2 w(int m, int L, double s) const {
        const double2 v = t[(m % L) * (N / L)];
        return s > 0 ? make_double2(v.x, -v.y) : v;
    }
};

template <int A, int B> __device__ __host__ __forceinline__ int perm_ab(int m) { return B * (m % A) + m / A; }

// ---------------------------------------------------------------------------
// In-register DFT of R points, natural order in and out.
// ---------------------------------------------------------------------------
template <int R> struct Dft;
template <> struct Dft<1> { __device__ __forceinline__ static void run(double2 *, double, const TwT &) {} };
template <> struct Dft<2> {
    __device__ __forceinline__ static void run(double2 *v, double, const TwT &) {
        const double2 a = v[0], b = v[1];
        v[0] = cadd(a, b); v[1] = csub(a, b);
    }
};
template <> struct Dft<3> {
    __device__ __forceinline__ static void run(double2 *v, double s, const TwT &tw) {
        const double h = -tw.w(1, 3, -1.0).y;   // sin(2 pi/3)
        const double2 a0 = v[0], t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
        const double2 c = make_double2(a0.x - 0.5 * t1.x, a0.y - 0.5 * t1.y);
        const double2 jt2 = cmuli(t2, s * h);
        v[0] = cadd(a0, t1); v[1] = cadd(c, jt2); v[2] = csub(c, jt2);
    }
};
template <> struct Dft<4> {
    __device__ __forceinline__ static void run(double2 *v, double s, const TwT &) {
        const double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]), t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
        const double2 jt3 = cmuli(t3, s);
        v[0] = cadd(t0, t2); v[1] = cadd(t1, jt3); v[2] = csub(t0, t2); v[3] = csub(t1, jt3);
    }
};
// composite R = P*Q by the same four-step in registers
template <int P, int Q> struct DftComp {
    __device__ __forceinline__ static void run(double2 *v, double s, const TwT &tw) {
        constexpr int R = P * Q;
        double2 t[R];
#pragma unroll
        for (int n2 = 0; n2 < Q; ++n2) {
            double2 a[P];
#pragma unroll
            for (int n1 = 0; n1 < P; ++n1) a[n1] = v[Q * n1 + n2];
            Dft<P>::run(a, s, tw);
#pragma unroll
            for (int k1 = 0; k1 < P; ++k1) t[Q * k1 + n2] = (n2 * k1 == 0) ? a[k1] : cmul(a[k1], tw.w(n2 * k1, R, s));
        }
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) {
            double2 b[Q];
#pragma unroll
            for (int n2 = 0; n2 < Q; ++n2) b[n2] = t[Q * k1 + n2];
            Dft<Q>::run(b, s, tw);
#pragma unroll
            for (int k2 = 0; k2 < Q; ++k2) v[k1 + P * k2] = b[k2];
        }
    }
};
template <> struct Dft<6> : DftComp<2, 3> {};
template <> struct Dft<8> : DftComp<4, 2> {};
template <> struct Dft<12> : DftComp<4, 3> {};
template <> struct Dft<16> : DftComp<4, 4> {};

// ---------------------------------------------------------------------------
// Passes over S sequences: element e of sequence s at buf[s*ss + e*es].
// Work units are distributed with the sequence index fastest so that
// consecutive threads touch consecutive rows/columns.  Ends with __syncthreads.
// ---------------------------------------------------------------------------
template <int A, int B>
__device__ __forceinline__ void fft_v1(double2 *buf, int S, int ss, int es, double s, const TwT &tw) {
    constexpr int L = A * B;
    const int T = blockDim.x;
    for (int u = threadIdx.x; u < S * B; u += T) {
        const int q = u % S, n2 = u / S;
        double2 *base = buf + (size_t)q * ss + n2 * es;
        double2 v[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) v[n1] = base[(size_t)(B * n1) * es];
        Dft<A>::run(v, s, tw);
#pragma unroll
        for (int k1 = 1; k1 < A; ++k1) v[k1] = cmul(v[k1], tw.w(n2 * k1, L, s));
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) base[(size_t)(B * k1) * es] = v[k1];
    }
    __syncthreads();
    for (int u = threadIdx.x; u < S * A; u += T) {
        const int q = u % S, k1 = u / S;
        double2 *base = buf + (size_t)q * ss + (size_t)(B * k1) * es;
        double2 v[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) v[n2] = base[(size_t)n2 * es];
        Dft<B>::run(v, s, tw);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) base[(size_t)k2 * es] = v[k2];
    }
    __syncthreads();
}

template <int A, int B>
__device__ __forceinline__ void fft_v2(double2 *buf, int S, int ss, int es, double s, const TwT &tw) {
    constexpr int L = A * B;
    const int T = blockDim.x;
    for (int u = threadIdx.x; u < S * A; u += T) {
        const int q = u % S, n1 = u / S;
        double2 *base = buf + (size_t)q * ss + (size_t)(B * n1) * es;
        double2 v[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) v[n2] = base[(size_t)n2 * es];
        Dft<B>::run(v, s, tw);
#pragma unroll
        for (int k2 = 1; k2 < B; ++k2) v[k2] = cmul(v[k2], tw.w(n1 * k2, L, s));
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) base[(size_t)k2 * es] = v[k2];
    }
    __syncthreads();
    for (int u = threadIdx.x; u < S * B; u += T) {
        const int q = u % S, k2 = u / S;
        double2 *base = buf + (size_t)q * ss + k2 * es;
        double2 v[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) v[n1] = base[(size_t)(B * n1) * es];
        Dft<A>::run(v, s, tw);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) base[(size_t)(B * k1) * es] = v[k1];
    }
    __syncthreads();
}

// c2r reconstruction of the half-length complex sequence of every row (natural
// order): Z[n] = (X[n] + conj X[M-n]) + i w+^n (X[n] - conj X[M-n]), n < M,
// with Im X[0] = Im X[M] = 0 (FFTW / numpy irfft semantics).
__device__ __forceinline__ double2 c2r_pre_one(double2 xk, double2 xm, double2 wp) {
    const double2 e = make_double2(xk.x + xm.x, xk.y - xm.y);
    const double2 d = make_double2(xk.x - xm.x, xk.y + xm.y);
    const double2 od = cmul(d, wp);
    return make_double2(e.x - od.y, e.y + od.x);
}
__device__ __forceinline__ void y_c2r_pre(double2 *buf, int rows, int pitch, int M, const TwT &tw) {
    const int T = blockDim.x;
    const int npair = M / 2 + 1;
    for (int u = threadIdx.x; u < rows * npair; u += T) {
        const int k = u % rows, n = u / rows;
        double2 *row = buf + (size_t)k * pitch;
        if (n == 0) {
            double2 x0 = row[0], xM = row[M];
            x0.y = 0.0; xM.y = 0.0;
            row[0] = c2r_pre_one(x0, xM, make_double2(1.0, 0.0));
        } else if (2 * n == M) {
            const double2 x = row[n];
            row[n] = c2r_pre_one(x, x, tw.w(n, 2 * M, +1.0));
        } else {
            const double2 xa = row[n], xb = row[M - n];
            row[n] = c2r_pre_one(xa, xb, tw.w(n, 2 * M, +1.0));
            row[M - n] = c2r_pre_one(xb, xa, tw.w(M - n, 2 * M, +1.0));
        }
    }
    __syncthreads();
}

// r2c split of every row: X[n] = (Z[n] + conj Z[M-n])/2 + w-^n (Z[n] - conj Z[M-n])/(2i),
// n = 0..M, Z[M] = Z[0].
__device__ __forceinline__ double2 r2c_post_one(double2 zk, double2 zm, double2 wm) {
    const double2 e = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
    const double2 o = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
    return cadd(e, cmul(wm, o));
}
__device__ __forceinline__ void y_r2c_post(double2 *buf, int rows, int pitch, int M, const TwT &tw) {
    const int T = blockDim.x;
    const int npair = M / 2 + 1;
    for (int u = threadIdx.x; u < rows * npair; u += T) {
        const int k = u % rows, n = u / rows;
        double2 *row = buf + (size_t)k * pitch;
        if (n == 0) {
            const double2 z0 = row[0];
            row[0] = make_double2(z0.x + z0.y, 0.0);
            row[M] = make_double2(z0.x - z0.y, 0.0);
        } else if (2 * n == M) {
            const double2 z = row[n];
            row[n] = r2c_post_one(z, z, tw.w(n, 2 * M, -1.0));
        } else {
            const double2 za = row[n], zb = row[M - n];
            row[n] = r2c_post_one(za, zb, tw.w(n, 2 * M, -1.0));
            row[M - n] = r2c_post_one(zb, za, tw.w(M - n, 2 * M, -1.0));
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Per-size plans: z length N = A_z*B_z, y half length M = N/2 = A_y*B_y.
// ---------------------------------------------------------------------------
template <int N> struct Plan;  // AZ*BZ = N, AY*BY = N/2
template <> struct Plan<32>  { static constexpr int AZ = 8,  BZ = 4, AY = 4,  BY = 4, T = 256, EPT = 3; };
template <> struct Plan<64>  { static constexpr int AZ = 8,  BZ = 8, AY = 8,  BY = 4, T = 256, EPT = 9; };
template <> struct Plan<96>  { static constexpr int AZ = 12, BZ = 8, AY = 12, BY = 4, T = 512, EPT = 10; };
template <> struct Plan<128> { static constexpr int AZ = 16, BZ = 8, AY = 8,  BY = 8, T = 512, EPT = 17; };

// smem row of spectral z index kz after a z pass (fft_v1 output order), and
// the slot of real pair index m in a row (fft_v1 output / fft_v2 input order).
template <int N> __device__ __forceinline__ int zrow(int kz) { return perm_ab<Plan<N>::AZ, Plan<N>::BZ>(kz); }
template <int N> __device__ __forceinline__ int yslot(int m) { return perm_ab<Plan<N>::AY, Plan<N>::BY>(m); }
// inverse of zrow: the kz held by smem row p
template <int N> __device__ __forceinline__ int kz_of_row(int p) { return p / Plan<N>::BZ + Plan<N>::AZ * (p % Plan<N>::BZ); }

// c2r of the plane in buf (natural spectral rows kz, columns ky).  On return,
// real value (z, y) is ((double*)&buf[zrow(z)*pitch + yslot(y/2)])[y&1].
template <int N>
__device__ __forceinline__ void plane_c2r(double2 *buf, const TwT &tw) {
    constexpr int my2 = N / 2 + 1, M = N / 2;
    fft_v1<Plan<N>::AZ, Plan<N>::BZ>(buf, my2, 1, my2, +1.0, tw);
    y_c2r_pre(buf, N, my2, M, tw);
    fft_v1<Plan<N>::AY, Plan<N>::BY>(buf, N, my2, 1, +1.0, tw);
}
// r2c of the plane whose real value (z, y) is stored in the c2r output order
// above.  On return the unscaled spectrum (kz, ky) is at buf[kz*pitch + ky]
// (natural order).
template <int N>
__device__ __forceinline__ void plane_r2c(double2 *buf, const TwT &tw) {
    constexpr int my2 = N / 2 + 1, M = N / 2;
    fft_v2<Plan<N>::AY, Plan<N>::BY>(buf, N, my2, 1, -1.0, tw);
    y_r2c_post(buf, N, my2, M, tw);
    fft_v2<Plan<N>::AZ, Plan<N>::BZ>(buf, my2, 1, my2, -1.0, tw);
}

// Offset of real node (z, y) inside one physical plane of the HBM real fields,
// which are stored exactly as plane_c2r leaves the shared-memory buffer (rows
// of my+2 doubles), so plane loads and stores are single bulk copies.
template <int N> __device__ __host__ __forceinline__ int real_off(int z, int y) {
    return (Plan<N>::BZ * (z % Plan<N>::AZ) + z / Plan<N>::AZ) * (N + 2) + 2 * (Plan<N>::BY * ((y >> 1) % Plan<N>::AY) + (y >> 1) / Plan<N>::AY) + (y & 1);
}

}  // namespace pibm
