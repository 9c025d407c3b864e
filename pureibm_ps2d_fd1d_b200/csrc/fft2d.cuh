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
// Per-size plans: z length N = AZ*BZ, y half length M = N/2 = AY*BY, T threads.
// EPT = spectral elements per thread (ceil(my2*N / T)).
// ---------------------------------------------------------------------------
template <int N> struct Plan;
template <> struct Plan<32>  { static constexpr int AZ = 8,  BZ = 4, AY = 4,  BY = 4, T = 256, EPT = 3; };
template <> struct Plan<64>  { static constexpr int AZ = 8,  BZ = 8, AY = 8,  BY = 4, T = 256, EPT = 9; };
template <> struct Plan<96>  { static constexpr int AZ = 12, BZ = 8, AY = 12, BY = 4, T = 512, EPT = 10; };
template <> struct Plan<128> { static constexpr int AZ = 16, BZ = 8, AY = 8,  BY = 8, T = 512, EPT = 17; };
template <> struct Plan<256> { static constexpr int AZ = 16, BZ = 16, AY = 16, BY = 8, T = 512, EPT = 65; };

// smem row of physical z after an inverse z pass (bfft_v1 output order), and
// the slot of real pair index m in a row (bfft_v1 output / bfft_v2 input order).
template <int N> __device__ __forceinline__ int zrow(int z) { return perm_ab<Plan<N>::AZ, Plan<N>::BZ>(z); }
template <int N> __device__ __forceinline__ int yslot(int m) { return perm_ab<Plan<N>::AY, Plan<N>::BY>(m); }

// c2r reconstruction of one element pair: Z[n] = (X[n] + conj X[M-n]) + i w+^n (X[n] - conj X[M-n]).
__device__ __forceinline__ double2 c2r_pre_one(double2 xk, double2 xm, double2 wp) {
    const double2 e = make_double2(xk.x + xm.x, xk.y - xm.y);
    const double2 d = make_double2(xk.x - xm.x, xk.y + xm.y);
    const double2 od = cmul(d, wp);
    return make_double2(e.x - od.y, e.y + od.x);
}
// r2c split of one element pair: X[n] = (Z[n] + conj Z[M-n])/2 + w-^n (Z[n] - conj Z[M-n])/(2i).
__device__ __forceinline__ double2 r2c_post_one(double2 zk, double2 zm, double2 wm) {
    const double2 e = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
    const double2 o = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
    return cadd(e, cmul(wm, o));
}

// ---------------------------------------------------------------------------
// Block-wide passes over S sequences (element e of sequence q at
// buf[q*ss + e*es]) with a compile-time thread count T, so that the rounds a
// thread executes are unrolled and interleaved.  Units are distributed with
// the sequence index fastest: consecutive threads touch consecutive columns
// (stride 1) or rows (stride pitch = my2, 4 banks apart), conflict-free.
// Each pass ends with __syncthreads.
// ---------------------------------------------------------------------------
template <int A, int B, int S, int T>
__device__ __forceinline__ void bfft_v1(double2 *buf, int ss, int es, double s, const TwT &tw) {
    constexpr int L = A * B;
#pragma unroll
    for (int u0 = 0; u0 < S * B; u0 += T) {
        const int u = u0 + (int)threadIdx.x;
        if (u < S * B) {
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
    }
    __syncthreads();
#pragma unroll
    for (int u0 = 0; u0 < S * A; u0 += T) {
        const int u = u0 + (int)threadIdx.x;
        if (u < S * A) {
            const int q = u % S, k1 = u / S;
            double2 *base = buf + (size_t)q * ss + (size_t)(B * k1) * es;
            double2 v[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) v[n2] = base[(size_t)n2 * es];
            Dft<B>::run(v, s, tw);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) base[(size_t)k2 * es] = v[k2];
        }
    }
    __syncthreads();
}

template <int A, int B, int S, int T>
__device__ __forceinline__ void bfft_v2(double2 *buf, int ss, int es, double s, const TwT &tw) {
    constexpr int L = A * B;
#pragma unroll
    for (int u0 = 0; u0 < S * A; u0 += T) {
        const int u = u0 + (int)threadIdx.x;
        if (u < S * A) {
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
    }
    __syncthreads();
#pragma unroll
    for (int u0 = 0; u0 < S * B; u0 += T) {
        const int u = u0 + (int)threadIdx.x;
        if (u < S * B) {
            const int q = u % S, k2 = u / S;
            double2 *base = buf + (size_t)q * ss + k2 * es;
            double2 v[A];
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) v[n1] = base[(size_t)(B * n1) * es];
            Dft<A>::run(v, s, tw);
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1) base[(size_t)(B * k1) * es] = v[k1];
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Packed ky = 0 / ky = M columns.  The two columns share one complex z
// transform held in column 0:
//  c2r: only Re of their inverse z transforms is used (the y reconstruction
//       drops the imaginary parts of ky = 0 and ky = M), and
//       Re(IFFT X) = IFFT(Herm X), Herm X[k] = (X[k] + conj X[-k])/2, so
//       column 0 <- Herm X0 + i Herm XM; the y reconstruction reads
//       Re -> ky = 0 and Im -> ky = M back from column 0.
//  r2c: both columns are real after the y pass, column 0 <- X0 + i XM; the
//       spectrum is read back with cl_unpack (A = (Y[k] + conj Y[-k])/2,
//       B = (Y[k] - conj Y[-k])/(2i)).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 herm_pack(double2 a, double2 am, double2 b, double2 bm) {
    const double2 h0 = make_double2(0.5 * (a.x + am.x), 0.5 * (a.y - am.y));
    const double2 hm = make_double2(0.5 * (b.x + bm.x), 0.5 * (b.y - bm.y));
    return make_double2(h0.x - hm.y, h0.y + hm.x);
}
// Offset of real node (z, y) inside one physical plane of the HBM real fields,
// which are stored exactly as the c2r plane transform leaves its rows in
// shared memory (rows of my+2 doubles), so plane loads and stores are bulk copies.
template <int N> __device__ __host__ __forceinline__ int real_off(int z, int y) {
    return (Plan<N>::BZ * (z % Plan<N>::AZ) + z / Plan<N>::AZ) * (N + 2) + 2 * (Plan<N>::BY * ((y >> 1) % Plan<N>::AY) + (y >> 1) / Plan<N>::AY) + (y & 1);
}

}  // namespace pibm
