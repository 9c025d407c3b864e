// plane_cl.cuh -- y-z plane transforms split over a thread-block cluster.
//
// A whole complex half-plane (N rows kz x N/2+1 columns ky, FP64) is 133 KB
// at N = 128, so a CTA that holds one leaves room for no second CTA on the SM
// and its loads, stores and barriers cannot overlap anything.  Here a plane
// is shared by a cluster of C CTAs, each holding 1/C of it:
//
//   column phase (z transforms)  CTA r holds columns ky in [r*MC, (r+1)*MC) of
//                                all N rows at pitch PZ = MC+1; CTA 0 also
//                                keeps column ky = M = N/2 in slot MC.
//   row phase (y transforms)     CTA r holds rows [r*NR, (r+1)*NR) of the plane
//                                in z-transform output order at pitch P = M+1:
//                                exactly those rows of the single-CTA image,
//                                so a real plane keeps its HBM layout and CTA r
//                                moves its rows with one contiguous bulk copy.
//
// Between the phases the elements cross between the CTAs' shared memory
// (distributed shared memory, map_shared_rank) between two cluster barriers,
// fused with the half-length real-transform step of the y direction (c2r:
// each CTA pulls its rows; r2c: each CTA pushes its rows to the column
// owners).  The arithmetic of every element is the same as in the single-CTA
// transform.
#pragma once
#include <cooperative_groups.h>

#include "fft2d.cuh"

namespace pibm {

namespace cg = cooperative_groups;

// CTAs per plane (C) and threads per CTA (T) for each supported size.
template <int N> struct ClCfg;
template <> struct ClCfg<32>  { static constexpr int C = 1, T = 256; };
template <> struct ClCfg<64>  { static constexpr int C = 2, T = 128; };
template <> struct ClCfg<96>  { static constexpr int C = 2, T = 256; };
template <> struct ClCfg<128> { static constexpr int C = 2, T = 256; };
template <> struct ClCfg<256> { static constexpr int C = 8, T = 256; };

template <int N> struct PL {
    static constexpr int C = ClCfg<N>::C, T = ClCfg<N>::T;
    static constexpr int M = N / 2, P = M + 1;          // row-phase pitch (complex slots)
    static constexpr int MC = M / C, PZ = MC + 1;       // columns per CTA, column-phase pitch
    static constexpr int NR = N / C;                    // rows per CTA in the row phase
    static constexpr int BUF = (N * PZ > NR * P) ? N * PZ : NR * P;   // complex slots of the buffer
    static constexpr int RL = NR * (N + 2);             // doubles of one CTA's real rows
    static constexpr uint32_t RBYTES = RL * 8;
    static constexpr int NOUT = N * PZ;                 // column-phase slots (slot MC: rank 0 only)
    static constexpr int EPT = (NOUT + T - 1) / T;
    // CTAs per SM the register budget is sized for: at 128^3 three CTAs of
    // 256 threads (80 registers, 24 warps per SM) measured faster than two
    // (128 registers), spills of the nonlinear kernels' epilogue included;
    // the other sizes keep 128 registers (their nonlinear kernels spill more,
    // and the batched ensemble measured slower with them at 80)
    static constexpr int MINB = (N == 128) ? 3 : 512 / T;
    static_assert(M % C == 0 && N % C == 0, "plane split");
    static_assert(RBYTES % 16 == 0, "bulk copies move 16-byte multiples");
};
// Dynamic shared memory of a plane kernel: buffer + twiddle table.
template <int N> constexpr size_t cl_smem() { return (size_t)(PL<N>::BUF + N) * sizeof(double2); }

// Physical z of shared-memory row R (inverse of zrow), and pair index m of
// row slot s (inverse of yslot).
template <int N> __device__ __forceinline__ int zinv(int R) { return (R % Plan<N>::BZ) * Plan<N>::AZ + R / Plan<N>::BZ; }
template <int N> __device__ __forceinline__ int yinv(int s) { return (s % Plan<N>::BY) * Plan<N>::AY + s / Plan<N>::BY; }

// Global column ky of column-phase slot jl of CTA `rank`.
template <int N> __device__ __forceinline__ int cl_col(int jl, int rank) {
    return jl == PL<N>::MC ? PL<N>::M : rank * PL<N>::MC + jl;
}

// 32-bit shared::cluster address of element `slot` of CTA `rank`'s buffer,
// and a 16-byte store through it (distributed shared memory).
__device__ __forceinline__ uint32_t cl_addr(const double2 *buf, int slot, int rank) {
    uint32_t r;
    asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"((uint32_t)__cvta_generic_to_shared(buf + slot)), "r"(rank));
    return r;
}
__device__ __forceinline__ void cl_st(uint32_t addr, double2 v) {
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v.x), "d"(v.y) : "memory");
}

// CTA 0, warp 0: column 0 <- Herm(ky = 0) + i Herm(ky = M) (see herm_pack).
template <int N>
__device__ __forceinline__ void cl_pack_col0(double2 *buf) {
    using L = PL<N>;
    constexpr int R = (N + 31) / 32;
    const int lane = threadIdx.x & 31;
    double2 y[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        if (k < N) {
            const int km = (N - k) % N;
            y[r] = herm_pack(buf[k * L::PZ], buf[km * L::PZ], buf[k * L::PZ + L::MC], buf[km * L::PZ + L::MC]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        if (k < N) buf[k * L::PZ] = y[r];
    }
}

// Spectral value of column-phase slot (kz, jl) after cl_r2c (unscaled).
// CTA 0 reads ky = 0 (jl = 0) and ky = M (jl = MC) from the packed column 0.
template <int N>
__device__ __forceinline__ double2 cl_unpack(const double2 *buf, int kz, int jl, int rank) {
    using L = PL<N>;
    if (rank != 0 || (jl != 0 && jl != L::MC)) return buf[kz * L::PZ + jl];
    const double2 y = buf[kz * L::PZ], ym = buf[((N - kz) % N) * L::PZ];
    if (jl == 0) return make_double2(0.5 * (y.x + ym.x), 0.5 * (y.y - ym.y));
    return make_double2(0.5 * (y.y + ym.y), -0.5 * (y.x - ym.x));
}

// c2r reconstruction of ROWS rows at pitch P: each row's M+1 spectral values
// X[0..M] (ky = 0 in Re and ky = M in Im of slot 0) become the M complex
// points Z[n] = (X[n] + conj X[M-n]) + i w+^n (X[n] - conj X[M-n]) of the
// half-length inverse transform.
template <int N, int T, int ROWS>
__device__ __forceinline__ void rows_c2r_pre(double2 *buf, const TwT &tw) {
    constexpr int M = N / 2, P = N / 2 + 1, NP = M / 2 + 1;
#pragma unroll 3
    for (int u0 = 0; u0 < ROWS * NP; u0 += T) {
        const int u = u0 + (int)threadIdx.x;
        if (u < ROWS * NP) {
            const int k = u % ROWS, n = u / ROWS;
            double2 *row = buf + (size_t)k * P;
            if (n == 0) {
                const double2 y = row[0];
                row[0] = c2r_pre_one(make_double2(y.x, 0.0), make_double2(y.y, 0.0), make_double2(1.0, 0.0));
            } else if (2 * n == M) {
                const double2 x = row[n];
                row[n] = c2r_pre_one(x, x, tw.w(n, 2 * M, +1.0));
            } else {
                const double2 xa = row[n], xb = row[M - n];
                row[n] = c2r_pre_one(xa, xb, tw.w(n, 2 * M, +1.0));
                row[M - n] = c2r_pre_one(xb, xa, tw.w(M - n, 2 * M, +1.0));
            }
        }
    }
    __syncthreads();
}
// r2c split of ROWS rows at pitch P: the half-length transform Z[0..M-1] of a
// real row becomes X[n] = (Z[n] + conj Z[M-n])/2 + w-^n (Z[n] - conj Z[M-n])/(2i);
// the two real values X[0] and X[M] are packed into slot 0 as X[0] + i X[M].
template <int N, int T, int ROWS>
__device__ __forceinline__ void rows_r2c_post(double2 *buf, const TwT &tw) {
    constexpr int M = N / 2, P = N / 2 + 1, NP = M / 2 + 1;
#pragma unroll 3
    for (int u0 = 0; u0 < ROWS * NP; u0 += T) {
        const int u = u0 + (int)threadIdx.x;
        if (u < ROWS * NP) {
            const int k = u % ROWS, n = u / ROWS;
            double2 *row = buf + (size_t)k * P;
            if (n == 0) {
                const double2 z0 = row[0];
                row[0] = make_double2(z0.x + z0.y, z0.x - z0.y);
            } else if (2 * n == M) {
                const double2 z = row[n];
                row[n] = r2c_post_one(z, z, tw.w(n, 2 * M, -1.0));
            } else {
                const double2 za = row[n], zb = row[M - n];
                row[n] = r2c_post_one(za, zb, tw.w(n, 2 * M, -1.0));
                row[M - n] = r2c_post_one(zb, za, tw.w(M - n, 2 * M, -1.0));
            }
        }
    }
    __syncthreads();
}

// The exchanges fused with the half-length real-transform step.  Row r of a
// CTA's row phase is processed as M/2 units: unit j = 0 takes slot 0 (ky = 0
// in Re, ky = M in Im after the packed z pass) and slot M/2, unit j in
// [1, M/2) the mirror pair (j, M - j).  Each unit produces its two outputs
// from its two inputs, so the separate row pass of rows_c2r_pre /
// rows_r2c_post disappears and every element crosses shared memory once.
template <int N> __device__ __forceinline__ int cl_mirror(int j) { return j == 0 ? N / 4 : N / 2 - j; }

// c2r: column phase -> row phase with the reconstruction Z[n] of rows_c2r_pre.
// Pull: every CTA reads its rows' mirror pairs from the column owners, then
// rewrites its own buffer in the row layout.
template <int N>
__device__ __forceinline__ void cl_cols_to_rows_pre(double2 *buf, const TwT &tw, int rank) {
    using L = PL<N>;
    constexpr int H = L::M / 2, TOT = L::NR * H, K = (TOT + L::T - 1) / L::T;
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();   // every CTA of the plane finished its z pass
    double2 va[K], vb[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int u = (int)threadIdx.x + k * L::T;
        if (u < TOT) {
            const int r = u / H, j = u - r * H, nb = cl_mirror<N>(j);
            const int ha = j / L::MC, hb = nb / L::MC, row = (rank * L::NR + r) * L::PZ;
            const double2 xa = cl.map_shared_rank(buf, ha)[row + j - ha * L::MC];
            const double2 xb = cl.map_shared_rank(buf, hb)[row + nb - hb * L::MC];
            if (j == 0) {
                va[k] = c2r_pre_one(make_double2(xa.x, 0.0), make_double2(xa.y, 0.0), make_double2(1.0, 0.0));
                vb[k] = c2r_pre_one(xb, xb, tw.w(H, N, +1.0));
            } else {
                va[k] = c2r_pre_one(xa, xb, tw.w(j, N, +1.0));
                vb[k] = c2r_pre_one(xb, xa, tw.w(nb, N, +1.0));
            }
        }
    }
    cl.sync();   // every CTA finished reading: buffers may be rewritten
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int u = (int)threadIdx.x + k * L::T;
        if (u < TOT) {
            const int r = u / H, j = u - r * H;
            buf[r * L::P + j] = va[k];
            buf[r * L::P + cl_mirror<N>(j)] = vb[k];
        }
    }
    __syncthreads();
}

// r2c: row phase -> column phase with the split X[n] of rows_r2c_post.
// Push: every CTA forms the outputs of its own rows, and after a cluster
// barrier (all rows read) stores them into the column owners' buffers.
template <int N>
__device__ __forceinline__ void cl_rows_to_cols_post(double2 *buf, const TwT &tw, int rank) {
    using L = PL<N>;
    constexpr int H = L::M / 2, TOT = L::NR * H, K = (TOT + L::T - 1) / L::T;
    cg::cluster_group cl = cg::this_cluster();
    double2 va[K], vb[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int u = (int)threadIdx.x + k * L::T;
        if (u < TOT) {
            const int r = u / H, j = u - r * H, nb = cl_mirror<N>(j);
            const double2 za = buf[r * L::P + j], zb = buf[r * L::P + nb];
            if (j == 0) {
                va[k] = make_double2(za.x + za.y, za.x - za.y);
                vb[k] = r2c_post_one(zb, zb, tw.w(H, N, -1.0));
            } else {
                va[k] = r2c_post_one(za, zb, tw.w(j, N, -1.0));
                vb[k] = r2c_post_one(zb, za, tw.w(nb, N, -1.0));
            }
        }
    }
    cl.sync();   // every CTA read its rows: buffers may be rewritten
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int u = (int)threadIdx.x + k * L::T;
        if (u < TOT) {
            const int r = u / H, j = u - r * H, nb = cl_mirror<N>(j);
            const int ha = j / L::MC, hb = nb / L::MC, row = (rank * L::NR + r) * L::PZ;
            cl_st(cl_addr(buf, row + j - ha * L::MC, ha), va[k]);
            cl_st(cl_addr(buf, row + nb - hb * L::MC, hb), vb[k]);
        }
    }
    cl.sync();   // every column of the plane is in place
}

// c2r of the CTA's columns (natural kz, column-phase layout; CTA 0 with
// ky = M in slot MC).  Call after a __syncthreads.  On return the CTA holds
// rows [rank*NR, (rank+1)*NR) of the real plane image: real value (z, y) of
// such a row R = zrow(z) is ((double*)buf)[(R - rank*NR)*(N+2) + 2*yslot(y/2) + (y&1)].
template <int N>
__device__ __forceinline__ void cl_c2r(double2 *buf, const TwT &tw, int rank) {
    using L = PL<N>;
    if (rank == 0) {
        if (threadIdx.x < 32) cl_pack_col0<N>(buf);
        __syncthreads();
    }
    bfft_v1<Plan<N>::AZ, Plan<N>::BZ, L::MC, L::T>(buf, 1, L::PZ, +1.0, tw);
    if constexpr (L::C > 1) {
        cl_cols_to_rows_pre<N>(buf, tw, rank);
    } else {
        rows_c2r_pre<N, L::T, L::NR>(buf, tw);
    }
    bfft_v1<Plan<N>::AY, Plan<N>::BY, L::NR, L::T>(buf, L::P, 1, +1.0, tw);
}

// r2c of the CTA's real rows (row-phase layout, as cl_c2r leaves them).  Call
// after a __syncthreads.  On return the CTA holds its columns, natural in kz,
// unscaled; read them with cl_unpack.
template <int N>
__device__ __forceinline__ void cl_r2c(double2 *buf, const TwT &tw, int rank) {
    using L = PL<N>;
    bfft_v2<Plan<N>::AY, Plan<N>::BY, L::NR, L::T>(buf, L::P, 1, -1.0, tw);
    if constexpr (L::C > 1) {
        cl_rows_to_cols_post<N>(buf, tw, rank);
    } else {
        rows_r2c_post<N, L::T, L::NR>(buf, tw);
    }
    bfft_v2<Plan<N>::AZ, Plan<N>::BZ, L::MC, L::T>(buf, 1, L::PZ, -1.0, tw);
}

}  // namespace pibm
