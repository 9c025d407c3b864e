// step_common.cuh -- device helpers shared by the flow and scalar kernels:
// twiddle loads, bounded bulk-copy waits, deterministic block reductions,
// the order-2 interpolation stencil, and the cluster launch of plane kernels.
#pragma once
#include "engine.cuh"
#include "fft2d.cuh"
#include "plane_cl.cuh"
#include "bulk.cuh"
#include "../../include/pibm.h"

namespace pibm {

constexpr int kDragSplit = 8;   // CTAs per sphere of the surface-quadrature kernels
constexpr double kSmallD = 1.0000000180025095e-35;   // (double)1.0E-35f, SMALL_NUMBER of constants.F90:92

template <int N>
__device__ __forceinline__ void load_tw(double2 *tws, const Geo &g) {
    for (int t = threadIdx.x; t < N; t += blockDim.x) tws[t] = g.tw[t];
}
// Physical real planes are RSP = N*(N+2) doubles: the shared-memory image of a
// transformed plane (rows of N data doubles + 2 unused).
template <int N> struct RP { static constexpr int RSP = N * (N + 2); static constexpr uint32_t BYTES = RSP * 8; };
// a / b from the reciprocal y = 1/b (correctly rounded, computed once by the
// caller): q = a*y, then one correction with the exact FMA remainder,
// q + (a - q*b)*y (Markstein, IBM J. Res. Dev. 34(1), 1990; "Markstein's
// theorem" in Muller et al., Handbook of Floating-Point Arithmetic).  For
// normal operands and quotients the result is the correctly rounded a / b
// (checked against the division on the device in the tests); a zero
// remainder means q is exact and is kept as is, sign of zero included.
__device__ __forceinline__ double qdiv(double a, double b, double y) {
    const double q = a * y;
    const double e = fma(-q, b, a);
    return e == 0.0 ? q : fma(e, y, q);
}

// The r2c normalisation x / nrm, nrm = my*mz = N*N (ff2rc).  For N a power of
// two 1/nrm is exact, so x * (1/nrm) and x / nrm are the same correctly rounded
// value and the multiplication replaces the longer division sequence; other
// sizes keep the division.
template <int N> __device__ __forceinline__ double2 r2c_norm(double2 x, double nrm) {
    if constexpr ((N & (N - 1)) == 0) {
        constexpr double r = 1.0 / ((double)N * (double)N);
        return make_double2(x.x * r, x.y * r);
    } else {
        return make_double2(x.x / nrm, x.y / nrm);
    }
}
// The run's status word for a block-wide early return: the OR over the
// block's threads, so that every thread takes the same branch before the
// block's barriers although another kernel, or another block of this one,
// may set the word while the block starts.  Call with every thread present.
__device__ __forceinline__ bool block_failed(const Scal *sc) { return __syncthreads_or(sc->status != 0) != 0; }

// Bounded wait on the CTA's load barrier; records a timeout in the status word.
__device__ __forceinline__ void load_wait(uint64_t *mb, uint32_t &phase, Scal *sc) {
    if (!mbar_wait(mb, phase)) atomicCAS(&sc->status, 0, PIBM_ERR_TIMEOUT);
    phase ^= 1u;
}

// Deterministic block sum (fixed lane/warp tree).
__device__ __forceinline__ double block_sum(double v, double *scr) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) scr[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < nw ? scr[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    if (threadIdx.x == 0) scr[0] = r;
    __syncthreads();
    r = scr[0];
    __syncthreads();
    return r;
}
// K block sums (or maxima) at once, each with block_sum's (block_max's)
// lane/warp tree, so every result is bitwise that of a separate call; two
// barriers for all K instead of four each.  scr holds 32*K doubles.
template <int K, bool kMax = false>
__device__ __forceinline__ void block_reduce_k(double (&v)[K], double *scr) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_xor_sync(0xffffffffu, v[k], o);
            v[k] = kMax ? fmax(v[k], t) : v[k] + t;
        }
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) scr[k * 32 + w] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double r = lane < nw ? scr[k * 32 + lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_xor_sync(0xffffffffu, r, o);
            r = kMax ? fmax(r, t) : r + t;
        }
        v[k] = r;   // every warp computes the same tree: no third barrier
    }
    __syncthreads();
}
__device__ __forceinline__ double block_max(double v, double *scr) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) scr[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < nw ? scr[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
    }
    __syncthreads();
    if (threadIdx.x == 0) scr[0] = r;
    __syncthreads();
    r = scr[0];
    __syncthreads();
    return r;
}

// ============================================================================
// Interpolation stencils ('lpi', order 2, periodic): stencil = [pc, pc+1]
// (dependent_functions.F90:45-275; interpolation.F90:202-381,740-751).
// Geometry uses explicitly rounded operations so host and device agree.
// ============================================================================
struct Sten {
    int ii[2], jj[2], kk[2];
    double xv[2], yv[2], zv[2];
    __device__ __forceinline__ double w(int a, int b, int c) const { return __dmul_rn(__dmul_rn(xv[a], yv[b]), zv[c]); }
};

__device__ __forceinline__ int cell_of(double x) { return x < 0.0 ? (int)(x - 1.0) : (int)x; }

__device__ __forceinline__ int wrapi(int v, int n) { return v < 1 ? v + n : (v > n ? v - n : v); }

__device__ __forceinline__ void make_sten(const Geo &g, const double pos[3], Sten &s) {
    int pc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) pc[d] = cell_of(pos[d]);
    const double zx = __dsub_rn(pos[0], (double)pc[0]);
    const double zy = __dsub_rn(pos[1], (double)pc[1]);
    const double zz = __dsub_rn(pos[2], (double)pc[2]);
    s.xv[0] = __dsub_rn(1.0, zx); s.xv[1] = zx;
    s.yv[0] = __dsub_rn(1.0, zy); s.yv[1] = zy;
    s.zv[0] = __dsub_rn(1.0, zz); s.zv[1] = zz;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        s.ii[q] = wrapi(pc[0] + q, g.nx) - 1;   // 0-based
        s.jj[q] = wrapi(pc[1] + q, g.my) - 1;
        s.kk[q] = wrapi(pc[2] + q, g.mz) - 1;
    }
}

// Contribution of a reversal point to one node of its inner stencil, entry
// ent = 8 p + a + 2 b + 4 c of the spreading lists: w * force_tmp / dx^3
// (boundary_condition.F90:1425-1462), w the trilinear weight of corner
// (a, b, c) formed from the point's cell offsets rz[3p..3p+2] as make_sten and
// Sten::w form it, force_tmp = rec[6p..6p+2].  k_rev forms the same values
// for its sums, so they are bitwise those it would have stored.
__device__ __forceinline__ void corner_contrib(const double *__restrict__ rz, const double *__restrict__ rec, int ent,
                                               double dx3, double rdx3, double t[3]) {
    const size_t p = (size_t)(ent >> 3);
    const double zx = __ldg(rz + 3 * p), zy = __ldg(rz + 3 * p + 1), zz = __ldg(rz + 3 * p + 2);
    const double wx = (ent & 1) ? zx : __dsub_rn(1.0, zx);
    const double wy = (ent & 2) ? zy : __dsub_rn(1.0, zy);
    const double wz = (ent & 4) ? zz : __dsub_rn(1.0, zz);
    const double w = __dmul_rn(__dmul_rn(wx, wy), wz);
#pragma unroll
    for (int n = 0; n < 3; ++n) t[n] = qdiv(w * __ldg(rec + 6 * p + n), dx3, rdx3);
}

// value at node (x=i, y=j, z=k) of a physical field (one component)
template <int N>
__device__ __forceinline__ double fat(const double *f, int i, int j, int k) {
    return __ldg(f + (size_t)i * RP<N>::RSP + real_off<N>(k, j));
}
// interpolator order (k, j, i)
template <int N>
__device__ __forceinline__ double interp_kji(const Sten &s, const double *f, double add = 0.0) {
    double r = 0.0;
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int a = 0; a < 2; ++a) r = r + (fat<N>(f, s.ii[a], s.jj[b], s.kk[c]) + add) * s.w(a, b, c);
    return r;
}
// array_dot_product order (i, j, k)
template <int N>
__device__ __forceinline__ double dot_ijk(const Sten &s, const double *f) {
    double r = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < 2; ++c) r = r + fat<N>(f, s.ii[a], s.jj[b], s.kk[c]) * s.w(a, b, c);
    return r;
}

// ============================================================================
// Plane-kernel launches
// ============================================================================
template <int N>
inline size_t plane_smem() { return cl_smem<N>(); }

// Launch a plane kernel on nplanes planes: PL<N>::C CTAs per plane, grouped
// into clusters of that size (the plane's CTAs exchange data through
// distributed shared memory).
template <int N, typename... KArgs, typename... Args>
inline void launch_planes(void (*k)(KArgs...), int nplanes, int items, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nplanes * PL<N>::C), (unsigned)items, 1);
    cfg.blockDim = dim3(PL<N>::T, 1, 1);
    cfg.dynamicSmemBytes = plane_smem<N>();
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = PL<N>::C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, args...);
}


// Planes one thread of the scalar's x-flux kernel covers (flux_segment gives
// the flow's).
constexpr int kScalarFluxSeg = 32;

// launch_planes for a fused batch: nz runs of the same size along gridDim.z.
template <int N, typename... KArgs, typename... Args>
inline void launch_planes_z(void (*k)(KArgs...), int nplanes, int items, int nz, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nplanes * PL<N>::C), (unsigned)items, (unsigned)nz);
    cfg.blockDim = dim3(PL<N>::T, 1, 1);
    cfg.dynamicSmemBytes = plane_smem<N>();
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = PL<N>::C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, args...);
}

// Tile row pitch of the x-line kernels' [line][i] tiles (double2 elements).  A 16-byte shared access is
// served per 8 threads (128 bytes = 8 slots of 4 banks); the element loops put
// thread t on (line t % LT, plane t / LT), so 8 threads cover 8 lines of one
// plane for LT = 8 (an odd pitch puts them in distinct slots) and 4 lines of two
// planes for LT = 4 (a pitch of 2 mod 8 does: slot 2*line + i).
template <int NX, int LT> __host__ __device__ constexpr int lines_pitch() { return LT == 4 ? NX + 2 : NX + 1; }

}  // namespace pibm
