// lines_pipe.cuh -- the x-line part of velstep (pressure -> ustep -> divcorr,
// poisson.F90:55-508, usteptime.F90:45-269, check_divergence
// steptheflow.F90:219-240) as a persistent kernel fed by tensor-map copies.
//
// The staged kernel (b_lines) loads a tile's 13 input fields with ordinary
// loads in a few passes separated by barriers, so few bytes are in flight per
// SM and its solves wait on its loads.  Here one producer warp streams the
// tile's fields, one field at a time, as "slabs" (one field's values over 4
// lines x NX planes, 64-byte rows: the 4 lines are contiguous in the
// [comp][i][kz][ky] layout) through a ring of KR shared-memory slots with
// tiled bulk-tensor copies, and runs ahead into the next tile while the four
// consumer warps (one line each) solve.  The consumers take the fields in the
// order the reference forms the pressure source -- (nl, ff) of each component,
// then onl -- and accumulate the source (in registers) and the explicit ustep
// terms (in the u tiles) with every rounding written out (psrc_term_rt,
// cadd_rn), so the results are bitwise those of b_lines.  u and p leave
// through tensor-map stores of the tile's work tiles.  Tiles are handed out
// dynamically (an atomic ticket), so the block that draws the (0,0) line,
// whose Thomas solves are serial, takes fewer tiles.
//
// Every slab and work tile is a [i][line] box with the 64-byte swizzle: line
// l of plane i sits at byte i*64 + 16*(l ^ ((i >> 1) & 3)), so a warp reading
// one line at 32 consecutive planes touches 32 distinct bank groups.
#pragma once
#include <cuda.h>

#include "bulk.cuh"
#include "line_solve.cuh"

namespace pibm {

// Tensor maps of the kernel's fields, each [comp][i][PS complex] seen as
// FLOAT64 {2 PS, nx, ncomp} with the box {8, NX, 1} and the 64-byte swizzle.
struct LineMaps {
    CUtensorMap u, p, nl, onl, ff;
};

template <int NX> struct LPipe {
    static constexpr int R = NX / 32;          // planes per lane
    static constexpr int LT = 4;               // lines per tile = consumer warps
    static constexpr int KR = 3;               // slab ring depth
    static constexpr int NSLAB = 13;           // input slabs per tile
    static constexpr int SLAB = NX * 64;       // bytes of one field over a tile
    static constexpr int T = (LT + 1) * 32;    // consumers + producer warp
    static constexpr int MINB = 3;             // blocks per SM the budget is sized for
    // shared-memory byte offsets from a 1024-byte aligned base
    static constexpr int O_RING = 0;
    static constexpr int O_P = O_RING + KR * SLAB;           // p tile (TMA store source)
    static constexpr int O_U = O_P + SLAB;                   // 3 u tiles (TMA store sources)
    static constexpr int O_ROW = O_U + 3 * SLAB;             // per-warp rows [LT][NX] double2
    static constexpr int O_TWS = O_ROW + LT * NX * 16;       // twiddles, NX double2
    static constexpr int O_ST = O_TWS + NX * 16;             // stage table, 32 double2
    static constexpr int O_LCS = O_ST + 32 * 16;             // per-lane cosines, R*32 doubles
    static constexpr int O_LTR = O_LCS + R * 32 * 8;         // per-lane twiddles, (R-1)*32 double2
    static constexpr int O_GAM = O_LTR + (R - 1) * 32 * 16;  // Thomas scratch, NX doubles
    static constexpr int O_BAR = O_GAM + NX * 8;             // full[KR], empty[KR]
    static constexpr int O_TID = O_BAR + 2 * KR * 8;         // ticket of the tile in flight, 2 ints
    static constexpr int BYTES = O_TID + 16;
    static constexpr int SMEM = BYTES + 1024;                // + alignment slack
    static_assert(SLAB % 1024 == 0, "slabs keep the swizzle's 1024-byte alignment");
};

// Byte offset of (plane i, line l) in a swizzled slab or tile.
__device__ __forceinline__ int sw64(int i, int l) { return i * 64 + ((l ^ ((i >> 1) & 3)) << 4); }
__device__ __forceinline__ double2 &tel(unsigned char *tile, int i, int l) { return *reinterpret_cast<double2 *>(tile + sw64(i, l)); }

// Input slab j of a tile: its map and component, in the order of consumption.
__device__ __forceinline__ const CUtensorMap *slab_map(const LineMaps &mp, int j, int &comp) {
    if (j < 6) { comp = j >> 1; return (j & 1) ? &mp.ff : &mp.nl; }
    if (j < 9) { comp = j - 6; return &mp.onl; }
    if (j == 9) { comp = 0; return &mp.p; }
    comp = j - 10;
    return &mp.u;
}

template <int NX>
__device__ __forceinline__ void lines_pipe_body(const Geo &g, const LineMaps &mp, Scal *__restrict__ sc) {
    using L = LPipe<NX>;
    constexpr int R = L::R, KR = L::KR;
    extern __shared__ unsigned char lp_raw[];
    unsigned char *sm = lp_raw + ((1024u - (smem_u32(lp_raw) & 1023u)) & 1023u);
    unsigned char *ring = sm + L::O_RING, *Pt = sm + L::O_P, *Ut = sm + L::O_U;   // u tile n at Ut + n*SLAB
    double2 *tws = reinterpret_cast<double2 *>(sm + L::O_TWS);
    double2 *st = reinterpret_cast<double2 *>(sm + L::O_ST);
    double *lcs = reinterpret_cast<double *>(sm + L::O_LCS);
    double2 *ltr = reinterpret_cast<double2 *>(sm + L::O_LTR);
    double *gam = reinterpret_cast<double *>(sm + L::O_GAM);
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + L::O_BAR), *empty = full + KR;
    volatile int *tid_ring = reinterpret_cast<int *>(sm + L::O_TID);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = g.PS / L::LT;

    if (threadIdx.x == 0)
        for (int k = 0; k < KR; ++k) { mbar_init(full + k, 1); mbar_init(empty + k, L::LT); }
    for (int t = threadIdx.x; t < NX; t += blockDim.x) tws[t] = g.tw[t];
    fill_stage_table<32>(st, g.tw, NX);
    fill_line_tw<R>(lcs, ltr, g.tw);
    grid_dep_wait();   // the tables above are set-up data; the fields and the status come from earlier kernels
    // one barrier: the early-return vote, the barrier inits and the tables
    const bool failed = block_failed(sc);

    if (!failed && warp == L::LT) {
        // ---------------- producer: tickets and slab copies ----------------
        if (lane == 0) {
            uint32_t k = 0;
            for (int c = 0;; ++c) {
                const int t = (int)atomicAdd(&sc->lines_next, 1u);
                for (int j = 0; j < L::NSLAB; ++j, ++k) {
                    const int slot = k % KR;
                    if (k >= KR && !mbar_wait(empty + slot, ((k / KR) - 1) & 1)) atomicCAS(&sc->status, 0, PIBM_ERR_TIMEOUT);
                    if (j == 0) {
                        tid_ring[c & 1] = t < ntiles ? t : -1;
                        if (t >= ntiles) { mbar_arrive(full + slot); break; }   // no more tiles: wake the consumers
                    }
                    int comp;
                    const CUtensorMap *m = slab_map(mp, j, comp);
                    mbar_expect_tx(full + slot, L::SLAB);
                    tma_load_3d(ring + slot * L::SLAB, m, 8 * t, 0, comp, full + slot);
                }
                if (t >= ntiles) break;
            }
        }
    } else if (!failed) {
        // ---------------- consumers: warp w solves line 4 t + w ----------------
        const int w = warp;
        const LineTw<R> tw{{tws, NX, 1, st}, lcs, ltr};
        const double dx = g.dx, dx2 = g.dx2, dt = sc->dt, vis = g.vis;
        const double c1 = g.c1, c2 = g.c2, c3 = g.c3, c4 = g.c4;
        const double c12 = c1 + c2, rdx = 1.0 / dx, rdx2 = 1.0 / dx2, rc12 = 1.0 / c12;
        double2 *row = reinterpret_cast<double2 *>(sm + L::O_ROW) + w * NX;   // this warp's scratch row
        bool ok = true;
        uint32_t k = 0;
        auto next_slab = [&](bool wait_done) -> unsigned char * {
            const int slot = k % KR;
            if (!wait_done && !mbar_wait(full + slot, (k / KR) & 1)) atomicCAS(&sc->status, 0, PIBM_ERR_TIMEOUT);
            return ring + slot * L::SLAB;
        };
        auto release = [&]() {
            __syncwarp();
            if (lane == 0) mbar_arrive(empty + (k % KR));
            ++k;
        };
        for (int c = 0;; ++c) {
            if (!mbar_wait(full + (k % KR), (k / KR) & 1)) atomicCAS(&sc->status, 0, PIBM_ERR_TIMEOUT);
            const int t = tid_ring[c & 1];
            // the previous tile's stores have read the work tiles, which this tile overwrites
            if (threadIdx.x == 0) bulk_wait_read();
            // one decision for the four warps (they meet at the tile's named barriers)
            if (!named_bar_and(1, L::LT * 32, t >= 0)) break;
            const int q = t * L::LT + w;
            const double ky = g.ky[q % g.my2], kz = g.kz[q / g.my2], w2w = g.w2[q];
            const LineCoef kw = line_coef(dt, vis, c1, c2, dx2, w2w);
            // ---- pressure source (poisson.F90:97-116) in registers; explicit ustep
            // parts (usteptime.F90:291-297) in the u tiles until each component's solve
            double2 tt[R];
#pragma unroll
            for (int r = 0; r < R; ++r) tt[r] = make_double2(0.0, 0.0);
#pragma unroll 1
            for (int j = 0; j < 9; ++j) {
                unsigned char *S = next_slab(j == 0);
                const int n = j < 6 ? (j >> 1) : j - 6, kind = j < 6 ? (j & 1) : 2;   // kind: 0 nl, 1 ff, 2 onl
                const double cf = kind == 0 ? c3 : (kind == 1 ? 1.0 : c4);
                unsigned char *E = Ut + n * L::SLAB;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = lane + 32 * r, ip = i == NX - 1 ? 0 : i + 1;
                    const double2 x0 = tel(S, i, w), x1 = tel(S, ip, w);
                    tt[r] = cadd_rn(tt[r], psrc_term_rt(n, kind != 1, cf, x0, x1, ky, kz, dx, rdx));
                    double2 &e = tel(E, i, w);
                    if (kind == 0) e = cscale_rn(x0, dt * c3);
                    else e = cadd_rn(e, cscale_rn(x0, kind == 1 ? dt : dt * c4));
                }
                release();
            }
            // ---- pressure (poisson.F90:118-239): old p, solve, p = p + (phi - p)
            double2 po[R], v[R];
            {
                unsigned char *S = next_slab(false);
#pragma unroll
                for (int r = 0; r < R; ++r) po[r] = tel(S, lane + 32 * r, w);
                release();
            }
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = make_double2(qdiv(tt[r].x, c12, rc12), qdiv(tt[r].y, c12, rc12));
            if (q == 0) {
#pragma unroll
                for (int r = 0; r < R; ++r) row[lane + 32 * r] = v[r];
                __syncwarp();
                if (lane == 0) ok = thomas_real(row, gam, kw.pa, kw.pb, kw.pc, NX - 1) && ok;
                __syncwarp();
#pragma unroll
                for (int r = 0; r < R; ++r) v[r] = row[lane + 32 * r];
            } else {
                circulant_solve_reg<R>(v, kw.pa, kw.pb, tw, lane);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) tel(Pt, lane + 32 * r, w) = p_update(po[r], v[r]);
            __syncwarp();
            // ---- ustep per component (usteptime.F90:73-470)
#pragma unroll 1
            for (int n = 0; n < 3; ++n) {
                unsigned char *S = next_slab(false);
                unsigned char *U = Ut + n * L::SLAB;
                double2 rr[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = lane + 32 * r, im = i == 0 ? NX - 1 : i - 1, ip = i == NX - 1 ? 0 : i + 1;
                    rr[r] = ustep_rhs(n, kw, tel(S, i, w), tel(S, im, w), tel(S, ip, w), tel(U, i, w), tel(Pt, im, w), tel(Pt, i, w), i == 0, ky,
                                      kz, dx, rdx, dx2, rdx2);
                }
                release();
                circulant_solve_reg<R>(rr, kw.ua, kw.ub, tw, lane);
#pragma unroll
                for (int r = 0; r < R; ++r) tel(U, lane + 32 * r, w) = rr[r];
            }
            __syncwarp();
            unsigned char *U1 = Ut, *U2 = Ut + L::SLAB, *U3 = Ut + 2 * L::SLAB;
            // ---- divcorr (poisson.F90:241-508)
            const double ralpc = 1.0 / kw.alp;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r, ip = i == NX - 1 ? 0 : i + 1;
                const double2 t2 = div_term(tel(U1, i, w), tel(U1, ip, w), tel(U2, i, w), tel(U2, ip, w), tel(U3, i, w), tel(U3, ip, w), ky, kz,
                                            dx, rdx);
                v[r] = make_double2(qdiv(t2.x, kw.alp, ralpc), qdiv(t2.y, kw.alp, ralpc));
            }
            if (q == 0) {
#pragma unroll
                for (int r = 0; r < R; ++r) row[lane + 32 * r] = v[r];
                __syncwarp();
                if (lane == 0) ok = thomas_real(row, gam, kw.pa, kw.pb, kw.pc, NX - 1) && ok;
                __syncwarp();
            } else {
                circulant_solve_reg<R>(v, kw.pa, kw.pb, tw, lane);
#pragma unroll
                for (int r = 0; r < R; ++r) row[lane + 32 * r] = v[r];
                __syncwarp();
            }
            {
                double2 nu1[R], nu2[R], nu3[R], np[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = lane + 32 * r;
                    const int im = i == 0 ? NX - 1 : i - 1, ip = i == NX - 1 ? 0 : i + 1;
                    divcorr_update(kw, row[i], row[im], row[ip], i == 0, tel(U1, i, w), tel(U2, i, w), tel(U3, i, w), tel(Pt, i, w), ky, kz, w2w,
                                   dx, rdx, dx2, rdx2, nu1[r], nu2[r], nu3[r], np[r]);
                }
                __syncwarp();
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = lane + 32 * r;
                    tel(U1, i, w) = nu1[r]; tel(U2, i, w) = nu2[r]; tel(U3, i, w) = nu3[r]; tel(Pt, i, w) = np[r];
                }
                __syncwarp();
            }
            // check_divergence for this line
            double dmax = 0.0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r, ip = i == NX - 1 ? 0 : i + 1;
                dmax = fmax(dmax, cabs_rn(div_term(tel(U1, i, w), tel(U1, ip, w), tel(U2, i, w), tel(U2, ip, w), tel(U3, i, w), tel(U3, ip, w),
                                                   ky, kz, dx, rdx)));
            }
            for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
            if (lane == 0) atomicMax(&sc->divmax_bits, (unsigned long long)__double_as_longlong(dmax));
            // ---- the tile's u and p leave through tensor-map stores
            fence_async_smem();
            named_bar_sync(1, L::LT * 32);
            if (threadIdx.x == 0) {
#pragma unroll
                for (int n = 0; n < 3; ++n) tma_store_3d(&mp.u, Ut + n * L::SLAB, 8 * t, 0, n);
                tma_store_3d(&mp.p, Pt, 8 * t, 0, 0);
                bulk_commit();
            }
        }
        if (!ok) atomicCAS(&sc->status, 0, PIBM_ERR_PIVOT);
        if (threadIdx.x == 0) bulk_wait_all();
    }
    // the last block to finish resets the tickets for the next launch
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&sc->lines_done, 1u) == gridDim.x - 1) {
            atomicExch(&sc->lines_next, 0u);
            atomicExch(&sc->lines_done, 0u);
        }
    }
}

template <int NX>
__global__ void __launch_bounds__(LPipe<NX>::T, LPipe<NX>::MINB) k_lines_pipe(const Geo g, const __grid_constant__ LineMaps mp,
                                                                              Scal *__restrict__ sc) {
    lines_pipe_body<NX>(g, mp, sc);
}

}  // namespace pibm
