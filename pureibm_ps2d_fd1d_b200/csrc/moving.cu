// moving.cu -- moving particles (IMOVE = 1): the soft-sphere DEM of
// des_time_march (SRC/FLO/collision_mod.F90, soft_sphere_coll.F90) and the
// per-step rebuild of the immersed-boundary geometry that bcset does after it
// (grid_nodes_insphere, update_nrpr_array: dependent_functions.F90:783-1051).
//
// Compiled with --fmad=false: every expression is evaluated with the
// reference's operation order and no contraction, so positions, cell
// indices, contact and neighbour lists and the solid mask come out bit-equal
// to a serial evaluation of the same expressions.
//
// The reference keeps the contact lists with one sequential loop over the
// particles.  Here each sub-step is three launches:
//   k_dem_update  one thread per particle L: every pair (J, L) is evaluated by
//                 both its threads with the same arithmetic; L applies what the
//                 serial loop does to L's list at J's turn (J < L), then at
//                 its own turn (compaction, own pairs), forms FC(L) in the
//                 serial order (lower partners ascending, then its own pairs in
//                 NEIGHBOURS order) and advances L (CFNEWVALUES)
//   k_dem_bin     one CTA: particles per coarse cell, ascending
//   k_dem_search  one warp per particle: GRID_BASED_NEIGHBOR_SEARCH's list of L
//                 (entries appended by lower particles' searches, L itself,
//                 L's own finds in cell-scan order), then CFUPDATEOLD
// What makes this exact: within a sub-step the reference changes L's entries
// for a partner P > L only at L's own turn and its entries for P < L only at
// P's turn, so every decision reads lists as they were at the sub-step start.
#include <cuda_runtime.h>
#include <stdint.h>

#include "step_common.cuh"

namespace pibm {

namespace {

constexpr double kPiD = 3.14159265358979323846;

// One contact pair as CALC_FORCE_DES evaluates it at LL = A's turn, I = B
// (soft_sphere_coll.F90:300-420, CFRELVEL :728-776): periodic unwrap of B,
// overlap test, normal spring-dashpot force on A.  Reads the sub-step's
// starting positions and velocities.
__device__ bool pair_force(const Mov &m, int A, int B, double fn[3], Scal *sc) {
    const double L3[3] = {m.XL, m.YL, m.ZL};
    double pB[3], dist[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double a = m.pos_old[3 * A + d], b = m.pos_old[3 * B + d];
        pB[d] = b;
        if (fabs(a - b) > 4.0 * m.max_radius) pB[d] = b > a ? b - L3[d] : b + L3[d];
        dist[d] = pB[d] - a;
    }
    double dd = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) dd = dd + dist[d] * dist[d];
    const double rlm = m.rad + m.rad;
    const double distmod = sqrt(dd);
    if (!(rlm - distmod > kSmallD)) return false;
    if (distmod == 0.0) { atomicCAS(&sc->status, 0, PIBM_ERR_DEM_MOVE); return false; }
    double nrm[3], vrel[3], osum[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        nrm[d] = dist[d] / distmod;
        vrel[d] = m.vel_old[3 * A + d] - m.vel_old[3 * B + d];
        osum[d] = 0.0 * m.rad + 0.0 * m.rad;   // OMEGA stays zero (rotation update disabled)
    }
    const double vrot[3] = {osum[1] * nrm[2] - osum[2] * nrm[1], osum[2] * nrm[0] - osum[0] * nrm[2],
                            osum[0] * nrm[1] - osum[1] * nrm[0]};
    double vrn = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) { vrel[d] = vrel[d] + vrot[d]; vrn = vrn + vrel[d] * nrm[d]; }
    const double ov_n = rlm - distmod;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double fns1 = -(m.kn * ov_n) * nrm[d];
        const double fns2 = -(m.eta_n * vrn) * nrm[d];
        fn[d] = fns1 + fns2;
    }
    return true;
}

// Sub-step count of this flow step (des_time_march :272-279) and the reset of
// the geometry counters rebuilt after the DEM.
__global__ void k_dem_start(Mov m, Scal *sc) {
    if (threadIdx.x != 0) return;
    sc->count_solid = 0;
    if (sc->status) return;
    const double dt = sc->dt;
    int factor = 1;
    double dts = dt;
    if (m.soft) {
        factor = (int)(dt / m.dtsolid);
        dts = m.dtsolid;
        if (factor < 1) { factor = 1; dts = dt; }
    }
    if (factor > m.max_factor) { sc->status = PIBM_ERR_ARG; factor = 0; }
    m.factor[0] = factor;
    m.dts[0] = dts;
    sc->dem_substeps = factor;
}

// CALC_FORCE_DES + CFNEWVALUES for particle L (see the file comment), one warp
// per particle: the lanes evaluate L's pairs (every entry of NEIGHBOURS(L)
// other than L), lane 0 then applies them in the serial order.
constexpr int kUpdWarps = 4;
constexpr int kMaxList = 40;   // >= MAXNEIGHBORS
__global__ void __launch_bounds__(32 * kUpdWarps) k_dem_update(Mov m, Scal *sc, const double *__restrict__ pres,
                                                               const double *__restrict__ visc, int ifac) {
    if (ifac > m.factor[0] || sc->status) return;
    __shared__ double fn_s[kUpdWarps][kMaxList][3];
    __shared__ int cf_s[kUpdWarps][kMaxList], wl_s[kUpdWarps][kMaxList], wv_s[kUpdWarps][kMaxList];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int L = blockIdx.x * kUpdWarps + wid;
    if (L >= m.N) return;
    const int MX = m.maxn, nc = m.ncnt[L];
    // pair (J, L) for J < L as at J's turn (flag bit 0 contact, bit 1 "already
    // in J's contact list"), pair (L, I) for I > L as at L's turn
    for (int q = lane; q < nc; q += 32) {
        const int P = m.neigh[L * MX + q];
        int f = 0;
        double fn[3] = {0.0, 0.0, 0.0};
        if (P < L) {
            if (pair_force(m, P, L, fn, sc)) {
                f = 1;
                for (int p = 0; p < m.pncnt[P]; ++p)
                    if (m.pn[P * MX + p] == L) { if (m.pv[P * MX + p] == 1) f |= 2; break; }
            }
        } else if (P > L) {
            if (pair_force(m, L, P, fn, sc)) f = 1;
        }
        cf_s[wid][q] = f;
#pragma unroll
        for (int d = 0; d < 3; ++d) fn_s[wid][q][d] = fn[d];
    }
    __syncwarp();
    if (lane != 0) return;
    int *wl = wl_s[wid], *wv = wv_s[wid];
    int wc = m.pncnt[L];
    for (int q = 0; q < wc; ++q) { wl[q] = m.pn[L * MX + q]; wv[q] = m.pv[L * MX + q]; }
    double fc[3] = {0.0, 0.0, 0.0};
    bool over = false;
    // turns of the lower partners J (ascending: they precede L in NEIGHBOURS(L))
    for (int q = 0; q < nc; ++q) {
        const int J = m.neigh[L * MX + q];
        if (J >= L || !(cf_s[wid][q] & 1)) continue;
        if (cf_s[wid][q] & 2) {
            for (int p = 0; p < wc; ++p) if (wl[p] == J) { wv[p] = 1; break; }
        } else if (wc + 1 < MX) {
            wl[wc] = J; wv[wc] = 1; ++wc;
        } else {
            over = true;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) fc[d] = fc[d] - fn_s[wid][q][d];
    }
    // L's turn: drop the entries whose contact ended, clear the flags, own pairs
    int w = 0;
    for (int p = 0; p < wc; ++p) if (wv[p]) { wl[w] = wl[p]; ++w; }
    wc = w;
    for (int p = 0; p < wc; ++p) wv[p] = 0;
    for (int q = 0; q < nc; ++q) {
        const int I = m.neigh[L * MX + q];
        if (I <= L || !(cf_s[wid][q] & 1)) continue;
        int found = -1;
        for (int p = 0; p < wc; ++p) if (wl[p] == I) { found = p; break; }
        if (found >= 0) {
            wv[found] = 1;
        } else if (wc + 1 < MX) {
            wl[wc] = I; wv[wc] = 1; ++wc;
        } else {
            over = true;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) fc[d] = fc[d] + fn_s[wid][q][d];
    }
    if (over) atomicCAS(&sc->status, 0, PIBM_ERR_NEIGH_OVERFLOW);
    m.pncnt2[L] = wc;
    for (int p = 0; p < wc; ++p) { m.pn2[L * MX + p] = wl[p]; m.pv2[L * MX + p] = wv[p]; }
    // CFNEWVALUES (collision_mod.F90:1335-1462), softsphere coupled to the flow
    const double dts = m.dts[0];
    const int N = m.N;
    double pn[3], dd = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const size_t q = (size_t)L + (size_t)N * d;
        double a = fc[d] / m.pmass + (m.rhof * (pres[q] + visc[q])) / m.pmass;
        a = a - sc->frame_accln[d];
        a = a - (sc->mpg[d] * m.pvol) / m.pmass;
        const double v = m.vel_old[3 * L + d] + a * dts;
        m.vel[3 * L + d] = v;
        pn[d] = m.pos_old[3 * L + d] + v * dts;
        const double t = pn[d] - m.pos_old[3 * L + d];
        dd = dd + t * t;
    }
    if (sqrt(dd) >= m.rad) atomicCAS(&sc->status, 0, PIBM_ERR_DEM_MOVE);
    const double L3[3] = {m.XL, m.YL, m.ZL};
    const double dc[3] = {m.dxc, m.dyc, m.dzc};
    const int cmax[3] = {m.cx, m.cy, m.cz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (pn[d] > L3[d]) pn[d] = pn[d] - (L3[d] - 0.0);
        else if (pn[d] < 0.0) pn[d] = pn[d] + (L3[d] - 0.0);
        m.pos[3 * L + d] = pn[d];
        m.pijk[3 * L + d] = min((int)(pn[d] / dc[d]) + 2, cmax[d]);   // FIND_CELL_INDEX (:743-762)
    }
}

// 'none' collision type (des_time_march :295-328): velocities kept, positions
// advanced over dt; the neighbour lists are not rebuilt.
__global__ void k_dem_none(Mov m, Scal *sc) {
    const int L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= m.N || sc->status) return;
    const double dt = sc->dt;
    const double L3[3] = {m.XL, m.YL, m.ZL};
    double pn[3], dd = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double v = m.vel_old[3 * L + d];
        m.vel[3 * L + d] = v;
        pn[d] = m.pos_old[3 * L + d] + v * dt;
        const double t = pn[d] - m.pos_old[3 * L + d];
        dd = dd + t * t;
    }
    if (sqrt(dd) >= m.rad) atomicCAS(&sc->status, 0, PIBM_ERR_DEM_MOVE);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (pn[d] > L3[d]) pn[d] = pn[d] - (L3[d] - 0.0);
        else if (pn[d] < 0.0) pn[d] = pn[d] + (L3[d] - 0.0);
        m.pos[3 * L + d] = pn[d];
        m.pos_old[3 * L + d] = pn[d];
    }
}

__device__ __forceinline__ int cell_id(const Mov &m, int i, int j, int k) {
    return (i - 2) + (m.cx - 1) * ((j - 2) + (m.cy - 1) * (k - 2));
}

// PARTICLES_IN_CELL (collision_mod.F90:764-805): particles of every coarse
// cell in ascending order.  One CTA of 1024 threads; smem holds ncell counts,
// starts and fill counters and N particle slots.
__global__ void __launch_bounds__(1024) k_dem_bin(Mov m, Scal *sc, int ifac) {
    if (ifac > m.factor[0] || sc->status) return;
    extern __shared__ int sh[];
    int *cnt = sh, *start = sh + m.ncell, *fill = start + m.ncell + 1, *tmp = fill + m.ncell;
    __shared__ int wsum[32];
    const int T = blockDim.x, t = threadIdx.x, N = m.N, NC = m.ncell;
    for (int c = t; c < NC; c += T) { cnt[c] = 0; fill[c] = 0; }
    __syncthreads();
    for (int l = t; l < N; l += T) atomicAdd(&cnt[cell_id(m, m.pijk[3 * l], m.pijk[3 * l + 1], m.pijk[3 * l + 2])], 1);
    __syncthreads();
    // exclusive scan of cnt: each thread a contiguous chunk, then a block scan of the chunk sums
    const int per = (NC + T - 1) / T, c0 = min(t * per, NC), c1 = min(c0 + per, NC);
    int s = 0;
    for (int c = c0; c < c1; ++c) s += cnt[c];
    int x = s;
    const int lane = t & 31, wid = t >> 5;
    for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int v = lane < (T >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, v, o); if (lane >= o) v += y; }
        wsum[lane] = v;
    }
    __syncthreads();
    int run = x - s + (wid > 0 ? wsum[wid - 1] : 0);
    for (int c = c0; c < c1; ++c) { start[c] = run; run += cnt[c]; }
    if (t == 0) start[NC] = N;
    __syncthreads();
    for (int l = t; l < N; l += T) {
        const int c = cell_id(m, m.pijk[3 * l], m.pijk[3 * l + 1], m.pijk[3 * l + 2]);
        tmp[start[c] + atomicAdd(&fill[c], 1)] = l;
    }
    __syncthreads();
    for (int l = t; l < N; l += T) {
        const int c = cell_id(m, m.pijk[3 * l], m.pijk[3 * l + 1], m.pijk[3 * l + 2]);
        int rank = 0;
        for (int e = start[c]; e < start[c + 1]; ++e) rank += tmp[e] < l ? 1 : 0;
        m.clist[start[c] + rank] = l;
    }
    for (int c = t; c <= NC; c += T) m.cstart[c] = start[c];
}

// Neighbourhood cell `o` (0..26, the reference's kk/jj/ii scan order) of a
// particle in cell (ci, cj, ck): wrapped cell and periodic image factors
// (collision_mod.F90:866-945).
__device__ __forceinline__ int nb_cell(const Mov &m, int ci, int cj, int ck, int o, double sh[3]) {
    int ii = ci + (o % 3) - 1, jj = cj + (o / 3) % 3 - 1, kk = ck + o / 9 - 1;
    sh[0] = sh[1] = sh[2] = 0.0;
    if (ii > m.cx) { ii = 2; sh[0] = 1.0; }
    if (ii < 2) { ii = m.cx; sh[0] = -1.0; }
    if (jj > m.cy) { jj = 2; sh[1] = 1.0; }
    if (jj < 2) { jj = m.cy; sh[1] = -1.0; }
    if (kk > m.cz) { kk = 2; sh[2] = 1.0; }
    if (kk < 2) { kk = m.cz; sh[2] = -1.0; }
    return cell_id(m, ii, jj, kk);
}
// The search's distance test of PNO seen from LL through image sh.
__device__ __forceinline__ bool near_img(const Mov &m, int LL, int PNO, const double sh[3]) {
    const double rlm = 1.2 * (m.rad + m.rad);
    const double c0 = m.pos[3 * PNO + 0] + sh[0] * m.LXs;
    const double c1 = m.pos[3 * PNO + 1] + sh[1] * m.LYs;
    const double c2 = m.pos[3 * PNO + 2] + sh[2] * m.LZs;
    const double d0 = c0 - m.pos[3 * LL + 0], d1 = c1 - m.pos[3 * LL + 1], d2 = c2 - m.pos[3 * LL + 2];
    double dd = 0.0;
    dd = dd + d0 * d0;
    dd = dd + d1 * d1;
    dd = dd + d2 * d2;
    return rlm - sqrt(dd) > kSmallD;
}

// The image factor through which a search from cell cJ sees cell cL along one
// direction when the coarse grid has at least 3 cells there (then exactly one
// of the offsets -1, 0, +1 wraps onto cL).
__device__ __forceinline__ double img_dir(int cJ, int cL, int cmax) {
    if (cJ - 1 >= 2 && cJ - 1 == cL) return 0.0;
    if (cJ + 1 <= cmax && cJ + 1 == cL) return 0.0;
    if (cJ == cL) return 0.0;
    return cJ + 1 > cmax ? 1.0 : -1.0;   // the wrapped neighbour: across the upper or the lower boundary
}

// GRID_BASED_NEIGHBOR_SEARCH (collision_mod.F90:807-1062) for one particle per
// warp, then CFUPDATEOLD and the contact lists of the next sub-step.
//  - coarse grids with >= 3 cells per direction: the 27 neighbourhood cells
//    are distinct, so lane o < 27 scans cell o; finds are placed by a prefix
//    sum over the lanes, which keeps the reference's cell-scan order
//  - smaller grids (cells repeat through the periodic wrap): lane 0 follows
//    the serial loop, first accepted image of a particle only
constexpr int kSearchWarps = 4;
__global__ void __launch_bounds__(32 * kSearchWarps) k_dem_search(Mov m, Scal *sc, int ifac) {
    if (ifac > m.factor[0] || sc->status) return;
    __shared__ int own_s[kSearchWarps][64], mir_s[kSearchWarps][64];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int L = blockIdx.x * kSearchWarps + wid;
    if (L >= m.N) return;
    const int MX = m.maxn;
    int *own = own_s[wid], *mir = mir_s[wid];
    const int ci = m.pijk[3 * L], cj = m.pijk[3 * L + 1], ck = m.pijk[3 * L + 2];
    const int cL = cell_id(m, ci, cj, ck);
    int nown = 0, nmir = 0;
    const bool fast = m.cx >= 4 && m.cy >= 4 && m.cz >= 4;
    if (fast) {
        double sh[3] = {0.0, 0.0, 0.0};
        int c = 0, s0 = 0, s1 = 0;
        if (lane < 27) { c = nb_cell(m, ci, cj, ck, lane, sh); s0 = m.cstart[c]; s1 = m.cstart[c + 1]; }
        // own finds P > L of this lane's cell
        int cnt = 0;
        for (int e = s0; e < s1; ++e) { const int P = m.clist[e]; if (P > L && near_img(m, L, P, sh)) ++cnt; }
        int x = cnt;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        nown = __shfl_sync(0xffffffffu, x, 31);
        int pos = x - cnt;
        for (int e = s0; e < s1; ++e) {
            const int P = m.clist[e];
            if (P > L && near_img(m, L, P, sh)) { if (pos < 64) own[pos] = P; ++pos; }
        }
        // lower particles J whose search accepts L: J sees cell cL through one image
        cnt = 0;
        for (int e = s0; e < s1; ++e) {
            const int J = m.clist[e];
            if (J >= L) continue;
            const double shj[3] = {img_dir(m.pijk[3 * J], ci, m.cx), img_dir(m.pijk[3 * J + 1], cj, m.cy),
                                   img_dir(m.pijk[3 * J + 2], ck, m.cz)};
            if (near_img(m, J, L, shj)) ++cnt;
        }
        x = cnt;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        nmir = __shfl_sync(0xffffffffu, x, 31);
        pos = x - cnt;
        for (int e = s0; e < s1; ++e) {
            const int J = m.clist[e];
            if (J >= L) continue;
            const double shj[3] = {img_dir(m.pijk[3 * J], ci, m.cx), img_dir(m.pijk[3 * J + 1], cj, m.cy),
                                   img_dir(m.pijk[3 * J + 2], ck, m.cz)};
            if (near_img(m, J, L, shj)) { if (pos < 64) mir[pos] = J; ++pos; }
        }
        __syncwarp();
    } else if (lane == 0) {
        for (int o = 0; o < 27; ++o) {
            double sh[3];
            const int c = nb_cell(m, ci, cj, ck, o, sh);
            for (int e = m.cstart[c]; e < m.cstart[c + 1]; ++e) {
                const int P = m.clist[e];
                if (P <= L || !near_img(m, L, P, sh)) continue;
                bool already = false;
                for (int q = 0; q < nown && q < 64; ++q) if (own[q] == P) { already = true; break; }
                if (!already) { if (nown < 64) own[nown] = P; ++nown; }
            }
        }
        for (int o = 0; o < 27; ++o) {
            double sh[3];
            const int c = nb_cell(m, ci, cj, ck, o, sh);
            bool seen = false;
            for (int o2 = 0; o2 < o; ++o2) { double t[3]; if (nb_cell(m, ci, cj, ck, o2, t) == c) { seen = true; break; } }
            if (seen) continue;
            for (int e = m.cstart[c]; e < m.cstart[c + 1]; ++e) {
                const int J = m.clist[e];
                if (J >= L) continue;
                const int ji = m.pijk[3 * J], jj = m.pijk[3 * J + 1], jk = m.pijk[3 * J + 2];
                bool acc = false;
                for (int oj = 0; oj < 27 && !acc; ++oj) {
                    double shj[3];
                    if (nb_cell(m, ji, jj, jk, oj, shj) == cL && near_img(m, J, L, shj)) acc = true;
                }
                if (acc) { if (nmir < 64) mir[nmir] = J; ++nmir; }
            }
        }
    }
    if (!fast) {   // counts of the serial path are in lane 0
        nown = __shfl_sync(0xffffffffu, nown, 0);
        nmir = __shfl_sync(0xffffffffu, nmir, 0);
    }
    __syncwarp();
    const bool over = nmir > 64 || nown > 64 || nmir + 1 + nown + 1 > MX;
    if (lane == 0 && !over) {
        for (int a = 1; a < nmir; ++a) {   // ascending J
            const int v = mir[a];
            int b = a - 1;
            while (b >= 0 && mir[b] > v) { mir[b + 1] = mir[b]; --b; }
            mir[b + 1] = v;
        }
    }
    __syncwarp();
    if (over) {
        if (lane == 0) atomicCAS(&sc->status, 0, PIBM_ERR_NEIGH_OVERFLOW);
        return;
    }
    const int tot = nmir + 1 + nown;
    for (int q = lane; q < tot; q += 32)
        m.neigh[L * MX + q] = q < nmir ? mir[q] : (q == nmir ? L : own[q - nmir - 1]);
    if (lane == 0) m.ncnt[L] = tot;
    // CFUPDATEOLD and the contact lists written by this sub-step
    if (lane < 3) { m.pos_old[3 * L + lane] = m.pos[3 * L + lane]; m.vel_old[3 * L + lane] = m.vel[3 * L + lane]; }
    const int pc = m.pncnt2[L];
    for (int q = lane; q < pc; q += 32) { m.pn[L * MX + q] = m.pn2[L * MX + q]; m.pv[L * MX + q] = m.pv2[L * MX + q]; }
    if (lane == 0) m.pncnt[L] = pc;
}

// IBMUPDATE (collision_mod.F90:1464-1474): grid-unit centres and velocities.
__global__ void k_dem_ibm(Mov m, Scal *sc, double dx) {
    const int L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= m.N || sc->status) return;
    const int N = m.N;
    m.xc[L] = m.pos[3 * L + 0] / dx + 1.0 - 0.0;
    m.xc[L + N] = m.pos[3 * L + 1] / dx + 1.0;
    m.xc[L + 2 * N] = m.pos[3 * L + 2] / dx + 1.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) m.vel_ibm[L + (size_t)N * d] = m.vel[3 * L + d];
}

// grid_nodes_insphere (dependent_functions.F90:783-963): one CTA per sphere
// clears the nodes of its bounding box that lie in the sphere (nodes covered
// by two spheres are counted twice, as in the reference).
template <int N>
__global__ void __launch_bounds__(256) k_mask(Geo g, Mov m, Scal *sc) {
    __shared__ double scr[32];
    if (block_failed(sc)) return;
    const int s = blockIdx.x, NB = g.nbody, nx = g.nx;
    const double cx = m.xc[s], cy = m.xc[s + NB], cz = m.xc[s + 2 * NB], r = g.rb;
    const int i0 = (int)ceil(cx - r), i1 = (int)floor(cx + r);
    const int j0 = (int)ceil(cy - r), j1 = (int)floor(cy + r);
    const int k0 = (int)ceil(cz - r), k1 = (int)floor(cz + r);
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
    double cnt = 0.0;
    for (int e = threadIdx.x; e < ni * nj * nk; e += blockDim.x) {
        const int k = k0 + e / (ni * nj), j = j0 + (e / ni) % nj, i = i0 + e % ni;
        const double a = (double)i - cx, b = (double)j - cy, c = (double)k - cz;
        double d2 = a * a;
        d2 = d2 + b * b + c * c;
        if (sqrt(d2) - r <= kSmallD) {
            const int ii = wrapi(i, nx), jj = wrapi(j, N), kk = wrapi(k, N);
            m.fluid[(size_t)(ii - 1) * RP<N>::RSP + real_off<N>(kk - 1, jj - 1)] = 0;
            cnt += 1.0;
        }
    }
    cnt = block_sum(cnt, scr);
    if (threadIdx.x == 0) atomicAdd((unsigned long long *)&sc->count_solid, (unsigned long long)cnt);
}

// update_nrpr_array + check_external_pt (dependent_functions.F90:966-1051):
// one CTA per sphere flags its reversal points whose outer point lies in a
// neighbour sphere, counts the active ones and sets da(2) of bcset.
__global__ void __launch_bounds__(256) k_nrpr(Geo g, Mov m, Scal *sc) {
    __shared__ double scr[32];
    if (block_failed(sc)) return;
    const int s = blockIdx.x, NB = g.nbody, nb = g.nbnd;
    const double px = (double)(g.nx + 1), py = (double)g.my, pz = (double)g.mz;
    const int nc = m.ncnt[s];
    double act = 0.0;
    for (int l = threadIdx.x; l < nb; l += blockDim.x) {
        double xo[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) xo[d] = m.xc[s + d * NB] + g.bnd[3 * l + d] * g.ro;
        if (xo[0] < 1.0) xo[0] = px + xo[0];
        if (xo[0] > px) xo[0] = xo[0] - px;
        if (xo[1] < 1.0) xo[1] = py + 1.0 + xo[1];
        if (xo[1] > py) xo[1] = xo[1] - py - 1.0;
        if (xo[2] < 1.0) xo[2] = pz + 1.0 + xo[2];
        if (xo[2] > pz) xo[2] = xo[2] - pz - 1.0;
        bool active = true;
        if (nc > 1) {
            for (int q = 0; q < nc; ++q) {
                const int P = m.neigh[s * m.maxn + q];
                double d2 = 0.0;
#pragma unroll
                for (int d = 0; d < 3; ++d) { const double a = m.xc[P + d * NB] - xo[d]; d2 = d2 + a * a; }
                if (sqrt(d2) < g.rb) { active = false; break; }
            }
        }
        m.revflag[(size_t)s * nb + l] = active ? 1 : 0;
        act += active ? 1.0 : 0.0;
    }
    act = block_sum(act, scr);
    if (threadIdx.x == 0) {
        const int n = (int)act;
        m.nrpr[s] = n;
        m.da2[s] = 4.0 * kPiD * ((g.ri * g.dx) * (g.ri * g.dx)) / (double)n;
    }
}

// Offsets of every sphere's active points in the (sphere, point) list, the
// point count, and the solid/fluid counts of the new mask.
__global__ void __launch_bounds__(1024) k_pts_scan(Geo g, Mov m, Scal *sc) {
    __shared__ int wsum[32];
    if (block_failed(sc)) return;
    const int T = blockDim.x, t = threadIdx.x, NB = g.nbody;
    const int per = (NB + T - 1) / T, c0 = min(t * per, NB), c1 = min(c0 + per, NB);
    int s = 0;
    for (int c = c0; c < c1; ++c) s += m.nrpr[c];
    int x = s;
    const int lane = t & 31, wid = t >> 5;
    for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int v = lane < (T >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, v, o); if (lane >= o) v += y; }
        wsum[lane] = v;
    }
    __syncthreads();
    int run = x - s + (wid > 0 ? wsum[wid - 1] : 0);
    for (int c = c0; c < c1; ++c) { m.ptoff[c] = run; run += m.nrpr[c]; }
    if (t == T - 1) {
        sc->npts = run;
        sc->count_fluid = g.ncell - sc->count_solid;
        sc->maxvolfrac = (double)sc->count_solid / (double)g.ncell;
    }
}

// Active points of one sphere written in point order at its offset.
__global__ void __launch_bounds__(256) k_pts_write(Geo g, Mov m, Scal *sc) {
    __shared__ int wsum[8];
    __shared__ int base;
    if (block_failed(sc)) return;
    const int s = blockIdx.x, nb = g.nbnd, t = threadIdx.x, lane = t & 31, wid = t >> 5;
    if (t == 0) base = m.ptoff[s];
    __syncthreads();
    for (int l0 = 0; l0 < nb; l0 += blockDim.x) {
        const int l = l0 + t;
        const int f = l < nb ? m.revflag[(size_t)s * nb + l] : 0;
        const unsigned bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) wsum[wid] = __popc(bal);
        __syncthreads();
        int before = 0;
        for (int w = 0; w < wid; ++w) before += wsum[w];
        if (f) {
            const int p = base + before + __popc(bal & ((1u << lane) - 1u));
            m.pt_m[p] = s;
            m.pt_l[p] = l;
        }
        __syncthreads();
        if (t == 0) { int a = 0; for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += wsum[w]; base += a; }
        __syncthreads();
    }
}

// Spreading targets (boundary_condition.F90:1379-1462): every (point, corner)
// whose node receives force goes into that node's bucket.
template <int N>
__global__ void __launch_bounds__(256) k_sp_count(Geo g, Mov m, Scal *sc) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (sc->status || p >= sc->npts) return;
    const int s = m.pt_m[p], l = m.pt_l[p], NB = g.nbody;
    int base[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) base[d] = cell_of(m.xc[s + d * NB] + g.bnd[3 * l + d] * g.ri);
    for (int ck = 0; ck < 2; ++ck)
        for (int cj = 0; cj < 2; ++cj)
            for (int ci = 0; ci < 2; ++ci) {
                const int i = wrapi(base[0] + ci, g.nx), j = wrapi(base[1] + cj, N), k = wrapi(base[2] + ck, N);
                const size_t node = (size_t)(i - 1) * RP<N>::RSP + real_off<N>(k - 1, j - 1);
                if (!g.include_frmeanfluid && m.fluid[node]) continue;
                const int slot = atomicAdd(&m.spcnt[node], 1);
                if (slot < m.kmax) m.spbuf[node * m.kmax + slot] = p * 8 + ci + 2 * cj + 4 * ck;
                else atomicCAS(&sc->status, 0, PIBM_ERR_SPREAD_OVERFLOW);
            }
}

// A node's bucket in ascending entry order, the reference's accumulation
// order ((point, corner) or (evaluation, corner)): buckets of up to 8 entries
// (nearly all) through a 19-comparator sorting network in registers, longer
// ones by insertion sort.  f(entry) is called in that order.
template <class F>
__device__ __forceinline__ void bucket_in_order(const int *bucket, int c, F f) {
    if (c <= 8) {
        int v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = q < c ? bucket[q] : 0x7fffffff;
        auto ce = [&](int a, int b) { const int x = min(v[a], v[b]), y = max(v[a], v[b]); v[a] = x; v[b] = y; };
        ce(0, 1); ce(2, 3); ce(4, 5); ce(6, 7);
        ce(0, 2); ce(1, 3); ce(4, 6); ce(5, 7);
        ce(1, 2); ce(5, 6);
        ce(0, 4); ce(1, 5); ce(2, 6); ce(3, 7);
        ce(2, 4); ce(3, 5);
        ce(1, 2); ce(3, 4); ce(5, 6);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (q < c) f(v[q]);
    } else {
        int e[64];
        const int cc = min(c, 64);
        for (int q = 0; q < cc; ++q) {
            const int x = bucket[q];
            int b = q - 1;
            while (b >= 0 && e[b] > x) { e[b + 1] = e[b]; --b; }
            e[b + 1] = x;
        }
        for (int q = 0; q < cc; ++q) f(e[q]);
    }
}

// fr at every node: the bucket's contributions in ascending (point, corner)
// order, the reference's accumulation order; nodes without force get zero.
__global__ void __launch_bounds__(256) k_spread_dyn(Geo g, Mov m, const double *__restrict__ rec,
                                                    const double *__restrict__ rz, double *__restrict__ fr, Scal *sc) {
    const size_t node = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t CR = (size_t)g.nx * g.RS;
    if (node >= CR || sc->status) return;
    const double rdx3 = 1.0 / g.dx3;
    double acc[3] = {0.0, 0.0, 0.0};
    const int c = min(m.spcnt[node], m.kmax);
    if (c > 0)
        bucket_in_order(m.spbuf + node * m.kmax, c, [&](int ent) {
            double t[3];
            corner_contrib(rz, rec, ent, g.dx3, rdx3, t);
            if (g.include_frmeanfluid) {
#pragma unroll
                for (int n = 0; n < 3; ++n) acc[n] = acc[n] + t[n];
            } else {
                const double *r = rec + (size_t)(ent >> 3) * 6 + 3;
#pragma unroll
                for (int n = 0; n < 3; ++n) acc[n] = (acc[n] + t[n]) + r[n];
            }
        });
#pragma unroll
    for (int n = 0; n < 3; ++n) fr[n * CR + node] = acc[n];
}

// ---------------------------------------------------------------------------
// Passive scalar with moving particles: the reversal-point evaluations of
// calc_inner_rev_data (SRC/SCALAR/bc_scalar.F90:558-932, serial branch) for
// the step's active points.  Inner point x = xc + bnd*radibdy, its cell
// wrapped into 1..nx (WEST/EAST_PERIODIC_IMAGE, ibm.h:148-149); a point in
// cell nx is evaluated a second time one period west (EAST_PERIODIC_IMAGE_MOD,
// ibm.h:150).  Evaluations are ordered (sphere, point, evaluation).
// ---------------------------------------------------------------------------
struct ScalEval {
    double x[3];
    int c[3], nev;
};
__device__ __forceinline__ ScalEval scal_eval(const Geo &g, const Mov &m, int s, int l) {
    ScalEval e;
    const int NB = g.nbody, nx = g.nx, mxf = g.nx + 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        e.x[d] = m.xc[s + d * NB] + g.bnd[3 * l + d] * g.ri;
        e.c[d] = cell_of(e.x[d]);
    }
    int pct = e.c[0];
    double xlt = e.x[0];
    if (!(1 <= pct && pct <= nx)) {
        if (e.c[0] < 1) { pct = mxf + e.c[0] - 1; xlt = mxf + e.x[0] - 1; }
        else if (e.c[0] >= mxf) { pct = e.c[0] - (mxf - 1); xlt = e.x[0] - (mxf - 1); }
    }
    e.nev = pct == nx ? 2 : 1;
    e.c[0] = pct;
    e.x[0] = xlt;
    return e;
}

// Evaluations per sphere.
__global__ void __launch_bounds__(256) k_sev_count(Geo g, Mov m, Scal *sc) {
    __shared__ double scr[32];
    if (block_failed(sc)) return;
    const int s = blockIdx.x, nb = g.nbnd;
    double n = 0.0;
    for (int l = threadIdx.x; l < nb; l += blockDim.x)
        if (m.revflag[(size_t)s * nb + l]) n += (double)scal_eval(g, m, s, l).nev;
    n = block_sum(n, scr);
    if (threadIdx.x == 0) m.sev_cnt[s] = (int)n;
}

// Offsets of every sphere's evaluations and their total.
__global__ void __launch_bounds__(1024) k_sev_scan(Geo g, Mov m, Scal *sc) {
    __shared__ int wsum[32];
    if (block_failed(sc)) return;
    const int T = blockDim.x, t = threadIdx.x, NB = g.nbody;
    const int per = (NB + T - 1) / T, c0 = min(t * per, NB), c1 = min(c0 + per, NB);
    int s = 0;
    for (int c = c0; c < c1; ++c) s += m.sev_cnt[c];
    int x = s;
    const int lane = t & 31, wid = t >> 5;
    for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int v = lane < (T >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, v, o); if (lane >= o) v += y; }
        wsum[lane] = v;
    }
    __syncthreads();
    int run = x - s + (wid > 0 ? wsum[wid - 1] : 0);
    for (int c = c0; c < c1; ++c) { m.sev_off[c] = run; run += m.sev_cnt[c]; }
    if (t == T - 1) sc->nsev = run;
}

// One sphere's evaluations written in (point, evaluation) order at its offset.
__global__ void __launch_bounds__(256) k_sev_write(Geo g, Mov m, Scal *sc) {
    __shared__ int wsum[8];
    __shared__ int base;
    if (block_failed(sc)) return;
    const int s = blockIdx.x, nb = g.nbnd, t = threadIdx.x, lane = t & 31, wid = t >> 5, mxf = g.nx + 1;
    if (t == 0) base = m.sev_off[s];
    __syncthreads();
    for (int l0 = 0; l0 < nb; l0 += blockDim.x) {
        const int l = l0 + t;
        ScalEval e;
        int n = 0;
        if (l < nb && m.revflag[(size_t)s * nb + l]) { e = scal_eval(g, m, s, l); n = e.nev; }
        int x = n;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        int before = 0;
        for (int w = 0; w < wid; ++w) before += wsum[w];
        int q = base + before + x - n;
        for (int ev = 1; ev <= n; ++ev, ++q) {
            if (ev == 2 && e.c[0] >= mxf - 1) { e.c[0] = e.c[0] - (mxf - 1); e.x[0] = e.x[0] - (mxf - 1); }
            m.sev_m[q] = s;
            m.sev_l[q] = l;
#pragma unroll
            for (int d = 0; d < 3; ++d) { m.sev_x[3 * (size_t)q + d] = e.x[d]; m.sev_c[3 * (size_t)q + d] = e.c[d]; }
        }
        __syncthreads();
        if (t == 0) { int a = 0; for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += wsum[w]; base += a; }
        __syncthreads();
    }
}

// Scalar spreading targets: stencil corners on planes 1..nx (planes 0 and
// nx+1 are never transformed), solid nodes unless INCLUDE_FRMEANFLUID.
template <int N>
__global__ void __launch_bounds__(256) k_ssp_count(Geo g, Mov m, Scal *sc) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (sc->status || e >= sc->nsev) return;
    const int nx = g.nx, mxf = g.nx + 1;
    const int c0 = m.sev_c[3 * (size_t)e], c1 = m.sev_c[3 * (size_t)e + 1], c2 = m.sev_c[3 * (size_t)e + 2];
    for (int ck = 0; ck < 2; ++ck)
        for (int cj = 0; cj < 2; ++cj)
            for (int ci = 0; ci < 2; ++ci) {
                int i = c0 + ci;
                if (i < 0) i = mxf + i - 1;
                if (i < 1 || i > nx) continue;
                const int j = wrapi(c1 + cj, N), k = wrapi(c2 + ck, N);
                const size_t node = (size_t)(i - 1) * RP<N>::RSP + real_off<N>(k - 1, j - 1);
                if (!g.include_frmeanfluid && m.fluid[node]) continue;
                const int slot = atomicAdd(&m.sspcnt[node], 1);
                if (slot < m.kmax) m.sspbuf[node * m.kmax + slot] = e * 8 + ci + 2 * cj + 4 * ck;
                else atomicCAS(&sc->status, 0, PIBM_ERR_SPREAD_OVERFLOW);
            }
}

// Scalar forcing at every node of planes 1..nx in (evaluation, corner) order.
__global__ void __launch_bounds__(256) k_sspread_dyn(Geo g, Mov m, const double *__restrict__ sctb,
                                                     const double *__restrict__ sfd, double *__restrict__ sfr, Scal *sc) {
    const size_t node = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= (size_t)g.nx * g.RS || sc->status) return;
    double v = 0.0;
    const int c = min(m.sspcnt[node], m.kmax);
    if (c > 0)
        bucket_in_order(m.sspbuf + node * m.kmax, c, [&](int ent) {
            v = v + sctb[ent];
            if (!g.include_frmeanfluid) v = v + sfd[ent >> 3];
        });
    sfr[node] = v;
}

template <int N>
void enqueue_moving_scalar_t(const Geo &g, const Mov &m, Scal *sc, cudaStream_t s) {
    k_sev_count<<<g.nbody, 256, 0, s>>>(g, m, sc);
    k_sev_scan<<<1, 1024, 0, s>>>(g, m, sc);
    k_sev_write<<<g.nbody, 256, 0, s>>>(g, m, sc);
    cudaMemsetAsync(m.sspcnt, 0, (size_t)g.nx * RP<N>::RSP * sizeof(int), s);
    k_ssp_count<N><<<(g.nsev + 255) / 256, 256, 0, s>>>(g, m, sc);
}

template <int N>
void enqueue_moving_t(const Geo &g, const Mov &m, Scal *sc, const double *pres, const double *visc, cudaStream_t s) {
    const int pb = (m.N + 127) / 128;
    k_dem_start<<<1, 32, 0, s>>>(m, sc);
    if (m.soft) {
        const size_t bin_smem = (size_t)(3 * m.ncell + 1 + m.N) * sizeof(int);
        for (int ifac = 1; ifac <= m.max_factor; ++ifac) {
            k_dem_update<<<(m.N + kUpdWarps - 1) / kUpdWarps, 32 * kUpdWarps, 0, s>>>(m, sc, pres, visc, ifac);
            k_dem_bin<<<1, 1024, bin_smem, s>>>(m, sc, ifac);
            k_dem_search<<<(m.N + kSearchWarps - 1) / kSearchWarps, 32 * kSearchWarps, 0, s>>>(m, sc, ifac);
        }
    } else {
        k_dem_none<<<pb, 128, 0, s>>>(m, sc);
    }
    k_dem_ibm<<<pb, 128, 0, s>>>(m, sc, g.dx);
    cudaMemsetAsync(m.fluid, 1, (size_t)g.nx * RP<N>::RSP, s);
    cudaMemsetAsync(m.spcnt, 0, (size_t)g.nx * RP<N>::RSP * sizeof(int), s);
    k_mask<N><<<g.nbody, 256, 0, s>>>(g, m, sc);
    k_nrpr<<<g.nbody, 256, 0, s>>>(g, m, sc);
    k_pts_scan<<<1, 1024, 0, s>>>(g, m, sc);
    k_pts_write<<<g.nbody, 256, 0, s>>>(g, m, sc);
    k_sp_count<N><<<(g.npts + 255) / 256, 256, 0, s>>>(g, m, sc);
}

}  // namespace

// The DEM of one flow step and the geometry rebuild that follows it
// (bcset, boundary_condition.F90:539-554), enqueued after compute_mpg_at_n.
void enqueue_moving(const Geo &g, const Mov &m, Scal *sc, const double *pres, const double *visc, cudaStream_t s) {
    switch (g.my) {
        case 32: enqueue_moving_t<32>(g, m, sc, pres, visc, s); break;
        case 64: enqueue_moving_t<64>(g, m, sc, pres, visc, s); break;
        case 96: enqueue_moving_t<96>(g, m, sc, pres, visc, s); break;
        case 128: enqueue_moving_t<128>(g, m, sc, pres, visc, s); break;
        case 256: enqueue_moving_t<256>(g, m, sc, pres, visc, s); break;
    }
}
int moving_kernels_per_step(const Mov &m) { return 1 + (m.soft ? 3 * m.max_factor : 1) + 6; }

// Scalar geometry of the step (before calc_inner_rev_data) and its spreading.
void enqueue_moving_scalar(const Geo &g, const Mov &m, Scal *sc, cudaStream_t s) {
    switch (g.my) {
        case 32: enqueue_moving_scalar_t<32>(g, m, sc, s); break;
        case 64: enqueue_moving_scalar_t<64>(g, m, sc, s); break;
        case 96: enqueue_moving_scalar_t<96>(g, m, sc, s); break;
        case 128: enqueue_moving_scalar_t<128>(g, m, sc, s); break;
        case 256: enqueue_moving_scalar_t<256>(g, m, sc, s); break;
    }
}
void enqueue_sspread_dyn(const Geo &g, const Mov &m, const double *sctb, const double *sfd, double *sfr, Scal *sc, cudaStream_t s) {
    const size_t CR = (size_t)g.nx * g.RS;
    k_sspread_dyn<<<(unsigned)((CR + 255) / 256), 256, 0, s>>>(g, m, sctb, sfd, sfr, sc);
}
int moving_scalar_kernels_per_step() { return 4; }

void enqueue_spread_dyn(const Geo &g, const Mov &m, const double *rec, const double *rz, double *fr, Scal *sc, cudaStream_t s) {
    const size_t CR = (size_t)g.nx * g.RS;
    k_spread_dyn<<<(unsigned)((CR + 255) / 256), 256, 0, s>>>(g, m, rec, rz, fr, sc);
}

// Set-up: cells and the first neighbour search of des_time_march(.TRUE.)
// (initialize_flo.F90:631-639) on the uploaded positions.
void enqueue_dem_init(const Mov &m, Scal *sc, cudaStream_t s) {
    k_dem_start<<<1, 32, 0, s>>>(m, sc);   // also sets factor >= 1 for the two launches below
    const size_t bin_smem = (size_t)(3 * m.ncell + 1 + m.N) * sizeof(int);
    k_dem_bin<<<1, 1024, bin_smem, s>>>(m, sc, 1);
    k_dem_search<<<(m.N + kSearchWarps - 1) / kSearchWarps, 32 * kSearchWarps, 0, s>>>(m, sc, 1);
}

cudaError_t configure_moving_kernels(const Mov &m) {
    const int smem = (int)((size_t)(3 * m.ncell + 1 + m.N) * sizeof(int));
    return cudaFuncSetAttribute(k_dem_bin, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

}  // namespace pibm
