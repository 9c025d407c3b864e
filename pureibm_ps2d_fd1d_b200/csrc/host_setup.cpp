// host_setup.cpp -- run set-up for the engine (see host_setup.h).
#include "host_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace pibm {
int real_offset(int n, int z, int y);   // plane-transform order of a real node (kernels.cu)

namespace {
const double kSmall = (double)1.0E-35f;   // SMALL_NUMBER, a REAL(4) literal (constants.F90:92)
const double kLarge = (double)1.0E+32f;   // LARGE_NUMBER (constants.F90:93)
const double kPi = 3.14159265358979323846;
const double kTwoPi = 2.0 * kPi;

inline int trunc_int(double x) { return (int)x; }                  // Fortran INT
inline int cell_index(double x) { return x < 0.0 ? trunc_int(x - 1) : trunc_int(x); }   // boundary_condition.F90:1182-1198
}  // namespace

// Surface points of one octant mirrored into the whole sphere with outward
// unit normals: quadgener / generbnd / dcgen (geom_init.F90:44-242, 244-369, 573-586).
void surface_points(double r, double f2, std::vector<double> &bnd, std::vector<double> &cdv, int &nbnd) {
    struct P { double x, y, z; };
    std::vector<P> oct;
    const int ntheta = (int)std::lround(kTwoPi * r / 4.0 * f2);
    const double dtheta = kTwoPi / ntheta / 4.0;
    double theta = 0.0;
    for (int it = 0; it <= ntheta; ++it) {
        const int nphi = (int)std::lround(kTwoPi * r * std::sin(theta) / 4 * f2);
        const double dphi = kTwoPi / nphi / 4;   // nphi = 0 at the pole: one point, dphi unused
        double phi = 0.0;
        for (int ip = 0; ip <= nphi; ++ip) {
            P q;
            q.z = r * std::cos(theta) / r;
            q.y = r * std::sin(theta) * std::cos(phi) / r;
            q.x = r * std::sin(theta) * std::sin(phi) / r;
            if (std::fabs(q.z) < 1.0e-5) q.z = 0.0;
            if (std::fabs(q.y) < 1.0e-5) q.y = 0.0;
            if (std::fabs(q.x) < 1.0e-5) q.x = 0.0;
            oct.push_back(q);
            phi = phi + dphi;
        }
        theta = theta + dtheta;
    }
    // mirror images in the reference's order: identity, -x, -y, -z, -x-y, -x-z, -y-z, -x-y-z,
    // each image only for points whose mirrored coordinates are nonzero
    static const int sx[8] = {1, -1, 1, 1, -1, -1, 1, -1};
    static const int sy[8] = {1, 1, -1, 1, -1, 1, -1, -1};
    static const int sz[8] = {1, 1, 1, -1, 1, -1, -1, -1};
    bnd.clear(); cdv.clear();
    for (int im = 0; im < 8; ++im) {
        for (const P &q : oct) {
            if ((sx[im] < 0 && q.x == 0) || (sy[im] < 0 && q.y == 0) || (sz[im] < 0 && q.z == 0)) continue;
            const double a = sx[im] * q.x, b = sy[im] * q.y, c = sz[im] * q.z;
            const double len = std::sqrt(a * a + b * b + c * c);
            bnd.push_back(a); bnd.push_back(b); bnd.push_back(c);
            cdv.push_back(a / len); cdv.push_back(b / len); cdv.push_back(c / len);
        }
    }
    nbnd = (int)(bnd.size() / 3);
}

namespace {

// Solid mask and counts: grid_nodes_insphere (dependent_functions.F90:783-963).
// Nodes covered by two spheres are counted twice, as in the reference.
void build_mask(RunSetup &S) {
    const int nx = S.nx, my = S.my, mz = S.mz;
    S.fluid.assign((size_t)nx * my * mz, 1);
    long long solid = 0;
    for (int m = 0; m < S.nbody; ++m) {
        const double cx = S.xc[m], cy = S.xc[m + S.nbody], cz = S.xc[m + 2 * S.nbody];
        const double r = S.radbdy;
        const int i0 = (int)std::ceil(cx - r), i1 = (int)std::floor(cx + r);
        const int j0 = (int)std::ceil(cy - r), j1 = (int)std::floor(cy + r);
        const int k0 = (int)std::ceil(cz - r), k1 = (int)std::floor(cz + r);
        for (int i = i0; i <= i1; ++i) {
            const int ii = i < 1 ? i + nx : (i > nx ? i - nx : i);
            for (int j = j0; j <= j1; ++j) {
                const int jj = j < 1 ? j + my : (j > my ? j - my : j);
                for (int k = k0; k <= k1; ++k) {
                    const int kk = k < 1 ? k + mz : (k > mz ? k - mz : k);
                    const double a = (double)i - cx, b = (double)j - cy, c = (double)k - cz;
                    double d2 = a * a;
                    d2 = d2 + b * b + c * c;
                    if (std::sqrt(d2) - r <= kSmall) {
                        S.fluid[(size_t)(ii - 1) * my * mz + (size_t)(kk - 1) * my + (jj - 1)] = 0;
                        ++solid;
                    }
                }
            }
        }
    }
    S.count_solid = solid;
    S.count_fluid = (long long)nx * my * mz - solid;
    S.maxvolfrac = (double)S.count_solid / (double)((long long)nx * my * mz);
}

// Neighbour sets from the DEM coarse-grid search done at set-up
// (collision_mod.F90:346-499 grid, :743-805 binning, :807-1062 search).
void build_neighbours(RunSetup &S) {
    const int N = S.nbody;
    S.neighbours.assign(N, {});
    if (N == 0) return;
    for (int l = 0; l < N; ++l) S.neighbours[l].push_back(l);
    const double rphys = S.radbdy * S.dx;
    const double dxeff = 2.0 * S.radbdy * 1.5 * S.dx;
    int nc[3];
    double dc[3], len[3];
    for (int d = 0; d < 3; ++d) {
        nc[d] = std::max((int)std::lround(S.doml[d] / dxeff), 2);
        dc[d] = S.doml[d] / (double)(nc[d] - 1);
        // XE(1)=0, XE(i)=XE(i-1)+dxc; period = XE(cx) - XE(1)
        double e = 0.0;
        for (int i = 2; i <= nc[d]; ++i) e = e + dc[d];
        len[d] = e;
    }
    std::vector<double> pos(3 * (size_t)N);
    std::vector<int> cell(3 * (size_t)N);
    for (int l = 0; l < N; ++l)
        for (int d = 0; d < 3; ++d) {
            pos[3 * l + d] = (S.xc[l + (size_t)d * N] - 1.0) * S.dx;
            cell[3 * l + d] = std::min(trunc_int(pos[3 * l + d] / dc[d]) + 2, nc[d]);
        }
    // physical cells are 2..nc (nc-1 of them); bins in ascending particle order
    const int W = nc[0] + 2, H = nc[1] + 2;
    std::vector<std::vector<int>> bins((size_t)W * H * (nc[2] + 2));
    auto bin = [&](int i, int j, int k) -> std::vector<int> & { return bins[(size_t)i + (size_t)W * ((size_t)j + (size_t)H * k)]; };
    for (int l = 0; l < N; ++l) bin(cell[3 * l], cell[3 * l + 1], cell[3 * l + 2]).push_back(l);
    for (int L = 0; L < N; ++L) {
        for (int dk = -1; dk <= 1; ++dk)
            for (int dj = -1; dj <= 1; ++dj)
                for (int di = -1; di <= 1; ++di) {
                    int c[3] = {cell[3 * L] + di, cell[3 * L + 1] + dj, cell[3 * L + 2] + dk};
                    double shift[3] = {0, 0, 0};
                    for (int d = 0; d < 3; ++d) {
                        if (c[d] > nc[d]) { c[d] = 2; shift[d] = 1.0; }
                        if (c[d] < 2) { c[d] = nc[d]; shift[d] = -1.0; }
                    }
                    for (int P : bin(c[0], c[1], c[2])) {
                        if (P <= L) continue;
                        const double rlm = 1.2 * (rphys + rphys);
                        double d2 = 0.0;
                        double dd[3];
                        for (int d = 0; d < 3; ++d) dd[d] = (pos[3 * P + d] + shift[d] * len[d]) - pos[3 * L + d];
                        d2 = dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2];
                        const double dist = std::sqrt(d2);
                        std::vector<int> &nl = S.neighbours[L];
                        if (rlm - dist > kSmall && std::find(nl.begin() + 1, nl.end(), P) == nl.end()) {
                            nl.push_back(P);
                            S.neighbours[P].push_back(L);
                        }
                    }
                }
    }
}

// Active reversal points: update_nrpr_array + check_external_pt
// (dependent_functions.F90:966-1051), including its periodic-image offsets.
void build_if_rev(RunSetup &S) {
    const int N = S.nbody, nb = S.nbnd;
    S.if_rev.assign((size_t)nb * N, 1);
    S.nrpr_active.assign(N, nb);
    const double period_x = (double)(S.nx + 1), py = (double)S.my, pz = (double)S.mz;
    for (int m = 0; m < N; ++m) {
        const std::vector<int> &nl = S.neighbours[m];
        for (int l = 0; l < nb; ++l) {
            double xo[3];
            for (int d = 0; d < 3; ++d) xo[d] = S.xc[m + (size_t)d * N] + S.bnd[3 * l + d] * S.radobdy;
            if (xo[0] < 1.0) xo[0] = period_x + xo[0];
            if (xo[0] > period_x) xo[0] = xo[0] - period_x;
            if (xo[1] < 1.0) xo[1] = py + 1.0 + xo[1];
            if (xo[1] > py) xo[1] = xo[1] - py - 1.0;
            if (xo[2] < 1.0) xo[2] = pz + 1.0 + xo[2];
            if (xo[2] > pz) xo[2] = xo[2] - pz - 1.0;
            bool active = true;
            if (nl.size() > 1) {
                for (int P : nl) {
                    double s = 0.0;
                    for (int d = 0; d < 3; ++d) { const double a = S.xc[P + (size_t)d * N] - xo[d]; s = s + a * a; }
                    if (std::sqrt(s) < S.radbdy) { active = false; break; }
                }
            }
            if (!active) { S.if_rev[(size_t)l + (size_t)nb * m] = 0; S.nrpr_active[m] -= 1; }
        }
    }
}

// Spreading map for the inner reversal points (boundary_condition.F90:1379-1462):
// every node that receives force, with its contributing (point, corner) pairs in
// the reference's accumulation order.  With include_frmeanfluid=F only solid
// nodes receive force.
void build_spread_map(RunSetup &S, bool all_nodes, bool renumber) {
    const int N = S.nbody, nb = S.nbnd, nx = S.nx, my = S.my, mz = S.mz;
    S.pt_m.clear(); S.pt_l.clear();
    for (int m = 0; m < N; ++m)
        for (int l = 0; l < nb; ++l)
            if (S.if_rev[(size_t)l + (size_t)nb * m]) { S.pt_m.push_back(m); S.pt_l.push_back(l); }
    const int np = (int)S.pt_m.size();
    std::vector<std::pair<long long, int>> ent;   // (node, point*8+corner)
    ent.reserve((size_t)np * 8);
    for (int p = 0; p < np; ++p) {
        const int m = S.pt_m[p], l = S.pt_l[p];
        int base[3];
        for (int d = 0; d < 3; ++d) {
            const double x = S.xc[m + (size_t)d * N] + S.bnd[3 * l + d] * S.radibdy;
            base[d] = cell_index(x);
        }
        for (int ck = 0; ck < 2; ++ck)
            for (int cj = 0; cj < 2; ++cj)
                for (int ci = 0; ci < 2; ++ci) {
                    int i = base[0] + ci, j = base[1] + cj, k = base[2] + ck;
                    i = i < 1 ? i + nx : (i > nx ? i - nx : i);
                    j = j < 1 ? j + my : (j > my ? j - my : j);
                    k = k < 1 ? k + mz : (k > mz ? k - mz : k);
                    const long long node = (long long)(i - 1) * my * mz + (long long)(k - 1) * my + (j - 1);
                    if (!all_nodes && S.fluid[(size_t)node]) continue;
                    ent.push_back({node, p * 8 + ci + 2 * cj + 4 * ck});
                }
    }
    if (renumber && np > 1) {
        // Renumber the points in the memory order of their inner stencil's base
        // corner (x plane, then the plane-transform order of (z, y)), so that
        // the threads of a warp in the reversal-forcing kernel gather from
        // neighbouring sectors and its point records land near those of the
        // spreading gather.  Each node's contributions keep the reference's
        // (sphere, point, corner) order: only the indices change.
        const int rsp = my * (my + 2);
        std::vector<long long> key((size_t)np);
        for (int p = 0; p < np; ++p) {
            const int m = S.pt_m[p], l = S.pt_l[p];
            int c[3];
            for (int d = 0; d < 3; ++d) c[d] = cell_index(S.xc[m + (size_t)d * N] + S.bnd[3 * l + d] * S.radibdy);
            const int i = c[0] < 1 ? c[0] + nx : (c[0] > nx ? c[0] - nx : c[0]);
            const int j = c[1] < 1 ? c[1] + my : (c[1] > my ? c[1] - my : c[1]);
            const int k = c[2] < 1 ? c[2] + mz : (c[2] > mz ? c[2] - mz : c[2]);
            key[(size_t)p] = (long long)(i - 1) * rsp + real_offset(my, k - 1, j - 1);
        }
        std::vector<int> ord((size_t)np), inv((size_t)np);
        for (int p = 0; p < np; ++p) ord[(size_t)p] = p;
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return key[(size_t)a] < key[(size_t)b]; });
        std::vector<int> pm((size_t)np), pl((size_t)np);
        for (int t = 0; t < np; ++t) {
            inv[(size_t)ord[(size_t)t]] = t;
            pm[(size_t)t] = S.pt_m[(size_t)ord[(size_t)t]];
            pl[(size_t)t] = S.pt_l[(size_t)ord[(size_t)t]];
        }
        S.pt_m.swap(pm);
        S.pt_l.swap(pl);
        for (auto &e : ent) e.second = inv[(size_t)(e.second >> 3)] * 8 + (e.second & 7);
    }
    std::stable_sort(ent.begin(), ent.end(), [](const std::pair<long long, int> &a, const std::pair<long long, int> &b) { return a.first < b.first; });
    S.sp_node.clear(); S.sp_ptr.clear(); S.sp_ent.clear();
    for (size_t q = 0; q < ent.size(); ++q) {
        if (q == 0 || ent[q].first != ent[q - 1].first) { S.sp_node.push_back((int)ent[q].first); S.sp_ptr.push_back((int)q); }
        S.sp_ent.push_back(ent[q].second);
    }
    S.sp_ptr.push_back((int)ent.size());
}

}  // namespace

// Scalar reversal-point evaluations and their spreading map
// (calc_inner_rev_data, SRC/SCALAR/bc_scalar.F90:558-932, serial branch):
// inner point x = xc + bnd*radibdy, its cell wrapped into 1..nx with
// WEST/EAST_PERIODIC_IMAGE (ibm.h:148-149); a point in cell nx is evaluated
// again shifted by -nx (EAST_PERIODIC_IMAGE_MOD, ibm.h:150).  Stencil corners
// below plane 0 wrap by mxf-1; corners on planes 0 and nx+1 are never
// transformed (ff2rc runs over planes 1..nx), so the map leaves them out.
void build_scalar_evals(RunSetup &S, bool all_nodes) {
    const int N = S.nbody, nb = S.nbnd, nx = S.nx, my = S.my, mz = S.mz, mxf = S.mxf;
    S.sev_m.clear(); S.sev_l.clear(); S.sev_c.clear(); S.sev_x.clear();
    std::vector<std::pair<long long, int>> ent;
    for (int m = 0; m < N; ++m)
        for (int l = 0; l < nb; ++l) {
            if (!S.if_rev[(size_t)l + (size_t)nb * m]) continue;
            double x[3];
            int c[3];
            for (int d = 0; d < 3; ++d) {
                x[d] = S.xc[m + (size_t)d * N] + S.bnd[3 * l + d] * S.radibdy;
                c[d] = cell_index(x[d]);
            }
            int pct = c[0];
            double xlt = x[0];
            if (!(1 <= pct && pct <= nx)) {
                if (c[0] < 1) { pct = mxf + c[0] - 1; xlt = mxf + x[0] - 1; }
                else if (c[0] >= mxf) { pct = c[0] - (mxf - 1); xlt = x[0] - (mxf - 1); }
            }
            const int nev = pct == nx ? 2 : 1;
            for (int ev = 1; ev <= nev; ++ev) {
                if (ev == 1) { c[0] = pct; x[0] = xlt; }
                else if (c[0] >= mxf - 1) { c[0] = c[0] - (mxf - 1); x[0] = x[0] - (mxf - 1); }
                const int e = (int)S.sev_m.size();
                S.sev_m.push_back(m); S.sev_l.push_back(l);
                for (int d = 0; d < 3; ++d) { S.sev_x.push_back(x[d]); S.sev_c.push_back(c[d]); }
                for (int ck = 0; ck < 2; ++ck)
                    for (int cj = 0; cj < 2; ++cj)
                        for (int ci = 0; ci < 2; ++ci) {
                            int i = c[0] + ci, j = c[1] + cj, k = c[2] + ck;
                            if (i < 0) i = mxf + i - 1;
                            if (i < 1 || i > nx) continue;
                            j = j < 1 ? j + my : (j > my ? j - my : j);
                            k = k < 1 ? k + mz : (k > mz ? k - mz : k);
                            const long long node = (long long)(i - 1) * my * mz + (long long)(k - 1) * my + (j - 1);
                            if (!all_nodes && S.fluid[(size_t)node]) continue;
                            ent.push_back({node, e * 8 + ci + 2 * cj + 4 * ck});
                        }
            }
        }
    std::stable_sort(ent.begin(), ent.end(), [](const std::pair<long long, int> &a, const std::pair<long long, int> &b) { return a.first < b.first; });
    S.ssp_node.clear(); S.ssp_ptr.clear(); S.ssp_ent.clear();
    for (size_t q = 0; q < ent.size(); ++q) {
        if (q == 0 || ent[q].first != ent[q - 1].first) { S.ssp_node.push_back((int)ent[q].first); S.ssp_ptr.push_back((int)q); }
        S.ssp_ent.push_back(ent[q].second);
    }
    S.ssp_ptr.push_back((int)ent.size());
}

// DEM constants for moving particles: initialize_coarse_grid
// (collision_mod.F90:346-492: cgrid_fac 1.5, KN = 800000, MEW = 0),
// DES_INIT_ARRAYS / CFASSIGN (:582-741: masses, KT, the collision time and
// DTSOLID = TCOLL/50 from the phase diameter) and the pair damping of
// CALC_FORCE_DES (soft_sphere_coll.F90:408-414), all spheres of one phase.
static void build_dem(RunSetup &S, const pibm_params &prm) {
    S.moving = true;
    S.dem_soft = prm.collision_softsphere ? 1 : 0;
    const double dxeff = 2.0 * S.radbdy * 1.5 * S.dx;
    S.dem_cy = std::max((int)std::lround(S.doml[1] / dxeff), 2);
    S.dem_cx = std::max((int)std::lround(S.doml[0] / dxeff), 2);
    S.dem_cz = std::max((int)std::lround(S.doml[2] / dxeff), 2);
    S.dem_dyc = S.doml[1] / (double)(S.dem_cy - 1);
    S.dem_dxc = S.doml[0] / (double)(S.dem_cx - 1);
    S.dem_dzc = S.doml[2] / (double)(S.dem_cz - 1);
    // search periods XE(IMAX1) - XE(1), XE accumulated cell by cell (:471-483, 823-825)
    double e = 0.0;
    for (int i = 2; i <= S.dem_cx; ++i) e = e + S.dem_dxc;
    S.dem_LXs = e;
    e = 0.0;
    for (int j = 2; j <= S.dem_cy; ++j) e = e + S.dem_dyc;
    S.dem_LYs = e;
    e = 0.0;
    for (int k = 2; k <= S.dem_cz; ++k) e = e + S.dem_dzc;
    S.dem_LZs = e;
    S.dem_kn = 800000.0;
    S.dem_rad = S.radbdy * S.dx;
    const double r2 = S.dem_rad * S.dem_rad;
    S.dem_pvol = (4.0 / 3.0) * kPi * r2 * S.dem_rad;
    S.dem_pmass = S.dem_pvol * prm.rhos;
    const double len = std::log(prm.coeff_rest);
    {
        const double mi = (kPi * std::pow(prm.dia_phys, 3.0) * prm.rhos) / 6.0;
        const double meff = (mi * mi) / (mi + mi);
        double etan = 2.0 * std::sqrt(S.dem_kn * meff) * std::fabs(len);
        etan = etan / std::sqrt(kPi * kPi + std::pow(len, 2.0));
        const double tcoll = kPi / std::sqrt(S.dem_kn / meff - std::pow(etan / meff, 2.0) / 4.0);
        S.dem_dtsolid = std::min(tcoll, kLarge) / 50.0;
    }
    {
        const double mi = (kPi * std::pow(2.0 * S.dem_rad, 3.0) * prm.rhos) / 6.0;
        const double meff = (mi * mi) / (mi + mi);
        S.dem_eta_n = 2.0 * std::sqrt(S.dem_kn * meff) * std::fabs(len);
        S.dem_eta_n = S.dem_eta_n / std::sqrt(kPi * kPi + std::pow(len, 2.0));
    }
}

bool setup_run(const pibm_params &prm, const pibm_particles *parts, RunSetup &S, std::string &err) {
    if (prm.my < 4 || (prm.my % 2) != 0) { err = "MY must be an even integer >= 4"; return false; }
    const int mz = prm.mz > 0 ? prm.mz : prm.my;
    if (mz != prm.my) { err = "only MZ == MY is supported"; return false; }
    if (prm.discr_scheme != PIBM_SCHEME_UPWIND && prm.discr_scheme != PIBM_SCHEME_CENTER) { err = "bad discr_scheme"; return false; }
    if (prm.imove != 0 && prm.imove != 1) { err = "IMOVE must be 0 or 1"; return false; }
    // reference options whose code paths are not part of this engine: refused, never ignored
    if (prm.dobnd) { err = "DOBND = T (surface-point forcing, calc_bnd_forcing) is not supported: set DOBND = F"; return false; }
    if (prm.aliasflag) { err = "ALIASFLAG = 1 (dealiased nonlinear term) is not supported: set ALIASFLAG = 0"; return false; }
    if (prm.nlcons_false) { err = "NLCONS = F is not supported: set NLCONS = T"; return false; }
    S.my = prm.my; S.mz = mz; S.mx = S.my + 1; S.mxf = S.mx; S.nx = S.mx - 1; S.my2 = S.my / 2 + 1;
    S.nbody = parts ? parts->nbody : 0;
    if (S.nbody < 0 || (S.nbody > 0 && !parts->xc)) { err = "bad particle list"; return false; }
    S.doml[1] = prm.lybyd * prm.dia_phys;
    S.dx = S.doml[1] / S.my;
    S.doml[0] = (S.mx - 1) * S.dx; S.doml[2] = S.doml[1];
    S.voldom = S.doml[0] * S.doml[1] * S.doml[2];
    S.radbdy = 0.5 * (double)S.my / prm.lybyd;
    S.dr = prm.dr;
    S.radibdy = S.radbdy - prm.dr; S.radobdy = S.radbdy + prm.dr;
    S.xc.assign(parts && S.nbody ? parts->xc : nullptr, parts && S.nbody ? parts->xc + 3 * (size_t)S.nbody : nullptr);
    S.vel.assign((size_t)S.nbody * 3, 0.0);
    if (parts && parts->velbdy) for (size_t q = 0; q < (size_t)S.nbody * 3; ++q) S.vel[q] = parts->velbdy[q];
    S.char_length = prm.dia_phys;
    S.vis = prm.vis;
    {
        double vf = 0.0;
        for (int m = 0; m < S.nbody; ++m) { const double dia = 2.0 * S.radbdy * S.dx; vf = vf + kPi * std::pow(dia, 3.0) / 6.0; }
        S.mean_volfrac = S.nbody ? vf / S.voldom : 0.0;
    }
    build_mask(S);
    const double ut = (prm.re * S.vis) / S.char_length;
    for (int d = 0; d < 3; ++d) S.uchar[d] = ut * std::cos(kPi * prm.flo_ang[d] / 180.0);
    S.ucharmod = std::sqrt(S.uchar[0] * S.uchar[0] + S.uchar[1] * S.uchar[1] + S.uchar[2] * S.uchar[2]);
    for (int d = 0; d < 3; ++d) {
        double s = 0.0;
        for (int m = 0; m < S.nbody; ++m) s = s + S.vel[m + (size_t)d * S.nbody];
        S.usmean_des[d] = S.nbody ? s / (double)S.nbody : 0.0;
        S.ufmean_des[d] = S.uchar[d] / (1.0 - S.maxvolfrac);
        S.umean0[d] = (prm.set_mpg || prm.initialize_zero) ? 0.0
                      : (1.0 - S.maxvolfrac) * S.ufmean_des[d] + S.maxvolfrac * S.usmean_des[d];
    }
    surface_points(0.5 * prm.dia_phys / S.doml[1] * S.my, prm.f2, S.bnd, S.cd, S.nbnd);
    // initial time step (initialize_flo.F90:557-676)
    const double umeanslip = S.ucharmod / (1.0 - S.maxvolfrac);
    double umax = umeanslip;
    for (double v : S.vel) umax = std::max(umax, std::fabs(v));
    const double dt_conv = S.dx / umax;
    double dt_vis = kLarge;
    if (prm.re < 1.0) dt_vis = prm.re * prm.dbydx * dt_conv / (prm.cfl * prm.vfl);
    build_neighbours(S);
    build_if_rev(S);
    build_spread_map(S, prm.include_frmeanfluid != 0, prm.imove == 0);   // moving runs rebuild theirs every step
    double dt_diff = kLarge;
    if (prm.iscalon) {
        // initscal: SRC/SCALAR/scalar_init.F90:58-122
        if (!(prm.pr_or_sc_nu > 0.0)) { err = "PR_OR_SC_NU must be positive"; return false; }
        S.scal = true;
        S.gamma_s = S.vis / prm.pr_or_sc_nu;
        S.phisurf = prm.phisurf;
        S.phistream = prm.phistream;
        dt_diff = (S.dx * S.dx * (1.0 - S.maxvolfrac)) / S.gamma_s;
        build_scalar_evals(S, prm.include_frmeanfluid != 0);
    }
    if (prm.imove == 1 && S.nbody > 0) {
        if (!(prm.rhos > 0.0) || !(prm.rhof > 0.0)) { err = "RHOF and RHOS must be positive with IMOVE=1"; return false; }
        if (prm.collision_softsphere && !(prm.coeff_rest > 0.0)) { err = "COEFF_REST must be positive"; return false; }
        build_dem(S, prm);
    }
    S.dt = prm.cfl * std::min(std::min(dt_conv, dt_vis), std::min(kLarge, dt_diff));
    S.dt = std::min(S.dt, kLarge);
    S.cf = -1.0 / S.dt;
    S.ramp_frac_time = prm.ramp_frac_steps * S.ucharmod * S.dt / ((double)(float)(S.mx - 1) * S.dx);
    S.dx2 = S.dx * S.dx;
    S.dx3 = std::pow(S.dx, 3.0);
    // wavenumbers (initialize_flo.F90:735-763)
    S.ky.resize(S.my2); S.kz.resize(S.mz); S.w2.resize((size_t)S.my2 * S.mz);
    for (int j = 0; j < S.my2; ++j) S.ky[j] = kTwoPi * (double)j / ((double)S.my * S.dx);
    for (int k = 1; k <= S.mz / 2; ++k) {
        S.kz[k - 1] = kTwoPi * (double)(k - 1) / ((double)S.mz * S.dx);
        S.kz[S.mz - k] = -kTwoPi * (double)k / ((double)S.mz * S.dx);
    }
    for (int k = 0; k < S.mz; ++k)
        for (int j = 0; j < S.my2; ++j) {
            const double re = (0.0 * 0.0 - S.ky[j] * S.ky[j]) + (0.0 * 0.0 - S.kz[k] * S.kz[k]);
            S.w2[(size_t)j + (size_t)S.my2 * k] = -re;
        }
    return true;
}

}  // namespace pibm
