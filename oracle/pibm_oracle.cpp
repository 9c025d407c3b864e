// pibm_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the CPU oracle.
//
// A plain C++ restatement of the reference's serial (PARALLEL=0, x-periodic,
// AB2, order-2 'lpi' interpolation, conservative nonlinear term) time step and
// of the initialisation that defines its inputs.  It is the parity checker for
// the CUDA engine and the timed CPU baseline of bench.py; nothing in the
// product links or calls it.
//
// Parity status: the reference cannot be built here (no Fortran compiler, FFTW
// ships only as prebuilt archives), so the step itself is "parity unpinned"
// against reference outputs.  The plane FFT conventions are pinned against
// numpy (tests/golden); the time integration, the viscous and scalar line
// solves, both x fluxes, the spectral nonlinear products and the projection
// against closed-form shear-wave solutions (tests/test_oracle_decay.py,
// tests/test_oracle_scalar.py); the immersed-boundary set-up and forcing
// against whole-cell translation across the periodic boundaries
// (tests/test_oracle_invariance.py).  Every routine below cites the reference
// lines it restates.  Reference paths are relative to the project root
// PUReIBM_PS2D-FD1D/.
//
// Summation order: global sums that the reference accumulates in a single
// serial accumulator over (i,k,j) are accumulated here per x-plane and then
// combined in plane order, so results do not depend on the thread count.
#include "fft_oracle.h"
#include "../include/pibm.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace orc;

namespace {

// SRC/SHARED_MODULES/constants.F90:84-94 (single-precision literals widened).
const double SMALL_NUMBER = (double)1.0E-35f;
const double LARGE_NUMBER = (double)1.0E+32f;
const double PI = 3.14159265358979323846;   // 4*atan(1) in double == M_PI
const double TWOPI = 2.0 * PI;

thread_local std::string g_err;

inline int fint(double x) { return (int)x; }   // Fortran INT: truncation toward zero

// Soft-sphere DEM state (IMOVE = 1, COLLISION_TYPE = 'softsphere'): dem_mod.F90
// arrays for one phase.  Particle indices are 0-based here; list order is the
// reference's.  Positions and velocities are physical (DES_POS = (XC-1)*dx).
struct Dem {
    int N = 0;
    int cx = 0, cy = 0, cz = 0;               // coarse grid nodes; physical cells 2..c (IMAX1 = cx)
    double dxc = 0, dyc = 0, dzc = 0;
    double LXs = 0, LYs = 0, LZs = 0;         // search periods XE(IMAX1)-XE(1) (collision_mod.F90:823-825)
    double XL = 0, YL = 0, ZL = 0;            // XLENGTH/YLENGTH/ZLENGTH = wall positions EX2/TY2/NZ2
    double kn = 0, kt = 0, eta_n = 0, eta_t = 0, mew = 0;
    double dtsolid_orig = 0, max_radius = 0, rhof = 0;
    int maxneigh = 0;
    std::vector<double> pos, pos_old, vel, vel_old, om, om_old;   // [3*l + d]
    std::vector<double> rad, pmass, pvol;
    std::vector<int> pijk;                                        // [3*l + d], cells 2..c
    std::vector<std::vector<int>> neigh;                          // NEIGHBOURS(l, 2..): mirrors, self, found
    std::vector<std::vector<int>> pn, pv;                         // PN(l, 2..), PV(l, 2..)
};

struct Orc {
    // ---- parameters -------------------------------------------------------
    pibm_params prm;
    int nx, my, mz, my2, mx, mxf;
    double dx, dy, dz, dx2, vis, doml[3], voldom;
    double coef[4];                 // coef(rks,1:4) of the current stage
    double coef_tab[3][4];          // AB2 (one stage) or RK3 (three): initialize_flo.F90:861-884
    int itrmax = 1;
    double char_length, uchar[3], ucharmod, umeanslip;
    double cfl, cfl_max;
    double ramp_frac_time;
    // ---- particles --------------------------------------------------------
    int nbody;
    std::vector<double> xc;         // (nbody,3) col-major, grid units
    std::vector<double> velbdy;     // (nbody,3)
    std::vector<double> radbdy, radibdy, radobdy;
    int nbnd, nrpr;
    std::vector<double> bndpts;     // (3,nbnd)
    std::vector<double> cd;         // (3,nbnd)
    std::vector<uint8_t> if_rev;    // (nbnd, nbody)
    std::vector<int> nrpr_active;   // (nbody)
    std::vector<std::vector<int>> neighbours;  // DEM neighbour lists incl. self
    bool moving = false;            // IMOVE = 1: particles move (DEM every step)
    Dem dem;
    double mean_volfrac, maxvolfrac;
    long long count_solid, count_fluid;
    std::vector<uint8_t> fluid;     // fluid_atijk(0:nx+1, my, mz)
    // ---- means / scalars ---------------------------------------------------
    double umean[3], ufmean[3], ufmean_old[3], usmean[3], usmean_des[3], ufmean_des[3],
        usmean_act[3], mpg[3], frmean[3], frmeanfluid[3], frame_accln[3], frame_vel[3],
        frame_pos[3], pres_total[3], visc_total[3], dufmeandt[3], meanslip[3], mesh_vel[3];
    double dt, t, cf, cforig, mixmeanslipmod, meanslipmod, umax_last, divmax;
    double ferror, fold, norm_drag, pres_drag, visc_drag, total_drag;
    std::vector<double> ferror_array;
    int nerr_steps;
    // ---- spectral state -----------------------------------------------------
    std::vector<cplx> wy, wz;
    std::vector<double> w2;         // (my2,mz)
    std::vector<cplx> u, nl, onl, ff, p;
    // ---- real-space work fields ----------------------------------------------
    std::vector<double> ubcp, pbcp, nlbc, onlbc, diffn, omega, ppr, fr;
    // ---- per-particle ---------------------------------------------------------
    std::vector<double> pres, visc, force;
    // ---- passive scalar (ISCALON = 1, one species) ------------------------------
    bool scal = false;
    double gamma_s = 0, phisurf = 0, phistream = 0;
    double heat_ratio = 1, heat_ratio_old = 1, heat_ratio_new = 1;
    std::vector<cplx> phif, nlphif, onlphif, ffphi;        // (nx+1,my2,mz)
    std::vector<double> phir, nlphir, onlphir, sdiffn;     // (nx+1,my,mz)
    std::vector<double> gradphi;                           // (nx+1,my,mz,3)
    std::vector<double> sfr;                               // fr(0:nx+1,my,mz)
    std::vector<double> flux_body;                         // (nbody)
    double flux_global = 0, nusselt = 0;
    int nthreads = 1;

    // index helpers, 1-based like the reference
    size_t CI(int i, int j, int k, int n) const { return (size_t)(i - 1) + (size_t)(nx + 1) * ((size_t)(j - 1) + (size_t)my2 * ((size_t)(k - 1) + (size_t)mz * (size_t)(n - 1))); }
    size_t PI3(int i, int j, int k) const { return (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)my2 * (size_t)(k - 1)); }
    size_t RI(int i, int j, int k, int n) const { return (size_t)(i - 1) + (size_t)(nx + 1) * ((size_t)(j - 1) + (size_t)my * ((size_t)(k - 1) + (size_t)mz * (size_t)(n - 1))); }
    size_t QI(int i, int j, int k, int n) const { return (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)my * ((size_t)(k - 1) + (size_t)mz * (size_t)(n - 1))); }
    bool FL(int i, int j, int k) const { return fluid[(size_t)i + (size_t)(nx + 2) * ((size_t)(j - 1) + (size_t)my * (size_t)(k - 1))] != 0; }
    void SETFL(int i, int j, int k, bool v) { fluid[(size_t)i + (size_t)(nx + 2) * ((size_t)(j - 1) + (size_t)my * (size_t)(k - 1))] = v ? 1 : 0; }
    size_t SF(int i, int j, int k) const { return (size_t)i + (size_t)(nx + 2) * ((size_t)(j - 1) + (size_t)my * (size_t)(k - 1)); }
    double XC(int m, int n) const { return xc[(size_t)(m - 1) + (size_t)nbody * (n - 1)]; }
    double &XCr(int m, int n) { return xc[(size_t)(m - 1) + (size_t)nbody * (n - 1)]; }
    double VB(int m, int n) const { return velbdy[(size_t)(m - 1) + (size_t)nbody * (n - 1)]; }
    double BND(int n, int l) const { return bndpts[(size_t)(n - 1) + 3 * (size_t)(l - 1)]; }
    double CD(int n, int l) const { return cd[(size_t)(n - 1) + 3 * (size_t)(l - 1)]; }
    double W2(int j, int k) const { return w2[(size_t)(j - 1) + (size_t)my2 * (k - 1)]; }

    // ---- plane helpers (gather/scatter around the thread's PlaneFFT) ----------
    std::vector<PlaneFFT> ffts;
    std::vector<std::vector<cplx>> cbuf;
    std::vector<std::vector<double>> rbuf;
    int tid() const {
#ifdef _OPENMP
        return omp_get_thread_num();
#else
        return 0;
#endif
    }
};

// ============================================================================
// Set-up: initflo restated (SRC/FLO/initialize_flo.F90:61-1013).
// ============================================================================

// quadgener + generbnd + dcgen: SRC/FLO/geom_init.F90:44-242, 244-369, 573-586.
void quadgener(double r, double f2, std::vector<double> &xs, std::vector<double> &cdv, int &nb) {
    std::vector<double> nxb, nyb, nzb;
    int imax = (int)std::lround(TWOPI * r / 4.0 * f2);   // NINT(twopi*r/four*f2)
    double dtheta = TWOPI / imax / 4.0;
    double theta = 0.0;
    for (int i = 1; i <= imax + 1; ++i) {
        int jmax = (int)std::lround(TWOPI * r * std::sin(theta) / 4 * f2);
        double dphi = TWOPI / jmax / 4;
        double phi = 0.0;
        for (int j = 1; j <= jmax + 1; ++j) {
            double z = r * std::cos(theta) / r;
            if (std::fabs(z) < 1.0e-5) z = 0.;
            double y = r * std::sin(theta) * std::cos(phi) / r;
            if (std::fabs(y) < 1.0e-5) y = 0.;
            double x = r * std::sin(theta) * std::sin(phi) / r;
            if (std::fabs(x) < 1.0e-5) x = 0.;
            phi = phi + dphi;
            nzb.push_back(z); nyb.push_back(y); nxb.push_back(x);
        }
        theta = theta + dtheta;
    }
    const int npt = (int)nxb.size();
    xs.clear(); cdv.clear();
    auto add = [&](double a, double b, double c) {
        double rr = std::sqrt(a * a + b * b + c * c);
        xs.push_back(a); xs.push_back(b); xs.push_back(c);
        cdv.push_back(a / rr); cdv.push_back(b / rr); cdv.push_back(c / rr);
    };
    for (int i = 0; i < npt; ++i) add(nxb[i], nyb[i], nzb[i]);
    for (int i = 0; i < npt; ++i) if (nxb[i] != 0) add(-nxb[i], nyb[i], nzb[i]);
    for (int i = 0; i < npt; ++i) if (nyb[i] != 0) add(nxb[i], -nyb[i], nzb[i]);
    for (int i = 0; i < npt; ++i) if (nzb[i] != 0) add(nxb[i], nyb[i], -nzb[i]);
    for (int i = 0; i < npt; ++i) if (nxb[i] != 0 && nyb[i] != 0) add(-nxb[i], -nyb[i], nzb[i]);
    for (int i = 0; i < npt; ++i) if (nxb[i] != 0 && nzb[i] != 0) add(-nxb[i], nyb[i], -nzb[i]);
    for (int i = 0; i < npt; ++i) if (nyb[i] != 0 && nzb[i] != 0) add(nxb[i], -nyb[i], -nzb[i]);
    for (int i = 0; i < npt; ++i) if (nxb[i] != 0 && nyb[i] != 0 && nzb[i] != 0) add(-nxb[i], -nyb[i], -nzb[i]);
    nb = (int)(xs.size() / 3);
}

// grid_nodes_insphere: SRC/FLO/dependent_functions.F90:783-963 (serial branch).
void grid_nodes_insphere(Orc &o) {
    o.fluid.assign((size_t)(o.nx + 2) * o.my * o.mz, 1);
    long long count_solid_tmp = 0, count_fluid_tmp = (long long)o.nx * o.my * o.mz;
    for (int m = 1; m <= o.nbody; ++m) {
        double xlr[3], xll[3];
        for (int d = 1; d <= 3; ++d) { xlr[d - 1] = o.XC(m, d) + o.radbdy[m - 1]; xll[d - 1] = o.XC(m, d) - o.radbdy[m - 1]; }
        int imin = (int)std::ceil(xll[0]), imax = (int)std::floor(xlr[0]);
        int jmin = (int)std::ceil(xll[1]), jmax = (int)std::floor(xlr[1]);
        int kmin = (int)std::ceil(xll[2]), kmax = (int)std::floor(xlr[2]);
        for (int i = imin; i <= imax; ++i) {
            int ii = i;
            if (i < 1) ii = o.mxf + i - 1;
            if (i > o.mxf - 1) ii = i - (o.mxf - 1);
            for (int j = jmin; j <= jmax; ++j) {
                int jj = j;
                if (j < 1) jj = o.my + j;
                if (j > o.my) jj = j - o.my;
                for (int k = kmin; k <= kmax; ++k) {
                    int kk = k;
                    if (k < 1) kk = o.mz + k;
                    if (k > o.mz) kk = k - o.mz;
                    double a = (double)i - o.XC(m, 1), b = (double)j - o.XC(m, 2), c = (double)k - o.XC(m, 3);
                    double dist = a * a;
                    dist = dist + b * b + c * c;
                    dist = std::sqrt(dist);
                    if ((dist - o.radbdy[m - 1]) <= SMALL_NUMBER) {
                        o.SETFL(ii, jj, kk, false);
                        count_solid_tmp += 1;
                        count_fluid_tmp -= 1;
                    }
                }
            }
        }
    }
    o.count_solid = count_solid_tmp;
    o.count_fluid = count_fluid_tmp;
    o.maxvolfrac = (double)o.count_solid / (double)((long long)o.nx * o.my * o.mz);
    for (int k = 1; k <= o.mz; ++k)
        for (int j = 1; j <= o.my; ++j) {
            o.SETFL(o.mxf, j, k, o.FL(1, j, k));
            o.SETFL(0, j, k, o.FL(o.mxf - 1, j, k));
        }
}

// DEM coarse-grid neighbour search restated for the set-up call
// des_time_march(.TRUE.): initialize_coarse_grid (collision_mod.F90:346-499),
// DES_INIT_ARRAYS positions (:1279-1289), find_cell_index (:743-762),
// particles_in_cell (:764-805), GRID_BASED_NEIGHBOR_SEARCH (:807-1062).
// neighbours[LL] lists LL itself first, then neighbours in discovery order.
void neighbor_search(Orc &o) {
    const int N = o.nbody;
    o.neighbours.assign(N, std::vector<int>());
    if (N == 0) return;
    double rmax = 0;
    for (int m = 0; m < N; ++m) rmax = std::max(rmax, o.radbdy[m]);
    const double XL = o.doml[0], YL = o.doml[1], ZL = o.doml[2];
    const double dxeff = 2.0 * rmax * 1.5 * o.dx;
    int cy = std::max((int)std::lround(YL / dxeff), 2);
    int cx = std::max((int)std::lround(XL / dxeff), 2);
    int cz = std::max((int)std::lround(ZL / dxeff), 2);
    double dyc = YL / (double)(cy - 1), dxc = XL / (double)(cx - 1), dzc = ZL / (double)(cz - 1);
    const int IMAX1 = cx, JMAX1 = cy, KMAX1 = cz, IMIN1 = 2, JMIN1 = 2, KMIN1 = 2;
    const int IMAX2 = cx + 1, JMAX2 = cy + 1, KMAX2 = cz + 1;
    std::vector<double> XE(IMAX2 + 1, 0.0), YN(JMAX2 + 1, 0.0), ZT(KMAX2 + 1, 0.0);
    for (int i = IMIN1; i <= IMAX2; ++i) XE[i] = XE[i - 1] + dxc;
    for (int j = JMIN1; j <= JMAX2; ++j) YN[j] = YN[j - 1] + dyc;
    for (int k = KMIN1; k <= KMAX2; ++k) ZT[k] = ZT[k - 1] + dzc;
    const double LX = XE[IMAX1] - XE[1], LY = YN[JMAX1] - YN[1], LZ = ZT[KMAX1] - ZT[1];
    std::vector<double> pos(3 * N), rad(N);
    for (int l = 0; l < N; ++l) {
        pos[3 * l + 0] = (o.XC(l + 1, 1) + 0 - 1.0) * o.dx;
        pos[3 * l + 1] = (o.XC(l + 1, 2) - 1.0) * o.dy;
        pos[3 * l + 2] = (o.XC(l + 1, 3) - 1.0) * o.dz;
        rad[l] = o.radbdy[l] * o.dx;
    }
    std::vector<int> pijk(3 * N);
    // cell -> particle list (ascending particle index)
    auto cell_id = [&](int i, int j, int k) { return (size_t)i + (size_t)(IMAX2 + 1) * ((size_t)j + (size_t)(JMAX2 + 1) * (size_t)k); };
    std::vector<std::vector<int>> pic((size_t)(IMAX2 + 1) * (JMAX2 + 1) * (KMAX2 + 1));
    for (int ip = 0; ip < N; ++ip) {
        pijk[3 * ip + 0] = std::min(fint(pos[3 * ip + 0] / dxc) + 2, IMAX1);
        pijk[3 * ip + 1] = std::min(fint(pos[3 * ip + 1] / dyc) + 2, JMAX1);
        pijk[3 * ip + 2] = std::min(fint(pos[3 * ip + 2] / dzc) + 2, KMAX1);
        pic[cell_id(pijk[3 * ip], pijk[3 * ip + 1], pijk[3 * ip + 2])].push_back(ip);
    }
    for (int LL = 0; LL < N; ++LL) o.neighbours[LL].push_back(LL);
    for (int LL = 0; LL < N; ++LL) {
        int II = pijk[3 * LL], JJ = pijk[3 * LL + 1], KK = pijk[3 * LL + 2];
        for (int kk = KK - 1; kk <= KK + 1; ++kk)
            for (int jj = JJ - 1; jj <= JJ + 1; ++jj)
                for (int ii = II - 1; ii <= II + 1; ++ii) {
                    int I = ii, J = jj, K = kk;
                    double xper = 0, yper = 0, zper = 0;
                    if (ii > IMAX1) { I = IMIN1; xper = 1.0; }
                    if (ii < IMIN1) { I = IMAX1; xper = -1.0; }
                    if (jj > JMAX1) { J = JMIN1; yper = 1.0; }
                    if (jj < JMIN1) { J = JMAX1; yper = -1.0; }
                    if (kk > KMAX1) { K = KMIN1; zper = 1.0; }
                    if (kk < KMIN1) { K = KMAX1; zper = -1.0; }
                    const std::vector<int> &lst = pic[cell_id(I, J, K)];
                    for (int PNO : lst) {
                        if (PNO <= LL) continue;
                        double R_LM = 1.2 * (rad[LL] + rad[PNO]);
                        double c0 = pos[3 * PNO + 0] + xper * LX, c1 = pos[3 * PNO + 1] + yper * LY, c2 = pos[3 * PNO + 2] + zper * LZ;
                        double d0 = c0 - pos[3 * LL + 0], d1 = c1 - pos[3 * LL + 1], d2 = c2 - pos[3 * LL + 2];
                        double distmag = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                        bool already = false;
                        for (size_t q = 1; q < o.neighbours[LL].size(); ++q) if (o.neighbours[LL][q] == PNO) already = true;
                        if (R_LM - distmag > SMALL_NUMBER && !already) {
                            o.neighbours[LL].push_back(PNO);
                            o.neighbours[PNO].push_back(LL);
                        }
                    }
                }
    }
}

// update_nrpr_array + check_external_pt: SRC/FLO/dependent_functions.F90:966-1051.
void update_nrpr(Orc &o) {
    o.if_rev.assign((size_t)o.nbnd * o.nbody, 1);
    o.nrpr_active.assign(o.nbody, o.nrpr);
    for (int m = 1; m <= o.nbody; ++m) {
        for (int l = 1; l <= o.nrpr; ++l) {
            double XLO[3];
            for (int n = 1; n <= 3; ++n) XLO[n - 1] = o.XC(m, n) + o.BND(n, l) * o.radobdy[m - 1];
            bool rev = true;
            if (XLO[0] < 1.0) XLO[0] = o.mxf + XLO[0];
            if (XLO[0] > o.mxf) XLO[0] = XLO[0] - o.mxf;
            if (XLO[1] < 1.0) XLO[1] = o.my + 1.0 + XLO[1];
            if (XLO[1] > o.my) XLO[1] = XLO[1] - o.my - 1.0;
            if (XLO[2] < 1.0) XLO[2] = o.mz + 1.0 + XLO[2];
            if (XLO[2] > o.mz) XLO[2] = XLO[2] - o.mz - 1.0;
            const std::vector<int> &nb = o.neighbours[m - 1];
            if (nb.size() > 1) {
                for (size_t ip = 0; ip < nb.size(); ++ip) {
                    int PNO = nb[ip] + 1;
                    double dist = 0.0;
                    for (int d = 1; d <= 3; ++d) { double a = o.XC(PNO, d) - XLO[d - 1]; dist = dist + a * a; }
                    dist = std::sqrt(dist);
                    if (dist < o.radbdy[PNO - 1]) { rev = false; break; }
                }
            }
            o.if_rev[(size_t)(l - 1) + (size_t)o.nbnd * (m - 1)] = rev ? 1 : 0;
            if (!rev) o.nrpr_active[m - 1] -= 1;
        }
    }
}

// ============================================================================
// Soft-sphere DEM for moving particles (IMOVE = 1, COLLISION_TYPE =
// 'softsphere', one phase, x/y/z-periodic walls, no wall contacts since
// WALLDTSPLIT = F).  initialize_coarse_grid sets MEW = MEW_W = 0
// (collision_mod.F90:388-389), so CFSLIDE always returns a tangential force of
// (signed) zero and the tangential history PFN/PFT never reaches a force; the
// rotation update is commented out (CFNEWVALUES, :1388), so OMEGA stays 0.
// What moves the particles is the normal spring-dashpot force of each contact
// pair; the contact lists PN/PV are kept exactly as the reference keeps them.
// ============================================================================

// initialize_coarse_grid (collision_mod.F90:346-492), DES_INIT_ARRAYS (:1203-1316)
// and CFASSIGN (:582-741) for the 'default' particle input.
void dem_init(Orc &o) {
    Dem &D = o.dem;
    const int N = o.nbody;
    D.N = N;
    D.XL = o.doml[0]; D.YL = o.doml[1]; D.ZL = o.doml[2];
    double rmax = 0.0;
    for (int m = 0; m < N; ++m) rmax = std::max(rmax, o.radbdy[m]);
    const double dxeff = 2.0 * rmax * 1.5 * o.dx;                  // cgrid_fac = 1.5
    D.cy = std::max((int)std::lround(D.YL / dxeff), 2);
    D.cx = std::max((int)std::lround(D.XL / dxeff), 2);
    D.cz = std::max((int)std::lround(D.ZL / dxeff), 2);
    D.dyc = D.YL / (double)(D.cy - 1);
    D.dxc = D.XL / (double)(D.cx - 1);
    D.dzc = D.ZL / (double)(D.cz - 1);
    // XE(1) = 0, XE(i) = XE(i-1) + dxc (i = 2..IMAX2); period = XE(IMAX1) - XE(1)
    double e = 0.0;
    for (int i = 2; i <= D.cx; ++i) e = e + D.dxc;
    D.LXs = e;
    e = 0.0;
    for (int j = 2; j <= D.cy; ++j) e = e + D.dyc;
    D.LYs = e;
    e = 0.0;
    for (int k = 2; k <= D.cz; ++k) e = e + D.dzc;
    D.LZs = e;
    D.kn = 800000.0;                                              // KN (:384-386)
    D.kt = (2.0 / 7.0) * D.kn;                                    // KT (CFASSIGN :627)
    D.mew = 0.0;
    D.maxneigh = 30 + 1 + 6;                                      // MN + 1 + NWALLS (:508)
    D.rhof = o.prm.rhof;
    D.pos.assign(3 * (size_t)N, 0.0); D.vel.assign(3 * (size_t)N, 0.0); D.om.assign(3 * (size_t)N, 0.0);
    D.rad.assign(N, 0.0); D.pmass.assign(N, 0.0); D.pvol.assign(N, 0.0);
    D.max_radius = 0.0;
    for (int l = 0; l < N; ++l) {
        D.pos[3 * l + 0] = (o.XC(l + 1, 1) + 0.0 - 1.0) * o.dx;   // foffset = 0
        D.pos[3 * l + 1] = (o.XC(l + 1, 2) - 1.0) * o.dy;
        D.pos[3 * l + 2] = (o.XC(l + 1, 3) - 1.0) * o.dz;
        D.rad[l] = o.radbdy[l] * o.dx;
        for (int d = 0; d < 3; ++d) D.vel[3 * l + d] = o.VB(l + 1, d + 1);
        const double r2 = D.rad[l] * D.rad[l];
        D.pvol[l] = (4.0 / 3.0) * PI * r2 * D.rad[l];
        D.pmass[l] = D.pvol[l] * o.prm.rhos;
        D.max_radius = std::max(D.max_radius, D.rad[l]);
    }
    D.pos_old = D.pos; D.vel_old = D.vel; D.om_old = D.om;
    // collision time from the phase diameter (CFASSIGN :664-680); DTSOLID = TCOLL/50
    const double en = o.prm.coeff_rest, len = std::log(en);
    {
        const double mi = (PI * std::pow(o.prm.dia_phys, 3.0) * o.prm.rhos) / 6.0;
        const double meff = (mi * mi) / (mi + mi);
        double etan = 2.0 * std::sqrt(D.kn * meff) * std::fabs(len);
        etan = etan / std::sqrt(PI * PI + std::pow(len, 2.0));
        const double tcoll = PI / std::sqrt(D.kn / meff - std::pow(etan / meff, 2.0) / 4.0);
        D.dtsolid_orig = std::min(tcoll, LARGE_NUMBER) / 50.0;
    }
    // pair damping of CALC_FORCE_DES (soft_sphere_coll.F90:408-414): one phase,
    // so every pair has the same masses
    if (N > 0) {
        const double mi = (PI * std::pow(2.0 * D.rad[0], 3.0) * o.prm.rhos) / 6.0;
        const double meff = (mi * mi) / (mi + mi);
        D.eta_n = 2.0 * std::sqrt(D.kn * meff) * std::fabs(len);
        D.eta_n = D.eta_n / std::sqrt(PI * PI + std::pow(len, 2.0));
        D.eta_t = 0.5 * D.eta_n;
    }
    D.pn.assign(N, {}); D.pv.assign(N, {});
}

// FIND_CELL_INDEX (collision_mod.F90:743-762).
void dem_cells(Dem &D) {
    D.pijk.assign(3 * (size_t)D.N, 0);
    for (int l = 0; l < D.N; ++l) {
        D.pijk[3 * l + 0] = std::min(fint(D.pos[3 * l + 0] / D.dxc) + 2, D.cx);
        D.pijk[3 * l + 1] = std::min(fint(D.pos[3 * l + 1] / D.dyc) + 2, D.cy);
        D.pijk[3 * l + 2] = std::min(fint(D.pos[3 * l + 2] / D.dzc) + 2, D.cz);
    }
}

// PARTICLES_IN_CELL + GRID_BASED_NEIGHBOR_SEARCH (collision_mod.F90:764-1062).
// NEIGHBOURS(LL) ends up as: entries appended by lower particles' searches
// (ascending), LL itself, then LL's own finds in cell-scan order.
bool dem_search(Dem &D) {
    const int N = D.N;
    const int W = D.cx + 2, H = D.cy + 2;
    std::vector<std::vector<int>> pic((size_t)W * H * (D.cz + 2));
    auto bin = [&](int i, int j, int k) -> std::vector<int> & { return pic[(size_t)i + (size_t)W * ((size_t)j + (size_t)H * k)]; };
    for (int l = 0; l < N; ++l) bin(D.pijk[3 * l], D.pijk[3 * l + 1], D.pijk[3 * l + 2]).push_back(l);
    D.neigh.assign(N, {});
    for (int LL = 0; LL < N; ++LL) {
        D.neigh[LL].push_back(LL);
        if ((int)D.neigh[LL].size() + 1 > D.maxneigh) { g_err = "DEM neighbour list overflow"; return false; }
        const int II = D.pijk[3 * LL], JJ = D.pijk[3 * LL + 1], KK = D.pijk[3 * LL + 2];
        for (int kk = KK - 1; kk <= KK + 1; ++kk)
            for (int jj = JJ - 1; jj <= JJ + 1; ++jj)
                for (int ii = II - 1; ii <= II + 1; ++ii) {
                    int I = ii, J = jj, K = kk;
                    double xper = 0.0, yper = 0.0, zper = 0.0;
                    if (ii > D.cx) { I = 2; xper = 1.0; }
                    if (ii < 2) { I = D.cx; xper = -1.0; }
                    if (jj > D.cy) { J = 2; yper = 1.0; }
                    if (jj < 2) { J = D.cy; yper = -1.0; }
                    if (kk > D.cz) { K = 2; zper = 1.0; }
                    if (kk < 2) { K = D.cz; zper = -1.0; }
                    for (int PNO : bin(I, J, K)) {
                        if (PNO <= LL) continue;
                        const double rlm = 1.2 * (D.rad[LL] + D.rad[PNO]);   // FACTOR_RLM
                        const double c0 = D.pos[3 * PNO + 0] + xper * D.LXs;
                        const double c1 = D.pos[3 * PNO + 1] + yper * D.LYs;
                        const double c2 = D.pos[3 * PNO + 2] + zper * D.LZs;
                        const double d0 = c0 - D.pos[3 * LL + 0], d1 = c1 - D.pos[3 * LL + 1], d2 = c2 - D.pos[3 * LL + 2];
                        double dd = 0.0;
                        dd = dd + d0 * d0; dd = dd + d1 * d1; dd = dd + d2 * d2;
                        const double distmag = std::sqrt(dd);
                        bool already = false;
                        for (size_t q = 0; q < D.neigh[LL].size(); ++q) if (D.neigh[LL][q] == PNO) already = true;
                        if (rlm - distmag > SMALL_NUMBER && !already) {
                            D.neigh[LL].push_back(PNO);
                            if ((int)D.neigh[LL].size() + 1 > D.maxneigh) { g_err = "DEM neighbour list overflow"; return false; }
                            D.neigh[PNO].push_back(LL);
                            if ((int)D.neigh[PNO].size() + 1 > D.maxneigh) { g_err = "DEM neighbour list overflow"; return false; }
                        }
                    }
                }
    }
    return true;
}

// CALC_FORCE_DES (soft_sphere_coll.F90:52-551) without walls: contact-list
// upkeep and the contact force FC of every particle.
bool dem_forces(Dem &D, double dtsolid, std::vector<double> &fc) {
    const int N = D.N;
    const double L[3] = {D.XL, D.YL, D.ZL};
    fc.assign(3 * (size_t)N, 0.0);
    for (int LL = 0; LL < N; ++LL) {
        std::vector<int> &pn = D.pn[LL], &pv = D.pv[LL];
        {   // drop the entries whose contact ended (PV = 0), keeping the order
            size_t w = 0;
            for (size_t q = 0; q < pn.size(); ++q)
                if (pv[q] != 0) { pn[w] = pn[q]; pv[w] = pv[q]; ++w; }
            pn.resize(w); pv.resize(w);
        }
        std::fill(pv.begin(), pv.end(), 0);
        for (int I : D.neigh[LL]) {
            if (I <= LL) continue;
            int ni = -1, ni_i = -1;
            for (size_t q = 0; q < pn.size(); ++q) if (pn[q] == I) { ni = (int)q; break; }
            if (ni >= 0)
                for (size_t q = 0; q < D.pn[I].size(); ++q) if (D.pn[I][q] == LL) { ni_i = (int)q; break; }
            double pI[3];
            for (int d = 0; d < 3; ++d) {
                pI[d] = D.pos[3 * I + d];
                const double tempd = std::fabs(D.pos[3 * LL + d] - D.pos[3 * I + d]);
                if (tempd > 4.0 * D.max_radius) pI[d] = pI[d] > D.pos[3 * LL + d] ? pI[d] - L[d] : pI[d] + L[d];
            }
            const double rlm = D.rad[LL] + D.rad[I];
            double dist[3], dd = 0.0;
            for (int d = 0; d < 3; ++d) dist[d] = pI[d] - D.pos[3 * LL + d];
            for (int d = 0; d < 3; ++d) dd = dd + dist[d] * dist[d];
            const double distmod = std::sqrt(dd);
            if (!(rlm - distmod > SMALL_NUMBER)) continue;
            if (distmod == 0.0) { g_err = "DEM: coincident particle centres"; return false; }
            double nrm[3];
            for (int d = 0; d < 3; ++d) nrm[d] = dist[d] / distmod;
            // CFRELVEL (:728-776)
            double vrel[3], osum[3], vrot[3];
            for (int d = 0; d < 3; ++d) vrel[d] = D.vel[3 * LL + d] - D.vel[3 * I + d];
            for (int d = 0; d < 3; ++d) osum[d] = D.om[3 * LL + d] * D.rad[LL] + D.om[3 * I + d] * D.rad[I];
            vrot[0] = osum[1] * nrm[2] - osum[2] * nrm[1];
            vrot[1] = osum[2] * nrm[0] - osum[0] * nrm[2];
            vrot[2] = osum[0] * nrm[1] - osum[1] * nrm[0];
            for (int d = 0; d < 3; ++d) vrel[d] = vrel[d] + vrot[d];
            double vrn = 0.0;
            for (int d = 0; d < 3; ++d) vrn = vrn + vrel[d] * nrm[d];
            double ov_n;
            if (ni >= 0) {
                pv[ni] = 1;
                if (ni_i >= 0) D.pv[I][ni_i] = 1;
                ov_n = rlm - distmod;
            } else {
                pn.push_back(I); pv.push_back(1);
                D.pn[I].push_back(LL); D.pv[I].push_back(1);
                ov_n = rlm - distmod;
            }
            if ((int)pn.size() + 1 > D.maxneigh || (int)D.pn[I].size() + 1 > D.maxneigh) { g_err = "DEM contact list overflow"; return false; }
            // normal force FNS1 + FNS2; the tangential force is zero (MEW = 0)
            for (int d = 0; d < 3; ++d) {
                const double fns1 = -(D.kn * ov_n) * nrm[d];
                const double fns2 = -(D.eta_n * vrn) * nrm[d];
                const double fn = fns1 + fns2;
                fc[3 * LL + d] = fc[3 * LL + d] + fn;       // CFFCTOW (:873-905)
                fc[3 * I + d] = fc[3 * I + d] - fn;
            }
        }
    }
    return true;
}

// des_time_march(.FALSE.) for 'softsphere' (collision_mod.F90:272-294) and
// IBMUPDATE (:1464-1474): FACTOR sub-steps of SOFT_SPHERE_COLLISION
// (CALC_FORCE_DES + CFNEWVALUES, :1658-1761), CFUPDATEOLD, FIND_CELL_INDEX,
// PARTICLES_IN_CELL and GRID_BASED_NEIGHBOR_SEARCH.
int des_time_march(Orc &o) {
    Dem &D = o.dem;
    const int N = D.N;
    const double L[3] = {D.XL, D.YL, D.ZL};
    if (!o.prm.collision_softsphere) {
        // COLLISION_TYPE = 'none' (:295-328): DTSOLID = dt, velocities kept,
        // positions advanced by CFNEWVALUES; the neighbour lists are not rebuilt
        for (int l = 0; l < N; ++l) {
            double dd = 0.0;
            for (int d = 0; d < 3; ++d) {
                D.vel[3 * l + d] = D.vel_old[3 * l + d];
                D.om[3 * l + d] = D.om_old[3 * l + d];
                D.pos[3 * l + d] = D.pos_old[3 * l + d] + D.vel[3 * l + d] * o.dt;
                const double t = D.pos[3 * l + d] - D.pos_old[3 * l + d];
                dd = dd + t * t;
            }
            if (std::sqrt(dd) >= D.rad[l]) { g_err = "DEM: particle moved a radius in one sub-step"; return PIBM_ERR_DEM_MOVE; }
            for (int d = 0; d < 3; ++d) {
                if (D.pos[3 * l + d] > L[d]) D.pos[3 * l + d] = D.pos[3 * l + d] - (L[d] - 0.0);
                else if (D.pos[3 * l + d] < 0.0) D.pos[3 * l + d] = D.pos[3 * l + d] + (L[d] - 0.0);
            }
            for (int d = 0; d < 3; ++d) { D.pos_old[3 * l + d] = D.pos[3 * l + d]; D.vel_old[3 * l + d] = D.vel[3 * l + d]; }
        }
    } else {
    int factor = fint(o.dt / D.dtsolid_orig);
    double dts = D.dtsolid_orig;
    if (factor < 1) { factor = 1; dts = o.dt; }
    std::vector<double> fc;
    for (int ifac = 1; ifac <= factor; ++ifac) {
        if (!dem_forces(D, dts, fc)) return PIBM_ERR_NEIGH_OVERFLOW;
        // CFNEWVALUES (:1335-1462), softsphere, coupled to the flow
        for (int l = 0; l < N; ++l) {
            for (int d = 0; d < 3; ++d) {
                const size_t q = (size_t)l + (size_t)N * d;
                double a = fc[3 * l + d] / D.pmass[l] + (D.rhof * (o.pres[q] + o.visc[q])) / D.pmass[l];
                a = a - o.frame_accln[d];
                a = a - (o.mpg[d] * D.pvol[l]) / D.pmass[l];
                D.vel[3 * l + d] = D.vel_old[3 * l + d] + a * dts;
                D.om[3 * l + d] = D.om_old[3 * l + d];
                D.pos[3 * l + d] = D.pos_old[3 * l + d] + D.vel[3 * l + d] * dts;
            }
            double dd = 0.0;
            for (int d = 0; d < 3; ++d) { const double t = D.pos[3 * l + d] - D.pos_old[3 * l + d]; dd = dd + t * t; }
            if (std::sqrt(dd) >= D.rad[l]) { g_err = "DEM: particle moved a radius in one sub-step"; return PIBM_ERR_DEM_MOVE; }
            for (int d = 0; d < 3; ++d) {
                if (D.pos[3 * l + d] > L[d]) D.pos[3 * l + d] = D.pos[3 * l + d] - (L[d] - 0.0);
                else if (D.pos[3 * l + d] < 0.0) D.pos[3 * l + d] = D.pos[3 * l + d] + (L[d] - 0.0);
            }
        }
        D.pos_old = D.pos; D.vel_old = D.vel; D.om_old = D.om;   // CFUPDATEOLD
        dem_cells(D);
        if (!dem_search(D)) return PIBM_ERR_NEIGH_OVERFLOW;
    }
    }
    for (int m = 1; m <= N; ++m) {
        o.XCr(m, 1) = D.pos[3 * (m - 1) + 0] / o.dx + 1.0 - 0.0;
        o.XCr(m, 2) = D.pos[3 * (m - 1) + 1] / o.dy + 1.0;
        o.XCr(m, 3) = D.pos[3 * (m - 1) + 2] / o.dz + 1.0;
        for (int d = 0; d < 3; ++d) o.velbdy[(size_t)(m - 1) + (size_t)N * d] = D.vel[3 * (m - 1) + d];
    }
    o.neighbours = D.neigh;
    return PIBM_OK;
}

bool setup(Orc &o, const pibm_params *prm, const pibm_particles *parts) {
    o.prm = *prm;
    if (prm->my <= 0 || (prm->my % 2) != 0) { g_err = "my must be positive and even"; return false; }
    o.my = prm->my;
    o.mz = prm->mz > 0 ? prm->mz : prm->my;
    o.mx = o.my + 1; o.mxf = o.mx; o.nx = o.mx - 1; o.my2 = o.my / 2 + 1;
    o.nbody = parts ? parts->nbody : 0;
    // 'default' particle input: initialize_flo.F90:1555-1590
    o.doml[1] = prm->lybyd * prm->dia_phys;
    o.radbdy.assign(o.nbody, 0.5 * (double)o.my / prm->lybyd);
    o.dx = o.doml[1] / o.my; o.dy = o.dx; o.dz = o.dx;
    o.doml[0] = (o.mx - 1) * o.dx; o.doml[2] = o.doml[1];
    o.xc.assign((size_t)o.nbody * 3, 0.0);
    o.velbdy.assign((size_t)o.nbody * 3, 0.0);
    for (int m = 0; m < o.nbody * 3; ++m) {
        o.xc[m] = parts->xc[m];
        if (parts->velbdy) o.velbdy[m] = parts->velbdy[m];
    }
    o.char_length = prm->dia_phys;
    o.vis = prm->vis;
    o.cfl = prm->cfl; o.cfl_max = prm->cfl_max;
    // phase volume fraction: INPUT_CHECK formula (initialize_flo.F90:2293-2306);
    // the reference's 'default' branch leaves vol_frac1 = 0 (:1493,1536).
    o.voldom = o.doml[0] * o.doml[1] * o.doml[2];
    {
        double vf = 0.0;
        for (int m = 0; m < o.nbody; ++m) { double dia = 2.0 * o.radbdy[m] * o.dx; vf = vf + PI * std::pow(dia, 3.0) / 6.0; }
        o.mean_volfrac = o.nbody > 0 ? vf / o.voldom : 0.0;
    }
    grid_nodes_insphere(o);
    // uchar: initialize_flo.F90:277-283
    double uchar_tmp = (prm->re * o.vis) / o.char_length;
    for (int d = 0; d < 3; ++d) o.uchar[d] = uchar_tmp * std::cos(PI * prm->flo_ang[d] / 180.0);
    o.ucharmod = std::sqrt(o.uchar[0] * o.uchar[0] + o.uchar[1] * o.uchar[1] + o.uchar[2] * o.uchar[2]);
    // desired means and initial umean: :318-353
    for (int d = 0; d < 3; ++d) {
        double s = 0.0;
        for (int m = 1; m <= o.nbody; ++m) s = s + o.VB(m, d + 1);
        o.usmean_des[d] = o.nbody > 0 ? s / (double)o.nbody : 0.0;
        o.ufmean_des[d] = o.uchar[d] / (1.0 - o.maxvolfrac);
        o.umean[d] = (prm->set_mpg || prm->initialize_zero) ? 0.0
                     : (1.0 - o.maxvolfrac) * o.ufmean_des[d] + o.maxvolfrac * o.usmean_des[d];
        o.frame_accln[d] = 0; o.frame_vel[d] = 0; o.frame_pos[d] = 1.0;
        o.mpg[d] = prm->mpg[d];
        o.ufmean[d] = 0; o.ufmean_old[d] = 0; o.usmean[d] = 0; o.frmean[d] = 0; o.frmeanfluid[d] = 0;
        o.pres_total[d] = 0; o.visc_total[d] = 0; o.dufmeandt[d] = 0; o.usmean_act[d] = 0;
        o.mesh_vel[d] = 0;
    }
    // surface points: :450-495
    double r = 0.5 * prm->dia_phys / o.doml[1] * o.my;
    quadgener(r, prm->f2, o.bndpts, o.cd, o.nbnd);
    o.nrpr = o.nbnd;
    o.radibdy.resize(o.nbody); o.radobdy.resize(o.nbody);
    for (int m = 0; m < o.nbody; ++m) { o.radibdy[m] = o.radbdy[m] - prm->dr; o.radobdy[m] = o.radbdy[m] + prm->dr; }
    // time step: :557-676
    o.umeanslip = std::sqrt(o.uchar[0] * o.uchar[0] + o.uchar[1] * o.uchar[1] + o.uchar[2] * o.uchar[2]) / (1.0 - o.maxvolfrac);
    double umax_tmp = o.umeanslip;
    for (int m = 0; m < o.nbody * 3; ++m) umax_tmp = std::max(umax_tmp, std::fabs(o.velbdy[m]));
    double dt_tmp_conv = o.dx / umax_tmp;
    double dt_tmp_vis = LARGE_NUMBER, dt_tmp_grav = LARGE_NUMBER, dt_tmp_diff = LARGE_NUMBER, dtcoll = LARGE_NUMBER;
    if (prm->re < 1.0) dt_tmp_vis = prm->re * prm->dbydx * dt_tmp_conv / (prm->cfl * prm->vfl);
    if (prm->iscalon) {
        // initscal: SRC/SCALAR/scalar_init.F90:58-122 (gamma = vis/Pr, diffusive dt limit)
        o.scal = true;
        o.gamma_s = o.vis / prm->pr_or_sc_nu;
        o.phisurf = prm->phisurf;
        o.phistream = prm->phistream;
        dt_tmp_diff = (o.dx * o.dx * (1.0 - o.maxvolfrac)) / o.gamma_s;
    }
    o.moving = prm->imove == 1 && o.nbody > 0;
    if (o.moving) {
        // des_time_march(.TRUE.) (initialize_flo.F90:631-639): the DEM arrays,
        // cells and the first neighbour search
        dem_init(o);
        dem_cells(o.dem);
        if (!dem_search(o.dem)) return false;
        o.neighbours = o.dem.neigh;
    } else {
        neighbor_search(o);
    }
    update_nrpr(o);
    o.dt = std::min(std::min(dt_tmp_conv, dt_tmp_vis), std::min(dt_tmp_grav, dt_tmp_diff));
    o.dt = prm->cfl * o.dt;
    o.dt = std::min(o.dt, dtcoll);
    o.cf = -1.0 / o.dt; o.cforig = o.cf;
    o.nerr_steps = 100;
    o.ferror = 1.0; o.fold = 0.0; o.ferror_array.assign(o.nerr_steps, 1.0);
    o.ramp_frac_time = prm->ramp_frac_steps * o.ucharmod * o.dt / ((double)(float)(o.mx - 1) * o.dx);
    o.dx2 = o.dx * o.dx;
    // wavenumbers: :735-742, 759-763
    o.wy.resize(o.my2); o.wz.resize(o.mz); o.w2.resize((size_t)o.my2 * o.mz);
    for (int i = 1; i <= o.my2; ++i) o.wy[i - 1] = cplx(0.0, TWOPI * (double)(i - 1) / ((double)o.my * o.dy));
    for (int i = 1; i <= o.mz / 2; ++i) {
        o.wz[i - 1] = cplx(0.0, TWOPI * (double)(i - 1) / ((double)o.mz * o.dz));
        o.wz[o.mz + 1 - i - 1] = cplx(0.0, -TWOPI * (double)i / ((double)o.mz * o.dz));
    }
    for (int k = 1; k <= o.mz; ++k)
        for (int j = 1; j <= o.my2; ++j) {
            cplx s = o.wy[j - 1] * o.wy[j - 1] + o.wz[k - 1] * o.wz[k - 1];
            o.w2[(size_t)(j - 1) + (size_t)o.my2 * (k - 1)] = -s.real();
        }
    if (prm->rk3) {
        const double t[3][4] = {{4.0 / 15.0, 4.0 / 15.0, 8.0 / 15.0, 0.0},
                                {1.0 / 15.0, 1.0 / 15.0, 5.0 / 12.0, -17.0 / 60.0},
                                {1.0 / 6.0, 1.0 / 6.0, 3.0 / 4.0, -5.0 / 12.0}};
        std::memcpy(o.coef_tab, t, sizeof(t));
        o.itrmax = 3;
    } else {
        const double t[4] = {0.5, 0.5, 3.0 / 2.0, -0.5};
        for (int r = 0; r < 3; ++r) std::memcpy(o.coef_tab[r], t, sizeof(t));
        o.itrmax = 1;
    }
    std::memcpy(o.coef, o.coef_tab[0], sizeof(o.coef));
    o.t = 0.0;
    const size_t NC = (size_t)(o.nx + 1) * o.my2 * o.mz * 3;
    o.u.assign(NC, 0.0); o.nl.assign(NC, 0.0); o.onl.assign(NC, 0.0); o.ff.assign(NC, 0.0);
    o.p.assign((size_t)o.nx * o.my2 * o.mz, 0.0);
    const size_t NR = (size_t)(o.nx + 1) * o.my * o.mz * 3;
    o.ubcp.assign(NR, 0.0); o.nlbc.assign(NR, 0.0); o.onlbc.assign(NR, 0.0); o.diffn.assign(NR, 0.0);
    o.omega.assign(NR, 0.0); o.fr.assign(NR, 0.0);
    o.pbcp.assign((size_t)o.nx * o.my * o.mz, 0.0);
    o.ppr.assign((size_t)o.nx * o.my * o.mz * 3, 0.0);
    o.pres.assign((size_t)o.nbody * 3, 0.0); o.visc.assign((size_t)o.nbody * 3, 0.0); o.force.assign((size_t)o.nbody * 3, 0.0);
    o.mixmeanslipmod = 0; o.meanslipmod = 0; o.umax_last = 0; o.divmax = 0; o.norm_drag = 0;
    if (o.scal) {
        // phi = 1 on every plane (scalar_init.F90:136-152): ff2rc of a constant
        // plane is exactly 1 at ky = kz = 0 and 0 elsewhere
        const size_t SC = (size_t)(o.nx + 1) * o.my2 * o.mz, SR = (size_t)(o.nx + 1) * o.my * o.mz;
        o.phif.assign(SC, 0.0); o.nlphif.assign(SC, 0.0); o.onlphif.assign(SC, 0.0); o.ffphi.assign(SC, 0.0);
        for (int i = 1; i <= o.nx + 1; ++i) o.phif[o.CI(i, 1, 1, 1)] = 1.0;
        o.phir.assign(SR, 0.0); o.nlphir.assign(SR, 0.0); o.onlphir.assign(SR, 0.0); o.sdiffn.assign(SR, 0.0);
        o.gradphi.assign(SR * 3, 0.0);
        o.sfr.assign((size_t)(o.nx + 2) * o.my * o.mz, 0.0);
        o.flux_body.assign(o.nbody, 0.0);
    }
#ifdef _OPENMP
    o.nthreads = omp_get_max_threads();
#endif
    o.ffts.resize(o.nthreads); o.cbuf.resize(o.nthreads); o.rbuf.resize(o.nthreads);
    for (int q = 0; q < o.nthreads; ++q) {
        o.ffts[q].init(o.my, o.mz);
        o.cbuf[q].resize((size_t)o.my2 * o.mz);
        o.rbuf[q].resize((size_t)o.my * o.mz);
    }
    if (!o.ffts[0].fy.ok() || !o.ffts[0].fz.ok()) { g_err = "grid size must be 2^a 3^b"; return false; }
    return true;
}

// ============================================================================
// Plane transforms between the x-fastest 4-D arrays and contiguous planes.
// ============================================================================
void c2r_plane(Orc &o, const cplx *src, size_t stride_x_offset_fn_dummy, double *dst);

// c2r of a complex plane given by a gather lambda, scatter into a real field.
template <class G, class S>
void c2r_with(Orc &o, G gather, S scatter) {
    int q = o.tid();
    cplx *cb = o.cbuf[q].data();
    double *rb = o.rbuf[q].data();
    for (int k = 1; k <= o.mz; ++k)
        for (int j = 1; j <= o.my2; ++j) cb[(j - 1) + (size_t)o.my2 * (k - 1)] = gather(j, k);
    o.ffts[q].c2r(cb, rb);
    for (int k = 1; k <= o.mz; ++k)
        for (int j = 1; j <= o.my; ++j) scatter(j, k, rb[(j - 1) + (size_t)o.my * (k - 1)]);
}
template <class G, class S>
void r2c_with(Orc &o, G gather, S scatter) {
    int q = o.tid();
    cplx *cb = o.cbuf[q].data();
    double *rb = o.rbuf[q].data();
    for (int k = 1; k <= o.mz; ++k)
        for (int j = 1; j <= o.my; ++j) rb[(j - 1) + (size_t)o.my * (k - 1)] = gather(j, k);
    o.ffts[q].r2c(rb, cb);
    for (int k = 1; k <= o.mz; ++k)
        for (int j = 1; j <= o.my2; ++j) scatter(j, k, cb[(j - 1) + (size_t)o.my2 * (k - 1)]);
}

// ============================================================================
// compute_new_timestep (+ calc_pressure): dependent_functions.F90:1054-1288, 298-351.
// ============================================================================
void compute_new_timestep(Orc &o, int rks) {
    const int nx = o.nx, my = o.my, mz = o.mz;
    std::vector<double> part((size_t)nx * 12, 0.0);   // per plane: uf(3) us(3) um(3) max(3)
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; ++i) {
        for (int n = 1; n <= 3; ++n)
            c2r_with(o, [&](int j, int k) { return o.u[o.CI(i, j, k, n)]; },
                     [&](int j, int k, double v) { o.ubcp[o.RI(i, j, k, n)] = v; });
        double *pp = &part[(size_t)(i - 1) * 12];
        pp[9] = pp[10] = pp[11] = SMALL_NUMBER;
        for (int k = 1; k <= mz; ++k)
            for (int j = 1; j <= my; ++j) {
                double v[3];
                for (int n = 1; n <= 3; ++n) { double &r = o.ubcp[o.RI(i, j, k, n)]; r = r + o.umean[n - 1]; v[n - 1] = r; }
                if (o.FL(i, j, k)) { for (int d = 0; d < 3; ++d) pp[d] = pp[d] + v[d]; }
                else { for (int d = 0; d < 3; ++d) pp[3 + d] = pp[3 + d] + v[d]; }
                for (int d = 0; d < 3; ++d) pp[6 + d] = pp[6 + d] + v[d];
                for (int d = 0; d < 3; ++d) pp[9 + d] = std::max(pp[9 + d], std::fabs(v[d] - o.mesh_vel[d]));
            }
    }
    for (int n = 1; n <= 3; ++n)
        for (int k = 1; k <= mz; ++k)
            for (int j = 1; j <= my; ++j) o.ubcp[o.RI(o.mx, j, k, n)] = o.ubcp[o.RI(1, j, k, n)];
    double uf[3] = {0, 0, 0}, us[3] = {0, 0, 0}, um[3] = {0, 0, 0}, mx3[3] = {SMALL_NUMBER, SMALL_NUMBER, SMALL_NUMBER};
    for (int i = 1; i <= nx; ++i) {
        double *pp = &part[(size_t)(i - 1) * 12];
        for (int d = 0; d < 3; ++d) {
            uf[d] += pp[d]; us[d] += pp[3 + d]; um[d] += pp[6 + d]; mx3[d] = std::max(mx3[d], pp[9 + d]);
        }
    }
    double umax_tmp = std::max(std::max(mx3[0], mx3[1]), mx3[2]);
    o.umax_last = umax_tmp;
    double dtnew;
    if (umax_tmp * o.dt / o.dx > o.cfl_max) dtnew = o.cfl_max * o.dx / umax_tmp;
    else dtnew = o.dt;
    if (o.moving) {
        // particle speed limit (dependent_functions.F90:1156-1164); the new dt
        // is taken from the fluid speed, as the reference writes it
        double up_max = SMALL_NUMBER;
        for (int m = 1; m <= o.nbody; ++m) {
            double s2 = 0.0;
            for (int d = 1; d <= 3; ++d) s2 = s2 + o.VB(m, d) * o.VB(m, d);
            up_max = std::max(up_max, std::sqrt(s2));
        }
        if (up_max * o.dt / o.dx > o.cfl_max) dtnew = o.cfl_max * o.dx / umax_tmp;
    }
    double ufmean_temp[3];
    for (int d = 0; d < 3; ++d) ufmean_temp[d] = uf[d] / (double)o.count_fluid;
    for (int d = 0; d < 3; ++d) { o.ufmean_old[d] = o.ufmean[d]; o.ufmean[d] = ufmean_temp[d]; }
    for (int d = 0; d < 3; ++d) {
        double s = 0; for (int m = 1; m <= o.nbody; ++m) s = s + o.VB(m, d + 1);
        o.usmean_act[d] = o.nbody > 0 ? s / (double)o.nbody : 0.0;
        o.dufmeandt[d] = -o.cf * (o.ufmean[d] - o.ufmean_old[d]);
        o.meanslip[d] = (o.ufmean[d] - o.usmean_des[d]) * (1.0 - o.maxvolfrac);
    }
    o.meanslipmod = std::sqrt(o.meanslip[0] * o.meanslip[0] + o.meanslip[1] * o.meanslip[1] + o.meanslip[2] * o.meanslip[2]);
    // single phase: usmean = volfrac*mean_spec_vel/mean_volfrac (:1191-1205)
    double mixmeanslip[3];
    for (int d = 0; d < 3; ++d) {
        double msv = o.nbody > 0 ? o.usmean_act[d] : 0.0;
        o.usmean[d] = o.nbody > 0 ? (o.mean_volfrac * msv) / o.mean_volfrac : 0.0;
        mixmeanslip[d] = (1.0 - o.maxvolfrac) * (o.usmean[d] - o.ufmean[d]);
    }
    o.mixmeanslipmod = std::sqrt(mixmeanslip[0] * mixmeanslip[0] + mixmeanslip[1] * mixmeanslip[1] + mixmeanslip[2] * mixmeanslip[2]);
    // calc_pressure
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; ++i)
        c2r_with(o, [&](int j, int k) { return o.p[o.PI3(i, j, k)]; },
                 [&](int j, int k, double v) { o.pbcp[o.QI(i, j, k, 1)] = v; });
    if (rks == o.itrmax && o.prm.adaptive) o.dt = dtnew;
    o.t = o.t + o.dt * (o.coef[0] + o.coef[1]);
    double utemp = o.ucharmod;
    double tempt = o.ramp_frac_time * (double)(float)(o.mx - 1) * o.dx / utemp;
    if (o.t < tempt) { o.cf = -1.0 / o.dt; o.cforig = o.cf; o.cf = o.cf * (o.t / tempt); }
    else { o.cf = -1.0 / o.dt; o.cforig = o.cf; }
}

// ============================================================================
// form_nl: SRC/FLO/nl_allflow.F90:71-327 (serial branch).  fdderiv is a
// private array here (the reference aliases it on fr, which bcset re-zeroes).
// ============================================================================
void form_nl(Orc &o) {
    const int nx = o.nx, my = o.my, mz = o.mz, mxf = o.mxf;
    const bool center = o.prm.discr_scheme == PIBM_SCHEME_CENTER;
    const bool upwind = o.prm.discr_scheme == PIBM_SCHEME_UPWIND;
    const double *mv = o.mesh_vel;
    std::vector<double> fd((size_t)(nx + 1) * my * mz * 3, 0.0);
    auto FD = [&](int i, int j, int k, int n) -> double & { return fd[o.RI(i, j, k, n)]; };
    auto U = [&](int i, int j, int k, int n) { return o.ubcp[o.RI(i, j, k, n)]; };
    // products, y/z spectral derivatives
#pragma omp parallel
    {
        std::vector<cplx> f22((size_t)o.my2 * mz), f33((size_t)o.my2 * mz), f12((size_t)o.my2 * mz), f13((size_t)o.my2 * mz), f23((size_t)o.my2 * mz);
#pragma omp for schedule(static)
        for (int i = 1; i <= nx; ++i) {
            auto sp = [&](int a, int b, std::vector<cplx> &dst) {
                r2c_with(o, [&](int j, int k) { return (U(i, j, k, a) - mv[a - 1]) * (U(i, j, k, b) - mv[b - 1]); },
                         [&](int j, int k, cplx v) { dst[(j - 1) + (size_t)o.my2 * (k - 1)] = v; });
            };
            sp(2, 2, f22); sp(3, 3, f33); sp(1, 2, f12); sp(1, 3, f13); sp(2, 3, f23);
            for (int k = 1; k <= mz; ++k)
                for (int j = 1; j <= o.my2; ++j) {
                    size_t q = (j - 1) + (size_t)o.my2 * (k - 1);
                    cplx wy = o.wy[j - 1], wz = o.wz[k - 1];
                    o.nl[o.CI(i, j, k, 1)] = wy * f12[q] + wz * f13[q];
                    o.nl[o.CI(i, j, k, 2)] = wy * f22[q] + wz * f23[q];
                    o.nl[o.CI(i, j, k, 3)] = wy * f23[q] + wz * f33[q];
                }
            for (int k = 1; k <= mz; ++k)
                for (int j = 1; j <= my; ++j) {
                    if (center) {
                        double u1 = U(i, j, k, 1) - mv[0];
                        FD(i, j, k, 1) = u1 * u1;
                        FD(i, j, k, 2) = (U(i, j, k, 1) - mv[0]) * (U(i, j, k, 2) - mv[1]);
                        FD(i, j, k, 3) = (U(i, j, k, 1) - mv[0]) * (U(i, j, k, 3) - mv[2]);
                    } else {
                        FD(i, j, k, 1) = FD(i, j, k, 2) = FD(i, j, k, 3) = 0.0;
                    }
                }
        }
    }
    if (center)
        for (int n = 1; n <= 3; ++n) for (int k = 1; k <= mz; ++k) for (int j = 1; j <= my; ++j) FD(o.mx, j, k, n) = FD(1, j, k, n);
    if (upwind) {
        const bool minmod = o.prm.limiter == PIBM_LIMITER_MINMOD;
        const double dx = o.dx;
#pragma omp parallel
        {
            std::vector<double> uplus(nx + 1), uminus(nx + 1), Up(nx + 1), Um(nx + 1), slope(nx + 1);
#pragma omp for schedule(static)
            for (int k = 1; k <= mz; ++k)
                for (int j = 1; j <= my; ++j) {
                    double phi_ri = 1.0;
                    for (int idim = 1; idim <= 3; ++idim) {
                        for (int i = 1; i <= nx; ++i) {
                            int im1 = i - 1, ip1 = i + 1;
                            if (im1 < 1) im1 = mxf + im1 - 1;
                            if (ip1 > mxf - 1) ip1 = ip1 - (mxf - 1);
                            slope[i] = (U(ip1, j, k, idim) - U(im1, j, k, idim)) / (2.0 * dx);
                            if (!minmod) phi_ri = 1.0;
                            else {
                                phi_ri = (U(i, j, k, idim) - U(im1, j, k, idim)) / (U(ip1, j, k, idim) - U(i, j, k, idim) + SMALL_NUMBER);
                                if (phi_ri <= 0.0) phi_ri = 0.0; else phi_ri = std::min(1.0, phi_ri);
                            }
                            slope[i] = slope[i] * phi_ri * 1.0;
                            if (idim == 1) {
                                uplus[im1] = U(i, j, k, idim) - slope[i] * (dx / 2.0);
                                uminus[i] = U(i, j, k, idim) + slope[i] * (dx / 2.0);
                                Up[im1] = uplus[im1];
                                Um[i] = uminus[i];
                            } else {
                                Up[im1] = U(i, j, k, idim) - slope[i] * (dx / 2.0);
                                Um[i] = U(i, j, k, idim) + slope[i] * (dx / 2.0);
                            }
                            FD(im1, j, k, idim) = FD(im1, j, k, idim) + 0.5 * (uplus[im1] - mv[0]) * (Up[im1] - mv[idim - 1]);
                            FD(i, j, k, idim) = FD(i, j, k, idim) + 0.5 * (uminus[i] - mv[0]) * (Um[i] - mv[idim - 1]);
                            if (i != 1) {
                                double ms = std::max(std::fabs(uminus[im1] - mv[0]), std::fabs(uplus[im1] - mv[0]));
                                FD(im1, j, k, idim) = FD(im1, j, k, idim) - 0.5 * ms * (Up[im1] - Um[im1]);
                            }
                        }
                        double ms = std::max(std::fabs(uminus[nx] - mv[0]), std::fabs(uplus[nx] - mv[0]));
                        FD(nx, j, k, idim) = FD(nx, j, k, idim) - 0.5 * ms * (Up[nx] - Um[nx]);
                        FD(o.mx, j, k, idim) = FD(1, j, k, idim);
                    }
                }
        }
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; ++i)
        for (int idim = 1; idim <= 3; ++idim) {
            int im1 = i - 1, ip1 = i + 1;
            if (im1 < 1) im1 = mxf + im1 - 1;
            if (ip1 > mxf - 1) ip1 = ip1 - (mxf - 1);
            r2c_with(o, [&](int j, int k) {
                         if (center) return (FD(ip1, j, k, idim) - FD(im1, j, k, idim)) / (2.0 * o.dx);
                         return (FD(i, j, k, idim) - FD(im1, j, k, idim)) / o.dx; },
                     [&](int j, int k, cplx v) { cplx &d = o.nl[o.CI(i, j, k, idim)]; d = d + v; });
        }
    for (int n = 1; n <= 3; ++n)
        for (int k = 1; k <= mz; ++k)
            for (int j = 1; j <= o.my2; ++j) o.nl[o.CI(nx + 1, j, k, n)] = o.nl[o.CI(1, j, k, n)];
}

// ============================================================================
// bcset helpers: calc_visc, compute_omega, calc_pgrad (boundary_condition.F90:1648-1896).
// ============================================================================
void calc_visc(Orc &o) {
    const int nx = o.nx;
    const double rdx2 = 1.0 / o.dx2;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx + 1; ++i)
        for (int n = 1; n <= 3; ++n) {
            int im = i - 1, ip = i + 1;
            if (i == 1) im = nx;
            if (i == nx + 1) ip = 2;
            c2r_with(o, [&](int j, int k) {
                         cplx f = rdx2 * ((o.u[o.CI(im, j, k, n)] - 2.0 * o.u[o.CI(i, j, k, n)]) + o.u[o.CI(ip, j, k, n)]);
                         f = f - o.W2(j, k) * o.u[o.CI(i, j, k, n)];
                         return f * o.vis; },
                     [&](int j, int k, double v) { o.diffn[o.RI(i, j, k, n)] = v; });
        }
}

void compute_omega(Orc &o) {
    const int nx = o.nx, mxf = o.mxf;
    const double tdx = 2.0 * o.dx;
    auto U = [&](int i, int j, int k, int n) { return o.ubcp[o.RI(i, j, k, n)]; };
#pragma omp parallel
    {
        std::vector<double> a((size_t)o.my * o.mz), b((size_t)o.my * o.mz);
#pragma omp for schedule(static)
        for (int i = 1; i <= nx + 1; ++i) {
            int ip = i + 1, im = i - 1;
            if (i == 1) { ip = 2; im = mxf - 1; }
            if (i == mxf) { ip = 2; im = mxf - 1; }
            // omega3 = dv/dx - du/dy
            c2r_with(o, [&](int j, int k) { return o.wy[j - 1] * o.u[o.CI(i, j, k, 1)]; },
                     [&](int j, int k, double v) { a[(j - 1) + (size_t)o.my * (k - 1)] = v; });
            for (int k = 1; k <= o.mz; ++k) for (int j = 1; j <= o.my; ++j)
                o.omega[o.RI(i, j, k, 3)] = (U(ip, j, k, 2) - U(im, j, k, 2)) / tdx - a[(j - 1) + (size_t)o.my * (k - 1)];
            // omega2 = du/dz - dw/dx
            c2r_with(o, [&](int j, int k) { return o.wz[k - 1] * o.u[o.CI(i, j, k, 1)]; },
                     [&](int j, int k, double v) { a[(j - 1) + (size_t)o.my * (k - 1)] = v; });
            for (int k = 1; k <= o.mz; ++k) for (int j = 1; j <= o.my; ++j)
                o.omega[o.RI(i, j, k, 2)] = a[(j - 1) + (size_t)o.my * (k - 1)] - (U(ip, j, k, 3) - U(im, j, k, 3)) / tdx;
            // omega1 = dw/dy - dv/dz
            c2r_with(o, [&](int j, int k) { return o.wz[k - 1] * o.u[o.CI(i, j, k, 2)]; },
                     [&](int j, int k, double v) { a[(j - 1) + (size_t)o.my * (k - 1)] = v; });
            c2r_with(o, [&](int j, int k) { return o.wy[j - 1] * o.u[o.CI(i, j, k, 3)]; },
                     [&](int j, int k, double v) { b[(j - 1) + (size_t)o.my * (k - 1)] = v; });
            for (int k = 1; k <= o.mz; ++k) for (int j = 1; j <= o.my; ++j) {
                size_t q = (j - 1) + (size_t)o.my * (k - 1);
                o.omega[o.RI(i, j, k, 1)] = b[q] - a[q];
            }
        }
    }
}

void calc_pgrad(Orc &o) {
    const int nx = o.nx;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; ++i) {
        int ip = i + 1, im = i - 1;
        if (i == 1) im = nx;
        if (i == nx) ip = 1;
        c2r_with(o, [&](int j, int k) { return (o.p[o.PI3(ip, j, k)] - o.p[o.PI3(im, j, k)]) / (2.0 * o.dx); },
                 [&](int j, int k, double v) { o.ppr[o.QI(i, j, k, 1)] = v + o.mpg[0]; });
        c2r_with(o, [&](int j, int k) { return o.p[o.PI3(i, j, k)] * o.wy[j - 1]; },
                 [&](int j, int k, double v) { o.ppr[o.QI(i, j, k, 2)] = v + o.mpg[1]; });
        c2r_with(o, [&](int j, int k) { return o.p[o.PI3(i, j, k)] * o.wz[k - 1]; },
                 [&](int j, int k, double v) { o.ppr[o.QI(i, j, k, 3)] = v + o.mpg[2]; });
    }
}

// ============================================================================
// Interpolation: set_interpolation_stencil / _pstencil ('lpi', order 2),
// interpolate_udata / interpolate_pdata and interp_threed_* with shape2
// (dependent_functions.F90:45-158,612-781; interpolation.F90:202-381,740-751).
// For order 2 with periodic y,z (and x) the stencil is always [pc, pc+1].
// ============================================================================
struct Stencil {
    int ib, jb, kb;
    int ii[2], jj[2], kk[2];   // wrapped indices
    double w[2][2][2];         // weights(i,j,k)
};

inline void make_stencil(const Orc &o, const int pc[3], const double pos[3], int im_x, Stencil &s) {
    // set_interpolation_stencil / _pstencil: lpi, order 2, ob2l = ob2r = 1
    int ib = std::max(1, pc[0]), ie = std::min(im_x, pc[0] + 1);
    if (ib == 1) ib = ie - 2 + 1;
    if (ie == im_x) ie = ib + 2 - 1;
    int jb = std::max(1, pc[1]), je = std::min(o.my, pc[1] + 1);
    if (jb == 1) jb = je - 2 + 1;
    if (je == o.my) je = jb + 2 - 1;
    int kb = std::max(1, pc[2]), ke = std::min(o.mz, pc[2] + 1);
    if (kb == 1) kb = ke - 2 + 1;
    if (ke == o.mz) ke = kb + 2 - 1;
    s.ib = ib; s.jb = jb; s.kb = kb;
    for (int q = 0; q < 2; ++q) {
        int ii = ib + q, jj = jb + q, kk = kb + q;
        if (ii < 1) ii = o.mxf + ii - 1;
        if (ii > o.mxf - 1) ii = ii - o.mxf + 1;
        if (jj < 1) jj = o.my + jj;
        if (jj > o.my) jj = jj - o.my;
        if (kk < 1) kk = o.mz + kk;
        if (kk > o.mz) kk = kk - o.mz;
        s.ii[q] = ii; s.jj[q] = jj; s.kk[q] = kk;
    }
    // interp_threed_scalar: zeta = ppos - coor(1); dx(1) = coor(2)-coor(1) = 1
    double zx = (pos[0] - (double)ib) / (double)((ib + 1) - ib);
    double zy = (pos[1] - (double)jb) / (double)((jb + 1) - jb);
    double zz = (pos[2] - (double)kb) / (double)((kb + 1) - kb);
    double xv[2] = {1.0 - zx, zx}, yv[2] = {1.0 - zy, zy}, zv[2] = {1.0 - zz, zz};
    for (int k = 0; k < 2; ++k) for (int j = 0; j < 2; ++j) for (int i = 0; i < 2; ++i) s.w[i][j][k] = xv[i] * yv[j] * zv[k];
}

// interpolator (k, j, i loop order, accumulator starts at 0.0)
template <class F>
inline double interp_kji(const Stencil &s, F val) {
    double r = 0.0;
    for (int k = 0; k < 2; ++k) for (int j = 0; j < 2; ++j) for (int i = 0; i < 2; ++i) r = r + val(s.ii[i], s.jj[j], s.kk[k]) * s.w[i][j][k];
    return r;
}
// array_dot_product_3d (i, j, k loop order)
template <class F>
inline double dot_ijk(const Stencil &s, F val) {
    double r = 0.0;
    for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) for (int k = 0; k < 2; ++k) r = r + val(s.ii[i], s.jj[j], s.kk[k]) * s.w[i][j][k];
    return r;
}

inline int cell_of(double x) { return x < 0.0 ? fint(x - 1) : fint(x); }

// ============================================================================
// compute_mpg_at_n + calc_pres_visc_drag: boundary_condition.F90:302-464, 1481-1645.
// ============================================================================
void compute_mpg_at_n(Orc &o, int rks) {
    (void)rks;
    compute_omega(o);
    for (int d = 0; d < 3; ++d) { o.pres_total[d] = 0; o.visc_total[d] = 0; }
    for (int m = 1; m <= o.nbody; ++m) {
        double presm[3] = {0, 0, 0}, viscm[3] = {0, 0, 0};
        double rb = o.radbdy[m - 1];
        double da1 = 4.0 * PI * ((rb * o.dx) * (rb * o.dx)) / (double)o.nbnd;
        for (int l = 1; l <= o.nbnd; ++l) {
            double xl[3], xpb[3];
            for (int n = 1; n <= 3; ++n) xl[n - 1] = o.XC(m, n) + o.BND(n, l) * rb;
            xpb[0] = xl[0] - 0.5; xpb[1] = xl[1]; xpb[2] = xl[2];
            int pcell[3], vcell[3];
            for (int n = 0; n < 3; ++n) { pcell[n] = cell_of(xpb[n]); vcell[n] = cell_of(xl[n]); }
            Stencil sp, sv;
            make_stencil(o, pcell, xpb, o.mxf - 1, sp);
            double pl = dot_ijk(sp, [&](int i, int j, int k) { return o.pbcp[o.QI(i, j, k, 1)]; });
            make_stencil(o, vcell, xl, o.mxf, sv);
            double vort[3] = {0, 0, 0};
            for (int k = 0; k < 2; ++k) for (int j = 0; j < 2; ++j) for (int i = 0; i < 2; ++i)
                for (int n = 1; n <= 3; ++n) vort[n - 1] = vort[n - 1] + sv.w[i][j][k] * o.omega[o.RI(sv.ii[i], sv.jj[j], sv.kk[k], n)];
            double df[3];
            df[0] = vort[2] * o.CD(2, l); df[0] = df[0] - vort[1] * o.CD(3, l);
            df[1] = vort[0] * o.CD(3, l); df[1] = df[1] - vort[2] * o.CD(1, l);
            df[2] = vort[1] * o.CD(1, l); df[2] = df[2] - vort[0] * o.CD(2, l);
            for (int d = 0; d < 3; ++d) df[d] = -df[d];
            for (int d = 1; d <= 3; ++d) {
                presm[d - 1] = presm[d - 1] - pl * o.CD(d, l) * da1;
                o.pres_total[d - 1] = o.pres_total[d - 1] + pl * o.CD(d, l) * da1;
                viscm[d - 1] = viscm[d - 1] + df[d - 1] * o.vis * da1;
                o.visc_total[d - 1] = o.visc_total[d - 1] + df[d - 1] * o.vis * da1;
            }
        }
        for (int d = 0; d < 3; ++d) { o.pres[(m - 1) + (size_t)o.nbody * d] = presm[d]; o.visc[(m - 1) + (size_t)o.nbody * d] = viscm[d]; }
    }
    double pa[3], va[3];
    for (int d = 0; d < 3; ++d) {
        double s = 0, v = 0;
        for (int m = 0; m < o.nbody; ++m) { s = s + o.pres[m + (size_t)o.nbody * d]; v = v + o.visc[m + (size_t)o.nbody * d]; }
        pa[d] = s; va[d] = v;
    }
    double norm_factor = (3.0 * PI * o.vis * (o.mixmeanslipmod + SMALL_NUMBER) * o.char_length) * (double)o.nbody;
    o.pres_drag = std::sqrt(pa[0] * pa[0] + pa[1] * pa[1] + pa[2] * pa[2]) / norm_factor / (1.0 - o.maxvolfrac);
    o.visc_drag = std::sqrt(va[0] * va[0] + va[1] * va[1] + va[2] * va[2]) / norm_factor / (1.0 - o.maxvolfrac);
    o.total_drag = o.pres_drag + o.visc_drag;
    const double rhof = o.prm.rhof, rhos = o.prm.rhos, mvf = o.mean_volfrac;
    if (!o.prm.set_mpg) {
        if (o.moving) {
            for (int d = 0; d < 3; ++d) {
                double g = o.cf * (o.ufmean_des[d] - o.ufmean[d]) + o.cf * (o.usmean[d] - o.usmean_des[d]);
                g = g + (o.pres_total[d] - (o.visc_total[d])) * (1.0 / (rhof * (1.0 - mvf)) + 1.0 / (mvf * rhos)) / o.voldom;
                g = g / (1.0 / rhof - 1.0 / rhos);
                o.mpg[d] = g;
                o.frame_accln[d] = -o.mpg[d] / rhos - (o.pres_total[d] - o.visc_total[d]) / (mvf * rhos * o.voldom) + o.cf * (o.usmean_des[d] - o.usmean[d]);
            }
        } else {
            for (int d = 0; d < 3; ++d)
                o.mpg[d] = o.cf * (o.ufmean_des[d] - o.ufmean[d]) + (o.pres_total[d] / o.voldom - (o.visc_total[d]) / o.voldom) / (1.0 - o.maxvolfrac);
        }
        if (o.prm.include_frmeanfluid)
            for (int d = 0; d < 3; ++d) o.mpg[d] = o.mpg[d] + o.frmeanfluid[d];
    } else if (o.moving) {
        for (int d = 0; d < 3; ++d)
            o.frame_accln[d] = -o.mpg[d] / rhos - (o.pres_total[d] - o.visc_total[d]) / (mvf * rhos * o.voldom) + o.cf * (o.usmean_des[d] - o.usmean[d]);
    }
    const double c12 = o.coef[0] + o.coef[1];
    for (int m = 1; m <= o.nbody; ++m) {
        double vol = PI * std::pow(2.0 * o.radbdy[m - 1] * o.dx, 3.0) / 6.0;
        for (int d = 0; d < 3; ++d) {
            size_t q = (m - 1) + (size_t)o.nbody * d;
            o.force[q] = c12 * (o.pres[q] + o.visc[q]) - c12 * o.mpg[d] * vol;
        }
    }
}

// ============================================================================
// calc_inner_reversal_forcing: boundary_condition.F90:1104-1479 (serial branch).
// ============================================================================
void calc_inner_reversal_forcing(Orc &o, int m, double da2) {
    const double rb = o.radbdy[m - 1], ri = o.radibdy[m - 1], ro = o.radobdy[m - 1];
    const double drm = o.prm.dr;
    const double dx3 = std::pow(o.dx, 3.0);
    const double c12 = o.coef[0] + o.coef[1];
    for (int l = 1; l <= o.nrpr; ++l) {
        if (!o.if_rev[(size_t)(l - 1) + (size_t)o.nbnd * (m - 1)]) continue;
        double xli[3], xlo[3], rad = 0.0, snorm[3], xpi[3];
        for (int n = 1; n <= 3; ++n) {
            xli[n - 1] = o.XC(m, n) + o.BND(n, l) * ri;
            xlo[n - 1] = o.XC(m, n) + o.BND(n, l) * ro;
            double a = o.BND(n, l) * ri;
            rad = rad + a * a;
        }
        rad = std::sqrt(rad);
        for (int n = 0; n < 3; ++n) snorm[n] = (o.BND(n + 1, l) * ri) / rad;
        xpi[0] = xli[0] - 0.5; xpi[1] = xli[1]; xpi[2] = xli[2];
        int vcello[3], pcelli[3], vcelli[3];
        for (int n = 0; n < 3; ++n) { vcello[n] = cell_of(xlo[n]); pcelli[n] = cell_of(xpi[n]); vcelli[n] = cell_of(xli[n]); }
        // outer velocity
        Stencil so, spi, si;
        make_stencil(o, vcello, xlo, o.mxf, so);
        double ulo[3];
        for (int n = 1; n <= 3; ++n) ulo[n - 1] = interp_kji(so, [&](int i, int j, int k) { return o.ubcp[o.RI(i, j, k, n)]; });
        // inner pressure point: ppr (includes mpg)
        make_stencil(o, pcelli, xpi, o.mxf - 1, spi);
        double ppll[3];
        for (int n = 1; n <= 3; ++n) ppll[n - 1] = interp_kji(spi, [&](int i, int j, int k) { return o.ppr[o.QI(i, j, k, n)]; });
        // inner velocity point
        make_stencil(o, vcelli, xli, o.mxf, si);
        double uli[3], nll[3], onll[3], dfll[3];
        for (int n = 1; n <= 3; ++n) {
            uli[n - 1] = interp_kji(si, [&](int i, int j, int k) { return o.ubcp[o.RI(i, j, k, n)]; });
            nll[n - 1] = dot_ijk(si, [&](int i, int j, int k) { return o.nlbc[o.RI(i, j, k, n)]; });
            onll[n - 1] = dot_ijk(si, [&](int i, int j, int k) { return o.onlbc[o.RI(i, j, k, n)]; });
            dfll[n - 1] = dot_ijk(si, [&](int i, int j, int k) { return o.diffn[o.RI(i, j, k, n)]; });
        }
        double unmag = 0.0, ubnmag = 0.0, linvel[3];
        for (int d = 0; d < 3; ++d) linvel[d] = o.VB(m, d + 1) + 0.0 * rb * o.dx;  // angv = 0
        for (int d = 0; d < 3; ++d) { unmag = unmag + snorm[d] * ulo[d]; ubnmag = ubnmag + snorm[d] * linvel[d]; }
        double ucar[3];
        for (int d = 0; d < 3; ++d) {
            double unorm = snorm[d] * unmag;
            double utang = ulo[d] - unorm;
            double ubnorm = snorm[d] * ubnmag;
            double ubtang = linvel[d] - ubnorm;
            double utangi = ubtang * (ro - ri) - utang * (rb - ri);
            utangi = utangi / (ro - rb);
            double unormi = 0.0;
            if (o.prm.revernorm == 1) { unormi = ubnorm * (ro - ri) - unorm * (rb - ri); unormi = unormi / (ro - rb); }
            ucar[d] = utangi + unormi;
        }
        double ft[3];
        for (int n = 0; n < 3; ++n) {
            ft[n] = o.cf * (-ucar[n] + uli[n]);
            ft[n] = ft[n] - o.coef[2] * nll[n] - o.coef[3] * onll[n];
            ft[n] = ft[n] + c12 * (ppll[n] - dfll[n]);
            ft[n] = ft[n] * da2 * drm * o.dx;
        }
        int count_fl = 0;
        double force_fl[3] = {0, 0, 0};
        for (int k = 0; k < 2; ++k) for (int j = 0; j < 2; ++j) for (int i = 0; i < 2; ++i)
            if (o.FL(si.ii[i], si.jj[j], si.kk[k])) {
                count_fl += 1;
                for (int n = 0; n < 3; ++n) { double tmppa = si.w[i][j][k] * ft[n]; force_fl[n] = force_fl[n] + tmppa / dx3; }
            }
        int count_so = 8 - count_fl;
        double force_dist[3];
        for (int n = 0; n < 3; ++n) force_dist[n] = count_so > 0 ? force_fl[n] / (double)(float)count_so : 0.0;
        for (int k = 0; k < 2; ++k) for (int j = 0; j < 2; ++j) for (int i = 0; i < 2; ++i) {
            int ii = si.ii[i], jj = si.jj[j], kk = si.kk[k];
            bool isfl = o.FL(ii, jj, kk);
            for (int n = 1; n <= 3; ++n) {
                double tmppa = si.w[i][j][k] * ft[n - 1];
                double &f = o.fr[o.RI(ii, jj, kk, n)];
                if (o.prm.include_frmeanfluid) {
                    if (isfl) o.frmeanfluid[n - 1] = o.frmeanfluid[n - 1] + tmppa / dx3;
                    f = f + tmppa / dx3;
                } else if (!isfl) {
                    f = f + tmppa / dx3 + force_dist[n - 1];
                }
                o.frmean[n - 1] = o.frmean[n - 1] + tmppa / dx3;
            }
        }
    }
}

// ============================================================================
// bcset: boundary_condition.F90:467-900 (fixed particles, dorpr, not dobnd).
// ============================================================================
int bcset(Orc &o, int rks) {
    calc_visc(o);
    compute_mpg_at_n(o, rks);
    if (o.moving) {
        const int rc = des_time_march(o);
        if (rc) return rc;
        grid_nodes_insphere(o);
        update_nrpr(o);
    }
    calc_pgrad(o);
    std::fill(o.fr.begin(), o.fr.end(), 0.0);
    for (int d = 0; d < 3; ++d) { o.frmean[d] = 0; o.frmeanfluid[d] = 0; }
    for (int m = 1; m <= o.nbody; ++m) {
        double da2 = 4.0 * PI * ((o.radibdy[m - 1] * o.dx) * (o.radibdy[m - 1] * o.dx)) / (double)o.nrpr_active[m - 1];
        if (o.prm.dorpr) calc_inner_reversal_forcing(o, m, da2);
    }
    for (int d = 0; d < 3; ++d) {
        o.frmean[d] = o.frmean[d] / (double)((long long)o.nx * o.my * o.mz);
        o.frmeanfluid[d] = o.frmeanfluid[d] / (double)o.count_fluid;
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= o.nx; ++i)
        for (int n = 1; n <= 3; ++n)
            r2c_with(o, [&](int j, int k) { return o.fr[o.RI(i, j, k, n)] - o.frmean[n - 1]; },
                     [&](int j, int k, cplx v) { o.ff[o.CI(i, j, k, n)] = v; });
    for (int n = 1; n <= 3; ++n)
        for (int k = 1; k <= o.mz; ++k)
            for (int j = 1; j <= o.my2; ++j) o.ff[o.CI(o.nx + 1, j, k, n)] = o.ff[o.CI(1, j, k, n)];
    // diagnostics: :701-841 (single phase)
    double avg[3];
    for (int d = 0; d < 3; ++d) {
        double s = 0; for (int m = 0; m < o.nbody; ++m) s = s + o.force[m + (size_t)o.nbody * d];
        avg[d] = (s / o.nbody) * o.mean_volfrac / o.mean_volfrac;
    }
    double nd = std::sqrt(avg[0] * avg[0] + avg[1] * avg[1] + avg[2] * avg[2]);
    double nf = (3.0 * PI * o.vis * o.ucharmod * o.char_length);
    if (o.prm.set_mpg) nf = (3.0 * PI * o.vis * (o.mixmeanslipmod + SMALL_NUMBER) * o.char_length);
    o.norm_drag = nd / nf;
    o.ferror = o.norm_drag > 0.0 ? std::fabs(o.norm_drag - o.fold) / o.norm_drag : 1.0;
    o.fold = o.norm_drag;
    for (int q = o.nerr_steps - 1; q >= 1; --q) o.ferror_array[q] = o.ferror_array[q - 1];
    o.ferror_array[0] = o.ferror;
    if (o.norm_drag > 1.0E+06) return PIBM_ERR_BLOWUP;
    return PIBM_OK;
}

int nonlinear(Orc &o, int rks) {
    o.onl = o.nl;
    std::fill(o.nl.begin(), o.nl.end(), cplx(0.0, 0.0));
    form_nl(o);
    for (auto &v : o.nl) v = -v;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= o.nx + 1; ++i)
        for (int n = 1; n <= 3; ++n) {
            c2r_with(o, [&](int j, int k) { return o.nl[o.CI(i, j, k, n)]; },
                     [&](int j, int k, double v) { o.nlbc[o.RI(i, j, k, n)] = v; });
            c2r_with(o, [&](int j, int k) { return o.onl[o.CI(i, j, k, n)]; },
                     [&](int j, int k, double v) { o.onlbc[o.RI(i, j, k, n)] = v; });
        }
    if (o.nbody > 0) return bcset(o, rks);
    return PIBM_OK;
}

// ============================================================================
// Tridiagonal solvers: tridag / tridag3 (tridiagonal.F90:47-150).
// ============================================================================
bool tridag(const double *a, const double *b, const double *c, const double *r, double *u, int n, double *gam) {
    for (int i = 0; i < n; ++i) u[i] = 0.0;
    if (b[0] == 0.0) return false;
    double bet = b[0];
    u[0] = r[0] / bet;
    for (int j = 1; j < n; ++j) {
        gam[j] = c[j - 1] / bet;
        bet = b[j] - a[j] * gam[j];
        if (bet == 0.0) return false;
        u[j] = (r[j] - a[j] * u[j - 1]) / bet;
    }
    for (int j = n - 2; j >= 0; --j) u[j] = u[j] - gam[j + 1] * u[j + 1];
    return true;
}
bool tridag3(const double *a, const double *b, const double *c, const double *r1, const double *r2, const double *r3,
             double *u1, double *u2, double *u3, int n, double *gam) {
    if (b[0] == 0.0) return false;
    double bet = b[0];
    u1[0] = r1[0] / bet; u2[0] = r2[0] / bet; u3[0] = r3[0] / bet;
    for (int j = 1; j < n; ++j) {
        gam[j] = c[j - 1] / bet;
        bet = b[j] - a[j] * gam[j];
        if (bet == 0.0) return false;
        u1[j] = (r1[j] - a[j] * u1[j - 1]) / bet;
        u2[j] = (r2[j] - a[j] * u2[j - 1]) / bet;
        u3[j] = (r3[j] - a[j] * u3[j - 1]) / bet;
    }
    for (int j = n - 2; j >= 0; --j) {
        u1[j] = u1[j] - gam[j + 1] * u1[j + 1];
        u2[j] = u2[j] - gam[j + 1] * u2[j + 1];
        u3[j] = u3[j] - gam[j + 1] * u3[j + 1];
    }
    return true;
}

// Cyclic solve via Sherman-Morrison as in pressure/ustep/divcorr
// (poisson.F90:144-182, usteptime.F90:344-349,431-470).  b is modified.
bool cyclic_solve(int nx, const double *a, double *b, const double *c, const double *rr, const double *ri,
                  double *outr, double *outi, double *auxz, double *gam) {
    std::vector<double> auxu(nx, 0.0), auxv(nx, 0.0);
    auxu[0] = 1.0; auxu[nx - 1] = 1.0;
    auxv[0] = c[nx - 1] / auxu[nx - 1];
    auxv[nx - 1] = a[0] / auxu[0];
    b[0] = b[0] - auxu[0] * auxv[0];
    b[nx - 1] = b[nx - 1] - auxu[nx - 1] * auxv[nx - 1];
    if (!tridag3(a, b, c, rr, auxu.data(), ri, outr, auxz, outi, nx, gam)) return false;
    double vdotz = auxv[0] * auxz[0] + auxv[nx - 1] * auxz[nx - 1];
    double vdotyr = auxv[0] * outr[0] + auxv[nx - 1] * outr[nx - 1];
    double vdotyi = auxv[0] * outi[0] + auxv[nx - 1] * outi[nx - 1];
    for (int i = 0; i < nx; ++i) {
        outr[i] = outr[i] - vdotyr * auxz[i] / (1.0 + vdotz);
        outi[i] = outi[i] - vdotyi * auxz[i] / (1.0 + vdotz);
    }
    return true;
}

// velstep: pressure -> ustep -> divcorr per (j,k) line, then check_divergence
// and the umean update (steptheflow.F90:52-160, poisson.F90:55-508,
// usteptime.F90:45-269).  Lines are independent, so each line runs all three.
int velstep(Orc &o, int rks) {
    (void)rks;
    const int nx = o.nx, mz = o.mz, my2 = o.my2;
    const double dx = o.dx, dx2 = o.dx2, dt = o.dt, vis = o.vis;
    const double c1 = o.coef[0], c2 = o.coef[1], c3 = o.coef[2], c4 = o.coef[3];
    int bad = 0;
    std::vector<double> divline((size_t)my2 * mz, 0.0);
#pragma omp parallel
    {
        std::vector<double> a(nx), b(nx), c(nx), dv(nx), dvi(nx), outr(nx), outi(nx), auxz(nx), gam(nx);
        std::vector<cplx> r(nx), div(nx);
#pragma omp for schedule(static) collapse(2)
        for (int jj = 1; jj <= my2; ++jj)
            for (int kk = 1; kk <= mz; ++kk) {
                const int j = jj, k = kk;
                const double w2 = o.W2(j, k);
                const cplx wy = o.wy[j - 1], wz = o.wz[k - 1];
                auto NL = [&](int i, int n) { return o.nl[o.CI(i, j, k, n)]; };
                auto ONL = [&](int i, int n) { return o.onl[o.CI(i, j, k, n)]; };
                auto FF = [&](int i, int n) { return o.ff[o.CI(i, j, k, n)]; };
                auto Ur = [&](int i, int n) -> cplx & { return o.u[o.CI(i, j, k, n)]; };
                auto P = [&](int i) -> cplx & { return o.p[o.PI3(i, j, k)]; };
                // ---------------- pressure ----------------
                for (int i = 0; i < nx; ++i) { a[i] = 1.0 / dx2 - 0.25 * w2; b[i] = -2.0 / dx2 - 0.5 * w2; c[i] = 1.0 / dx2 - 0.25 * w2; }
                for (int i = 1; i <= nx; ++i) {
                    cplx tmpc(0.0, 0.0);
                    tmpc = tmpc + c3 * (NL(i + 1, 1) - NL(i, 1)) / dx + (FF(i + 1, 1) - FF(i, 1)) / dx;
                    tmpc = tmpc + c3 * wy * (NL(i + 1, 2) + NL(i, 2)) / 2.0 + wy * (FF(i + 1, 2) + FF(i, 2)) / 2.0;
                    tmpc = tmpc + c3 * wz * (NL(i + 1, 3) + NL(i, 3)) / 2.0 + wz * (FF(i + 1, 3) + FF(i, 3)) / 2.0;
                    tmpc = tmpc + c4 * (ONL(i + 1, 1) - ONL(i, 1)) / dx;
                    tmpc = tmpc + c4 * wy * (ONL(i + 1, 2) + ONL(i, 2)) / 2.0;
                    tmpc = tmpc + c4 * wz * (ONL(i + 1, 3) + ONL(i, 3)) / 2.0;
                    tmpc = 0.5 * (1.0 + 1.0) * tmpc;
                    dv[i - 1] = tmpc.real() / (c1 + c2);
                    dvi[i - 1] = tmpc.imag() / (c1 + c2);
                }
                if (j == 1 && k == 1) {
                    if (!tridag(a.data(), b.data(), c.data(), dv.data(), outr.data(), nx - 1, gam.data())) { bad = 1; }
                    outr[nx - 1] = 0.0;
                    for (int i = 0; i < nx; ++i) outi[i] = 0.0;
                } else {
                    if (!cyclic_solve(nx, a.data(), b.data(), c.data(), dv.data(), dvi.data(), outr.data(), outi.data(), auxz.data(), gam.data())) bad = 1;
                }
                for (int i = 1; i <= nx; ++i) { cplx tmpp(outr[i - 1], outi[i - 1]); P(i) = P(i) + 1.0 * (tmpp - P(i)); }
                // ---------------- ustep ----------------
                for (int i = 0; i < nx; ++i) {
                    a[i] = -(1.0 * dt * vis * c2 / dx2);
                    b[i] = 1.0 + dt * vis * c2 * (1.0 * 2.0 / dx2 + w2);
                    c[i] = -(1.0 * dt * vis * c2 / dx2);
                }
                {
                    // auxiliary Sherman-Morrison modification of b (shared across idim)
                    std::vector<double> bmod(b);
                    for (int idim = 1; idim <= 3; ++idim) {
                        for (int i = 1; i <= nx; ++i) {
                            cplx rv = Ur(i, idim) * (1.0 - dt * vis * c1 * w2);
                            rv = rv + dt * c3 * NL(i, idim) + dt * FF(i, idim);
                            rv = rv + dt * c4 * ONL(i, idim);
                            r[i - 1] = rv;
                        }
                        const double alp = dt * (c1 + c2);
                        for (int i = 2; i <= nx; ++i) {
                            cplx &rv = r[i - 1];
                            if (idim == 1) rv = rv - alp * (P(i) - P(i - 1)) / dx;
                            else if (idim == 2) rv = rv - alp * 0.5 * (P(i - 1) + P(i)) * wy;
                            else rv = rv - alp * 0.5 * (P(i - 1) + P(i)) * wz;
                            rv = rv + 1.0 * dt * vis * c1 * (Ur(i - 1, idim) + Ur(i + 1, idim) - 2.0 * Ur(i, idim)) / dx2;
                        }
                        {
                            cplx &rv = r[0];
                            if (idim == 1) rv = rv - alp * (P(1) - P(nx)) / dx;
                            else if (idim == 2) rv = rv - alp * 0.5 * (P(nx) + P(1)) * wy;
                            else rv = rv - alp * 0.5 * (P(nx) + P(1)) * wz;
                            rv = rv + 1.0 * dt * vis * c1 * (Ur(2, idim) - 2.0 * Ur(1, idim) + Ur(nx, idim)) / dx2;
                        }
                        for (int i = 0; i < nx; ++i) { dv[i] = r[i].real(); dvi[i] = r[i].imag(); }
                        std::vector<double> bb(bmod);
                        if (!cyclic_solve(nx, a.data(), bb.data(), c.data(), dv.data(), dvi.data(), outr.data(), outi.data(), auxz.data(), gam.data())) bad = 1;
                        for (int i = 1; i <= nx; ++i) Ur(i, idim) = cplx(outr[i - 1], outi[i - 1]);
                        Ur(nx + 1, idim) = Ur(1, idim);
                    }
                }
                // ---------------- divcorr ----------------
                const double alp = (c1 + c2) * dt;
                for (int i = 0; i < nx; ++i) { a[i] = 1.0 / dx2 - 0.25 * w2; b[i] = -2.0 / dx2 - 0.5 * w2; c[i] = 1.0 / dx2 - 0.25 * w2; }
                for (int i = 1; i <= nx; ++i) {
                    cplx tmpc = (Ur(i + 1, 1) - Ur(i, 1)) / dx;
                    tmpc = tmpc + 0.5 * wy * (Ur(i, 2) + Ur(i + 1, 2));
                    tmpc = tmpc + 0.5 * wz * (Ur(i, 3) + Ur(i + 1, 3));
                    dv[i - 1] = 0.5 * (1.0 + 1.0) * tmpc.real();
                    dvi[i - 1] = 0.5 * (1.0 + 1.0) * tmpc.imag();
                    dv[i - 1] = dv[i - 1] / alp;
                    dvi[i - 1] = dvi[i - 1] / alp;
                }
                if (j == 1 && k == 1) {
                    if (!tridag(a.data(), b.data(), c.data(), dv.data(), outr.data(), nx - 1, gam.data())) bad = 1;
                    outr[nx - 1] = 0.0;
                    for (int i = 0; i < nx; ++i) outi[i] = 0.0;
                } else {
                    if (!cyclic_solve(nx, a.data(), b.data(), c.data(), dv.data(), dvi.data(), outr.data(), outi.data(), auxz.data(), gam.data())) bad = 1;
                }
                for (int i = 0; i < nx; ++i) div[i] = cplx(outr[i], outi[i]);
                Ur(1, 1) = Ur(1, 1) - alp * (div[0] - div[nx - 1]) / dx;
                Ur(1, 2) = Ur(1, 2) - alp * wy * 0.5 * (div[0] + div[nx - 1]);
                Ur(1, 3) = Ur(1, 3) - alp * wz * 0.5 * (div[0] + div[nx - 1]);
                for (int i = 2; i <= nx; ++i) {
                    Ur(i, 1) = Ur(i, 1) - alp * (div[i - 1] - div[i - 2]) / dx;
                    Ur(i, 2) = Ur(i, 2) - alp * 0.5 * wy * (div[i - 2] + div[i - 1]);
                    Ur(i, 3) = Ur(i, 3) - alp * 0.5 * wz * (div[i - 2] + div[i - 1]);
                }
                for (int n = 1; n <= 3; ++n) Ur(nx + 1, n) = Ur(1, n);
                const double c2dtv = (c2 * dt) * vis;
                for (int i = 1; i <= nx; ++i) {
                    cplx dm = (i == 1) ? div[nx - 1] : div[i - 2];
                    cplx dp = (i == nx) ? div[0] : div[i];
                    cplx d0 = div[i - 1];
                    P(i) = P(i) + d0 - c2dtv * (((dm - 2.0 * d0) + dp) / dx2 - w2 * d0);
                }
                // check_divergence for this line
                double dmax = 0.0;
                for (int i = 1; i <= nx; ++i) {
                    cplx tmpc = (Ur(i + 1, 1) - Ur(i, 1)) / dx;
                    tmpc = tmpc + 0.5 * wy * (Ur(i, 2) + Ur(i + 1, 2));
                    tmpc = tmpc + 0.5 * wz * (Ur(i, 3) + Ur(i + 1, 3));
                    double tmp = std::sqrt(tmpc.real() * tmpc.real() + tmpc.imag() * tmpc.imag());
                    if (tmp > dmax) dmax = tmp;
                }
                divline[(size_t)(j - 1) + (size_t)my2 * (k - 1)] = dmax;
            }
    }
    o.divmax = 0.0;
    for (double v : divline) o.divmax = std::max(o.divmax, v);
    for (int d = 0; d < 3; ++d) o.umean[d] = o.umean[d] + (-o.mpg[d] + o.frmean[d] - o.frame_accln[d]) * dt;
    if (o.moving)
        for (int d = 0; d < 3; ++d) { o.frame_vel[d] = o.frame_vel[d] + o.frame_accln[d] * dt; o.frame_pos[d] = o.frame_pos[d] + o.frame_vel[d] * dt; }
    return bad ? PIBM_ERR_PIVOT : PIBM_OK;
}

// ============================================================================
// Passive scalar, one species (ISCALON = 1): scalstep, SRC/SCALAR/stepthescalar.F90:51-94.
// The scalar is periodic in x up to the factor heat_ratio (fully developed
// heat transfer): phi(x + L) = phi(x) / heat_ratio, so every x wrap below
// carries that factor.  Array roles follow the reference's aliases: phir is
// the real scalar (ubcp(:,:,:,1) there), nlphir/onlphir the real nonlinear
// terms (nlbcp/onlbcp), sdiffn the real diffusion term (diffn), gradphi the
// real gradient (ppr), sfr the real forcing (fr(0:nx+1)).
// ============================================================================

// form_nlphi + compute_phim_heat_ratio: SRC/SCALAR/nl_allphi.F90:59-253, 256-330 (serial).
void form_nlphi(Orc &o) {
    const int nx = o.nx, my = o.my, mz = o.mz, my2 = o.my2, mxf = o.mxf;
    const bool center = o.prm.discr_scheme == PIBM_SCHEME_CENTER;
    const double h = o.heat_ratio, dx = o.dx;
    std::vector<double> pb((size_t)(nx + 1) * my * mz);            // phirbcp (nlbcp there), planes 1..nx+1
    std::vector<double> fd((size_t)(nx + 2) * my * mz, 0.0);       // fdderiv(0:nx+1)
    auto PB = [&](int i, int j, int k) -> double & { return pb[o.RI(i, j, k, 1)]; };
    auto FD = [&](int i, int j, int k) -> double & { return fd[o.SF(i, j, k)]; };
    auto U = [&](int i, int j, int k, int n) { return o.ubcp[o.RI(i, j, k, n)]; };
#pragma omp parallel
    {
        std::vector<cplx> f2((size_t)my2 * mz), f3((size_t)my2 * mz);
#pragma omp for schedule(static)
        for (int i = 1; i <= nx + 1; ++i) {
            c2r_with(o, [&](int j, int k) { return o.phif[o.CI(i, j, k, 1)]; }, [&](int j, int k, double v) { PB(i, j, k) = v; });
            r2c_with(o, [&](int j, int k) { return U(i, j, k, 2) * PB(i, j, k); },
                     [&](int j, int k, cplx v) { f2[(j - 1) + (size_t)my2 * (k - 1)] = v; });
            r2c_with(o, [&](int j, int k) { return U(i, j, k, 3) * PB(i, j, k); },
                     [&](int j, int k, cplx v) { f3[(j - 1) + (size_t)my2 * (k - 1)] = v; });
            for (int k = 1; k <= mz; ++k)
                for (int j = 1; j <= my2; ++j) {
                    const size_t q = (j - 1) + (size_t)my2 * (k - 1);
                    o.nlphif[o.CI(i, j, k, 1)] = o.wy[j - 1] * f2[q] + o.wz[k - 1] * f3[q];
                }
            for (int k = 1; k <= mz; ++k)
                for (int j = 1; j <= my; ++j) FD(i, j, k) = center ? U(i, j, k, 1) * PB(i, j, k) : 0.0;
        }
    }
    // compute_phim_heat_ratio(.TRUE.): only the last plane's mixed mean sets heat_ratio_new
    {
        const int i = nx + 1;
        double phim = 0.0, um = 0.0;
        long long cnt = 0;
        for (int k = 1; k <= mz; ++k)
            for (int j = 1; j <= my; ++j)
                if (o.FL(i, j, k)) {
                    phim = phim + U(i, j, k, 1) * PB(i, j, k);
                    um = um + U(i, j, k, 1);
                    cnt = cnt + 1;
                }
        um = um / (double)cnt;
        phim = phim / (um * (double)cnt);
        o.heat_ratio_new = 1.0 / phim;
    }
    for (int k = 1; k <= mz; ++k)
        for (int j = 1; j <= my; ++j) FD(0, j, k) = center ? FD(nx, j, k) * h : 0.0;
    if (!center) {
#pragma omp parallel
        {
            std::vector<double> uplus(nx + 2), uminus(nx + 2), Up(nx + 2), Um(nx + 2), sp(nx + 2), su(nx + 2);
#pragma omp for schedule(static)
            for (int k = 1; k <= mz; ++k)
                for (int j = 1; j <= my; ++j) {
                    sp[0] = (PB(1, j, k) - PB(nx - 1, j, k) * h) / (2.0 * dx);
                    Um[0] = PB(nx, j, k) * h + sp[0] * (dx / 2.0);
                    sp[nx + 1] = (PB(2, j, k) / h - PB(nx, j, k)) / (2.0 * dx);
                    Up[nx] = PB(1, j, k) / h - sp[nx + 1] * (dx / 2.0);
                    su[0] = (U(1, j, k, 1) - U(nx - 1, j, k, 1)) / (2.0 * dx);
                    uminus[0] = U(nx, j, k, 1) + su[0] * (dx / 2.0);
                    su[nx + 1] = (U(2, j, k, 1) - U(nx, j, k, 1)) / (2.0 * dx);
                    uplus[nx] = U(1, j, k, 1) - su[nx + 1] * (dx / 2.0);
                    for (int i = 1; i <= nx; ++i) {
                        int im1 = i - 1, ip1 = i + 1;
                        double pfm = 1.0, pfp = 1.0;
                        if (im1 < 1) { im1 = mxf + im1 - 1; pfm = h; }
                        if (ip1 > mxf) { ip1 = ip1 - (mxf - 1); pfp = 1.0 / h; }
                        sp[i] = (pfp * PB(ip1, j, k) - pfm * PB(im1, j, k)) / (2.0 * dx);
                        su[i] = (U(ip1, j, k, 1) - U(im1, j, k, 1)) / (2.0 * dx);
                        uplus[i - 1] = U(i, j, k, 1) - su[i] * (dx / 2.0);
                        uminus[i] = U(i, j, k, 1) + su[i] * (dx / 2.0);
                        Up[i - 1] = PB(i, j, k) - sp[i] * (dx / 2.0);
                        Um[i] = PB(i, j, k) + sp[i] * (dx / 2.0);
                    }
                    for (int i = 0; i <= nx; ++i) {
                        const double ms = std::max(std::fabs(uminus[i]), std::fabs(uplus[i]));
                        double f = 0.5 * (uplus[i] * Up[i]) + 0.5 * (uminus[i] * Um[i]);
                        FD(i, j, k) = f - 0.5 * ms * (Up[i] - Um[i]);
                    }
                }
        }
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; ++i)
        r2c_with(o, [&](int j, int k) {
                     if (center) return (FD(i + 1, j, k) - FD(i - 1, j, k)) / (2.0 * dx);
                     return (FD(i, j, k) - FD(i - 1, j, k)) / dx; },
                 [&](int j, int k, cplx v) { cplx &d = o.nlphif[o.CI(i, j, k, 1)]; d = d + v; });
    for (int k = 1; k <= mz; ++k)
        for (int j = 1; j <= my2; ++j) o.nlphif[o.CI(nx + 1, j, k, 1)] = o.nlphif[o.CI(1, j, k, 1)] / h;
    for (int i = 1; i <= nx; ++i)
        for (int k = 1; k <= mz; ++k) {
            for (int j = 1; j <= my; ++j) o.phir[o.RI(i, j, k, 1)] = PB(i, j, k);
            for (int j = 1; j <= my2; ++j) { cplx &v = o.nlphif[o.CI(i, j, k, 1)]; v = -v; }
        }
    for (int k = 1; k <= mz; ++k) {
        for (int j = 1; j <= my2; ++j) { cplx &v = o.nlphif[o.CI(nx + 1, j, k, 1)]; v = -v; }
        for (int j = 1; j <= my; ++j) o.phir[o.RI(nx + 1, j, k, 1)] = o.phir[o.RI(1, j, k, 1)] / h;
    }
}

// calc_diffn: SRC/SCALAR/bc_scalar.F90:935-1033 (serial branch, planes 1..nx+1).
void calc_diffn_scal(Orc &o) {
    const int nx = o.nx, my2 = o.my2, mz = o.mz;
    const double h = o.heat_ratio, dx = o.dx, dx2 = o.dx2;
    auto PF = [&](int i, int j, int k) { return o.phif[o.CI(i, j, k, 1)]; };
#pragma omp parallel
    {
        std::vector<cplx> f1((size_t)my2 * mz), f2((size_t)my2 * mz), f3((size_t)my2 * mz), f4((size_t)my2 * mz);
#pragma omp for schedule(static)
        for (int i = 1; i <= nx + 1; ++i) {
            for (int k = 1; k <= mz; ++k)
                for (int j = 1; j <= my2; ++j) {
                    const size_t q = (j - 1) + (size_t)my2 * (k - 1);
                    cplx a;
                    if (i == 1) a = (1.0 / dx2) * (PF(nx, j, k) * h - 2.0 * PF(1, j, k) + PF(2, j, k));
                    else if (i == nx) a = (1.0 / dx2) * (PF(i - 1, j, k) - 2.0 * PF(i, j, k) + PF(1, j, k) / h);
                    else if (i == nx + 1) a = (1.0 / dx2) * (PF(i - 1, j, k) - 2.0 * PF(i, j, k) + PF(2, j, k) / h);
                    else a = (1.0 / dx2) * (PF(i - 1, j, k) - 2.0 * PF(i, j, k) + PF(i + 1, j, k));
                    a = a - o.W2(j, k) * PF(i, j, k);
                    f1[q] = a * o.gamma_s;
                    if (i == 1) f2[q] = (PF(2, j, k) - PF(nx, j, k) * h) / (2.0 * dx);
                    else if (i == nx) f2[q] = (PF(1, j, k) / h - PF(i - 1, j, k)) / (2.0 * dx);
                    else if (i == nx + 1) f2[q] = (PF(2, j, k) / h - PF(i - 1, j, k)) / (2.0 * dx);
                    else f2[q] = (PF(i + 1, j, k) - PF(i - 1, j, k)) / (2.0 * dx);
                    f3[q] = PF(i, j, k) * o.wy[j - 1];
                    f4[q] = PF(i, j, k) * o.wz[k - 1];
                }
            auto out = [&](std::vector<cplx> &f, std::vector<double> &dst, int n) {
                c2r_with(o, [&](int j, int k) { return f[(j - 1) + (size_t)my2 * (k - 1)]; },
                         [&](int j, int k, double v) { dst[o.RI(i, j, k, n)] = v; });
            };
            out(f1, o.sdiffn, 1); out(f2, o.gradphi, 1); out(f3, o.gradphi, 2); out(f4, o.gradphi, 3);
        }
    }
}

// set_interpolation_stencil ('lpi', order 2, x periodic; dependent_functions.F90:45-158)
// without wrapping, and the weights of interp_threed with shape2.
struct RawSten {
    int ib, jb, kb;
    double w[2][2][2];
};
inline void raw_stencil(const Orc &o, const int pc[3], const double pos[3], RawSten &s) {
    int ib = std::max(1, pc[0]), ie = std::min(o.mxf, pc[0] + 1);
    if (ib == 1) ib = ie - 2 + 1;
    int jb = std::max(1, pc[1]), je = std::min(o.my, pc[1] + 1);
    if (jb == 1) jb = je - 2 + 1;
    int kb = std::max(1, pc[2]), ke = std::min(o.mz, pc[2] + 1);
    if (kb == 1) kb = ke - 2 + 1;
    s.ib = ib; s.jb = jb; s.kb = kb;
    const double zx = (pos[0] - (double)ib) / (double)((ib + 1) - ib);
    const double zy = (pos[1] - (double)jb) / (double)((jb + 1) - jb);
    const double zz = (pos[2] - (double)kb) / (double)((kb + 1) - kb);
    const double xv[2] = {1.0 - zx, zx}, yv[2] = {1.0 - zy, zy}, zv[2] = {1.0 - zz, zz};
    for (int k = 0; k < 2; ++k) for (int j = 0; j < 2; ++j) for (int i = 0; i < 2; ++i) s.w[i][j][k] = xv[i] * yv[j] * zv[k];
}
inline int wrap_yz(int v, int n) { return v < 1 ? v + n : (v > n ? v - n : v); }

// interpolate_phidata: SRC/SCALAR/bc_scalar.F90:1036-1153 (serial).  x indices
// below 1 wrap with the factor heat_ratio (heat_ratio_old for onlphir), above
// mxf with 1/heat_ratio.  flag 1 also interpolates nl, onl and diffn.
void interp_phi(const Orc &o, const int pc[3], const double pos[3], int flag, RawSten &s,
                double &ul, double &nll, double &onll, double &dfll) {
    raw_stencil(o, pc, pos, s);
    double v[2][2][2], nl[2][2][2], onl[2][2][2], df[2][2][2];
    for (int k = 0; k < 2; ++k)
        for (int j = 0; j < 2; ++j)
            for (int i = 0; i < 2; ++i) {
                int ii = s.ib + i, jj = wrap_yz(s.jb + j, o.my), kk = wrap_yz(s.kb + k, o.mz);
                double pf = 1.0, pfo = 1.0;
                if (ii < 1) { ii = o.mxf + ii - 1; pf = o.heat_ratio; pfo = o.heat_ratio_old; }
                else if (ii > o.mxf) { ii = ii - o.mxf + 1; pf = 1.0 / o.heat_ratio; }
                v[i][j][k] = o.phir[o.RI(ii, jj, kk, 1)] * pf;
                if (flag == 1) {
                    nl[i][j][k] = o.nlphir[o.RI(ii, jj, kk, 1)] * pf;
                    onl[i][j][k] = o.onlphir[o.RI(ii, jj, kk, 1)] * pfo;
                    df[i][j][k] = o.sdiffn[o.RI(ii, jj, kk, 1)] * pf;
                }
            }
    ul = 0.0;
    for (int k = 0; k < 2; ++k) for (int j = 0; j < 2; ++j) for (int i = 0; i < 2; ++i) ul = ul + v[i][j][k] * s.w[i][j][k];
    if (flag == 1) {
        nll = 0.0; onll = 0.0; dfll = 0.0;
        for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) for (int k = 0; k < 2; ++k) nll = nll + nl[i][j][k] * s.w[i][j][k];
        for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) for (int k = 0; k < 2; ++k) onll = onll + onl[i][j][k] * s.w[i][j][k];
        for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) for (int k = 0; k < 2; ++k) dfll = dfll + df[i][j][k] * s.w[i][j][k];
    }
}

// calc_bndrev_data with DOBND = F: surface flux of sphere m from the
// interpolated gradient (SRC/SCALAR/bc_scalar.F90:385-556, serial branch).
double scal_surface_flux(const Orc &o, int m) {
    double fluxloc = 0.0;
    for (int l = 1; l <= o.nbnd; ++l) {
        double xl[3];
        int is[3];
        for (int n = 1; n <= 3; ++n) {
            xl[n - 1] = o.XC(m, n) + o.BND(n, l) * o.radbdy[m - 1];
            is[n - 1] = cell_of(xl[n - 1]);
        }
        // CELL_IN_BOX / WEST_PERIODIC_IMAGE / EAST_PERIODIC_IMAGE (ibm.h:147-149)
        if (!(1 <= is[0] && is[0] <= o.nx)) {
            if (is[0] < 1) { xl[0] = o.mxf + xl[0] - 1; is[0] = o.mxf + is[0] - 1; }
            else if (is[0] >= o.mxf) { xl[0] = xl[0] - (o.mxf - 1); is[0] = is[0] - (o.mxf - 1); }
        }
        RawSten s;
        raw_stencil(o, is, xl, s);
        double g[3][2][2][2];
        for (int k = 0; k < 2; ++k)
            for (int j = 0; j < 2; ++j)
                for (int i = 0; i < 2; ++i) {
                    int ii = s.ib + i, jj = wrap_yz(s.jb + j, o.my), kk = wrap_yz(s.kb + k, o.mz);
                    double pf = 1.0;
                    if (ii < 1) { ii = o.mxf + ii - 1; pf = o.heat_ratio; }
                    if (ii > o.mxf) { ii = ii - o.mxf + 1; pf = 1.0 / o.heat_ratio; }
                    for (int n = 1; n <= 3; ++n) g[n - 1][i][j][k] = o.gradphi[o.RI(ii, jj, kk, n)] * pf;
                }
        double gb[3];
        for (int n = 0; n < 3; ++n) {
            double r = 0.0;
            for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) for (int k = 0; k < 2; ++k) r = r + g[n][i][j][k] * s.w[i][j][k];
            gb[n] = r;
        }
        double d = 0.0;
        for (int n = 1; n <= 3; ++n) d = d + gb[n - 1] * o.BND(n, l);
        fluxloc = fluxloc + d;
    }
    return fluxloc;
}

// calc_inner_rev_data: SRC/SCALAR/bc_scalar.F90:558-932 (serial branch).  A
// point whose cell is the last one (i = nx) is evaluated twice, as itself and
// shifted one period west; each evaluation spreads onto its own stencil and
// the forcing on planes 0 and nx+1 is not transformed.
void scal_inner_forcing(Orc &o, int m, double da2) {
    const double dx3 = std::pow(o.dx, 3.0), drm = 1.0;
    const double c1 = o.coef[0], c2 = o.coef[1], c3 = o.coef[2], c4 = o.coef[3];
    const double rb = o.radbdy[m - 1], ri = o.radibdy[m - 1], ro = o.radobdy[m - 1];
    for (int l = 1; l <= o.nbnd; ++l) {
        if (!o.if_rev[(size_t)(l - 1) + (size_t)o.nbnd * (m - 1)]) continue;
        double xli[3];
        int iii[3];
        for (int n = 1; n <= 3; ++n) {
            xli[n - 1] = o.XC(m, n) + o.BND(n, l) * ri;
            iii[n - 1] = cell_of(xli[n - 1]);
        }
        int pct = iii[0];
        double xlt = xli[0];
        if (!(1 <= pct && pct <= o.nx)) {
            if (iii[0] < 1) { pct = o.mxf + iii[0] - 1; xlt = o.mxf + xli[0] - 1; }
            else if (iii[0] >= o.mxf) { pct = iii[0] - (o.mxf - 1); xlt = xli[0] - (o.mxf - 1); }
        }
        const int nev = pct == o.nx ? 2 : 1;
        for (int ev = 1; ev <= nev; ++ev) {
            if (ev == 1) { iii[0] = pct; xli[0] = xlt; }
            else if (iii[0] >= o.mxf - 1) { iii[0] = iii[0] - (o.mxf - 1); xli[0] = xli[0] - (o.mxf - 1); }
            double xlo[3];
            int io[3];
            for (int n = 1; n <= 3; ++n) {
                xlo[n - 1] = xli[n - 1] + o.BND(n, l) * (ro - ri);
                io[n - 1] = cell_of(xlo[n - 1]);
            }
            RawSten so, si;
            double philo, phili, nll = 0, onll = 0, dfll = 0, dum;
            interp_phi(o, io, xlo, 0, so, philo, dum, dum, dum);
            interp_phi(o, iii, xli, 1, si, phili, nll, onll, dfll);
            philo = o.phisurf * (ro - ri) - philo * (rb - ri);
            philo = philo / (ro - rb);
            const double phil = o.cf * (-philo + phili);
            double t = 0.0;
            t = t + phil;
            t = t - c3 * nll - c4 * onll;
            t = t - (c2 + c1) * dfll;
            t = t * da2 * drm * o.dx;
            int count_fl = 0;
            double force_fl = 0.0;
            auto node = [&](int i, int j, int k, int &ii, int &jj, int &kk) {
                ii = si.ib + i; jj = wrap_yz(si.jb + j, o.my); kk = wrap_yz(si.kb + k, o.mz);
                if (ii < 0) ii = o.mxf + ii - 1;
            };
            for (int k = 0; k < 2; ++k)
                for (int j = 0; j < 2; ++j)
                    for (int i = 0; i < 2; ++i) {
                        int ii, jj, kk;
                        node(i, j, k, ii, jj, kk);
                        if (o.FL(ii, jj, kk)) { count_fl += 1; force_fl = force_fl + si.w[i][j][k] * t / dx3; }
                    }
            const int count_so = 8 - count_fl;
            const double force_dist = force_fl / (double)count_so;
            for (int k = 0; k < 2; ++k)
                for (int j = 0; j < 2; ++j)
                    for (int i = 0; i < 2; ++i) {
                        int ii, jj, kk;
                        node(i, j, k, ii, jj, kk);
                        double &f = o.sfr[o.SF(ii, jj, kk)];
                        if (o.prm.include_frmeanfluid) f = f + si.w[i][j][k] * t / dx3;
                        else if (!o.FL(ii, jj, kk)) f = f + si.w[i][j][k] * t / dx3 + force_dist;
                    }
        }
    }
}

// bcsetscal (SRC/SCALAR/bc_scalar.F90:65-383) after nlphi_graduphi's
// transforms of the nonlinear terms (SRC/SCALAR/nlphi.F90:56-155).
void bcsetscal(Orc &o) {
    const int nx = o.nx;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx + 1; ++i) {
        c2r_with(o, [&](int j, int k) { return o.nlphif[o.CI(i, j, k, 1)]; }, [&](int j, int k, double v) { o.nlphir[o.RI(i, j, k, 1)] = v; });
        c2r_with(o, [&](int j, int k) { return o.onlphif[o.CI(i, j, k, 1)]; }, [&](int j, int k, double v) { o.onlphir[o.RI(i, j, k, 1)] = v; });
    }
    std::fill(o.sfr.begin(), o.sfr.end(), 0.0);
    calc_diffn_scal(o);
    o.flux_global = 0.0;
    for (int m = 1; m <= o.nbody; ++m) {
        const double da1 = 4.0 * PI * ((o.radbdy[m - 1] * o.dx) * (o.radbdy[m - 1] * o.dx)) / (double)o.nbnd;
        const double da2 = 4.0 * PI * ((o.radibdy[m - 1] * o.dx) * (o.radibdy[m - 1] * o.dx)) / (double)o.nrpr_active[m - 1];
        o.flux_body[m - 1] = scal_surface_flux(o, m);
        if (o.prm.dorpr) scal_inner_forcing(o, m, da2);
        o.flux_global = o.flux_global + o.flux_body[m - 1] * da1;
    }
    o.nusselt = -(o.flux_global * o.char_length * o.char_length) / (6.0 * o.voldom * o.maxvolfrac * (o.phisurf - o.phistream));
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; ++i)
        r2c_with(o, [&](int j, int k) { return o.sfr[o.SF(i, j, k)]; }, [&](int j, int k, cplx v) { o.ffphi[o.CI(i, j, k, 1)] = v; });
}

// phistep: SRC/SCALAR/stepthescalar.F90:99-213 (serial branch): per (ky,kz)
// line a cyclic Crank-Nicolson solve whose corners carry heat_ratio_new,
// by Thomas (tridag3) + Sherman-Morrison.
bool phistep(Orc &o) {
    const int nx = o.nx, my2 = o.my2, mz = o.mz;
    const double dt = o.dt, g = o.gamma_s, dx2 = o.dx2;
    const double c1 = o.coef[0], c2 = o.coef[1], c3 = o.coef[2], c4 = o.coef[3];
    const double hn = o.heat_ratio_new, h = o.heat_ratio;
    bool ok = true;
#pragma omp parallel reduction(&& : ok)
    {
        std::vector<double> a(nx), b(nx), c(nx), tr(nx), ti(nx), ur(nx), ui(nx), auxu(nx), auxv(nx), auxz(nx), gam(nx + 1);
        std::vector<cplx> r1(nx);
#pragma omp for schedule(static)
        for (int k = 1; k <= mz; ++k)
            for (int j = 1; j <= my2; ++j) {
                auto PF = [&](int i) { return o.phif[o.CI(i, j, k, 1)]; };
                const double alpha = hn, beta = 1.0 / hn, w2 = o.W2(j, k);
                for (int i = 1; i <= nx; ++i) {
                    a[i - 1] = -(dt * g * c2 / dx2);
                    b[i - 1] = 1.0 + dt * g * c2 * (2.0 / dx2 + w2);
                    c[i - 1] = -(dt * g * c2 / dx2);
                    auxu[i - 1] = 0.0; auxv[i - 1] = 0.0; auxz[i - 1] = 0.0;
                    cplx r = PF(i) * (1.0 - dt * c1 * g * w2);
                    r = r + dt * c3 * o.nlphif[o.CI(i, j, k, 1)] + dt * o.ffphi[o.CI(i, j, k, 1)];
                    r = r + dt * c4 * o.onlphif[o.CI(i, j, k, 1)];
                    r1[i - 1] = r;
                }
                a[0] = a[0] * hn;
                c[nx - 1] = c[nx - 1] / hn;
                for (int i = 2; i <= nx; ++i)
                    r1[i - 1] = r1[i - 1] + dt * g * c1 * (PF(i - 1) + PF(i + 1) - 2.0 * PF(i)) / dx2;
                r1[0] = r1[0] + dt * g * c1 * (PF(2) - 2.0 * PF(1) + PF(nx) * h) / dx2;
                for (int i = 0; i < nx; ++i) { tr[i] = r1[i].real(); ti[i] = r1[i].imag(); }
                auxu[0] = alpha;
                auxu[nx - 1] = beta;
                auxv[0] = c[nx - 1] / auxu[nx - 1];
                auxv[nx - 1] = a[0] / auxu[0];
                b[0] = b[0] - auxu[0] * auxv[0];
                b[nx - 1] = b[nx - 1] - auxu[nx - 1] * auxv[nx - 1];
                if (!tridag3(a.data(), b.data(), c.data(), tr.data(), auxu.data(), ti.data(), ur.data(), auxz.data(), ui.data(), nx, gam.data())) {
                    ok = false;
                    continue;
                }
                const double vdotz = auxv[0] * auxz[0] + auxv[nx - 1] * auxz[nx - 1];
                const double vdotyr = auxv[0] * ur[0] + auxv[nx - 1] * ur[nx - 1];
                const double vdotyi = auxv[0] * ui[0] + auxv[nx - 1] * ui[nx - 1];
                for (int i = 1; i <= nx; ++i)
                    o.phif[o.CI(i, j, k, 1)] = cplx(ur[i - 1] - vdotyr * auxz[i - 1] / (1.0 + vdotz),
                                                    ui[i - 1] - vdotyi * auxz[i - 1] / (1.0 + vdotz));
                o.phif[o.CI(nx + 1, j, k, 1)] = o.phif[o.CI(1, j, k, 1)] / hn;
            }
    }
    return ok;
}

// scalstep: SRC/SCALAR/stepthescalar.F90:51-94 (one species).
int scalstep(Orc &o) {
    std::swap(o.onlphif, o.nlphif);
    std::fill(o.nlphif.begin(), o.nlphif.end(), cplx(0.0, 0.0));
    form_nlphi(o);
    bcsetscal(o);
    if (!phistep(o)) return PIBM_ERR_PIVOT;
    o.heat_ratio_old = o.heat_ratio;
    o.heat_ratio = o.heat_ratio_new;
    return PIBM_OK;
}

void fill_report(Orc &o, pibm_step_report *rep) {
    std::memset(rep, 0, sizeof(*rep));
    rep->dt = o.dt; rep->t = o.t; rep->cf = o.cf; rep->umax = o.umax_last; rep->divmax = o.divmax;
    for (int d = 0; d < 3; ++d) {
        rep->ufmean[d] = o.ufmean[d]; rep->usmean[d] = o.usmean[d]; rep->umean[d] = o.umean[d];
        rep->mpg[d] = o.mpg[d]; rep->frmean[d] = o.frmean[d];
        rep->pres_total[d] = o.pres_total[d]; rep->visc_total[d] = o.visc_total[d];
    }
    rep->norm_drag = o.norm_drag; rep->ferror = o.ferror;
    rep->pres_drag = o.pres_drag; rep->visc_drag = o.visc_drag; rep->total_drag = o.total_drag;
    rep->mixmeanslipmod = o.mixmeanslipmod;
    long long s = 0; for (int v : o.nrpr_active) s += v;
    rep->nrpr_active_total = s;
    rep->heat_ratio = o.heat_ratio;
    rep->nusselt = o.nusselt;
}

// One iteration of the driver's rks loop (dtibm_main_scal_flo.F90:426-527)
// with the stage's coefficients coef(rks, 1:4).
int step_stage(Orc &o, int rks, pibm_step_report *rep) {
    std::memcpy(o.coef, o.coef_tab[rks - 1], sizeof(o.coef));
    compute_new_timestep(o, rks);
    int rc = nonlinear(o, rks);
    if (rc) return rc;
    rc = velstep(o, rks);
    if (!rc && o.scal) rc = scalstep(o);
    if (rep) fill_report(o, rep);
    for (const cplx &v : o.u) if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) return PIBM_ERR_NAN;
    return rc;
}

// One time step: rks = 1..itrmax.
int step(Orc &o, pibm_step_report *rep) {
    for (int rks = 1; rks <= o.itrmax; ++rks) {
        const int rc = step_stage(o, rks, rep);
        if (rc) return rc;
    }
    return PIBM_OK;
}

#include "adjoint_oracle.inc"

}  // namespace

// ============================================================================
// C interface (test-only entry points: orc_*).
// ============================================================================
extern "C" {

const char *orc_last_error(void) { return g_err.c_str(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_create(const pibm_params *prm, const pibm_particles *parts, void **out) {
    Orc *o = new Orc();
    if (!setup(*o, prm, parts)) { delete o; return PIBM_ERR_ARG; }
    *out = o;
    return PIBM_OK;
}

void orc_destroy(void *h) { delete (Orc *)h; }

int orc_info(void *h, pibm_info *info) {
    Orc &o = *(Orc *)h;
    info->nx = o.nx; info->my = o.my; info->mz = o.mz; info->my2 = o.my2; info->nbody = o.nbody; info->nbnd = o.nbnd;
    info->dx = o.dx; info->dt = o.dt; info->radbdy = o.nbody ? o.radbdy[0] : 0.0; info->maxvolfrac = o.maxvolfrac;
    info->count_solid = o.count_solid; info->count_fluid = o.count_fluid;
    long long s = 0; for (int v : o.nrpr_active) s += v;
    info->npts_active = (int32_t)s;
    info->kernels_per_step = 0;
    return PIBM_OK;
}

int orc_step(void *h, pibm_step_report *rep) { return step(*(Orc *)h, rep); }
int orc_step_rks(void *h, int rks, pibm_step_report *rep) {
    Orc &o = *(Orc *)h;
    if (rks < 1 || rks > o.itrmax) { g_err = "rks out of range"; return PIBM_ERR_ARG; }
    return step_stage(o, rks, rep);
}

int orc_get_state(void *h, pibm_state_view *s) {
    Orc &o = *(Orc *)h;
    if (s->u) std::memcpy((void *)s->u, (const void *)o.u.data(), o.u.size() * sizeof(cplx));
    if (s->nl) std::memcpy((void *)s->nl, (const void *)o.nl.data(), o.nl.size() * sizeof(cplx));
    if (s->p) std::memcpy((void *)s->p, (const void *)o.p.data(), o.p.size() * sizeof(cplx));
    for (int d = 0; d < 3; ++d) { s->umean[d] = o.umean[d]; s->mpg[d] = o.mpg[d]; s->ufmean[d] = o.ufmean[d]; }
    s->t = o.t; s->dt = o.dt; s->cf = o.cf;
    return PIBM_OK;
}

int orc_set_state(void *h, const pibm_state_view *s) {
    Orc &o = *(Orc *)h;
    if (s->u) std::memcpy((void *)o.u.data(), (const void *)s->u, o.u.size() * sizeof(cplx));
    if (s->nl) std::memcpy((void *)o.nl.data(), (const void *)s->nl, o.nl.size() * sizeof(cplx));
    if (s->p) std::memcpy((void *)o.p.data(), (const void *)s->p, o.p.size() * sizeof(cplx));
    for (int d = 0; d < 3; ++d) { o.umean[d] = s->umean[d]; o.mpg[d] = s->mpg[d]; o.ufmean[d] = s->ufmean[d]; }
    o.t = s->t; o.dt = s->dt; o.cf = s->cf;
    return PIBM_OK;
}

int orc_get_particles(void *h, double *pres, double *visc, double *force, double *xc, double *vel) {
    Orc &o = *(Orc *)h;
    size_t n = (size_t)o.nbody * 3 * sizeof(double);
    if (pres) std::memcpy(pres, o.pres.data(), n);
    if (visc) std::memcpy(visc, o.visc.data(), n);
    if (force) std::memcpy(force, o.force.data(), n);
    if (xc) std::memcpy(xc, o.xc.data(), n);
    if (vel) std::memcpy(vel, o.velbdy.data(), n);
    return PIBM_OK;
}

int orc_get_if_rev(void *h, uint8_t *out) {
    Orc &o = *(Orc *)h;
    std::memcpy(out, o.if_rev.data(), o.if_rev.size());
    return PIBM_OK;
}

int orc_get_fluid_mask(void *h, uint8_t *out) {
    Orc &o = *(Orc *)h;
    for (int k = 1; k <= o.mz; ++k)
        for (int j = 1; j <= o.my; ++j)
            for (int i = 1; i <= o.nx; ++i)
                out[(size_t)(i - 1) + (size_t)o.nx * ((size_t)(j - 1) + (size_t)o.my * (k - 1))] = o.FL(i, j, k) ? 1 : 0;
    return PIBM_OK;
}

int orc_get_geometry(void *h, double *bndpts, double *cdv) {
    Orc &o = *(Orc *)h;
    if (bndpts) std::memcpy(bndpts, o.bndpts.data(), o.bndpts.size() * sizeof(double));
    if (cdv) std::memcpy(cdv, o.cd.data(), o.cd.size() * sizeof(double));
    return PIBM_OK;
}

// Real fields after the last step (for kernel-level parity): which =
// 0 ubcp(nx+1,my,mz,3) 1 nlbc 2 onlbc 3 diffn 4 omega 5 fr 6 pbcp(nx,my,mz) 7 ppr(nx,my,mz,3)
// 8 ff complex (nx+1,my2,mz,3)
int orc_get_field(void *h, int which, double *out) {
    Orc &o = *(Orc *)h;
    const std::vector<double> *v = nullptr;
    switch (which) {
        case 0: v = &o.ubcp; break; case 1: v = &o.nlbc; break; case 2: v = &o.onlbc; break;
        case 3: v = &o.diffn; break; case 4: v = &o.omega; break; case 5: v = &o.fr; break;
        case 6: v = &o.pbcp; break; case 7: v = &o.ppr; break;
        case 8: std::memcpy((void *)out, (const void *)o.ff.data(), o.ff.size() * sizeof(cplx)); return PIBM_OK;
        default: return PIBM_ERR_ARG;
    }
    std::memcpy(out, v->data(), v->size() * sizeof(double));
    return PIBM_OK;
}

int orc_ff2rc(int my, int mz, int nplanes, const double *a, double *b) {
    PlaneFFT f; f.init(my, mz);
    if (!f.fy.ok() || !f.fz.ok()) return PIBM_ERR_ARG;
    const int my2 = my / 2 + 1;
    for (int q = 0; q < nplanes; ++q)
        f.r2c(a + (size_t)q * my * mz, (cplx *)b + (size_t)q * my2 * mz);
    return PIBM_OK;
}

int orc_ff2cr(int my, int mz, int nplanes, const double *a, double *b) {
    PlaneFFT f; f.init(my, mz);
    if (!f.fy.ok() || !f.fz.ok()) return PIBM_ERR_ARG;
    const int my2 = my / 2 + 1;
    for (int q = 0; q < nplanes; ++q)
        f.c2r((const cplx *)a + (size_t)q * my2 * mz, b + (size_t)q * my * mz);
    return PIBM_OK;
}

// Cyclic tridiagonal solve as used by ustep/pressure (for known-answer tests).
int orc_cyclic_solve(int n, const double *a, const double *b, const double *c, const double *rr, const double *ri,
                     double *outr, double *outi) {
    std::vector<double> bb(b, b + n), auxz(n), gam(n);
    return cyclic_solve(n, a, bb.data(), c, rr, ri, outr, outi, auxz.data(), gam.data()) ? 0 : PIBM_ERR_PIVOT;
}

}  // extern "C"

// Passive scalar state: phif complex (nx+1,my2,mz) interleaved, flux_body (nbody),
// ratios[0..2] = heat_ratio, heat_ratio_old, nusselt.  Any pointer may be NULL.
extern "C" int orc_get_scalar(void *h, double *phif, double *flux_body, double *ratios) {
    Orc &o = *(Orc *)h;
    if (!o.scal) return PIBM_ERR_ARG;
    if (phif) std::memcpy((void *)phif, o.phif.data(), o.phif.size() * sizeof(cplx));
    if (flux_body) for (int m = 0; m < o.nbody; ++m) flux_body[m] = o.flux_body[m];
    if (ratios) { ratios[0] = o.heat_ratio; ratios[1] = o.heat_ratio_old; ratios[2] = o.nusselt; }
    return PIBM_OK;
}

extern "C" int orc_get_scalar_nl(void *h, double *nlphif) {
    Orc &o = *(Orc *)h;
    if (!o.scal) return PIBM_ERR_ARG;
    std::memcpy((void *)nlphif, o.nlphif.data(), o.nlphif.size() * sizeof(cplx));
    return PIBM_OK;
}

// usmean_des / ufmean_des read from a restart (restart_funcs.F90:450-452).
extern "C" int orc_set_desired_means(void *h, const double *usd, const double *ufd) {
    Orc &o = *(Orc *)h;
    for (int d = 0; d < 3; ++d) { o.usmean_des[d] = usd[d]; o.ufmean_des[d] = ufd[d]; }
    return PIBM_OK;
}

// Frame motion of a moving run (frame_vel, frame_pos: steptheflow.F90:99-103,
// restart_funcs.F90:253-254).
extern "C" int orc_get_frame(void *h, double *frame_vel, double *frame_pos) {
    Orc &o = *(Orc *)h;
    for (int d = 0; d < 3; ++d) { frame_vel[d] = o.frame_vel[d]; frame_pos[d] = o.frame_pos[d]; }
    return PIBM_OK;
}
extern "C" int orc_set_frame(void *h, const double *frame_vel, const double *frame_pos) {
    Orc &o = *(Orc *)h;
    for (int d = 0; d < 3; ++d) { o.frame_vel[d] = frame_vel[d]; o.frame_pos[d] = frame_pos[d]; }
    return PIBM_OK;
}

// read_unformatted's scalar part (restart_funcs.F90:560-590).
extern "C" int orc_set_scalar(void *h, const double *phif, const double *nlphif, const double *ratios) {
    Orc &o = *(Orc *)h;
    if (!o.scal) return PIBM_ERR_ARG;
    std::memcpy((void *)o.phif.data(), phif, o.phif.size() * sizeof(cplx));
    std::memcpy((void *)o.nlphif.data(), nlphif, o.nlphif.size() * sizeof(cplx));
    o.heat_ratio = ratios[0];
    o.heat_ratio_old = ratios[1];
    return PIBM_OK;
}

// sizes of the ABI structs as compiled from include/pibm.h (for the ctypes mirror test)
// DEM lists in the reference layout NEIGHBOURS/PN/PV(nbody, maxn): column 1 the
// count (PV: 1), columns 2.. 1-based particle numbers, then -1 (PV: 0).
// Discrete adjoint (test infrastructure): K AB2 steps from the current state,
// J = (1/K) sum_n e . sum_m (pres + visc), gradients w.r.t. xc (nbody,3) and
// mpg(3); lu0/lp0/lnl0 (optional) receive lambda of the initial u, p, nl in
// the state layout, lumean0 lambda of the initial umean.
extern "C" int orc_adjoint(void *h, int K, const double *e, double *J, double *gxc, double *gmpg,
                           double *lu0, double *lp0, double *lnl0, double *lumean0) {
    Orc &o = *(Orc *)h;
    AdjState A;
    const int rc = adjoint_run(o, K, e, J, gxc, gmpg, &A);
    if (rc) return rc;
    if (lu0) std::memcpy(lu0, A.lu.data(), A.lu.size() * sizeof(cplx));
    if (lp0) std::memcpy(lp0, A.lp.data(), A.lp.size() * sizeof(cplx));
    if (lnl0) std::memcpy(lnl0, A.lnl.data(), A.lnl.size() * sizeof(cplx));
    if (lumean0) for (int d = 0; d < 3; ++d) lumean0[d] = A.lumean[d];
    return PIBM_OK;
}

extern "C" int orc_get_contacts(void *h, int maxn, int32_t *neigh, int32_t *pn, int32_t *pv) {
    Orc &o = *(Orc *)h;
    if (!o.moving) return PIBM_ERR_ARG;
    const Dem &D = o.dem;
    const int N = D.N;
    for (int l = 0; l < N; ++l)
        if ((int)D.neigh[l].size() + 1 > maxn || (int)D.pn[l].size() + 1 > maxn) return PIBM_ERR_ARG;
    for (int l = 0; l < N; ++l) {
        neigh[l] = (int32_t)D.neigh[l].size();
        pn[l] = (int32_t)D.pn[l].size();
        pv[l] = 1;
        for (int c = 1; c < maxn; ++c) {
            const size_t q = (size_t)l + (size_t)N * c;
            neigh[q] = c - 1 < (int)D.neigh[l].size() ? D.neigh[l][c - 1] + 1 : -1;
            pn[q] = c - 1 < (int)D.pn[l].size() ? D.pn[l][c - 1] + 1 : -1;
            pv[q] = c - 1 < (int)D.pv[l].size() ? D.pv[l][c - 1] : 0;
        }
    }
    return PIBM_OK;
}

extern "C" int orc_sizeof(int which) {
    switch (which) {
        case 0: return (int)sizeof(pibm_params);
        case 1: return (int)sizeof(pibm_particles);
        case 2: return (int)sizeof(pibm_state_view);
        case 3: return (int)sizeof(pibm_step_report);
        case 4: return (int)sizeof(pibm_info);
        default: return -1;
    }
}
