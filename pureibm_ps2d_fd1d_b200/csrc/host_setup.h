// host_setup.h -- host-side set-up of a run (the parts of the reference's
// initflo, SRC/FLO/initialize_flo.F90:61-1013, that define the step's inputs).
// Compiled without floating-point contraction so that every geometric
// quantity (cell indices, weights, mask distances) matches the device
// kernels, which use explicitly rounded operations for the same expressions.
#pragma once
#include <stdint.h>
#include <vector>
#include <string>
#include "../../include/pibm.h"

namespace pibm {

struct RunSetup {
    // grid
    int nx = 0, my = 0, mz = 0, my2 = 0, mx = 0, mxf = 0;
    double dx = 0, dx2 = 0, dx3 = 0, vis = 0, doml[3] = {0, 0, 0}, voldom = 0;
    double coef[4] = {0.5, 0.5, 1.5, -0.5};
    double char_length = 0, uchar[3] = {0, 0, 0}, ucharmod = 0;
    double dt = 0, cf = 0, ramp_frac_time = 0;
    std::vector<double> ky, kz, w2;        // wy = i*ky, wz = i*kz, w2 (my2 x mz, j fastest)
    // particles (all spheres share one radius for input_type='default')
    int nbody = 0;
    std::vector<double> xc, vel;           // (nbody,3) column-major, grid units
    double radbdy = 0, radibdy = 0, radobdy = 0, dr = 1.0;
    int nbnd = 0;
    std::vector<double> bnd, cd;           // (3, nbnd)
    std::vector<uint8_t> if_rev;           // (nbnd, nbody)
    std::vector<int> nrpr_active;          // (nbody)
    std::vector<std::vector<int>> neighbours;
    std::vector<uint8_t> fluid;            // device layout [i][k][j] (1 = fluid)
    long long count_solid = 0, count_fluid = 0;
    double maxvolfrac = 0, mean_volfrac = 0;
    double ufmean_des[3] = {0, 0, 0}, usmean_des[3] = {0, 0, 0}, umean0[3] = {0, 0, 0};
    // active reversal points in (m, l) order
    std::vector<int> pt_m, pt_l;
    // spreading map: nodes (device layout linear index i*my*mz + k*my + j), CSR rows of
    // (point index * 8 + corner) in ascending point order
    std::vector<int> sp_node, sp_ptr, sp_ent;
    // passive scalar (iscalon): diffusivity, surface and stream values, and the
    // reversal-point evaluations of calc_inner_rev_data: each active point once,
    // a second time one period west when its cell is the last one; positions
    // (after the x wrap) and cells per evaluation, and the spreading map of
    // (evaluation * 8 + corner) per node of planes 1..nx in reference order
    bool scal = false;
    double gamma_s = 0, phisurf = 0, phistream = 0;
    std::vector<int> sev_m, sev_l, sev_c;     // sev_c: 3 cells per evaluation
    std::vector<double> sev_x;                // 3 coordinates per evaluation
    std::vector<int> ssp_node, ssp_ptr, ssp_ent;
    // moving particles (IMOVE = 1): soft-sphere DEM constants of
    // initialize_coarse_grid / CFASSIGN (collision_mod.F90:346-741) for one
    // phase; positions are physical, DES_POS = (XC - 1) * dx
    bool moving = false;
    int dem_soft = 0;                          // COLLISION_TYPE = 'softsphere' (else 'none')
    int dem_cx = 0, dem_cy = 0, dem_cz = 0;    // coarse grid nodes (physical cells 2..c)
    double dem_dxc = 0, dem_dyc = 0, dem_dzc = 0, dem_LXs = 0, dem_LYs = 0, dem_LZs = 0;
    double dem_kn = 0, dem_eta_n = 0, dem_rad = 0, dem_pmass = 0, dem_pvol = 0, dem_dtsolid = 0;
};

bool setup_run(const pibm_params &prm, const pibm_particles *parts, RunSetup &S, std::string &err);
// Surface quadrature (exposed for tests through the handle).
void surface_points(double r, double f2, std::vector<double> &bnd, std::vector<double> &cd, int &nbnd);

}  // namespace pibm
