// api.cu -- the pibm_* C ABI (include/pibm.h) on top of the sm_100a kernels.
//
// A handle owns: the device copy of the run geometry, every field of the
// step, one stream, and two CUDA graphs of one step each (the nonlinear-term
// buffers alternate between steps, so even and odd steps differ only in which
// buffer is "current").  pibm_run replays the graphs without host
// synchronisation; pibm_step launches one step and reads the diagnostics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pibm.h"
#include "engine.cuh"
#include "host_setup.h"

namespace pibm {
cudaError_t configure_kernels(int n);
bool supported_size(int n);
void enqueue_step(const Geo &g, DevBufs &b, int cur, cudaStream_t s, cudaEvent_t *ev, const StepStreams *ss,
                  cudaEvent_t *kev = nullptr);
int kernels_per_step(const Geo &g, const Mov &m);
void enqueue_batch_step(int n, const MemberSet &ms, const BatchShape &bs, cudaStream_t s, cudaStream_t side,
                        cudaEvent_t fork, cudaEvent_t join);
int batch_kernels_per_step(const BatchShape &bs);
void enqueue_dem_init(const Mov &m, Scal *sc, cudaStream_t s);
cudaError_t configure_moving_kernels(const Mov &m);
void enqueue_c2r(const Geo &g, const double2 *a, double *b, int nplanes, cudaStream_t s);
void enqueue_r2c(const Geo &g, const double *a, double2 *b, int nplanes, cudaStream_t s);
void enqueue_f2d(const double2 *f, double2 *d, int nx, int nxf, int PS, int ncomp, cudaStream_t s);
void enqueue_d2f(const double2 *d, double2 *f, int nx, int nxf, int PS, int ncomp, cudaStream_t s);
int real_offset(int n, int z, int y);
int plane_ctas(int n);
void enqueue_scalar(const Geo &g, DevBufs &b, int cur, cudaStream_t s);
void enqueue_scalar_c2r(const Geo &g, const double2 *src, double *dst, int nplanes, cudaStream_t s);
int scalar_kernels_per_step(const Geo &g);
cudaError_t configure_scalar_kernels(int n);
void enqueue_adjoint_step(const Geo &g, const DevBufs &b, const AdjBufs &a, const double e[3], double wJ, cudaStream_t s);
void enqueue_adjoint_jacc(const Scal *sc, AdjScal *as, const double e[3], cudaStream_t s);
int adjoint_kernels_per_step(const Geo &g);
cudaError_t configure_adjoint_kernels(int n);
cudaError_t autotune_lines(Geo &g, DevBufs &b, int cur, cudaStream_t s, double ms[2]);
extern const int kLinesTiles[2];
}  // namespace pibm

using namespace pibm;

namespace {
thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
#define CUDA_OR_FAIL(expr)                                                                  \
    do {                                                                                    \
        cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess) return fail(PIBM_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

// e^{-2 pi i m/n} in extended precision, rounded to double.
std::vector<double2> twiddles(int n) {
    std::vector<double2> t(n);
    for (int m = 0; m < n; ++m) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
        t[m] = make_double2((double)cosl(a), (double)sinl(a));
    }
    return t;
}
}  // namespace

struct pibm_handle {
    RunSetup S;
    pibm_params prm;
    Geo g;                // the run's constants (stage 1)
    Geo gs[3];            // per stage rks: coef(rks, 1:4) and the dt update of the last stage
    int itrmax = 1;       // 1 (AB2) or 3 (RK3)
    int next_rks = 1;     // the rks the next pibm_step call is expected to run
    DevBufs b;
    std::vector<void *> allocs;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    unsigned geo_ver = 0; // bumped whenever the Geo copies change (graphs hold them by value)
    int cur = 0;          // buffer index the next step writes its nonlinear term to
    int device = 0;
    double2 *stage = nullptr;   // reference-layout staging buffer of get/set_state (allocated once)
    StepStreams ss;             // side streams of the forked step (graphs and pibm_step)
    AdjBufs adj{};              // adjoint work arrays (allocated by the first adjoint call)
    bool adj_ready = false;
    int adj_left = 0;           // host-driven sweep: reverse steps still expected
    double lines_ms[2] = {0.0, 0.0};   // autotuner: best time of each x-line tile width
    char *adj_fields = nullptr;        // host-driven sweep with RK3: the fields of the step's stages
    double adj_e[3] = {0, 0, 0}, adj_wJ = 0.0;

    template <class T> cudaError_t alloc(T **p, size_t n) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, n * sizeof(T) > 0 ? n * sizeof(T) : 16);
        if (e == cudaSuccess) { allocs.push_back(q); cudaMemset(q, 0, n * sizeof(T) > 0 ? n * sizeof(T) : 16); }
        *p = (T *)q;
        return e;
    }
    template <class T> cudaError_t upload(const T **p, const std::vector<T> &v) {
        T *q = nullptr;
        cudaError_t e = alloc(&q, v.size());
        if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(q, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
        *p = q;
        return e;
    }
    ~pibm_handle() {
        for (auto &gx : graph) if (gx) cudaGraphExecDestroy(gx);
        if (stream) cudaStreamDestroy(stream);
        if (ss.side) cudaStreamDestroy(ss.side);
        if (ss.scal) cudaStreamDestroy(ss.scal);
        for (cudaEvent_t e : {ss.fork, ss.drag_done, ss.scal_done, ss.geo_done, ss.rev_done, ss.frmean_done})
            if (e) cudaEventDestroy(e);
        for (void *q : allocs) cudaFree(q);
    }
};

// The step graphs hold the Geo copies by value: drop them after a change
// (recaptured by the next pibm_run; batches compare geo_ver).
static void drop_graphs(pibm_handle *h) {
    for (auto &gx : h->graph) if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
    ++h->geo_ver;
}

// Moving particles: DEM state on the device and the first neighbour search
// of des_time_march(.TRUE.) (DES_INIT_ARRAYS positions, FIND_CELL_INDEX).
static int setup_moving(pibm_handle *h) {
    const RunSetup &S = h->S;
    Geo &g = h->g;
    Mov &m = h->b.mov;
    std::memset(&m, 0, sizeof(m));
    const int N = S.nbody;
    m.N = N;
    m.maxn = 30 + 1 + 6;   // MN + 1 + NWALLS (collision_mod.F90:508)
    m.soft = S.dem_soft;
    m.cx = S.dem_cx; m.cy = S.dem_cy; m.cz = S.dem_cz;
    m.ncell = (m.cx - 1) * (m.cy - 1) * (m.cz - 1);
    m.dxc = S.dem_dxc; m.dyc = S.dem_dyc; m.dzc = S.dem_dzc;
    m.LXs = S.dem_LXs; m.LYs = S.dem_LYs; m.LZs = S.dem_LZs;
    m.XL = S.doml[0]; m.YL = S.doml[1]; m.ZL = S.doml[2];
    m.kn = S.dem_kn; m.eta_n = S.dem_eta_n; m.rad = S.dem_rad; m.pmass = S.dem_pmass; m.pvol = S.dem_pvol;
    m.rhof = h->prm.rhof; m.dtsolid = S.dem_dtsolid; m.max_radius = S.dem_rad;
    m.max_factor = m.soft ? std::max(1, (int)(S.dt / m.dtsolid)) : 1;
    m.kmax = S.my >= 256 ? 32 : 48;
    if (m.ncell > 8192 || 3 * m.ncell + 1 + N > 40000)
        return fail(PIBM_ERR_ARG, "moving particles: coarse DEM grid or particle count too large for the binning kernel");
    std::vector<double> pos(3 * (size_t)N);
    std::vector<int> pijk(3 * (size_t)N);
    const double dc[3] = {m.dxc, m.dyc, m.dzc};
    const int cm[3] = {m.cx, m.cy, m.cz};
    for (int l = 0; l < N; ++l) {
        pos[3 * l + 0] = (S.xc[l] + 0.0 - 1.0) * S.dx;
        pos[3 * l + 1] = (S.xc[l + (size_t)N] - 1.0) * S.dx;
        pos[3 * l + 2] = (S.xc[l + 2 * (size_t)N] - 1.0) * S.dx;
        for (int d = 0; d < 3; ++d) pijk[3 * l + d] = std::min((int)(pos[3 * l + d] / dc[d]) + 2, cm[d]);
    }
    std::vector<double> vel(3 * (size_t)N);
    for (int l = 0; l < N; ++l)
        for (int d = 0; d < 3; ++d) vel[3 * l + d] = S.vel[l + (size_t)d * N];
    int rc = PIBM_OK;
    auto guard = [&](cudaError_t e, const char *what) -> bool {
        if (e != cudaSuccess) { rc = fail(PIBM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)); return false; }
        return true;
    };
    const size_t NL = (size_t)N * m.maxn, nodes = (size_t)g.nx * g.RS;
    const int one = 1;
    bool ok = guard(h->alloc(&m.pos, 3 * (size_t)N), "dem pos") && guard(h->alloc(&m.pos_old, 3 * (size_t)N), "dem pos") &&
              guard(h->alloc(&m.vel, 3 * (size_t)N), "dem vel") && guard(h->alloc(&m.vel_old, 3 * (size_t)N), "dem vel") &&
              guard(h->alloc(&m.pijk, 3 * (size_t)N), "dem cells") && guard(h->alloc(&m.neigh, NL), "dem neighbours") &&
              guard(h->alloc(&m.ncnt, (size_t)N), "dem neighbours") && guard(h->alloc(&m.pn, NL), "dem contacts") &&
              guard(h->alloc(&m.pv, NL), "dem contacts") && guard(h->alloc(&m.pncnt, (size_t)N), "dem contacts") &&
              guard(h->alloc(&m.pn2, NL), "dem contacts") && guard(h->alloc(&m.pv2, NL), "dem contacts") &&
              guard(h->alloc(&m.pncnt2, (size_t)N), "dem contacts") && guard(h->alloc(&m.cstart, (size_t)m.ncell + 1), "dem cells") &&
              guard(h->alloc(&m.clist, (size_t)N), "dem cells") && guard(h->alloc(&m.factor, 1), "dem factor") &&
              guard(h->alloc(&m.dts, 1), "dem dts") && guard(h->alloc(&m.revflag, (size_t)N * S.nbnd), "revflag") &&
              guard(h->alloc(&m.nrpr, (size_t)N), "nrpr") && guard(h->alloc(&m.ptoff, (size_t)N), "ptoff") &&
              guard(h->alloc(&m.spcnt, nodes), "spread counts") && guard(h->alloc(&m.spbuf, nodes * (size_t)m.kmax), "spread buckets") &&
              guard(cudaMemcpy(m.pos, pos.data(), pos.size() * sizeof(double), cudaMemcpyHostToDevice), "dem pos") &&
              guard(cudaMemcpy(m.pos_old, pos.data(), pos.size() * sizeof(double), cudaMemcpyHostToDevice), "dem pos") &&
              guard(cudaMemcpy(m.vel, vel.data(), vel.size() * sizeof(double), cudaMemcpyHostToDevice), "dem vel") &&
              guard(cudaMemcpy(m.vel_old, vel.data(), vel.size() * sizeof(double), cudaMemcpyHostToDevice), "dem vel") &&
              guard(cudaMemcpy(m.pijk, pijk.data(), pijk.size() * sizeof(int), cudaMemcpyHostToDevice), "dem cells") &&
              guard(cudaMemcpy(m.factor, &one, sizeof(int), cudaMemcpyHostToDevice), "dem factor") &&
              guard(cudaMemcpy(m.revflag, S.if_rev.data(), S.if_rev.size(), cudaMemcpyHostToDevice), "revflag");
    if (!ok) return rc;
    if (g.scal) {
        ok = guard(h->alloc(&m.sev_cnt, (size_t)N), "sev counts") && guard(h->alloc(&m.sev_off, (size_t)N), "sev offsets") &&
             guard(h->alloc(&m.sspcnt, nodes), "scalar spread counts") &&
             guard(h->alloc(&m.sspbuf, nodes * (size_t)m.kmax), "scalar spread buckets");
        if (!ok) return rc;
        m.sev_m = const_cast<int *>(g.sev_m); m.sev_l = const_cast<int *>(g.sev_l);
        m.sev_c = const_cast<int *>(g.sev_c); m.sev_x = const_cast<double *>(g.sev_x);
    }
    m.xc = const_cast<double *>(g.xc);
    m.vel_ibm = const_cast<double *>(g.vel);
    m.fluid = const_cast<uint8_t *>(g.fluid);
    m.pt_m = const_cast<int *>(g.pt_m);
    m.pt_l = const_cast<int *>(g.pt_l);
    m.da2 = const_cast<double *>(g.da2);
    CUDA_OR_FAIL(configure_moving_kernels(m));
    enqueue_dem_init(m, h->b.sc, h->stream);
    CUDA_OR_FAIL(cudaGetLastError());
    Scal sc;
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    if (sc.status) return fail(sc.status, "moving particles: the first DEM neighbour search failed (list overflow)");
    return PIBM_OK;
}

// One time step = stages rks = 1..itrmax; stage k writes the nonlinear term
// into buffer cur ^ (k & 1) (the onl = nl swap of every nonlinear call).
static void enqueue_time_step(pibm_handle *h, int cur, cudaStream_t s, const StepStreams *ss) {
    for (int k = 0; k < h->itrmax; ++k) enqueue_step(h->gs[k], h->b, cur ^ (k & 1), s, nullptr, ss);
}

extern "C" {

const char *pibm_last_error(void) { return g_last_error.c_str(); }

int pibm_create(const pibm_params *prm, const pibm_particles *parts, pibm_handle **out) {
    if (!prm || !out) return fail(PIBM_ERR_ARG, "null argument");
    *out = nullptr;
    pibm_handle *h = new pibm_handle();
    h->prm = *prm;
    std::string err;
    if (!setup_run(*prm, parts, h->S, err)) { delete h; return fail(PIBM_ERR_ARG, err); }
    RunSetup &S = h->S;
    if (!supported_size(S.my)) { delete h; return fail(PIBM_ERR_ARG, "MY must be one of 32, 64, 96, 128, 256"); }
    int rc;
    auto guard = [&](cudaError_t e, const char *what) -> bool {
        if (e != cudaSuccess) { rc = fail(PIBM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)); return false; }
        return true;
    };
    if (!guard(cudaGetDevice(&h->device), "cudaGetDevice") || !guard(configure_kernels(S.my), "configure_kernels") ||
        !guard(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate") ||
        !guard(cudaStreamCreateWithFlags(&h->ss.side, cudaStreamNonBlocking), "cudaStreamCreate") ||
        !guard(cudaStreamCreateWithFlags(&h->ss.scal, cudaStreamNonBlocking), "cudaStreamCreate") ||
        !guard(cudaEventCreateWithFlags(&h->ss.fork, cudaEventDisableTiming), "cudaEventCreate") ||
        !guard(cudaEventCreateWithFlags(&h->ss.drag_done, cudaEventDisableTiming), "cudaEventCreate") ||
        !guard(cudaEventCreateWithFlags(&h->ss.scal_done, cudaEventDisableTiming), "cudaEventCreate") ||
        !guard(cudaEventCreateWithFlags(&h->ss.geo_done, cudaEventDisableTiming), "cudaEventCreate") ||
        !guard(cudaEventCreateWithFlags(&h->ss.rev_done, cudaEventDisableTiming), "cudaEventCreate") ||
        !guard(cudaEventCreateWithFlags(&h->ss.frmean_done, cudaEventDisableTiming), "cudaEventCreate")) { delete h; return rc; }
    Geo &g = h->g;
    std::memset(&g, 0, sizeof(g));
    g.nx = S.nx; g.my = S.my; g.mz = S.mz; g.my2 = S.my2;
    g.PS = S.my2 * S.mz; g.RS = (S.my + 2) * S.mz;   // physical real plane: rows of my+2 doubles
    g.dx = S.dx; g.dx2 = S.dx2; g.rdx2 = 1.0 / S.dx2; g.dx3 = S.dx3; g.vis = S.vis;
    g.nrm = (double)(float)(S.my * S.mz);
    g.plane_ctas = plane_ctas(S.my);
    g.c1 = S.coef[0]; g.c2 = S.coef[1]; g.c3 = S.coef[2]; g.c4 = S.coef[3];
    g.scheme = prm->discr_scheme; g.limiter = prm->limiter;
    g.flux_seg = flux_segment(S.my, S.scal);
    g.include_frmeanfluid = prm->include_frmeanfluid; g.revernorm = prm->revernorm;
    g.set_mpg = prm->set_mpg; g.adaptive = prm->adaptive; g.dt_update = 1;
    g.cfl_max = prm->cfl_max; g.ramp_frac_time = S.ramp_frac_time; g.ucharmod = S.ucharmod;
    g.char_length = S.char_length; g.voldom = S.voldom; g.maxvolfrac = S.maxvolfrac; g.mean_volfrac = S.mean_volfrac;
    g.count_fluid = S.count_fluid; g.ncell = (long long)S.nx * S.my * S.mz;
    for (int d = 0; d < 3; ++d) { g.ufmean_des[d] = S.ufmean_des[d]; g.usmean_des[d] = S.usmean_des[d]; g.usmean_act[d] = S.usmean_des[d]; }
    g.nbody = S.nbody; g.nbnd = S.nbnd; g.npts = (int)S.pt_m.size();
    g.rhof = prm->rhof; g.rhos = prm->rhos;
    g.moving = S.moving ? 1 : 0;
    // moving particles: the point lists are rebuilt every step, sized for all points
    std::vector<int> pt_m = S.pt_m, pt_l = S.pt_l;
    if (g.moving) { g.npts = S.nbody * S.nbnd; pt_m.resize((size_t)g.npts, 0); pt_l.resize((size_t)g.npts, 0); }
    g.rb = S.radbdy; g.ri = S.radibdy; g.ro = S.radobdy; g.dr = S.dr;
    g.da1 = 4.0 * 3.14159265358979323846 * ((S.radbdy * S.dx) * (S.radbdy * S.dx)) / (double)S.nbnd;
    g.sphere_vol = 3.14159265358979323846 * std::pow(2.0 * S.radbdy * S.dx, 3.0) / 6.0;
    g.sp_nnodes = (int)S.sp_node.size();
    std::vector<double> da2(S.nbody);
    for (int m = 0; m < S.nbody; ++m)
        da2[m] = 4.0 * 3.14159265358979323846 * ((S.radibdy * S.dx) * (S.radibdy * S.dx)) / (double)S.nrpr_active[m];
    std::vector<double2> tw = twiddles(S.my);
    const size_t NC = (size_t)g.nx * g.PS, NR = (size_t)g.nx * g.RS;
    // physical fields are stored in the plane-transform order: permute the
    // solid mask and the spreading targets accordingly
    const int nat = S.my * S.mz;   // natural plane size of the set-up arrays
    std::vector<int> roff((size_t)nat);
    for (int z = 0; z < S.mz; ++z)
        for (int y = 0; y < S.my; ++y) roff[(size_t)z * S.my + y] = real_offset(S.my, z, y);
    std::vector<uint8_t> fluid_p((size_t)S.nx * g.RS, 1);
    for (int i = 0; i < S.nx; ++i)
        for (int e = 0; e < nat; ++e) fluid_p[(size_t)i * g.RS + roff[e]] = S.fluid[(size_t)i * nat + e];
    std::vector<int> sp_node_p(S.sp_node.size());
    for (size_t q = 0; q < S.sp_node.size(); ++q) {
        const int node = S.sp_node[q], i = node / nat, e = node - i * nat;
        sp_node_p[q] = i * g.RS + roff[e];
    }
    DevBufs &b = h->b;
    bool ok = guard(h->upload(&g.tw, tw), "tw") && guard(h->upload(&g.ky, S.ky), "ky") && guard(h->upload(&g.kz, S.kz), "kz") &&
              guard(h->upload(&g.w2, S.w2), "w2") && guard(h->upload(&g.fluid, fluid_p), "mask") &&
              guard(h->upload(&g.xc, S.xc), "xc") && guard(h->upload(&g.vel, S.vel), "vel") &&
              guard(h->upload(&g.bnd, S.bnd), "bnd") && guard(h->upload(&g.cd, S.cd), "cd") &&
              guard(h->upload(&g.pt_m, pt_m), "pt_m") && guard(h->upload(&g.pt_l, pt_l), "pt_l") &&
              guard(h->upload(&g.da2, da2), "da2") && guard(h->upload(&g.sp_node, sp_node_p), "sp_node") &&
              guard(h->upload(&g.sp_ptr, S.sp_ptr), "sp_ptr") && guard(h->upload(&g.sp_ent, S.sp_ent), "sp_ent") &&
              guard(h->alloc(&b.u, 3 * NC), "u") && guard(h->alloc(&b.p, NC), "p") &&
              guard(h->alloc(&b.nl[0], 3 * NC), "nl0") && guard(h->alloc(&b.nl[1], 3 * NC), "nl1") &&
              guard(h->alloc(&b.ff, 3 * NC), "ff") && guard(h->alloc(&b.ubcp, 3 * NR), "ubcp") &&
              guard(h->alloc(&b.pbcp, NR), "pbcp") && guard(h->alloc(&b.Q, 3 * NR), "Q") && guard(h->alloc(&b.Dx, 3 * NR), "Dx") &&
              guard(h->alloc(&b.omega, 3 * NR), "omega") && guard(h->alloc(&b.pgr, 3 * NR), "pgr") &&
              (S.nbody == 0 || guard(h->alloc(&b.fr, 3 * NR), "fr")) &&
              guard(h->alloc(&b.part, (size_t)g.nx * 8 * 12), "part") &&
              guard(h->alloc(&b.pres, 3 * (size_t)S.nbody), "pres") && guard(h->alloc(&b.visc, 3 * (size_t)S.nbody), "visc") &&
              guard(h->alloc(&b.ptot, 3 * (size_t)S.nbody), "ptot") && guard(h->alloc(&b.force, 3 * (size_t)S.nbody), "force") &&
              guard(h->alloc(&b.rec, 6 * (size_t)g.npts), "rec") && guard(h->alloc(&b.rz, 3 * (size_t)g.npts), "rz") &&
              guard(h->alloc(&b.dpart, 6 * 8 * (size_t)S.nbody), "dpart") &&
              guard(h->alloc(&b.blockpart, 6 * (size_t)((g.npts + 255) / 256 + 1)), "blockpart") &&
              guard(h->alloc(&b.sc, 1), "scalars");
    if (!ok) { delete h; return rc; }
    if (S.scal) {
        // passive scalar: geometry of the reversal-point evaluations, the
        // spreading map in plane-transform order, and phi = 1 (scalar_init.F90:136-152)
        g.scal = 1; g.gamma_s = S.gamma_s; g.phisurf = S.phisurf; g.phistream = S.phistream;
        g.nsev = (int)S.sev_m.size();
        if (g.moving) g.nsev = 2 * S.nbody * S.nbnd;   // rebuilt every step: capacity
        g.ssp_nnodes = (int)S.ssp_node.size();
        std::vector<int> ssp_node_p(S.ssp_node.size());
        for (size_t q = 0; q < S.ssp_node.size(); ++q) {
            const int node = S.ssp_node[q], i = node / nat, e = node - i * nat;
            ssp_node_p[q] = i * g.RS + roff[e];
        }
        std::vector<double2> phi0(NC, make_double2(0.0, 0.0));
        for (int i = 0; i < g.nx; ++i) phi0[(size_t)i * g.PS] = make_double2(1.0, 0.0);
        const size_t NR1 = (size_t)(g.nx + 1) * g.RS, nsev = (size_t)g.nsev;
        std::vector<int> sev_m = S.sev_m, sev_l = S.sev_l, sev_c = S.sev_c;
        std::vector<double> sev_x = S.sev_x;
        if (g.moving) { sev_m.resize(nsev, 0); sev_l.resize(nsev, 0); sev_c.resize(3 * nsev, 0); sev_x.resize(3 * nsev, 0.0); }
        ok = guard(h->upload(&g.sev_m, sev_m), "sev_m") && guard(h->upload(&g.sev_l, sev_l), "sev_l") &&
             guard(h->upload(&g.sev_c, sev_c), "sev_c") && guard(h->upload(&g.sev_x, sev_x), "sev_x") &&
             guard(h->upload(&g.ssp_node, ssp_node_p), "ssp_node") && guard(h->upload(&g.ssp_ptr, S.ssp_ptr), "ssp_ptr") &&
             guard(h->upload(&g.ssp_ent, S.ssp_ent), "ssp_ent") &&
             guard(h->alloc(&b.phif, NC), "phif") && guard(h->alloc(&b.nls[0], NC), "nls0") &&
             guard(h->alloc(&b.nls[1], NC), "nls1") && guard(h->alloc(&b.ffs, NC), "ffs") &&
             guard(h->alloc(&b.phr, NR), "phr") && guard(h->alloc(&b.phimg, (size_t)g.RS), "phimg") &&
             guard(h->alloc(&b.nlr[0], NR1), "nlr0") && guard(h->alloc(&b.nlr[1], NR1), "nlr1") &&
             guard(h->alloc(&b.sdf, NR1), "sdf") && guard(h->alloc(&b.gph, 3 * NR1), "gph") &&
             guard(h->alloc(&b.sfr, NR), "sfr") && guard(h->alloc(&b.dsx, NR), "dsx") &&
             guard(h->alloc(&b.spart, 8 * 3), "spart") && guard(h->alloc(&b.sctb, 8 * nsev), "sctb") &&
             guard(h->alloc(&b.sfd, nsev), "sfd") && guard(h->alloc(&b.sdpart, 8 * (size_t)S.nbody), "sdpart") &&
             guard(h->alloc(&b.flux_body, (size_t)S.nbody), "flux_body") &&
             guard(cudaMemcpy(b.phif, phi0.data(), NC * sizeof(double2), cudaMemcpyHostToDevice), "phi0") &&
             guard(configure_scalar_kernels(S.my), "configure_scalar_kernels");
        if (!ok) { delete h; return rc; }
    }
    Scal sc;
    std::memset(&sc, 0, sizeof(sc));
    for (int d = 0; d < 3; ++d) { sc.umean[d] = S.umean0[d]; sc.mpg[d] = prm->mpg[d]; }
    sc.dt = S.dt; sc.cf = S.cf; sc.cforig = S.cf; sc.t = 0.0; sc.fold = 0.0; sc.ferror = 1.0;
    sc.heat_ratio = sc.heat_ratio_old = sc.heat_ratio_new = 1.0;
    sc.count_solid = S.count_solid; sc.count_fluid = S.count_fluid; sc.maxvolfrac = S.maxvolfrac;
    sc.npts = (int)S.pt_m.size();
    sc.nsev = (int)S.sev_m.size();
    for (int d = 0; d < 3; ++d) { sc.usmean_act[d] = S.usmean_des[d]; sc.frame_vel[d] = 0.0; sc.frame_pos[d] = 1.0; }
    if (!guard(cudaMemcpy(b.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice), "scalars")) { delete h; return rc; }
    if (g.moving && (rc = setup_moving(h)) != PIBM_OK) { delete h; return rc; }
    // x-line tile width measured on this run's grid
    if (!guard(autotune_lines(g, h->b, h->cur, h->stream, h->lines_ms), "x-line tile autotune")) { delete h; return rc; }
    // time-integration stages (initialize_flo.F90:861-884)
    static const double kAB2[4] = {0.5, 0.5, 3.0 / 2.0, -0.5};
    static const double kRK3[3][4] = {{4.0 / 15.0, 4.0 / 15.0, 8.0 / 15.0, 0.0},
                                      {1.0 / 15.0, 1.0 / 15.0, 5.0 / 12.0, -17.0 / 60.0},
                                      {1.0 / 6.0, 1.0 / 6.0, 3.0 / 4.0, -5.0 / 12.0}};
    h->itrmax = prm->rk3 ? 3 : 1;
    for (int k = 0; k < h->itrmax; ++k) {
        const double *c = prm->rk3 ? kRK3[k] : kAB2;
        h->gs[k] = g;
        h->gs[k].c1 = c[0]; h->gs[k].c2 = c[1]; h->gs[k].c3 = c[2]; h->gs[k].c4 = c[3];
        h->gs[k].dt_update = k == h->itrmax - 1;
    }
    g = h->gs[0];
    *out = h;
    return PIBM_OK;
}

int pibm_info_get(pibm_handle *h, pibm_info *info) {
    if (!h || !info) return fail(PIBM_ERR_ARG, "null argument");
    const RunSetup &S = h->S;
    info->nx = S.nx; info->my = S.my; info->mz = S.mz; info->my2 = S.my2; info->nbody = S.nbody; info->nbnd = S.nbnd;
    info->dx = S.dx; info->dt = S.dt; info->radbdy = S.radbdy; info->maxvolfrac = S.maxvolfrac;
    info->count_solid = S.count_solid; info->count_fluid = S.count_fluid;
    info->npts_active = (int32_t)S.pt_m.size();
    info->kernels_per_step = kernels_per_step(h->g, h->b.mov) * h->itrmax;
    return PIBM_OK;
}

static int fill_report(pibm_handle *h, pibm_step_report *rep) {
    Scal sc;
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        rep->dt = sc.dt; rep->t = sc.t; rep->cf = sc.cf; rep->umax = sc.umax;
        long long bits = (long long)sc.divmax_bits;
        std::memcpy(&rep->divmax, &bits, sizeof(double));
        for (int d = 0; d < 3; ++d) {
            rep->ufmean[d] = sc.ufmean[d]; rep->usmean[d] = sc.usmean[d]; rep->umean[d] = sc.umean[d];
            rep->mpg[d] = sc.mpg[d]; rep->frmean[d] = sc.frmean[d];
            rep->pres_total[d] = sc.pres_total[d]; rep->visc_total[d] = sc.visc_total[d];
        }
        rep->norm_drag = sc.norm_drag; rep->ferror = sc.ferror;
        rep->pres_drag = sc.pres_drag; rep->visc_drag = sc.visc_drag; rep->total_drag = sc.total_drag;
        rep->mixmeanslipmod = sc.mixmeanslipmod;
        rep->heat_ratio = sc.heat_ratio;
        rep->nusselt = sc.nusselt;
        long long s = 0;
        for (int v : h->S.nrpr_active) s += v;
        rep->nrpr_active_total = h->g.moving ? (long long)sc.npts : s;
    }
    if (sc.status) return fail(sc.status, "step reported a solver stop condition");
    return PIBM_OK;
}

int pibm_step(pibm_handle *h, int rks, pibm_step_report *rep) {
    if (!h) return fail(PIBM_ERR_ARG, "null handle");
    if (rks < 1 || rks > h->itrmax) return fail(PIBM_ERR_ARG, h->itrmax == 1 ? "AB2 has a single stage (rks = 1)" : "rks must be 1, 2 or 3 (RK3)");
    if (rks != h->next_rks) return fail(PIBM_ERR_ARG, "stages must run in the order rks = 1..itrmax");
    enqueue_step(h->gs[rks - 1], h->b, h->cur, h->stream, nullptr, &h->ss);
    CUDA_OR_FAIL(cudaGetLastError());
    h->cur ^= 1;
    h->next_rks = rks == h->itrmax ? 1 : rks + 1;
    return fill_report(h, rep);
}

int pibm_run(pibm_handle *h, int nsteps, pibm_step_report *last) {
    if (!h || nsteps < 0) return fail(PIBM_ERR_ARG, "bad argument");
    if (h->next_rks != 1) return fail(PIBM_ERR_ARG, "pibm_run starts at a step boundary (finish the rks stages with pibm_step)");
    for (int par = 0; par < 2; ++par) {
        if (h->graph[par]) continue;
        cudaGraph_t gr;
        CUDA_OR_FAIL(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_time_step(h, par, h->stream, &h->ss);
        CUDA_OR_FAIL(cudaStreamEndCapture(h->stream, &gr));
        CUDA_OR_FAIL(cudaGraphInstantiate(&h->graph[par], gr, 0));
        cudaGraphDestroy(gr);
    }
    for (int s = 0; s < nsteps; ++s) {
        CUDA_OR_FAIL(cudaGraphLaunch(h->graph[h->cur], h->stream));
        h->cur ^= 1;
    }
    return fill_report(h, last);
}

int pibm_run_timed(pibm_handle *h, int nsteps, pibm_step_report *last, double *total_ms) {
    if (!h || nsteps <= 0 || !total_ms) return fail(PIBM_ERR_ARG, "bad argument");
    int rc = pibm_run(h, 0, nullptr);   // captures the step graphs on first use
    if (rc) return rc;
    cudaEvent_t e0, e1;
    CUDA_OR_FAIL(cudaEventCreate(&e0));
    CUDA_OR_FAIL(cudaEventCreate(&e1));
    CUDA_OR_FAIL(cudaEventRecord(e0, h->stream));
    for (int s = 0; s < nsteps; ++s) {
        CUDA_OR_FAIL(cudaGraphLaunch(h->graph[h->cur], h->stream));
        h->cur ^= 1;
    }
    CUDA_OR_FAIL(cudaEventRecord(e1, h->stream));
    CUDA_OR_FAIL(cudaEventSynchronize(e1));
    float ms = 0.f;
    CUDA_OR_FAIL(cudaEventElapsedTime(&ms, e0, e1));
    *total_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return fill_report(h, last);
}

int pibm_run_profiled(pibm_handle *h, int nsteps, pibm_step_report *last, double *total_ms, double *phase_ms, int nphase) {
    if (!h || nsteps <= 0 || nphase < 0 || nphase > PIBM_NPHASE) return fail(PIBM_ERR_ARG, "bad argument");
    if (h->next_rks != 1) return fail(PIBM_ERR_ARG, "pibm_run_profiled starts at a step boundary");
    const int nst = nsteps * h->itrmax;   // stages, each with its own phase events
    std::vector<cudaEvent_t> ev((size_t)nst * (PIBM_NPHASE + 1));
    for (auto &e : ev) CUDA_OR_FAIL(cudaEventCreate(&e));
    for (int s = 0; s < nst; ++s) {
        enqueue_step(h->gs[s % h->itrmax], h->b, h->cur, h->stream, &ev[(size_t)s * (PIBM_NPHASE + 1)], nullptr);
        h->cur ^= 1;
    }
    CUDA_OR_FAIL(cudaGetLastError());
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    for (int q = 0; q < nphase; ++q) phase_ms[q] = 0.0;
    for (int s = 0; s < nst; ++s)
        for (int q = 0; q < nphase; ++q) {
            float ms = 0.f;
            CUDA_OR_FAIL(cudaEventElapsedTime(&ms, ev[(size_t)s * (PIBM_NPHASE + 1) + q], ev[(size_t)s * (PIBM_NPHASE + 1) + q + 1]));
            phase_ms[q] += ms;
        }
    if (total_ms) {
        float ms = 0.f;
        CUDA_OR_FAIL(cudaEventElapsedTime(&ms, ev.front(), ev.back()));
        *total_ms = ms;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return fill_report(h, last);
}

int pibm_kernel_times(pibm_handle *h, int nsteps, double *total_ms, double *kernel_ms, int nkernel) {
    if (!h || nsteps <= 0 || nkernel < 0 || nkernel > PIBM_NKERNEL || (nkernel > 0 && !kernel_ms))
        return fail(PIBM_ERR_ARG, "bad argument");
    if (h->next_rks != 1) return fail(PIBM_ERR_ARG, "pibm_kernel_times starts at a step boundary");
    const int nst = nsteps * h->itrmax;
    const size_t per = 2 * (size_t)PIBM_NKERNEL;
    std::vector<cudaEvent_t> ev((size_t)nst * per);
    for (auto &e : ev) CUDA_OR_FAIL(cudaEventCreate(&e));
    for (int s = 0; s < nst; ++s) {
        enqueue_step(h->gs[s % h->itrmax], h->b, h->cur, h->stream, nullptr, nullptr, &ev[(size_t)s * per]);
        h->cur ^= 1;
    }
    CUDA_OR_FAIL(cudaGetLastError());
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < nkernel; ++k) kernel_ms[k] = 0.0;
    for (int s = 0; s < nst; ++s)
        for (int k = 0; k < nkernel; ++k) {
            float ms = 0.f;
            CUDA_OR_FAIL(cudaEventElapsedTime(&ms, ev[(size_t)s * per + 2 * k], ev[(size_t)s * per + 2 * k + 1]));
            kernel_ms[k] += ms;
        }
    if (total_ms) {
        float ms = 0.f;
        CUDA_OR_FAIL(cudaEventElapsedTime(&ms, ev.front(), ev[(size_t)(nst - 1) * per + 2 * PIBM_K_SCAL_D + 1]));
        *total_ms = ms;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return fill_report(h, nullptr);
}

const char *pibm_kernel_name(int k) {
    static const char *names[PIBM_NKERNEL] = {"k_a0", "k_scal_a", "k_flux", "k_nl", "k_drag", "k_scal_b",
                                              "k_rev", "k_scal_c", "k_spread", "k_ff", "k_lines", "k_scal_d"};
    return (k >= 0 && k < PIBM_NKERNEL) ? names[k] : nullptr;
}

int pibm_get_state(pibm_handle *h, pibm_state_view *s) {
    if (!h || !s) return fail(PIBM_ERR_ARG, "null argument");
    const Geo &g = h->g;
    const int nxf = g.nx + 1;
    const size_t nfu = (size_t)nxf * g.PS * 3, nfp = (size_t)g.nx * g.PS;
    if (!h->stage) CUDA_OR_FAIL(h->alloc(&h->stage, nfu));
    double2 *tmp = h->stage;
    const int prev = h->cur ^ 1;   // buffer holding the latest nl
    if (s->u) {
        enqueue_d2f(h->b.u, tmp, g.nx, nxf, g.PS, 3, h->stream);
        CUDA_OR_FAIL(cudaMemcpyAsync(s->u, tmp, nfu * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    }
    if (s->nl) {
        enqueue_d2f(h->b.nl[prev], tmp, g.nx, nxf, g.PS, 3, h->stream);
        CUDA_OR_FAIL(cudaMemcpyAsync(s->nl, tmp, nfu * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    }
    if (s->p) {
        enqueue_d2f(h->b.p, tmp, g.nx, g.nx, g.PS, 1, h->stream);
        CUDA_OR_FAIL(cudaMemcpyAsync(s->p, tmp, nfp * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    }
    Scal sc;
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    for (int d = 0; d < 3; ++d) { s->umean[d] = sc.umean[d]; s->mpg[d] = sc.mpg[d]; s->ufmean[d] = sc.ufmean[d]; }
    s->t = sc.t; s->dt = sc.dt; s->cf = sc.cf;
    return PIBM_OK;
}

int pibm_set_state(pibm_handle *h, const pibm_state_view *s) {
    if (!h || !s) return fail(PIBM_ERR_ARG, "null argument");
    const Geo &g = h->g;
    const int nxf = g.nx + 1;
    const size_t nfu = (size_t)nxf * g.PS * 3, nfp = (size_t)g.nx * g.PS;
    if (!h->stage) CUDA_OR_FAIL(h->alloc(&h->stage, nfu));
    double2 *tmp = h->stage;
    const int prev = h->cur ^ 1;
    if (s->u) {
        CUDA_OR_FAIL(cudaMemcpyAsync(tmp, s->u, nfu * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
        enqueue_f2d(tmp, h->b.u, g.nx, nxf, g.PS, 3, h->stream);
    }
    if (s->nl) {
        CUDA_OR_FAIL(cudaMemcpyAsync(tmp, s->nl, nfu * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
        enqueue_f2d(tmp, h->b.nl[prev], g.nx, nxf, g.PS, 3, h->stream);
    }
    if (s->p) {
        CUDA_OR_FAIL(cudaMemcpyAsync(tmp, s->p, nfp * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
        enqueue_f2d(tmp, h->b.p, g.nx, g.nx, g.PS, 1, h->stream);
    }
    Scal sc;
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    for (int d = 0; d < 3; ++d) { sc.umean[d] = s->umean[d]; sc.mpg[d] = s->mpg[d]; sc.ufmean[d] = s->ufmean[d]; }
    sc.t = s->t; sc.dt = s->dt; sc.cf = s->cf;
    sc.status = 0;
    h->next_rks = 1;   // a restart begins a time step
    if (h->g.moving && h->S.dem_soft) {
        // the step graphs hold max_factor DEM sub-steps; a larger dt needs more
        Mov &m = h->b.mov;
        const int need = std::max(1, (int)(s->dt / m.dtsolid));
        if (need > m.max_factor) {
            m.max_factor = need;
            drop_graphs(h);
        }
    }
    CUDA_OR_FAIL(cudaMemcpyAsync(h->b.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    return PIBM_OK;
}

int pibm_get_particles(pibm_handle *h, double *pres, double *visc, double *force, double *xc, double *vel) {
    if (!h) return fail(PIBM_ERR_ARG, "null handle");
    const size_t n = (size_t)h->S.nbody * 3;
    if (n == 0) return PIBM_OK;
    if (pres) CUDA_OR_FAIL(cudaMemcpyAsync(pres, h->b.pres, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (visc) CUDA_OR_FAIL(cudaMemcpyAsync(visc, h->b.visc, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (force) CUDA_OR_FAIL(cudaMemcpyAsync(force, h->b.force, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (h->g.moving) {   // the positions and velocities the DEM has advanced
        if (xc) CUDA_OR_FAIL(cudaMemcpyAsync(xc, h->g.xc, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        if (vel) CUDA_OR_FAIL(cudaMemcpyAsync(vel, h->g.vel, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    if (!h->g.moving) {
        if (xc) std::memcpy(xc, h->S.xc.data(), n * sizeof(double));
        if (vel) std::memcpy(vel, h->S.vel.data(), n * sizeof(double));
    }
    return PIBM_OK;
}

// ---------------------------------------------------------------------------
// Discrete adjoint: forward with checkpoints, reverse sweep segment by segment.
// A state slot holds u, p, the latest nl (the next step's onl) and Scal; the
// parity of the nl ping-pong at the slot is kept on the host.
// ---------------------------------------------------------------------------
namespace {
struct SlotSet {
    char *base = nullptr;
    size_t bytes = 0;          // per slot
    std::vector<int> cur;
};
size_t slot_bytes(const pibm_handle *h) {
    const size_t SC = (size_t)h->g.nx * h->g.PS * sizeof(double2);
    return 7 * SC + ((sizeof(Scal) + 255) / 256) * 256;
}
void slot_save(pibm_handle *h, char *slot) {
    const size_t SC = (size_t)h->g.nx * h->g.PS * sizeof(double2);
    cudaMemcpyAsync(slot, h->b.u, 3 * SC, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(slot + 3 * SC, h->b.p, SC, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(slot + 4 * SC, h->b.nl[h->cur ^ 1], 3 * SC, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(slot + 7 * SC, h->b.sc, sizeof(Scal), cudaMemcpyDeviceToDevice, h->stream);
}
void slot_restore(pibm_handle *h, const char *slot, int cur) {
    const size_t SC = (size_t)h->g.nx * h->g.PS * sizeof(double2);
    h->cur = cur;
    cudaMemcpyAsync(h->b.u, slot, 3 * SC, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->b.p, slot + 3 * SC, SC, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->b.nl[h->cur ^ 1], slot + 4 * SC, 3 * SC, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->b.sc, slot + 7 * SC, sizeof(Scal), cudaMemcpyDeviceToDevice, h->stream);
}
}  // namespace

// Fields of one stage that its adjoint reads: ubcp(3) pbcp omega(3) pgr(3)
// Q(3) real components, the point forces rec and the stage's Scal.
static size_t fields_bytes(const pibm_handle *h, size_t *crb, size_t *recb) {
    const Geo &g = h->g;
    *crb = (size_t)g.nx * (size_t)g.RS * sizeof(double);
    *recb = ((6 * (size_t)g.npts * sizeof(double) + 255) / 256) * 256;
    return 13 * *crb + *recb + ((sizeof(Scal) + 255) / 256) * 256;
}
static void fields_save(pibm_handle *h, char *f) {
    size_t CRb, recb;
    fields_bytes(h, &CRb, &recb);
    cudaStream_t s = h->stream;
    cudaMemcpyAsync(f, h->b.ubcp, 3 * CRb, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(f + 3 * CRb, h->b.pbcp, CRb, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(f + 4 * CRb, h->b.omega, 3 * CRb, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(f + 7 * CRb, h->b.pgr, 3 * CRb, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(f + 10 * CRb, h->b.Q, 3 * CRb, cudaMemcpyDeviceToDevice, s);
    if (h->g.npts > 0) cudaMemcpyAsync(f + 13 * CRb, h->b.rec, 6 * (size_t)h->g.npts * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(f + 13 * CRb + recb, h->b.sc, sizeof(Scal), cudaMemcpyDeviceToDevice, s);
}
static DevBufs fields_view(const pibm_handle *h, char *f) {
    size_t CRb, recb;
    fields_bytes(h, &CRb, &recb);
    DevBufs v = h->b;
    v.ubcp = (double *)f;
    v.pbcp = (double *)(f + 3 * CRb);
    v.omega = (double *)(f + 4 * CRb);
    v.pgr = (double *)(f + 7 * CRb);
    v.Q = (double *)(f + 10 * CRb);
    v.rec = (double *)(f + 13 * CRb);
    v.sc = (Scal *)(f + 13 * CRb + recb);
    return v;
}
// The stages of one time step from the current state, each stage's fields
// kept in slots f0 + k*fb (the parity of the nl ping-pong flips per stage).
static void stages_with_fields(pibm_handle *h, char *f0, size_t fb) {
    for (int k = 0; k < h->itrmax; ++k) {
        enqueue_step(h->gs[k], h->b, h->cur, h->stream, nullptr, &h->ss);
        h->cur ^= 1;
        fields_save(h, f0 + fb * (size_t)k);
    }
}

static int adjoint_check(pibm_handle *h) {
    const Geo &g = h->g;
    if (g.moving || g.scal || !g.set_mpg || g.adaptive || !h->prm.dorpr || g.nbody < 1)
        return fail(PIBM_ERR_ARG, "adjoint: fixed spheres, SET_MPG, ADAPTIVE = F, DORPR and no scalar only");
    if (h->next_rks != 1) return fail(PIBM_ERR_ARG, "the adjoint starts at a step boundary");
    return PIBM_OK;
}
// adjoint work arrays, allocated on first use and kept by the handle
static int adjoint_alloc(pibm_handle *h) {
    const Geo &g = h->g;
    AdjBufs &a = h->adj;
    const size_t SC = (size_t)g.nx * g.PS, CR = (size_t)g.nx * (size_t)(g.my * (g.my + 2));
    if (!h->adj_ready) {
        CUDA_OR_FAIL(configure_adjoint_kernels(g.my));
        double *R10 = nullptr;
        const bool ok = h->alloc(&a.lu, 3 * SC) == cudaSuccess && h->alloc(&a.lp, SC) == cudaSuccess &&
                        h->alloc(&a.lnl, 3 * SC) == cudaSuccess && h->alloc(&a.lu2, 3 * SC) == cudaSuccess &&
                        h->alloc(&a.lp2, SC) == cudaSuccess && h->alloc(&a.lnl_new, 3 * SC) == cudaSuccess &&
                        h->alloc(&a.lonl, 3 * SC) == cudaSuccess && h->alloc(&a.lff, 3 * SC) == cudaSuccess &&
                        h->alloc(&a.T, 10 * SC) == cudaSuccess && h->alloc(&a.lfr, 3 * CR) == cudaSuccess &&
                        h->alloc(&R10, 10 * CR) == cudaSuccess && h->alloc(&a.lQ, 3 * CR) == cudaSuccess &&
                        h->alloc(&a.W8, 8 * CR) == cudaSuccess && h->alloc(&a.gxc, 3 * (size_t)g.nbody) == cudaSuccess &&
                        h->alloc(&a.as, 1) == cudaSuccess;
        if (!ok) return fail(PIBM_ERR_NOMEM, "adjoint work arrays");
        a.lubcp = R10; a.lomega = R10 + 3 * CR; a.lpbcp = R10 + 6 * CR; a.lpgr = R10 + 7 * CR;
        h->adj_ready = true;
    }
    return PIBM_OK;
}
// zero the adjoint state and the gradients
static void adjoint_zero(pibm_handle *h) {
    const Geo &g = h->g;
    AdjBufs &a = h->adj;
    const size_t SC = (size_t)g.nx * g.PS;
    cudaMemsetAsync(a.lu, 0, 3 * SC * sizeof(double2), h->stream);
    cudaMemsetAsync(a.lp, 0, SC * sizeof(double2), h->stream);
    cudaMemsetAsync(a.lnl, 0, 3 * SC * sizeof(double2), h->stream);
    cudaMemsetAsync(a.gxc, 0, 3 * (size_t)g.nbody * sizeof(double), h->stream);
    cudaMemsetAsync(a.as, 0, sizeof(AdjScal), h->stream);
}

int pibm_adjoint_run(pibm_handle *h, int nsteps, int checkpoint_every, const double direction[3], double *g_xc, double g_mpg[3],
                     pibm_adjoint_report *rep) {
    if (!h || nsteps < 1 || !direction || !g_xc || !g_mpg) return fail(PIBM_ERR_ARG, "bad argument");
    const Geo &g = h->g;
    int rc = adjoint_check(h);
    if (rc) return rc;
    if ((rc = pibm_run(h, 0, nullptr))) return rc;   // step graphs
    AdjBufs &a = h->adj;
    if ((rc = adjoint_alloc(h))) return rc;
    const int K = nsteps, S = h->itrmax;
    // state slots (checkpoints and the final state) and, for one segment, the
    // fields every reverse stage reads
    const size_t sb = slot_bytes(h);
    size_t CRb, recb;
    const size_t fb = fields_bytes(h, &CRb, &recb);
    int ck = checkpoint_every;
    if (ck <= 0) {   // as many steps per segment as 80% of the free memory holds
        size_t fr = 0, tot = 0;
        CUDA_OR_FAIL(cudaMemGetInfo(&fr, &tot));
        const double per_step = (double)fb * S + (double)sb;
        ck = (int)std::max(1.0, std::min((double)K, 0.8 * (double)fr / per_step));
    }
    const int nseg = (K + ck - 1) / ck, seglen = std::min(ck, K);
    const int last0 = (nseg - 1) * ck;   // the last segment keeps its fields in the forward pass
    // the slot pool and the timing events live for this call only; released on every return path
    struct Scratch {
        char *pool = nullptr;
        cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
        ~Scratch() {
            for (auto &x : ev) if (x) cudaEventDestroy(x);
            if (pool) cudaFree(pool);
        }
    } scratch;
    CUDA_OR_FAIL(cudaMalloc(&scratch.pool, sb * (size_t)(nseg + 1) + fb * (size_t)seglen * S));
    char *pool = scratch.pool;
    std::vector<int> cur_ck((size_t)nseg);
    char *slots_ck = pool, *slot_fin = pool + sb * (size_t)nseg, *fslots = pool + sb * (size_t)(nseg + 1);
    cudaStream_t s = h->stream;
    const double e[3] = {direction[0], direction[1], direction[2]};
    cudaEvent_t *ev = scratch.ev;
    for (int q = 0; q < 3; ++q) CUDA_OR_FAIL(cudaEventCreate(&ev[q]));
    adjoint_zero(h);
    // forward: K steps, a checkpoint every ck steps, J accumulated on the device
    CUDA_OR_FAIL(cudaEventRecord(ev[0], s));
    for (int n = 0; n < K; ++n) {
        if (n % ck == 0) { slot_save(h, slots_ck + sb * (size_t)(n / ck)); cur_ck[(size_t)(n / ck)] = h->cur; }
        if (n >= last0 && S > 1) {
            stages_with_fields(h, fslots + fb * (size_t)(n - last0) * S, fb);
        } else {
            CUDA_OR_FAIL(cudaGraphLaunch(h->graph[h->cur], s));
            h->cur ^= 1;
            if (n >= last0) fields_save(h, fslots + fb * (size_t)(n - last0));
        }
        enqueue_adjoint_jacc(h->b.sc, a.as, e, s);
    }
    slot_save(h, slot_fin);
    const int cur_fin = h->cur;
    CUDA_OR_FAIL(cudaEventRecord(ev[1], s));
    // reverse sweep: per segment, recompute its steps from the checkpoint
    // keeping each step's fields, then run the adjoint steps backwards
    AdjBufs w = a;
    const double wJ = 1.0 / (double)K;
    for (int sg = nseg - 1; sg >= 0; --sg) {
        const int n0 = sg * ck, n1 = std::min(K, n0 + ck);
        if (sg < nseg - 1) slot_restore(h, slots_ck + sb * (size_t)sg, cur_ck[(size_t)sg]);
        for (int n = n0; n < n1 && sg < nseg - 1; ++n) {
            char *f = fslots + fb * (size_t)(n - n0) * S;
            if (S == 1) {   // AB2: the step graph, then its fields
                CUDA_OR_FAIL(cudaGraphLaunch(h->graph[h->cur], s));
                h->cur ^= 1;
                fields_save(h, f);
            } else {
                stages_with_fields(h, f, fb);
            }
        }
        for (int n = n1 - 1; n >= n0; --n)
            for (int k = S - 1; k >= 0; --k) {   // the objective reads the last stage's drag
                enqueue_adjoint_step(h->gs[k], fields_view(h, fslots + fb * ((size_t)(n - n0) * S + k)), w, e, k == S - 1 ? wJ : 0.0, s);
                std::swap(w.lu, w.lu2);
                std::swap(w.lp, w.lp2);
                std::swap(w.lnl, w.lonl);
            }
    }
    CUDA_OR_FAIL(cudaEventRecord(ev[2], s));
    CUDA_OR_FAIL(cudaGetLastError());
    slot_restore(h, slot_fin, cur_fin);
    Scal sc_fin;
    AdjScal as;
    std::vector<double> gx(3 * (size_t)g.nbody);
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc_fin, h->b.sc, sizeof(Scal), cudaMemcpyDeviceToHost, s));
    CUDA_OR_FAIL(cudaMemcpyAsync(&as, a.as, sizeof(AdjScal), cudaMemcpyDeviceToHost, s));
    CUDA_OR_FAIL(cudaMemcpyAsync(gx.data(), a.gxc, gx.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_OR_FAIL(cudaStreamSynchronize(s));
    float fms = 0.f, rms = 0.f;
    cudaEventElapsedTime(&fms, ev[0], ev[1]);
    cudaEventElapsedTime(&rms, ev[1], ev[2]);
    // the work buffers were swapped K times: keep the handle's set consistent
    a = w;
    if (sc_fin.status) return fail(sc_fin.status, "adjoint: a forward step reported a solver stop condition");
    if (as.status) return fail(as.status, "adjoint: an adjoint kernel reported a bounded-wait timeout or a zero pivot");
    for (size_t q = 0; q < gx.size(); ++q) g_xc[q] = gx[q];
    for (int d = 0; d < 3; ++d) g_mpg[d] = as.gmpg[d];
    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        rep->J = as.J / (double)K;
        rep->forward_ms = fms;
        rep->reverse_ms = rms;
        rep->nsteps = K;
        rep->checkpoint_every = ck;
        rep->adjoint_kernels_per_step = adjoint_kernels_per_step(g);
    }
    return PIBM_OK;
}

int pibm_adjoint_begin(pibm_handle *h, int nsteps, const double direction[3]) {
    if (!h || nsteps < 1 || !direction) return fail(PIBM_ERR_ARG, "bad argument");
    int rc = adjoint_check(h);
    if (rc) return rc;
    if ((rc = pibm_run(h, 0, nullptr))) return rc;   // step graphs
    if ((rc = adjoint_alloc(h))) return rc;
    if (h->itrmax > 1 && !h->adj_fields) {
        size_t CRb, recb;
        const size_t fb = fields_bytes(h, &CRb, &recb);
        if (h->alloc(&h->adj_fields, fb * (size_t)h->itrmax) != cudaSuccess) return fail(PIBM_ERR_NOMEM, "adjoint stage fields");
    }
    adjoint_zero(h);
    for (int d = 0; d < 3; ++d) h->adj_e[d] = direction[d];
    h->adj_wJ = 1.0 / (double)nsteps;
    h->adj_left = nsteps;
    CUDA_OR_FAIL(cudaGetLastError());
    return PIBM_OK;
}

int pibm_adjoint_step(pibm_handle *h) {
    if (!h) return fail(PIBM_ERR_ARG, "null handle");
    if (h->adj_left < 1) return fail(PIBM_ERR_ARG, "pibm_adjoint_step: call pibm_adjoint_begin first (or every step was reversed)");
    if (h->next_rks != 1) return fail(PIBM_ERR_ARG, "pibm_adjoint_step starts at a step boundary");
    AdjBufs &a = h->adj;
    auto swap_state = [&]() {
        std::swap(a.lu, a.lu2);
        std::swap(a.lp, a.lp2);
        std::swap(a.lnl, a.lonl);
    };
    if (h->itrmax == 1) {
        CUDA_OR_FAIL(cudaGraphLaunch(h->graph[h->cur], h->stream));   // step n's fields
        h->cur ^= 1;
        enqueue_adjoint_step(h->g, h->b, a, h->adj_e, h->adj_wJ, h->stream);
        swap_state();
    } else {
        size_t CRb, recb;
        const size_t fb = fields_bytes(h, &CRb, &recb);
        stages_with_fields(h, h->adj_fields, fb);   // the stages of step n, each stage's fields kept
        for (int k = h->itrmax - 1; k >= 0; --k) {
            enqueue_adjoint_step(h->gs[k], fields_view(h, h->adj_fields + fb * (size_t)k), a, h->adj_e,
                                 k == h->itrmax - 1 ? h->adj_wJ : 0.0, h->stream);
            swap_state();
        }
    }
    h->adj_left -= 1;
    CUDA_OR_FAIL(cudaGetLastError());
    return PIBM_OK;
}

int pibm_adjoint_end(pibm_handle *h, double *g_xc, double g_mpg[3]) {
    if (!h || !g_xc || !g_mpg) return fail(PIBM_ERR_ARG, "bad argument");
    if (!h->adj_ready) return fail(PIBM_ERR_ARG, "pibm_adjoint_end without pibm_adjoint_begin");
    const Geo &g = h->g;
    Scal sc;
    AdjScal as;
    std::vector<double> gx(3 * (size_t)g.nbody);
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(Scal), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaMemcpyAsync(&as, h->adj.as, sizeof(AdjScal), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaMemcpyAsync(gx.data(), h->adj.gxc, gx.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    if (sc.status) return fail(sc.status, "adjoint: a recomputed step reported a solver stop condition");
    if (as.status) return fail(as.status, "adjoint: an adjoint kernel reported a bounded-wait timeout or a zero pivot");
    if (h->adj_left != 0) return fail(PIBM_ERR_ARG, "pibm_adjoint_end before every step was reversed");
    for (size_t q = 0; q < gx.size(); ++q) g_xc[q] = gx[q];
    for (int d = 0; d < 3; ++d) g_mpg[d] = as.gmpg[d];
    return PIBM_OK;
}

int pibm_get_tuning(pibm_handle *h, int32_t *lines_per_cta, double lines_ms[2]) {
    if (!h) return fail(PIBM_ERR_ARG, "null handle");
    if (lines_per_cta) *lines_per_cta = h->g.lines_lt;
    if (lines_ms) for (int k = 0; k < 2; ++k) lines_ms[k] = h->lines_ms[k];
    return PIBM_OK;
}

int pibm_set_tuning(pibm_handle *h, int32_t lines_per_cta) {
    if (!h) return fail(PIBM_ERR_ARG, "null handle");
    if (lines_per_cta != kLinesTiles[0] && lines_per_cta != kLinesTiles[1]) return fail(PIBM_ERR_ARG, "x-line tile width must be 4 or 8");
    h->g.lines_lt = lines_per_cta;
    for (int k = 0; k < h->itrmax; ++k) h->gs[k].lines_lt = lines_per_cta;
    drop_graphs(h);
    return PIBM_OK;
}

int pibm_get_contacts(pibm_handle *h, int32_t maxn, int32_t *neigh, int32_t *pn, int32_t *pv) {
    if (!h) return fail(PIBM_ERR_ARG, "null handle");
    if (!h->g.moving) return fail(PIBM_ERR_ARG, "this run has no DEM (IMOVE = 0)");
    const Mov &m = h->b.mov;
    const int N = m.N, MX = m.maxn;
    std::vector<int> nb((size_t)N * MX), nc(N), cn((size_t)N * MX), cv((size_t)N * MX), cc(N);
    CUDA_OR_FAIL(cudaMemcpyAsync(nb.data(), m.neigh, nb.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaMemcpyAsync(nc.data(), m.ncnt, nc.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaMemcpyAsync(cn.data(), m.pn, cn.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaMemcpyAsync(cv.data(), m.pv, cv.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaMemcpyAsync(cc.data(), m.pncnt, cc.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    for (int l = 0; l < N; ++l)
        if (nc[l] + 1 > maxn || cc[l] + 1 > maxn) return fail(PIBM_ERR_ARG, "maxn is smaller than a list");
    for (int l = 0; l < N; ++l) {
        if (neigh) neigh[l] = nc[l];
        if (pn) pn[l] = cc[l];
        if (pv) pv[l] = 1;
        for (int c = 1; c < maxn; ++c) {
            const size_t q = (size_t)l + (size_t)N * c;
            if (neigh) neigh[q] = c - 1 < nc[l] ? nb[(size_t)l * MX + c - 1] + 1 : -1;
            if (pn) pn[q] = c - 1 < cc[l] ? cn[(size_t)l * MX + c - 1] + 1 : -1;
            if (pv) pv[q] = c - 1 < cc[l] ? cv[(size_t)l * MX + c - 1] : 0;
        }
    }
    return PIBM_OK;
}

int pibm_get_scalar(pibm_handle *h, double *phif, double *flux_body, double *ratios) {
    if (!h) return fail(PIBM_ERR_ARG, "null handle");
    if (!h->g.scal) return fail(PIBM_ERR_ARG, "this run has no scalar (ISCALON = 0)");
    const Geo &g = h->g;
    Scal sc;
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    std::vector<double2> dev((size_t)g.nx * g.PS);
    if (phif) CUDA_OR_FAIL(cudaMemcpyAsync(dev.data(), h->b.phif, dev.size() * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    std::vector<double> fb((size_t)g.nbody);
    if (flux_body && g.nbody) CUDA_OR_FAIL(cudaMemcpyAsync(fb.data(), h->b.flux_body, fb.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    if (phif) {
        // reference layout phif(nx+1, my2, mz), x fastest; plane nx+1 = phif(1)/heat_ratio
        const size_t nxf = (size_t)g.nx + 1;
        for (int k = 0; k < g.mz; ++k)
            for (int j = 0; j < g.my2; ++j) {
                const size_t e = (size_t)k * g.my2 + j;
                for (int i = 0; i < g.nx; ++i) {
                    const double2 v = dev[(size_t)i * g.PS + e];
                    phif[2 * (i + nxf * e)] = v.x;
                    phif[2 * (i + nxf * e) + 1] = v.y;
                }
                const double2 v = dev[e];
                phif[2 * (g.nx + nxf * e)] = v.x / sc.heat_ratio;
                phif[2 * (g.nx + nxf * e) + 1] = v.y / sc.heat_ratio;
            }
    }
    if (flux_body) for (int m = 0; m < g.nbody; ++m) flux_body[m] = fb[m];
    if (ratios) { ratios[0] = sc.heat_ratio; ratios[1] = sc.heat_ratio_old; ratios[2] = sc.nusselt; }
    return PIBM_OK;
}

// usmean_des / ufmean_des of a restarted run (read_unformatted reads them from
// the u file, restart_funcs.F90:450-452) instead of the set-up's values.
int pibm_set_desired_means(pibm_handle *h, const double *usmean_des, const double *ufmean_des) {
    if (!h || !usmean_des || !ufmean_des) return fail(PIBM_ERR_ARG, "null argument");
    for (Geo *g : {&h->g, &h->gs[0], &h->gs[1], &h->gs[2]})
        for (int d = 0; d < 3; ++d) { g->usmean_des[d] = usmean_des[d]; g->ufmean_des[d] = ufmean_des[d]; }
    drop_graphs(h);
    return PIBM_OK;
}

// The scalar's nonlinear term of the last step, nlphif(nx+1, my2, mz) in the
// reference layout; plane nx+1 is nlphif(1)/heat_ratio of that step
// (nl_allphi.F90:219), i.e. /heat_ratio_old after the step.
int pibm_get_scalar_nl(pibm_handle *h, double *nlphif) {
    if (!h || !nlphif) return fail(PIBM_ERR_ARG, "null argument");
    if (!h->g.scal) return fail(PIBM_ERR_ARG, "this run has no scalar (ISCALON = 0)");
    const Geo &g = h->g;
    Scal sc;
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    std::vector<double2> dev((size_t)g.nx * g.PS);
    CUDA_OR_FAIL(cudaMemcpyAsync(dev.data(), h->b.nls[h->cur ^ 1], dev.size() * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    const size_t nxf = (size_t)g.nx + 1;
    for (int k = 0; k < g.mz; ++k)
        for (int j = 0; j < g.my2; ++j) {
            const size_t e = (size_t)k * g.my2 + j;
            for (int i = 0; i < g.nx; ++i) {
                const double2 v = dev[(size_t)i * g.PS + e];
                nlphif[2 * (i + nxf * e)] = v.x;
                nlphif[2 * (i + nxf * e) + 1] = v.y;
            }
            nlphif[2 * (g.nx + nxf * e)] = dev[e].x / sc.heat_ratio_old;
            nlphif[2 * (g.nx + nxf * e) + 1] = dev[e].y / sc.heat_ratio_old;
        }
    return PIBM_OK;
}

// Restart of the scalar (read_unformatted, restart_funcs.F90:560-590): phif and
// the last step's nlphif in the reference layout (nx+1, my2, mz), and
// ratios[0..1] = heat_ratio, heat_ratio_old.  The real nonlinear term the next
// step's forcing reads is the c2r of nlphif's nx+1 planes.
int pibm_set_scalar(pibm_handle *h, const double *phif, const double *nlphif, const double *ratios) {
    if (!h || !phif || !nlphif || !ratios) return fail(PIBM_ERR_ARG, "null argument");
    if (!h->g.scal) return fail(PIBM_ERR_ARG, "this run has no scalar (ISCALON = 0)");
    const Geo &g = h->g;
    const int nxf = g.nx + 1;
    const size_t nf = (size_t)nxf * g.PS;
    if (!h->stage) CUDA_OR_FAIL(h->alloc(&h->stage, 3 * nf));
    double2 *fin = h->stage, *dplanes = h->stage + nf;   // reference layout in, device planes out
    const int prev = h->cur ^ 1;
    CUDA_OR_FAIL(cudaMemcpyAsync(fin, phif, nf * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    enqueue_f2d(fin, h->b.phif, g.nx, nxf, g.PS, 1, h->stream);
    CUDA_OR_FAIL(cudaMemcpyAsync(fin, nlphif, nf * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    enqueue_f2d(fin, dplanes, nxf, nxf, g.PS, 1, h->stream);
    CUDA_OR_FAIL(cudaMemcpyAsync(h->b.nls[prev], dplanes, (size_t)g.nx * g.PS * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    enqueue_scalar_c2r(g, dplanes, h->b.nlr[prev], nxf, h->stream);
    CUDA_OR_FAIL(cudaGetLastError());
    Scal sc;
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    sc.heat_ratio = ratios[0];
    sc.heat_ratio_old = ratios[1];
    CUDA_OR_FAIL(cudaMemcpyAsync(h->b.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    return PIBM_OK;
}

// Unit directions of the surface quadrature points (quadgener,
// geom_init.F90:44-242), (nbnd, 3) row-major.
int pibm_get_surface_points(pibm_handle *h, double *bnd) {
    if (!h || !bnd) return fail(PIBM_ERR_ARG, "null argument");
    std::copy(h->S.bnd.begin(), h->S.bnd.end(), bnd);
    return PIBM_OK;
}

// Frame motion of a moving-particle run (frame_vel, frame_pos of global_data;
// updated in velstep, steptheflow.F90:99-103; restart records of
// restart_funcs.F90:253-254, read back in initialize_flo.F90:1891-1898).
int pibm_get_frame(pibm_handle *h, double *frame_vel, double *frame_pos) {
    if (!h) return fail(PIBM_ERR_ARG, "null handle");
    Scal sc;
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    for (int d = 0; d < 3; ++d) {
        if (frame_vel) frame_vel[d] = sc.frame_vel[d];
        if (frame_pos) frame_pos[d] = sc.frame_pos[d];
    }
    return PIBM_OK;
}

int pibm_set_frame(pibm_handle *h, const double *frame_vel, const double *frame_pos) {
    if (!h || !frame_vel || !frame_pos) return fail(PIBM_ERR_ARG, "null argument");
    if (h->next_rks != 1) return fail(PIBM_ERR_ARG, "pibm_set_frame at a step boundary only");
    Scal sc;
    CUDA_OR_FAIL(cudaMemcpyAsync(&sc, h->b.sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    for (int d = 0; d < 3; ++d) { sc.frame_vel[d] = frame_vel[d]; sc.frame_pos[d] = frame_pos[d]; }
    CUDA_OR_FAIL(cudaMemcpyAsync(h->b.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, h->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    return PIBM_OK;
}

int pibm_get_if_rev(pibm_handle *h, uint8_t *if_rev) {
    if (!h || !if_rev) return fail(PIBM_ERR_ARG, "null argument");
    if (h->g.moving) {   // flags of the last step's geometry rebuild
        CUDA_OR_FAIL(cudaMemcpyAsync(if_rev, h->b.mov.revflag, h->S.if_rev.size(), cudaMemcpyDeviceToHost, h->stream));
        CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
        return PIBM_OK;
    }
    std::memcpy(if_rev, h->S.if_rev.data(), h->S.if_rev.size());
    return PIBM_OK;
}

int pibm_get_fluid_mask(pibm_handle *h, uint8_t *mask) {
    if (!h || !mask) return fail(PIBM_ERR_ARG, "null argument");
    const RunSetup &S = h->S;
    if (h->g.moving) {   // the device mask, stored in plane-transform order
        std::vector<uint8_t> dev((size_t)S.nx * h->g.RS);
        CUDA_OR_FAIL(cudaMemcpyAsync(dev.data(), h->g.fluid, dev.size(), cudaMemcpyDeviceToHost, h->stream));
        CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
        for (int i = 0; i < S.nx; ++i)
            for (int k = 0; k < S.mz; ++k)
                for (int j = 0; j < S.my; ++j)
                    mask[(size_t)i + (size_t)S.nx * ((size_t)j + (size_t)S.my * k)] = dev[(size_t)i * h->g.RS + real_offset(S.my, k, j)];
        return PIBM_OK;
    }
    for (int i = 0; i < S.nx; ++i)
        for (int k = 0; k < S.mz; ++k)
            for (int j = 0; j < S.my; ++j)
                mask[(size_t)i + (size_t)S.nx * ((size_t)j + (size_t)S.my * k)] = S.fluid[(size_t)i * S.my * S.mz + (size_t)k * S.my + j];
    return PIBM_OK;
}

void pibm_destroy(pibm_handle *h) { delete h; }

static int plane_transform(int my, int mz, int nplanes, const double *a, double *b, bool forward) {
    if (my != mz || !supported_size(my) || nplanes < 0 || !a || !b) return fail(PIBM_ERR_ARG, "unsupported plane size");
    if (nplanes == 0) return PIBM_OK;
    Geo g;
    std::memset(&g, 0, sizeof(g));
    g.nx = 1; g.my = my; g.mz = mz; g.my2 = my / 2 + 1; g.PS = g.my2 * mz; g.RS = my * mz;
    g.nrm = (double)(float)(my * mz);
    g.plane_ctas = plane_ctas(my);
    CUDA_OR_FAIL(configure_kernels(my));
    std::vector<double2> tw = twiddles(my);
    double2 *dtw = nullptr, *dc = nullptr;
    double *dr = nullptr;
    const size_t nc = (size_t)g.PS * nplanes, nr = (size_t)g.RS * nplanes;
    CUDA_OR_FAIL(cudaMalloc(&dtw, tw.size() * sizeof(double2)));
    CUDA_OR_FAIL(cudaMalloc(&dc, nc * sizeof(double2)));
    CUDA_OR_FAIL(cudaMalloc(&dr, nr * sizeof(double)));
    CUDA_OR_FAIL(cudaMemcpy(dtw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice));
    g.tw = dtw;
    if (forward) {
        CUDA_OR_FAIL(cudaMemcpy(dr, a, nr * sizeof(double), cudaMemcpyHostToDevice));
        enqueue_r2c(g, dr, dc, nplanes, 0);
        CUDA_OR_FAIL(cudaGetLastError());
        CUDA_OR_FAIL(cudaMemcpy(b, dc, nc * sizeof(double2), cudaMemcpyDeviceToHost));
    } else {
        CUDA_OR_FAIL(cudaMemcpy(dc, a, nc * sizeof(double2), cudaMemcpyHostToDevice));
        enqueue_c2r(g, dc, dr, nplanes, 0);
        CUDA_OR_FAIL(cudaGetLastError());
        CUDA_OR_FAIL(cudaMemcpy(b, dr, nr * sizeof(double), cudaMemcpyDeviceToHost));
    }
    cudaFree(dtw); cudaFree(dc); cudaFree(dr);
    return PIBM_OK;
}

int pibm_ff2rc(int my, int mz, int nplanes, const double *a, double *b) { return plane_transform(my, mz, nplanes, a, b, true); }
int pibm_ff2cr(int my, int mz, int nplanes, const double *a, double *b) { return plane_transform(my, mz, nplanes, a, b, false); }

}  // extern "C"

// ---- allocation-free ff2cr: twiddles for every supported size live in one
// static device array, written once per device context by the first call ----
namespace {
constexpr int kNoAllocSizes[4] = {32, 64, 96, 128};
constexpr int kNoAllocMaxN = 128;
constexpr int kNoAllocEntries = 32 + 64 + 96 + 128;
static __device__ __align__(256) double2 g_noalloc_twiddles[kNoAllocEntries];
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double2 *g_noalloc_ptr[kNoAllocMaxDevices] = {};
// unique id of the context whose copy of g_noalloc_twiddles was filled (a
// device reset destroys the context, and the next one starts with a zeroed
// array under a new id, so the table is written again)
unsigned long long g_noalloc_ctx[kNoAllocMaxDevices] = {};

// Offset of the size-n table inside g_noalloc_twiddles, or -1.
int noalloc_offset(int n) {
    int off = 0;
    for (int s : kNoAllocSizes) {
        if (s == n) return off;
        off += s;
    }
    return -1;
}

// Unique id of the current thread's CUDA context (driver cuCtxGetId through
// the runtime's entry-point table; no link-time dependency on libcuda).
cudaError_t current_context_id(unsigned long long *id) {
    typedef int (*get_cur_t)(void **);
    typedef int (*get_id_t)(void *, unsigned long long *);
    static get_cur_t get_cur = nullptr;
    static get_id_t get_id = nullptr;
    if (!get_cur || !get_id) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa);
        if (e != cudaSuccess) return e;
        e = cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb);
        if (e != cudaSuccess) return e;
        if (qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b) return cudaErrorNotSupported;
        get_cur = (get_cur_t)a;
        get_id = (get_id_t)b;
    }
    void *ctx = nullptr;
    if (get_cur(&ctx) != 0 || !ctx) return cudaErrorDeviceUninitialized;
    if (get_id(ctx, id) != 0) return cudaErrorDeviceUninitialized;
    return cudaSuccess;
}
}  // namespace

extern "C" {

int pibm_ff2cr_noalloc(int my, int mz, int nplanes, const double *d_a, double *d_b, void *stream) {
    if (my > kNoAllocMaxN || mz > kNoAllocMaxN)
        return fail(PIBM_ERR_ARG, "pibm_ff2cr_noalloc: plane " + std::to_string(my) + "x" + std::to_string(mz) +
                                      " exceeds the static twiddle table (largest size 128)");
    if (my != mz || noalloc_offset(my) < 0)
        return fail(PIBM_ERR_ARG, "pibm_ff2cr_noalloc: unsupported plane size (my = mz in {32, 64, 96, 128})");
    if (nplanes < 0 || (nplanes > 0 && (!d_a || !d_b))) return fail(PIBM_ERR_ARG, "pibm_ff2cr_noalloc: bad argument");
    int dev = 0;
    CUDA_OR_FAIL(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(PIBM_ERR_ARG, "pibm_ff2cr_noalloc: device index out of range");
    double2 *table = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        // the array's device address in the current context (this call also
        // brings the device's context up if nothing has yet)
        void *p = nullptr;
        CUDA_OR_FAIL(cudaGetSymbolAddress(&p, g_noalloc_twiddles));
        unsigned long long ctx = 0;
        CUDA_OR_FAIL(current_context_id(&ctx));
        if (!g_noalloc_ptr[dev] || g_noalloc_ctx[dev] != ctx) {
            // first call in this device context (it is current): fill every size, wait
            std::vector<double2> host;
            host.reserve(kNoAllocEntries);
            for (int s : kNoAllocSizes) {
                std::vector<double2> t = twiddles(s);
                host.insert(host.end(), t.begin(), t.end());
            }
            CUDA_OR_FAIL(cudaMemcpy(p, host.data(), host.size() * sizeof(double2), cudaMemcpyHostToDevice));
            CUDA_OR_FAIL(cudaDeviceSynchronize());
            g_noalloc_ptr[dev] = (double2 *)p;
            g_noalloc_ctx[dev] = ctx;
        }
        table = g_noalloc_ptr[dev];
    }
    if (nplanes == 0) return PIBM_OK;
    CUDA_OR_FAIL(configure_kernels(my));
    Geo g;
    std::memset(&g, 0, sizeof(g));
    g.nx = 1; g.my = my; g.mz = mz; g.my2 = my / 2 + 1; g.PS = g.my2 * mz; g.RS = my * mz;
    g.nrm = (double)(float)(my * mz);
    g.plane_ctas = plane_ctas(my);
    g.tw = table + noalloc_offset(my);
    enqueue_c2r(g, (const double2 *)d_a, d_b, nplanes, (cudaStream_t)stream);
    CUDA_OR_FAIL(cudaGetLastError());
    return PIBM_OK;
}

// ---- batched independent realizations ----
// All members step together through ONE CUDA graph per step parity.  Members
// with fixed spheres and no scalar are grouped by grid size and scheme; a
// group steps through one launch per kernel with its members along gridDim.z
// (enqueue_batch_step), so a group of small grids fills the GPU the way one
// large grid does.  The groups run one after another; then the other members
// run one step each as branches of the graph (members whose plane kernels
// alone fill the GPU, my >= 128, one after the other in one chain).
struct BatchGroup {
    int n = 0, itrmax = 1;
    std::vector<int> idx;       // the members in the group, in batch order
    BatchShape shape{};
    std::vector<MemberSet> sets;   // the launches' members: [parity][stage]
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

struct pibm_batch {
    std::vector<pibm_handle *> members;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    std::vector<int> base;      // each member's parity when the graphs were captured
    std::vector<unsigned> ver;  // each member's geo_ver when the graphs were captured
    int flip = 0;               // graph[flip] is the next batch step
    bool fused = true;          // the graphs use the fused group launches
    bool captured_fused = true;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    std::vector<BatchGroup> groups;
    std::vector<char> in_group;
    ~pibm_batch() {
        for (auto &gx : graph) if (gx) cudaGraphExecDestroy(gx);
        if (fork) cudaEventDestroy(fork);
        for (auto e : join) cudaEventDestroy(e);
        for (auto &G : groups) {
            for (cudaEvent_t e : {G.fork, G.join}) if (e) cudaEventDestroy(e);
            if (G.side) cudaStreamDestroy(G.side);
        }
        if (stream) cudaStreamDestroy(stream);
        for (auto *h : members) pibm_destroy(h);
    }
};

// Fused groups of a new batch: members with fixed spheres (or none) and no
// scalar, keyed by grid size and stages per step, at most kFuseMax members
// per group; groups of one member stay on the members' own step.
static cudaError_t batch_groups(pibm_batch *bt) {
    const int n = (int)bt->members.size();
    bt->in_group.assign((size_t)n, 0);
    for (int q = 0; q < n; ++q) {
        const pibm_handle *h = bt->members[q];
        if (h->g.moving || h->g.scal) continue;
        BatchGroup *G = nullptr;
        for (auto &x : bt->groups)
            if (x.n == h->g.my && x.itrmax == h->itrmax && (int)x.idx.size() < kFuseMax) G = &x;
        if (!G) { bt->groups.emplace_back(); G = &bt->groups.back(); G->n = h->g.my; G->itrmax = h->itrmax; }
        G->idx.push_back(q);
    }
    std::vector<BatchGroup> keep;
    for (auto &G : bt->groups) if (G.idx.size() > 1) keep.push_back(G);
    bt->groups.swap(keep);
    for (auto &G : bt->groups) {
        for (int q : G.idx) bt->in_group[q] = 1;
        G.sets.resize((size_t)2 * G.itrmax);
        cudaError_t e;
        if ((e = cudaStreamCreateWithFlags(&G.side, cudaStreamNonBlocking)) != cudaSuccess) return e;
        for (cudaEvent_t *ev : {&G.fork, &G.join})
            if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int pibm_batch_create(int n, const pibm_params *prm, const pibm_particles *parts, pibm_batch **out) {
    if (n <= 0 || !prm || !out) return fail(PIBM_ERR_ARG, "bad argument");
    *out = nullptr;
    pibm_batch *bt = new pibm_batch();
    for (int q = 0; q < n; ++q) {
        pibm_handle *h = nullptr;
        int rc = pibm_create(&prm[q], parts ? &parts[q] : nullptr, &h);
        if (rc) { delete bt; return rc; }
        bt->members.push_back(h);
    }
    bt->join.resize((size_t)n, nullptr);
    cudaError_t e = cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&bt->fork, cudaEventDisableTiming);
    for (int q = 0; q < n && e == cudaSuccess; ++q) e = cudaEventCreateWithFlags(&bt->join[q], cudaEventDisableTiming);
    if (e == cudaSuccess) e = batch_groups(bt);
    if (e != cudaSuccess) { delete bt; return fail(PIBM_ERR_CUDA, std::string("batch stream/events: ") + cudaGetErrorString(e)); }
    *out = bt;
    return PIBM_OK;
}

// The members of every group's launches for the members' current parities
// and Geo copies (the graphs take them by value, as kernel parameters).
static void batch_members(pibm_batch *bt) {
    for (auto &G : bt->groups) {
        BatchShape &bs = G.shape;
        bs = BatchShape{(int)G.idx.size(), 0, 0, 0, bt->members[G.idx[0]]->gs[0].lines_lt, bt->members[G.idx[0]]->gs[0].flux_seg};
        for (int par = 0; par < 2; ++par)
            for (int k = 0; k < G.itrmax; ++k) {
                MemberSet &ms = G.sets[(size_t)par * G.itrmax + k];
                std::memset(&ms, 0, sizeof(ms));
                for (size_t z = 0; z < G.idx.size(); ++z) {
                    const int q = G.idx[z];
                    pibm_handle *h = bt->members[q];
                    Member &m = ms.m[z];
                    m.g = h->gs[k];
                    m.b = h->b;
                    m.cur = bt->base[q] ^ par ^ (k & 1);
                    m.nbk = h->g.nbody > 0 ? (h->g.npts + 255) / 256 : 0;
                    bs.max_nbody = std::max(bs.max_nbody, h->g.nbody);
                    bs.max_nbk = std::max(bs.max_nbk, m.nbk);
                    if (h->g.nbody > 0 && h->g.npts > 0) bs.max_spn = std::max(bs.max_spn, h->g.sp_nnodes);
                }
            }
    }
}

// (Re)capture the two batch graphs if any member's parity or Geo no longer
// matches them.
static int batch_graphs(pibm_batch *bt) {
    const int n = (int)bt->members.size();
    bool ok = bt->graph[0] && bt->graph[1] && (int)bt->base.size() == n && bt->captured_fused == bt->fused;
    for (int q = 0; ok && q < n; ++q)
        ok = bt->members[q]->cur == (bt->base[q] ^ bt->flip) && bt->members[q]->geo_ver == bt->ver[q];
    if (ok) return PIBM_OK;
    for (auto &gx : bt->graph) if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
    bt->base.resize((size_t)n);
    bt->ver.resize((size_t)n);
    for (int q = 0; q < n; ++q) { bt->base[q] = bt->members[q]->cur; bt->ver[q] = bt->members[q]->geo_ver; }
    bt->flip = 0;
    bt->captured_fused = bt->fused;
    batch_members(bt);
    for (int par = 0; par < 2; ++par) {
        cudaGraph_t gr;
        CUDA_OR_FAIL(cudaStreamBeginCapture(bt->stream, cudaStreamCaptureModeThreadLocal));
        // the groups one after another (run side by side, their launches
        // compete for SMs and L2 and the step takes longer), then the others
        if (bt->fused)
            for (auto &G : bt->groups)
                for (int k = 0; k < G.itrmax; ++k)
                    enqueue_batch_step(G.n, G.sets[(size_t)par * G.itrmax + k], G.shape, bt->stream, G.side, G.fork,
                                       G.join);
        CUDA_OR_FAIL(cudaEventRecord(bt->fork, bt->stream));
        // members whose plane kernels alone fill the GPU (nx*C CTAs per transform item
        // of at least one per SM slot) form one chain, one after the other; the
        // smaller members run as parallel branches beside that chain
        int prev_big = -1;
        for (int q = 0; q < n; ++q) {
            if (bt->fused && bt->in_group[q]) continue;
            pibm_handle *h = bt->members[q];
            const bool big = h->g.my >= 128;
            CUDA_OR_FAIL(cudaStreamWaitEvent(h->stream, (big && prev_big >= 0) ? bt->join[prev_big] : bt->fork, 0));
            enqueue_time_step(h, bt->base[q] ^ par, h->stream, &h->ss);
            CUDA_OR_FAIL(cudaEventRecord(bt->join[q], h->stream));
            CUDA_OR_FAIL(cudaStreamWaitEvent(bt->stream, bt->join[q], 0));
            if (big) prev_big = q;
        }
        CUDA_OR_FAIL(cudaStreamEndCapture(bt->stream, &gr));
        const cudaError_t e = cudaGraphInstantiate(&bt->graph[par], gr, 0);
        cudaGraphDestroy(gr);
        CUDA_OR_FAIL(e);
    }
    return PIBM_OK;
}

// Enqueue nsteps batch steps on the batch stream (no synchronisation).
static int batch_enqueue(pibm_batch *bt, int nsteps) {
    int rc = batch_graphs(bt);
    if (rc) return rc;
    for (int s = 0; s < nsteps; ++s) {
        CUDA_OR_FAIL(cudaGraphLaunch(bt->graph[bt->flip], bt->stream));
        bt->flip ^= 1;
        for (auto *h : bt->members) h->cur ^= 1;
    }
    return PIBM_OK;
}

// Every member's status after the batch stream has drained.
static int batch_reports(pibm_batch *bt) {
    CUDA_OR_FAIL(cudaStreamSynchronize(bt->stream));
    int rc = PIBM_OK;
    for (auto *h : bt->members) { int r = fill_report(h, nullptr); if (r && !rc) rc = r; }
    return rc;
}

int pibm_batch_run(pibm_batch *bt, int nsteps) {
    if (!bt || nsteps < 0) return fail(PIBM_ERR_ARG, "bad argument");
    int rc = batch_enqueue(bt, nsteps);
    if (rc) return rc;
    return batch_reports(bt);
}

int pibm_batch_time(pibm_batch *bt, int nsteps, int sequential, double *ms) {
    if (!bt || nsteps <= 0 || !ms || sequential < 0 || sequential > 2) return fail(PIBM_ERR_ARG, "bad argument");
    for (auto *h : bt->members)
        if (!h->graph[0] || !h->graph[1]) { int rc = pibm_run(h, 0, nullptr); if (rc) return rc; }
    if (sequential != 1) bt->fused = sequential == 0;
    int rc = batch_graphs(bt);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    CUDA_OR_FAIL(cudaEventCreate(&e0));
    CUDA_OR_FAIL(cudaEventCreate(&e1));
    CUDA_OR_FAIL(cudaStreamSynchronize(bt->stream));
    for (auto *h : bt->members) CUDA_OR_FAIL(cudaStreamSynchronize(h->stream));
    CUDA_OR_FAIL(cudaEventRecord(e0, bt->stream));
    if (sequential) {
        // the plain loop: one realization after another, each on its own graphs
        for (auto *h : bt->members)
            for (int s = 0; s < nsteps; ++s) {
                CUDA_OR_FAIL(cudaGraphLaunch(h->graph[h->cur], bt->stream));
                h->cur ^= 1;
            }
    } else {
        rc = batch_enqueue(bt, nsteps);
        bt->fused = true;
        if (rc) return rc;
    }
    CUDA_OR_FAIL(cudaEventRecord(e1, bt->stream));
    CUDA_OR_FAIL(cudaEventSynchronize(e1));
    float t = 0.f;
    CUDA_OR_FAIL(cudaEventElapsedTime(&t, e0, e1));
    *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return batch_reports(bt);
}

pibm_handle *pibm_batch_member(pibm_batch *bt, int i) {
    if (!bt || i < 0 || i >= (int)bt->members.size()) return nullptr;
    return bt->members[i];
}

void pibm_batch_destroy(pibm_batch *bt) { delete bt; }

}  // extern "C"
