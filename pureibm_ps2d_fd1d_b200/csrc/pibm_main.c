/*
 * pibm_main.c -- a host driver in C for libpibm: the time loop of the
 * reference's driver (SRC/FLO/dtibm_main_scal_flo.F90:393-651) for the
 * 'default' input type, with its per-step rank-0 records.
 *
 *     pibm_main RUN_NAME [MAX_STEPS]
 *
 * reads RUN_NAME_floparam.in (namelists read in read_nmls's order,
 * SRC/FLO/initialize.F90:274-359, unknown variables refused) and
 * RUN_NAME_sphr_center.inp (initialize_flo.F90:1485-1590: the first line is
 * skipped, columns x y z in diameters, scaled by DBYDX), creates the engine,
 * and steps it until t >= TEND or MAX_STEPS time steps (every rks stage of a
 * step through pibm_step, as the reference's DO intstep = 1, itrmax loop),
 * appending after each step
 *     RUN_NAME_norm_drag.dat, RUN_NAME_norm_drag_chem.dat,
 *     RUN_NAME_drag_components.dat   (bcset, boundary_condition.F90:849-870)
 *     RUN_NAME_dt_history.dat        (the driver, dtibm_main_scal_flo.F90:319-322, 460)
 * in the reference's columns and Fortran edit descriptors (2x,e20.12 and
 * 2x,g17.8).  Error returns of the engine stop the run like the reference's
 * STOP, with pibm_last_error() printed.
 *
 *     pibm_main --print-params FILE    parse FILE and print the pibm_params fields
 *     pibm_main --format X...          print each X with e20.12 and g17.8
 * are the library-free modes (no GPU needed).
 *
 * Built by pureibm_ps2d_fd1d_b200/build.py with gcc -ffp-contract=off and
 * linked to libpibm.so; no torch, no Python.
 */
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/pibm.h"

#define SMALL_NUMBER ((double)1.0e-35f)   /* the reference's single-precision literal, widened */
#define LARGE_NUMBER ((double)1.0e32f)

/* ------------------------------------------------------------------------ */
/* Fortran edit descriptors                                                  */
/* ------------------------------------------------------------------------ */
static void rjust(char *out, const char *s, int w) {
    const int n = (int)strlen(s);
    int k = 0;
    for (; k < w - n; ++k) out[k] = ' ';
    strcpy(out + k, s);
}

/* Ew.d: 0.ddd...E+ee (three exponent digits without the E beyond 99). */
static void fmt_e(char *out, double x, int w, int d) {
    char s[96], m[64];
    if (x != x) { rjust(out, "NaN", w); return; }
    if (isinf(x)) { rjust(out, x < 0 ? "-Infinity" : "Infinity", w); return; }
    if (x == 0.0) {
        char z[64];
        int k = 0;
        if (signbit(x)) z[k++] = '-';
        z[k++] = '0'; z[k++] = '.';
        for (int i = 0; i < d; ++i) z[k++] = '0';
        strcpy(z + k, "E+00");
        rjust(out, z, w);
        return;
    }
    snprintf(m, sizeof m, "%.*e", d - 1, fabs(x));
    char *e = strchr(m, 'e');
    const int exp = atoi(e + 1) + 1;
    char digits[64];
    int nd = 0;
    for (char *c = m; c < e; ++c)
        if (*c != '.') digits[nd++] = *c;
    digits[nd] = 0;
    if (exp >= -99 && exp <= 99)
        snprintf(s, sizeof s, "%s0.%sE%c%02d", x < 0 ? "-" : "", digits, exp < 0 ? '-' : '+', abs(exp));
    else
        snprintf(s, sizeof s, "%s0.%s%c%03d", x < 0 ? "-" : "", digits, exp < 0 ? '-' : '+', abs(exp));
    rjust(out, s, w);
}

/* Gw.d: F editing with d significant digits and 4 trailing blanks when
 * 0.1 <= |x| < 10**d after rounding to d digits, else Ew.d. */
static void fmt_g(char *out, double x, int w, int d) {
    const double ax = fabs(x);
    char s[96], t[96];
    if (x == x && !isinf(x) && ax != 0.0) {
        snprintf(t, sizeof t, "%.*e", d - 1, ax);
        const double r = strtod(t, NULL);
        if (0.1 <= r && r < pow(10.0, d)) {
            const int k = (int)floor(log10(r)) + 1;
            snprintf(t, sizeof t, "%s%.*f", x < 0 ? "-" : "", d - k, ax);
            rjust(s, t, w - 4);
            snprintf(out, 96, "%s    ", s);
            return;
        }
    }
    if (ax == 0.0 && x == x) {
        int k = 0;
        t[k++] = '0'; t[k++] = '.';
        for (int i = 0; i < d - 1; ++i) t[k++] = '0';
        t[k] = 0;
        rjust(s, t, w - 4);
        snprintf(out, 96, "%s    ", s);
        return;
    }
    fmt_e(out, x, w, d);
}

static void write_line(FILE *f, const double *v, int n, int g) {
    char b[128];
    for (int i = 0; i < n; ++i) {
        if (g) fmt_g(b, v[i], 17, 8); else fmt_e(b, v[i], 20, 12);
        fprintf(f, "  %s", b);
    }
    fputc('\n', f);
}

/* ------------------------------------------------------------------------ */
/* Namelist input (the groups and variables the reference declares,         */
/* SRC/FLO/global_data.F90:300-336, SRC/SCALAR/scalar_data.F90:89-91)       */
/* ------------------------------------------------------------------------ */
static const char *NML_FLOANDGRID = " mx mxf my mz tstart ramp_frac_steps tend nerr_steps wtime_maxhrs saveforres_time "
    "tol_ferror vis re rhof cpf kf archno cfl cfl_max vfl foffset mbuffer mpg ret flo_ang tol_gran_error ";
static const char *NML_PART_PROPT = " nbody dr f1 f2 tstartmove lybyd dbydx dia_phys rhos cps ks input_type discr_scheme "
    "limiter vol_frac1 min_part_sep nphases collision_type vel_distrib nl_slope_factor ";
static const char *NML_FLAGS = " aliasflag maxzeroflag revernorm imove iscalon irestart iscal_restart saveforrestart "
    "saveforres_time xperiodic adaptive set_umean set_mpg nlcons rk3 mean_vel_to_particles dorpr dobnd "
    "include_frmeanfluid impose_grav debug_check cage_simul fixed_moving gof_avg only_dem movingcv iturbon "
    "moving_from_fixed_bed from_post change_frame use_drag_law initialize_zero ";
static const char *NML_FILES = " outputfile rstsave outformat saveitns minunitno maxunitno errfile rstread write_output "
    "write_snapshot ";
static const char *NML_PSD = " psd_type nphases sigmabydavg phiavg equal_momentum ";
static const char *NML_GCG = " coeff_rest pvel_var min_colisions mis_hs ";
static const char *NML_BIDISPERSE = " volfrac_rat red1 dia_ratio yalpha ";
static const char *NML_LUBTEST = " hbyd ";
static const char *NML_MATINPUT = " hhat mis_mat ibordel matern_treshold ";
static const char *NML_RISER = " volume_fraction widthbyd aspect_ratio ";
static const char *NML_SCAL_PROPT = " nspmx phistream setphimean phisurf sourcepresent lumped_cap pr_or_sc_nu "
    "zero_flow_in_solid dorpr_scal ";
static const char *NML_POSTLIST = " nmis nbins skip_num post_no_flow_mem_alloc rad_factor power sa_max_itr post_error "
    "post_small rad_ratio func_rad_ratio cooling_rate temp_init sa_error objective_coef1 objective_coef2 igeometry "
    "isa sa_in_itr rad_reduction_ratio icohesive nsmall_length lybyd_small cluster_part_min cluster_part_max "
    "rotated include_nmis ";

/* Values the run needs, with the reference's defaults (initialize.F90:73-271). */
typedef struct Input {
    int my, mz, ramp_frac_steps, revernorm, imove, iscalon, aliasflag;
    int adaptive, set_mpg, set_umean, initialize_zero, dorpr, dobnd, include_frmeanfluid, rk3, nlcons, xperiodic;
    double lybyd, dbydx, dia_phys, vis, re, cfl, cfl_max, vfl, dr, f1, f2, rhof, rhos, coeff_rest;
    double flo_ang[3], mpg[3], pr_or_sc_nu, phisurf, phistream, tend;
    int have_dbydx, have_cfl_max, have_tend;
    char discr_scheme[32], limiter[32], collision_type[32], input_type[32], psd_type[32];
} Input;

static void input_defaults(Input *in) {
    memset(in, 0, sizeof *in);
    in->dia_phys = 1.0; in->vis = 0.012; in->re = 100.0; in->cfl = 0.5; in->vfl = 1.0; in->dr = 1.0;
    in->f1 = 1.6; in->f2 = 1.6; in->flo_ang[1] = 90.0; in->flo_ang[2] = 90.0;
    in->rhof = 1.0; in->rhos = 1.0; in->coeff_rest = 1.0; in->ramp_frac_steps = 20;
    in->adaptive = 1; in->dorpr = 1; in->revernorm = 1; in->dobnd = 1; in->nlcons = 1; in->xperiodic = 1;
    in->pr_or_sc_nu = 0.7; in->phisurf = 0.0; in->phistream = 1.0;
    strcpy(in->discr_scheme, "center"); strcpy(in->limiter, "none"); strcpy(in->collision_type, "none");
    strcpy(in->input_type, "default"); strcpy(in->psd_type, "");
}

static void lower(char *s) { for (; *s; ++s) *s = (char)tolower((unsigned char)*s); }

/* Logical value: T, .TRUE., F, .FALSE. (any case); returns -1 if not logical. */
static int logical_of(const char *v) {
    char b[32];
    snprintf(b, sizeof b, "%s", v);
    lower(b);
    const char *p = b[0] == '.' ? b + 1 : b;
    if (p[0] == 't') return 1;
    if (p[0] == 'f') return 0;
    return -1;
}

static double real_of(const char *v) {
    char b[64];
    snprintf(b, sizeof b, "%s", v);
    for (char *c = b; *c; ++c) if (*c == 'd' || *c == 'D') *c = 'e';
    return strtod(b, NULL);
}

static int err_input(const char *path, const char *what, const char *name) {
    fprintf(stderr, "%s: %s %s\n", path, what, name);
    return -1;
}

static void copy_lower(char *dst, size_t cap, const char *v) {
    size_t k = 0;
    for (; v[k] && k + 1 < cap; ++k) dst[k] = (char)tolower((unsigned char)v[k]);
    dst[k] = 0;
}

/* Assign one value (element idx >= 1 of an array variable, or idx = 0). */
static void assign(Input *in, const char *key, int idx, const char *v) {
#define R(name) if (!strcmp(key, #name)) { in->name = real_of(v); return; }
#define I(name) if (!strcmp(key, #name)) { in->name = (int)real_of(v); return; }
#define L(name) if (!strcmp(key, #name)) { in->name = logical_of(v) == 1; return; }
#define S(name) if (!strcmp(key, #name)) { copy_lower(in->name, sizeof in->name, v); return; }
    I(my) I(mz) I(ramp_frac_steps) I(revernorm) I(imove) I(iscalon) I(aliasflag)
    L(adaptive) L(set_mpg) L(set_umean) L(initialize_zero) L(dorpr) L(dobnd) L(include_frmeanfluid) L(rk3)
    L(nlcons) L(xperiodic)
    R(lybyd) R(dia_phys) R(vis) R(re) R(cfl) R(vfl) R(dr) R(f1) R(f2) R(rhof) R(rhos) R(coeff_rest)
    R(pr_or_sc_nu) R(phisurf) R(phistream)
    S(discr_scheme) S(limiter) S(collision_type) S(input_type) S(psd_type)
#undef R
#undef I
#undef L
#undef S
    if (!strcmp(key, "dbydx")) { in->dbydx = real_of(v); in->have_dbydx = 1; return; }
    if (!strcmp(key, "cfl_max")) { in->cfl_max = real_of(v); in->have_cfl_max = 1; return; }
    if (!strcmp(key, "tend")) { in->tend = real_of(v); in->have_tend = 1; return; }
    if (!strcmp(key, "flo_ang") && idx >= 1 && idx <= 3) { in->flo_ang[idx - 1] = real_of(v); return; }
    if (!strcmp(key, "mpg") && idx >= 1 && idx <= 3) { in->mpg[idx - 1] = real_of(v); return; }
}

/* Read one token of a group body: a quoted string or a run of characters
 * other than blanks, commas, '=' and '/'.  Returns its end or NULL. */
static const char *token(const char *p, const char *end, char *out, int cap) {
    int n = 0;
    if (p < end && (*p == '\'' || *p == '"')) {
        const char q = *p++;
        while (p < end && *p != q) { if (n < cap - 1) out[n++] = *p; ++p; }
        if (p < end) ++p;
    } else {
        while (p < end && !isspace((unsigned char)*p) && *p != ',' && *p != '=' && *p != '/' && *p != '(') {
            if (n < cap - 1) out[n++] = *p;
            ++p;
        }
    }
    out[n] = 0;
    return p;
}

static const char *skip_sep(const char *p, const char *end) {
    while (p < end && (isspace((unsigned char)*p) || *p == ',')) ++p;
    return p;
}

/* Is "NAME [(i)] =" at p (the start of the next assignment)? */
static int at_assignment(const char *p, const char *end) {
    if (p >= end || !(isalpha((unsigned char)*p) || *p == '_')) return 0;
    while (p < end && (isalnum((unsigned char)*p) || *p == '_')) ++p;
    while (p < end && isspace((unsigned char)*p)) ++p;
    if (p < end && *p == '(') {
        while (p < end && *p != ')') ++p;
        if (p < end) ++p;
        while (p < end && isspace((unsigned char)*p)) ++p;
    }
    return p < end && *p == '=';
}

/* Parse the body [p, end) of group `group` whose variables are `decl`. */
static int parse_group(Input *in, const char *path, const char *group, const char *decl, const char *p, const char *end) {
    char key[64], val[256], probe[72];
    for (;;) {
        p = skip_sep(p, end);
        if (p >= end) return 0;
        int idx = 0;
        p = token(p, end, key, sizeof key);
        lower(key);
        if (!key[0]) return err_input(path, "cannot read an assignment in group", group);
        snprintf(probe, sizeof probe, " %s ", key);
        if (!strstr(decl, probe)) {
            fprintf(stderr, "%s: &%s has no variable %s\n", path, group, key);
            return -1;
        }
        while (p < end && isspace((unsigned char)*p)) ++p;
        if (p < end && *p == '(') { idx = atoi(p + 1); while (p < end && *p != ')') ++p; if (p < end) ++p; }
        while (p < end && isspace((unsigned char)*p)) ++p;
        if (p >= end || *p != '=') return err_input(path, "missing '=' after", key);
        ++p;
        int k = idx ? idx : 1;
        for (;;) {
            p = skip_sep(p, end);
            if (p >= end || at_assignment(p, end)) break;
            p = token(p, end, val, sizeof val);
            if (!val[0]) { ++p; continue; }
            int rep = 1;
            char *star = strchr(val, '*');
            const char *v = val;
            if (star && star != val && isdigit((unsigned char)val[0])) { *star = 0; rep = atoi(val); v = star + 1; }
            for (int r = 0; r < rep; ++r, ++k) assign(in, key, (idx || k > 1 || !strcmp(key, "flo_ang") || !strcmp(key, "mpg")) ? k : 0, v);
        }
    }
}

/* Find group `name` at or after *pos (gfortran skips other groups on the way). */
static int find_group(const char *text, size_t *pos, const char *name, const char **body, const char **bend) {
    const size_t n = strlen(text), ln = strlen(name);
    for (size_t i = *pos; i < n; ++i) {
        if (text[i] != '&' && text[i] != '$') continue;
        if (strncasecmp(text + i + 1, name, ln) != 0) continue;
        const char c = text[i + 1 + ln];
        if (isalnum((unsigned char)c) || c == '_') continue;
        const char *b = text + i + 1 + ln, *e = b;
        /* the group ends at a '/' outside quotes */
        char q = 0;
        for (; *e; ++e) {
            if (q) { if (*e == q) q = 0; continue; }
            if (*e == '\'' || *e == '"') { q = *e; continue; }
            if (*e == '/') break;
        }
        if (!*e) return 0;
        *body = b; *bend = e;
        *pos = (size_t)(e - text) + 1;
        return 1;
    }
    return 0;
}

static int read_floparam(const char *path, Input *in) {
    FILE *f = fopen(path, "rb");
    if (!f) { fprintf(stderr, "%s: cannot open\n", path); return -1; }
    fseek(f, 0, SEEK_END);
    const long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *text = (char *)malloc((size_t)n + 1);
    if (!text || fread(text, 1, (size_t)n, f) != (size_t)n) { fclose(f); free(text); return -1; }
    fclose(f);
    text[n] = 0;
    /* '!' starts a comment outside quotes */
    char q = 0;
    for (long i = 0; i < n; ++i) {
        if (q) { if (text[i] == q) q = 0; continue; }
        if (text[i] == '\'' || text[i] == '"') { q = text[i]; continue; }
        if (text[i] == '!') while (i < n && text[i] != '\n') text[i++] = ' ';
    }
    input_defaults(in);
    struct { const char *name, *decl; } order[12];
    int no = 0;
    order[no].name = "floandgrid"; order[no++].decl = NML_FLOANDGRID;
    order[no].name = "part_propt"; order[no++].decl = NML_PART_PROPT;
    order[no].name = "flags"; order[no++].decl = NML_FLAGS;
    order[no].name = "files"; order[no++].decl = NML_FILES;
    order[no].name = "psd"; order[no++].decl = NML_PSD;
    order[no].name = "gcg"; order[no++].decl = NML_GCG;
    size_t pos = 0;
    int rc = 0;
    for (int g = 0; g < 12 && rc == 0; ++g) {
        if (g == no) {
            /* groups after GCG depend on values read so far (initialize.F90:295-328) */
            if (g != 6) break;
            if (!strcmp(in->input_type, "lubtest")) { order[no].name = "lubtest"; order[no++].decl = NML_LUBTEST;
                                                      order[no].name = "bidisperse"; order[no++].decl = NML_BIDISPERSE; }
            if (!strcmp(in->input_type, "random") && !strcmp(in->psd_type, "bidisp")) { order[no].name = "bidisperse"; order[no++].decl = NML_BIDISPERSE; }
            if (!strcmp(in->input_type, "mat")) { order[no].name = "matinput"; order[no++].decl = NML_MATINPUT; }
            if (!strcmp(in->input_type, "risers")) { order[no].name = "riser"; order[no++].decl = NML_RISER; }
            if (in->iscalon == 1) { order[no].name = "scal_propt"; order[no++].decl = NML_SCAL_PROPT; }
            order[no].name = "postlist"; order[no++].decl = NML_POSTLIST;
        }
        const char *b, *e;
        if (!find_group(text, &pos, order[g].name, &b, &e)) {
            fprintf(stderr, "%s: namelist group &%s is missing or out of read_nmls's order\n", path, order[g].name);
            rc = -1;
            break;
        }
        rc = parse_group(in, path, order[g].name, order[g].decl, b, e);
    }
    free(text);
    if (rc) return rc;
    if (in->set_umean) in->set_mpg = 1;
    return 0;
}

static int make_params(const Input *in, pibm_params *p) {
    memset(p, 0, sizeof *p);
    p->my = in->my;
    p->mz = in->mz ? in->mz : in->my;
    p->lybyd = in->lybyd;
    p->dbydx = in->have_dbydx ? in->dbydx : in->my / in->lybyd;
    p->dia_phys = in->dia_phys;
    p->vis = in->vis; p->re = in->re; p->cfl = in->cfl;
    p->cfl_max = in->have_cfl_max ? in->cfl_max : in->cfl;
    p->vfl = in->vfl; p->dr = in->dr; p->f1 = in->f1; p->f2 = in->f2;
    for (int d = 0; d < 3; ++d) { p->flo_ang[d] = in->flo_ang[d]; p->mpg[d] = in->mpg[d]; }
    p->rhof = in->rhof; p->rhos = in->rhos; p->coeff_rest = in->coeff_rest;
    p->ramp_frac_steps = in->ramp_frac_steps;
    if (!strcmp(in->discr_scheme, "upwind")) p->discr_scheme = PIBM_SCHEME_UPWIND;
    else if (!strcmp(in->discr_scheme, "center")) p->discr_scheme = PIBM_SCHEME_CENTER;
    else { fprintf(stderr, "DISCR_SCHEME must be 'center' or 'upwind'\n"); return -1; }
    p->limiter = !strcmp(in->limiter, "minmod") ? PIBM_LIMITER_MINMOD : PIBM_LIMITER_NONE;
    p->adaptive = in->adaptive; p->set_mpg = in->set_mpg; p->initialize_zero = in->initialize_zero;
    p->dorpr = in->dorpr; p->revernorm = in->revernorm; p->include_frmeanfluid = in->include_frmeanfluid;
    p->imove = in->imove;
    if (strcmp(in->collision_type, "none") && strcmp(in->collision_type, "softsphere") && strcmp(in->collision_type, "eventdriven")) {
        fprintf(stderr, "COLLISION_TYPE = '%s' is not a reference collision model\n", in->collision_type);
        return -1;
    }
    if (in->imove == 1 && !strcmp(in->collision_type, "eventdriven")) {
        fprintf(stderr, "COLLISION_TYPE = 'eventdriven' is not supported (soft-sphere DEM or 'none')\n");
        return -1;
    }
    p->collision_softsphere = !strcmp(in->collision_type, "softsphere");
    p->iscalon = in->iscalon;
    p->pr_or_sc_nu = in->pr_or_sc_nu; p->phisurf = in->phisurf; p->phistream = in->phistream;
    p->rk3 = in->rk3;
    p->dobnd = in->dobnd; p->aliasflag = in->aliasflag; p->nlcons_false = !in->nlcons;
    if (!in->xperiodic) { fprintf(stderr, "XPERIODIC=F is not supported (x-periodic only)\n"); return -1; }
    if (strcmp(in->input_type, "default")) {
        fprintf(stderr, "INPUT_TYPE = '%s': this driver reads particle lists (INPUT_TYPE = 'default')\n", in->input_type);
        return -1;
    }
    return 0;
}

/* Sphere centres from a sphr_center.inp: (nbody,3) column-major, grid units. */
static int read_sphr_center(const char *path, double dbydx, double **xc, int *nbody) {
    FILE *f = fopen(path, "r");
    if (!f) { fprintf(stderr, "%s: cannot open\n", path); return -1; }
    char line[1024];
    int cap = 64, n = 0;
    double *rows = (double *)malloc(sizeof(double) * 3 * cap);
    if (!fgets(line, sizeof line, f)) { fclose(f); *nbody = 0; *xc = rows; return 0; }
    while (fgets(line, sizeof line, f)) {
        char a[3][64];
        if (sscanf(line, "%63s %63s %63s", a[0], a[1], a[2]) != 3) continue;
        if (n == cap) { cap *= 2; rows = (double *)realloc(rows, sizeof(double) * 3 * cap); }
        for (int d = 0; d < 3; ++d) rows[3 * n + d] = real_of(a[d]);
        ++n;
    }
    fclose(f);
    double *out = (double *)malloc(sizeof(double) * 3 * (n ? n : 1));
    for (int m = 0; m < n; ++m)
        for (int d = 0; d < 3; ++d) out[m + (size_t)n * d] = rows[3 * m + d] * dbydx;
    free(rows);
    *xc = out;
    *nbody = n;
    return 0;
}

static void print_params(const pibm_params *p) {
    printf("my %d\nmz %d\n", p->my, p->mz);
    printf("lybyd %.17g\ndbydx %.17g\ndia_phys %.17g\nvis %.17g\nre %.17g\ncfl %.17g\ncfl_max %.17g\nvfl %.17g\n",
           p->lybyd, p->dbydx, p->dia_phys, p->vis, p->re, p->cfl, p->cfl_max, p->vfl);
    printf("dr %.17g\nf1 %.17g\nf2 %.17g\n", p->dr, p->f1, p->f2);
    for (int d = 0; d < 3; ++d) printf("flo_ang%d %.17g\n", d, p->flo_ang[d]);
    for (int d = 0; d < 3; ++d) printf("mpg%d %.17g\n", d, p->mpg[d]);
    printf("rhof %.17g\nrhos %.17g\ncoeff_rest %.17g\n", p->rhof, p->rhos, p->coeff_rest);
    printf("ramp_frac_steps %d\ndiscr_scheme %d\nlimiter %d\nadaptive %d\nset_mpg %d\ninitialize_zero %d\n",
           p->ramp_frac_steps, p->discr_scheme, p->limiter, p->adaptive, p->set_mpg, p->initialize_zero);
    printf("dorpr %d\nrevernorm %d\ninclude_frmeanfluid %d\nimove %d\ncollision_softsphere %d\niscalon %d\n",
           p->dorpr, p->revernorm, p->include_frmeanfluid, p->imove, p->collision_softsphere, p->iscalon);
    printf("pr_or_sc_nu %.17g\nphisurf %.17g\nphistream %.17g\nrk3 %d\n", p->pr_or_sc_nu, p->phisurf, p->phistream, p->rk3);
    printf("dobnd %d\naliasflag %d\nnlcons_false %d\n", p->dobnd, p->aliasflag, p->nlcons_false);
}

/* ------------------------------------------------------------------------ */
/* The time loop                                                             */
/* ------------------------------------------------------------------------ */
static FILE *open_record(const char *run, const char *name, const char *mode) {
    char path[1024];
    snprintf(path, sizeof path, "%s_%s.dat", run, name);
    FILE *f = fopen(path, mode);
    if (!f) fprintf(stderr, "%s: cannot open\n", path);
    return f;
}

static int stop(const char *what, int rc) {
    fprintf(stderr, "%s failed (%d): %s\n", what, rc, pibm_last_error());
    return 1;
}

int main(int argc, char **argv) {
    if (argc >= 3 && !strcmp(argv[1], "--print-params")) {
        Input in;
        pibm_params p;
        if (read_floparam(argv[2], &in) || make_params(&in, &p)) return 2;
        print_params(&p);
        printf("tend %.17g\n", in.have_tend ? in.tend : -1.0);
        return 0;
    }
    if (argc >= 2 && !strcmp(argv[1], "--format")) {
        char b[128];
        for (int i = 2; i < argc; ++i) {
            const double x = strtod(argv[i], NULL);
            fmt_e(b, x, 20, 12);
            printf("%s|", b);
            fmt_g(b, x, 17, 8);
            printf("%s|\n", b);
        }
        return 0;
    }
    if (argc < 2) {
        fprintf(stderr, "usage: %s RUN_NAME [MAX_STEPS]\n", argv[0]);
        return 2;
    }
    const char *run = argv[1];
    const long max_steps = argc >= 3 ? atol(argv[2]) : -1;
    char path[1024];
    Input in;
    pibm_params prm;
    snprintf(path, sizeof path, "%s_floparam.in", run);
    if (read_floparam(path, &in) || make_params(&in, &prm)) return 2;
    double *xc = NULL;
    int nbody = 0;
    snprintf(path, sizeof path, "%s_sphr_center.inp", run);
    if (read_sphr_center(path, prm.dbydx, &xc, &nbody)) return 2;

    pibm_particles parts = {nbody, nbody ? xc : NULL, NULL};
    pibm_handle *h = NULL;
    int rc = pibm_create(&prm, &parts, &h);
    if (rc) return stop("pibm_create", rc);
    pibm_info info;
    if ((rc = pibm_info_get(h, &info))) return stop("pibm_info_get", rc);

    /* initflo constants (initialize_flo.F90:277-283, 550-627; scalar_init.F90:79) */
    const int itrmax = prm.rk3 ? 3 : 1;
    const double uchar0 = (prm.re * prm.vis) / prm.dia_phys;
    double uchar[3];
    for (int d = 0; d < 3; ++d) uchar[d] = uchar0 * cos(M_PI * prm.flo_ang[d] / 180.0);
    const double ucharmod = sqrt(((0.0 + uchar[0] * uchar[0]) + uchar[1] * uchar[1]) + uchar[2] * uchar[2]);
    const double char_length = prm.dia_phys, mvf = info.maxvolfrac;
    const double umeanslip = ucharmod / (1.0 - mvf);
    const double t_conv = char_length / (umeanslip * (1.0 - mvf));
    const double t_vis = (char_length * char_length) / prm.vis;
    const double t_diff = prm.iscalon ? (char_length * char_length) / (prm.vis / prm.pr_or_sc_nu) : LARGE_NUMBER;
    const double d1 = prm.lybyd * prm.dia_phys, dx = d1 / prm.my;
    const double voldom = ((prm.my * dx) * d1) * d1;
    const double c12 = itrmax == 3 ? (1.0 / 6.0 + 1.0 / 6.0) : (0.5 + 0.5);

    FILE *fnd = open_record(run, "norm_drag", "w"), *fch = open_record(run, "norm_drag_chem", "w");
    FILE *fdc = open_record(run, "drag_components", "w"), *fdt = open_record(run, "dt_history", "w");
    if (!fnd || !fch || !fdc || !fdt) return 2;
    {
        const char *hd[4] = {"ISTEP", "DT", "#STEPS REQD", "CFL"};
        char b[32];
        for (int i = 0; i < 4; ++i) { rjust(b, hd[i], 17); fprintf(fdt, "  %s", b); }
        fputc('\n', fdt);
    }
    double *pres = (double *)calloc(3 * (size_t)(nbody ? nbody : 1), sizeof(double));
    double *visc = (double *)calloc(3 * (size_t)(nbody ? nbody : 1), sizeof(double));
    double *vel = (double *)calloc(3 * (size_t)(nbody ? nbody : 1), sizeof(double));
    long istep = 0;
    pibm_step_report rep;
    memset(&rep, 0, sizeof rep);
    for (;;) {
        if (max_steps >= 0 && istep >= max_steps) break;
        if (in.have_tend && istep > 0 && rep.t >= in.tend) break;
        for (int rks = 1; rks <= itrmax; ++rks)
            if ((rc = pibm_step(h, rks, &rep))) return stop("pibm_step", rc);
        ++istep;
        /* bcset records (boundary_condition.F90:849-870), last stage of the step */
        const double t = rep.t, dt = rep.dt, nd = rep.norm_drag;
        double usact[3] = {0.0, 0.0, 0.0}, nd_chem = 0.0;
        if (nbody) {
            if ((rc = pibm_get_particles(h, pres, visc, NULL, NULL, vel))) return stop("pibm_get_particles", rc);
            double avg[3];
            for (int d = 0; d < 3; ++d) {
                double acc = 0.0, ac = 0.0;
                for (int m = 0; m < nbody; ++m) {
                    acc = acc + vel[m + (size_t)nbody * d];
                    ac = ac + c12 * (pres[m + (size_t)nbody * d] + visc[m + (size_t)nbody * d]);
                }
                usact[d] = acc / nbody;
                avg[d] = ac / nbody;
            }
            nd_chem = sqrt((pow(avg[0], 2.0) + pow(avg[1], 2.0)) + pow(avg[2], 2.0));
            const double slip = prm.set_mpg ? (rep.mixmeanslipmod + SMALL_NUMBER) : ucharmod;
            const double nf = (((3.0 * M_PI) * prm.vis) * slip) * char_length;
            nd_chem = nd_chem / nf;
        }
        double v[11];
        v[0] = t / t_conv / (1.0 - mvf); v[1] = t / t_vis; v[2] = t / t_diff;
        v[3] = nd; v[4] = nd;
        for (int d = 0; d < 3; ++d) { v[5 + d] = usact[d]; v[8 + d] = rep.ufmean[d] / ucharmod; }
        write_line(fnd, v, 11, 0);
        v[3] = nd_chem; v[4] = nd_chem;
        write_line(fch, v, 5, 0);
        const double norm_factor = ((((3.0 * M_PI) * prm.vis) * (rep.mixmeanslipmod + SMALL_NUMBER)) * char_length) * nbody;
        const double mpg_avg = sqrt((rep.mpg[0] * rep.mpg[0] + rep.mpg[1] * rep.mpg[1]) + rep.mpg[2] * rep.mpg[2]);
        const double tdm = norm_factor > 0 ? (mpg_avg * voldom) / norm_factor : 0.0;
        const double td = rep.total_drag;
        double w[6] = {rep.pres_drag, rep.visc_drag, td, tdm, nd, fabs(td - tdm) / (td + SMALL_NUMBER)};
        write_line(fdc, w, 6, 0);
        /* driver record (dtibm_main_scal_flo.F90:460) */
        const double tend = in.have_tend ? in.tend : t;
        double g[4] = {(double)istep, dt, (tend - t) / dt + (double)istep, uchar[0] * dt / dx};
        write_line(fdt, g, 4, 1);
        fflush(fnd); fflush(fch); fflush(fdc); fflush(fdt);
    }
    fclose(fnd); fclose(fch); fclose(fdc); fclose(fdt);
    printf("%ld steps, t = %.10g, dt = %.10g, norm_drag = %.10g\n", istep, rep.t, rep.dt, rep.norm_drag);
    free(pres); free(visc); free(vel); free(xc);
    pibm_destroy(h);
    return 0;
}
