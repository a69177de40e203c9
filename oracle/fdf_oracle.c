/*
 * CPU oracle for the fdfault time-stepping path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of edaub/fdfault's single-process solver path: input
 * parsing of the .in sections the path needs, transfinite grid and SBP
 * metrics, outer-boundary and interface normals, friction parameters, the
 * time step, and the per-stage update domain::do_rk_stage
 * (src/domain.cpp:228-305) with everything it calls.  Each function names the
 * reference lines it restates.  Arithmetic is written in the reference's
 * operation order (left-to-right products, same parenthesisation, same
 * accumulation order per node), and this file is compiled without FP
 * contraction, so results are bit-identical to the reference compiled the
 * same way (tests/test_oracle_golden.py pins this against fixtures written by oracle/_ref).
 *
 * Scope: ndim 2 (mode II and mode III) and 3; sbporder 2, 3, 4; RK orders
 * 1-4; elastic and plastic material; outer boundaries none / absorbing /
 * free / rigid; interfaces locked / frictionless / slipweak / stz; load,
 * parameter and state files; heterogeneous initial stress; artificial
 * dissipation; surfaces from files.  Heterogeneous material files are not
 * supported (orc_load reports an error).  No MPI: one process owns the whole
 * grid, so there are no ghost cells.
 */
#include "fdf_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXB 64
#define MAXI 32
#define MAXP 64
#define PATHLEN 1024

typedef struct {
    int type; /* 0 constant, 1 gaussian, 2 ellipse, 3 linear, 4 boxcar */
    double t0, x0, dx, y0, dy;
    double a, b, c, d;
    double val[9];
} pert_t;

typedef struct {
    int active;
    int location;
    double r, alpha, theta, cp, cs, zp, zs, gamma;
    int mlb[3], prb[3];
    int n0, n1;
    double *nx[3];
    double *dl;
} bound_t;

typedef struct {
    int coords[3], nx[3], xm[3];
    int mlb[3], mc[3], mrb[3], prb[3];
    double dx[3], xb[3], lb[3];
    double rho, lam, g, mu, coh, beta, eta;
    char btype[6][64];
    char bfile[6][PATHLEN];
    bound_t bound[6];
} block_t;

typedef struct {
    int kind; /* 0 locked, 1 frictionless, 2 slipweak, 3 stz */
    int direction;
    int b1, b2; /* flat block indices */
    int n[2];
    int xm[3], xp[3];
    int mlb[3], prb[3], delta[3];
    double cp1, cs1, zp1, zs1, cp2, cs2, zp2, zs2, gamma1, gamma2;
    double xb[3], lb[3];
    double *nx[3], *dl1, *dl2;
    int is_friction, has_state;
    double *u, *du, *v, *s, *sn, *ux, *dux, *vx, *sx, *state, *dstate, *dstatedt;
    int nloads;
    pert_t loads[MAXP];
    int load_file;
    double *s1, *s2, *s3;
    int nperts;
    pert_t perts[MAXP];
    int param_file;
    double *par[9];
    double *tfront;
} iface_t;

struct orc_problem {
    char infile[PATHLEN];
    char name[256], datadir[PATHLEN];
    int nt;
    double dt, ttot, cfl;
    int ninfo, rkorder;
    int ndim, mode, nx[3], nblocks[3];
    int *nx_block[3], *xm_block[3];
    int nifaces;
    char iftype[MAXI][64];
    int sbporder;
    char material[64];
    int is_plastic;
    double s0[6];
    char loadfile[PATHLEN], matfile[PATHLEN];
    int plastic_tensor;
    int nfields, nfieldsp, nv, ns, index[6];
    int nxyz, nxd[3];
    double *f, *df, *x, *metric, *jac, *s;
    int hetstress;
    int hetmat;   /* material file: rho, lambda, G per node (fields.cpp:582-711) */
    double *mat;
    double cdiss;
    int dissipation;
    block_t *blocks;
    int nbt;
    iface_t ifaces[MAXI];
    double fdc[12][16], dsc[12][16], h0;
    int nstages;
    double A[5], B[5], C[6];
    int front_on, front_field;
    double front_value;
    char err[2048];
};

/* ------------------------------------------------------------------------- */
/* input reading: sectioned text, values read token by token like operator>> */

typedef struct {
    FILE *fp;
    int ok;
} rd_t;

static int line_is(const char *line, const char *hdr) {
    size_t n = strlen(line);
    while (n > 0 && (line[n - 1] == '\n')) n--;
    return n == strlen(hdr) && strncmp(line, hdr, n) == 0;
}

/* open infile, scan past `first` (if given) then to the line equal to `hdr` */
static int rd_open(rd_t *r, const char *infile, const char *first, const char *hdr) {
    char line[4096];
    r->ok = 0;
    r->fp = fopen(infile, "r");
    if (!r->fp) return 0;
    if (first) {
        int found = 0;
        while (fgets(line, sizeof line, r->fp)) {
            if (line_is(line, first)) {
                found = 1;
                break;
            }
        }
        if (!found) {
            fclose(r->fp);
            r->fp = NULL;
            return 0;
        }
    }
    while (fgets(line, sizeof line, r->fp)) {
        if (line_is(line, hdr)) {
            r->ok = 1;
            return 1;
        }
    }
    fclose(r->fp);
    r->fp = NULL;
    return 0;
}

static void rd_close(rd_t *r) {
    if (r->fp) fclose(r->fp);
    r->fp = NULL;
}

static void rd_str(rd_t *r, char *buf, int n) {
    char fmt[16];
    snprintf(fmt, sizeof fmt, "%%%ds", n - 1);
    if (fscanf(r->fp, fmt, buf) != 1) {
        buf[0] = 0;
        r->ok = 0;
    }
}

static double rd_dbl(rd_t *r) {
    char buf[256];
    rd_str(r, buf, sizeof buf);
    return strtod(buf, NULL);
}

static int rd_int(rd_t *r) {
    char buf[256];
    rd_str(r, buf, sizeof buf);
    return (int)strtol(buf, NULL, 10);
}

static int read_doubles(const char *path, double *dst, long n, long offset) {
    FILE *fp = fopen(path, "rb");
    if (!fp) return 0;
    if (fseek(fp, offset * (long)sizeof(double), SEEK_SET) != 0) {
        fclose(fp);
        return 0;
    }
    size_t got = fread(dst, sizeof(double), (size_t)n, fp);
    fclose(fp);
    return got == (size_t)n;
}

static double *zalloc(long n) {
    double *p = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    return p;
}

/* ------------------------------------------------------------------------- */
/* SBP coefficients: src/fd.cpp:33-155 (same rational and decimal constants) */

static void set_fd(orc_problem *p) {
    int s = p->sbporder;
    memset(p->fdc, 0, sizeof p->fdc);
    memset(p->dsc, 0, sizeof p->dsc);
    double(*c)[16] = p->fdc;
    double(*d)[16] = p->dsc;
    if (s == 2) {
        c[0][0] = -0.5; c[0][1] = 0.; c[0][2] = 0.5;
        d[0][0] = 0.5; d[0][1] = -1.; d[0][2] = 0.5;
        c[1][0] = -1.; c[1][1] = 1.; c[1][2] = 0.;
        c[2][0] = -0.5; c[2][1] = 0.; c[2][2] = 0.5;
        d[1][0] = -1.; d[1][1] = 1.; d[1][2] = 0.;
        d[2][0] = 0.5; d[2][1] = -1.; d[2][2] = 0.5;
        p->h0 = 0.5;
    } else if (s == 3) {
        c[0][0] = 1. / 12.; c[0][1] = -2. / 3.; c[0][2] = 0.; c[0][3] = 2. / 3.; c[0][4] = -1. / 12.;
        d[0][0] = -1. / 12.; d[0][1] = 1. / 3.; d[0][2] = -1. / 2.; d[0][3] = 1. / 3.; d[0][4] = -1. / 12.;
        c[1][0] = -24. / 17.; c[1][1] = 59. / 34.; c[1][2] = -4. / 17.; c[1][3] = -3. / 34.;
        c[2][0] = -0.5; c[2][1] = 0.; c[2][2] = 0.5;
        c[3][0] = 4. / 43.; c[3][1] = -59. / 86.; c[3][2] = 0.; c[3][3] = 59. / 86.; c[3][4] = -4. / 43.;
        c[4][0] = 3. / 98.; c[4][1] = 0.; c[4][2] = -59. / 98.; c[4][3] = 0.; c[4][4] = 32. / 49.; c[4][5] = -4. / 49.;
        d[1][0] = -8. / 17.; d[1][1] = 16. / 17.; d[1][2] = -8. / 17.;
        d[2][0] = 16. / 59.; d[2][1] = -36. / 59.; d[2][2] = 24. / 59.; d[2][3] = -4. / 59.;
        d[3][0] = -8. / 43.; d[3][1] = 24. / 43.; d[3][2] = -28. / 43.; d[3][3] = 16. / 43.; d[3][4] = -4. / 43;
        d[4][0] = 0.; d[4][1] = -4. / 49.; d[4][2] = 16. / 49.; d[4][3] = -24. / 49.; d[4][4] = 16. / 49.; d[4][5] = -4. / 49.;
        p->h0 = 17. / 48.;
    } else {
        c[0][0] = -1. / 60.; c[0][1] = 3. / 20.; c[0][2] = -3. / 4.; c[0][3] = 0.; c[0][4] = 3. / 4.; c[0][5] = -3. / 20.; c[0][6] = 1. / 60.;
        d[0][0] = 1. / 60.; d[0][1] = -1. / 10.; d[0][2] = 1. / 4.; d[0][3] = -1. / 3.; d[0][4] = 1. / 4.; d[0][5] = -1. / 10.; d[0][6] = 1. / 60.;
        static const double b4[6][9] = {
            {-1.582533518939116, 2.033378678700676, -0.141512858744873, -0.450398306578272, 0.104488069284042, 0.036577936277544, 0., 0., 0.},
            {-0.462059195631158, 0., 0.287258622978251, 0.258816087376832, -0.069112065532624, -0.014903449191300, 0., 0., 0.},
            {0.071247104721830, -0.636451095137907, 0., 0.606235523609147, -0.022902190275815, -0.018129342917256, 0., 0., 0.},
            {0.114713313798970, -0.290087484386815, -0.306681191361148, 0., 0.520262285050482, -0.051642265516119, 0.013435342414630, 0., 0.},
            {-0.036210680656541, 0.105400944933782, 0.015764336127392, -0.707905442575989, 0., 0.769199413962647, -0.164529643265203, 0.018281071473911, 0.},
            {-0.011398193015050, 0.020437334208704, 0.011220896474665, 0.063183694641876, -0.691649024426814, 0., 0.739709139060752, -0.147941827812150, 0.016437980868017}};
        static const double d4[6][9] = {
            {-0.105502234595941, 0.316506703787823, -0.316506703787823, 0.105502234595941, 0., 0., 0., 0., 0.},
            {0.071922084408557, -0.227753267293765, 0.251727295429951, -0.107883126612836, 0.011987014068093, 0., 0., 0., 0.},
            {-0.159350793065290, 0.557727775728513, -0.743637034304685, 0.478052379195869, -0.159350793065290, 0.026558465510882, 0., 0., 0.},
            {0.026870684829259, -0.120918081731666, 0.241836163463333, -0.282142190707221, 0.201530136219444, -0.080612054487778, 0.013435342414630, 0., 0.},
            {0., 0.018281071473911, -0.109686428843468, 0.274216072108671, -0.365621429478228, 0.274216072108671, -0.109686428843468, 0.018281071473911, 0.},
            {0., 0., 0.016437980868017, -0.098627885208100, 0.246569713020251, -0.328759617360334, 0.246569713020251, -0.098627885208100, 0.016437980868017}};
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 9; j++) {
                c[i + 1][j] = b4[i][j];
                d[i + 1][j] = d4[i][j];
            }
        p->h0 = 13649. / 43200.;
    }
}

/* RK coefficients: src/rk.cpp:8-98 */
static int set_rk(orc_problem *p) {
    switch (p->rkorder) {
        case 1:
            p->nstages = 1;
            p->A[0] = 0.; p->B[0] = 1.; p->C[0] = 0.; p->C[1] = 1.;
            break;
        case 2:
            p->nstages = 2;
            p->A[0] = 0.; p->A[1] = -1.; p->B[0] = 1.; p->B[1] = 0.5;
            p->C[0] = 0.; p->C[1] = 1.; p->C[2] = 1.;
            break;
        case 3:
            p->nstages = 3;
            p->A[0] = 0.; p->A[1] = -5. / 9.; p->A[2] = -153. / 128.;
            p->B[0] = 1. / 3.; p->B[1] = 15. / 16.; p->B[2] = 8. / 15.;
            p->C[0] = 0.; p->C[1] = 1. / 3.; p->C[2] = 3. / 4.; p->C[3] = 1.;
            break;
        case 4:
            p->nstages = 5;
            p->A[0] = 0.;
            p->A[1] = -567301805773. / 1357537059087.;
            p->A[2] = -2404267990393. / 2016746695238.;
            p->A[3] = -3550918686646. / 2091501179385.;
            p->A[4] = -1275806237668. / 842570457699.;
            p->B[0] = 1432997174477. / 9575080441755.;
            p->B[1] = 5161836677717. / 13612068292357.;
            p->B[2] = 1720146321549. / 2090206949498.;
            p->B[3] = 3134564353537. / 4481467310338.;
            p->B[4] = 2277821191437. / 14882151754819.;
            p->C[0] = 0.;
            p->C[1] = 1432997174477. / 9575080441755.;
            p->C[2] = 2526269341429. / 6820363962896.;
            p->C[3] = 2006345519317. / 3224310063776.;
            p->C[4] = 2802321613138. / 2924317926251.;
            p->C[5] = 1.;
            break;
        default:
            return 0;
    }
    return 1;
}

/* ------------------------------------------------------------------------- */
/* parametric perturbations: src/pert.cpp:7-136 */

static int pert_type(const char *s) {
    if (!strcmp(s, "constant")) return 0;
    if (!strcmp(s, "gaussian")) return 1;
    if (!strcmp(s, "ellipse")) return 2;
    if (!strcmp(s, "linear")) return 3;
    if (!strcmp(s, "boxcar")) return 4;
    return -1;
}

static void pert_init(pert_t *q, const int n[2], const int xm[2], const int xm_loc[2],
                      const double x[2], const double l[2]) {
    q->a = (double)(xm_loc[0] - xm[0]) / (double)(n[0] - 1) * l[0] + x[0];
    q->b = l[0] / (double)(n[0] - 1);
    q->c = (double)(xm_loc[1] - xm[1]) / (double)(n[1] - 1) * l[1] + x[1];
    q->d = l[1] / (double)(n[1] - 1);
}

static double pert_tfunc(const pert_t *q, double t) {
    return (t >= q->t0) ? 1. : t / q->t0;
}

static double pert_xyfunc(const pert_t *q, int i, int j) {
    double xyval = 0., xval, yval, eps = 1.e-14;
    double xi = q->b * (double)i + q->a, yj = q->d * (double)j + q->c;
    switch (q->type) {
        case 0:
            xyval = 1.;
            break;
        case 1:
            xval = (q->dx < eps) ? 0. : ((xi - q->x0) / q->dx) * ((xi - q->x0) / q->dx);
            yval = (q->dy < eps) ? 0. : ((yj - q->y0) / q->dy) * ((yj - q->y0) / q->dy);
            xyval = exp(-xval - yval);
            break;
        case 2:
            xval = (q->dx < eps) ? 0. : ((xi - q->x0) / q->dx) * ((xi - q->x0) / q->dx);
            yval = (q->dy < eps) ? 0. : ((yj - q->y0) / q->dy) * ((yj - q->y0) / q->dy);
            if (xval + yval <= 1.) xyval = 1.;
            break;
        case 3:
            xval = (q->dx < eps) ? 1 : xi / q->dx + q->x0;
            yval = (q->dy < eps) ? 1 : yj / q->dy + q->y0;
            xyval = xval * yval;
            break;
        case 4:
            if (q->dx < eps) {
                xval = 1.;
            } else if (fabs(fabs(xi - q->x0) - q->dx) < eps) {
                xval = 0.5;
            } else if (fabs(xi - q->x0) < q->dx) {
                xval = 1.;
            } else {
                xval = 0.;
            }
            if (q->dy < eps) {
                yval = 1.;
            } else if (fabs(fabs(yj - q->y0) - q->dy) < eps) {
                yval = 0.5;
            } else if (fabs(yj - q->y0) < q->dy) {
                yval = 1.;
            } else {
                yval = 0.;
            }
            xyval = xval * yval;
            break;
    }
    return xyval;
}

/* value k of perturbation q at fault node (i,j), time t: src/load.cpp:20-37 and friends */
static double pert_get(const pert_t *q, int k, int i, int j, double t) {
    return q->val[k] * pert_xyfunc(q, i, j) * pert_tfunc(q, t);
}

/* ------------------------------------------------------------------------- */
/* grid set-up: src/block.cpp:769-1046, surfaces src/surface.cpp:11-101 */

typedef struct {
    int n[2];
    double *x; /* [ndim][n0][n1] */
} surf_t;

static int surf_make(orc_problem *p, block_t *b, int loc, surf_t *sf) {
    int dirn = loc / 2;
    int index[2];
    if (dirn == 0) {
        index[0] = 1; index[1] = 2;
    } else if (dirn == 1) {
        index[0] = 0; index[1] = 2;
    } else {
        index[0] = 0; index[1] = 1;
    }
    int ndim = p->ndim;
    sf->n[0] = b->nx[index[0]];
    sf->n[1] = b->nx[index[1]];
    long nn = (long)sf->n[0] * sf->n[1];
    sf->x = zalloc(ndim * nn);
    if (strcmp(b->bfile[loc], "none") != 0) {
        if (!read_doubles(b->bfile[loc], sf->x, ndim * nn, 0)) {
            snprintf(p->err, sizeof p->err, "cannot read surface file %s", b->bfile[loc]);
            return 0;
        }
        return 1;
    }
    /* flat surface: x_in and l_in from block.cpp:183-213 */
    double xin[3], lin[2];
    for (int i = 0; i < 3; i++) xin[i] = b->xb[i];
    if (loc % 2 == 1) xin[dirn] = b->xb[dirn] + b->lb[dirn];
    lin[0] = b->lb[index[0]];
    lin[1] = b->lb[index[1]];
    for (int j = 0; j < sf->n[0]; j++)
        for (int k = 0; k < sf->n[1]; k++) sf->x[dirn * nn + j * sf->n[1] + k] = xin[dirn];
    for (int j = 0; j < sf->n[0]; j++)
        for (int k = 0; k < sf->n[1]; k++) {
            sf->x[index[0] * nn + j * sf->n[1] + k] = xin[index[0]] + lin[0] * (double)(j) / (double)(sf->n[0] - 1);
            if (ndim == 3)
                sf->x[index[1] * nn + j * sf->n[1] + k] = xin[index[1]] + lin[1] * (double)(k) / (double)(sf->n[1] - 1);
        }
    return 1;
}

static double sx(const surf_t *s, int i, int a, int b) {
    return s->x[(long)i * s->n[0] * s->n[1] + (long)a * s->n[1] + b];
}

static int set_grid(orc_problem *p, block_t *b) {
    int ndim = p->ndim;
    surf_t surf[6];
    memset(surf, 0, sizeof surf);
    for (int i = 0; i < 2 * ndim; i++)
        if (!surf_make(p, b, i, &surf[i])) return 0;
    for (int i = 0; i < 3; i++) b->dx[i] = 1. / (double)(b->nx[i] - 1);
    int nx = b->nx[0], ny = b->nx[1], nz = b->nx[2];
    const int *nxd = p->nxd;
    double *X = p->x;
    for (int i = 0; i < ndim; i++)
        for (int j = b->mlb[0]; j < b->prb[0]; j++)
            for (int k = b->mlb[1]; k < b->prb[1]; k++)
                for (int l = b->mlb[2]; l < b->prb[2]; l++) {
                    int jj = j - b->mlb[0], kk = k - b->mlb[1], ll = l - b->mlb[2];
                    double pp = (double)jj * b->dx[0], q = (double)kk * b->dx[1], r = (double)ll * b->dx[2];
                    long id = (long)i * nxd[0] + (long)j * nxd[1] + (long)k * nxd[2] + l;
                    X[id] = ((1. - pp) * sx(&surf[0], i, kk, ll) + pp * sx(&surf[1], i, kk, ll) +
                             (1. - q) * sx(&surf[2], i, jj, ll) + q * sx(&surf[3], i, jj, ll));
                    if (ndim == 3) X[id] += (1. - r) * sx(&surf[4], i, jj, kk) + r * sx(&surf[5], i, jj, kk);
                    X[id] -= ((1. - q) * (1. - pp) * sx(&surf[0], i, 0, ll) + (1. - q) * pp * sx(&surf[1], i, 0, ll) +
                              q * (1. - pp) * sx(&surf[0], i, ny - 1, ll) + q * pp * sx(&surf[1], i, ny - 1, ll));
                    if (ndim == 3) {
                        X[id] -= ((1. - pp) * (1. - r) * sx(&surf[0], i, kk, 0) + pp * (1. - r) * sx(&surf[1], i, kk, 0) +
                                  (1. - q) * (1. - r) * sx(&surf[2], i, jj, 0) + q * (1. - r) * sx(&surf[3], i, jj, 0) +
                                  (1. - pp) * r * sx(&surf[0], i, kk, nz - 1) + pp * r * sx(&surf[1], i, kk, nz - 1) +
                                  (1. - q) * r * sx(&surf[2], i, jj, nz - 1) + q * r * sx(&surf[3], i, jj, nz - 1));
                        X[id] += ((1. - pp) * (1. - q) * (1. - r) * sx(&surf[0], i, 0, 0) +
                                  pp * (1. - q) * (1. - r) * sx(&surf[1], i, 0, 0) +
                                  (1. - pp) * q * (1. - r) * sx(&surf[0], i, ny - 1, 0) +
                                  (1. - pp) * (1. - q) * r * sx(&surf[0], i, 0, nz - 1) +
                                  pp * q * (1. - r) * sx(&surf[1], i, ny - 1, 0) +
                                  pp * (1. - q) * r * sx(&surf[1], i, 0, nz - 1) +
                                  (1. - pp) * q * r * sx(&surf[0], i, ny - 1, nz - 1) +
                                  pp * q * r * sx(&surf[1], i, ny - 1, nz - 1));
                    }
                }
    (void)nx;
    for (int i = 0; i < 2 * ndim; i++) free(surf[i].x);

    /* metric derivatives: block.cpp:831-986 */
    long nloc = (long)b->nx[0] * b->nx[1] * b->nx[2];
    double *xp[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            xp[i][j] = zalloc(nloc);
            for (long m = 0; m < nloc; m++) xp[i][j][m] = (i == j) ? 1. : 0.;
        }
    int s = p->sbporder;
#define LOC(a, bb, c) (((long)((a)-b->mlb[0]) * b->nx[1] + ((bb)-b->mlb[1])) * b->nx[2] + ((c)-b->mlb[2]))
    for (int dirn = 0; dirn < ndim; dirn++) {
        for (int i = b->mlb[0]; i < b->prb[0]; i++)
            for (int j = b->mlb[1]; j < b->prb[1]; j++)
                for (int k = b->mlb[2]; k < b->prb[2]; k++) {
                    int pos[3] = {i, j, k};
                    int pcur = pos[dirn];
                    for (int l = 0; l < ndim; l++) {
                        double acc = 0.;
                        if (pcur < b->mc[dirn]) {
                            for (int n = 0; n < 3 * (s - 1); n++) {
                                int tp[3] = {i, j, k};
                                tp[dirn] = b->mlb[dirn] + n;
                                acc += p->fdc[pcur - b->mlb[dirn] + 1][n] *
                                       X[(long)l * nxd[0] + (long)tp[0] * nxd[1] + (long)tp[1] * nxd[2] + tp[2]] / b->dx[dirn];
                            }
                        } else if (pcur < b->mrb[dirn]) {
                            for (int n = 0; n < 2 * s - 1; n++) {
                                int tp[3] = {i, j, k};
                                tp[dirn] = pcur - s + 1 + n;
                                acc += p->fdc[0][n] *
                                       X[(long)l * nxd[0] + (long)tp[0] * nxd[1] + (long)tp[1] * nxd[2] + tp[2]] / b->dx[dirn];
                            }
                        } else {
                            for (int n = 0; n < 3 * (s - 1); n++) {
                                int tp[3] = {i, j, k};
                                tp[dirn] = b->prb[dirn] - 1 - n;
                                acc -= p->fdc[b->prb[dirn] - pcur][n] *
                                       X[(long)l * nxd[0] + (long)tp[0] * nxd[1] + (long)tp[1] * nxd[2] + tp[2]] / b->dx[dirn];
                            }
                        }
                        xp[l][dirn][LOC(i, j, k)] = acc;
                    }
                }
    }
    /* jacobian and metric: block.cpp:988-1014 */
    for (int i = b->mlb[0]; i < b->prb[0]; i++)
        for (int j = b->mlb[1]; j < b->prb[1]; j++)
            for (int k = b->mlb[2]; k < b->prb[2]; k++) {
                long L = LOC(i, j, k);
                long id = (long)i * nxd[1] + (long)j * nxd[2] + k;
                double jac = (xp[0][0][L] * (xp[1][1][L] * xp[2][2][L] - xp[1][2][L] * xp[2][1][L]) -
                              xp[1][0][L] * (xp[0][1][L] * xp[2][2][L] - xp[0][2][L] * xp[2][1][L]) +
                              xp[2][0][L] * (xp[0][1][L] * xp[1][2][L] - xp[0][2][L] * xp[1][1][L]));
                p->jac[id] = jac;
                if (!(jac > 0.)) {
                    snprintf(p->err, sizeof p->err, "non-positive jacobian at node %ld", id);
                    return 0;
                }
                for (int l = 0; l < ndim; l++)
                    for (int m = 0; m < ndim; m++)
                        p->metric[(long)l * ndim * nxd[0] + (long)m * nxd[0] + id] =
                            ((xp[(m + 1) % 3][(l + 1) % 3][L] * xp[(m + 2) % 3][(l + 2) % 3][L] -
                              xp[(m + 1) % 3][(l + 2) % 3][L] * xp[(m + 2) % 3][(l + 1) % 3][L]) /
                             jac);
            }
#undef LOC
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) free(xp[i][j]);
    return 1;
}

/* ------------------------------------------------------------------------- */
/* material helpers: src/material.cpp */

static double mat_cs(const block_t *b) { return sqrt(b->g / b->rho); }
static double mat_cp(const block_t *b) { return sqrt((b->lam + 2. * b->g) / b->rho); }

/* wave speeds, impedances and gamma of one node of a heterogeneous material:
   boundary.cpp:303-314 and interface.cpp:614-638 (pow(x, 2) is x * x) */
typedef struct {
    double cp, cs, zp, zs, gamma;
} nodemat_t;
static nodemat_t node_mat(const orc_problem *p, long id) {
    const long n = p->nxd[0];
    const double rho = p->mat[id], lam = p->mat[n + id], g = p->mat[2 * n + id];
    nodemat_t m;
    m.cp = sqrt((lam + 2. * g) / rho);
    m.cs = sqrt(g / rho);
    m.zp = rho * m.cp;
    m.zs = rho * m.cs;
    m.gamma = 1. - 2. * ((m.cs / m.cp) * (m.cs / m.cp));
    return m;
}

/* outer boundary set-up: src/boundary.cpp:15-240 */
static void bound_init(orc_problem *p, block_t *b, int loc) {
    bound_t *bd = &b->bound[loc];
    int ndim = p->ndim;
    const char *bt = b->btype[loc];
    bd->location = loc;
    bd->active = strcmp(bt, "none") != 0;
    if (!bd->active) return;
    int mlb[3], prb[3];
    for (int i = 0; i < 3; i++) mlb[i] = b->mlb[i];
    int dirn = loc / 2;
    int oth[2];
    if (dirn == 0) {
        oth[0] = 1; oth[1] = 2;
    } else if (dirn == 1) {
        oth[0] = 0; oth[1] = 2;
    } else {
        oth[0] = 0; oth[1] = 1;
    }
    bd->n0 = b->nx[oth[0]];
    bd->n1 = b->nx[oth[1]];
    if (loc % 2 == 1) mlb[dirn] += b->nx[dirn] - 1;
    prb[dirn] = mlb[dirn] + 1;
    prb[oth[0]] = mlb[oth[0]] + bd->n0;
    prb[oth[1]] = mlb[oth[1]] + bd->n1;
    for (int i = 0; i < 3; i++) {
        bd->mlb[i] = mlb[i];
        bd->prb[i] = prb[i];
    }
    bd->cp = mat_cp(b);
    bd->cs = mat_cs(b);
    bd->zp = b->rho * bd->cp;
    bd->zs = b->rho * bd->cs;
    bd->gamma = 1. - 2. * ((bd->cs / bd->cp) * (bd->cs / bd->cp));
    if (!strcmp(bt, "absorbing")) {
        bd->r = 0.; bd->alpha = 2.; bd->theta = 0.;
    } else if (!strcmp(bt, "free")) {
        bd->r = -1.; bd->alpha = 1.; bd->theta = 0.;
    } else {
        bd->r = 1.; bd->alpha = 0.; bd->theta = 1.;
    }
    long nn = (long)bd->n0 * bd->n1;
    for (int k = 0; k < ndim; k++) bd->nx[k] = zalloc(nn);
    bd->dl = zalloc(nn);
    const int *nxd = p->nxd;
    for (int i = 0; i < bd->n0; i++)
        for (int j = 0; j < bd->n1; j++) {
            int pos[3];
            pos[dirn] = mlb[dirn];
            pos[oth[0]] = i + mlb[oth[0]];
            pos[oth[1]] = j + mlb[oth[1]];
            long id = (long)pos[0] * nxd[1] + (long)pos[1] * nxd[2] + pos[2];
            long ij = (long)i * bd->n1 + j;
            double dl = 0.;
            for (int k = 0; k < ndim; k++) {
                double m = p->metric[(long)dirn * ndim * nxd[0] + (long)k * nxd[0] + id];
                dl += m * m;
                bd->nx[k][ij] = m;
            }
            dl = sqrt(dl);
            for (int k = 0; k < ndim; k++) bd->nx[k][ij] /= dl;
            dl /= p->h0 * b->dx[dirn];
            bd->dl[ij] = dl;
            if (loc % 2 == 0)
                for (int k = 0; k < ndim; k++) bd->nx[k][ij] = -bd->nx[k][ij];
        }
}

/* ------------------------------------------------------------------------- */
/* rotations: src/boundary.cpp:505-568 */

typedef struct {
    double v1, v2, v3, s11, s12, s13, s22, s23, s33;
} bf_t;

static bf_t rot_xy_nt(bf_t b, const double nn[3], const double t1[3], const double t2[3]) {
    bf_t o;
    o.v1 = nn[0] * b.v1 + nn[1] * b.v2 + nn[2] * b.v3;
    o.v2 = t1[0] * b.v1 + t1[1] * b.v2 + t1[2] * b.v3;
    o.v3 = t2[0] * b.v1 + t2[1] * b.v2 + t2[2] * b.v3;
    o.s11 = (nn[0] * (b.s11 * nn[0] + b.s12 * nn[1] + b.s13 * nn[2]) + nn[1] * (b.s12 * nn[0] + b.s22 * nn[1] + b.s23 * nn[2]) +
             nn[2] * (b.s13 * nn[0] + b.s23 * nn[1] + b.s33 * nn[2]));
    o.s12 = (nn[0] * (b.s11 * t1[0] + b.s12 * t1[1] + b.s13 * t1[2]) + nn[1] * (b.s12 * t1[0] + b.s22 * t1[1] + b.s23 * t1[2]) +
             nn[2] * (b.s13 * t1[0] + b.s23 * t1[1] + b.s33 * t1[2]));
    o.s13 = (nn[0] * (b.s11 * t2[0] + b.s12 * t2[1] + b.s13 * t2[2]) + nn[1] * (b.s12 * t2[0] + b.s22 * t2[1] + b.s23 * t2[2]) +
             nn[2] * (b.s13 * t2[0] + b.s23 * t2[1] + b.s33 * t2[2]));
    o.s22 = (t1[0] * (b.s11 * t1[0] + b.s12 * t1[1] + b.s13 * t1[2]) + t1[1] * (b.s12 * t1[0] + b.s22 * t1[1] + b.s23 * t1[2]) +
             t1[2] * (b.s13 * t1[0] + b.s23 * t1[1] + b.s33 * t1[2]));
    o.s23 = (t1[0] * (b.s11 * t2[0] + b.s12 * t2[1] + b.s13 * t2[2]) + t1[1] * (b.s12 * t2[0] + b.s22 * t2[1] + b.s23 * t2[2]) +
             t1[2] * (b.s13 * t2[0] + b.s23 * t2[1] + b.s33 * t2[2]));
    o.s33 = (t2[0] * (b.s11 * t2[0] + b.s12 * t2[1] + b.s13 * t2[2]) + t2[1] * (b.s12 * t2[0] + b.s22 * t2[1] + b.s23 * t2[2]) +
             t2[2] * (b.s13 * t2[0] + b.s23 * t2[1] + b.s33 * t2[2]));
    return o;
}

static bf_t rot_nt_xy(bf_t b, const double nn[3], const double t1[3], const double t2[3]) {
    bf_t o;
    o.v1 = nn[0] * b.v1 + t1[0] * b.v2 + t2[0] * b.v3;
    o.v2 = nn[1] * b.v1 + t1[1] * b.v2 + t2[1] * b.v3;
    o.v3 = nn[2] * b.v1 + t1[2] * b.v2 + t2[2] * b.v3;
    o.s11 = (nn[0] * (b.s11 * nn[0] + b.s12 * t1[0] + b.s13 * t2[0]) + t1[0] * (b.s12 * nn[0] + b.s22 * t1[0] + b.s23 * t2[0]) +
             t2[0] * (b.s13 * nn[0] + b.s23 * t1[0] + b.s33 * t2[0]));
    o.s12 = (nn[0] * (b.s11 * nn[1] + b.s12 * t1[1] + b.s13 * t2[1]) + t1[0] * (b.s12 * nn[1] + b.s22 * t1[1] + b.s23 * t2[1]) +
             t2[0] * (b.s13 * nn[1] + b.s23 * t1[1] + b.s33 * t2[1]));
    o.s13 = (nn[0] * (b.s11 * nn[2] + b.s12 * t1[2] + b.s13 * t2[2]) + t1[0] * (b.s12 * nn[2] + b.s22 * t1[2] + b.s23 * t2[2]) +
             t2[0] * (b.s13 * nn[2] + b.s23 * t1[2] + b.s33 * t2[2]));
    o.s22 = (nn[1] * (b.s11 * nn[1] + b.s12 * t1[1] + b.s13 * t2[1]) + t1[1] * (b.s12 * nn[1] + b.s22 * t1[1] + b.s23 * t2[1]) +
             t2[1] * (b.s13 * nn[1] + b.s23 * t1[1] + b.s33 * t2[1]));
    o.s23 = (nn[1] * (b.s11 * nn[2] + b.s12 * t1[2] + b.s13 * t2[2]) + t1[1] * (b.s12 * nn[2] + b.s22 * t1[2] + b.s23 * t2[2]) +
             t2[1] * (b.s13 * nn[2] + b.s23 * t1[2] + b.s33 * t2[2]));
    o.s33 = (nn[2] * (b.s11 * nn[2] + b.s12 * t1[2] + b.s13 * t2[2]) + t1[2] * (b.s12 * nn[2] + b.s22 * t1[2] + b.s23 * t2[2]) +
             t2[2] * (b.s13 * nn[2] + b.s23 * t1[2] + b.s33 * t2[2]));
    return o;
}

/* ------------------------------------------------------------------------- */
/* block rate: src/block.cpp:1048-1278 (mode II), 1384-1539 (mode III), 1541-2050 (3D) */

static void calc_df(orc_problem *p, block_t *b, double dt) {
    const int ndim = p->ndim, mode = p->mode, s = p->sbporder;
    const long n0 = p->nxd[0];
    const int *nxd = p->nxd;
    double *F = p->f, *DF = p->df, *M = p->metric, *J = p->jac;
    double invrho = dt / b->rho / b->dx[0];
    double g2lam = dt * (2. * b->g + b->lam) / b->dx[0];
    double g = dt * b->g / b->dx[0];
    double lambda = dt * b->lam / b->dx[0];
    const double cdiss = p->cdiss;
    const int nf = (ndim == 3) ? 9 : ((mode == 2) ? 5 : 3);
    for (int d = 0; d < ndim; d++) {
        if (d > 0) {
            invrho *= b->dx[d - 1] / b->dx[d];
            g2lam *= b->dx[d - 1] / b->dx[d];
            g *= b->dx[d - 1] / b->dx[d];
            lambda *= b->dx[d - 1] / b->dx[d];
        }
        const long stride = (d == 0) ? nxd[1] : ((d == 1) ? nxd[2] : 1);
        for (int i = b->mlb[0]; i < b->prb[0]; i++)
            for (int j = b->mlb[1]; j < b->prb[1]; j++)
                for (int k = b->mlb[2]; k < b->prb[2]; k++) {
                    const long i1 = (long)i * nxd[1] + (long)j * nxd[2] + k;
                    const int pos = (d == 0) ? i : ((d == 1) ? j : k);
                    int index3, ntap;
                    long base;
                    long step;
                    double sg;
                    if (pos < b->mc[d]) {
                        index3 = pos - b->mlb[d] + 1;
                        ntap = 3 * (s - 1);
                        base = i1 + (long)(b->mlb[d] - pos) * stride;
                        step = stride;
                        sg = 1.;
                    } else if (pos < b->mrb[d]) {
                        index3 = 0;
                        ntap = 2 * s - 1;
                        base = i1 + (long)(-s + 1) * stride;
                        step = stride;
                        sg = 1.;
                    } else {
                        index3 = b->prb[d] - pos;
                        ntap = 3 * (s - 1);
                        base = i1 + (long)(b->prb[d] - 1 - pos) * stride;
                        step = -stride;
                        sg = -1.;
                    }
                    double ir = invrho, gl = g2lam, gg = g, la = lambda;
                    if (p->hetmat) { /* per node (block.cpp:1061-1065 and the other passes) */
                        const double rh = p->mat[i1], lm = p->mat[n0 + i1], gm = p->mat[2 * n0 + i1];
                        ir = dt / rh / b->dx[d];
                        gl = dt * (2. * gm + lm) / b->dx[d];
                        gg = dt * gm / b->dx[d];
                        la = dt * lm / b->dx[d];
                    }
                    const double invjac = ir / J[i1];
                    const double *cf = p->fdc[index3];
                    const double *dc = p->dsc[index3];
                    for (int n = 0; n < ntap; n++) {
                        const long i2 = base + (long)n * step;
                        const double c = cf[n];
                        double t[9];
                        if (ndim == 3) {
                            const double *m2 = M + (long)(d * ndim) * n0;
                            const double ma = m2[i2], mb = m2[n0 + i2], mcc = m2[2 * n0 + i2];
                            const double ca = m2[i1], cb = m2[n0 + i1], cc = m2[2 * n0 + i1];
                            t[0] = (invjac * c * J[i2] * (ma * F[3 * n0 + i2] + mb * F[4 * n0 + i2] + mcc * F[5 * n0 + i2]));
                            t[1] = (invjac * c * J[i2] * (ma * F[4 * n0 + i2] + mb * F[6 * n0 + i2] + mcc * F[7 * n0 + i2]));
                            t[2] = (invjac * c * J[i2] * (ma * F[5 * n0 + i2] + mb * F[7 * n0 + i2] + mcc * F[8 * n0 + i2]));
                            t[3] = c * (gl * ca * F[i2] + la * (cb * F[n0 + i2] + cc * F[2 * n0 + i2]));
                            t[4] = c * gg * (ca * F[n0 + i2] + cb * F[i2]);
                            t[5] = c * gg * (ca * F[2 * n0 + i2] + cc * F[i2]);
                            t[6] = c * (gl * cb * F[n0 + i2] + la * (ca * F[i2] + cc * F[2 * n0 + i2]));
                            t[7] = c * gg * (cb * F[2 * n0 + i2] + cc * F[n0 + i2]);
                            t[8] = c * (gl * cc * F[2 * n0 + i2] + la * (ca * F[i2] + cb * F[n0 + i2]));
                        } else if (mode == 2) {
                            const double *m2 = M + (long)(d * ndim) * n0;
                            const double ma = m2[i2], mb = m2[n0 + i2];
                            const double ca = m2[i1], cb = m2[n0 + i1];
                            t[0] = (invjac * c * J[i2] * (ma * F[2 * n0 + i2] + mb * F[3 * n0 + i2]));
                            t[1] = (invjac * c * J[i2] * (ma * F[3 * n0 + i2] + mb * F[4 * n0 + i2]));
                            t[2] = c * (gl * ca * F[i2] + la * cb * F[n0 + i2]);
                            t[3] = gg * c * (ca * F[n0 + i2] + cb * F[i2]);
                            t[4] = c * (gl * cb * F[n0 + i2] + la * ca * F[i2]);
                        } else {
                            const double *m2 = M + (long)(d * ndim) * n0;
                            const double ma = m2[i2], mb = m2[n0 + i2];
                            const double ca = m2[i1], cb = m2[n0 + i1];
                            t[0] = invjac * c * J[i2] * (ma * F[n0 + i2] + mb * F[2 * n0 + i2]);
                            t[1] = gg * ca * c * F[i2];
                            t[2] = gg * cb * c * F[i2];
                        }
                        for (int q = 0; q < nf; q++) {
                            if (sg > 0.)
                                DF[q * n0 + i1] += t[q];
                            else
                                DF[q * n0 + i1] -= t[q];
                        }
                        if (cdiss > 0.) {
                            for (int q = 0; q < nf; q++)
                                DF[q * n0 + i1] += cdiss * (dc[n] * J[i2] * F[q * n0 + i2]) / J[i1];
                        }
                    }
                }
    }
    /* mode II plastic szz rate: block.cpp:1280-1294 */
    if (ndim == 2 && mode == 2 && p->is_plastic) {
        double nu = 0.5 * b->lam / (b->lam + b->g);
        for (int i = b->mlb[0]; i < b->prb[0]; i++)
            for (int j = b->mlb[1]; j < b->prb[1]; j++) {
                long id = (long)i * nxd[1] + j;
                /* the second term reads the material array one x row on
                   (mat[nxd[1] + index], block.cpp:1289-1291): rho of (i+1, j),
                   past the last row lambda of (0, j) */
                if (p->hetmat) nu = 0.5 * p->mat[n0 + id] / (p->mat[n0 + id] + p->mat[nxd[1] + id]);
                DF[5 * n0 + id] = nu * (DF[2 * n0 + id] + DF[4 * n0 + id]);
            }
    }
}

/* outer boundary SAT: src/boundary.cpp:265-503 */
static void apply_bound(orc_problem *p, block_t *b, bound_t *bd, double dt) {
    if (!bd->active) return;
    const int ndim = p->ndim, mode = p->mode;
    const long n0 = p->nxd[0];
    const int *nxd = p->nxd;
    double *F = p->f, *DF = p->df;
    double nn[3] = {0., 0., 0.}, t1[3], t2[3], h = 0.;
    const double r = bd->r;
    (void)b;
    for (int i = bd->mlb[0]; i < bd->prb[0]; i++)
        for (int j = bd->mlb[1]; j < bd->prb[1]; j++)
            for (int k = bd->mlb[2]; k < bd->prb[2]; k++) {
                long id = (long)i * nxd[1] + (long)j * nxd[2] + k;
                long ij;
                switch (bd->location) {
                    case 0: case 1: ij = (long)(j - bd->mlb[1]) * bd->n1 + (k - bd->mlb[2]); break;
                    case 2: case 3: ij = (long)(i - bd->mlb[0]) * bd->n1 + (k - bd->mlb[2]); break;
                    default: ij = (long)(i - bd->mlb[0]) * bd->n1 + (j - bd->mlb[1]);
                }
                for (int l = 0; l < ndim; l++) {
                    nn[l] = bd->nx[l][ij];
                    h = dt * bd->dl[ij];
                }
                double cp = bd->cp, cs = bd->cs, zp = bd->zp, zs = bd->zs, gamma = bd->gamma;
                if (p->hetmat) {
                    const nodemat_t m = node_mat(p, id);
                    cp = m.cp; cs = m.cs; zp = m.zp; zs = m.zs; gamma = m.gamma;
                }
                if (fabs(nn[0]) > fabs(nn[1]) && fabs(nn[0]) > fabs(nn[2])) {
                    t1[2] = 0.;
                    t1[1] = nn[0] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
                    t1[0] = -nn[1] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
                } else if (fabs(nn[1]) > fabs(nn[2])) {
                    t1[2] = 0.;
                    t1[0] = nn[1] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
                    t1[1] = -nn[0] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
                } else {
                    t1[1] = 0.;
                    t1[0] = nn[2] / sqrt(nn[0] * nn[0] + nn[2] * nn[2]);
                    t1[2] = -nn[0] / sqrt(nn[0] * nn[0] + nn[2] * nn[2]);
                }
                t2[0] = nn[1] * t1[2] - nn[2] * t1[1];
                t2[1] = nn[2] * t1[0] - nn[0] * t1[2];
                t2[2] = nn[0] * t1[1] - nn[1] * t1[0];
                bf_t bb, brots, brot;
                if (ndim == 3) {
                    bb.v1 = F[id]; bb.v2 = F[n0 + id]; bb.v3 = F[2 * n0 + id];
                    bb.s11 = F[3 * n0 + id]; bb.s12 = F[4 * n0 + id]; bb.s13 = F[5 * n0 + id];
                    bb.s22 = F[6 * n0 + id]; bb.s23 = F[7 * n0 + id]; bb.s33 = F[8 * n0 + id];
                } else if (mode == 2) {
                    bb.v1 = F[id]; bb.v2 = F[n0 + id]; bb.v3 = 0.;
                    bb.s11 = F[2 * n0 + id]; bb.s12 = F[3 * n0 + id]; bb.s13 = 0.;
                    bb.s22 = F[4 * n0 + id]; bb.s23 = 0.; bb.s33 = 0.;
                } else {
                    bb.v1 = 0.; bb.v2 = 0.; bb.v3 = F[id];
                    bb.s11 = 0.; bb.s12 = 0.; bb.s13 = F[n0 + id];
                    bb.s22 = 0.; bb.s23 = F[2 * n0 + id]; bb.s33 = 0.;
                }
                brot = rot_xy_nt(bb, nn, t1, t2);
                brots = brot;
                /* calc_hat: boundary.cpp:494-503 */
                double hps = (r + 1.) * 0.5 * (brot.s11 - zp * brot.v1), hpv = (r - 1.) * 0.5 * (brot.s11 / zp - brot.v1);
                double h1s = (r + 1.) * 0.5 * (brot.s12 - zs * brot.v2), h1v = (r - 1.) * 0.5 * (brot.s12 / zs - brot.v2);
                double h2s = (r + 1.) * 0.5 * (brot.s13 - zs * brot.v3), h2v = (r - 1.) * 0.5 * (brot.s13 / zs - brot.v3);
                brot.v1 -= hpv;
                brot.v2 = 0.;
                brot.v3 = 0.;
                brot.s22 = gamma * (brot.s11 - hps);
                brot.s33 = gamma * (brot.s11 - hps);
                brot.s11 -= hps;
                brot.s12 = 0.;
                brot.s13 = 0.;
                brot.s23 = 0.;
                bb = rot_nt_xy(brot, nn, t1, t2);
                const double alpha = bd->alpha, theta = bd->theta;
                if (ndim == 3) {
                    DF[id] -= alpha * cp * h * bb.v1;
                    DF[n0 + id] -= alpha * cp * h * bb.v2;
                    DF[2 * n0 + id] -= alpha * cp * h * bb.v3;
                    DF[3 * n0 + id] -= theta * cp * h * bb.s11;
                    DF[4 * n0 + id] -= theta * cp * h * bb.s12;
                    DF[5 * n0 + id] -= theta * cp * h * bb.s13;
                    DF[6 * n0 + id] -= theta * cp * h * bb.s22;
                    DF[7 * n0 + id] -= theta * cp * h * bb.s23;
                    DF[8 * n0 + id] -= theta * cp * h * bb.s33;
                } else if (mode == 2) {
                    DF[id] -= cp * h * bb.v1;
                    DF[n0 + id] -= cp * h * bb.v2;
                    DF[2 * n0 + id] -= cp * h * bb.s11;
                    DF[3 * n0 + id] -= cp * h * bb.s12;
                    DF[4 * n0 + id] -= cp * h * bb.s22;
                    if (p->is_plastic) DF[5 * n0 + id] -= cp * h * bb.s33;
                }
                brots.v1 = 0.;
                brots.v2 -= h1v;
                brots.v3 -= h2v;
                brots.s11 = 0.;
                brots.s12 -= h1s;
                brots.s13 -= h2s;
                brots.s22 = 0.;
                brots.s23 = 0.;
                brots.s33 = 0.;
                bb = rot_nt_xy(brots, nn, t1, t2);
                if (ndim == 3) {
                    DF[id] -= alpha * cs * h * bb.v1;
                    DF[n0 + id] -= alpha * cs * h * bb.v2;
                    DF[2 * n0 + id] -= alpha * cs * h * bb.v3;
                    DF[3 * n0 + id] -= theta * cs * h * bb.s11;
                    DF[4 * n0 + id] -= theta * cs * h * bb.s12;
                    DF[5 * n0 + id] -= theta * cs * h * bb.s13;
                    DF[6 * n0 + id] -= theta * cs * h * bb.s22;
                    DF[7 * n0 + id] -= theta * cs * h * bb.s23;
                    DF[8 * n0 + id] -= theta * cs * h * bb.s33;
                } else if (mode == 2) {
                    DF[id] -= cs * h * bb.v1;
                    DF[n0 + id] -= cs * h * bb.v2;
                    DF[2 * n0 + id] -= cs * h * bb.s11;
                    DF[3 * n0 + id] -= cs * h * bb.s12;
                    DF[4 * n0 + id] -= cs * h * bb.s22;
                } else {
                    DF[id] -= cs * h * bb.v3;
                    DF[n0 + id] -= cs * h * bb.s13;
                    DF[2 * n0 + id] -= cs * h * bb.s23;
                }
            }
}

/* ------------------------------------------------------------------------- */
/* friction laws */

typedef struct {
    double v11, v12, v13, s11, s12, s13;
    double v21, v22, v23, s21, s22, s23;
} iff_t;

/* interface::solve_locked: src/interface.cpp:1017-1028 */
static void solve_locked(double v1, double v2, double s1, double s2, double z1, double z2, double *ov1,
                         double *ov2, double *os1, double *os2) {
    double s = (z2 * (s1 - z1 * v1) + z1 * (s2 + z2 * v2)) / (z1 + z2);
    double v = (s - s1) / z1 + v1;
    *os1 = s;
    *os2 = s;
    *ov1 = v;
    *ov2 = v;
}

/* slipweak::calc_mu: src/slipweak.cpp:253-308 */
static double sw_calc_mu(const iface_t *f, int ii, int jj, double t) {
    double dct = 0., must = 0., mudt = 0., trupt = 0., tct = 0.;
    for (int m = 0; m < f->nperts; m++) {
        dct += pert_get(&f->perts[m], 0, ii, jj, t);
        must += pert_get(&f->perts[m], 1, ii, jj, t);
        mudt += pert_get(&f->perts[m], 2, ii, jj, t);
        trupt += pert_get(&f->perts[m], 4, ii, jj, t);
        tct += pert_get(&f->perts[m], 5, ii, jj, t);
    }
    long index = (long)ii * f->n[1] + jj;
    if (f->param_file) {
        dct += f->par[0][index];
        must += f->par[1][index];
        mudt += f->par[2][index];
        trupt += f->par[4][index];
        tct += f->par[5][index];
    }
    double f1, f2;
    if (dct == 0. || f->u[index] >= dct)
        f1 = 1.;
    else
        f1 = f->u[index] / dct;
    if (trupt <= 0. || t < trupt)
        f2 = 0.;
    else if (t >= trupt && t < trupt + tct)
        f2 = (tct == 0.) ? 1. : (t - trupt) / tct;
    else
        f2 = 1.;
    return (f1 >= f2) ? must + (mudt - must) * f1 : must + (mudt - must) * f2;
}

/* stz: src/stz.cpp:436-484 */
static double stz_vpl(double mu, const double *pr) {
    double chi = pr[3], v0 = pr[4], f0 = pr[5], a = pr[6], muy = pr[7];
    if (mu <= muy) return 0.;
    return v0 * exp(-f0 + mu / a - 1. / chi) * (1. - muy / mu);
}
static double stz_dvpldmu(double mu, const double *pr) {
    double a = pr[6], muy = pr[7];
    if (mu <= muy) return 0.;
    return stz_vpl(mu, pr) * (1. / a - muy / mu / (mu - muy));
}
static double stz_func(double mu, const double *pr) { return pr[1] * stz_vpl(mu, pr) - pr[2] * mu - pr[0]; }
static double stz_der(double mu, const double *pr) { return pr[1] * stz_dvpldmu(mu, pr) - pr[2]; }

/* bracketed Newton: src/utilities.cpp:89-179; returns 0 on failure */
static int solve_newton(double xmin, double xmax, const double *pr, double *out) {
    int i = 0;
    const int nmax = 100;
    const double tol = 2.e-16;
    double func, der, x, xl, xh, fh, dx, dxold, temp;
    x = 0.5 * (xmin + xmax);
    xh = xmax;
    xl = xmin;
    func = stz_func(x, pr);
    fh = stz_func(xh, pr);
    if (isinf(fh)) {
        int guard = 0;
        while (1) {
            if (!isinf(func)) {
                if (func > 0.) {
                    xh = x;
                    break;
                } else {
                    xl = x;
                }
            } else {
                xh = x;
            }
            x = 0.5 * (xh + xl);
            func = stz_func(x, pr);
            if (++guard > 4000) return 0;
        }
    }
    x = 0.5 * (xh + xl);
    func = stz_func(x, pr);
    der = stz_der(x, pr);
    dx = fabs(xh - xl);
    dxold = dx;
    while (i < nmax) {
        if (der == 0.) return 0;
        if ((((x - xh) * der - func) * ((x - xl) * der - func) > 0.) || fabs(2. * func) > fabs(dxold * der)) {
            dxold = dx;
            dx = 0.5 * (xh - xl);
            x = xl + dx;
            if (xl == x) break;
        } else {
            dxold = dx;
            dx = func / der;
            temp = x;
            x = x - dx;
            if (temp == x) break;
        }
        if (fabs(dx) < tol) break;
        func = stz_func(x, pr);
        der = stz_der(x, pr);
        if (func < 0.)
            xl = x;
        else
            xh = x;
        i++;
    }
    if (i == nmax) return 0;
    *out = x;
    return 1;
}

/* stz::calc_mu: src/stz.cpp:263-309 */
static int stz_calc_mu(const iface_t *f, double phi, double eta, double snc, int ii, int jj, double t,
                       double *mu) {
    double pr[8];
    long index = (long)ii * f->n[1] + jj;
    pr[0] = phi; pr[1] = eta; pr[2] = snc; pr[3] = f->state[index];
    pr[4] = 0.; pr[5] = 0.; pr[6] = 0.; pr[7] = 0.;
    for (int m = 0; m < f->nperts; m++) {
        pr[4] += pert_get(&f->perts[m], 0, ii, jj, t);
        pr[5] += pert_get(&f->perts[m], 1, ii, jj, t);
        pr[6] += pert_get(&f->perts[m], 2, ii, jj, t);
        pr[7] += pert_get(&f->perts[m], 3, ii, jj, t);
    }
    if (f->param_file) {
        pr[4] += f->par[0][index];
        pr[5] += f->par[1][index];
        pr[6] += f->par[2][index];
        pr[7] += f->par[3][index];
    }
    if (pr[7] >= -phi / snc) {
        *mu = -phi / snc;
        return 1;
    }
    return solve_newton(pr[7], -phi / snc, pr, mu);
}

/* stz::calc_dstatedt + chihat: src/stz.cpp:311-356; returns 0 if V exceeds v1 */
static int stz_dstatedt(const iface_t *f, double vhat, double shat, int ii, int jj, double t, double *out) {
    double c0t = 0., Rt = 0., betat = 0., chiwt = 0., v1t = 0.;
    for (int m = 0; m < f->nperts; m++) {
        c0t += pert_get(&f->perts[m], 4, ii, jj, t);
        Rt += pert_get(&f->perts[m], 5, ii, jj, t);
        betat += pert_get(&f->perts[m], 6, ii, jj, t);
        chiwt += pert_get(&f->perts[m], 7, ii, jj, t);
        v1t += pert_get(&f->perts[m], 8, ii, jj, t);
    }
    long index = (long)ii * f->n[1] + jj;
    if (f->param_file) {
        c0t += f->par[4][index];
        Rt += f->par[5][index];
        betat += f->par[6][index];
        chiwt += f->par[7][index];
        v1t += f->par[8][index];
    }
    if (vhat > v1t) return 0;
    double chihat = (vhat == 0.) ? chiwt : chiwt / log(v1t / vhat);
    *out = vhat * shat / c0t * (1. - f->state[index] / chihat) - Rt * exp(-betat / f->state[index]);
    return 1;
}

/* friction::solve_fs / slipweak::solve_fs: src/friction.cpp:400-435, src/slipweak.cpp:206-251 */
static int solve_fs(orc_problem *p, iface_t *f, double phi, double eta, double snc, int ii, int jj, double t,
                    double *bv, double *bs) {
    (void)p;
    if (f->kind == 2) {
        double c0t = 0.;
        for (int m = 0; m < f->nperts; m++) c0t += pert_get(&f->perts[m], 3, ii, jj, t);
        long index = (long)ii * f->n[1] + jj;
        if (f->param_file) c0t += f->par[3][index];
        if (snc < 0.) {
            double mu = sw_calc_mu(f, ii, jj, t);
            if (c0t + mu * fabs(snc) > phi) {
                *bv = 0.;
                *bs = phi;
            } else {
                *bs = c0t + mu * fabs(snc);
                *bv = (phi - *bs) / eta;
            }
        } else {
            if (phi > c0t) {
                *bs = c0t;
                *bv = (phi - *bs) / eta;
            } else {
                *bv = 0.;
                *bs = phi;
            }
        }
        return 1;
    }
    if (snc < 0.) {
        double mu = 0.;
        if (f->kind == 3) {
            if (!stz_calc_mu(f, phi, eta, snc, ii, jj, t, &mu)) {
                snprintf(p->err, sizeof p->err, "Newton's method failed to converge");
                return 0;
            }
        }
        if (mu * fabs(snc) > phi) {
            *bv = 0.;
            *bs = phi;
        } else {
            *bs = mu * fabs(snc);
            *bv = (phi - *bs) / eta;
        }
    } else {
        *bs = 0.;
        *bv = phi / eta;
    }
    if (f->has_state) {
        if (!stz_dstatedt(f, *bv, *bs, ii, jj, t, &f->dstatedt[(long)ii * f->n[1] + jj])) {
            snprintf(p->err, sizeof p->err, "Slip velocity exceeds melting value");
            return 0;
        }
    }
    return 1;
}

/* friction::solve_friction: src/friction.cpp:293-398 */
static int solve_friction(orc_problem *p, iface_t *f, iff_t *in, double snc, double z1, double z2, int ii, int jj,
                          double t, iff_t *out) {
    const double eta = z1 * z2 / (z1 + z2);
    double phi, phi2, phi3, v2, v3;
    long index = (long)ii * f->n[1] + jj;
    if (f->load_file) {
        snc += f->s1[index];
        in->s12 += f->s2[index];
        in->s22 += f->s2[index];
        in->s13 += f->s3[index];
        in->s23 += f->s3[index];
    }
    for (int k = 0; k < f->nloads; k++) {
        snc += pert_get(&f->loads[k], 0, ii, jj, t);
        in->s12 += pert_get(&f->loads[k], 1, ii, jj, t);
        in->s22 += pert_get(&f->loads[k], 1, ii, jj, t);
        in->s13 += pert_get(&f->loads[k], 2, ii, jj, t);
        in->s23 += pert_get(&f->loads[k], 2, ii, jj, t);
    }
    phi2 = eta * (in->s12 / z1 - in->v12 + in->s22 / z2 + in->v22);
    phi3 = eta * (in->s13 / z1 - in->v13 + in->s23 / z2 + in->v23);
    phi = sqrt(phi2 * phi2 + phi3 * phi3);
    double bv, bs;
    if (!solve_fs(p, f, phi, eta, snc, ii, jj, t, &bv, &bs)) return 0;
    if (bv == 0.) {
        v2 = 0.;
        v3 = 0.;
    } else {
        v2 = bv * phi2 / (eta * bv + bs);
        v3 = bv * phi3 / (eta * bv + bs);
    }
    out->s12 = phi2 - eta * v2;
    out->s22 = out->s12;
    out->s13 = phi3 - eta * v3;
    out->s23 = out->s13;
    out->v12 = (out->s12 - in->s12) / z1 + in->v12;
    out->v22 = (-out->s22 + in->s22) / z2 + in->v22;
    out->v13 = (out->s13 - in->s13) / z1 + in->v13;
    out->v23 = (-out->s23 + in->s23) / z2 + in->v23;
    f->v[index] = bv;
    f->s[index] = bs;
    f->sn[index] = snc;
    long nn = (long)f->n[0] * f->n[1];
    if (p->ndim == 3) {
        f->vx[index] = v2;
        f->vx[nn + index] = v3;
        f->sx[index] = out->s12;
        f->sx[nn + index] = out->s13;
    } else if (p->mode == 2) {
        f->vx[index] = v2;
        f->sx[index] = out->s12;
    } else {
        f->vx[index] = v3;
        f->sx[index] = out->s13;
    }
    if (f->load_file) {
        out->s12 -= f->s2[index];
        out->s22 -= f->s2[index];
        out->s13 -= f->s3[index];
        out->s23 -= f->s3[index];
    }
    for (int k = 0; k < f->nloads; k++) {
        out->s12 -= pert_get(&f->loads[k], 1, ii, jj, t);
        out->s22 -= pert_get(&f->loads[k], 1, ii, jj, t);
        out->s13 -= pert_get(&f->loads[k], 2, ii, jj, t);
        out->s23 -= pert_get(&f->loads[k], 2, ii, jj, t);
    }
    return 1;
}

/* interface::apply_bcs: src/interface.cpp:573-970 (+ solve_interface variants) */
static int iface_apply(orc_problem *p, iface_t *f, double dt, double t, int no_sat) {
    if (!f->is_friction && no_sat) return 1;
    const int ndim = p->ndim, mode = p->mode;
    const long n0 = p->nxd[0];
    const int *nxd = p->nxd;
    double *F = p->f, *DF = p->df, *S = p->s;
    const double *s0 = p->s0;
    double nn[3] = {0., 0., 0.}, t1[3], t2[3];
    for (int i = f->mlb[0]; i < f->prb[0]; i++)
        for (int j = f->mlb[1]; j < f->prb[1]; j++)
            for (int k = f->mlb[2]; k < f->prb[2]; k++) {
                long i1 = (long)i * nxd[1] + (long)j * nxd[2] + k;
                long i2 = (long)(i + f->delta[0]) * nxd[1] + (long)(j + f->delta[1]) * nxd[2] + k + f->delta[2];
                int ii, jj;
                switch (f->direction) {
                    case 0: ii = j - f->mlb[1]; jj = k - f->mlb[2]; break;
                    case 1: ii = i - f->mlb[0]; jj = k - f->mlb[2]; break;
                    default: ii = i - f->mlb[0]; jj = j - f->mlb[1];
                }
                long ij = (long)ii * f->n[1] + jj;
                double cp1 = f->cp1, cs1 = f->cs1, zp1 = f->zp1, zs1 = f->zs1;
                double cp2 = f->cp2, cs2 = f->cs2, zp2 = f->zp2, zs2 = f->zs2;
                double gamma1 = f->gamma1, gamma2 = f->gamma2;
                if (p->hetmat) {
                    const nodemat_t m1 = node_mat(p, i1), m2 = node_mat(p, i2);
                    cp1 = m1.cp; cs1 = m1.cs; zp1 = m1.zp; zs1 = m1.zs; gamma1 = m1.gamma;
                    cp2 = m2.cp; cs2 = m2.cs; zp2 = m2.zp; zs2 = m2.zs; gamma2 = m2.gamma;
                }
                double h1 = dt * f->dl1[ij], h2 = dt * f->dl2[ij];
                for (int l = 0; l < ndim; l++) nn[l] = f->nx[l][ij];
                switch (f->direction) {
                    case 0:
                        t1[2] = 0.;
                        t1[1] = nn[0] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
                        t1[0] = -nn[1] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
                        break;
                    case 1:
                        t1[2] = 0.;
                        t1[0] = nn[1] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
                        t1[1] = -nn[0] / sqrt(nn[0] * nn[0] + nn[1] * nn[1]);
                        break;
                    default:
                        t1[1] = 0.;
                        t1[0] = nn[2] / sqrt(nn[0] * nn[0] + nn[2] * nn[2]);
                        t1[2] = -nn[0] / sqrt(nn[0] * nn[0] + nn[2] * nn[2]);
                }
                t2[0] = nn[1] * t1[2] - nn[2] * t1[1];
                t2[1] = nn[2] * t1[0] - nn[0] * t1[2];
                t2[2] = nn[0] * t1[1] - nn[1] * t1[0];
                if (f->direction == 1) {
                    t2[0] = -t2[0];
                    t2[1] = -t2[1];
                    t2[2] = -t2[2];
                }
                bf_t b1, b2, br1, br2, bs1, bs2;
                if (ndim == 3) {
                    b1.v1 = F[i1]; b1.v2 = F[n0 + i1]; b1.v3 = F[2 * n0 + i1];
                    b1.s11 = F[3 * n0 + i1] + s0[0]; b1.s12 = F[4 * n0 + i1] + s0[1]; b1.s13 = F[5 * n0 + i1] + s0[2];
                    b1.s22 = F[6 * n0 + i1] + s0[3]; b1.s23 = F[7 * n0 + i1] + s0[4]; b1.s33 = F[8 * n0 + i1] + s0[5];
                    b2.v1 = F[i2]; b2.v2 = F[n0 + i2]; b2.v3 = F[2 * n0 + i2];
                    b2.s11 = F[3 * n0 + i2] + s0[0]; b2.s12 = F[4 * n0 + i2] + s0[1]; b2.s13 = F[5 * n0 + i2] + s0[2];
                    b2.s22 = F[6 * n0 + i2] + s0[3]; b2.s23 = F[7 * n0 + i2] + s0[4]; b2.s33 = F[8 * n0 + i2] + s0[5];
                    if (p->hetstress) {
                        b1.s11 += S[i1]; b1.s12 += S[n0 + i1]; b1.s13 += S[2 * n0 + i1];
                        b1.s22 += S[3 * n0 + i1]; b1.s23 += S[4 * n0 + i1]; b1.s33 += S[5 * n0 + i1];
                        b2.s11 += S[i2]; b2.s12 += S[n0 + i2]; b2.s13 += S[2 * n0 + i2];
                        b2.s22 += S[3 * n0 + i2]; b2.s23 += S[4 * n0 + i2]; b2.s33 += S[5 * n0 + i2];
                    }
                } else if (mode == 2) {
                    b1.v1 = F[i1]; b1.v2 = F[n0 + i1]; b1.v3 = 0.;
                    b1.s11 = F[2 * n0 + i1] + s0[0]; b1.s12 = F[3 * n0 + i1] + s0[1]; b1.s13 = 0.;
                    b1.s22 = F[4 * n0 + i1] + s0[3]; b1.s23 = 0.; b1.s33 = 0.;
                    b2.v1 = F[i2]; b2.v2 = F[n0 + i2]; b2.v3 = 0.;
                    b2.s11 = F[2 * n0 + i2] + s0[0]; b2.s12 = F[3 * n0 + i2] + s0[1]; b2.s13 = 0.;
                    b2.s22 = F[4 * n0 + i2] + s0[3]; b2.s23 = 0.; b2.s33 = 0.;
                    if (p->hetstress) {
                        b1.s11 += S[i1]; b1.s12 += S[n0 + i1]; b1.s22 += S[2 * n0 + i1];
                        b2.s11 += S[i2]; b2.s12 += S[n0 + i2]; b2.s22 += S[2 * n0 + i2];
                    }
                } else {
                    b1.v1 = 0.; b1.v2 = 0.; b1.v3 = F[i1];
                    b1.s11 = s0[0]; b1.s12 = 0.; b1.s13 = F[n0 + i1] + s0[2];
                    b1.s22 = s0[3]; b1.s23 = F[2 * n0 + i1] + s0[4]; b1.s33 = 0.;
                    b2.v1 = 0.; b2.v2 = 0.; b2.v3 = F[i2];
                    b2.s11 = s0[0]; b2.s12 = 0.; b2.s13 = F[n0 + i2] + s0[2];
                    b2.s22 = s0[3]; b2.s23 = F[2 * n0 + i2] + s0[4]; b2.s33 = 0.;
                    if (p->hetstress) {
                        b1.s13 += S[i1]; b1.s23 += S[n0 + i1];
                        b2.s13 += S[i2]; b2.s23 += S[n0 + i2];
                    }
                }
                br1 = rot_xy_nt(b1, nn, t1, t2);
                br2 = rot_xy_nt(b2, nn, t1, t2);
                bs1 = br1;
                bs2 = br2;
                iff_t hat;
                if (!f->is_friction) {
                    solve_locked(br1.v1, br2.v1, br1.s11, br2.s11, zp1, zp2, &hat.v11, &hat.v21, &hat.s11, &hat.s21);
                    solve_locked(br1.v2, br2.v2, br1.s12, br2.s12, zs1, zs2, &hat.v12, &hat.v22, &hat.s12, &hat.s22);
                    solve_locked(br1.v3, br2.v3, br1.s13, br2.s13, zs1, zs2, &hat.v13, &hat.v23, &hat.s13, &hat.s23);
                } else {
                    double pv1, pv2, ps1, ps2;
                    solve_locked(br1.v1, br2.v1, br1.s11, br2.s11, zp1, zp2, &pv1, &pv2, &ps1, &ps2);
                    iff_t in;
                    memset(&in, 0, sizeof in);
                    in.v12 = br1.v2; in.v22 = br2.v2; in.v13 = br1.v3; in.v23 = br2.v3;
                    in.s12 = br1.s12; in.s22 = br2.s12; in.s13 = br1.s13; in.s23 = br2.s13;
                    if (!solve_friction(p, f, &in, ps1, zs1, zs2, ii, jj, t, &hat)) return 0;
                    hat.v11 = pv1; hat.v21 = pv2; hat.s11 = ps1; hat.s21 = ps2;
                }
                if (no_sat) continue;
                br1.v1 -= hat.v11;
                br1.v2 = 0.; br1.v3 = 0.;
                br1.s22 = gamma1 * (br1.s11 - hat.s11);
                br1.s33 = gamma1 * (br1.s11 - hat.s11);
                br1.s11 -= hat.s11;
                br1.s12 = 0.; br1.s13 = 0.; br1.s23 = 0.;
                br2.v1 -= hat.v21;
                br2.v2 = 0.; br2.v3 = 0.;
                br2.s22 = gamma2 * (br2.s11 - hat.s21);
                br2.s33 = gamma2 * (br2.s11 - hat.s21);
                br2.s11 -= hat.s21;
                br2.s12 = 0.; br2.s13 = 0.; br2.s23 = 0.;
                b1 = rot_nt_xy(br1, nn, t1, t2);
                b2 = rot_nt_xy(br2, nn, t1, t2);
                if (ndim == 3) {
                    DF[i1] -= cp1 * h1 * b1.v1; DF[n0 + i1] -= cp1 * h1 * b1.v2; DF[2 * n0 + i1] -= cp1 * h1 * b1.v3;
                    DF[3 * n0 + i1] -= cp1 * h1 * b1.s11; DF[4 * n0 + i1] -= cp1 * h1 * b1.s12; DF[5 * n0 + i1] -= cp1 * h1 * b1.s13;
                    DF[6 * n0 + i1] -= cp1 * h1 * b1.s22; DF[7 * n0 + i1] -= cp1 * h1 * b1.s23; DF[8 * n0 + i1] -= cp1 * h1 * b1.s33;
                    DF[i2] -= cp2 * h2 * b2.v1; DF[n0 + i2] -= cp2 * h2 * b2.v2; DF[2 * n0 + i2] -= cp2 * h2 * b2.v3;
                    DF[3 * n0 + i2] -= cp2 * h2 * b2.s11; DF[4 * n0 + i2] -= cp2 * h2 * b2.s12; DF[5 * n0 + i2] -= cp2 * h2 * b2.s13;
                    DF[6 * n0 + i2] -= cp2 * h2 * b2.s22; DF[7 * n0 + i2] -= cp2 * h2 * b2.s23; DF[8 * n0 + i2] -= cp2 * h2 * b2.s33;
                } else if (mode == 2) {
                    DF[i1] -= cp1 * h1 * b1.v1; DF[n0 + i1] -= cp1 * h1 * b1.v2; DF[2 * n0 + i1] -= cp1 * h1 * b1.s11;
                    DF[3 * n0 + i1] -= cp1 * h1 * b1.s12; DF[4 * n0 + i1] -= cp1 * h1 * b1.s22;
                    if (p->is_plastic) DF[5 * n0 + i1] -= cp1 * h1 * b1.s33;
                    DF[i2] -= cp2 * h2 * b2.v1; DF[n0 + i2] -= cp2 * h2 * b2.v2; DF[2 * n0 + i2] -= cp2 * h2 * b2.s11;
                    DF[3 * n0 + i2] -= cp2 * h2 * b2.s12; DF[4 * n0 + i2] -= cp2 * h2 * b2.s22;
                    if (p->is_plastic) DF[5 * n0 + i2] -= cp2 * h2 * b2.s33;
                }
                bs1.v1 = 0.; bs1.v2 -= hat.v12; bs1.v3 -= hat.v13;
                bs1.s11 = 0.; bs1.s12 -= hat.s12; bs1.s13 -= hat.s13;
                bs1.s22 = 0.; bs1.s23 = 0.; bs1.s33 = 0.;
                bs2.v1 = 0.; bs2.v2 -= hat.v22; bs2.v3 -= hat.v23;
                bs2.s11 = 0.; bs2.s12 -= hat.s22; bs2.s13 -= hat.s23;
                bs2.s22 = 0.; bs2.s23 = 0.; bs2.s33 = 0.;
                b1 = rot_nt_xy(bs1, nn, t1, t2);
                b2 = rot_nt_xy(bs2, nn, t1, t2);
                if (ndim == 3) {
                    DF[i1] -= cs1 * h1 * b1.v1; DF[n0 + i1] -= cs1 * h1 * b1.v2; DF[2 * n0 + i1] -= cs1 * h1 * b1.v3;
                    DF[3 * n0 + i1] -= cs1 * h1 * b1.s11; DF[4 * n0 + i1] -= cs1 * h1 * b1.s12; DF[5 * n0 + i1] -= cs1 * h1 * b1.s13;
                    DF[6 * n0 + i1] -= cs1 * h1 * b1.s22; DF[7 * n0 + i1] -= cs1 * h1 * b1.s23; DF[8 * n0 + i1] -= cs1 * h1 * b1.s33;
                    DF[i2] -= cs2 * h2 * b2.v1; DF[n0 + i2] -= cs2 * h2 * b2.v2; DF[2 * n0 + i2] -= cs2 * h2 * b2.v3;
                    DF[3 * n0 + i2] -= cs2 * h2 * b2.s11; DF[4 * n0 + i2] -= cs2 * h2 * b2.s12; DF[5 * n0 + i2] -= cs2 * h2 * b2.s13;
                    DF[6 * n0 + i2] -= cs2 * h2 * b2.s22; DF[7 * n0 + i2] -= cs2 * h2 * b2.s23; DF[8 * n0 + i2] -= cs2 * h2 * b2.s33;
                } else if (mode == 2) {
                    DF[i1] -= cs1 * h1 * b1.v1; DF[n0 + i1] -= cs1 * h1 * b1.v2; DF[2 * n0 + i1] -= cs1 * h1 * b1.s11;
                    DF[3 * n0 + i1] -= cs1 * h1 * b1.s12; DF[4 * n0 + i1] -= cs1 * h1 * b1.s22;
                    DF[i2] -= cs2 * h2 * b2.v1; DF[n0 + i2] -= cs2 * h2 * b2.v2; DF[2 * n0 + i2] -= cs2 * h2 * b2.s11;
                    DF[3 * n0 + i2] -= cs2 * h2 * b2.s12; DF[4 * n0 + i2] -= cs2 * h2 * b2.s22;
                } else {
                    DF[i1] -= cs1 * h1 * b1.v3; DF[n0 + i1] -= cs1 * h1 * b1.s13; DF[2 * n0 + i1] -= cs1 * h1 * b1.s23;
                    DF[i2] -= cs2 * h2 * b2.v3; DF[n0 + i2] -= cs2 * h2 * b2.s13; DF[2 * n0 + i2] -= cs2 * h2 * b2.s23;
                }
            }
    return 1;
}

/* friction::scale_df / calc_df / update: src/friction.cpp:444-505.  The
 * reference's state scale loop runs over (ndim-1)*n entries of an n-entry
 * array (friction.cpp:459-461); only the first n entries hold state, so the
 * restatement scales those. */
static void iface_scale(orc_problem *p, iface_t *f, double A) {
    if (!f->is_friction) return;
    long nn = (long)f->n[0] * f->n[1];
    for (long i = 0; i < (p->ndim - 1) * nn; i++) f->dux[i] *= A;
    for (long i = 0; i < nn; i++) f->du[i] *= A;
    if (!f->has_state) return;
    for (long i = 0; i < nn; i++) f->dstate[i] *= A;
}
static void iface_calc_df(orc_problem *p, iface_t *f, double dt) {
    if (!f->is_friction) return;
    long nn = (long)f->n[0] * f->n[1];
    for (long i = 0; i < (p->ndim - 1) * nn; i++) f->dux[i] += dt * f->vx[i];
    for (long i = 0; i < nn; i++) f->du[i] += dt * f->v[i];
    if (!f->has_state) return;
    for (long i = 0; i < nn; i++) f->dstate[i] += dt * f->dstatedt[i];
}
static void iface_update(orc_problem *p, iface_t *f, double B) {
    if (!f->is_friction) return;
    long nn = (long)f->n[0] * f->n[1];
    for (long i = 0; i < (p->ndim - 1) * nn; i++) f->ux[i] += B * f->dux[i];
    for (long i = 0; i < nn; i++) f->u[i] += B * f->du[i];
    if (!f->has_state) return;
    for (long i = 0; i < nn; i++) f->state[i] += B * f->dstate[i];
}

/* ------------------------------------------------------------------------- */
/* plasticity: src/block.cpp:442-697 */

typedef struct {
    double sxx, sxy, sxz, syy, syz, szz, gammap, lambda, epxx, epxy, epxz, epyy, epyz, epzz;
} plastp;

static plastp plastic_flow(const block_t *b, double dt, plastp in, double k, double g) {
    double sigma = (in.sxx + in.syy + in.szz) / 3.;
    double tau = sqrt(((in.sxx - in.syy) * (in.sxx - in.syy) + (in.syy - in.szz) * (in.syy - in.szz) +
                       (in.szz - in.sxx) * (in.szz - in.sxx)) / 6. +
                      in.sxy * in.sxy + in.sxz * in.sxz + in.syz * in.syz);
    double yf = b->coh - b->mu * sigma;
    if (yf < 0.) yf = 0.;
    double y = tau - yf;
    plastp out;
    double sd[6];
    if (y <= 0.) {
        out = in;
        out.lambda = 0.;
    } else {
        if (tau * b->mu * b->beta * k > (b->mu * sigma - b->coh) * g)
            out.lambda = (tau + b->mu * sigma - b->coh) / (b->eta + dt * (g + b->mu * b->beta * k));
        else
            out.lambda = tau / (b->eta + dt * g);
        out.gammap = in.gammap + dt * out.lambda;
        sd[0] = in.sxx - sigma; sd[1] = in.sxy; sd[2] = in.sxz;
        sd[3] = in.syy - sigma; sd[4] = in.syz; sd[5] = in.szz - sigma;
        tau -= dt * out.lambda * g;
        sigma -= dt * out.lambda * b->beta * k;
        for (int i = 0; i < 6; i++) sd[i] *= tau / (tau + dt * out.lambda * g);
        out.sxx = sd[0] + sigma; out.sxy = sd[1]; out.sxz = sd[2];
        out.syy = sd[3] + sigma; out.syz = sd[4]; out.szz = sd[5] + sigma;
        out.epxx = in.epxx + dt * out.lambda * (sd[0] / (2. * tau) + (b->beta / 3.));
        out.epxy = in.epxy + dt * out.lambda * (sd[1] / (2. * tau));
        out.epxz = in.epxz + dt * out.lambda * (sd[2] / (2. * tau));
        out.epyy = in.epyy + dt * out.lambda * (sd[3] / (2. * tau) + (b->beta / 3.));
        out.epyz = in.epyz + dt * out.lambda * (sd[4] / (2. * tau));
        out.epzz = in.epzz + dt * out.lambda * (sd[5] / (2. * tau) + (b->beta / 3.));
    }
    return out;
}

/* block::calc_plastic, src/block.cpp:442-589.  Its loops declare `double k`
   and then an `int k` loop index over z, so the bulk modulus it assigns
   (k = lambda + 2/3 G, lines 519-524) lands in the loop index: the modulus
   passed to plastic_flow is truncated to an integer, and the z loop continues
   from that integer + 1.  A column therefore visits its first node, then
   trunc(K) + 1 and so on; the reference only finishes when every column
   leaves the block this way (in 2D always, in 3D normally after the first z
   node).  This follows that control flow node by node and reports the
   columns where the reference would loop for ever. */
static int calc_plastic(orc_problem *p, block_t *b, double dt) {
    const long n0 = p->nxd[0];
    double *F = p->f;
    const int pt = p->plastic_tensor;
    int st, o;
    if (p->ndim == 3) { st = 3; o = 9; } else if (p->mode == 2) { st = 2; o = 6; } else { st = 1; o = 3; }
    for (int i = b->mlb[0]; i < b->prb[0]; i++)
        for (int j = b->mlb[1]; j < b->prb[1]; j++) {
            int visits = 0;
            for (int kk = b->mlb[2]; kk < b->prb[2]; kk++) {
                if (++visits > p->nx[2] + 1) {
                    snprintf(p->err, sizeof p->err,
                             "the reference's plastic update does not terminate at column (%d, %d) of a block", i, j);
                    return 0;
                }
                long id = (long)i * p->nxd[1] + (long)j * p->nxd[2] + kk;
                double kb = b->lam + 2. / 3. * b->g, g = b->g;
                if (p->hetmat) { /* block.cpp:519-521 */
                    kb = p->mat[n0 + id] + 2. / 3. * p->mat[2 * n0 + id];
                    g = p->mat[2 * n0 + id];
                }
                if (!(kb < 2147483647.)) {
                    snprintf(p->err, sizeof p->err, "bulk modulus out of the range of the reference's int loop index");
                    return 0;
                }
                const int kint = (int)kb;
                const double k = (double)kint;
                plastp in;
                memset(&in, 0, sizeof in);
                if (p->ndim == 3) {
                    in.sxx = F[3 * n0 + id]; in.sxy = F[4 * n0 + id]; in.sxz = F[5 * n0 + id];
                    in.syy = F[6 * n0 + id]; in.syz = F[7 * n0 + id]; in.szz = F[8 * n0 + id];
                } else if (p->mode == 2) {
                    in.sxx = F[2 * n0 + id]; in.sxy = F[3 * n0 + id]; in.sxz = 0.;
                    in.syy = F[4 * n0 + id]; in.syz = 0.; in.szz = F[5 * n0 + id];
                } else {
                    in.sxx = p->s0[0]; in.sxy = 0.; in.sxz = F[n0 + id];
                    in.syy = p->s0[3]; in.syz = F[2 * n0 + id]; in.szz = p->s0[5];
                }
                in.lambda = F[o * n0 + id];
                in.gammap = F[(o + 1) * n0 + id];
                if (pt) {
                    in.epxx = F[(o + 2) * n0 + id]; in.epxy = F[(o + 3) * n0 + id]; in.epxz = F[(o + 4) * n0 + id];
                    in.epyy = F[(o + 5) * n0 + id]; in.epyz = F[(o + 6) * n0 + id]; in.epzz = F[(o + 7) * n0 + id];
                }
                plastp out = plastic_flow(b, dt, in, k, g);
                if (p->ndim == 3) {
                    F[3 * n0 + id] = out.sxx; F[4 * n0 + id] = out.sxy; F[5 * n0 + id] = out.sxz;
                    F[6 * n0 + id] = out.syy; F[7 * n0 + id] = out.syz; F[8 * n0 + id] = out.szz;
                } else if (p->mode == 2) {
                    F[2 * n0 + id] = out.sxx; F[3 * n0 + id] = out.sxy; F[4 * n0 + id] = out.syy; F[5 * n0 + id] = out.szz;
                } else {
                    F[n0 + id] = out.sxz; F[2 * n0 + id] = out.syz;
                }
                F[o * n0 + id] = out.lambda;
                F[(o + 1) * n0 + id] = out.gammap;
                if (pt) {
                    F[(o + 2) * n0 + id] = out.epxx; F[(o + 3) * n0 + id] = out.epxy; F[(o + 4) * n0 + id] = out.epxz;
                    F[(o + 5) * n0 + id] = out.epyy; F[(o + 6) * n0 + id] = out.epyz; F[(o + 7) * n0 + id] = out.epzz;
                }
                (void)st;
                kk = kint;
            }
        }
    return 1;
}

/* fields::set_stress / remove_stress: src/fields.cpp:184-220 */
void orc_set_stress(orc_problem *p) {
    long n = p->nxyz;
    for (int i = 0; i < p->ns; i++)
        for (long j = 0; j < n; j++) p->f[(p->nv + i) * n + j] += p->s0[p->index[i]];
    if (!p->hetstress) return;
    for (int i = 0; i < p->ns; i++)
        for (long j = 0; j < n; j++) p->f[(p->nv + i) * n + j] += p->s[i * n + j];
}
void orc_remove_stress(orc_problem *p) {
    long n = p->nxyz;
    for (int i = 0; i < p->ns; i++)
        for (long j = 0; j < n; j++) p->f[(p->nv + i) * n + j] -= p->s0[p->index[i]];
    if (!p->hetstress) return;
    for (int i = 0; i < p->ns; i++)
        for (long j = 0; j < n; j++) p->f[(p->nv + i) * n + j] -= p->s[i * n + j];
}

/* ------------------------------------------------------------------------- */
/* domain::do_rk_stage: src/domain.cpp:228-305 */

int orc_do_rk_stage(orc_problem *p, double dt, int stage, double t) {
    double A = p->A[stage], B = p->B[stage];
    long ndf = (long)p->nfields * p->nxyz;
    for (long i = 0; i < ndf; i++) p->df[i] *= A;
    for (int i = 0; i < p->nifaces; i++) iface_scale(p, &p->ifaces[i], A);
    for (int b = 0; b < p->nbt; b++) {
        calc_df(p, &p->blocks[b], dt);
        for (int l = 0; l < 2 * p->ndim; l++) apply_bound(p, &p->blocks[b], &p->blocks[b].bound[l], dt);
    }
    double tc = t + p->C[stage] * dt;
    for (int i = 0; i < p->nifaces; i++)
        if (!iface_apply(p, &p->ifaces[i], dt, tc, 0)) return 2;
    for (int i = 0; i < p->nifaces; i++) iface_calc_df(p, &p->ifaces[i], dt);
    for (int i = 0; i < p->nifaces; i++) iface_update(p, &p->ifaces[i], B);
    for (long i = 0; i < ndf; i++) p->f[i] += B * p->df[i];
    if (stage + 1 == p->nstages && p->is_plastic) {
        orc_set_stress(p);
        for (int b = 0; b < p->nbt; b++)
            if (!calc_plastic(p, &p->blocks[b], dt)) return 3;
        orc_remove_stress(p);
        for (int i = 0; i < p->nifaces; i++)
            if (!iface_apply(p, &p->ifaces[i], dt, tc, 1)) return 2;
    }
    return 0;
}

/* front::set_front: src/front.cpp:103-125 (the "U" field never records) */
static void set_front(orc_problem *p, double t) {
    if (!p->front_on) return;
    for (int i = 0; i < p->nifaces; i++) {
        iface_t *f = &p->ifaces[i];
        if (!f->is_friction) continue;
        long nn = (long)f->n[0] * f->n[1];
        for (long m = 0; m < nn; m++)
            if (f->tfront[m] < 0. && p->front_field == 0 && f->v[m] >= p->front_value) f->tfront[m] = t;
    }
}

/* problem::solve inner body for step i: src/problem.cpp:151-168 */
int orc_step(orc_problem *p, int i) {
    for (int st = 0; st < p->nstages; st++) {
        int rc = orc_do_rk_stage(p, p->dt, st, (double)i * p->dt);
        if (rc) return rc;
    }
    /* output happens on absolute stress; the add/subtract round trip is part
     * of the reference's arithmetic on every step (problem.cpp:160-164) */
    orc_set_stress(p);
    orc_remove_stress(p);
    set_front(p, (double)(i + 1) * p->dt);
    return 0;
}

/* absolute value of field component c ((f + s0) + s for stresses), as the
 * reference writes it between set_stress and remove_stress */
void orc_abs_field(const orc_problem *p, int c, double *out) {
    long n = p->nxyz;
    int si = -1;
    for (int i = 0; i < p->ns; i++)
        if (p->nv + i == c) si = i;
    for (long j = 0; j < n; j++) {
        double v = p->f[(long)c * n + j];
        if (si >= 0) {
            v += p->s0[p->index[si]];
            if (p->hetstress) v += p->s[(long)si * n + j];
        }
        out[j] = v;
    }
}

int orc_run(orc_problem *p, int first_step, int nsteps) {
    for (int i = first_step; i < first_step + nsteps; i++) {
        int rc = orc_step(p, i);
        if (rc) return rc;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* loading: problem.cpp:16-84, domain.cpp:19-153, fields.cpp:13-164,
 * block.cpp:22-264, interface.cpp:17-403, friction.cpp:19-227,
 * slipweak.cpp:19-182, stz.cpp:19-232, problem.cpp:94-134 */

static int load_iface(orc_problem *p, int idx) {
    iface_t *f = &p->ifaces[idx];
    char hdr[64], dirs[16];
    rd_t r;
    snprintf(hdr, sizeof hdr, "[fdfault.interface%d]", idx);
    if (!rd_open(&r, p->infile, NULL, hdr)) {
        snprintf(p->err, sizeof p->err, "Error reading interface %d from input file", idx);
        return 0;
    }
    int i1[3], i2[3];
    rd_str(&r, dirs, sizeof dirs);
    for (int i = 0; i < 3; i++) i1[i] = rd_int(&r);
    for (int i = 0; i < 3; i++) i2[i] = rd_int(&r);
    rd_close(&r);
    f->direction = (!strcmp(dirs, "x")) ? 0 : ((!strcmp(dirs, "y")) ? 1 : 2);
    int D = f->direction;
    for (int i = 0; i < 3; i++)
        if (i2[i] != i1[i] + (i == D ? 1 : 0)) {
            snprintf(p->err, sizeof p->err, "interface %d joins non-adjacent blocks", idx);
            return 0;
        }
    f->b1 = (i1[0] * p->nblocks[1] + i1[1]) * p->nblocks[2] + i1[2];
    f->b2 = (i2[0] * p->nblocks[1] + i2[1]) * p->nblocks[2] + i2[2];
    block_t *b1 = &p->blocks[f->b1], *b2 = &p->blocks[f->b2];
    int oth[2];
    if (D == 0) { oth[0] = 1; oth[1] = 2; } else if (D == 1) { oth[0] = 0; oth[1] = 2; } else { oth[0] = 0; oth[1] = 1; }
    f->n[0] = b1->nx[oth[0]];
    f->n[1] = b2->nx[oth[1]];
    for (int i = 0; i < 3; i++) {
        f->xm[i] = b2->xm[i];
        f->xp[i] = b2->xm[i] + b2->nx[i] - 1;
        f->mlb[i] = b1->mlb[i];
        f->delta[i] = (i == D) ? 1 : 0;
    }
    f->xp[D] = b2->xm[D];
    f->mlb[D] = b1->mlb[D] + b1->nx[D] - 1;
    f->prb[D] = f->mlb[D] + 1;
    f->prb[oth[0]] = f->mlb[oth[0]] + f->n[0];
    f->prb[oth[1]] = f->mlb[oth[1]] + f->n[1];
    /* edge check: interface.cpp:331-347 */
    const int *nxd = p->nxd;
    for (int l = 0; l < p->ndim; l++)
        for (int a = f->mlb[0]; a < f->prb[0]; a++)
            for (int b = f->mlb[1]; b < f->prb[1]; b++)
                for (int c = f->mlb[2]; c < f->prb[2]; c++) {
                    double va = p->x[(long)l * nxd[0] + (long)a * nxd[1] + (long)b * nxd[2] + c];
                    double vb = p->x[(long)l * nxd[0] + (long)(a + f->delta[0]) * nxd[1] + (long)(b + f->delta[1]) * nxd[2] + c + f->delta[2]];
                    if (!(fabs(va - vb) <= (1.e-8 + 1.e-5 * fabs(vb)))) {
                        snprintf(p->err, sizeof p->err, "interface %d block edges do not match", idx);
                        return 0;
                    }
                }
    f->cp1 = mat_cp(b1); f->cs1 = mat_cs(b1); f->zp1 = b1->rho * f->cp1; f->zs1 = b1->rho * f->cs1;
    f->cp2 = mat_cp(b2); f->cs2 = mat_cs(b2); f->zp2 = b2->rho * f->cp2; f->zs2 = b2->rho * f->cs2;
    f->gamma1 = 1. - 2. * ((f->cs1 / f->cp1) * (f->cs1 / f->cp1));
    f->gamma2 = 1. - 2. * ((f->cs2 / f->cp2) * (f->cs2 / f->cp2));
    for (int i = 0; i < 3; i++) {
        f->xb[i] = b1->xb[i];
        f->lb[i] = b1->lb[i];
    }
    /* normals: interface.cpp:414-534 */
    long nn = (long)f->n[0] * f->n[1];
    for (int k = 0; k < p->ndim; k++) f->nx[k] = zalloc(nn);
    f->dl1 = zalloc(nn);
    f->dl2 = zalloc(nn);
    for (int i = 0; i < f->n[0]; i++)
        for (int j = 0; j < f->n[1]; j++) {
            int pos[3];
            pos[D] = f->mlb[D];
            pos[oth[0]] = i + f->mlb[oth[0]];
            pos[oth[1]] = j + f->mlb[oth[1]];
            long id1 = (long)pos[0] * nxd[1] + (long)pos[1] * nxd[2] + pos[2];
            long id2 = id1 + ((D == 0) ? nxd[1] : ((D == 1) ? nxd[2] : 1));
            long ij = (long)i * f->n[1] + j;
            double dl = 0.;
            for (int k = 0; k < p->ndim; k++) {
                double m = p->metric[(long)D * p->ndim * nxd[0] + (long)k * nxd[0] + id1];
                dl += m * m;
                f->nx[k][ij] = m;
            }
            dl = sqrt(dl);
            for (int k = 0; k < p->ndim; k++) f->nx[k][ij] /= dl;
            f->dl1[ij] = dl / (p->h0 * b1->dx[D]);
            dl = 0.;
            for (int k = 0; k < p->ndim; k++) {
                double m = p->metric[(long)D * p->ndim * nxd[0] + (long)k * nxd[0] + id2];
                dl += m * m;
            }
            dl = sqrt(dl);
            f->dl2[ij] = dl / (p->h0 * b2->dx[D]);
        }
    const char *ty = p->iftype[idx];
    f->kind = (!strcmp(ty, "locked")) ? 0 : (!strcmp(ty, "frictionless")) ? 1 : (!strcmp(ty, "slipweak")) ? 2 : (!strcmp(ty, "stz")) ? 3 : -1;
    if (f->kind < 0) {
        snprintf(p->err, sizeof p->err, "unknown interface type %s", ty);
        return 0;
    }
    f->is_friction = f->kind >= 1;
    f->has_state = f->kind == 3;
    if (!f->is_friction) return 1;
    f->u = zalloc(nn); f->du = zalloc(nn); f->v = zalloc(nn); f->s = zalloc(nn); f->sn = zalloc(nn);
    f->ux = zalloc((p->ndim - 1) * nn); f->dux = zalloc((p->ndim - 1) * nn);
    f->vx = zalloc((p->ndim - 1) * nn); f->sx = zalloc((p->ndim - 1) * nn);
    f->tfront = zalloc(nn);
    for (long m = 0; m < nn; m++) f->tfront[m] = -1.;
    /* fault-plane coordinate mapping for perturbations: friction.cpp:131-176 */
    double x2[2], l2[2];
    int xm2[2], xml2[2];
    x2[0] = f->xb[oth[0]]; x2[1] = f->xb[oth[1]];
    l2[0] = f->lb[oth[0]]; l2[1] = f->lb[oth[1]];
    xm2[0] = f->xm[oth[0]]; xm2[1] = f->xm[oth[1]];
    xml2[0] = xm2[0]; xml2[1] = xm2[1];
    char tok[PATHLEN];
    if (!rd_open(&r, p->infile, hdr, "[fdfault.friction]")) {
        snprintf(p->err, sizeof p->err, "Error reading interface %d friction", idx);
        return 0;
    }
    f->nloads = rd_int(&r);
    if (f->nloads > MAXP) return 0;
    for (int i = 0; i < f->nloads; i++) {
        pert_t *q = &f->loads[i];
        rd_str(&r, tok, sizeof tok);
        q->type = pert_type(tok);
        q->t0 = rd_dbl(&r); q->x0 = rd_dbl(&r); q->dx = rd_dbl(&r); q->y0 = rd_dbl(&r); q->dy = rd_dbl(&r);
        q->val[0] = rd_dbl(&r); q->val[1] = rd_dbl(&r); q->val[2] = rd_dbl(&r);
        if (p->ndim == 2 && p->mode == 2) q->val[2] = 0.;
        else if (p->ndim == 2 && p->mode == 3) q->val[1] = 0.;
        pert_init(q, f->n, xm2, xml2, x2, l2);
    }
    rd_str(&r, tok, sizeof tok);
    rd_close(&r);
    if (strcmp(tok, "none") != 0) {
        f->load_file = 1;
        f->s1 = zalloc(nn); f->s2 = zalloc(nn); f->s3 = zalloc(nn);
        if (!read_doubles(tok, f->s1, nn, 0) || !read_doubles(tok, f->s2, nn, nn) || !read_doubles(tok, f->s3, nn, 2 * nn)) {
            snprintf(p->err, sizeof p->err, "Error opening load file %s", tok);
            return 0;
        }
        if (p->ndim == 2 && p->mode == 2) for (long m = 0; m < nn; m++) f->s3[m] = 0.;
        else if (p->ndim == 2 && p->mode == 3) for (long m = 0; m < nn; m++) f->s2[m] = 0.;
    }
    if (f->kind == 2) {
        if (!rd_open(&r, p->infile, hdr, "[fdfault.slipweak]")) {
            snprintf(p->err, sizeof p->err, "Error reading slipweak from input file");
            return 0;
        }
        f->nperts = rd_int(&r);
        if (f->nperts > MAXP) return 0;
        for (int i = 0; i < f->nperts; i++) {
            pert_t *q = &f->perts[i];
            rd_str(&r, tok, sizeof tok);
            q->type = pert_type(tok);
            q->t0 = rd_dbl(&r); q->x0 = rd_dbl(&r); q->dx = rd_dbl(&r); q->y0 = rd_dbl(&r); q->dy = rd_dbl(&r);
            for (int k = 0; k < 6; k++) q->val[k] = rd_dbl(&r);
            pert_init(q, f->n, xm2, xml2, x2, l2);
        }
        rd_str(&r, tok, sizeof tok);
        rd_close(&r);
        if (strcmp(tok, "none") != 0) {
            f->param_file = 1;
            for (int k = 0; k < 6; k++) {
                f->par[k] = zalloc(nn);
                if (!read_doubles(tok, f->par[k], nn, k * nn)) {
                    snprintf(p->err, sizeof p->err, "Error opening parameter file %s", tok);
                    return 0;
                }
            }
        }
    } else if (f->kind == 3) {
        if (!rd_open(&r, p->infile, hdr, "[fdfault.stz]")) {
            snprintf(p->err, sizeof p->err, "Error reading stz from input file");
            return 0;
        }
        double chi0 = rd_dbl(&r);
        char statefile[PATHLEN];
        rd_str(&r, statefile, sizeof statefile);
        f->nperts = rd_int(&r);
        if (f->nperts > MAXP) return 0;
        for (int i = 0; i < f->nperts; i++) {
            pert_t *q = &f->perts[i];
            rd_str(&r, tok, sizeof tok);
            q->type = pert_type(tok);
            q->t0 = rd_dbl(&r); q->x0 = rd_dbl(&r); q->dx = rd_dbl(&r); q->y0 = rd_dbl(&r); q->dy = rd_dbl(&r);
            for (int k = 0; k < 9; k++) q->val[k] = rd_dbl(&r);
            pert_init(q, f->n, xm2, xml2, x2, l2);
        }
        rd_str(&r, tok, sizeof tok);
        rd_close(&r);
        f->state = zalloc(nn); f->dstate = zalloc(nn); f->dstatedt = zalloc(nn);
        if (strcmp(statefile, "none") != 0) {
            if (!read_doubles(statefile, f->state, nn, 0)) {
                snprintf(p->err, sizeof p->err, "Error opening state file %s", statefile);
                return 0;
            }
        }
        for (long m = 0; m < nn; m++) f->state[m] += chi0;
        if (strcmp(tok, "none") != 0) {
            f->param_file = 1;
            for (int k = 0; k < 9; k++) {
                f->par[k] = zalloc(nn);
                if (!read_doubles(tok, f->par[k], nn, k * nn)) {
                    snprintf(p->err, sizeof p->err, "Error opening parameter file %s", tok);
                    return 0;
                }
            }
        }
    }
    return 1;
}

static int load_all(orc_problem *p) {
    rd_t r;
    char tok[PATHLEN];
    if (!rd_open(&r, p->infile, NULL, "[fdfault.problem]")) {
        snprintf(p->err, sizeof p->err, "Error reading problem from input file");
        return 0;
    }
    rd_str(&r, p->name, sizeof p->name);
    rd_str(&r, p->datadir, sizeof p->datadir);
    p->nt = rd_int(&r);
    p->dt = rd_dbl(&r);
    p->ttot = rd_dbl(&r);
    p->cfl = rd_dbl(&r);
    p->ninfo = rd_int(&r);
    p->rkorder = rd_int(&r);
    rd_close(&r);
    if (!set_rk(p)) {
        snprintf(p->err, sizeof p->err, "Error in initializing RK method");
        return 0;
    }
    if (!rd_open(&r, p->infile, NULL, "[fdfault.domain]")) {
        snprintf(p->err, sizeof p->err, "Error reading domain from input file");
        return 0;
    }
    p->ndim = rd_int(&r);
    p->mode = rd_int(&r);
    for (int i = 0; i < 3; i++) p->nx[i] = rd_int(&r);
    for (int i = 0; i < 3; i++) p->nblocks[i] = rd_int(&r);
    for (int i = 0; i < 3; i++) {
        p->nx_block[i] = (int *)calloc((size_t)p->nblocks[i], sizeof(int));
        p->xm_block[i] = (int *)calloc((size_t)p->nblocks[i], sizeof(int));
        for (int j = 0; j < p->nblocks[i]; j++) p->nx_block[i][j] = rd_int(&r);
    }
    p->nifaces = rd_int(&r);
    if (p->nifaces > MAXI) return 0;
    for (int i = 0; i < p->nifaces; i++) rd_str(&r, p->iftype[i], sizeof p->iftype[i]);
    p->sbporder = rd_int(&r);
    rd_str(&r, p->material, sizeof p->material);
    rd_close(&r);
    if (p->sbporder < 2 || p->sbporder > 4) {
        snprintf(p->err, sizeof p->err, "sbporder must be 2, 3 or 4");
        return 0;
    }
    p->is_plastic = !strcmp(p->material, "plastic");
    for (int i = 0; i < 3; i++) {
        int sum = 0;
        for (int j = 0; j < p->nblocks[i]; j++) {
            p->xm_block[i][j] = sum;
            sum += p->nx_block[i][j];
        }
        if (sum != p->nx[i]) {
            snprintf(p->err, sizeof p->err, "block sizes do not sum to domain size");
            return 0;
        }
    }
    set_fd(p);
    /* fields: fields.cpp:13-164 */
    if (!rd_open(&r, p->infile, NULL, "[fdfault.fields]")) {
        snprintf(p->err, sizeof p->err, "Error reading fields from input file");
        return 0;
    }
    for (int i = 0; i < 6; i++) p->s0[i] = rd_dbl(&r);
    rd_str(&r, p->loadfile, sizeof p->loadfile);
    rd_str(&r, p->matfile, sizeof p->matfile);
    p->plastic_tensor = rd_int(&r);
    rd_close(&r);
    if (strcmp(p->matfile, "none") != 0 && p->ndim == 2 && p->mode == 3) {
        /* the reference's time step reads a third material array that mode III
           does not have (block.cpp:387-388, fields.cpp:58-61) */
        snprintf(p->err, sizeof p->err, "heterogeneous material files are not supported for mode III");
        return 0;
    }
    int nfields, nfieldsp;
    if (p->ndim == 3) nfields = 9; else if (p->mode == 2) nfields = 5; else nfields = 3;
    if (!p->is_plastic) nfieldsp = 0;
    else {
        nfieldsp = p->plastic_tensor ? 8 : 2;
        if (p->ndim == 2 && p->mode == 2) nfields = 6;
    }
    p->nfields = nfields;
    p->nfieldsp = nfieldsp;
    p->nxyz = p->nx[0] * p->nx[1] * p->nx[2];
    p->nxd[0] = p->nxyz;
    p->nxd[1] = p->nx[1] * p->nx[2];
    p->nxd[2] = p->nx[2];
    long n = p->nxyz;
    p->f = zalloc((long)(nfields + nfieldsp) * n);
    p->df = zalloc((long)nfields * n);
    p->x = zalloc((long)p->ndim * n);
    p->metric = zalloc((long)p->ndim * p->ndim * n);
    p->jac = zalloc(n);
    if (p->ndim == 3) {
        p->ns = 6; p->nv = 3;
        for (int i = 0; i < 6; i++) p->index[i] = i;
    } else if (p->mode == 2) {
        p->ns = 3; p->nv = 2;
        p->index[0] = 0; p->index[1] = 1; p->index[2] = 3;
        if (p->is_plastic) {
            p->ns = 4;
            p->index[3] = 5;
        }
    } else {
        p->ns = 2; p->nv = 1;
        p->index[0] = 2; p->index[1] = 4;
    }
    if (strcmp(p->loadfile, "none") != 0) {
        p->hetstress = 1;
        p->s = zalloc((long)p->ns * n);
        if (!read_doubles(p->loadfile, p->s, (long)p->ns * n, 0)) {
            snprintf(p->err, sizeof p->err, "Error opening stress file %s", p->loadfile);
            return 0;
        }
    }
    if (strcmp(p->matfile, "none") != 0) {
        p->hetmat = 1;
        p->mat = zalloc(3L * n);
        if (!read_doubles(p->matfile, p->mat, 3L * n, 0)) {
            snprintf(p->err, sizeof p->err, "Error opening material file %s", p->matfile);
            return 0;
        }
        for (long q = 0; q < 3L * n; q++)
            if (!(p->mat[q] > 0.)) { /* fields.cpp:648 */
                snprintf(p->err, sizeof p->err, "material properties must be positive (%s)", p->matfile);
                return 0;
            }
    }
    /* operator: block.cpp:87-107 */
    p->cdiss = 0.;
    if (rd_open(&r, p->infile, NULL, "[fdfault.operator]")) {
        p->cdiss = rd_dbl(&r);
        rd_close(&r);
    }
    p->dissipation = p->cdiss > 0.;
    /* blocks */
    p->nbt = p->nblocks[0] * p->nblocks[1] * p->nblocks[2];
    if (p->nbt > MAXB) return 0;
    p->blocks = (block_t *)calloc((size_t)p->nbt, sizeof(block_t));
    int s = p->sbporder;
    for (int bi = 0; bi < p->nblocks[0]; bi++)
        for (int bj = 0; bj < p->nblocks[1]; bj++)
            for (int bk = 0; bk < p->nblocks[2]; bk++) {
                block_t *b = &p->blocks[(bi * p->nblocks[1] + bj) * p->nblocks[2] + bk];
                b->coords[0] = bi; b->coords[1] = bj; b->coords[2] = bk;
                char hdr[64];
                snprintf(hdr, sizeof hdr, "[fdfault.block%d%d%d]", bi, bj, bk);
                if (!rd_open(&r, p->infile, NULL, hdr)) {
                    snprintf(p->err, sizeof p->err, "Error reading block %d%d%d from input file", bi, bj, bk);
                    return 0;
                }
                b->rho = rd_dbl(&r);
                b->lam = rd_dbl(&r);
                b->g = rd_dbl(&r);
                if (p->is_plastic) {
                    b->mu = rd_dbl(&r);
                    b->coh = rd_dbl(&r);
                    b->beta = rd_dbl(&r);
                    b->eta = rd_dbl(&r);
                }
                for (int i = 0; i < p->ndim; i++) b->xb[i] = rd_dbl(&r);
                for (int i = 0; i < p->ndim; i++) b->lb[i] = rd_dbl(&r);
                for (int i = 0; i < 2 * p->ndim; i++) rd_str(&r, b->btype[i], sizeof b->btype[i]);
                for (int i = 0; i < 2 * p->ndim; i++) rd_str(&r, b->bfile[i], sizeof b->bfile[i]);
                rd_close(&r);
                int coords[3] = {bi, bj, bk};
                for (int i = 0; i < 3; i++) {
                    b->nx[i] = (i < p->ndim) ? p->nx_block[i][coords[i]] : 1;
                    b->xm[i] = (i < p->ndim) ? p->xm_block[i][coords[i]] : 0;
                    if (i < p->ndim && b->nx[i] < 4 * s - 3) {
                        snprintf(p->err, sizeof p->err, "block too small for the SBP operator");
                        return 0;
                    }
                    b->mlb[i] = b->xm[i];
                    if (b->nx[i] > 1) {
                        b->mc[i] = b->mlb[i] + 2 * (s - 1);
                        b->mrb[i] = b->mlb[i] + b->nx[i] - 2 * (s - 1);
                        b->prb[i] = b->mrb[i] + 2 * (s - 1);
                    } else {
                        b->mc[i] = b->mlb[i];
                        b->mrb[i] = b->mlb[i] + b->nx[i];
                        b->prb[i] = b->mrb[i];
                    }
                }
                if (!set_grid(p, b)) return 0;
                for (int l = 0; l < 2 * p->ndim; l++) bound_init(p, b, l);
            }
    for (int i = 0; i < p->nifaces; i++)
        if (!load_iface(p, i)) return 0;
    /* initial interface solve: domain.cpp:141-143 */
    for (int i = 0; i < p->nifaces; i++)
        if (!iface_apply(p, &p->ifaces[i], 0., 0., 1)) return 0;
    /* time step: problem.cpp:94-134 with block.cpp:368-403 */
    double dxmin = 0.;
    for (int bb = 0; bb < p->nbt; bb++) {
        block_t *b = &p->blocks[bb];
        double dxmax = 0.;
        double cs = mat_cs(b);
        for (int i = b->mlb[0]; i < b->prb[0]; i++)
            for (int j = b->mlb[1]; j < b->prb[1]; j++)
                for (int k = b->mlb[2]; k < b->prb[2]; k++) {
                    long id = (long)i * p->nxd[1] + (long)j * p->nxd[2] + k;
                    if (p->hetmat) cs = sqrt(p->mat[2 * n + id] / p->mat[id]);
                    for (int l = 0; l < p->ndim; l++) {
                        double dxt = 0.;
                        for (int m = 0; m < p->ndim; m++) {
                            double mm = p->metric[(long)l * p->ndim * n + (long)m * n + id];
                            dxt += mm * mm;
                        }
                        dxt = cs * sqrt(dxt) / b->dx[l];
                        if (dxt > dxmax) dxmax = dxt;
                    }
                }
        double dxt = 1. / dxmax;
        if (dxt > 1.e-14 && (dxmin <= 1.e-14 || dxt < dxmin)) dxmin = dxt;
    }
    if ((p->ttot > 0. && p->nt > 0) && (p->dt == 0 && p->cfl == 0.)) {
        p->dt = p->ttot / (double)p->nt;
        p->cfl = p->dt / dxmin;
    } else {
        if (p->dt > 0.)
            p->cfl = p->dt / dxmin;
        else
            p->dt = p->cfl * dxmin;
        if (p->ttot > 0.) {
            p->nt = (int)ceil(p->ttot / p->dt);
            p->ttot = (double)p->nt * p->dt;
        } else {
            p->ttot = (double)p->nt * p->dt;
        }
    }
    /* front list: frontlist.cpp:20-67 */
    if (rd_open(&r, p->infile, NULL, "[fdfault.frontlist]")) {
        p->front_on = rd_int(&r);
        if (p->front_on) {
            rd_str(&r, tok, sizeof tok);
            p->front_field = (!strcmp(tok, "V")) ? 0 : 1;
            p->front_value = rd_dbl(&r);
        }
        rd_close(&r);
    }
    /* initial output on absolute stress (problem.cpp:74-78), then the
     * initial front values at t = 0 (problem.cpp:82) */
    orc_set_stress(p);
    orc_remove_stress(p);
    set_front(p, 0.);
    return 1;
}

orc_problem *orc_load(const char *infile, char *err, int errlen) {
    orc_problem *p = (orc_problem *)calloc(1, sizeof(orc_problem));
    if (!p) return NULL;
    snprintf(p->infile, sizeof p->infile, "%s", infile);
    if (!load_all(p)) {
        if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s", p->err[0] ? p->err : "invalid input");
        orc_free(p);
        return NULL;
    }
    return p;
}

void orc_free(orc_problem *p) {
    if (!p) return;
    free(p->f); free(p->df); free(p->x); free(p->metric); free(p->jac); free(p->s); free(p->mat);
    for (int i = 0; i < 3; i++) {
        free(p->nx_block[i]);
        free(p->xm_block[i]);
    }
    if (p->blocks) {
        for (int b = 0; b < p->nbt; b++)
            for (int l = 0; l < 6; l++) {
                for (int k = 0; k < 3; k++) free(p->blocks[b].bound[l].nx[k]);
                free(p->blocks[b].bound[l].dl);
            }
        free(p->blocks);
    }
    for (int i = 0; i < MAXI; i++) {
        iface_t *f = &p->ifaces[i];
        for (int k = 0; k < 3; k++) free(f->nx[k]);
        free(f->dl1); free(f->dl2);
        free(f->u); free(f->du); free(f->v); free(f->s); free(f->sn);
        free(f->ux); free(f->dux); free(f->vx); free(f->sx);
        free(f->state); free(f->dstate); free(f->dstatedt);
        free(f->s1); free(f->s2); free(f->s3); free(f->tfront);
        for (int k = 0; k < 9; k++) free(f->par[k]);
    }
    free(p);
}

void orc_info(const orc_problem *p, int *ints, double *dbls) {
    ints[0] = p->ndim; ints[1] = p->mode; ints[2] = p->nx[0]; ints[3] = p->nx[1]; ints[4] = p->nx[2];
    ints[5] = p->nfields; ints[6] = p->nfieldsp; ints[7] = p->nifaces; ints[8] = p->nstages; ints[9] = p->nt;
    ints[10] = p->sbporder; ints[11] = p->nblocks[0]; ints[12] = p->nblocks[1]; ints[13] = p->nblocks[2];
    ints[14] = p->is_plastic; ints[15] = p->rkorder;
    dbls[0] = p->dt; dbls[1] = p->ttot; dbls[2] = p->cfl;
}

double *orc_field(orc_problem *p, int which) {
    switch (which) {
        case ORC_F: return p->f;
        case ORC_DF: return p->df;
        case ORC_X: return p->x;
        case ORC_METRIC: return p->metric;
        case ORC_JAC: return p->jac;
        case ORC_S: return p->s;
    }
    return NULL;
}

double *orc_fault(orc_problem *p, int iface, int which, int *n0, int *n1) {
    if (iface < 0 || iface >= p->nifaces) return NULL;
    iface_t *f = &p->ifaces[iface];
    *n0 = f->n[0];
    *n1 = f->n[1];
    switch (which) {
        case ORC_U: return f->u;
        case ORC_DU: return f->du;
        case ORC_V: return f->v;
        case ORC_SS: return f->s;
        case ORC_SN: return f->sn;
        case ORC_UX: return f->ux;
        case ORC_DUX: return f->dux;
        case ORC_VX: return f->vx;
        case ORC_SX: return f->sx;
        case ORC_STATE: return f->state;
        case ORC_DSTATE: return f->dstate;
        case ORC_DSTATEDT: return f->dstatedt;
        case ORC_TFRONT: return f->tfront;
    }
    return NULL;
}

int orc_iface_info(const orc_problem *p, int iface, int *ints) {
    if (iface < 0 || iface >= p->nifaces) return -1;
    const iface_t *f = &p->ifaces[iface];
    ints[0] = f->kind; ints[1] = f->direction; ints[2] = f->n[0]; ints[3] = f->n[1];
    for (int i = 0; i < 3; i++) {
        ints[4 + i] = f->mlb[i];
        ints[7 + i] = f->xm[i];
        ints[10 + i] = f->xp[i];
    }
    return 0;
}

const char *orc_last_error(const orc_problem *p) { return p->err; }
