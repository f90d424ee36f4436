/*
 * fdtd_oracle.c -- FP64 CPU restatement of GSvit's stepping loop.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; never part of the product path).
 *
 * Each routine restates one reference routine, cited by file:line of the
 * GSvit sources (src3d/).  The reference's own quirks on this path are kept
 * deliberately, because parity is judged against the reference CPU path:
 *   - CPML psi_E of dispersive (ADE) cells is updated twice per step, once in
 *     the ADE branch of ystep_e (yee.c:950-1057) and once in boundary_estep;
 *   - the x0-face correction inside the ADE branch multiplies by cb == 0
 *     (yee.c:577, yee.c:961-966);
 *   - the z0-face E correction of Ex is gated by ztbc (boundary.c:758-759);
 *   - TSF corrections use the epsilon of the face cell (source.c:566);
 *   - vacuum cells in FULL/ELECTRIC/MAGNETIC matmode take their coefficients
 *     from the float voxel arrays filled with (float)EPSILON_0 / (float)MU_0
 *     (yee.c:107-116).
 * Only the material types LINTAB, ADE and PEC (plus voxel LINEAR data) are on
 * this path; the RC Drude / CP / CP3 / PLRC branches are rejected.
 */
#include "fdtd_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define C0    299792458.0                 /* constants.h:29 */
#define MU0   1.256637061435917295e-6     /* constants.h:31 */
#define EPS0  8.854187817620389850e-12    /* constants.h:32 */
#define PI_D  3.1415926535897932384626433832795028841971693993751

enum { FX0 = 0, FXN, FY0, FYN, FZ0, FZN };

struct oracle_state {
    int xres, yres, zres;
    size_t n;
    double dx, dy, dz, dt;
    int matmode, nmat;
    fdtd_material *mats;
    int32_t *mat;
    double *veps, *vsig, *vmu, *vsigast;
    int32_t *bnds, *sskip;
    double *f[6];                 /* ex ey ez hx hy hz */
    int disp;                     /* ADE arrays allocated */
    double *ep[3], *dp[3], *dpp[3], *p[3][2], *pp[3][2];
    fdtd_cpml_face cp[6];
    double *be[6], *ce[6], *bh[6], *ch[6], *ke[6], *kh[6];
    double *pe[6][2], *ph[6][2];  /* psi slabs, see cpml_alloc() */
    int tsf;
    fdtd_tsf t;
    double *wave;
    double corr;
    int jres;
    double jdx;
    double *je, *jh, *jeps, *jmu;
    double jb[8];                 /* fbnx0_e_0, e_1, h_0, h_1, fbnxn_e_0, e_1, h_0, h_1 */
    int nfff;
    fdtd_nfff ff;
    int32_t *ffpts;
    int32_t *ffistart;
    int ndata;
    double *ffr[6], *ffct[6];     /* per point, per face: r and cos(theta) tables */
    double *ffser;                /* (p*3 + c)*ndata */
    int nprobes;
    int32_t *probes;
    double *probe_out;
    int nsteps_planned;
    int step;
};

#define IDX(s, i, j, k) ((((size_t)(i)) * (size_t)(s)->yres + (size_t)(j)) * (size_t)(s)->zres + (size_t)(k))
#define EX(s) ((s)->f[0])
#define EY(s) ((s)->f[1])
#define EZ(s) ((s)->f[2])
#define HX(s) ((s)->f[3])
#define HY(s) ((s)->f[4])
#define HZ(s) ((s)->f[5])

static int is_tab(int type)   /* the "tabulated material" set of yee.c:220-225 */
{
    return type == FDTD_MAT_LINTAB || type == FDTD_MAT_DRUDE || type == FDTD_MAT_PLRC ||
           type == FDTD_MAT_ADE || type == FDTD_MAT_CP || type == FDTD_MAT_CP3;
}

static int is_disp(int type)  /* the dispersive set of yee.c:469-471 */
{
    return type == FDTD_MAT_DRUDE || type == FDTD_MAT_CP3 || type == FDTD_MAT_CP ||
           type == FDTD_MAT_ADE || type == FDTD_MAT_PLRC;
}

static int matidx(const oracle_state *s, int i, int j, int k)
{
    return s->nmat > 0 ? s->mat[IDX(s, i, j, k)] : -1;
}

/* sv_yee_data_get_epsilon_sigma, yee.c:1318-1350 */
static int get_eps_sig(const oracle_state *s, int i, int j, int k, double *eps, double *sig)
{
    int m = matidx(s, i, j, k);
    double e = EPS0, g = 0;
    if (m > 0 && is_tab(s->mats[m].type)) {
        e = s->mats[m].epsilon;
        g = s->mats[m].sigma;
    } else if (s->veps && s->vsig) {
        size_t c = IDX(s, i, j, k);
        e = s->veps[c];
        g = s->vsig[c];
    }
    *eps = e;
    *sig = g;
    return m;
}

/* sv_yee_data_get_epsilon, yee.c:1266-1289 */
static double get_eps(const oracle_state *s, int i, int j, int k)
{
    int m = matidx(s, i, j, k);
    if (m > 0 && is_tab(s->mats[m].type))
        return s->mats[m].epsilon;
    if (s->matmode == FDTD_MATMODE_FULL || s->matmode == FDTD_MATMODE_ELECTRIC)
        return s->veps[IDX(s, i, j, k)];
    return EPS0;
}

/* sv_yee_data_is_pec, yee.c:1250-1263 */
static int is_pec(const oracle_state *s, int i, int j, int k)
{
    int m = matidx(s, i, j, k);
    return m > 0 && s->mats[m].type == FDTD_MAT_PEC;
}

/* sv_yee_data_get_db, yee.c:1620-1647 */
static double get_db(const oracle_state *s, int i, int j, int k)
{
    int m = matidx(s, i, j, k);
    double dt = s->dt;
    if (m > 0 && is_tab(s->mats[m].type)) {
        const fdtd_material *q = &s->mats[m];
        return (dt / q->mu / s->dx) / (1 + q->sigast * dt / 2 / q->mu);
    }
    if (s->matmode == FDTD_MATMODE_FULL || s->matmode == FDTD_MATMODE_MAGNETIC) {
        size_t c = IDX(s, i, j, k);
        return (dt / s->vmu[c] / s->dx) / (1 + s->vsigast[c] * dt / 2 / s->vmu[c]);
    }
    return dt / MU0 / s->dx;
}

/* sv_yee_data_get_tsf_mattype, yee.c:1686-1707 */
static int tsf_mattype(const oracle_state *s, int i, int j, int k)
{
    int m = matidx(s, i, j, k);
    if (m == 0 || m == -1) {
        if ((s->matmode == FDTD_MATMODE_FULL || s->matmode == FDTD_MATMODE_ELECTRIC) &&
            fabs(1.0 - s->veps[IDX(s, i, j, k)] / EPS0) < 0.001)
            return 0;
        if (s->matmode == FDTD_MATMODE_NONE)
            return 0;
    }
    if (m > 0 && s->mats[m].type == FDTD_MAT_LINTAB && fabs(1.0 - s->mats[m].epsilon / EPS0) < 0.001)
        return 0;
    return 1;
}

/* sv_yee_data_get_tbc, yee.c:454-526: which E components are left for the
 * ordinary update (1) and which are taken by the dispersive branch (0). */
static int get_tbc(const oracle_state *s, int i, int j, int k, int *xt, int *yt, int *zt)
{
    int m;
    *xt = *yt = *zt = 1;
    if (s->nmat <= 0)
        return -1;
    m = s->mat[IDX(s, i, j, k)];
    if (m > 0 && is_disp(s->mats[m].type)) {
        *xt = *yt = *zt = 0;
        return m;
    }
#define NB(ii, jj, kk, cond, act)                                                      \
    if ((cond) && s->mat[IDX(s, ii, jj, kk)] > 0 && is_disp(s->mats[s->mat[IDX(s, ii, jj, kk)]].type)) { \
        m = s->mat[IDX(s, ii, jj, kk)];                                                \
        act;                                                                           \
    }
    NB(i - 1, j, k, i > 0, (*yt = *zt = 0));
    NB(i, j - 1, k, j > 0, (*xt = *zt = 0));
    NB(i, j, k - 1, k > 0, (*xt = *yt = 0));
    NB(i - 1, j - 1, k, i > 0 && j > 0, (*zt = 0));
    NB(i, j - 1, k - 1, j > 0 && k > 0, (*xt = 0));
    NB(i - 1, j, k - 1, i > 0 && k > 0, (*yt = 0));
#undef NB
    return m;
}

/* sv_yee_data_get_cabs, yee.c:1397-1493: per-component ca/cb with the
 * interface averaging of epsilon and sigma over the cells sharing an edge. */
static void get_cabs(const oracle_state *s, int i, int j, int k, double ca[3], double cb[3])
{
    double e, g, ex, ey, ez, gx, gy, gz;
    int nx, ny, nz;
    double dt = s->dt;
    get_eps_sig(s, i, j, k, &e, &g);
    ex = ey = ez = e;
    gx = gy = gz = g;
    if (s->bnds[IDX(s, i, j, k)] > 0) {
        nx = ny = nz = 1;
        if (i > 0) {
            get_eps_sig(s, i - 1, j, k, &e, &g);
            ey += e; gy += g; ez += e; gz += g; ny++; nz++;
        }
        if (j > 0) {
            get_eps_sig(s, i, j - 1, k, &e, &g);
            ex += e; gx += g; ez += e; gz += g; nx++; nz++;
        }
        if (k > 0) {
            get_eps_sig(s, i, j, k - 1, &e, &g);
            ex += e; gx += g; ey += e; gy += g; nx++; ny++;
        }
        if (j > 0 && k > 0) {
            get_eps_sig(s, i, j - 1, k - 1, &e, &g);
            ex += e; gx += g; nx++;
        }
        if (i > 0 && k > 0) {
            get_eps_sig(s, i - 1, j, k - 1, &e, &g);
            ey += e; gy += g; ny++;
        }
        if (i > 0 && j > 0) {
            get_eps_sig(s, i - 1, j - 1, k, &e, &g);
            ez += e; gz += g; nz++;
        }
        ex /= nx; gx /= nx;
        ey /= ny; gy /= ny;
        ez /= nz; gz /= nz;
    }
    ca[0] = (1 - gx * dt / 2 / ex) / (1 + gx * dt / 2 / ex);
    cb[0] = (dt / ex / s->dx) / (1 + gx * dt / 2 / ex);
    if (s->bnds[IDX(s, i, j, k)] > 0 || (s->dx != s->dy || s->dx != s->dz)) {
        ca[1] = (1 - gy * dt / 2 / ey) / (1 + gy * dt / 2 / ey);
        cb[1] = (dt / ey / s->dy) / (1 + gy * dt / 2 / ey);
        ca[2] = (1 - gz * dt / 2 / ez) / (1 + gz * dt / 2 / ez);
        cb[2] = (dt / ez / s->dz) / (1 + gz * dt / 2 / ez);
    } else {
        ca[1] = ca[2] = ca[0];
        cb[1] = cb[2] = cb[0];
    }
}

/* ---------------------------------------------------------------- set-up */

/* CPML grading, becebhch0 / becebhch of boundary.c:34-99.  `pos` is the
 * grading position (i for the 0-faces, depth-i for the n-faces) and hsign the
 * half-cell offset of the H samples (-0.5 on 0-faces, +0.5 on n-faces). */
static void cpml_grade(int pos, int imax, double sigma, double kappa, double a, int m, double dt,
                       double hsign, double *be, double *ce, double *bh, double *ch, double *ke, double *kh)
{
    double pe = pow((imax - pos) / (double)(imax - 0), m);
    double phh = pow((imax - pos - hsign) / (double)(imax - 0), m);
    double sve = sigma * pe, kve = 1 + (kappa - 1) * pe, ave = a * pow(((pos - 0) / ((double)imax - 0)), 1);
    double svh = sigma * phh, kvh = 1 + (kappa - 1) * phh, avh = a * pow(((pos - hsign) / ((double)imax - 0)), 1);
    *be = exp(-(sve / kve + ave) * dt / EPS0);
    *ce = (sve == 0) ? 0 : (sve / (sve + kve * ave) / kve) * ((*be) - 1.0);
    *bh = exp(-(svh / kvh + avh) * dt / EPS0);
    *ch = (svh == 0) ? 0 : (svh / (svh + kvh * avh) / kvh) * ((*bh) - 1.0);
    *ke = kve;
    *kh = kvh;
}

/* slab of face f: x faces [d][yres][zres], y faces [xres][d][zres],
 * z faces [xres][yres][d]  (boundary.c:102-280) */
static size_t slab_idx(const oracle_state *s, int f, int a, int b, int c)
{
    int d = s->cp[f].depth;
    if (f == FX0 || f == FXN)
        return ((size_t)a * s->yres + b) * s->zres + c;
    if (f == FY0 || f == FYN)
        return ((size_t)a * d + b) * s->zres + c;
    return ((size_t)a * s->yres + b) * d + c;
}

static int cpml_alloc(oracle_state *s)
{
    int f, i;
    for (f = 0; f < 6; f++) {
        int d = s->cp[f].depth;
        size_t cnt;
        if (!s->cp[f].enabled)
            continue;
        if (f <= FXN) cnt = (size_t)d * s->yres * s->zres;
        else if (f <= FYN) cnt = (size_t)s->xres * d * s->zres;
        else cnt = (size_t)s->xres * s->yres * d;
        s->be[f] = calloc(d, sizeof(double)); s->ce[f] = calloc(d, sizeof(double));
        s->bh[f] = calloc(d, sizeof(double)); s->ch[f] = calloc(d, sizeof(double));
        s->ke[f] = calloc(d, sizeof(double)); s->kh[f] = calloc(d, sizeof(double));
        s->pe[f][0] = calloc(cnt, sizeof(double)); s->pe[f][1] = calloc(cnt, sizeof(double));
        s->ph[f][0] = calloc(cnt, sizeof(double)); s->ph[f][1] = calloc(cnt, sizeof(double));
        if (!s->pe[f][0] || !s->pe[f][1] || !s->ph[f][0] || !s->ph[f][1])
            return -1;
        for (i = 0; i < d; i++) {
            int low = (f == FX0 || f == FY0 || f == FZ0);
            cpml_grade(low ? i : d - i, d, s->cp[f].sigma, s->cp[f].kappa, s->cp[f].a, s->cp[f].m, s->dt,
                       low ? 0.5 : -0.5, &s->be[f][i], &s->ce[f][i], &s->bh[f][i], &s->ch[f][i],
                       &s->ke[f][i], &s->kh[f][i]);
        }
    }
    return 0;
}

/* internal boundary map, plan.c:5387-5416 */
static void make_bnds(oracle_state *s)
{
    int i, j, k, ii, jj, kk;
    for (i = 0; i < s->xres; i++)
        for (j = 0; j < s->yres; j++)
            for (k = 0; k < s->zres; k++) {
                size_t c = IDX(s, i, j, k);
                double e, g, ne, ng;
                int m, nm;
                s->bnds[c] = 0;
                if (i == 0 || j == 0 || k == 0 || i == s->xres - 1 || j == s->yres - 1 || k == s->zres - 1) {
                    s->bnds[c] = 1;
                    continue;
                }
                m = get_eps_sig(s, i, j, k, &e, &g);
                for (ii = -1; ii <= 1; ii++)
                    for (jj = -1; jj <= 1; jj++)
                        for (kk = -1; kk <= 1; kk++) {
                            if (s->bnds[c] == 1)
                                continue;
                            nm = get_eps_sig(s, i + ii, j + jj, k + kk, &ne, &ng);
                            if (nm != m || ne != e || ng != g)
                                s->bnds[c] = 1;
                        }
            }
}

/* eval_closecheck, plan.c:3857-3873 */
static int closecheck(const oracle_state *s, int ip, int jp, int kp, int sd)
{
    int i, j, k;
    for (i = (ip - sd > 0 ? ip - sd : 0); i < (ip + sd < s->xres ? ip + sd : s->xres); i++)
        for (j = (jp - sd > 0 ? jp - sd : 0); j < (jp + sd < s->yres ? jp + sd : s->yres); j++)
            for (k = (kp - sd > 0 ? kp - sd : 0); k < (kp + sd < s->zres ? kp + sd : s->zres); k++)
                if (tsf_mattype(s, i, j, k) != 0)
                    return 1;
    return 0;
}

/* TSF source-skip map, plan.c:5298-5326 */
static void make_sourceskip(oracle_state *s)
{
    int i, j, k, sd = s->t.skipdepth;
    memset(s->sskip, 0, s->n * sizeof(int32_t));
    if (!s->tsf || sd < 0)
        return;
    for (i = 0; i < s->xres; i++)
        for (j = 0; j < s->yres; j++)
            for (k = 0; k < s->zres; k++) {
                if (i > (s->t.i0 + sd) && j > (s->t.j0 + sd) && k > (s->t.k0 + sd) &&
                    i < (s->t.in - sd) && j < (s->t.jn - sd) && k < (s->t.kn - sd))
                    continue;
                if (closecheck(s, i, j, k, sd))
                    s->sskip[IDX(s, i, j, k)] = 1;
            }
}

/* far-field geometry, farfield.c:31-172 */
static double ff_dist(double x1, double y1, double z1, double x2, double y2, double z2)
{
    return sqrt((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2) + (z1 - z2) * (z1 - z2));
}

static double ff_angvec(double x1, double y1, double z1, double x2, double y2, double z2)
{
    return ((double)(x1 * x2 + y1 * y2 + z1 * z2) / (sqrt((double)(x1 * x1 + y1 * y1 + z1 * z1) * (x2 * x2 + y2 * y2 + z2 * z2))));
}

static double ff_angle(double x1, double y1, double z1, double x2, double y2, double z2, int side)
{
    static const double nv[6][3] = {{0, -1, 0}, {0, 1, 0}, {-1, 0, 0}, {1, 0, 0}, {0, 0, -1}, {0, 0, 1}};
    return ff_angvec(x2 - x1, y2 - y1, z2 - z1, nv[side][0], nv[side][1], nv[side][2]);
}

static int nfff_setup(oracle_state *s, const fdtd_desc *d)
{
    int n, npt = s->ff.npoints;
    int i0 = s->ff.i0, i1 = s->ff.in, j0 = s->ff.j0, j1 = s->ff.jn, k0 = s->ff.k0, k1 = s->ff.kn;
    int ix = i1 - i0, iy = j1 - j0, iz = k1 - k0;
    double div = C0 * s->dt / s->dx;
    s->ndata = (int)(2000 + 2 * d->nsteps +
                     sqrt(s->xres * s->xres + s->yres * s->yres + s->zres * s->zres) / (C0 * s->dt / s->dx));
    s->ffpts = malloc(sizeof(int32_t) * 3 * (size_t)npt);
    s->ffistart = malloc(sizeof(int32_t) * (size_t)npt);
    s->ffser = calloc((size_t)npt * 3 * (size_t)s->ndata, sizeof(double));
    if (!s->ffpts || !s->ffistart || !s->ffser)
        return -1;
    memcpy(s->ffpts, d->nfff.points, sizeof(int32_t) * 3 * (size_t)npt);
    for (n = 0; n < npt; n++) {
        double ri = s->ffpts[3 * n], rj = s->ffpts[3 * n + 1], rk = s->ffpts[3 * n + 2];
        if (d->nfff.istart)
            s->ffistart[n] = d->nfff.istart[n];
        else {
            double v = sqrt((ri / div) * (ri / div) + (rj / div) * (rj / div) + (rk / div) * (rk / div)) - 500;
            s->ffistart[n] = (int)(v > 0 ? v : 0);
        }
    }
    /* tables per point: faces 0 left(x0) 1 right(xn) 2 top(y0) 3 bottom(yn) 4 front(z0) 5 back(zn) */
    {
        size_t fsz[6];
        int f;
        fsz[0] = fsz[1] = (size_t)iy * iz;
        fsz[2] = fsz[3] = (size_t)ix * iz;
        fsz[4] = fsz[5] = (size_t)ix * iy;
        for (f = 0; f < 6; f++) {
            s->ffr[f] = malloc(sizeof(double) * fsz[f] * (size_t)npt);
            s->ffct[f] = malloc(sizeof(double) * fsz[f] * (size_t)npt);
            if (!s->ffr[f] || !s->ffct[f])
                return -1;
        }
        for (n = 0; n < npt; n++) {
            double x = s->ffpts[3 * n], y = s->ffpts[3 * n + 1], z = s->ffpts[3 * n + 2];
            int i, j, k;
            for (j = j0; j < j1; j++)
                for (k = k0; k < k1; k++) {
                    size_t c = (size_t)n * fsz[0] + (size_t)(j - j0) * iz + (k - k0);
                    s->ffr[0][c] = ff_dist(x, y, z, i0, j, k);
                    s->ffct[0][c] = ff_angle(i0, j, k, x, y, z, 2);
                    s->ffr[1][c] = ff_dist(x, y, z, i1, j, k);
                    s->ffct[1][c] = ff_angle(i1, j, k, x, y, z, 3);
                }
            for (i = i0; i < i1; i++)
                for (k = k0; k < k1; k++) {
                    size_t c = (size_t)n * fsz[2] + (size_t)(i - i0) * iz + (k - k0);
                    s->ffr[2][c] = ff_dist(x, y, z, i, j0, k);
                    s->ffct[2][c] = ff_angle(i, j0, k, x, y, z, 0);
                    s->ffr[3][c] = ff_dist(x, y, z, i, j1, k);
                    s->ffct[3][c] = ff_angle(i, j1, k, x, y, z, 1);
                }
            for (i = i0; i < i1; i++)
                for (j = j0; j < j1; j++) {
                    size_t c = (size_t)n * fsz[4] + (size_t)(i - i0) * iy + (j - j0);
                    s->ffr[4][c] = ff_dist(x, y, z, i, j, k0);
                    s->ffct[4][c] = ff_angle(i, j, k0, x, y, z, 4);
                    s->ffr[5][c] = ff_dist(x, y, z, i, j, k1);
                    s->ffct[5][c] = ff_angle(i, j, k1, x, y, z, 5);
                }
        }
    }
    return 0;
}

static void set_err(char *err, const char *msg)
{
    if (err) {
        strncpy(err, msg, 255);
        err[255] = 0;
    }
}

oracle_state *oracle_create(const fdtd_desc *d, char *err)
{
    oracle_state *s;
    size_t n, c;
    int m, comp, f;
    if (!d || d->abi_version != FDTD_ABI_VERSION) {
        set_err(err, "bad descriptor");
        return NULL;
    }
    if (d->xres < 3 || d->yres < 3 || d->zres < 3) {
        set_err(err, "grid too small");
        return NULL;
    }
    for (m = 1; m < d->nmat; m++) {
        int ty = d->mats[m].type;
        if (ty != FDTD_MAT_LINTAB && ty != FDTD_MAT_ADE && ty != FDTD_MAT_PEC) {
            set_err(err, "material type outside the stepped path (LINTAB, ADE, PEC)");
            return NULL;
        }
    }
    s = calloc(1, sizeof(*s));
    if (!s) return NULL;
    s->xres = d->xres; s->yres = d->yres; s->zres = d->zres;
    n = s->n = (size_t)d->xres * d->yres * d->zres;
    s->dx = d->dx; s->dy = d->dy; s->dz = d->dz; s->dt = d->dt;
    s->matmode = d->matmode;
    s->nmat = d->nmat;
    s->nsteps_planned = d->nsteps;
    for (comp = 0; comp < 6; comp++) {
        s->f[comp] = calloc(n, sizeof(double));
        if (!s->f[comp]) { set_err(err, "out of memory"); oracle_destroy(s); return NULL; }
    }
    if (s->nmat > 0) {
        s->mats = malloc(sizeof(fdtd_material) * (size_t)s->nmat);
        s->mat = malloc(sizeof(int32_t) * n);
        memcpy(s->mats, d->mats, sizeof(fdtd_material) * (size_t)s->nmat);
        if (d->mat) memcpy(s->mat, d->mat, sizeof(int32_t) * n);
        else memset(s->mat, 0, sizeof(int32_t) * n);
        for (c = 0; c < n; c++)
            if (s->mat[c] < 0 || s->mat[c] >= s->nmat) {
                set_err(err, "material index out of range");
                oracle_destroy(s);
                return NULL;
            }
        for (m = 1; m < s->nmat; m++)
            if (s->mats[m].type == FDTD_MAT_ADE) s->disp = 1;
    }
    /* voxel arrays, yee.c:104-116 */
    if (s->matmode == FDTD_MATMODE_FULL || s->matmode == FDTD_MATMODE_ELECTRIC) {
        s->veps = malloc(sizeof(double) * n);
        s->vsig = malloc(sizeof(double) * n);
        for (c = 0; c < n; c++) {
            s->veps[c] = d->epsilon ? (double)d->epsilon[c] : (double)(float)EPS0;
            s->vsig[c] = d->sigma ? (double)d->sigma[c] : 0.0;
        }
    }
    if (s->matmode == FDTD_MATMODE_FULL || s->matmode == FDTD_MATMODE_MAGNETIC) {
        s->vmu = malloc(sizeof(double) * n);
        s->vsigast = malloc(sizeof(double) * n);
        for (c = 0; c < n; c++) {
            s->vmu[c] = d->mu ? (double)d->mu[c] : (double)(float)MU0;
            s->vsigast[c] = d->sigast ? (double)d->sigast[c] : 0.0;
        }
    }
    if (s->disp) { /* allocate_ade, plan.c:4013-4060 */
        for (comp = 0; comp < 3; comp++) {
            s->ep[comp] = calloc(n, sizeof(double));
            s->dp[comp] = calloc(n, sizeof(double));
            s->dpp[comp] = calloc(n, sizeof(double));
            s->p[comp][0] = calloc(n, sizeof(double)); s->p[comp][1] = calloc(n, sizeof(double));
            s->pp[comp][0] = calloc(n, sizeof(double)); s->pp[comp][1] = calloc(n, sizeof(double));
            if (!s->ep[comp] || !s->dp[comp] || !s->dpp[comp] || !s->p[comp][0] || !s->p[comp][1] ||
                !s->pp[comp][0] || !s->pp[comp][1]) {
                set_err(err, "out of memory"); oracle_destroy(s); return NULL;
            }
        }
    }
    s->bnds = malloc(sizeof(int32_t) * n);
    s->sskip = malloc(sizeof(int32_t) * n);
    for (f = 0; f < 6; f++) s->cp[f] = d->cpml[f];
    if (cpml_alloc(s)) { set_err(err, "out of memory"); oracle_destroy(s); return NULL; }
    make_bnds(s);
    /* TSF, plan.c:1522-1597 */
    s->tsf = d->tsf.enabled;
    if (s->tsf) {
        int i;
        s->t = d->tsf;
        s->wave = malloc(sizeof(double) * (size_t)(d->tsf.nwave > 0 ? d->tsf.nwave : 1));
        if (d->tsf.nwave > 0) memcpy(s->wave, d->tsf.wave, sizeof(double) * (size_t)d->tsf.nwave);
        s->corr = 1.0 / sqrt(pow(sin(s->t.theta), 4) * (pow(cos(s->t.phi), 4) + pow(sin(s->t.phi), 4)) +
                             pow(cos(s->t.theta), 4));
        s->jres = (int)(sqrt((double)(s->xres * s->xres + s->yres * s->yres + s->zres * s->zres)) + 250);
        s->jdx = s->dx / s->corr;
        s->je = calloc((size_t)s->jres + 4, sizeof(double));   /* dval may touch data[res] */
        s->jh = calloc((size_t)s->jres + 4, sizeof(double));
        s->jeps = malloc(sizeof(double) * (size_t)s->jres);
        s->jmu = malloc(sizeof(double) * (size_t)s->jres);
        for (i = 0; i < s->jres; i++) {
            s->jeps[i] = s->t.layered_epsilon;
            s->jmu[i] = s->t.layered_mu;
        }
    }
    make_sourceskip(s);
    s->nfff = d->nfff.enabled && d->nfff.npoints > 0;
    if (s->nfff) {
        s->ff = d->nfff;
        if (nfff_setup(s, d)) { set_err(err, "out of memory"); oracle_destroy(s); return NULL; }
    }
    s->nprobes = d->nprobes;
    if (s->nprobes > 0) {
        s->probes = malloc(sizeof(int32_t) * 3 * (size_t)s->nprobes);
        memcpy(s->probes, d->probes, sizeof(int32_t) * 3 * (size_t)s->nprobes);
        s->probe_out = calloc((size_t)s->nprobes * 6 * (size_t)(d->nsteps > 0 ? d->nsteps : 1), sizeof(double));
    }
    return s;
}

void oracle_destroy(oracle_state *s)
{
    int c, f;
    if (!s) return;
    for (c = 0; c < 6; c++) free(s->f[c]);
    for (c = 0; c < 3; c++) {
        free(s->ep[c]); free(s->dp[c]); free(s->dpp[c]);
        free(s->p[c][0]); free(s->p[c][1]); free(s->pp[c][0]); free(s->pp[c][1]);
    }
    for (f = 0; f < 6; f++) {
        free(s->be[f]); free(s->ce[f]); free(s->bh[f]); free(s->ch[f]); free(s->ke[f]); free(s->kh[f]);
        free(s->pe[f][0]); free(s->pe[f][1]); free(s->ph[f][0]); free(s->ph[f][1]);
        free(s->ffr[f]); free(s->ffct[f]);
    }
    free(s->mats); free(s->mat); free(s->veps); free(s->vsig); free(s->vmu); free(s->vsigast);
    free(s->bnds); free(s->sskip); free(s->wave); free(s->je); free(s->jh); free(s->jeps); free(s->jmu);
    free(s->ffpts); free(s->ffistart); free(s->ffser); free(s->probes); free(s->probe_out);
    free(s);
}

/* ---------------------------------------------------------------- H step */

static double kappa_at(const oracle_state *s, int face, int pos, int h)
{
    const double *t = h ? s->kh[face] : s->ke[face];
    return t[pos];
}

/* sv_yee_data_ystep_h, yee.c:146-265 */
static void ystep_h(oracle_state *s)
{
    int i;
    const int xr = s->xres, yr = s->yres, zr = s->zres;
    const double dt = s->dt;
#pragma omp parallel for schedule(static)
    for (i = 0; i < xr; i++) {
        int j, k;
        for (j = 0; j < yr; j++)
            for (k = 0; k < zr; k++) {
                size_t c = IDX(s, i, j, k);
                int m = matidx(s, i, j, k);
                double kx = 1, ky = 1, kz = 1, da, dbx, dby, dbz, ex, ey, ez;
                if (s->cp[FX0].enabled && i < s->cp[FX0].depth) kx = fmax(kx, kappa_at(s, FX0, i, 1));
                if (s->cp[FXN].enabled && i >= xr - s->cp[FXN].depth) kx = fmax(kx, kappa_at(s, FXN, i - (xr - s->cp[FXN].depth), 1));
                if (s->cp[FY0].enabled && j < s->cp[FY0].depth) ky = fmax(ky, kappa_at(s, FY0, j, 1));
                if (s->cp[FYN].enabled && j >= yr - s->cp[FYN].depth) ky = fmax(ky, kappa_at(s, FYN, j - (yr - s->cp[FYN].depth), 1));
                if (s->cp[FZ0].enabled && k < s->cp[FZ0].depth) kz = fmax(kz, kappa_at(s, FZ0, k, 1));
                if (s->cp[FZN].enabled && k >= zr - s->cp[FZN].depth) kz = fmax(kz, kappa_at(s, FZN, k - (zr - s->cp[FZN].depth), 1));
                ex = EX(s)[c]; ey = EY(s)[c]; ez = EZ(s)[c];
                if (m > 0 && is_tab(s->mats[m].type)) {
                    const fdtd_material *q = &s->mats[m];
                    da = (1 - q->sigast * dt / 2 / q->mu) / (1 + q->sigast * dt / 2 / q->mu);
                    dbx = (dt / q->mu / s->dx) / (1 + q->sigast * dt / 2 / q->mu);
                    dby = (dt / q->mu / s->dy) / (1 + q->sigast * dt / 2 / q->mu);
                    dbz = (dt / q->mu / s->dz) / (1 + q->sigast * dt / 2 / q->mu);
                } else if (s->matmode == FDTD_MATMODE_FULL || s->matmode == FDTD_MATMODE_MAGNETIC) {
                    double mu = s->vmu[c], sa = s->vsigast[c];
                    da = (1 - sa * dt / 2 / mu) / (1 + sa * dt / 2 / mu);
                    dbx = (dt / mu / s->dx) / (1 + sa * dt / 2 / mu);
                    dby = (dt / mu / s->dy) / (1 + sa * dt / 2 / mu);
                    dbz = (dt / mu / s->dz) / (1 + sa * dt / 2 / mu);
                } else {
                    da = 1;
                    dbx = dt / MU0 / s->dx;
                    dby = dt / MU0 / s->dy;
                    dbz = dt / MU0 / s->dz;
                }
                if (!(j == yr - 1 || k == zr - 1))
                    HX(s)[c] = da * HX(s)[c] + dbx * ((EY(s)[c + 1] - ey) / kz - (EZ(s)[c + zr] - ez) / ky);
                if (!(i == xr - 1 || k == zr - 1))
                    HY(s)[c] = da * HY(s)[c] + dby * ((EZ(s)[c + (size_t)yr * zr] - ez) / kx - (EX(s)[c + 1] - ex) / kz);
                if (!(i == xr - 1 || j == yr - 1))
                    HZ(s)[c] = da * HZ(s)[c] + dbz * ((EX(s)[c + zr] - ex) / ky - (EY(s)[c + (size_t)yr * zr] - ey) / kx);
            }
    }
}

/* ------------------------------------------------------------ TSF source */

/* dcomp, source.c:54-107 (with the reference's i0=0, i1=xres, ... call) */
static double dcomp(const oracle_state *s, int i, int j, int k)
{
    double th = s->t.theta, ph = s->t.phi;
    double ax = sin(th) * cos(ph), ay = sin(th) * sin(ph), az = cos(th);
    double rx = 0, ry = 0, rz = 0;
    int i0 = 0, i1 = s->xres, j0 = 0, j1 = s->yres, k0 = 0, k1 = s->zres;
    if (th >= 0 && th <= (PI_D / 2.0)) {
        if (ph >= 0 && ph <= (PI_D / 2.0)) { rx = i - i0; ry = j - j0; rz = k - k0; }
        else if (ph > (PI_D / 2.0) && ph <= PI_D) { rx = i - i1; ry = j - j0; rz = k - k0; }
        else if (ph > PI_D && ph <= (3.0 * PI_D / 2.0)) { rx = i - i1; ry = j - j1; rz = k - k0; }
        else { rx = i - i0; ry = j - j1; rz = k - k0; }
    } else if (th < PI_D && th > (PI_D / 2.0)) {
        if (ph >= 0 && ph <= (PI_D / 2.0)) { rx = i - i0; ry = j - j0; rz = k - k1; }
        else if (ph > (PI_D / 2.0) && ph <= PI_D) { ry = j - j0; rz = k - k1; }
        else if (ph > PI_D && ph <= (3.0 * PI_D / 2.0)) { rx = i - i1; ry = j - j1; rz = k - k1; }
        else { rx = i - i0; ry = j - j1; rz = k - k1; }
    } else
        return -1;
    return 10 + (ax * rx + ay * ry + az * rz);
}

/* sv_dline_get_dval, dline.c:89-111 */
static double dval(const double *data, int res, double x)
{
    int l = (int)floor(x);
    double a = x - (double)l;
    if (x >= 1 && x < (res - 1)) {
        double w1 = a + 1, w2 = a, w3 = 1 - a, w4 = 2 - a;
        w1 = 4 - 8 * w1 + 5 * w1 * w1 - w1 * w1 * w1;
        w2 = 1 - 2 * w2 * w2 + w2 * w2 * w2;
        w3 = 1 - 2 * w3 * w3 + w3 * w3 * w3;
        w4 = 4 - 8 * w4 + 5 * w4 * w4 - w4 * w4 * w4;
        return w1 * data[l - 1] + w2 * data[l] + w3 * data[l + 1] + w4 * data[l + 2];
    } else if ((x < 1 && x >= 0) || (x >= (res - 1) && x < res))
        return (1 - a) * data[l] + a * data[l + 1];
    return 0;
}

/* projections gex..ghz, source.c:131-165 */
static double gex(double f, double t, double p, double q) { return f * (cos(q) * sin(p) - sin(q) * cos(t) * cos(p)); }
static double gey(double f, double t, double p, double q) { return f * (-cos(q) * cos(p) - sin(q) * cos(t) * sin(p)); }
static double gez(double f, double t, double p, double q) { (void)p; return f * (sin(q) * sin(t)); }
static double ghx(double f, double t, double p, double q) { return f * (sin(q) * sin(p) + cos(q) * cos(t) * cos(p)); }
static double ghy(double f, double t, double p, double q) { return f * (-sin(q) * cos(p) + cos(q) * cos(t) * sin(p)); }
static double ghz(double f, double t, double p, double q) { (void)p; return f * (-cos(q) * sin(t)); }

/* mat_too_close_check, source.c:253-265 (the LTSF skip depth is -1 here) */
static int mtc(const oracle_state *s, int i, int j, int k)
{
    if (s->t.skipdepth == -1)
        return 1;
    return s->sskip[IDX(s, i, j, k)] ? 0 : 1;
}

/* 1D auxiliary grid step, source.c:1469-1473 over 1dpool.c:84-162 */
static void aux_step(oracle_state *s)
{
    int i, r = s->jres;
    double multe = s->dt / (EPS0 * s->jdx) / 1;
    double multh = s->dt / (MU0 * s->jdx) / 1;
    double lc = (s->dt * C0 - s->jdx) / (s->dt * C0 + s->jdx);
    double *e = s->je, *h = s->jh;
    for (i = 0; i < r; i++)                 /* sv_1dpool_ystep_e */
        if (i > 0)
            e[i] += 1.0 / s->jeps[i] * multe * (h[i - 1] - h[i]);
    e[0] = s->jb[1] + lc * (e[1] - s->jb[0]);          /* sv_1dpool_boundary */
    h[0] = s->jb[3] + lc * (h[1] - s->jb[2]);
    e[r - 1] = s->jb[5] + lc * (e[r - 2] - s->jb[4]);
    h[r - 1] = s->jb[7] + lc * (h[r - 2] - s->jb[6]);
    s->jb[0] = e[0]; s->jb[1] = e[1]; s->jb[2] = h[0]; s->jb[3] = h[1];   /* _boundary_copy */
    s->jb[4] = e[r - 1]; s->jb[5] = e[r - 2]; s->jb[6] = h[r - 1]; s->jb[7] = h[r - 2];
    e[0] = (s->step < s->t.nwave) ? s->wave[s->step] : 0.0;              /* _apply_source */
    for (i = 0; i < r; i++)                 /* sv_1dpool_ystep_h */
        if (i < r - 1)
            h[i] += 1.0 / s->jmu[i] * multh * (e[i] - e[i + 1]);
}

/* TSF part of sv_pool_apply_source_hstep, source.c:1464-1672 */
static void tsf_h(oracle_state *s)
{
    const fdtd_tsf *t = &s->t;
    double hcor = s->dt / s->dx / MU0;
    double th = t->theta, ph = t->phi, ps = t->psi;
    int i, j, k;
    aux_step(s);
    for (j = t->j0; j <= t->jn; j++)
        for (k = t->k0; k <= t->kn; k++) {
            if (!t->skip[FX0] && mtc(s, t->i0, j, k)) {
                double ve = dval(s->je, s->jres, s->corr * dcomp(s, t->i0, j, k));
                if (k < t->kn) HY(s)[IDX(s, t->i0 - 1, j, k)] -= 1 * hcor * gez(ve, th, ph, ps);
                if (j < t->jn) HZ(s)[IDX(s, t->i0 - 1, j, k)] += hcor * gey(ve, th, ph, ps);
            }
            if (!t->skip[FXN] && mtc(s, t->in, j, k)) {
                double ve = dval(s->je, s->jres, s->corr * dcomp(s, t->in, j, k));
                if (k < t->kn) HY(s)[IDX(s, t->in, j, k)] += 1 * hcor * gez(ve, th, ph, ps);
                if (j < t->jn) HZ(s)[IDX(s, t->in, j, k)] -= hcor * gey(ve, th, ph, ps);
            }
        }
    for (i = t->i0; i <= t->in; i++)
        for (k = t->k0; k <= t->kn; k++) {
            if (!t->skip[FY0] && mtc(s, i, t->j0, k)) {
                double ve = dval(s->je, s->jres, s->corr * dcomp(s, i, t->j0, k));
                if (k < t->kn) HX(s)[IDX(s, i, t->j0 - 1, k)] += 1 * hcor * gez(ve, th, ph, ps);
                if (i < t->in) HZ(s)[IDX(s, i, t->j0 - 1, k)] -= hcor * gex(ve, th, ph, ps);
            }
            if (!t->skip[FYN] && mtc(s, i, t->jn, k)) {
                double ve = dval(s->je, s->jres, s->corr * dcomp(s, i, t->jn, k));
                if (k < t->kn) HX(s)[IDX(s, i, t->jn, k)] -= 1 * hcor * gez(ve, th, ph, ps);
                if (i < t->in) HZ(s)[IDX(s, i, t->jn, k)] += hcor * gex(ve, th, ph, ps);
            }
        }
    for (i = t->i0; i <= t->in; i++)
        for (j = t->j0; j <= t->jn; j++) {
            if (!t->skip[FZ0] && mtc(s, i, j, t->k0)) {
                double ve = dval(s->je, s->jres, s->corr * dcomp(s, i, j, t->k0));
                if (j < t->jn && !is_pec(s, i, j, t->k0)) HX(s)[IDX(s, i, j, t->k0 - 1)] -= 1 * hcor * gey(ve, th, ph, ps);
                if (i < t->in && !is_pec(s, i, j, t->k0)) HY(s)[IDX(s, i, j, t->k0 - 1)] += 1 * hcor * gex(ve, th, ph, ps);
            }
            if (!t->skip[FZN] && mtc(s, i, j, t->kn)) {
                double ve = dval(s->je, s->jres, s->corr * dcomp(s, i, j, t->kn));
                if (j < t->jn) HX(s)[IDX(s, i, j, t->kn)] += 1 * hcor * gey(ve, th, ph, ps);
                if (i < t->in) HY(s)[IDX(s, i, j, t->kn)] -= 1 * hcor * gex(ve, th, ph, ps);
            }
        }
}

/* TSF part of sv_pool_apply_source_estep, source.c:547-771 */
static void tsf_e(oracle_state *s)
{
    const fdtd_tsf *t = &s->t;
    double ecor = s->dt / s->dx;
    double th = t->theta, ph = t->phi, ps = t->psi;
    int i, j, k;
    for (j = t->j0; j <= t->jn; j++)
        for (k = t->k0; k <= t->kn; k++) {
            if (!t->skip[FX0] && mtc(s, t->i0, j, k)) {
                double vh = dval(s->jh, s->jres, s->corr * dcomp(s, t->i0 - 1, j, k));
                double eps = get_eps(s, t->i0, j, k);
                if (j < t->jn) EY(s)[IDX(s, t->i0, j, k)] += 1 * ecor / eps * ghz(vh, th, ph, ps);
                if (k < t->kn) EZ(s)[IDX(s, t->i0, j, k)] -= ecor / eps * ghy(vh, th, ph, ps);
            }
            if (!t->skip[FXN] && mtc(s, t->in, j, k)) {
                double vh = dval(s->jh, s->jres, s->corr * dcomp(s, t->in, j, k));
                double eps = get_eps(s, t->in, j, k);
                if (j < t->jn) EY(s)[IDX(s, t->in, j, k)] -= 1 * ecor / eps * ghz(vh, th, ph, ps);
                if (k < t->kn) EZ(s)[IDX(s, t->in, j, k)] += ecor / eps * ghy(vh, th, ph, ps);
            }
        }
    for (i = t->i0; i <= t->in; i++)
        for (k = t->k0; k <= t->kn; k++) {
            if (!t->skip[FY0] && mtc(s, i, t->j0, k)) {
                double vh = dval(s->jh, s->jres, s->corr * dcomp(s, i, t->j0 - 1, k));
                double eps = get_eps(s, i, t->j0, k);
                if (i < t->in) EX(s)[IDX(s, i, t->j0, k)] -= 1 * ecor / eps * ghz(vh, th, ph, ps);
                if (k < t->kn) EZ(s)[IDX(s, i, t->j0, k)] += ecor / eps * ghx(vh, th, ph, ps);
            }
            if (!t->skip[FYN] && mtc(s, i, t->jn, k)) {
                double vh = dval(s->jh, s->jres, s->corr * dcomp(s, i, t->jn, k));
                double eps = get_eps(s, i, t->jn, k);
                if (i < t->in) EX(s)[IDX(s, i, t->jn, k)] += 1 * ecor / eps * ghz(vh, th, ph, ps);
                if (k < t->kn) EZ(s)[IDX(s, i, t->jn, k)] -= ecor / eps * ghx(vh, th, ph, ps);
            }
        }
    for (i = t->i0; i <= t->in; i++)
        for (j = t->j0; j <= t->jn; j++) {
            if (!t->skip[FZ0] && mtc(s, i, j, t->k0)) {
                double vh = dval(s->jh, s->jres, s->corr * dcomp(s, i, j, t->k0 - 1));
                double eps = get_eps(s, i, j, t->k0);
                if (i < t->in && !is_pec(s, i, j, t->k0)) EX(s)[IDX(s, i, j, t->k0)] += 1 * ecor / eps * ghy(vh, th, ph, ps);
                if (j < t->jn && !is_pec(s, i, j, t->k0)) EY(s)[IDX(s, i, j, t->k0)] -= 1 * ecor / eps * ghx(vh, th, ph, ps);
            }
            if (!t->skip[FZN] && mtc(s, i, j, t->kn)) {
                double vh = dval(s->jh, s->jres, s->corr * dcomp(s, i, j, t->kn));
                double eps = get_eps(s, i, j, t->kn);
                if (i < t->in) EX(s)[IDX(s, i, j, t->kn)] -= 1 * ecor / eps * ghy(vh, th, ph, ps);
                if (j < t->jn) EY(s)[IDX(s, i, j, t->kn)] += 1 * ecor / eps * ghx(vh, th, ph, ps);
            }
        }
}

/* ----------------------------------------------------------- CPML H step */

/* CPML part of sv_pool_boundary_hstep, boundary.c:347-519 */
static void cpml_h(oracle_state *s)
{
    const int xr = s->xres, yr = s->yres, zr = s->zres;
    const double dx = s->dx, dy = s->dy, dz = s->dz;
    int i, j, k;
    if (s->cp[FX0].enabled) {
        for (i = 0; i < s->cp[FX0].depth - 1; i++) {
#pragma omp parallel for private(k) schedule(static)
            for (j = 1; j < yr - 1; j++)
                for (k = 1; k < zr - 1; k++) {
                    size_t c = IDX(s, i, j, k), q = slab_idx(s, FX0, i, j, k);
                    double db = get_db(s, i, j, k), bh = s->bh[FX0][i], ch = s->ch[FX0][i];
                    s->ph[FX0][1][q] = bh * s->ph[FX0][1][q] + ch * ((EY(s)[IDX(s, i + 1, j, k)] - EY(s)[c])) / dx; /* phzx */
                    s->ph[FX0][0][q] = bh * s->ph[FX0][0][q] + ch * ((EZ(s)[IDX(s, i + 1, j, k)] - EZ(s)[c])) / dx; /* phyx */
                    HY(s)[c] += dx * db * s->ph[FX0][0][q];
                    HZ(s)[c] -= dx * db * s->ph[FX0][1][q];
                }
        }
    }
    if (s->cp[FY0].enabled) {
        for (j = 0; j < s->cp[FY0].depth - 1; j++) {
#pragma omp parallel for private(k) schedule(static)
            for (i = 1; i < xr - 1; i++)
                for (k = 1; k < zr - 1; k++) {
                    size_t c = IDX(s, i, j, k), q = slab_idx(s, FY0, i, j, k);
                    double db = get_db(s, i, j, k), bh = s->bh[FY0][j], ch = s->ch[FY0][j];
                    s->ph[FY0][0][q] = bh * s->ph[FY0][0][q] + ch * ((EZ(s)[IDX(s, i, j + 1, k)] - EZ(s)[c])) / dy; /* phxy */
                    s->ph[FY0][1][q] = bh * s->ph[FY0][1][q] + ch * ((EX(s)[IDX(s, i, j + 1, k)] - EX(s)[c])) / dy; /* phzy */
                    HX(s)[c] -= dy * db * s->ph[FY0][0][q];
                    HZ(s)[c] += dy * db * s->ph[FY0][1][q];
                }
        }
    }
    if (s->cp[FZ0].enabled) {
        for (k = 0; k < s->cp[FZ0].depth - 1; k++) {
#pragma omp parallel for private(j) schedule(static)
            for (i = 1; i < xr - 1; i++)
                for (j = 1; j < yr - 1; j++) {
                    size_t c = IDX(s, i, j, k), q = slab_idx(s, FZ0, i, j, k);
                    double db = get_db(s, i, j, k), bh = s->bh[FZ0][k], ch = s->ch[FZ0][k];
                    s->ph[FZ0][1][q] = bh * s->ph[FZ0][1][q] + ch * ((EX(s)[IDX(s, i, j, k + 1)] - EX(s)[c])) / dz; /* phyz */
                    s->ph[FZ0][0][q] = bh * s->ph[FZ0][0][q] + ch * ((EY(s)[IDX(s, i, j, k + 1)] - EY(s)[c])) / dz; /* phxz */
                    HY(s)[c] -= dz * db * s->ph[FZ0][1][q];
                    HX(s)[c] += dz * db * s->ph[FZ0][0][q];
                }
        }
    }
    if (s->cp[FXN].enabled) {
        int d = s->cp[FXN].depth;
        for (j = 1; j < yr - 1; j++)
            for (k = 1; k < zr - 1; k++)
                HX(s)[IDX(s, xr - 1, j, k)] = HY(s)[IDX(s, xr - 1, j, k)] = HZ(s)[IDX(s, xr - 1, j, k)] = 0;
        for (i = xr - d + 1; i < xr - 1; i++) {
            int ir = i - (xr - d);
#pragma omp parallel for private(k) schedule(static)
            for (j = 1; j < yr - 1; j++)
                for (k = 1; k < zr - 1; k++) {
                    size_t c = IDX(s, i, j, k), q = slab_idx(s, FXN, ir, j, k);
                    double db = get_db(s, i, j, k), bh = s->bh[FXN][ir], ch = s->ch[FXN][ir];
                    s->ph[FXN][1][q] = bh * s->ph[FXN][1][q] + ch * ((EY(s)[IDX(s, i + 1, j, k)] - EY(s)[c])) / dx;
                    s->ph[FXN][0][q] = bh * s->ph[FXN][0][q] + ch * ((EZ(s)[IDX(s, i + 1, j, k)] - EZ(s)[c])) / dx;
                    HY(s)[c] += dx * db * s->ph[FXN][0][q];
                    HZ(s)[c] -= dx * db * s->ph[FXN][1][q];
                }
        }
    }
    if (s->cp[FYN].enabled) {
        int d = s->cp[FYN].depth;
        for (i = 1; i < xr - 1; i++)
            for (k = 1; k < zr - 1; k++)
                HX(s)[IDX(s, i, yr - 1, k)] = HY(s)[IDX(s, i, yr - 1, k)] = HZ(s)[IDX(s, i, yr - 1, k)] = 0;
        for (j = yr - d + 1; j < yr - 1; j++) {
            int jr = j - (yr - d);
#pragma omp parallel for private(k) schedule(static)
            for (i = 1; i < xr - 1; i++)
                for (k = 1; k < zr - 1; k++) {
                    size_t c = IDX(s, i, j, k), q = slab_idx(s, FYN, i, jr, k);
                    double db = get_db(s, i, j, k), bh = s->bh[FYN][jr], ch = s->ch[FYN][jr];
                    s->ph[FYN][0][q] = bh * s->ph[FYN][0][q] + ch * ((EZ(s)[IDX(s, i, j + 1, k)] - EZ(s)[c])) / dy;
                    s->ph[FYN][1][q] = bh * s->ph[FYN][1][q] + ch * ((EX(s)[IDX(s, i, j + 1, k)] - EX(s)[c])) / dy;
                    HX(s)[c] -= dy * db * s->ph[FYN][0][q];
                    HZ(s)[c] += dy * db * s->ph[FYN][1][q];
                }
        }
    }
    if (s->cp[FZN].enabled) {
        int d = s->cp[FZN].depth;
        for (i = 1; i < xr - 1; i++)
            for (j = 1; j < yr - 1; j++)
                HX(s)[IDX(s, i, j, zr - 1)] = HY(s)[IDX(s, i, j, zr - 1)] = HZ(s)[IDX(s, i, j, zr - 1)] = 0;
        for (k = zr - d + 1; k < zr - 1; k++) {
            int kr = k - (zr - d);
#pragma omp parallel for private(j) schedule(static)
            for (i = 1; i < xr - 1; i++)
                for (j = 1; j < yr - 1; j++) {
                    size_t c = IDX(s, i, j, k), q = slab_idx(s, FZN, i, j, kr);
                    double db = get_db(s, i, j, k), bh = s->bh[FZN][kr], ch = s->ch[FZN][kr];
                    s->ph[FZN][1][q] = bh * s->ph[FZN][1][q] + ch * ((EX(s)[IDX(s, i, j, k + 1)] - EX(s)[c])) / dz;
                    s->ph[FZN][0][q] = bh * s->ph[FZN][0][q] + ch * ((EY(s)[IDX(s, i, j, k + 1)] - EY(s)[c])) / dz;
                    HY(s)[c] -= dz * db * s->ph[FZN][1][q];
                    HX(s)[c] += dz * db * s->ph[FZN][0][q];
                }
        }
    }
}

/* ------------------------------------------------------------- E step */

/* CPML inside the ADE branch of ystep_e, yee.c:950-1057 */
static void ade_cpml(oracle_state *s, int i, int j, int k, const fdtd_material *q, double cb0, int xt, int yt, int zt)
{
    const int xr = s->xres, yr = s->yres, zr = s->zres;
    const double dx = s->dx, dy = s->dy, dz = s->dz, dt = s->dt;
    size_t c = IDX(s, i, j, k);
    double cbx = (dt / q->epsilon / dx) / (1 + q->sigma * dt / 2 / q->epsilon);
    double cby = (dt / q->epsilon / dy) / (1 + q->sigma * dt / 2 / q->epsilon);
    double cbz = (dt / q->epsilon / dz) / (1 + q->sigma * dt / 2 / q->epsilon);
    if (s->cp[FX0].enabled && i > 1 && i < s->cp[FX0].depth) {
        size_t w = slab_idx(s, FX0, i, j, k);
        double be = s->be[FX0][i], ce = s->ce[FX0][i];
        s->pe[FX0][0][w] = be * s->pe[FX0][0][w] + ce * ((HZ(s)[c] - HZ(s)[IDX(s, i - 1, j, k)])) / dy;
        s->pe[FX0][1][w] = be * s->pe[FX0][1][w] + ce * ((HY(s)[c] - HY(s)[IDX(s, i - 1, j, k)])) / dz;
        if (!(j == 0 || k == 0) && yt == 0) EY(s)[c] -= dy * cb0 * s->pe[FX0][0][w];
        if (!(j == 0 || k == 0) && zt == 0) EZ(s)[c] += dz * cb0 * s->pe[FX0][1][w];
    }
    if (s->cp[FY0].enabled && j > 1 && j < s->cp[FY0].depth) {
        size_t w = slab_idx(s, FY0, i, j, k);
        double be = s->be[FY0][j], ce = s->ce[FY0][j];
        s->pe[FY0][0][w] = be * s->pe[FY0][0][w] + ce * ((HZ(s)[c] - HZ(s)[IDX(s, i, j - 1, k)])) / dz;
        s->pe[FY0][1][w] = be * s->pe[FY0][1][w] + ce * ((HX(s)[c] - HX(s)[IDX(s, i, j - 1, k)])) / dx;
        if (!(i == 0 || k == 0) && xt == 0) EX(s)[c] += dx * cbx * s->pe[FY0][0][w];
        if (!(i == 0 || k == 0) && zt == 0) EZ(s)[c] -= dz * cbz * s->pe[FY0][1][w];
    }
    if (s->cp[FZ0].enabled && k > 1 && k < s->cp[FZ0].depth) {
        size_t w = slab_idx(s, FZ0, i, j, k);
        double be = s->be[FZ0][k], ce = s->ce[FZ0][k];
        s->pe[FZ0][1][w] = be * s->pe[FZ0][1][w] + ce * ((HX(s)[c] - HX(s)[IDX(s, i, j, k - 1)])) / dy; /* peyz */
        s->pe[FZ0][0][w] = be * s->pe[FZ0][0][w] + ce * ((HY(s)[c] - HY(s)[IDX(s, i, j, k - 1)])) / dx; /* pexz */
        if (!(i == 0 || j == 0) && yt == 0) EY(s)[c] += dy * cby * s->pe[FZ0][1][w];
        if (!(i == 0 || j == 0) && xt == 0) EX(s)[c] -= dx * cbx * s->pe[FZ0][0][w];
    }
    if (s->cp[FXN].enabled && (i >= (xr - s->cp[FXN].depth + 1)) && i < xr) {
        int ir = i - (xr - s->cp[FXN].depth);
        size_t w = slab_idx(s, FXN, ir, j, k);
        double be = s->be[FXN][ir], ce = s->ce[FXN][ir];
        s->pe[FXN][0][w] = be * s->pe[FXN][0][w] + ce * ((HZ(s)[c] - HZ(s)[IDX(s, i - 1, j, k)])) / dy;
        s->pe[FXN][1][w] = be * s->pe[FXN][1][w] + ce * ((HY(s)[c] - HY(s)[IDX(s, i - 1, j, k)])) / dz;
        if (!(j == 0 || k == 0) && yt == 0) EY(s)[c] -= dy * cby * s->pe[FXN][0][w];
        if (!(j == 0 || k == 0) && zt == 0) EZ(s)[c] += dz * cbz * s->pe[FXN][1][w];
    }
    if (s->cp[FYN].enabled && (j >= (yr - s->cp[FYN].depth + 1)) && j < yr) {
        int jr = j - (yr - s->cp[FYN].depth);
        size_t w = slab_idx(s, FYN, i, jr, k);
        double be = s->be[FYN][jr], ce = s->ce[FYN][jr];
        s->pe[FYN][0][w] = be * s->pe[FYN][0][w] + ce * ((HZ(s)[c] - HZ(s)[IDX(s, i, j - 1, k)])) / dx;
        s->pe[FYN][1][w] = be * s->pe[FYN][1][w] + ce * ((HX(s)[c] - HX(s)[IDX(s, i, j - 1, k)])) / dz;
        if (!(i == 0 || k == 0) && xt == 0) EX(s)[c] += dx * cbx * s->pe[FYN][0][w];
        if (!(i == 0 || k == 0) && zt == 0) EZ(s)[c] -= dz * cbz * s->pe[FYN][1][w];
    }
    if (s->cp[FZN].enabled && (k >= (zr - s->cp[FZN].depth + 1)) && k < zr) {
        int kr = k - (zr - s->cp[FZN].depth);
        size_t w = slab_idx(s, FZN, i, j, kr);
        double be = s->be[FZN][kr], ce = s->ce[FZN][kr];
        s->pe[FZN][1][w] = be * s->pe[FZN][1][w] + ce * ((HX(s)[c] - HX(s)[IDX(s, i, j, k - 1)])) / dy;
        s->pe[FZN][0][w] = be * s->pe[FZN][0][w] + ce * ((HY(s)[c] - HY(s)[IDX(s, i, j, k - 1)])) / dx;
        if (!(i == 0 || j == 0) && yt == 0) EY(s)[c] += dy * cby * s->pe[FZN][1][w];
        if (!(i == 0 || j == 0) && xt == 0) EX(s)[c] -= dx * cbx * s->pe[FZN][0][w];
    }
}

/* ADE (Drude + 2 critical points) branch of ystep_e, yee.c:914-1108 */
static void ade_cell(oracle_state *s, int i, int j, int k, int m, double kx, double ky, double kz,
                     int xt, int yt, int zt)
{
    const fdtd_material *q = &s->mats[m];
    size_t c = IDX(s, i, j, k);
    const size_t sj = (size_t)s->zres, si = (size_t)s->yres * s->zres;
    double ve[3], vd[3], vp[3][2];
    int a, n;
    double *E[3] = {EX(s), EY(s), EZ(s)};
    const double dd[3] = {s->dx, s->dy, s->dz};
    int go[3];
    ve[0] = EX(s)[c]; ve[1] = EY(s)[c]; ve[2] = EZ(s)[c];
    go[0] = (j > 0 && k > 0 && xt == 0);
    go[1] = (i > 0 && k > 0 && yt == 0);
    go[2] = (i > 0 && j > 0 && zt == 0);
    for (a = 0; a < 3; a++) {
        double curl;
        if (!go[a]) continue;   /* the curl is only formed where its neighbours exist */
        if (a == 0) curl = (HZ(s)[c] - HZ(s)[c - sj]) / ky - (HY(s)[c] - HY(s)[c - 1]) / kz;
        else if (a == 1) curl = (HX(s)[c] - HX(s)[c - 1]) / kz - (HZ(s)[c] - HZ(s)[c - si]) / kx;
        else curl = (HY(s)[c] - HY(s)[c - si]) / kx - (HX(s)[c] - HX(s)[c - sj]) / ky;
        E[a][c] = q->ade_c0 * curl / dd[a]
                  + q->ade_c1 * (-q->ade_a0 * s->dpp[a][c] + (1 - q->ade_a1) * s->dp[a][c])
                  + q->ade_c1 * (-q->ade_bp0[0] * s->pp[a][0][c] + (1 - q->ade_bp1[0]) * s->p[a][0][c])
                  + q->ade_c1 * (-q->ade_bp0[1] * s->pp[a][1][c] + (1 - q->ade_bp1[1]) * s->p[a][1][c])
                  + q->ade_c2 * s->ep[a][c] + q->ade_c3 * E[a][c];
    }
    ade_cpml(s, i, j, k, q, 0.0, xt, yt, zt);
    for (a = 0; a < 3; a++) {
        vd[a] = s->dp[a][c];
        for (n = 0; n < 2; n++) vp[a][n] = s->p[a][n][c];
    }
    for (a = 0; a < 3; a++) {
        s->dp[a][c] = q->ade_a0 * s->dpp[a][c] + q->ade_a1 * s->dp[a][c] + q->ade_a2 * (s->ep[a][c] + 2 * ve[a] + E[a][c]);
        for (n = 0; n < 2; n++)
            s->p[a][n][c] = q->ade_bp0[n] * s->pp[a][n][c] + q->ade_bp1[n] * s->p[a][n][c] +
                            q->ade_bp2[n] * s->ep[a][c] + q->ade_bp3[n] * ve[a] + q->ade_bp4[n] * E[a][c];
    }
    for (a = 0; a < 3; a++) {
        s->ep[a][c] = ve[a];
        s->dpp[a][c] = vd[a];
        for (n = 0; n < 2; n++) s->pp[a][n][c] = vp[a][n];
    }
}

/* sv_yee_data_ystep_e, yee.c:530-1247 */
static void ystep_e(oracle_state *s)
{
    int i;
    const int xr = s->xres, yr = s->yres, zr = s->zres;
#pragma omp parallel for schedule(static)
    for (i = 0; i < xr; i++) {
        int j, k;
        const size_t sj = (size_t)zr, si = (size_t)yr * zr;
        for (j = 0; j < yr; j++)
            for (k = 0; k < zr; k++) {
                size_t c = IDX(s, i, j, k);
                double kx = 1, ky = 1, kz = 1, hx, hy, hz;
                int xt, yt, zt, m;
                if (s->cp[FX0].enabled && i < s->cp[FX0].depth) kx = fmax(kx, s->ke[FX0][i]);
                if (s->cp[FXN].enabled && i >= xr - s->cp[FXN].depth) kx = fmax(kx, s->ke[FXN][i - (xr - s->cp[FXN].depth)]);
                if (s->cp[FY0].enabled && j < s->cp[FY0].depth) ky = fmax(ky, s->ke[FY0][j]);
                if (s->cp[FYN].enabled && j >= yr - s->cp[FYN].depth) ky = fmax(ky, s->ke[FYN][j - (yr - s->cp[FYN].depth)]);
                if (s->cp[FZ0].enabled && k < s->cp[FZ0].depth) kz = fmax(kz, s->ke[FZ0][k]);
                if (s->cp[FZN].enabled && k >= zr - s->cp[FZN].depth) kz = fmax(kz, s->ke[FZN][k - (zr - s->cp[FZN].depth)]);
                hx = HX(s)[c]; hy = HY(s)[c]; hz = HZ(s)[c];
                m = get_tbc(s, i, j, k, &xt, &yt, &zt);
                if (s->nmat > 0 && s->disp && xt * yt * zt == 0)
                    ade_cell(s, i, j, k, m, kx, ky, kz, xt, yt, zt);
                if ((xt + yt + zt) != 0) {
                    double ca[3], cb[3];
                    get_cabs(s, i, j, k, ca, cb);
                    if (j > 0 && k > 0 && xt)
                        EX(s)[c] = ca[0] * EX(s)[c] + cb[0] * ((hz - HZ(s)[c - sj]) / ky - (hy - HY(s)[c - 1]) / kz);
                    if (i > 0 && k > 0 && yt)
                        EY(s)[c] = ca[1] * EY(s)[c] + cb[1] * ((hx - HX(s)[c - 1]) / kz - (hz - HZ(s)[c - si]) / kx);
                    if (i > 0 && j > 0 && zt)
                        EZ(s)[c] = ca[2] * EZ(s)[c] + cb[2] * ((hy - HY(s)[c - si]) / kx - (hx - HX(s)[c - sj]) / ky);
                }
                /* PEC tangential components, yee.c:1138-1237 (no SF source on this path) */
                if (m >= 0 && i > 0 && j > 0 && k > 0) {
                    const int *mt = s->mat;
                    int t0 = s->mats[mt[c]].type, tx = s->mats[mt[c - si]].type, ty = s->mats[mt[c - sj]].type;
                    int tz = s->mats[mt[c - 1]].type, txy = s->mats[mt[c - si - sj]].type;
                    int tyz = s->mats[mt[c - sj - 1]].type, txz = s->mats[mt[c - si - 1]].type;
                    int txyz = s->mats[mt[c - si - sj - 1]].type;
                    const int P = FDTD_MAT_PEC;
                    if (s->mats[m].type == P || tx == P || ty == P || tz == P || txy == P || tyz == P || txz == P || txyz == P) {
                        if ((tx != P && t0 == P) || (tx == P && t0 != P)) { EY(s)[c] = 0; EZ(s)[c] = 0; }
                        if ((ty != P && t0 == P) || (ty == P && t0 != P)) { EX(s)[c] = 0; EZ(s)[c] = 0; }
                        if ((tz != P && t0 == P) || (tz == P && t0 != P)) { EX(s)[c] = 0; EY(s)[c] = 0; }
                        if (txy == P && t0 != P) EZ(s)[c] = 0;
                        if (txz == P && t0 != P) EY(s)[c] = 0;
                        if (tyz == P && t0 != P) EX(s)[c] = 0;
                    }
                }
            }
    }
}

/* CPML part of sv_pool_boundary_estep, boundary.c:691-884 */
static void cpml_e(oracle_state *s)
{
    const int xr = s->xres, yr = s->yres, zr = s->zres;
    const double dx = s->dx, dy = s->dy, dz = s->dz;
    int i, j, k;
    if (s->cp[FX0].enabled) {
        for (j = 0; j < yr; j++)
            for (k = 0; k < zr; k++)
                EY(s)[IDX(s, 0, j, k)] = EZ(s)[IDX(s, 0, j, k)] = EX(s)[IDX(s, 0, j, k)] = 0;
        for (i = 1; i < s->cp[FX0].depth; i++) {
#pragma omp parallel for private(k) schedule(static)
            for (j = 0; j < yr; j++)
                for (k = 0; k < zr; k++) {
                    size_t c = IDX(s, i, j, k), w = slab_idx(s, FX0, i, j, k);
                    int xt, yt, zt;
                    double ca[3], cb[3], be = s->be[FX0][i], ce = s->ce[FX0][i];
                    get_tbc(s, i, j, k, &xt, &yt, &zt);
                    get_cabs(s, i, j, k, ca, cb);
                    s->pe[FX0][0][w] = be * s->pe[FX0][0][w] + ce * ((HZ(s)[c] - HZ(s)[IDX(s, i - 1, j, k)])) / dx;
                    s->pe[FX0][1][w] = be * s->pe[FX0][1][w] + ce * ((HY(s)[c] - HY(s)[IDX(s, i - 1, j, k)])) / dx;
                    if (!(j == 0 || k == 0) && yt == 1) EY(s)[c] -= dx * cb[1] * s->pe[FX0][0][w];
                    if (!(j == 0 || k == 0) && zt == 1) EZ(s)[c] += dx * cb[2] * s->pe[FX0][1][w];
                }
        }
    }
    if (s->cp[FY0].enabled) {
        for (i = 0; i < xr; i++)
            for (k = 0; k < zr; k++)
                EY(s)[IDX(s, i, 0, k)] = EZ(s)[IDX(s, i, 0, k)] = EX(s)[IDX(s, i, 0, k)] = 0;
        for (j = 1; j < s->cp[FY0].depth; j++) {
#pragma omp parallel for private(k) schedule(static)
            for (i = 0; i < xr; i++)
                for (k = 0; k < zr; k++) {
                    size_t c = IDX(s, i, j, k), w = slab_idx(s, FY0, i, j, k);
                    int xt, yt, zt;
                    double ca[3], cb[3], be = s->be[FY0][j], ce = s->ce[FY0][j];
                    get_tbc(s, i, j, k, &xt, &yt, &zt);
                    get_cabs(s, i, j, k, ca, cb);
                    s->pe[FY0][0][w] = be * s->pe[FY0][0][w] + ce * ((HZ(s)[c] - HZ(s)[IDX(s, i, j - 1, k)])) / dy;
                    s->pe[FY0][1][w] = be * s->pe[FY0][1][w] + ce * ((HX(s)[c] - HX(s)[IDX(s, i, j - 1, k)])) / dy;
                    if (!(i == 0 || k == 0) && xt == 1) EX(s)[c] += dy * cb[0] * s->pe[FY0][0][w];
                    if (!(i == 0 || k == 0) && zt == 1) EZ(s)[c] -= dy * cb[2] * s->pe[FY0][1][w];
                }
        }
    }
    if (s->cp[FZ0].enabled) {
        for (i = 0; i < xr; i++)
            for (j = 0; j < yr; j++)
                EY(s)[IDX(s, i, j, 0)] = EZ(s)[IDX(s, i, j, 0)] = EX(s)[IDX(s, i, j, 0)] = 0;
        for (k = 1; k < s->cp[FZ0].depth; k++) {
#pragma omp parallel for private(j) schedule(static)
            for (i = 0; i < xr; i++)
                for (j = 0; j < yr; j++) {
                    size_t c = IDX(s, i, j, k), w = slab_idx(s, FZ0, i, j, k);
                    int xt, yt, zt;
                    double ca[3], cb[3], be = s->be[FZ0][k], ce = s->ce[FZ0][k];
                    get_tbc(s, i, j, k, &xt, &yt, &zt);
                    get_cabs(s, i, j, k, ca, cb);
                    s->pe[FZ0][1][w] = be * s->pe[FZ0][1][w] + ce * ((HX(s)[c] - HX(s)[IDX(s, i, j, k - 1)])) / dz;
                    s->pe[FZ0][0][w] = be * s->pe[FZ0][0][w] + ce * ((HY(s)[c] - HY(s)[IDX(s, i, j, k - 1)])) / dz;
                    if (!(i == 0 || j == 0) && yt == 1) EY(s)[c] += dx * cb[1] * s->pe[FZ0][1][w];
                    if (!(i == 0 || j == 0) && zt == 1) EX(s)[c] -= dx * cb[0] * s->pe[FZ0][0][w];
                }
        }
    }
    if (s->cp[FXN].enabled) {
        int d = s->cp[FXN].depth;
        for (i = xr - d + 1; i < xr; i++) {
            int ir = i - (xr - d);
#pragma omp parallel for private(k) schedule(static)
            for (j = 0; j < yr; j++)
                for (k = 0; k < zr; k++) {
                    size_t c = IDX(s, i, j, k), w = slab_idx(s, FXN, ir, j, k);
                    int xt, yt, zt;
                    double ca[3], cb[3], be = s->be[FXN][ir], ce = s->ce[FXN][ir];
                    get_tbc(s, i, j, k, &xt, &yt, &zt);
                    get_cabs(s, i, j, k, ca, cb);
                    s->pe[FXN][0][w] = be * s->pe[FXN][0][w] + ce * ((HZ(s)[c] - HZ(s)[IDX(s, i - 1, j, k)])) / dx;
                    s->pe[FXN][1][w] = be * s->pe[FXN][1][w] + ce * ((HY(s)[c] - HY(s)[IDX(s, i - 1, j, k)])) / dx;
                    if (!(j == 0 || k == 0) && yt == 1) EY(s)[c] -= dx * cb[1] * s->pe[FXN][0][w];
                    if (!(j == 0 || k == 0) && zt == 1) EZ(s)[c] += dx * cb[2] * s->pe[FXN][1][w];
                }
        }
    }
    if (s->cp[FYN].enabled) {
        int d = s->cp[FYN].depth;
        for (j = yr - d + 1; j < yr; j++) {
            int jr = j - (yr - d);
#pragma omp parallel for private(k) schedule(static)
            for (i = 0; i < xr; i++)
                for (k = 0; k < zr; k++) {
                    size_t c = IDX(s, i, j, k), w = slab_idx(s, FYN, i, jr, k);
                    int xt, yt, zt;
                    double ca[3], cb[3], be = s->be[FYN][jr], ce = s->ce[FYN][jr];
                    get_tbc(s, i, j, k, &xt, &yt, &zt);
                    get_cabs(s, i, j, k, ca, cb);
                    s->pe[FYN][0][w] = be * s->pe[FYN][0][w] + ce * ((HZ(s)[c] - HZ(s)[IDX(s, i, j - 1, k)])) / dy;
                    s->pe[FYN][1][w] = be * s->pe[FYN][1][w] + ce * ((HX(s)[c] - HX(s)[IDX(s, i, j - 1, k)])) / dy;
                    if (!(i == 0 || k == 0) && xt == 1) EX(s)[c] += dy * cb[0] * s->pe[FYN][0][w];
                    if (!(i == 0 || k == 0) && zt == 1) EZ(s)[c] -= dy * cb[2] * s->pe[FYN][1][w];
                }
        }
    }
    if (s->cp[FZN].enabled) {
        int d = s->cp[FZN].depth;
        for (k = zr - d + 1; k < zr; k++) {
            int kr = k - (zr - d);
#pragma omp parallel for private(j) schedule(static)
            for (i = 0; i < xr; i++)
                for (j = 0; j < yr; j++) {
                    size_t c = IDX(s, i, j, k), w = slab_idx(s, FZN, i, j, kr);
                    int xt, yt, zt;
                    double ca[3], cb[3], be = s->be[FZN][kr], ce = s->ce[FZN][kr];
                    get_tbc(s, i, j, k, &xt, &yt, &zt);
                    get_cabs(s, i, j, k, ca, cb);
                    s->pe[FZN][1][w] = be * s->pe[FZN][1][w] + ce * ((HX(s)[c] - HX(s)[IDX(s, i, j, k - 1)])) / dz;
                    s->pe[FZN][0][w] = be * s->pe[FZN][0][w] + ce * ((HY(s)[c] - HY(s)[IDX(s, i, j, k - 1)])) / dz;
                    if (!(i == 0 || j == 0) && yt == 1) EY(s)[c] += dx * cb[1] * s->pe[FZN][1][w];
                    if (!(i == 0 || j == 0) && xt == 1) EX(s)[c] -= dx * cb[0] * s->pe[FZN][0][w];
                }
        }
    }
}

/* ----------------------------------------------------------- far field */

/* sv_pool_farfield, farfield.c:175-405 (time-domain Kirchhoff, E only) */
static void farfield(oracle_state *s)
{
    int n;
    const int i0 = s->ff.i0, i1 = s->ff.in, j0 = s->ff.j0, j1 = s->ff.jn, k0 = s->ff.k0, k1 = s->ff.kn;
    const int ix = i1 - i0, iy = j1 - j0, iz = k1 - k0;
    const double dx = s->dx, dy = s->dy, dz = s->dz, dt = s->dt;
    const int nd = s->ndata;
#pragma omp parallel for schedule(dynamic)
    for (n = 0; n < s->ff.npoints; n++) {
        double *F[3];
        const double *E[3] = {EX(s), EY(s), EZ(s)};
        int a, f;
        for (a = 0; a < 3; a++) F[a] = s->ffser + ((size_t)n * 3 + a) * nd;
        /* face order of the reference: x (i0,i1), y (j0,j1), z (k0,k1) */
        for (f = 0; f < 3; f++) {
            int ua, ub, na, nb;
            double size = (f == 0) ? dy * dz : (f == 1) ? dx * dz : dx * dy;
            if (f == 0) { na = iy; nb = iz; } else if (f == 1) { na = ix; nb = iz; } else { na = ix; nb = iy; }
            for (ua = 0; ua < na; ua++)
                for (ub = 0; ub < nb; ub++) {
                    int side;
                    for (side = 0; side < 2; side++) {
                        int face = 2 * f + side;
                        int lo0, lo1, pos, ci, cj, ck;
                        size_t tab = (size_t)n * (size_t)na * nb + (size_t)ua * nb + ub;
                        double r, ct, a1, b1, c1;
                        int nn;
                        size_t cc, cp, cm;
                        if (f == 0) { ci = side ? i1 : i0; cj = j0 + ua; ck = k0 + ub; lo0 = cj; lo1 = ck; }
                        else if (f == 1) { ci = i0 + ua; cj = side ? j1 : j0; ck = k0 + ub; lo0 = ci; lo1 = ck; }
                        else { ci = i0 + ua; cj = j0 + ub; ck = side ? k1 : k0; lo0 = ci; lo1 = cj; }
                        if (s->ff.skip[face] && lo0 >= s->ff.skip_lo[face][0] && lo1 >= s->ff.skip_lo[face][1] &&
                            lo0 <= s->ff.skip_hi[face][0] && lo1 <= s->ff.skip_hi[face][1])
                            continue;
                        r = s->ffr[face][tab] * dx;
                        ct = s->ffct[face][tab];
                        nn = (int)(s->step + 1 + r / (C0 * dt)) - s->ffistart[n];
                        if (nn < 3 || nn >= nd)
                            continue;
                        a1 = 1.0 / (4.0 * PI_D * r);
                        b1 = -1.0 / (4.0 * PI_D) * ct / (r * r);
                        c1 = -1.0 / (4.0 * PI_D) * ct / (C0 * r);
                        cc = IDX(s, ci, cj, ck);
                        if (f == 0) { cp = IDX(s, ci + 1, cj, ck); cm = IDX(s, ci - 1, cj, ck); }
                        else if (f == 1) { cp = IDX(s, ci, cj + 1, ck); cm = IDX(s, ci, cj - 1, ck); }
                        else { cp = IDX(s, ci, cj, ck + 1); cm = IDX(s, ci, cj, ck - 1); }
                        pos = side ? 1 : -1;
                        for (a = 0; a < 3; a++) {
                            F[a][nn] += -c1 / 2.0 / dt * E[a][cc] * size;
                            F[a][nn - 1] += (pos * a1 * (E[a][cp] - E[a][cm]) / 2.0 / dx + b1 * E[a][cc]) * size;
                            F[a][nn - 2] += c1 / 2.0 / dt * E[a][cc] * size;
                        }
                    }
                }
        }
    }
}

/* ------------------------------------------------------------- driver */

int oracle_step(oracle_state *s, int nsteps)
{
    int it, p;
    for (it = 0; it < nsteps; it++) {
        ystep_h(s);
        if (s->tsf) tsf_h(s);
        cpml_h(s);
        ystep_e(s);
        cpml_e(s);
        if (s->tsf) tsf_e(s);
        if (s->nfff) farfield(s);
        if (s->step < s->nsteps_planned)
            for (p = 0; p < s->nprobes; p++) {
                size_t c = IDX(s, s->probes[3 * p], s->probes[3 * p + 1], s->probes[3 * p + 2]);
                double *o = s->probe_out + ((size_t)p * s->nsteps_planned + s->step) * 6;
                int a;
                for (a = 0; a < 6; a++) o[a] = s->f[a][c];
            }
        s->step++;
    }
    return 0;
}

int oracle_get_fields(const oracle_state *s, double *ex, double *ey, double *ez, double *hx, double *hy, double *hz)
{
    double *o[6] = {ex, ey, ez, hx, hy, hz};
    int a;
    for (a = 0; a < 6; a++)
        if (o[a]) memcpy(o[a], s->f[a], sizeof(double) * s->n);
    return 0;
}

int oracle_set_fields(oracle_state *s, const double *ex, const double *ey, const double *ez,
                      const double *hx, const double *hy, const double *hz)
{
    const double *o[6] = {ex, ey, ez, hx, hy, hz};
    int a;
    for (a = 0; a < 6; a++)
        if (o[a]) memcpy(s->f[a], o[a], sizeof(double) * s->n);
    return 0;
}

int oracle_get_map(const oracle_state *s, int which, int32_t *out)
{
    if (which == FDTD_MAP_MAT) {
        if (s->mat) memcpy(out, s->mat, sizeof(int32_t) * s->n);
        else { size_t c; for (c = 0; c < s->n; c++) out[c] = -1; }
    } else if (which == FDTD_MAP_BNDS)
        memcpy(out, s->bnds, sizeof(int32_t) * s->n);
    else if (which == FDTD_MAP_SOURCESKIP)
        memcpy(out, s->sskip, sizeof(int32_t) * s->n);
    else
        return -1;
    return 0;
}

int oracle_get_probes(const oracle_state *s, double *out)
{
    if (s->nprobes > 0)
        memcpy(out, s->probe_out, sizeof(double) * (size_t)s->nprobes * 6 * (size_t)s->nsteps_planned);
    return 0;
}

int oracle_nfff_ndata(const oracle_state *s) { return s->nfff ? s->ndata : 0; }

int oracle_get_nfff_series(const oracle_state *s, double *out)
{
    if (!s->nfff) return -1;
    memcpy(out, s->ffser, sizeof(double) * (size_t)s->ff.npoints * 3 * (size_t)s->ndata);
    return 0;
}

int oracle_get_nfff_istart(const oracle_state *s, int32_t *out)
{
    if (!s->nfff) return -1;
    memcpy(out, s->ffistart, sizeof(int32_t) * (size_t)s->ff.npoints);
    return 0;
}

int oracle_aux_res(const oracle_state *s) { return s->tsf ? s->jres : 0; }

int oracle_get_aux(const oracle_state *s, double *e, double *h)
{
    if (!s->tsf) return -1;
    memcpy(e, s->je, sizeof(double) * (size_t)s->jres);
    memcpy(h, s->jh, sizeof(double) * (size_t)s->jres);
    return 0;
}

int oracle_get_step(const oracle_state *s) { return s->step; }

/* ------------------------------------------------- linear-step coefficients */

/* The coefficients of the source-free step as the loops above apply them,
 * for the FP64 adjoint restatement (oracle/adjoint.py).  Per cell c (N cells,
 * component a): ca[a*N + c], cb[a*N + c] (get_cabs, yee.c:1397-1493), da[c],
 * db[c] (ystep_h, yee.c:219-243), flags[c]: bits 0-2 the tbc of get_tbc,
 * bits 3-5 the components the PEC rule of ystep_e zeroes (yee.c:1138-1237),
 * bit 6 a cell of the dispersive branch. */
int oracle_get_coeffs(const oracle_state *s, double *ca, double *cb, double *da, double *db, int32_t *flags)
{
    const int xr = s->xres, yr = s->yres, zr = s->zres;
    const size_t N = (size_t)xr * yr * zr, sj = (size_t)zr, si = (size_t)yr * zr;
    int i, j, k;
    for (i = 0; i < xr; i++)
        for (j = 0; j < yr; j++)
            for (k = 0; k < zr; k++) {
                size_t c = IDX(s, i, j, k);
                double a3[3], b3[3], dt = s->dt;
                int xt, yt, zt, m, f = 0, a;
                m = matidx(s, i, j, k);
                if (m > 0 && is_tab(s->mats[m].type)) {
                    const fdtd_material *q = &s->mats[m];
                    da[c] = (1 - q->sigast * dt / 2 / q->mu) / (1 + q->sigast * dt / 2 / q->mu);
                    db[c] = (dt / q->mu / s->dx) / (1 + q->sigast * dt / 2 / q->mu);
                } else if (s->matmode == FDTD_MATMODE_FULL || s->matmode == FDTD_MATMODE_MAGNETIC) {
                    double mu = s->vmu[c], sa = s->vsigast[c];
                    da[c] = (1 - sa * dt / 2 / mu) / (1 + sa * dt / 2 / mu);
                    db[c] = (dt / mu / s->dx) / (1 + sa * dt / 2 / mu);
                } else {
                    da[c] = 1;
                    db[c] = dt / MU0 / s->dx;
                }
                m = get_tbc(s, i, j, k, &xt, &yt, &zt);
                get_cabs(s, i, j, k, a3, b3);
                for (a = 0; a < 3; a++) { ca[a * N + c] = a3[a]; cb[a * N + c] = b3[a]; }
                f = (xt ? 1 : 0) | (yt ? 2 : 0) | (zt ? 4 : 0);
                if (s->nmat > 0 && s->disp && xt * yt * zt == 0) f |= 64;
                if (m >= 0 && i > 0 && j > 0 && k > 0) {
                    const int *mt = s->mat;
                    int t0 = s->mats[mt[c]].type, tx = s->mats[mt[c - si]].type, ty = s->mats[mt[c - sj]].type;
                    int tz = s->mats[mt[c - 1]].type, txy = s->mats[mt[c - si - sj]].type;
                    int tyz = s->mats[mt[c - sj - 1]].type, txz = s->mats[mt[c - si - 1]].type;
                    int txyz = s->mats[mt[c - si - sj - 1]].type;
                    const int P = FDTD_MAT_PEC;
                    if (s->mats[m].type == P || tx == P || ty == P || tz == P || txy == P || tyz == P || txz == P || txyz == P) {
                        if ((tx != P && t0 == P) || (tx == P && t0 != P)) f |= 16 | 32;
                        if ((ty != P && t0 == P) || (ty == P && t0 != P)) f |= 8 | 32;
                        if ((tz != P && t0 == P) || (tz == P && t0 != P)) f |= 8 | 16;
                        if (txy == P && t0 != P) f |= 32;
                        if (txz == P && t0 != P) f |= 16;
                        if (tyz == P && t0 != P) f |= 8;
                    }
                }
                flags[c] = f;
            }
    return 0;
}

/* The material whose ADE coefficients the dispersive branch of a cell uses
 * (get_tbc, yee.c:454-526), or -1 where the cell is outside that branch. */
int oracle_get_ade_mat(const oracle_state *s, int32_t *out)
{
    const int xr = s->xres, yr = s->yres, zr = s->zres;
    int i, j, k;
    for (i = 0; i < xr; i++)
        for (j = 0; j < yr; j++)
            for (k = 0; k < zr; k++) {
                int xt, yt, zt;
                const int m = get_tbc(s, i, j, k, &xt, &yt, &zt);
                out[IDX(s, i, j, k)] = (s->nmat > 0 && s->disp && xt * yt * zt == 0) ? m : -1;
            }
    return 0;
}

/* CPML profiles of one face (cpml_grade): depth entries each; returns the
 * depth, 0 for a disabled face. */
int oracle_get_cpml(const oracle_state *s, int face, double *be, double *ce, double *bh, double *ch, double *ke, double *kh)
{
    int i, d;
    if (face < 0 || face > 5 || !s->cp[face].enabled)
        return 0;
    d = s->cp[face].depth;
    for (i = 0; i < d; i++) {
        be[i] = s->be[face][i]; ce[i] = s->ce[face][i];
        bh[i] = s->bh[face][i]; ch[i] = s->ch[face][i];
        ke[i] = s->ke[face][i]; kh[i] = s->kh[face][i];
    }
    return d;
}

/* Transpose of farfield() for the E set of the step whose far-field call saw
 * s->step == step: for the far points pts[0..npts), out[a*N + c] += the sum
 * over the taps of farfield() that read E[a][c] of their coefficient times
 * lam[(p*3 + a)*ndata + m] (lam = dJ/dF of the time-domain series). */
int oracle_farfield_transpose(const oracle_state *s, int step, int npts, const int32_t *pts, const double *lam, double *out)
{
    const int i0 = s->ff.i0, i1 = s->ff.in, j0 = s->ff.j0, j1 = s->ff.jn, k0 = s->ff.k0, k1 = s->ff.kn;
    const int ix = i1 - i0, iy = j1 - j0, iz = k1 - k0;
    const double dx = s->dx, dy = s->dy, dz = s->dz, dt = s->dt;
    const int nd = s->ndata;
    const size_t N = (size_t)s->xres * s->yres * s->zres;
    int t;
    if (!s->nfff) return -1;
    for (t = 0; t < npts; t++) {
        const int n = pts[t];
        int f;
        for (f = 0; f < 3; f++) {
            int ua, ub, na, nb;
            double size = (f == 0) ? dy * dz : (f == 1) ? dx * dz : dx * dy;
            if (f == 0) { na = iy; nb = iz; } else if (f == 1) { na = ix; nb = iz; } else { na = ix; nb = iy; }
            for (ua = 0; ua < na; ua++)
                for (ub = 0; ub < nb; ub++) {
                    int side;
                    for (side = 0; side < 2; side++) {
                        int face = 2 * f + side;
                        int lo0, lo1, pos, ci, cj, ck, a, nn;
                        size_t tab = (size_t)n * (size_t)na * nb + (size_t)ua * nb + ub;
                        double r, ct, a1, b1, c1;
                        size_t cc, cp, cm;
                        if (f == 0) { ci = side ? i1 : i0; cj = j0 + ua; ck = k0 + ub; lo0 = cj; lo1 = ck; }
                        else if (f == 1) { ci = i0 + ua; cj = side ? j1 : j0; ck = k0 + ub; lo0 = ci; lo1 = ck; }
                        else { ci = i0 + ua; cj = j0 + ub; ck = side ? k1 : k0; lo0 = ci; lo1 = cj; }
                        if (s->ff.skip[face] && lo0 >= s->ff.skip_lo[face][0] && lo1 >= s->ff.skip_lo[face][1] &&
                            lo0 <= s->ff.skip_hi[face][0] && lo1 <= s->ff.skip_hi[face][1])
                            continue;
                        r = s->ffr[face][tab] * dx;
                        ct = s->ffct[face][tab];
                        nn = (int)(step + 1 + r / (C0 * dt)) - s->ffistart[n];
                        if (nn < 3 || nn >= nd)
                            continue;
                        a1 = 1.0 / (4.0 * PI_D * r);
                        b1 = -1.0 / (4.0 * PI_D) * ct / (r * r);
                        c1 = -1.0 / (4.0 * PI_D) * ct / (C0 * r);
                        cc = IDX(s, ci, cj, ck);
                        if (f == 0) { cp = IDX(s, ci + 1, cj, ck); cm = IDX(s, ci - 1, cj, ck); }
                        else if (f == 1) { cp = IDX(s, ci, cj + 1, ck); cm = IDX(s, ci, cj - 1, ck); }
                        else { cp = IDX(s, ci, cj, ck + 1); cm = IDX(s, ci, cj, ck - 1); }
                        pos = side ? 1 : -1;
                        for (a = 0; a < 3; a++) {
                            const double *L = lam + ((size_t)n * 3 + a) * nd;
                            out[a * N + cc] += (-c1 / 2.0 / dt * L[nn] + b1 * L[nn - 1] + c1 / 2.0 / dt * L[nn - 2]) * size;
                            out[a * N + cp] += pos * a1 / 2.0 / dx * L[nn - 1] * size;
                            out[a * N + cm] -= pos * a1 / 2.0 / dx * L[nn - 1] * size;
                        }
                    }
                }
        }
    }
    return 0;
}
