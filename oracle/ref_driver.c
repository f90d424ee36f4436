/*
 * ref_driver.c -- drives GSvit's own CPU solver sources (compiled unmodified
 * from the reference tree against oracle/shim) from an fdtd_desc.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into
 * oracle/_ref/libgsvit_ref.so together with src3d/{yee,boundary,source,1dpool,
 * dline,farfield,dcube,fcube,icube,pool,zpool}.c; never part of the product.
 *
 * plan.c itself needs GL/Gwyddion/FFTW and does not build here, so the few
 * planner steps the stepping code depends on are restated (each cited):
 * material table and maps, ADE array allocation (plan.c:4013-4060), the
 * interface map bnds (plan.c:5387-5416), the TSF skip map (plan.c:5298-5326,
 * eval_closecheck plan.c:3857-3873) and the TSF set-up (plan.c:1522-1597).
 * Everything inside the step (sv_yee_data_ystep_h/e, sv_pool_boundary_*step,
 * sv_pool_apply_source_*step, sv_1dpool_*, sv_dline_get_dval,
 * sv_pool_farfield, sv_boundary_new, sv_farfield_new, ...) is the reference's
 * own compiled code, called in the CPU order of svit.c:217-237.
 */
#include <math.h>
#include <string.h>

#include "pool.h"
#include "yee.h"
#include "constants.h"
#include "1dpool.h"
#include "../include/gsvit_b200.h"

/* symbols referenced by pool.c / source.c whose subsystems are not built */
SvOutput *sv_output_new(void)
{
    SvOutput *o = (SvOutput *)g_malloc0(sizeof(SvOutput));
    return o;
}
SvPFarfield *sv_pfarfield_new(SvPool *mp, SvSet *set) { (void)mp; (void)set; return NULL; }
SvSubgrid *sv_subgrid_new(SvPool *mp, SvSet *set) { (void)mp; (void)set; return NULL; }
int sv_pool_subgrid_copy(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_subgrid_step(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }

typedef struct ref_state {
    SvSet *set;
    SvPool *mp;
    int nprobes, nsteps;
    int32_t *probes;
    double *probe_out;
    int nfff;
} ref_state;

static void err_set(char *err, const char *m)
{
    if (err) { strncpy(err, m, 255); err[255] = 0; }
}

static SvDCube *cube(SvYeeData *d)
{
    return sv_dcube_new(d->xres, d->yres, d->zres, d->xres * d->dx, d->yres * d->dy, d->zres * d->dz, 1);
}

/* allocate_ade, plan.c:4013-4060 (arrays only) */
static void alloc_ade(SvYeeData *d)
{
    int j;
    d->exp = cube(d); d->eyp = cube(d); d->ezp = cube(d);
    d->dpxp = g_malloc(sizeof(SvDCube *)); d->dpyp = g_malloc(sizeof(SvDCube *)); d->dpzp = g_malloc(sizeof(SvDCube *));
    d->dpx = g_malloc(sizeof(SvDCube *)); d->dpy = g_malloc(sizeof(SvDCube *)); d->dpz = g_malloc(sizeof(SvDCube *));
    d->dpxp[0] = cube(d); d->dpyp[0] = cube(d); d->dpzp[0] = cube(d);
    d->dpx[0] = cube(d); d->dpy[0] = cube(d); d->dpz[0] = cube(d);
    d->pxp = g_malloc(2 * sizeof(SvDCube *)); d->pyp = g_malloc(2 * sizeof(SvDCube *)); d->pzp = g_malloc(2 * sizeof(SvDCube *));
    d->px = g_malloc(2 * sizeof(SvDCube *)); d->py = g_malloc(2 * sizeof(SvDCube *)); d->pz = g_malloc(2 * sizeof(SvDCube *));
    for (j = 0; j < 2; j++) {
        d->pxp[j] = cube(d); d->pyp[j] = cube(d); d->pzp[j] = cube(d);
        d->px[j] = cube(d); d->py[j] = cube(d); d->pz[j] = cube(d);
    }
}

static SvBoundaryType btype(const fdtd_cpml_face *f) { return f->enabled ? SV_BOUNDARY_CPML : SV_BOUNDARY_NONE; }

ref_state *ref_create(const fdtd_desc *desc, char *err)
{
    ref_state *r;
    SvSet *set;
    SvPool *mp;
    SvYeeData *d;
    int i, j, k, n;
    if (!desc || desc->abi_version != FDTD_ABI_VERSION) { err_set(err, "bad descriptor"); return NULL; }
    r = (ref_state *)g_malloc0(sizeof(ref_state));
    set = r->set = (SvSet *)g_malloc0(sizeof(SvSet));
    set->sp.xres = desc->xres; set->sp.yres = desc->yres; set->sp.zres = desc->zres;
    set->sp.dx = desc->dx; set->sp.dy = desc->dy; set->sp.dz = desc->dz;
    set->sc.nsteps = desc->nsteps;
    set->sc.step_act = 0;
    set->sc.verbose = 0;
    set->sc.usegpu = 0;
    set->plan.dt = desc->dt;
    set->plan.matmode = (SvMatMode)desc->matmode;
    set->plan.gpumode = SV_GPUMODE_NONE;
    set->sb.bx0 = btype(&desc->cpml[FDTD_FACE_X0]); set->sb.bxn = btype(&desc->cpml[FDTD_FACE_XN]);
    set->sb.by0 = btype(&desc->cpml[FDTD_FACE_Y0]); set->sb.byn = btype(&desc->cpml[FDTD_FACE_YN]);
    set->sb.bz0 = btype(&desc->cpml[FDTD_FACE_Z0]); set->sb.bzn = btype(&desc->cpml[FDTD_FACE_ZN]);
#define SETF(F, S) do { const fdtd_cpml_face *c = &desc->cpml[F]; set->sb.depth_##S = c->depth; set->sb.m_##S = c->m; \
        set->sb.sigma_##S = c->sigma; set->sb.a_##S = c->a; set->sb.kappa_##S = c->kappa; } while (0)
    SETF(FDTD_FACE_X0, bx0); SETF(FDTD_FACE_XN, bxn); SETF(FDTD_FACE_Y0, by0);
    SETF(FDTD_FACE_YN, byn); SETF(FDTD_FACE_Z0, bz0); SETF(FDTD_FACE_ZN, bzn);
#undef SETF
    set->smb.bx0 = set->smb.bxn = set->smb.by0 = set->smb.byn = set->smb.bz0 = set->smb.bzn = SV_BOUNDARY_NONE;
    set->ss.tsf.box_boundary_skipdepth = desc->tsf.enabled ? desc->tsf.skipdepth : -1;
    set->ss.ltsf.box_boundary_skipdepth = -1;
    set->ss.npnts = 0;
    set->ss.nlocals = 0;
    if (desc->tsf.enabled) {
        set->ss.tsf.valid = 1;
        set->ss.tsf.box_i0 = desc->tsf.i0; set->ss.tsf.box_j0 = desc->tsf.j0; set->ss.tsf.box_k0 = desc->tsf.k0;
        set->ss.tsf.box_in = desc->tsf.in; set->ss.tsf.box_jn = desc->tsf.jn; set->ss.tsf.box_kn = desc->tsf.kn;
        set->ss.tsf.box_boundary_skipi0 = desc->tsf.skip[FDTD_FACE_X0];
        set->ss.tsf.box_boundary_skipin = desc->tsf.skip[FDTD_FACE_XN];
        set->ss.tsf.box_boundary_skipj0 = desc->tsf.skip[FDTD_FACE_Y0];
        set->ss.tsf.box_boundary_skipjn = desc->tsf.skip[FDTD_FACE_YN];
        set->ss.tsf.box_boundary_skipk0 = desc->tsf.skip[FDTD_FACE_Z0];
        set->ss.tsf.box_boundary_skipkn = desc->tsf.skip[FDTD_FACE_ZN];
        set->ss.tsf.ia_theta = desc->tsf.theta; set->ss.tsf.ia_phi = desc->tsf.phi; set->ss.tsf.ia_psi = desc->tsf.psi;
        set->ss.tsf.layered_epsilon = desc->tsf.layered_epsilon;
        set->ss.tsf.layered_mu = desc->tsf.layered_mu;
    }
    /* far field settings */
    if (desc->nfff.enabled && desc->nfff.npoints > 0) {
        const fdtd_nfff *f = &desc->nfff;
        r->nfff = 1;
        set->sf.box_i0 = f->i0; set->sf.box_in = f->in; set->sf.box_j0 = f->j0;
        set->sf.box_jn = f->jn; set->sf.box_k0 = f->k0; set->sf.box_kn = f->kn;
        set->sf.nrs = f->npoints;
        set->sf.ri = g_malloc(sizeof(gint) * f->npoints);
        set->sf.rj = g_malloc(sizeof(gint) * f->npoints);
        set->sf.rk = g_malloc(sizeof(gint) * f->npoints);
        set->sf.individual = g_malloc0(sizeof(gint) * f->npoints);
        for (n = 0; n < f->npoints; n++) {
            set->sf.ri[n] = f->points[3 * n]; set->sf.rj[n] = f->points[3 * n + 1]; set->sf.rk[n] = f->points[3 * n + 2];
        }
        set->sf.box_boundary_skipi0 = f->skip[FDTD_FACE_X0];
        set->sf.skipi0_jmin = f->skip_lo[FDTD_FACE_X0][0]; set->sf.skipi0_kmin = f->skip_lo[FDTD_FACE_X0][1];
        set->sf.skipi0_jmax = f->skip_hi[FDTD_FACE_X0][0]; set->sf.skipi0_kmax = f->skip_hi[FDTD_FACE_X0][1];
        set->sf.box_boundary_skipin = f->skip[FDTD_FACE_XN];
        set->sf.skipin_jmin = f->skip_lo[FDTD_FACE_XN][0]; set->sf.skipin_kmin = f->skip_lo[FDTD_FACE_XN][1];
        set->sf.skipin_jmax = f->skip_hi[FDTD_FACE_XN][0]; set->sf.skipin_kmax = f->skip_hi[FDTD_FACE_XN][1];
        set->sf.box_boundary_skipj0 = f->skip[FDTD_FACE_Y0];
        set->sf.skipj0_imin = f->skip_lo[FDTD_FACE_Y0][0]; set->sf.skipj0_kmin = f->skip_lo[FDTD_FACE_Y0][1];
        set->sf.skipj0_imax = f->skip_hi[FDTD_FACE_Y0][0]; set->sf.skipj0_kmax = f->skip_hi[FDTD_FACE_Y0][1];
        set->sf.box_boundary_skipjn = f->skip[FDTD_FACE_YN];
        set->sf.skipjn_imin = f->skip_lo[FDTD_FACE_YN][0]; set->sf.skipjn_kmin = f->skip_lo[FDTD_FACE_YN][1];
        set->sf.skipjn_imax = f->skip_hi[FDTD_FACE_YN][0]; set->sf.skipjn_kmax = f->skip_hi[FDTD_FACE_YN][1];
        set->sf.box_boundary_skipk0 = f->skip[FDTD_FACE_Z0];
        set->sf.skipk0_imin = f->skip_lo[FDTD_FACE_Z0][0]; set->sf.skipk0_jmin = f->skip_lo[FDTD_FACE_Z0][1];
        set->sf.skipk0_imax = f->skip_hi[FDTD_FACE_Z0][0]; set->sf.skipk0_jmax = f->skip_hi[FDTD_FACE_Z0][1];
        set->sf.box_boundary_skipkn = f->skip[FDTD_FACE_ZN];
        set->sf.skipkn_imin = f->skip_lo[FDTD_FACE_ZN][0]; set->sf.skipkn_jmin = f->skip_lo[FDTD_FACE_ZN][1];
        set->sf.skipkn_imax = f->skip_hi[FDTD_FACE_ZN][0]; set->sf.skipkn_jmax = f->skip_hi[FDTD_FACE_ZN][1];
    }

    /* pool: sv_pool_new + the parts of sv_pool_allocate (pool.c:62-73) on this path */
    mp = r->mp = sv_pool_new(set);
    mp->set = set;
    sv_yee_data_allocate(mp->d, set, set->sp.xres, set->sp.yres, set->sp.zres, set->sp.dx, set->sp.dy, set->sp.dz);
    d = mp->d;
    d->sourceskip = NULL;   /* sv_yee_data_new leaves it unset (yee.c:43-78) */
    mp->bnd = sv_boundary_new(mp, set);
    mp->farfield = r->nfff ? sv_farfield_new(mp, set) : NULL;
    if (r->nfff) {
        sv_pool_farfield_allocate_storage(mp, set);
        if (desc->nfff.istart)
            for (n = 0; n < desc->nfff.npoints; n++)
                mp->farfield->rpoints[n].istart = desc->nfff.istart[n];
    }
    /* materials */
    mp->nmat = desc->nmat;
    if (desc->nmat > 0) {
        int ade = 0;
        mp->mats = (SvMatProp *)g_malloc0(sizeof(SvMatProp) * desc->nmat);
        for (n = 0; n < desc->nmat; n++) {
            const fdtd_material *s = &desc->mats[n];
            SvMatProp *q = &mp->mats[n];
            q->type = s->type; q->epsilon = s->epsilon; q->mu = s->mu; q->sigma = s->sigma; q->sigast = s->sigast;
            q->drude_omega_p = s->drude_omega_p; q->drude_nu = s->drude_nu;
            for (i = 0; i < 2; i++) {
                q->cp3_a[i] = s->cp_a[i]; q->cp3_phi[i] = s->cp_phi[i];
                q->cp3_omega[i] = s->cp_omega[i]; q->cp3_gamma[i] = s->cp_gamma[i];
                q->ade_bp0[i] = s->ade_bp0[i]; q->ade_bp1[i] = s->ade_bp1[i]; q->ade_bp2[i] = s->ade_bp2[i];
                q->ade_bp3[i] = s->ade_bp3[i]; q->ade_bp4[i] = s->ade_bp4[i];
            }
            q->ade_a0 = s->ade_a0; q->ade_a1 = s->ade_a1; q->ade_a2 = s->ade_a2;
            q->ade_c0 = s->ade_c0; q->ade_c1 = s->ade_c1; q->ade_c2 = s->ade_c2; q->ade_c3 = s->ade_c3;
            q->pos = n;
            if (n > 0 && s->type == FDTD_MAT_ADE) ade = 1;
            if (n > 0 && s->type != FDTD_MAT_LINTAB && s->type != FDTD_MAT_ADE && s->type != FDTD_MAT_PEC) {
                err_set(err, "material type outside the driven path");
                return NULL;
            }
        }
        d->mat = sv_icube_new(d->xres, d->yres, d->zres, d->xres * d->dx, d->yres * d->dy, d->zres * d->dz, 1);
        for (i = 0; i < d->xres; i++)
            for (j = 0; j < d->yres; j++)
                for (k = 0; k < d->zres; k++)
                    d->mat->data[i][j][k] = desc->mat ? desc->mat[((size_t)i * d->yres + j) * d->zres + k] : 0;
        if (ade) alloc_ade(d);
    }
    for (i = 0; i < d->xres; i++)
        for (j = 0; j < d->yres; j++)
            for (k = 0; k < d->zres; k++) {
                size_t c = ((size_t)i * d->yres + j) * d->zres + k;
                if (d->epsilon && desc->epsilon) d->epsilon->data[i][j][k] = desc->epsilon[c];
                if (d->sigma && desc->sigma) d->sigma->data[i][j][k] = desc->sigma[c];
                if (d->mu && desc->mu) d->mu->data[i][j][k] = desc->mu[c];
                if (d->sigast && desc->sigast) d->sigast->data[i][j][k] = desc->sigast[c];
            }
    /* TSF source, plan.c:1522-1597 */
    if (desc->tsf.enabled) {
        SvSourceTSF *t = (SvSourceTSF *)g_malloc0(sizeof(SvSourceTSF));
        mp->src->tsf = t;
        t->box_i0 = desc->tsf.i0; t->box_j0 = desc->tsf.j0; t->box_k0 = desc->tsf.k0;
        t->box_in = desc->tsf.in; t->box_jn = desc->tsf.jn; t->box_kn = desc->tsf.kn;
        t->box_boundary_skipi0 = desc->tsf.skip[FDTD_FACE_X0]; t->box_boundary_skipin = desc->tsf.skip[FDTD_FACE_XN];
        t->box_boundary_skipj0 = desc->tsf.skip[FDTD_FACE_Y0]; t->box_boundary_skipjn = desc->tsf.skip[FDTD_FACE_YN];
        t->box_boundary_skipk0 = desc->tsf.skip[FDTD_FACE_Z0]; t->box_boundary_skipkn = desc->tsf.skip[FDTD_FACE_ZN];
        t->ia_theta = desc->tsf.theta; t->ia_phi = desc->tsf.phi; t->ia_psi = desc->tsf.psi;
        t->layered_epsilon = desc->tsf.layered_epsilon; t->layered_mu = desc->tsf.layered_mu;
        t->ndata = desc->tsf.nwave > desc->nsteps ? desc->tsf.nwave : desc->nsteps;
        t->e = (gdouble *)g_malloc0(sizeof(gdouble) * (t->ndata + 1));
        memcpy(t->e, desc->tsf.wave, sizeof(double) * desc->tsf.nwave);
        t->layered_zpos = (gint *)g_malloc0(sizeof(gint) * (t->ndata + 1));
        t->corr = 1.0 / sqrt(pow(sin(t->ia_theta), 4) * (pow(cos(t->ia_phi), 4) + pow(sin(t->ia_phi), 4)) + pow(cos(t->ia_theta), 4));
        t->jp = sv_1dpool_new((gint)(sqrt((gdouble)(set->sp.xres * set->sp.xres + set->sp.yres * set->sp.yres + set->sp.zres * set->sp.zres)) + 250),
                              set->sp.dx / t->corr, set->plan.dt);
        sv_1dpool_set_source_pos(t->jp, 0);
        sv_1dpool_set_material(t->jp, t->layered_epsilon, t->layered_mu);
    }
    /* TSF skip map, plan.c:5298-5326 */
    if (desc->tsf.enabled && set->ss.tsf.box_boundary_skipdepth >= 0) {
        int sd = set->ss.tsf.box_boundary_skipdepth, ii, jj, kk;
        d->sourceskip = sv_icube_new(d->xres, d->yres, d->zres, d->xres * d->dx, d->yres * d->dy, d->zres * d->dz, 1);
        /* cells are independent (pure lookups): split over the host threads */
#pragma omp parallel for private(j, k, ii, jj, kk) schedule(dynamic, 1)
        for (i = 0; i < d->xres; i++)
            for (j = 0; j < d->yres; j++)
                for (k = 0; k < d->zres; k++) {
                    int hit = 0;
                    d->sourceskip->data[i][j][k] = 0;
                    if (i > (desc->tsf.i0 + sd) && j > (desc->tsf.j0 + sd) && k > (desc->tsf.k0 + sd) &&
                        i < (desc->tsf.in - sd) && j < (desc->tsf.jn - sd) && k < (desc->tsf.kn - sd))
                        continue;
                    for (ii = MAX(0, i - sd); ii < MIN(i + sd, d->xres) && !hit; ii++)
                        for (jj = MAX(0, j - sd); jj < MIN(j + sd, d->yres) && !hit; jj++)
                            for (kk = MAX(0, k - sd); kk < MIN(k + sd, d->zres) && !hit; kk++)
                                if (sv_yee_data_get_tsf_mattype(d, set, mp->mats, mp->nmat, ii, jj, kk) != 0)
                                    hit = 1;
                    if (hit) d->sourceskip->data[i][j][k] = 1;
                }
    }
    /* internal boundaries, plan.c:5387-5416 (cells independent, as above) */
#pragma omp parallel for private(j, k) schedule(dynamic, 1)
    for (i = 0; i < d->xres; i++)
        for (j = 0; j < d->yres; j++)
            for (k = 0; k < d->zres; k++) {
                gdouble eps, sig, neps, nsig;
                int m, nm, ii, jj, kk;
                d->bnds->data[i][j][k] = 0;
                if (i == 0 || j == 0 || k == 0 || i == d->xres - 1 || j == d->yres - 1 || k == d->zres - 1) {
                    d->bnds->data[i][j][k] = 1;
                    continue;
                }
                m = sv_yee_data_get_epsilon_sigma(d, set, mp->mats, mp->nmat, i, j, k, &eps, &sig);
                for (ii = -1; ii <= 1; ii++)
                    for (jj = -1; jj <= 1; jj++)
                        for (kk = -1; kk <= 1; kk++) {
                            if (d->bnds->data[i][j][k] == 1) continue;
                            nm = sv_yee_data_get_epsilon_sigma(d, set, mp->mats, mp->nmat, i + ii, j + jj, k + kk, &neps, &nsig);
                            if (nm != m || neps != eps || nsig != sig) d->bnds->data[i][j][k] = 1;
                        }
            }
    /* probes */
    r->nprobes = desc->nprobes;
    r->nsteps = desc->nsteps;
    if (r->nprobes > 0) {
        r->probes = g_malloc(sizeof(int32_t) * 3 * r->nprobes);
        memcpy(r->probes, desc->probes, sizeof(int32_t) * 3 * r->nprobes);
        r->probe_out = g_malloc0(sizeof(double) * 6 * (size_t)r->nprobes * (size_t)(r->nsteps > 0 ? r->nsteps : 1));
    }
    return r;
}

void ref_destroy(ref_state *r)
{
    /* the reference has no matching free functions for most of its pool; the
     * process that loads this library is a short-lived test process */
    if (!r) return;
    g_free(r->probes);
    g_free(r->probe_out);
    g_free(r);
}

/* one CPU step, svit.c:217-237 */
int ref_step(ref_state *r, int nsteps)
{
    SvPool *mp = r->mp;
    SvSet *set = r->set;
    int it, p, a;
    for (it = 0; it < nsteps; it++) {
        sv_pool_boundary_copy(mp, set);
        sv_pool_ystep_h(mp, set);
        sv_pool_apply_source_hstep(mp, set);
        sv_pool_boundary_hstep(mp, set);
        sv_pool_ystep_e(mp, set);
        sv_pool_boundary_estep(mp, set);
        sv_pool_apply_source_estep(mp, set);
        if (r->nfff) sv_pool_farfield(mp, set);
        if (set->sc.step_act < r->nsteps)        /* sv_pool_getpoints, output.c:341-352 */
            for (p = 0; p < r->nprobes; p++) {
                int i = r->probes[3 * p], j = r->probes[3 * p + 1], k = r->probes[3 * p + 2];
                double v[6];
                double *o = r->probe_out + ((size_t)p * r->nsteps + set->sc.step_act) * 6;
                v[0] = mp->d->ex->data[i][j][k]; v[1] = mp->d->ey->data[i][j][k]; v[2] = mp->d->ez->data[i][j][k];
                v[3] = mp->d->hx->data[i][j][k]; v[4] = mp->d->hy->data[i][j][k]; v[5] = mp->d->hz->data[i][j][k];
                for (a = 0; a < 6; a++) o[a] = v[a];
            }
        set->sc.step_act++;
    }
    return 0;
}

static void copy_out(SvDCube *c, double *o)
{
    int i, j;
    if (!o) return;
    for (i = 0; i < c->xres; i++)
        for (j = 0; j < c->yres; j++)
            memcpy(o + ((size_t)i * c->yres + j) * c->zres, c->data[i][j], sizeof(double) * c->zres);
}

static void copy_in(SvDCube *c, const double *o)
{
    int i, j;
    if (!o) return;
    for (i = 0; i < c->xres; i++)
        for (j = 0; j < c->yres; j++)
            memcpy(c->data[i][j], o + ((size_t)i * c->yres + j) * c->zres, sizeof(double) * c->zres);
}

int ref_get_fields(const ref_state *r, double *ex, double *ey, double *ez, double *hx, double *hy, double *hz)
{
    SvYeeData *d = r->mp->d;
    copy_out(d->ex, ex); copy_out(d->ey, ey); copy_out(d->ez, ez);
    copy_out(d->hx, hx); copy_out(d->hy, hy); copy_out(d->hz, hz);
    return 0;
}

int ref_set_fields(ref_state *r, const double *ex, const double *ey, const double *ez,
                   const double *hx, const double *hy, const double *hz)
{
    SvYeeData *d = r->mp->d;
    copy_in(d->ex, ex); copy_in(d->ey, ey); copy_in(d->ez, ez);
    copy_in(d->hx, hx); copy_in(d->hy, hy); copy_in(d->hz, hz);
    return 0;
}

int ref_get_map(const ref_state *r, int which, int32_t *out)
{
    SvYeeData *d = r->mp->d;
    int i, j, k;
    for (i = 0; i < d->xres; i++)
        for (j = 0; j < d->yres; j++)
            for (k = 0; k < d->zres; k++) {
                size_t c = ((size_t)i * d->yres + j) * d->zres + k;
                if (which == FDTD_MAP_MAT) out[c] = d->mat ? d->mat->data[i][j][k] : -1;
                else if (which == FDTD_MAP_BNDS) out[c] = d->bnds->data[i][j][k];
                else if (which == FDTD_MAP_SOURCESKIP) out[c] = d->sourceskip ? d->sourceskip->data[i][j][k] : 0;
                else return -1;
            }
    return 0;
}

int ref_get_probes(const ref_state *r, double *out)
{
    if (r->nprobes > 0)
        memcpy(out, r->probe_out, sizeof(double) * 6 * (size_t)r->nprobes * (size_t)r->nsteps);
    return 0;
}

int ref_nfff_ndata(const ref_state *r) { return r->nfff ? r->mp->farfield->ndata : 0; }

int ref_get_nfff_series(const ref_state *r, double *out)
{
    int n, nd;
    if (!r->nfff) return -1;
    nd = r->mp->farfield->ndata;
    for (n = 0; n < r->set->sf.nrs; n++) {
        memcpy(out + ((size_t)n * 3 + 0) * nd, r->mp->farfield->rpoints[n].ex->data, sizeof(double) * nd);
        memcpy(out + ((size_t)n * 3 + 1) * nd, r->mp->farfield->rpoints[n].ey->data, sizeof(double) * nd);
        memcpy(out + ((size_t)n * 3 + 2) * nd, r->mp->farfield->rpoints[n].ez->data, sizeof(double) * nd);
    }
    return 0;
}

int ref_get_nfff_istart(const ref_state *r, int32_t *out)
{
    int n;
    if (!r->nfff) return -1;
    for (n = 0; n < r->set->sf.nrs; n++) out[n] = r->mp->farfield->rpoints[n].istart;
    return 0;
}

int ref_aux_res(const ref_state *r) { return r->mp->src->tsf ? r->mp->src->tsf->jp->res : 0; }

int ref_get_aux(const ref_state *r, double *e, double *h)
{
    Sv1DPool *jp;
    if (!r->mp->src->tsf) return -1;
    jp = r->mp->src->tsf->jp;
    memcpy(e, jp->e->data, sizeof(double) * jp->res);
    memcpy(h, jp->h->data, sizeof(double) * jp->res);
    return 0;
}

int ref_get_step(const ref_state *r) { return r->set->sc.step_act; }

#ifdef GSVIT_DROPIN
/* ------------------------------------------------------------------------
 * Drop-in check (test infrastructure): the same planned SvPool / SvSet, but
 * stepped through the GPU branch of svit.c:204-256 -- sv_pool_allocate_gpus
 * (pool.c:76-81) and the sv_pool_gpu_* family, here provided by
 * gsvit_copy_b200/dropin/gpu_b200.c over libgsvit_b200.  Built into
 * oracle/_ref/libgsvit_dropin.so, with UCUDA defined for every object, and
 * (GSVIT_REFCUDA) into oracle/_ref/libgsvit_refcuda.so over GSvit's own
 * src3d/gpu.c and gpu_kernels.cu.
 */
int dropin_start(ref_state *r)
{
    SvPool *mp = r->mp;
    SvSet *set = r->set;
    int p;
    /* point outputs as the planner leaves them (set->so, output.c:110-120) */
    set->so.npnts = r->nprobes;
    set->so.pnts = (SvOutputPar *)g_malloc0(sizeof(SvOutputPar) * (r->nprobes > 0 ? r->nprobes : 1));
    for (p = 0; p < r->nprobes; p++) {
        set->so.pnts[p].i = r->probes[3 * p];
        set->so.pnts[p].j = r->probes[3 * p + 1];
        set->so.pnts[p].k = r->probes[3 * p + 2];
    }
    if (r->nprobes > 0) {
        mp->out->outpointdata = (gdouble **)g_malloc(sizeof(gdouble *) * r->nprobes);
        for (p = 0; p < r->nprobes; p++)
            mp->out->outpointdata[p] = (gdouble *)g_malloc0(sizeof(gdouble) * 6 * (size_t)(r->nsteps > 0 ? r->nsteps : 1));
    }
    set->plan.gpumode = SV_GPUMODE_FULL;
    set->sc.ugpu[0] = 0;
#ifdef GSVIT_REFCUDA
    /* a deck with GPU = 1 and the default device query (settings.c:968-975):
     * the first device, queried
     * (sv_gpu_new reads the block size of its far-field kernels from the
     * device properties, gpu.c:1976-2003) */
    set->sc.usegpu = 1;
    set->sc.devicequery = 1;
#endif
    sv_pool_allocate_gpus(mp, set);
    if (!mp->gpu) return -1;
#ifdef GSVIT_REFCUDA
    if (((SvGpu *)mp->gpu)->ngset < 1) return -1;   /* no device found (gpu.c:2022-2040) */
#endif
    if (sv_pool_gpu_init(mp, set)) return -1;
    return sv_pool_gpu_copyto(mp, set, SV_SYNC_ALL) ? -1 : 0;
}

/* the GPU branch of the loop, svit.c:240-256 */
int dropin_step(ref_state *r, int nsteps)
{
    SvPool *mp = r->mp;
    SvSet *set = r->set;
    int it, rc = 0;
    for (it = 0; it < nsteps; it++) {
        rc |= sv_pool_gpu_boundary_copy(mp, set);
        rc |= sv_pool_gpu_ystep_h(mp, set);
        rc |= sv_pool_gpu_apply_source_hstep(mp, set);
        rc |= sv_pool_gpu_boundary_hstep(mp, set);
        rc |= sv_pool_gpu_ystep_e(mp, set);
        rc |= sv_pool_gpu_apply_source_estep(mp, set);
        rc |= sv_pool_gpu_boundary_estep(mp, set);
        rc |= sv_pool_gpu_getsum(mp, set);
        rc |= sv_pool_gpu_apply_farfield(mp, set);
        rc |= sv_pool_gpu_apply_pfarfield(mp, set);
        rc |= sv_pool_gpu_getpoints(mp, set);
        rc |= sv_pool_gpu_getforce(mp, set);
        set->sc.step_act++;
    }
    return rc ? -1 : 0;
}

/* Marks the planned deck as asking for one feature the drop-in does not
 * step (test of sv_gpu_new's refusal): 0 Liao boundary, 1 periodic boundary,
 * 2 PEC wall, 3 inner medium boundary, 4 point source, 5 SF source, 6 LTSF
 * source, 7 TSFF source, 8 subgrid, 9 sum output, 10 force output, 11
 * periodic far field, 12 an RC Drude material.  Returns -1 for an unknown id. */
int dropin_request(ref_state *r, int feature)
{
    SvPool *mp = r->mp;
    SvSet *set = r->set;
    switch (feature) {
    case 0: set->sb.bx0 = SV_BOUNDARY_LIAO; break;
    case 1: set->sb.bzn = SV_BOUNDARY_PERIODIC; break;
    case 2: set->sb.byn = SV_BOUNDARY_PEC; break;
    case 3: set->smb.bz0 = SV_BOUNDARY_CPML; break;
    case 4: set->ss.npnts = 1; break;
    case 5: mp->src->sf = (SvSourceSF *)g_malloc0(sizeof(SvSourceSF)); break;
    case 6: mp->src->ltsf = (SvSourceLTSF *)g_malloc0(sizeof(SvSourceLTSF)); break;
    case 7: mp->src->tsff = (SvSourceTSFF *)g_malloc0(sizeof(SvSourceTSFF)); break;
    case 8: set->sg.nsg = 1; break;
    case 9: set->so.nsums = 1; break;
    case 10: set->so.nforces = 1; break;
    case 11: set->spf.nrs = 1; break;
    case 12:
        if (mp->nmat < 2) return -1;
        mp->mats[mp->nmat - 1].type = SV_MAT_DRUDE;
        break;
    default: return -1;
    }
    return 0;
}

/* sv_pool_gpu_copyfrom at output time (svit.c:251-253) */
int dropin_finish(ref_state *r) { return sv_pool_gpu_copyfrom(r->mp, r->set, SV_SYNC_EH) ? -1 : 0; }

/* the point outputs written by copyfrom, as out[(p*nsteps + step)*6 + c] */
int dropin_get_probes(const ref_state *r, double *out)
{
    int p;
    for (p = 0; p < r->nprobes; p++)
        memcpy(out + (size_t)p * r->nsteps * 6, r->mp->out->outpointdata[p], sizeof(double) * 6 * (size_t)r->nsteps);
    return 0;
}
#endif
