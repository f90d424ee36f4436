/*
 * gpu_b200.c -- drop-in replacement of GSvit's src3d/gpu.c.
 *
 * GSvit's stepping loop (src3d/svit.c:204-256) reaches the GPU only through
 * sv_gpu_new (gpu.c:1960, via sv_pool_allocate_gpus, pool.c:76-81) and the
 * sv_pool_gpu_* family declared at src3d/pool.h:98-128.  This file implements
 * that family over the C ABI of include/gsvit_b200.h: it flattens the
 * planner's SvSet / SvPool into an fdtd_desc, creates one plan, and maps each
 * stage call onto the library.  It is compiled inside GSvit's tree (its
 * headers, with UCUDA defined so that SvPool carries its `gpu` member) in
 * place of gpu.c and gpu_kernels.cu, and linked with libgsvit_b200.
 *
 * Errors: gpu.c prints CUDA errors and carries on (gpu_kernels.cu:6063-6068);
 * here a failed call prints the library's error text and returns 1, and
 * sv_gpu_new returns NULL (so sv_pool_allocate_gpus leaves mp->gpu unset).
 * sv_gpu_new also refuses, before any library or CUDA call, every deck that
 * asks for something the library does not step: outer boundaries other than
 * CPML or none (PEC walls, Liao, periodic), inner medium boundaries, sources
 * other than the TSF plane wave (point, local, SF, LTSF, TSFF, LTSFF,
 * sheet), subgrids, material types other than linear-tabulated, ADE
 * (Drude / critical points) and PEC (the RC Drude / CP3 / CP and PLRC
 * models), sums, forces and the periodic far field.
 * Behaviour kept from gpu.c: copyfrom writes the
 * fields back into mp->d, the point outputs into mp->out->outpointdata
 * (output.c:341-352 layout) and the far-field series into
 * mp->farfield->rpoints[n].ex/ey/ez->data (farfield.c:175-405).  One whole time
 * step (H, TSF, CPML, E, ADE, far field, probes) runs in
 * sv_pool_gpu_ystep_h; the other per-stage calls of the loop are no-ops.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pool.h"
#include "settings.h"
#include "gsvit_b200.h"

typedef struct {
    fdtd_plan *plan;
    double *stage;        /* contiguous staging of one field component set */
    size_t n;
    int nprobes, nsteps;
    int have_series, npoints, ndata;
} B200Gpu;

static int b200_fail(const char *what)
{
    fprintf(stderr, "Error: GSvit B200 %s: %s\n", what, fdtd_last_error());
    return 1;
}

static B200Gpu *gpu_of(SvPool *mp) { return (B200Gpu *)mp->gpu; }

/* data[i][j][k] rows (dcube.c:31-53) <-> contiguous, k fastest */
static void gather_d(SvDCube *c, double *dst)
{
    int i, j;
    for (i = 0; i < c->xres; i++)
        for (j = 0; j < c->yres; j++)
            memcpy(dst + ((size_t)i * c->yres + j) * c->zres, c->data[i][j], sizeof(double) * c->zres);
}

static void scatter_d(SvDCube *c, const double *src)
{
    int i, j;
    for (i = 0; i < c->xres; i++)
        for (j = 0; j < c->yres; j++)
            memcpy(c->data[i][j], src + ((size_t)i * c->yres + j) * c->zres, sizeof(double) * c->zres);
}

static float *gather_f(SvFCube *c)
{
    int i, j;
    float *o;
    if (!c) return NULL;
    o = (float *)malloc(sizeof(float) * (size_t)c->xres * c->yres * c->zres);
    for (i = 0; i < c->xres; i++)
        for (j = 0; j < c->yres; j++)
            memcpy(o + ((size_t)i * c->yres + j) * c->zres, c->data[i][j], sizeof(float) * c->zres);
    return o;
}

static int32_t *gather_i(SvICube *c)
{
    int i, j, k;
    int32_t *o;
    if (!c) return NULL;
    o = (int32_t *)malloc(sizeof(int32_t) * (size_t)c->xres * c->yres * c->zres);
    for (i = 0; i < c->xres; i++)
        for (j = 0; j < c->yres; j++)
            for (k = 0; k < c->zres; k++) o[((size_t)i * c->yres + j) * c->zres + k] = c->data[i][j][k];
    return o;
}

static void cpml_face(fdtd_cpml_face *f, SvBoundaryType t, int depth, int m, double sigma, double a, double kappa)
{
    memset(f, 0, sizeof(*f));
    if (t != SV_BOUNDARY_CPML) return;
    f->enabled = 1;
    f->depth = depth;
    f->m = m;
    f->sigma = sigma;
    f->a = a;
    f->kappa = kappa;
}

static int outer_ok(SvBoundaryType t) { return t == SV_BOUNDARY_NONE || t == SV_BOUNDARY_CPML; }

/* The first feature of the deck that this library does not step, or NULL.
 * Settings as the parser and planner leave them: SvSetBoundary /
 * SvSetMBoundary (settings.h:529-590), SvSetSource (settings.h:491-508) and the
 * planned SvSource (source.h:224-233), SvSetOutput sums/forces
 * (settings.h:625-650), SvSetPFarfield (settings.h:827-864), SvSetSubgrid
 * (settings.h:522-525), the material table (SvMatProp.type, settings.h:103-113). */
static const char *b200_unsupported(const SvPool *mp, const SvSet *set)
{
    const SvSetBoundary *b = &set->sb;
    const SvSetMBoundary *m = &set->smb;
    int n;
    if (!outer_ok(b->bx0) || !outer_ok(b->bxn) || !outer_ok(b->by0) || !outer_ok(b->byn) || !outer_ok(b->bz0) ||
        !outer_ok(b->bzn))
        return "outer boundary other than CPML or none (PEC wall, Liao or periodic)";
    if (m->bx0 != SV_BOUNDARY_NONE || m->bxn != SV_BOUNDARY_NONE || m->by0 != SV_BOUNDARY_NONE ||
        m->byn != SV_BOUNDARY_NONE || m->bz0 != SV_BOUNDARY_NONE || m->bzn != SV_BOUNDARY_NONE)
        return "inner medium boundary";
    /* sv_source_new (source.c:40-51) leaves sp and sl unset and the others
     * NULL; the planner fills the latter only for sources the deck has */
    if (set->ss.npnts > 0) return "point source";
    if (set->ss.nlocals > 0) return "local source";
    if (mp->src && mp->src->sf) return "SF source";
    if (mp->src && mp->src->ltsf) return "LTSF source";
    if (mp->src && mp->src->tsff) return "TSFF source";
    if (mp->src && mp->src->ltsff) return "LTSFF source";
    if (mp->src && mp->src->sh) return "sheet source";
    if (set->sg.nsg > 0) return "subgrid";
    if (set->so.nsums > 0) return "sum output";
    if (set->so.nforces > 0) return "force output";
    if (set->spf.nrs > 0) return "periodic far field";   /* mp->pfarfield exists even without points */
    for (n = 1; n < mp->nmat; n++) {   /* mats[0] is vacuum (plan.c:78, 2418) */
        const int t = mp->mats[n].type;
        if (t != SV_MAT_LINTAB && t != SV_MAT_ADE && t != SV_MAT_PEC)
            return "material type other than linear-tabulated, ADE (Drude / critical points) or PEC";
    }
    return NULL;
}

/* sv_gpu_new (gpu.c:1960): the planner's state as an fdtd_desc, one plan */
SvGpu *sv_gpu_new(SvPool *mp, SvSet *set)
{
    SvYeeData *d = mp->d;
    B200Gpu *g;
    fdtd_desc desc;
    fdtd_material *mats = NULL;
    int32_t *mat = NULL, *pts = NULL, *ist = NULL, *probes = NULL;
    float *eps = NULL, *sig = NULL, *mu = NULL, *sigast = NULL;
    const char *unsupported = b200_unsupported(mp, set);
    int n, rc;

    if (unsupported) {
        fprintf(stderr, "Error: GSvit B200 does not step this deck: unsupported %s\n", unsupported);
        return NULL;
    }
    g = (B200Gpu *)calloc(1, sizeof(B200Gpu));
    memset(&desc, 0, sizeof(desc));
    desc.abi_version = FDTD_ABI_VERSION;
    desc.xres = set->sp.xres; desc.yres = set->sp.yres; desc.zres = set->sp.zres;
    desc.dx = set->sp.dx; desc.dy = set->sp.dy; desc.dz = set->sp.dz;
    desc.dt = set->plan.dt;
    desc.nsteps = set->sc.nsteps;
    desc.matmode = (int32_t)set->plan.matmode;
    desc.storage = FDTD_STORE_F32;
    /* material table: SvMatProp after the scaling of plan.c:4669-4698 */
    desc.nmat = mp->nmat;
    if (mp->nmat > 0) {
        mats = (fdtd_material *)calloc((size_t)mp->nmat, sizeof(fdtd_material));
        for (n = 0; n < mp->nmat; n++) {
            const SvMatProp *q = &mp->mats[n];
            fdtd_material *o = &mats[n];
            int p;
            o->type = q->type;
            o->epsilon = q->epsilon; o->mu = q->mu; o->sigma = q->sigma; o->sigast = q->sigast;
            o->drude_omega_p = q->drude_omega_p; o->drude_nu = q->drude_nu;
            for (p = 0; p < 2; p++) {
                o->cp_a[p] = q->cp3_a[p]; o->cp_phi[p] = q->cp3_phi[p];
                o->cp_omega[p] = q->cp3_omega[p]; o->cp_gamma[p] = q->cp3_gamma[p];
                o->ade_bp0[p] = q->ade_bp0[p]; o->ade_bp1[p] = q->ade_bp1[p]; o->ade_bp2[p] = q->ade_bp2[p];
                o->ade_bp3[p] = q->ade_bp3[p]; o->ade_bp4[p] = q->ade_bp4[p];
            }
            o->ade_a0 = q->ade_a0; o->ade_a1 = q->ade_a1; o->ade_a2 = q->ade_a2;
            o->ade_c0 = q->ade_c0; o->ade_c1 = q->ade_c1; o->ade_c2 = q->ade_c2; o->ade_c3 = q->ade_c3;
        }
        desc.mats = mats;
    }
    mat = gather_i(d->mat);
    eps = gather_f(d->epsilon); sig = gather_f(d->sigma); mu = gather_f(d->mu); sigast = gather_f(d->sigast);
    desc.mat = mat; desc.epsilon = eps; desc.sigma = sig; desc.mu = mu; desc.sigast = sigast;
    /* CPML (settings.c:5129-5162) */
    cpml_face(&desc.cpml[FDTD_FACE_X0], set->sb.bx0, set->sb.depth_bx0, set->sb.m_bx0, set->sb.sigma_bx0, set->sb.a_bx0, set->sb.kappa_bx0);
    cpml_face(&desc.cpml[FDTD_FACE_XN], set->sb.bxn, set->sb.depth_bxn, set->sb.m_bxn, set->sb.sigma_bxn, set->sb.a_bxn, set->sb.kappa_bxn);
    cpml_face(&desc.cpml[FDTD_FACE_Y0], set->sb.by0, set->sb.depth_by0, set->sb.m_by0, set->sb.sigma_by0, set->sb.a_by0, set->sb.kappa_by0);
    cpml_face(&desc.cpml[FDTD_FACE_YN], set->sb.byn, set->sb.depth_byn, set->sb.m_byn, set->sb.sigma_byn, set->sb.a_byn, set->sb.kappa_byn);
    cpml_face(&desc.cpml[FDTD_FACE_Z0], set->sb.bz0, set->sb.depth_bz0, set->sb.m_bz0, set->sb.sigma_bz0, set->sb.a_bz0, set->sb.kappa_bz0);
    cpml_face(&desc.cpml[FDTD_FACE_ZN], set->sb.bzn, set->sb.depth_bzn, set->sb.m_bzn, set->sb.sigma_bzn, set->sb.a_bzn, set->sb.kappa_bzn);
    /* TSF source: the planned SvSourceTSF (plan.c:1522-1597) */
    if (mp->src && mp->src->tsf) {
        const SvSourceTSF *t = mp->src->tsf;
        desc.tsf.enabled = 1;
        desc.tsf.i0 = t->box_i0; desc.tsf.j0 = t->box_j0; desc.tsf.k0 = t->box_k0;
        desc.tsf.in = t->box_in; desc.tsf.jn = t->box_jn; desc.tsf.kn = t->box_kn;
        desc.tsf.skip[FDTD_FACE_X0] = t->box_boundary_skipi0; desc.tsf.skip[FDTD_FACE_XN] = t->box_boundary_skipin;
        desc.tsf.skip[FDTD_FACE_Y0] = t->box_boundary_skipj0; desc.tsf.skip[FDTD_FACE_YN] = t->box_boundary_skipjn;
        desc.tsf.skip[FDTD_FACE_Z0] = t->box_boundary_skipk0; desc.tsf.skip[FDTD_FACE_ZN] = t->box_boundary_skipkn;
        desc.tsf.skipdepth = set->ss.tsf.box_boundary_skipdepth;
        desc.tsf.theta = t->ia_theta; desc.tsf.phi = t->ia_phi; desc.tsf.psi = t->ia_psi;
        desc.tsf.layered_epsilon = t->layered_epsilon;
        desc.tsf.layered_mu = t->layered_mu;
        desc.tsf.nwave = t->ndata;
        desc.tsf.wave = t->e;
    }
    /* far field: the reference's own time-domain series (farfield.c:175-405) */
    if (set->sf.nrs > 0 && mp->farfield) {
        desc.nfff.enabled = 1;
        desc.nfff.i0 = set->sf.box_i0; desc.nfff.j0 = set->sf.box_j0; desc.nfff.k0 = set->sf.box_k0;
        desc.nfff.in = set->sf.box_in; desc.nfff.jn = set->sf.box_jn; desc.nfff.kn = set->sf.box_kn;
#define SKIP(F, S, A, B) do { desc.nfff.skip[F] = set->sf.box_boundary_skip##S; \
        desc.nfff.skip_lo[F][0] = set->sf.skip##S##_##A##min; desc.nfff.skip_lo[F][1] = set->sf.skip##S##_##B##min; \
        desc.nfff.skip_hi[F][0] = set->sf.skip##S##_##A##max; desc.nfff.skip_hi[F][1] = set->sf.skip##S##_##B##max; } while (0)
        SKIP(FDTD_FACE_X0, i0, j, k); SKIP(FDTD_FACE_XN, in, j, k);
        SKIP(FDTD_FACE_Y0, j0, i, k); SKIP(FDTD_FACE_YN, jn, i, k);
        SKIP(FDTD_FACE_Z0, k0, i, j); SKIP(FDTD_FACE_ZN, kn, i, j);
#undef SKIP
        desc.nfff.npoints = set->sf.nrs;
        desc.nfff.nfreq = 0;
        desc.nfff.series = 1;
        pts = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)set->sf.nrs);
        ist = (int32_t *)malloc(sizeof(int32_t) * (size_t)set->sf.nrs);
        for (n = 0; n < set->sf.nrs; n++) {
            pts[3 * n] = set->sf.ri[n]; pts[3 * n + 1] = set->sf.rj[n]; pts[3 * n + 2] = set->sf.rk[n];
            ist[n] = mp->farfield->rpoints[n].istart;
        }
        desc.nfff.points = pts;
        desc.nfff.istart = ist;
        g->have_series = 1;
        g->npoints = set->sf.nrs;
        g->ndata = mp->farfield->ndata;
    }
    /* point outputs (output.c:341-352) */
    if (set->so.npnts > 0) {
        probes = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)set->so.npnts);
        for (n = 0; n < set->so.npnts; n++) {
            probes[3 * n] = set->so.pnts[n].i; probes[3 * n + 1] = set->so.pnts[n].j; probes[3 * n + 2] = set->so.pnts[n].k;
        }
        desc.nprobes = set->so.npnts;
        desc.probes = probes;
    }
    g->nprobes = set->so.npnts;
    g->nsteps = set->sc.nsteps;
    g->n = (size_t)set->sp.xres * set->sp.yres * set->sp.zres;

    rc = fdtd_plan_create(&desc, set->sc.ugpu[0] >= 0 ? set->sc.ugpu[0] : 0, &g->plan);
    free(mats); free(mat); free(eps); free(sig); free(mu); free(sigast); free(pts); free(ist); free(probes);
    if (rc != FDTD_OK) {
        b200_fail("plan");
        free(g);
        return NULL;
    }
    if (g->have_series) {
        int nd = 0;
        if (fdtd_nfff_ndata(g->plan, &nd) != FDTD_OK || nd != g->ndata) {
            fprintf(stderr, "Error: GSvit B200 far-field series length %d differs from GSvit's %d\n", nd, g->ndata);
            fdtd_plan_destroy(g->plan);
            free(g);
            return NULL;
        }
    }
    g->stage = (double *)malloc(sizeof(double) * 6 * g->n);
    return (SvGpu *)g;
}

int sv_pool_gpu_init(SvPool *mp, SvSet *set)
{
    (void)set;
    return gpu_of(mp) ? 0 : 1;
}

static int sync_mask(SvGpuSync what)
{
    return what == SV_SYNC_E ? FDTD_E : what == SV_SYNC_H ? FDTD_H : FDTD_EH;
}

/* sv_pool_gpu_copyto (gpu.c:629-685) */
int sv_pool_gpu_copyto(SvPool *mp, SvSet *set, SvGpuSync what)
{
    B200Gpu *g = gpu_of(mp);
    SvDCube *f[6] = {mp->d->ex, mp->d->ey, mp->d->ez, mp->d->hx, mp->d->hy, mp->d->hz};
    const double *comps[6];
    int c, mask = sync_mask(what);
    (void)set;
    for (c = 0; c < 6; c++) {
        comps[c] = NULL;
        if (!(mask >> c & 1)) continue;
        gather_d(f[c], g->stage + c * g->n);
        comps[c] = g->stage + c * g->n;
    }
    if (fdtd_set_fields(g->plan, mask, comps) != FDTD_OK) return b200_fail("copyto");
    return 0;
}

/* sv_pool_gpu_copyfrom (gpu.c:687-785): fields, point outputs, far-field series */
int sv_pool_gpu_copyfrom(SvPool *mp, SvSet *set, SvGpuSync what)
{
    B200Gpu *g = gpu_of(mp);
    SvDCube *f[6] = {mp->d->ex, mp->d->ey, mp->d->ez, mp->d->hx, mp->d->hy, mp->d->hz};
    double *comps[6];
    int c, mask = sync_mask(what), step = 0;
    (void)set;
    for (c = 0; c < 6; c++) comps[c] = (mask >> c & 1) ? g->stage + c * g->n : NULL;
    if (fdtd_get_fields(g->plan, mask, comps) != FDTD_OK) return b200_fail("copyfrom");
    for (c = 0; c < 6; c++)
        if (comps[c]) scatter_d(f[c], comps[c]);
    if (fdtd_get_step(g->plan, &step) != FDTD_OK) return b200_fail("copyfrom");
    if (g->nprobes > 0 && mp->out && mp->out->outpointdata && g->nsteps > 0) {
        size_t len = (size_t)g->nprobes * g->nsteps * 6;
        double *pr = (double *)malloc(sizeof(double) * len);
        int p, s;
        if (fdtd_get_probes(g->plan, pr, len) != FDTD_OK) { free(pr); return b200_fail("copyfrom"); }
        for (p = 0; p < g->nprobes; p++)
            for (s = 0; s < step && s < g->nsteps; s++)
                memcpy(mp->out->outpointdata[p] + (size_t)s * 6, pr + ((size_t)p * g->nsteps + s) * 6, sizeof(double) * 6);
        free(pr);
    }
    if (g->have_series) {
        size_t len = (size_t)g->npoints * 3 * g->ndata;
        double *ser = (double *)malloc(sizeof(double) * len);
        int n;
        if (fdtd_nfff_series(g->plan, ser, len) != FDTD_OK) { free(ser); return b200_fail("copyfrom"); }
        for (n = 0; n < g->npoints; n++) {
            memcpy(mp->farfield->rpoints[n].ex->data, ser + ((size_t)n * 3 + 0) * g->ndata, sizeof(double) * g->ndata);
            memcpy(mp->farfield->rpoints[n].ey->data, ser + ((size_t)n * 3 + 1) * g->ndata, sizeof(double) * g->ndata);
            memcpy(mp->farfield->rpoints[n].ez->data, ser + ((size_t)n * 3 + 2) * g->ndata, sizeof(double) * g->ndata);
        }
        free(ser);
    }
    return 0;
}

/* one whole time step: ystep_h, TSF, CPML, ystep_e, ADE, far field, probes */
int sv_pool_gpu_ystep_h(SvPool *mp, SvSet *set)
{
    (void)set;
    return fdtd_step(gpu_of(mp)->plan, 1) == FDTD_OK ? 0 : b200_fail("step");
}

/* stages of the same step, already done by sv_pool_gpu_ystep_h */
int sv_pool_gpu_ystep_e(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_gpu_apply_source_hstep(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_gpu_apply_source_estep(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_gpu_boundary_copy(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_gpu_boundary_hstep(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_gpu_boundary_estep(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_gpu_apply_farfield(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_gpu_getpoints(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }

/* sums, forces and the periodic far field: sv_gpu_new refuses decks that
 * request them, so with a plan these have nothing to do */
int sv_pool_gpu_getsum(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_gpu_getforce(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
int sv_pool_gpu_apply_pfarfield(SvPool *mp, SvSet *set) { (void)mp; (void)set; return 0; }
