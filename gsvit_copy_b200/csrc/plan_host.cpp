// plan_host.cpp -- host-side planning of the B200 FDTD library.
//
// Turns the flat descriptor (SvSet/SvPool after GSvit's planner) into what
// the kernels consume: per-cell coefficient classes, the interface and
// TSF-skip maps, CPML grading profiles, per-axis kappa, TSF face tables and
// the ADE coefficient sets.  This is the work gpu.c does in sv_gpu_new
// (gpu.c:1960-2712: material table pack gpu.c:2120-2178) but it also folds
// the per-cell decisions the reference CPU path takes at every step
// (get_tbc yee.c:454-526, get_cabs yee.c:1397-1493, the PEC rule
// yee.c:1138-1237) into a one-byte class per cell, so that the kernels read
// one byte instead of recomputing 7-neighbour material logic.
#include "plan_host.h"

#include <cmath>
#include <cstring>
#include <unordered_map>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double C0 = 299792458.0;
constexpr double MU0 = 1.256637061435917295e-6;
constexpr double EPS0 = 8.854187817620389850e-12;
constexpr double PI_D = 3.1415926535897932384626433832795028841971693993751;

bool is_tab(int t)
{
    return t == FDTD_MAT_LINTAB || t == FDTD_MAT_DRUDE || t == FDTD_MAT_PLRC || t == FDTD_MAT_ADE ||
           t == FDTD_MAT_CP || t == FDTD_MAT_CP3;
}

bool is_disp(int t)
{
    return t == FDTD_MAT_DRUDE || t == FDTD_MAT_CP3 || t == FDTD_MAT_CP || t == FDTD_MAT_ADE || t == FDTD_MAT_PLRC;
}

struct Grid {
    const fdtd_desc *d;
    int xr, yr, zr;
    std::vector<float> veps, vsig, vmu, vsigast;   // voxel arrays present per matmode
    bool has_e = false, has_m = false;
    const fdtd_design *ds = nullptr;               // design region (epsilon per cell, lossless)

    bool in_design(int i, int j, int k) const
    {
        return ds && i >= ds->i0 && i < ds->i1 && j >= ds->j0 && j < ds->j1 && k >= ds->k0 && k < ds->k1;
    }
    double design_eps(int i, int j, int k) const
    {
        return ds->eps_r[((size_t)(i - ds->i0) * (ds->j1 - ds->j0) + (j - ds->j0)) * (ds->k1 - ds->k0) + (k - ds->k0)] * EPS0;
    }

    size_t idx(int i, int j, int k) const { return ((size_t)i * yr + j) * zr + k; }
    int mat(int i, int j, int k) const
    {
        if (d->nmat <= 0) return -1;
        return d->mat ? d->mat[idx(i, j, k)] : 0;
    }
    // sv_yee_data_get_epsilon_sigma, yee.c:1318-1350
    int eps_sig(int i, int j, int k, double *e, double *g) const
    {
        int m = mat(i, j, k);
        double ee = EPS0, gg = 0;
        if (in_design(i, j, k)) {
            ee = design_eps(i, j, k);
        } else if (m > 0 && is_tab(d->mats[m].type)) {
            ee = d->mats[m].epsilon;
            gg = d->mats[m].sigma;
        } else if (has_e) {
            size_t c = idx(i, j, k);
            ee = veps[c];
            gg = vsig[c];
        }
        *e = ee;
        *g = gg;
        return m;
    }
    // sv_yee_data_get_epsilon, yee.c:1266-1289
    double eps(int i, int j, int k) const
    {
        if (in_design(i, j, k)) return design_eps(i, j, k);
        int m = mat(i, j, k);
        if (m > 0 && is_tab(d->mats[m].type)) return d->mats[m].epsilon;
        if (has_e) return veps[idx(i, j, k)];
        return EPS0;
    }
    bool is_pec(int i, int j, int k) const
    {
        int m = mat(i, j, k);
        return m > 0 && d->mats[m].type == FDTD_MAT_PEC;
    }
    // sv_yee_data_get_tsf_mattype, yee.c:1686-1707
    int tsf_mattype(int i, int j, int k) const
    {
        if (in_design(i, j, k)) return std::fabs(1.0 - design_eps(i, j, k) / EPS0) < 0.001 ? 0 : 1;
        int m = mat(i, j, k);
        if (m == 0 || m == -1) {
            if (has_e && (d->matmode == FDTD_MATMODE_FULL || d->matmode == FDTD_MATMODE_ELECTRIC) &&
                std::fabs(1.0 - (double)veps[idx(i, j, k)] / EPS0) < 0.001)
                return 0;
            if (d->matmode == FDTD_MATMODE_NONE) return 0;
        }
        if (m > 0 && d->mats[m].type == FDTD_MAT_LINTAB && std::fabs(1.0 - d->mats[m].epsilon / EPS0) < 0.001)
            return 0;
        return 1;
    }
};

// dispersive-neighbour rule, yee.c:454-526
int get_tbc(const Grid &g, int i, int j, int k, int *xt, int *yt, int *zt)
{
    *xt = *yt = *zt = 1;
    if (g.d->nmat <= 0) return -1;
    int m = g.mat(i, j, k);
    const fdtd_material *M = g.d->mats;
    if (m > 0 && is_disp(M[m].type)) {
        *xt = *yt = *zt = 0;
        return m;
    }
    auto nb = [&](bool cond, int ii, int jj, int kk) -> int {
        if (!cond) return 0;
        int q = g.mat(ii, jj, kk);
        return (q > 0 && is_disp(M[q].type)) ? q : 0;
    };
    int q;
    if ((q = nb(i > 0, i - 1, j, k))) { m = q; *yt = *zt = 0; }
    if ((q = nb(j > 0, i, j - 1, k))) { m = q; *xt = *zt = 0; }
    if ((q = nb(k > 0, i, j, k - 1))) { m = q; *xt = *yt = 0; }
    if ((q = nb(i > 0 && j > 0, i - 1, j - 1, k))) { m = q; *zt = 0; }
    if ((q = nb(j > 0 && k > 0, i, j - 1, k - 1))) { m = q; *xt = 0; }
    if ((q = nb(i > 0 && k > 0, i - 1, j, k - 1))) { m = q; *yt = 0; }
    return m;
}

// per-component ca/cb with interface averaging, yee.c:1397-1493
void get_cabs(const Grid &g, const std::vector<int8_t> &bnds, int i, int j, int k, double dt, double dx,
              double ca[3], double cb[3])
{
    double e, s, ex, ey, ez, sx, sy, sz;
    g.eps_sig(i, j, k, &e, &s);
    ex = ey = ez = e;
    sx = sy = sz = s;
    if (bnds[g.idx(i, j, k)] > 0) {
        int nx = 1, ny = 1, nz = 1;
        if (i > 0) { g.eps_sig(i - 1, j, k, &e, &s); ey += e; sy += s; ez += e; sz += s; ny++; nz++; }
        if (j > 0) { g.eps_sig(i, j - 1, k, &e, &s); ex += e; sx += s; ez += e; sz += s; nx++; nz++; }
        if (k > 0) { g.eps_sig(i, j, k - 1, &e, &s); ex += e; sx += s; ey += e; sy += s; nx++; ny++; }
        if (j > 0 && k > 0) { g.eps_sig(i, j - 1, k - 1, &e, &s); ex += e; sx += s; nx++; }
        if (i > 0 && k > 0) { g.eps_sig(i - 1, j, k - 1, &e, &s); ey += e; sy += s; ny++; }
        if (i > 0 && j > 0) { g.eps_sig(i - 1, j - 1, k, &e, &s); ez += e; sz += s; nz++; }
        ex /= nx; sx /= nx;
        ey /= ny; sy /= ny;
        ez /= nz; sz /= nz;
    }
    const double E[3] = {ex, ey, ez}, S[3] = {sx, sy, sz};
    for (int a = 0; a < 3; a++) {
        ca[a] = (1 - S[a] * dt / 2 / E[a]) / (1 + S[a] * dt / 2 / E[a]);
        cb[a] = (dt / E[a] / dx) / (1 + S[a] * dt / 2 / E[a]);
    }
}

// CPML grading of boundary.c:34-99 (becebhch0 for 0-faces, becebhch for n-faces)
void cpml_grade(int pos, int imax, double sigma, double kappa, double a, int m, double dt, bool low,
                double *be, double *ce, double *bh, double *ch, double *ke, double *kh)
{
    double hoff = low ? -0.5 : 0.5;
    double pe = std::pow((imax - pos) / (double)imax, m);
    double ph = std::pow((imax - pos + hoff) / (double)imax, m);
    double sve = sigma * pe, kve = 1 + (kappa - 1) * pe, ave = a * (pos / (double)imax);
    double svh = sigma * ph, kvh = 1 + (kappa - 1) * ph, avh = a * ((pos + hoff) / (double)imax);
    *be = std::exp(-(sve / kve + ave) * dt / EPS0);
    *ce = (sve == 0) ? 0 : (sve / (sve + kve * ave) / kve) * (*be - 1.0);
    *bh = std::exp(-(svh / kvh + avh) * dt / EPS0);
    *ch = (svh == 0) ? 0 : (svh / (svh + kvh * avh) / kvh) * (*bh - 1.0);
    *ke = kve;
    *kh = kvh;
}

// a cell's class: the FP32 coefficients, and the FP64 ones for FP64 plans
// (zero otherwise, so that FP32 plans deduplicate on the FP32 values alone)
struct ClassKey {
    DevClass c;
    DevClass64 d;
};
struct ClassHash {
    size_t operator()(const ClassKey &c) const
    {
        const uint32_t *w = reinterpret_cast<const uint32_t *>(&c);
        size_t h = 1469598103934665603ull;
        for (size_t q = 0; q < sizeof(ClassKey) / 4; q++) h = (h ^ w[q]) * 1099511628211ull;
        return h;
    }
};
struct ClassEq {
    bool operator()(const ClassKey &a, const ClassKey &b) const { return std::memcmp(&a, &b, sizeof(ClassKey)) == 0; }
};

}  // namespace

int build_host_plan(const fdtd_desc *d, HostPlan *hp, std::string *err)
{
    if (!d || d->abi_version != FDTD_ABI_VERSION) { *err = "descriptor ABI version mismatch"; return FDTD_E_INVALID; }
    if (d->xres < 3 || d->yres < 3 || d->zres < 3) { *err = "grid must be at least 3 cells on every axis"; return FDTD_E_INVALID; }
    if (!(d->dt > 0) || !(d->dx > 0)) { *err = "dt and dx must be positive"; return FDTD_E_INVALID; }
    if (d->dx != d->dy || d->dx != d->dz) { *err = "non-cubic cells are outside the implemented path"; return FDTD_E_UNSUPPORTED; }
    if (d->nmat > 0 && !d->mats) { *err = "nmat > 0 but mats is NULL"; return FDTD_E_INVALID; }
    if (d->storage != FDTD_STORE_F32 && d->storage != FDTD_STORE_F16 && d->storage != FDTD_STORE_BF16 &&
        d->storage != FDTD_STORE_F64) {
        *err = "unknown storage mode"; return FDTD_E_INVALID;
    }
    hp->real64 = d->storage == FDTD_STORE_F64;
    for (int m = 1; m < d->nmat; m++) {
        int t = d->mats[m].type;
        if (t != FDTD_MAT_LINTAB && t != FDTD_MAT_ADE && t != FDTD_MAT_PEC) {
            *err = "material type " + std::to_string(t) + " is outside the implemented path (LINTAB, ADE, PEC)";
            return FDTD_E_UNSUPPORTED;
        }
    }
    const int xr = d->xres, yr = d->yres, zr = d->zres;
    const size_t n = (size_t)xr * yr * zr;
    hp->xr = xr; hp->yr = yr; hp->zr = zr; hp->n = n;
    hp->dx = d->dx; hp->dt = d->dt;
    hp->nsteps = d->nsteps;
    const double dt = d->dt, dx = d->dx;

    Grid g;
    g.d = d; g.xr = xr; g.yr = yr; g.zr = zr;
    // design region: the box, its affected box (one cell more above on each
    // axis: those cells average epsilon with the box) and the context box
    // (one cell more below: the cells the affected ones average over)
    hp->design = d->design.enabled != 0;
    if (hp->design) {
        const fdtd_design &ds = d->design;
        const int lo[3] = {ds.i0, ds.j0, ds.k0}, hi[3] = {ds.i1, ds.j1, ds.k1}, res[3] = {xr, yr, zr};
        if (!ds.eps_r) { *err = "design region without eps_r"; return FDTD_E_INVALID; }
        for (int ax = 0; ax < 3; ax++) {
            if (lo[ax] < 1 || hi[ax] > res[ax] - 2 || lo[ax] >= hi[ax]) {
                *err = "design box must lie inside [1, res-2) on every axis"; return FDTD_E_INVALID;
            }
            hp->dbox[2 * ax] = lo[ax]; hp->dbox[2 * ax + 1] = hi[ax];
            hp->abox[2 * ax] = lo[ax]; hp->abox[2 * ax + 1] = hi[ax] + 1;
            hp->cbox[2 * ax] = lo[ax] - 1; hp->cbox[2 * ax + 1] = hi[ax] + 1;
            const fdtd_cpml_face &c0 = d->cpml[2 * ax], &c1 = d->cpml[2 * ax + 1];
            if ((c0.enabled && hp->abox[2 * ax] < c0.depth) || (c1.enabled && hp->abox[2 * ax + 1] > res[ax] - c1.depth)) {
                *err = "design region (and the cells above it) must lie outside the CPML slabs"; return FDTD_E_INVALID;
            }
        }
        const size_t nd = (size_t)(ds.i1 - ds.i0) * (ds.j1 - ds.j0) * (ds.k1 - ds.k0);
        for (size_t q = 0; q < nd; q++)
            if (!(ds.eps_r[q] >= 1e-3 && ds.eps_r[q] < 1e6)) { *err = "design eps_r must be positive and finite"; return FDTD_E_INVALID; }
        if (d->tsf.enabled) {
            const int t0[3] = {d->tsf.i0, d->tsf.j0, d->tsf.k0}, t1[3] = {d->tsf.in, d->tsf.jn, d->tsf.kn};
            for (int ax = 0; ax < 3; ax++)
                if (!(hp->abox[2 * ax] > t0[ax] && hp->abox[2 * ax + 1] <= t1[ax])) {
                    *err = "design region (and the cells above it) must lie strictly inside the TSF box"; return FDTD_E_INVALID;
                }
        }
        g.ds = &ds;
    }
    g.has_e = (d->matmode == FDTD_MATMODE_FULL || d->matmode == FDTD_MATMODE_ELECTRIC);
    g.has_m = (d->matmode == FDTD_MATMODE_FULL || d->matmode == FDTD_MATMODE_MAGNETIC);
    try {
        if (g.has_e) {   // voxel arrays as sv_yee_data_allocate fills them (yee.c:104-111)
            g.veps.assign(n, (float)EPS0);
            g.vsig.assign(n, 0.0f);
            if (d->epsilon) std::memcpy(g.veps.data(), d->epsilon, n * sizeof(float));
            if (d->sigma) std::memcpy(g.vsig.data(), d->sigma, n * sizeof(float));
        }
        if (g.has_m) {
            g.vmu.assign(n, (float)MU0);
            g.vsigast.assign(n, 0.0f);
            if (d->mu) std::memcpy(g.vmu.data(), d->mu, n * sizeof(float));
            if (d->sigast) std::memcpy(g.vsigast.data(), d->sigast, n * sizeof(float));
        }
        hp->bnds.assign(n, 0);
        hp->sskip.assign(n, 0);
        hp->cls.assign(n, 0);
    } catch (const std::bad_alloc &) {
        *err = "host allocation failed";
        return FDTD_E_NOMEM;
    }
    if (d->nmat > 0 && d->mat) {
        for (size_t c = 0; c < n; c++)
            if (d->mat[c] < 0 || d->mat[c] >= d->nmat) { *err = "material index out of range at cell " + std::to_string(c); return FDTD_E_INVALID; }
    }
    bool disp = false;
    for (int m = 1; m < d->nmat; m++)
        if (d->mats[m].type == FDTD_MAT_ADE) disp = true;
    hp->has_ade = disp;

    // interface map, plan.c:5387-5416
#pragma omp parallel for schedule(static)
    for (int i = 0; i < xr; i++)
        for (int j = 0; j < yr; j++)
            for (int k = 0; k < zr; k++) {
                size_t c = g.idx(i, j, k);
                if (i == 0 || j == 0 || k == 0 || i == xr - 1 || j == yr - 1 || k == zr - 1) { hp->bnds[c] = 1; continue; }
                double e, s, ne, ns;
                int m = g.eps_sig(i, j, k, &e, &s);
                int8_t b = 0;
                for (int ii = -1; ii <= 1 && !b; ii++)
                    for (int jj = -1; jj <= 1 && !b; jj++)
                        for (int kk = -1; kk <= 1 && !b; kk++) {
                            int nm = g.eps_sig(i + ii, j + jj, k + kk, &ne, &ns);
                            if (nm != m || ne != e || ns != s) b = 1;
                        }
                hp->bnds[c] = b;
            }

    // TSF set-up, plan.c:1522-1597, and skip map plan.c:5298-5326
    hp->tsf = d->tsf.enabled != 0;
    if (hp->tsf) {
        const fdtd_tsf &t = d->tsf;
        if (t.i0 < 1 || t.j0 < 1 || t.k0 < 1 || t.in > xr - 1 || t.jn > yr - 1 || t.kn > zr - 1 || t.in <= t.i0 ||
            t.jn <= t.j0 || t.kn <= t.k0) {
            *err = "TSF box must lie inside [1, res-1] on every axis"; return FDTD_E_INVALID;
        }
        if (!(t.theta >= 0 && t.theta < PI_D)) { *err = "TSF theta outside [0, pi)"; return FDTD_E_INVALID; }
        if (t.nwave < 0 || (t.nwave > 0 && !t.wave)) { *err = "TSF waveform missing"; return FDTD_E_INVALID; }
        hp->corr = 1.0 / std::sqrt(std::pow(std::sin(t.theta), 4) * (std::pow(std::cos(t.phi), 4) + std::pow(std::sin(t.phi), 4)) +
                                   std::pow(std::cos(t.theta), 4));
        hp->jres = (int)(std::sqrt((double)(xr * xr + yr * yr + zr * zr)) + 250);
        hp->jdx = dx / hp->corr;
        hp->wave.assign(t.wave, t.wave + t.nwave);
        int sd = t.skipdepth;
        if (sd >= 0) {
#pragma omp parallel for schedule(dynamic)
            for (int i = 0; i < xr; i++)
                for (int j = 0; j < yr; j++)
                    for (int k = 0; k < zr; k++) {
                        if (i > t.i0 + sd && j > t.j0 + sd && k > t.k0 + sd && i < t.in - sd && j < t.jn - sd && k < t.kn - sd)
                            continue;
                        bool hit = false;   // eval_closecheck, plan.c:3857-3873
                        for (int ii = std::max(0, i - sd); ii < std::min(i + sd, xr) && !hit; ii++)
                            for (int jj = std::max(0, j - sd); jj < std::min(j + sd, yr) && !hit; jj++)
                                for (int kk = std::max(0, k - sd); kk < std::min(k + sd, zr) && !hit; kk++)
                                    if (g.tsf_mattype(ii, jj, kk) != 0) hit = true;
                        hp->sskip[g.idx(i, j, k)] = hit ? 1 : 0;
                    }
        }
        // face tables: bit0 = correction applies (mat_too_close_check, source.c:253-265),
        //              bit1 = the face cell is PEC (the k0-face test of source.c:753,1633)
        auto mtc = [&](int i, int j, int k) { return sd == -1 ? 1 : (hp->sskip[g.idx(i, j, k)] ? 0 : 1); };
        const int ni = t.in - t.i0 + 1, nj = t.jn - t.j0 + 1, nk = t.kn - t.k0 + 1;
        for (int f = 0; f < 6; f++) {
            int ax = f / 2;
            int na = (ax == 0) ? nj : ni, nb = (ax == 2) ? nj : nk;
            hp->tmap[f].assign((size_t)na * nb, 0);
            hp->tmap_dims[f][0] = na;
            hp->tmap_dims[f][1] = nb;
            for (int a = 0; a < na; a++)
                for (int b = 0; b < nb; b++) {
                    int i, j, k;
                    int pos = (f % 2 == 0) ? (ax == 0 ? t.i0 : ax == 1 ? t.j0 : t.k0) : (ax == 0 ? t.in : ax == 1 ? t.jn : t.kn);
                    if (ax == 0) { i = pos; j = t.j0 + a; k = t.k0 + b; }
                    else if (ax == 1) { i = t.i0 + a; j = pos; k = t.k0 + b; }
                    else { i = t.i0 + a; j = t.j0 + b; k = pos; }
                    uint8_t v = 0;
                    if (!t.skip[f] && mtc(i, j, k)) v |= 1;
                    if (g.is_pec(i, j, k)) v |= 2;
                    hp->tmap[f][(size_t)a * nb + b] = v;
                }
        }
    }

    // ADE coefficient sets
    std::vector<int> ade_slot(std::max(d->nmat, 1), -1);
    hp->maxpoles = 0;
    for (int m = 1; m < d->nmat; m++) {
        if (d->mats[m].type != FDTD_MAT_ADE) continue;
        if ((int)hp->ades.size() >= FDTD_MAX_ADE) { *err = "too many ADE materials"; return FDTD_E_UNSUPPORTED; }
        const fdtd_material &q = d->mats[m];
        DevAde64 w;   // the difference-form set in FP64 (DevAde)
        std::memset(&w, 0, sizeof(w));
        w.c0dx = q.ade_c0 / dx;
        w.c2 = q.ade_c2; w.c3 = q.ade_c3;
        w.qe = q.ade_c1 * q.ade_a0;
        w.ma0 = -q.ade_a0;
        w.a2 = q.ade_a2;
        for (int p = 0; p < 2; p++) {
            w.pe[p] = q.ade_c1 * ((1.0 - q.ade_bp0[p]) - q.ade_bp1[p]);
            w.qpe[p] = q.ade_c1 * q.ade_bp0[p];
            w.rp[p] = (q.ade_bp0[p] + q.ade_bp1[p]) - 1.0;
            w.rq[p] = -q.ade_bp0[p];
            w.bp2[p] = q.ade_bp2[p]; w.bp3[p] = q.ade_bp3[p]; w.bp4[p] = q.ade_bp4[p];
            if (q.ade_bp2[p] != 0 || q.ade_bp3[p] != 0 || q.ade_bp4[p] != 0) hp->maxpoles = 2;
        }
        DevAde a;
        std::memset(&a, 0, sizeof(a));
        a.c0dx = (float)w.c0dx;
        a.c2 = (float)w.c2; a.c3 = (float)w.c3;
        a.qe = (float)w.qe;
        a.ma0 = (float)w.ma0;
        a.a2 = (float)w.a2;
        for (int p = 0; p < 2; p++) {
            a.pe[p] = (float)w.pe[p]; a.qpe[p] = (float)w.qpe[p];
            a.rp[p] = (float)w.rp[p]; a.rq[p] = (float)w.rq[p];
            a.bp2[p] = (float)w.bp2[p]; a.bp3[p] = (float)w.bp3[p]; a.bp4[p] = (float)w.bp4[p];
        }
        ade_slot[m] = (int)hp->ades.size();
        hp->ades.push_back(a);
        hp->ades64.push_back(w);
    }

    // per-cell classes, deduplicated; thread-local tables merged afterwards
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    std::vector<std::vector<ClassKey>> local(nthr);
    std::vector<std::unordered_map<ClassKey, int, ClassHash, ClassEq>> lmap(nthr);
    const bool r64 = hp->real64;
    std::vector<int> plane_owner(xr, 0);
    std::vector<uint16_t> lid(n);
    std::string perr;
    const double ecor = dt / dx;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < xr; i++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        plane_owner[i] = tid;
        for (int j = 0; j < yr; j++)
            for (int k = 0; k < zr; k++) {
                ClassKey key;
                std::memset(&key, 0, sizeof(key));
                DevClass &c = key.c;
                DevClass64 &w = key.d;   // stays zero for FP32 plans
                int xt, yt, zt;
                int m = get_tbc(g, i, j, k, &xt, &yt, &zt);
                double ca[3], cb[3];
                get_cabs(g, hp->bnds, i, j, k, dt, dx, ca, cb);
                for (int a = 0; a < 3; a++) { c.ca[a] = (float)ca[a]; c.cb[a] = (float)cb[a]; }
                if (r64)
                    for (int a = 0; a < 3; a++) { w.ca[a] = ca[a]; w.cb[a] = cb[a]; }
                if (disp && xt * yt * zt == 0) {
                    c.flags |= CF_ADE_BRANCH;
                    if (!xt) c.flags |= CF_ADE_X;
                    if (!yt) c.flags |= CF_ADE_Y;
                    if (!zt) c.flags |= CF_ADE_Z;
                    c.ade = ade_slot[m];
                    const fdtd_material &q = d->mats[m];
                    double cba = (dt / q.epsilon / dx) / (1 + q.sigma * dt / 2 / q.epsilon);
                    c.cba[0] = c.cba[1] = c.cba[2] = (float)cba;
                    if (r64) w.cba[0] = w.cba[1] = w.cba[2] = cba;
                }
                // H coefficients (ystep_h, yee.c:213-243)
                int mi = g.mat(i, j, k);
                double da, db;
                if (mi > 0 && is_tab(d->mats[mi].type)) {
                    const fdtd_material &q = d->mats[mi];
                    da = (1 - q.sigast * dt / 2 / q.mu) / (1 + q.sigast * dt / 2 / q.mu);
                    db = (dt / q.mu / dx) / (1 + q.sigast * dt / 2 / q.mu);
                } else if (g.has_m) {
                    double mu = g.vmu[g.idx(i, j, k)], sa = g.vsigast[g.idx(i, j, k)];
                    da = (1 - sa * dt / 2 / mu) / (1 + sa * dt / 2 / mu);
                    db = (dt / mu / dx) / (1 + sa * dt / 2 / mu);
                } else {
                    da = 1;
                    db = dt / MU0 / dx;
                }
                c.da = (float)da;
                c.db = (float)db;
                c.tsfe = (float)(ecor / g.eps(i, j, k));
                if (r64) { w.da = da; w.db = db; w.tsfe = ecor / g.eps(i, j, k); }
                const bool affected = hp->design && i >= hp->abox[0] && i < hp->abox[1] && j >= hp->abox[2] &&
                                      j < hp->abox[3] && k >= hp->abox[4] && k < hp->abox[5];
                if (affected) {   // E coefficients per cell (design_coefficients); no TSF face here
                    for (int a = 0; a < 3; a++) { c.ca[a] = 0.f; c.cb[a] = 0.f; w.ca[a] = 0; w.cb[a] = 0; }
                    c.tsfe = 0.f;
                    w.tsfe = 0;
                    c.flags |= CF_DESIGN;
                }
                // PEC rule, yee.c:1138-1237 (no SF source on this path)
                if (m >= 0 && i > 0 && j > 0 && k > 0) {
                    const fdtd_material *M = d->mats;
                    const int P = FDTD_MAT_PEC;
                    int t0 = M[g.mat(i, j, k)].type, tx = M[g.mat(i - 1, j, k)].type, ty = M[g.mat(i, j - 1, k)].type;
                    int tz = M[g.mat(i, j, k - 1)].type, txy = M[g.mat(i - 1, j - 1, k)].type;
                    int tyz = M[g.mat(i, j - 1, k - 1)].type, txz = M[g.mat(i - 1, j, k - 1)].type;
                    int txyz = M[g.mat(i - 1, j - 1, k - 1)].type;
                    if (M[m].type == P || tx == P || ty == P || tz == P || txy == P || tyz == P || txz == P || txyz == P) {
                        if ((tx != P && t0 == P) || (tx == P && t0 != P)) c.flags |= CF_PEC_Y | CF_PEC_Z;
                        if ((ty != P && t0 == P) || (ty == P && t0 != P)) c.flags |= CF_PEC_X | CF_PEC_Z;
                        if ((tz != P && t0 == P) || (tz == P && t0 != P)) c.flags |= CF_PEC_X | CF_PEC_Y;
                        if (txy == P && t0 != P) c.flags |= CF_PEC_Z;
                        if (txz == P && t0 != P) c.flags |= CF_PEC_Y;
                        if (tyz == P && t0 != P) c.flags |= CF_PEC_X;
                    }
                }
                if (r64) { w.flags = c.flags; w.ade = c.ade; }
                auto &mp = lmap[tid];
                auto it = mp.find(key);
                int id;
                if (it == mp.end()) {
                    id = (int)local[tid].size();
                    local[tid].push_back(key);
                    mp.emplace(key, id);
                } else
                    id = it->second;
                lid[g.idx(i, j, k)] = (uint16_t)std::min(id, 65535);
            }
    }
    std::unordered_map<ClassKey, int, ClassHash, ClassEq> gmap;
    std::vector<std::vector<int>> remap(nthr);
    for (int t = 0; t < nthr; t++) {
        for (auto &c : local[t]) {
            auto it = gmap.find(c);
            int id;
            if (it == gmap.end()) {
                id = (int)hp->classes.size();
                hp->classes.push_back(c.c);
                if (r64) hp->classes64.push_back(c.d);
                gmap.emplace(c, id);
            } else
                id = it->second;
            remap[t].push_back(id);
        }
    }
    if (hp->classes.size() > FDTD_MAX_CLASSES) {
        *err = "the material layout needs " + std::to_string(hp->classes.size()) + " coefficient classes (limit 256)";
        return FDTD_E_UNSUPPORTED;
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < xr; i++) {
        const std::vector<int> &rm = remap[plane_owner[i]];
        for (size_t c = (size_t)i * yr * zr; c < (size_t)(i + 1) * yr * zr; c++) hp->cls[c] = (uint8_t)rm[lid[c]];
    }

    // CPML profiles and per-axis 1/kappa with the MAX rule of yee.c:179-203, yee.c:573-592
    for (int f = 0; f < 6; f++) {
        hp->cp[f] = d->cpml[f];
        if (!d->cpml[f].enabled) continue;
        int dep = d->cpml[f].depth;
        int res = (f < 2) ? xr : (f < 4) ? yr : zr;
        if (dep < 2 || dep > res / 2) { *err = "CPML depth must be in [2, res/2]"; return FDTD_E_INVALID; }
        bool low = (f % 2 == 0);
        hp->be[f].resize(dep); hp->ce[f].resize(dep); hp->bh[f].resize(dep); hp->ch[f].resize(dep);
        hp->ke[f].resize(dep); hp->kh[f].resize(dep);
        hp->be64[f].resize(dep); hp->ce64[f].resize(dep); hp->bh64[f].resize(dep); hp->ch64[f].resize(dep);
        for (int q = 0; q < dep; q++) {
            double be, ce, bh, ch, ke, kh;
            cpml_grade(low ? q : dep - q, dep, d->cpml[f].sigma, d->cpml[f].kappa, d->cpml[f].a, d->cpml[f].m, dt, low,
                       &be, &ce, &bh, &ch, &ke, &kh);
            hp->be[f][q] = (float)be; hp->ce[f][q] = (float)ce; hp->bh[f][q] = (float)bh; hp->ch[f][q] = (float)ch;
            hp->be64[f][q] = be; hp->ce64[f][q] = ce; hp->bh64[f][q] = bh; hp->ch64[f][q] = ch;
            hp->ke[f][q] = ke; hp->kh[f][q] = kh;
        }
    }
    for (int ax = 0; ax < 3; ax++) {
        int res = ax == 0 ? xr : ax == 1 ? yr : zr;
        hp->ike[ax].assign(res, 1.0f);
        hp->ikh[ax].assign(res, 1.0f);
        hp->ike64[ax].assign(res, 1.0);
        hp->ikh64[ax].assign(res, 1.0);
        for (int q = 0; q < res; q++) {
            double ke = 1, kh = 1;
            int f0 = 2 * ax, fn = 2 * ax + 1;
            if (d->cpml[f0].enabled && q < d->cpml[f0].depth) {
                ke = std::max(ke, hp->ke[f0][q]);
                kh = std::max(kh, hp->kh[f0][q]);
            }
            if (d->cpml[fn].enabled && q >= res - d->cpml[fn].depth) {
                ke = std::max(ke, hp->ke[fn][q - (res - d->cpml[fn].depth)]);
                kh = std::max(kh, hp->kh[fn][q - (res - d->cpml[fn].depth)]);
            }
            hp->ike[ax][q] = (float)(1.0 / ke);
            hp->ikh[ax][q] = (float)(1.0 / kh);
            hp->ike64[ax][q] = 1.0 / ke;
            hp->ikh64[ax][q] = 1.0 / kh;
        }
    }
    // probes
    if (hp->design) {
        // context: epsilon and sigma of every cell of cbox (design cells
        // included); the cells there must be lossless, non-magnetic and
        // neither PEC nor dispersive
        const int *b = hp->cbox;
        const size_t nc = (size_t)(b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]);
        hp->ctx_eps.assign(nc, 0.0);
        hp->ctx_sig.assign(nc, 0.0);
        size_t q = 0;
        for (int i = b[0]; i < b[1]; i++)
            for (int j = b[2]; j < b[3]; j++)
                for (int k = b[4]; k < b[5]; k++, q++) {
                    double e, s;
                    const int m = g.eps_sig(i, j, k, &e, &s);
                    if (s != 0 || (m > 0 && d->mats[m].type != FDTD_MAT_LINTAB) ||
                        (m > 0 && d->mats[m].sigast != 0) || (g.has_m && g.vsigast[g.idx(i, j, k)] != 0)) {
                        *err = "the design region and its neighbours must be lossless LINTAB or vacuum cells";
                        return FDTD_E_INVALID;
                    }
                    hp->ctx_eps[q] = e;
                    hp->ctx_sig[q] = s;
                }
        design_coefficients(hp, d->design.eps_r);
    }
    hp->probes.clear();
    if (d->nprobes > 0) {
        if (!d->probes) { *err = "nprobes > 0 but probes is NULL"; return FDTD_E_INVALID; }
        for (int p = 0; p < d->nprobes; p++) {
            int i = d->probes[3 * p], j = d->probes[3 * p + 1], k = d->probes[3 * p + 2];
            if (i < 0 || j < 0 || k < 0 || i >= xr || j >= yr || k >= zr) { *err = "probe outside the grid"; return FDTD_E_INVALID; }
            hp->probes.push_back((int64_t)g.idx(i, j, k));
        }
    }
    return FDTD_OK;
}

// get_cabs (yee.c:1397-1493) for the affected box from the context arrays,
// after writing the design cells' new permittivities into them
void design_coefficients(HostPlan *hp, const double *eps_r)
{
    const int *b = hp->cbox, *dbx = hp->dbox, *a = hp->abox;
    const int cj = b[3] - b[2], ck = b[5] - b[4];
    auto cidx = [&](int i, int j, int k) { return ((size_t)(i - b[0]) * cj + (j - b[2])) * ck + (k - b[4]); };
    size_t q = 0;
    for (int i = dbx[0]; i < dbx[1]; i++)
        for (int j = dbx[2]; j < dbx[3]; j++)
            for (int k = dbx[4]; k < dbx[5]; k++, q++) hp->ctx_eps[cidx(i, j, k)] = eps_r[q] * EPS0;
    const size_t na = (size_t)(a[1] - a[0]) * (a[3] - a[2]) * (a[5] - a[4]);
    hp->dcoef.assign(6 * na, 0.f);
    hp->dcoef64.assign(6 * na, 0.0);
    const double dt = hp->dt, dx = hp->dx;
    q = 0;
    for (int i = a[0]; i < a[1]; i++)
        for (int j = a[2]; j < a[3]; j++)
            for (int k = a[4]; k < a[5]; k++, q++) {
                double ex, ey, ez, sx, sy, sz;
                ex = ey = ez = hp->ctx_eps[cidx(i, j, k)];
                sx = sy = sz = hp->ctx_sig[cidx(i, j, k)];
                if (hp->bnds[((size_t)i * hp->yr + j) * hp->zr + k] > 0) {   // i, j, k >= 1 here
                    auto e = [&](int ii, int jj, int kk) { return hp->ctx_eps[cidx(ii, jj, kk)]; };
                    auto s = [&](int ii, int jj, int kk) { return hp->ctx_sig[cidx(ii, jj, kk)]; };
                    ey += e(i - 1, j, k); sy += s(i - 1, j, k); ez += e(i - 1, j, k); sz += s(i - 1, j, k);
                    ex += e(i, j - 1, k); sx += s(i, j - 1, k); ez += e(i, j - 1, k); sz += s(i, j - 1, k);
                    ex += e(i, j, k - 1); sx += s(i, j, k - 1); ey += e(i, j, k - 1); sy += s(i, j, k - 1);
                    ex += e(i, j - 1, k - 1); sx += s(i, j - 1, k - 1);
                    ey += e(i - 1, j, k - 1); sy += s(i - 1, j, k - 1);
                    ez += e(i - 1, j - 1, k); sz += s(i - 1, j - 1, k);
                    ex /= 4; sx /= 4; ey /= 4; sy /= 4; ez /= 4; sz /= 4;
                }
                const double E[3] = {ex, ey, ez}, S[3] = {sx, sy, sz};
                for (int c = 0; c < 3; c++) {
                    hp->dcoef64[6 * q + c] = (1 - S[c] * dt / 2 / E[c]) / (1 + S[c] * dt / 2 / E[c]);
                    hp->dcoef64[6 * q + 3 + c] = (dt / E[c] / dx) / (1 + S[c] * dt / 2 / E[c]);
                    hp->dcoef[6 * q + c] = (float)hp->dcoef64[6 * q + c];
                    hp->dcoef[6 * q + 3 + c] = (float)hp->dcoef64[6 * q + 3 + c];
                }
            }
}

void design_gradient(const HostPlan *hp, const double *dcb, double *grad)
{
    const int *b = hp->cbox, *dbx = hp->dbox, *a = hp->abox;
    const int cj = b[3] - b[2], ck = b[5] - b[4];
    const int dj = dbx[3] - dbx[2], dk = dbx[5] - dbx[4];
    auto cidx = [&](int i, int j, int k) { return ((size_t)(i - b[0]) * cj + (j - b[2])) * ck + (k - b[4]); };
    auto in_design = [&](int i, int j, int k) {
        return i >= dbx[0] && i < dbx[1] && j >= dbx[2] && j < dbx[3] && k >= dbx[4] && k < dbx[5];
    };
    const size_t nd = (size_t)(dbx[1] - dbx[0]) * dj * dk;
    for (size_t q = 0; q < nd; q++) grad[q] = 0.0;
    const double dt = hp->dt, dx = hp->dx;
    size_t q = 0;
    for (int i = a[0]; i < a[1]; i++)
        for (int j = a[2]; j < a[3]; j++)
            for (int k = a[4]; k < a[5]; k++, q++) {
                const bool avg = hp->bnds[((size_t)i * hp->yr + j) * hp->zr + k] > 0;
                // the cells each component averages over (get_cabs), own cell first
                const int sets[3][4][3] = {{{i, j, k}, {i, j - 1, k}, {i, j, k - 1}, {i, j - 1, k - 1}},
                                           {{i, j, k}, {i - 1, j, k}, {i, j, k - 1}, {i - 1, j, k - 1}},
                                           {{i, j, k}, {i - 1, j, k}, {i, j - 1, k}, {i - 1, j - 1, k}}};
                const int nc = avg ? 4 : 1;
                for (int c = 0; c < 3; c++) {
                    double e = 0;
                    for (int m = 0; m < nc; m++) e += hp->ctx_eps[cidx(sets[c][m][0], sets[c][m][1], sets[c][m][2])];
                    e /= nc;
                    const double w = dcb[3 * q + c] * (-dt / (e * e * dx)) / nc * EPS0;
                    for (int m = 0; m < nc; m++) {
                        const int ii = sets[c][m][0], jj = sets[c][m][1], kk = sets[c][m][2];
                        if (in_design(ii, jj, kk)) grad[((size_t)(ii - dbx[0]) * dj + (jj - dbx[2])) * dk + (kk - dbx[4])] += w;
                    }
                }
            }
}

