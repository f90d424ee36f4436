// fdtd_kernels.cu -- sm_100a kernels of one GSvit FDTD time step.
//
// One step = aux_step (1D TSF grid, 1 CTA) -> fused_step (H and E of the
// whole grid in one pass) -> nfff_accumulate (running DFT on the NFFF box).
//
// fused_step marches along i (the slowest axis of the reference layout
// data[i][j][k]) over a (j,k) tile.  For plane i it first forms H^{n+1/2}(i)
// -- ystep_h (yee.c:146-265), the TSF H corrections (source.c:1464-1672),
// the CPML psi_H update and corrections (boundary.c:347-519) -- on the tile
// plus the j0-1 row and k0-1 column that the E update needs, keeps it in
// shared memory, and then forms E^{n+1}(i) -- ystep_e with the ADE branch,
// its embedded CPML, the ordinary update and the PEC rule (yee.c:530-1247),
// the CPML psi_E update and corrections (boundary.c:691-884) and the TSF E
// corrections (source.c:547-771).  H^{n+1/2}(i-1) stays in registers from the
// previous plane.  Reads come from one field set and writes go to the other,
// so the recomputed halo row never races with the CTA that owns it.
// Per cell-update the pass moves 6 field reads + 6 field writes + 1 class
// byte through HBM (49 B); halo reads are served by L1/L2.
#include <cuda_runtime.h>

#include "fdtd_kernels.cuh"

namespace {

enum { X0 = 0, XN = 1, Y0 = 2, YN = 3, Z0 = 4, ZN = 5 };

// ---------------------------------------------------------------- TSF (FP64)

// dcomp of source.c:54-107 with the reference call (i0=0, i1=xres, ...): the
// corner offsets and the rx = 0 branch are resolved on the host.
__device__ __forceinline__ double dcomp(const DevPlan &P, int i, int j, int k)
{
    double rx = P.trx_zero ? 0.0 : (double)(i - P.trx_origin);
    double ry = (double)(j - P.try_origin);
    double rz = (double)(k - P.trz_origin);
    double s = __dadd_rn(__dadd_rn(__dmul_rn(P.tax, rx), __dmul_rn(P.tay, ry)), __dmul_rn(P.taz, rz));
    return __dmul_rn(P.corr, __dadd_rn(10.0, s));
}

// sv_dline_get_dval, dline.c:89-111 (4-point cubic, linear near the ends)
__device__ __forceinline__ double dval(const double *data, int res, double x)
{
    double fl = floor(x);
    int l = (int)fl;
    double a = x - fl;
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

__device__ __forceinline__ uint8_t tflag(const DevPlan &P, int f, int a, int b)
{
    int nb = (f < 4) ? (P.t1[2] - P.t0[2] + 1) : (P.t1[1] - P.t0[1] + 1);
    return P.tmap[f][a * nb + b];
}

// TSF corrections of the H cell (i,j,k), source.c:1476-1672
__device__ void tsf_h(const DevPlan &P, int i, int j, int k, float &hx, float &hy, float &hz)
{
    const int i0 = P.t0[0], j0 = P.t0[1], k0 = P.t0[2], in = P.t1[0], jn = P.t1[1], kn = P.t1[2];
    const double hc = P.hcor;
    // i faces: j in [j0,jn], k in [k0,kn]
    if (j >= j0 && j <= jn && k >= k0 && k <= kn) {
        if (i == i0 - 1 && (tflag(P, X0, j - j0, k - k0) & 1)) {
            double ve = dval(P.aux_e, P.jres, dcomp(P, i0, j, k));
            if (k < kn) hy -= (float)(hc * (ve * P.gez));
            if (j < jn) hz += (float)(hc * (ve * P.gey));
        }
        if (i == in && (tflag(P, XN, j - j0, k - k0) & 1)) {
            double ve = dval(P.aux_e, P.jres, dcomp(P, in, j, k));
            if (k < kn) hy += (float)(hc * (ve * P.gez));
            if (j < jn) hz -= (float)(hc * (ve * P.gey));
        }
    }
    if (i >= i0 && i <= in && k >= k0 && k <= kn) {
        if (j == j0 - 1 && (tflag(P, Y0, i - i0, k - k0) & 1)) {
            double ve = dval(P.aux_e, P.jres, dcomp(P, i, j0, k));
            if (k < kn) hx += (float)(hc * (ve * P.gez));
            if (i < in) hz -= (float)(hc * (ve * P.gex));
        }
        if (j == jn && (tflag(P, YN, i - i0, k - k0) & 1)) {
            double ve = dval(P.aux_e, P.jres, dcomp(P, i, jn, k));
            if (k < kn) hx -= (float)(hc * (ve * P.gez));
            if (i < in) hz += (float)(hc * (ve * P.gex));
        }
    }
    if (i >= i0 && i <= in && j >= j0 && j <= jn) {
        if (k == k0 - 1) {
            uint8_t fl = tflag(P, Z0, i - i0, j - j0);
            if (fl & 1) {
                double ve = dval(P.aux_e, P.jres, dcomp(P, i, j, k0));
                if (j < jn && !(fl & 2)) hx -= (float)(hc * (ve * P.gey));
                if (i < in && !(fl & 2)) hy += (float)(hc * (ve * P.gex));
            }
        }
        if (k == kn && (tflag(P, ZN, i - i0, j - j0) & 1)) {
            double ve = dval(P.aux_e, P.jres, dcomp(P, i, j, kn));
            if (j < jn) hx += (float)(hc * (ve * P.gey));
            if (i < in) hy -= (float)(hc * (ve * P.gex));
        }
    }
}

// TSF corrections of the E cell (i,j,k), source.c:547-771
__device__ void tsf_e(const DevPlan &P, int i, int j, int k, float tsfe, float &ex, float &ey, float &ez)
{
    const int i0 = P.t0[0], j0 = P.t0[1], k0 = P.t0[2], in = P.t1[0], jn = P.t1[1], kn = P.t1[2];
    const double ce = (double)tsfe;
    if (j >= j0 && j <= jn && k >= k0 && k <= kn) {
        if (i == i0 && (tflag(P, X0, j - j0, k - k0) & 1)) {
            double vh = dval(P.aux_h, P.jres, dcomp(P, i0 - 1, j, k));
            if (j < jn) ey += (float)(ce * (vh * P.ghz));
            if (k < kn) ez -= (float)(ce * (vh * P.ghy));
        }
        if (i == in && (tflag(P, XN, j - j0, k - k0) & 1)) {
            double vh = dval(P.aux_h, P.jres, dcomp(P, in, j, k));
            if (j < jn) ey -= (float)(ce * (vh * P.ghz));
            if (k < kn) ez += (float)(ce * (vh * P.ghy));
        }
    }
    if (i >= i0 && i <= in && k >= k0 && k <= kn) {
        if (j == j0 && (tflag(P, Y0, i - i0, k - k0) & 1)) {
            double vh = dval(P.aux_h, P.jres, dcomp(P, i, j0 - 1, k));
            if (i < in) ex -= (float)(ce * (vh * P.ghz));
            if (k < kn) ez += (float)(ce * (vh * P.ghx));
        }
        if (j == jn && (tflag(P, YN, i - i0, k - k0) & 1)) {
            double vh = dval(P.aux_h, P.jres, dcomp(P, i, jn, k));
            if (i < in) ex += (float)(ce * (vh * P.ghz));
            if (k < kn) ez -= (float)(ce * (vh * P.ghx));
        }
    }
    if (i >= i0 && i <= in && j >= j0 && j <= jn) {
        if (k == k0) {
            uint8_t fl = tflag(P, Z0, i - i0, j - j0);
            if (fl & 1) {
                double vh = dval(P.aux_h, P.jres, dcomp(P, i, j, k0 - 1));
                if (i < in && !(fl & 2)) ex += (float)(ce * (vh * P.ghy));
                if (j < jn && !(fl & 2)) ey -= (float)(ce * (vh * P.ghx));
            }
        }
        if (k == kn && (tflag(P, ZN, i - i0, j - j0) & 1)) {
            double vh = dval(P.aux_h, P.jres, dcomp(P, i, j, kn));
            if (i < in) ex -= (float)(ce * (vh * P.ghy));
            if (j < jn) ey += (float)(ce * (vh * P.ghx));
        }
    }
}

// ------------------------------------------------------------------- H cell

struct EOwn {           // E^n at the cell and its +1 neighbours, read once
    float ex, ey, ez;
    float ey_k1, ex_k1, ez_j1, ex_j1, ez_i1, ey_i1;
};

__device__ __forceinline__ void load_e(const DevPlan &P, int64_t c, int i, int j, int k, EOwn &e)
{
    const float *EX = P.fin[0], *EY = P.fin[1], *EZ = P.fin[2];
    e.ex = __ldg(EX + c); e.ey = __ldg(EY + c); e.ez = __ldg(EZ + c);
    const bool kl = (k == P.zr - 1), jl = (j == P.yr - 1), il = (i == P.xr - 1);
    e.ey_k1 = kl ? 0.f : __ldg(EY + c + 1);
    e.ex_k1 = kl ? 0.f : __ldg(EX + c + 1);
    e.ez_j1 = jl ? 0.f : __ldg(EZ + c + P.sj);
    e.ex_j1 = jl ? 0.f : __ldg(EX + c + P.sj);
    e.ez_i1 = il ? 0.f : __ldg(EZ + c + P.si);
    e.ey_i1 = il ? 0.f : __ldg(EY + c + P.si);
}

// H^{n+1/2} of cell (i,j,k): ystep_h + TSF + CPML (+ the zeroed outer planes).
// `owner` cells also write their psi_H.
__device__ void h_cell(const DevPlan &P, const DevClass *cls, int i, int j, int k, bool owner, const EOwn &e,
                       float h[3])
{
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const DevClass &C = cls[__ldg(P.cls + c)];
    float hx = __ldg(P.fin[3] + c), hy = __ldg(P.fin[4] + c), hz = __ldg(P.fin[5] + c);
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    const bool il = (i == xr - 1), jl = (j == yr - 1), kl = (k == zr - 1);
    const float ikx = __ldg(P.ikh[0] + i), iky = __ldg(P.ikh[1] + j), ikz = __ldg(P.ikh[2] + k);
    const float dey_i = e.ey_i1 - e.ey, dez_i = e.ez_i1 - e.ez;   // E differences along x
    const float dex_j = e.ex_j1 - e.ex, dez_j = e.ez_j1 - e.ez;   // along y
    const float dex_k = e.ex_k1 - e.ex, dey_k = e.ey_k1 - e.ey;   // along z
    // ystep_h, yee.c:246-256
    if (!(jl || kl)) hx = C.da * hx + C.db * (dey_k * ikz - dez_j * iky);
    if (!(il || kl)) hy = C.da * hy + C.db * (dez_i * ikx - dex_k * ikz);
    if (!(il || jl)) hz = C.da * hz + C.db * (dex_j * iky - dey_i * ikx);
    if (P.tsf_on) tsf_h(P, i, j, k, hx, hy, hz);
    // CPML H, boundary.c:347-519; face order x0 y0 z0 xn yn zn
    const bool jin = (j >= 1 && j < yr - 1), kin = (k >= 1 && k < zr - 1), iin = (i >= 1 && i < xr - 1);
    const float dbdx = C.db * P.dx;
    const float idx_ = 1.0f / P.dx;
    if (P.cp_on[X0] && i < P.cp_d[X0] - 1 && jin && kin) {
        const int64_t q = ((int64_t)i * yr + j) * zr + k;
        const float bh = __ldg(P.bh[X0] + i), ch = __ldg(P.ch[X0] + i);
        float pzx = bh * __ldg(P.psih_in[X0][1] + q) + ch * dey_i * idx_;
        float pyx = bh * __ldg(P.psih_in[X0][0] + q) + ch * dez_i * idx_;
        hy += dbdx * pyx;
        hz -= dbdx * pzx;
        if (owner) { P.psih_out[X0][1][q] = pzx; P.psih_out[X0][0][q] = pyx; }
    }
    if (P.cp_on[Y0] && j < P.cp_d[Y0] - 1 && iin && kin) {
        const int64_t q = ((int64_t)i * P.cp_d[Y0] + j) * zr + k;
        const float bh = __ldg(P.bh[Y0] + j), ch = __ldg(P.ch[Y0] + j);
        float pxy = bh * __ldg(P.psih_in[Y0][0] + q) + ch * dez_j * idx_;
        float pzy = bh * __ldg(P.psih_in[Y0][1] + q) + ch * dex_j * idx_;
        hx -= dbdx * pxy;
        hz += dbdx * pzy;
        if (owner) { P.psih_out[Y0][0][q] = pxy; P.psih_out[Y0][1][q] = pzy; }
    }
    if (P.cp_on[Z0] && k < P.cp_d[Z0] - 1 && iin && jin) {
        const int64_t q = ((int64_t)i * yr + j) * P.cp_d[Z0] + k;
        const float bh = __ldg(P.bh[Z0] + k), ch = __ldg(P.ch[Z0] + k);
        float pyz = bh * __ldg(P.psih_in[Z0][1] + q) + ch * dex_k * idx_;
        float pxz = bh * __ldg(P.psih_in[Z0][0] + q) + ch * dey_k * idx_;
        hy -= dbdx * pyz;
        hx += dbdx * pxz;
        if (owner) { P.psih_out[Z0][1][q] = pyz; P.psih_out[Z0][0][q] = pxz; }
    }
    if (P.cp_on[XN]) {
        const int d = P.cp_d[XN];
        if (i >= xr - d + 1 && i < xr - 1 && jin && kin) {
            const int ir = i - (xr - d);
            const int64_t q = ((int64_t)ir * yr + j) * zr + k;
            const float bh = __ldg(P.bh[XN] + ir), ch = __ldg(P.ch[XN] + ir);
            float pzx = bh * __ldg(P.psih_in[XN][1] + q) + ch * dey_i * idx_;
            float pyx = bh * __ldg(P.psih_in[XN][0] + q) + ch * dez_i * idx_;
            hy += dbdx * pyx;
            hz -= dbdx * pzx;
            if (owner) { P.psih_out[XN][1][q] = pzx; P.psih_out[XN][0][q] = pyx; }
        }
    }
    if (P.cp_on[YN]) {
        const int d = P.cp_d[YN];
        if (j >= yr - d + 1 && j < yr - 1 && iin && kin) {
            const int jr = j - (yr - d);
            const int64_t q = ((int64_t)i * d + jr) * zr + k;
            const float bh = __ldg(P.bh[YN] + jr), ch = __ldg(P.ch[YN] + jr);
            float pxy = bh * __ldg(P.psih_in[YN][0] + q) + ch * dez_j * idx_;
            float pzy = bh * __ldg(P.psih_in[YN][1] + q) + ch * dex_j * idx_;
            hx -= dbdx * pxy;
            hz += dbdx * pzy;
            if (owner) { P.psih_out[YN][0][q] = pxy; P.psih_out[YN][1][q] = pzy; }
        }
    }
    if (P.cp_on[ZN]) {
        const int d = P.cp_d[ZN];
        if (k >= zr - d + 1 && k < zr - 1 && iin && jin) {
            const int kr = k - (zr - d);
            const int64_t q = ((int64_t)i * yr + j) * d + kr;
            const float bh = __ldg(P.bh[ZN] + kr), ch = __ldg(P.ch[ZN] + kr);
            float pyz = bh * __ldg(P.psih_in[ZN][1] + q) + ch * dex_k * idx_;
            float pxz = bh * __ldg(P.psih_in[ZN][0] + q) + ch * dey_k * idx_;
            hy -= dbdx * pyz;
            hx += dbdx * pxz;
            if (owner) { P.psih_out[ZN][1][q] = pyz; P.psih_out[ZN][0][q] = pxz; }
        }
    }
    // outer H planes zeroed by boundary_hstep (boundary.c:418-420, 455-457, 490-492)
    if ((P.cp_on[XN] && il && jin && kin) || (P.cp_on[YN] && jl && iin && kin) || (P.cp_on[ZN] && kl && iin && jin))
        hx = hy = hz = 0.f;
    h[0] = hx; h[1] = hy; h[2] = hz;
}

// ------------------------------------------------------------------- E cell

template <bool ADE, int NPOLES>
__device__ void e_cell(const DevPlan &P, const DevClass *cls, int i, int j, int k, const EOwn &e, const float h[3],
                       float hx_jm, float hz_jm, float hx_km, float hy_km, float hy_im, float hz_im)
{
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const DevClass &C = cls[__ldg(P.cls + c)];
    const unsigned fl = C.flags;
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    const float ikx = __ldg(P.ike[0] + i), iky = __ldg(P.ike[1] + j), ikz = __ldg(P.ike[2] + k);
    const float hx = h[0], hy = h[1], hz = h[2];
    const bool gx = (j > 0 && k > 0), gy = (i > 0 && k > 0), gz = (i > 0 && j > 0);
    // H differences along each axis (only formed where the neighbour exists)
    const float dhz_i = i > 0 ? hz - hz_im : 0.f, dhy_i = i > 0 ? hy - hy_im : 0.f;
    const float dhz_j = j > 0 ? hz - hz_jm : 0.f, dhx_j = j > 0 ? hx - hx_jm : 0.f;
    const float dhx_k = k > 0 ? hx - hx_km : 0.f, dhy_k = k > 0 ? hy - hy_km : 0.f;
    const float curlx = dhz_j * iky - dhy_k * ikz;
    const float curly = dhx_k * ikz - dhz_i * ikx;
    const float curlz = dhy_i * ikx - dhx_j * iky;
    float nx = e.ex, ny = e.ey, nz = e.ez;
    const float idx_ = 1.0f / P.dx;
    // CPML psi_E values carried from the ADE-branch update to boundary_estep
    float px0[2], pxn[2], py0[2], pyn[2], pz0[2], pzn[2];
    const bool inx0 = P.cp_on[X0] && i >= 1 && i < P.cp_d[X0];
    const bool iny0 = P.cp_on[Y0] && j >= 1 && j < P.cp_d[Y0];
    const bool inz0 = P.cp_on[Z0] && k >= 1 && k < P.cp_d[Z0];
    const bool inxn = P.cp_on[XN] && i >= xr - P.cp_d[XN] + 1;
    const bool inyn = P.cp_on[YN] && j >= yr - P.cp_d[YN] + 1;
    const bool inzn = P.cp_on[ZN] && k >= zr - P.cp_d[ZN] + 1;
    const bool zero = (P.cp_on[X0] && i == 0) || (P.cp_on[Y0] && j == 0) || (P.cp_on[Z0] && k == 0);
    int64_t qx0 = 0, qxn = 0, qy0 = 0, qyn = 0, qz0 = 0, qzn = 0;
    if (!zero) {
        if (inx0) { qx0 = ((int64_t)i * yr + j) * zr + k; px0[0] = P.psie[X0][0][qx0]; px0[1] = P.psie[X0][1][qx0]; }
        if (inxn) { qxn = ((int64_t)(i - (xr - P.cp_d[XN])) * yr + j) * zr + k; pxn[0] = P.psie[XN][0][qxn]; pxn[1] = P.psie[XN][1][qxn]; }
        if (iny0) { qy0 = ((int64_t)i * P.cp_d[Y0] + j) * zr + k; py0[0] = P.psie[Y0][0][qy0]; py0[1] = P.psie[Y0][1][qy0]; }
        if (inyn) { qyn = ((int64_t)i * P.cp_d[YN] + (j - (yr - P.cp_d[YN]))) * zr + k; pyn[0] = P.psie[YN][0][qyn]; pyn[1] = P.psie[YN][1][qyn]; }
        if (inz0) { qz0 = ((int64_t)i * yr + j) * P.cp_d[Z0] + k; pz0[0] = P.psie[Z0][0][qz0]; pz0[1] = P.psie[Z0][1][qz0]; }
        if (inzn) { qzn = ((int64_t)i * yr + j) * P.cp_d[ZN] + (k - (zr - P.cp_d[ZN])); pzn[0] = P.psie[ZN][0][qzn]; pzn[1] = P.psie[ZN][1][qzn]; }
    }
    if (ADE && (fl & CF_ADE_BRANCH)) {
        // ADE (Drude + critical points) branch, yee.c:914-1108
        const DevAde &A = P.ade[C.ade];
        const bool ax = (fl & CF_ADE_X) != 0, ay = (fl & CF_ADE_Y) != 0, az = (fl & CF_ADE_Z) != 0;
        float dp[3], dpp[3], ep[3], p[3][2], pp[3][2];
        const float eo[3] = {e.ex, e.ey, e.ez};
        const bool comp[3] = {ax, ay, az};
        for (int a = 0; a < 3; a++) {
            if (!comp[a]) continue;
            dp[a] = P.dp[a][c]; dpp[a] = P.dpp[a][c]; ep[a] = P.ep[a][c];
            for (int n = 0; n < NPOLES; n++) { p[a][n] = P.p_[a][n][c]; pp[a][n] = P.pp_[a][n][c]; }
        }
        const float curl[3] = {curlx, curly, curlz};
        const bool gd[3] = {gx, gy, gz};
        float ne[3] = {nx, ny, nz};
        for (int a = 0; a < 3; a++) {
            if (!(comp[a] && gd[a])) continue;
            float v = A.c0dx * curl[a] + A.c1 * (-A.a0 * dpp[a] + A.one_m_a1 * dp[a]);
            for (int n = 0; n < NPOLES; n++) v += A.c1 * (-A.bp0[n] * pp[a][n] + A.one_m_bp1[n] * p[a][n]);
            v += A.c2 * ep[a] + A.c3 * eo[a];
            ne[a] = v;
        }
        // CPML inside the ADE branch, yee.c:950-1057 (first psi_E update)
        if (!zero) {
            if (inx0 && i > 1) {   // x0: corrections scaled by cb == 0 (yee.c:577)
                const float be = __ldg(P.be[X0] + i), ce = __ldg(P.ce[X0] + i);
                px0[0] = be * px0[0] + ce * dhz_i * idx_;
                px0[1] = be * px0[1] + ce * dhy_i * idx_;
            }
            if (iny0 && j > 1) {
                const float be = __ldg(P.be[Y0] + j), ce = __ldg(P.ce[Y0] + j);
                py0[0] = be * py0[0] + ce * dhz_j * idx_;
                py0[1] = be * py0[1] + ce * dhx_j * idx_;
                if ((i > 0 && k > 0) && ax) ne[0] += P.dx * C.cba[0] * py0[0];
                if ((i > 0 && k > 0) && az) ne[2] -= P.dx * C.cba[2] * py0[1];
            }
            if (inz0 && k > 1) {
                const float be = __ldg(P.be[Z0] + k), ce = __ldg(P.ce[Z0] + k);
                pz0[1] = be * pz0[1] + ce * dhx_k * idx_;   // peyz
                pz0[0] = be * pz0[0] + ce * dhy_k * idx_;   // pexz
                if ((i > 0 && j > 0) && ay) ne[1] += P.dx * C.cba[1] * pz0[1];
                if ((i > 0 && j > 0) && ax) ne[0] -= P.dx * C.cba[0] * pz0[0];
            }
            if (inxn) {
                const int ir = i - (xr - P.cp_d[XN]);
                const float be = __ldg(P.be[XN] + ir), ce = __ldg(P.ce[XN] + ir);
                pxn[0] = be * pxn[0] + ce * dhz_i * idx_;
                pxn[1] = be * pxn[1] + ce * dhy_i * idx_;
                if ((j > 0 && k > 0) && ay) ne[1] -= P.dx * C.cba[1] * pxn[0];
                if ((j > 0 && k > 0) && az) ne[2] += P.dx * C.cba[2] * pxn[1];
            }
            if (inyn) {
                const int jr = j - (yr - P.cp_d[YN]);
                const float be = __ldg(P.be[YN] + jr), ce = __ldg(P.ce[YN] + jr);
                pyn[0] = be * pyn[0] + ce * dhz_j * idx_;
                pyn[1] = be * pyn[1] + ce * dhx_j * idx_;
                if ((i > 0 && k > 0) && ax) ne[0] += P.dx * C.cba[0] * pyn[0];
                if ((i > 0 && k > 0) && az) ne[2] -= P.dx * C.cba[2] * pyn[1];
            }
            if (inzn) {
                const int kr = k - (zr - P.cp_d[ZN]);
                const float be = __ldg(P.be[ZN] + kr), ce = __ldg(P.ce[ZN] + kr);
                pzn[1] = be * pzn[1] + ce * dhx_k * idx_;
                pzn[0] = be * pzn[0] + ce * dhy_k * idx_;
                if ((i > 0 && j > 0) && ay) ne[1] += P.dx * C.cba[1] * pzn[1];
                if ((i > 0 && j > 0) && ax) ne[0] -= P.dx * C.cba[0] * pzn[0];
            }
        }
        // polarisation recursions (only components the branch owns are ever read back)
        for (int a = 0; a < 3; a++) {
            if (!comp[a]) continue;
            const float en = ne[a];
            P.dp[a][c] = A.a0 * dpp[a] + A.a1 * dp[a] + A.a2 * (ep[a] + 2.f * eo[a] + en);
            for (int n = 0; n < NPOLES; n++) {
                P.p_[a][n][c] = A.bp0[n] * pp[a][n] + A.bp1[n] * p[a][n] + A.bp2[n] * ep[a] + A.bp3[n] * eo[a] + A.bp4[n] * en;
                P.pp_[a][n][c] = p[a][n];
            }
            P.ep[a][c] = eo[a];
            P.dpp[a][c] = dp[a];
        }
        nx = ne[0]; ny = ne[1]; nz = ne[2];
    }
    // ordinary update of the components left (yee.c:1113-1128)
    if (gx && !(ADE && (fl & CF_ADE_X))) nx = C.ca[0] * e.ex + C.cb[0] * curlx;
    if (gy && !(ADE && (fl & CF_ADE_Y))) ny = C.ca[1] * e.ey + C.cb[1] * curly;
    if (gz && !(ADE && (fl & CF_ADE_Z))) nz = C.ca[2] * e.ez + C.cb[2] * curlz;
    // PEC rule (yee.c:1138-1237)
    if (fl & CF_PEC_X) nx = 0.f;
    if (fl & CF_PEC_Y) ny = 0.f;
    if (fl & CF_PEC_Z) nz = 0.f;
    // boundary_estep: zeroed planes and psi_E (second update for ADE cells), boundary.c:691-884
    if (zero) {
        nx = ny = nz = 0.f;
    } else {
        const bool tx = !(fl & CF_ADE_X), ty = !(fl & CF_ADE_Y), tz = !(fl & CF_ADE_Z);
        const float dx = P.dx;
        if (inx0) {
            const float be = __ldg(P.be[X0] + i), ce = __ldg(P.ce[X0] + i);
            px0[0] = be * px0[0] + ce * dhz_i * idx_;
            px0[1] = be * px0[1] + ce * dhy_i * idx_;
            if (j > 0 && k > 0) {
                if (ty) ny -= dx * C.cb[1] * px0[0];
                if (tz) nz += dx * C.cb[2] * px0[1];
            }
            if (j > 0 && k > 0) { P.psie[X0][0][qx0] = px0[0]; P.psie[X0][1][qx0] = px0[1]; }
        }
        if (iny0) {
            const float be = __ldg(P.be[Y0] + j), ce = __ldg(P.ce[Y0] + j);
            py0[0] = be * py0[0] + ce * dhz_j * idx_;
            py0[1] = be * py0[1] + ce * dhx_j * idx_;
            if (i > 0 && k > 0) {
                if (tx) nx += dx * C.cb[0] * py0[0];
                if (tz) nz -= dx * C.cb[2] * py0[1];
                P.psie[Y0][0][qy0] = py0[0]; P.psie[Y0][1][qy0] = py0[1];
            }
        }
        if (inz0) {
            const float be = __ldg(P.be[Z0] + k), ce = __ldg(P.ce[Z0] + k);
            pz0[1] = be * pz0[1] + ce * dhx_k * idx_;
            pz0[0] = be * pz0[0] + ce * dhy_k * idx_;
            if (i > 0 && j > 0) {
                if (ty) ny += dx * C.cb[1] * pz0[1];
                if (tz) nx -= dx * C.cb[0] * pz0[0];     // gated by ztbc in the reference (boundary.c:758-759)
                P.psie[Z0][0][qz0] = pz0[0]; P.psie[Z0][1][qz0] = pz0[1];
            }
        }
        if (inxn) {
            const int ir = i - (xr - P.cp_d[XN]);
            const float be = __ldg(P.be[XN] + ir), ce = __ldg(P.ce[XN] + ir);
            pxn[0] = be * pxn[0] + ce * dhz_i * idx_;
            pxn[1] = be * pxn[1] + ce * dhy_i * idx_;
            if (j > 0 && k > 0) {
                if (ty) ny -= dx * C.cb[1] * pxn[0];
                if (tz) nz += dx * C.cb[2] * pxn[1];
                P.psie[XN][0][qxn] = pxn[0]; P.psie[XN][1][qxn] = pxn[1];
            }
        }
        if (inyn) {
            const int jr = j - (yr - P.cp_d[YN]);
            const float be = __ldg(P.be[YN] + jr), ce = __ldg(P.ce[YN] + jr);
            pyn[0] = be * pyn[0] + ce * dhz_j * idx_;
            pyn[1] = be * pyn[1] + ce * dhx_j * idx_;
            if (i > 0 && k > 0) {
                if (tx) nx += dx * C.cb[0] * pyn[0];
                if (tz) nz -= dx * C.cb[2] * pyn[1];
                P.psie[YN][0][qyn] = pyn[0]; P.psie[YN][1][qyn] = pyn[1];
            }
        }
        if (inzn) {
            const int kr = k - (zr - P.cp_d[ZN]);
            const float be = __ldg(P.be[ZN] + kr), ce = __ldg(P.ce[ZN] + kr);
            pzn[1] = be * pzn[1] + ce * dhx_k * idx_;
            pzn[0] = be * pzn[0] + ce * dhy_k * idx_;
            if (i > 0 && j > 0) {
                if (ty) ny += dx * C.cb[1] * pzn[1];
                if (tx) nx -= dx * C.cb[0] * pzn[0];
                P.psie[ZN][0][qzn] = pzn[0]; P.psie[ZN][1][qzn] = pzn[1];
            }
        }
    }
    if (P.tsf_on) tsf_e(P, i, j, k, C.tsfe, nx, ny, nz);
    P.fout[0][c] = nx;
    P.fout[1][c] = ny;
    P.fout[2][c] = nz;
}

// ------------------------------------------------------------ fused kernel

template <bool ADE, int NPOLES>
__global__ void __launch_bounds__(FDTD_TK * FDTD_TJ, 2) fused_step_kernel(const DevPlan P, int ichunk)
{
    constexpr int TK = FDTD_TK, TJ = FDTD_TJ;
    __shared__ float sh[3][TJ + 1][TK + 1];          // H^{n+1/2}(i) with the j0-1 row and k0-1 column
    __shared__ DevClass scls[FDTD_MAX_CLASSES];
    const int tid = threadIdx.x;
    const int tk = tid % TK, tj = tid / TK;
    const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
    const int k = k0 + tk, j = j0 + tj;
    const bool own = (k < P.zr) && (j < P.yr);
    const int ib = blockIdx.z * ichunk;
    const int ie = min(P.xr, ib + ichunk);
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(P.classes);
        uint32_t *dst = reinterpret_cast<uint32_t *>(scls);
        const int words = P.nclasses * (int)(sizeof(DevClass) / 4);
        for (int w = tid; w < words; w += TK * TJ) dst[w] = src[w];
    }
    // halo cell owned by this thread: row j0-1 (tid < TK) or column k0-1
    int hj = -1, hk = -1;
    if (tid < TK) { hj = j0 - 1; hk = k0 + tid; }
    else if (tid < TK + TJ) { hj = j0 + (tid - TK); hk = k0 - 1; }
    const bool halo = hj >= 0 && hk >= 0 && hj < P.yr && hk < P.zr;
    __syncthreads();

    float hy_im = 0.f, hz_im = 0.f;   // H^{n+1/2}(i-1) at this thread's cell
    if (ib > 0 && own) {
        EOwn e;
        float h[3];
        load_e(P, (int64_t)(ib - 1) * P.si + (int64_t)j * P.sj + k, ib - 1, j, k, e);
        h_cell(P, scls, ib - 1, j, k, false, e, h);
        hy_im = h[1];
        hz_im = h[2];
    }
    for (int i = ib; i < ie; i++) {
        EOwn e;
        float h[3] = {0.f, 0.f, 0.f};
        const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
        if (own) {
            load_e(P, c, i, j, k, e);
            h_cell(P, scls, i, j, k, true, e, h);
            sh[0][tj + 1][tk + 1] = h[0];
            sh[1][tj + 1][tk + 1] = h[1];
            sh[2][tj + 1][tk + 1] = h[2];
            P.fout[3][c] = h[0];
            P.fout[4][c] = h[1];
            P.fout[5][c] = h[2];
        }
        if (halo) {
            EOwn eh;
            float hh[3];
            load_e(P, (int64_t)i * P.si + (int64_t)hj * P.sj + hk, i, hj, hk, eh);
            h_cell(P, scls, i, hj, hk, false, eh, hh);
            sh[0][hj - j0 + 1][hk - k0 + 1] = hh[0];
            sh[1][hj - j0 + 1][hk - k0 + 1] = hh[1];
            sh[2][hj - j0 + 1][hk - k0 + 1] = hh[2];
        }
        __syncthreads();
        if (own) {
            e_cell<ADE, NPOLES>(P, scls, i, j, k, e, h, sh[0][tj][tk + 1], sh[2][tj][tk + 1], sh[0][tj + 1][tk],
                                sh[1][tj + 1][tk], hy_im, hz_im);
        }
        hy_im = h[1];
        hz_im = h[2];
        __syncthreads();
    }
}

// ------------------------------------------------------------ 1D aux grid

// 1D TSF grid step of source.c:1469-1473 over 1dpool.c:84-162, in FP64 with
// the reference's operation order (no contraction); also records the probes
// of the previous step (output.c:341-352).
__global__ void aux_step_kernel(const DevAux A)
{
    const int s = *A.step;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (s > 0 && s - 1 < A.nsteps_planned) {
        for (int q = tid; q < A.nprobes * 6; q += nt) {
            int p = q / 6, comp = q % 6;
            A.probe_out[((size_t)p * A.nsteps_planned + (s - 1)) * 6 + comp] = (double)A.fields[comp][A.probe_cells[p]];
        }
    }
    if (A.res > 0) {
        double *e = A.e, *h = A.h;
        const int r = A.res;
        for (int i = 1 + tid; i < r; i += nt)               // sv_1dpool_ystep_e
            e[i] = __dadd_rn(e[i], __dmul_rn(A.ce, __dadd_rn(h[i - 1], -h[i])));
        __syncthreads();
        if (tid == 0) {
            double *b = A.bnd;
            e[0] = __dadd_rn(b[1], __dmul_rn(A.lc, __dadd_rn(e[1], -b[0])));          // sv_1dpool_boundary
            h[0] = __dadd_rn(b[3], __dmul_rn(A.lc, __dadd_rn(h[1], -b[2])));
            e[r - 1] = __dadd_rn(b[5], __dmul_rn(A.lc, __dadd_rn(e[r - 2], -b[4])));
            h[r - 1] = __dadd_rn(b[7], __dmul_rn(A.lc, __dadd_rn(h[r - 2], -b[6])));
            b[0] = e[0]; b[1] = e[1]; b[2] = h[0]; b[3] = h[1];                          // _boundary_copy
            b[4] = e[r - 1]; b[5] = e[r - 2]; b[6] = h[r - 1]; b[7] = h[r - 2];
            e[0] = (s < A.nwave) ? A.wave[s] : 0.0;                                        // _apply_source
        }
        __syncthreads();
        for (int i = tid; i < r - 1; i += nt)               // sv_1dpool_ystep_h
            h[i] = __dadd_rn(h[i], __dmul_rn(A.chh, __dadd_rn(e[i], -e[i + 1])));
    }
    __syncthreads();
    if (tid == 0) *A.step = s + 1;
}

__global__ void probe_capture_kernel(const DevAux A)
{
    const int s = *A.step;     // number of completed steps
    if (s < 1 || s - 1 >= A.nsteps_planned) return;
    for (int q = threadIdx.x; q < A.nprobes * 6; q += blockDim.x) {
        int p = q / 6, comp = q % 6;
        A.probe_out[((size_t)p * A.nsteps_planned + (s - 1)) * 6 + comp] = (double)A.fields[comp][A.probe_cells[p]];
    }
}

// ------------------------------------------------------------ NFFF running DFT

// Per surface cell s and frequency f:  Ehat += E(step) w,  Dhat += dE/dn(step) w,
// w = exp(-i omega step dt).  FP64 accumulators.
__global__ void nfff_accumulate_kernel(const DevNfff N)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N.ns) return;
    const int step = *N.step - 1;
    const int64_t c = N.cell[s];
    const int64_t st = N.nstride[s];
    double v[6];
    for (int a = 0; a < 3; a++) {
        const float *E = N.e[a];
        v[a] = (double)E[c];
        v[3 + a] = ((double)E[c + st] - (double)E[c - st]) * N.inv2dx;
    }
    for (int f = 0; f < N.nfreq; f++) {
        double sn, cs;
        sincos(N.omega_dt[f] * (double)step, &sn, &cs);
        for (int q = 0; q < 6; q++) {
            double2 &A = N.acc[((size_t)f * 6 + q) * N.ns + s];
            A.x += v[q] * cs;
            A.y -= v[q] * sn;
        }
    }
}

// ------------------------------------------------------------ far-field integration

// F_hat_n(omega) = sum_s A_s exp(-i omega (1 + R_ns - istart_n) dt) *
//   [(-c' + b e^{i omega dt} + c' e^{2 i omega dt}) Ehat_s + sgn_f a e^{i omega dt} Dhat_s]
// with r, cos(theta), a, b, c, R of farfield.c:175-405 (the DFT of the
// reference time-domain series).  One block per (point, frequency).
__global__ void farfield_finalize_kernel(const DevFarfield F)
{
    const int pf = blockIdx.x;
    const int p = pf / F.nfreq, f = pf % F.nfreq;
    const double x = F.points[3 * p], y = F.points[3 * p + 1], z = F.points[3 * p + 2];
    const double om = F.omega[f], dt = F.dt, dx = F.dx;
    const double C0 = 299792458.0, PI = 3.14159265358979323846;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    double sw, cw, s2, c2;
    sincos(om * dt, &sw, &cw);
    sincos(2.0 * om * dt, &s2, &c2);
    for (int s = threadIdx.x; s < F.ns; s += blockDim.x) {
        const int fc = F.face[s];
        const double ci = F.cell_ijk[3 * s], cj = F.cell_ijk[3 * s + 1], ck = F.cell_ijk[3 * s + 2];
        const double rx = x - ci, ry = y - cj, rz = z - ck;
        const double rc = sqrt(rx * rx + ry * ry + rz * rz);
        // angle(): normal of the face (farfield.c:44-54)
        double dot;
        if (fc == 0) dot = -rx; else if (fc == 1) dot = rx; else if (fc == 2) dot = -ry;
        else if (fc == 3) dot = ry; else if (fc == 4) dot = -rz; else dot = rz;
        const double ct = dot / sqrt((rx * rx + ry * ry + rz * rz) * 1.0);
        const double area = dx * dx;
        const double r = rc * dx;
        const int R = (int)(1.0 + r / (C0 * dt));
        const double a = 1.0 / (4.0 * PI * r);
        const double b = -1.0 / (4.0 * PI) * ct / (r * r);
        const double cc = -1.0 / (4.0 * PI) * ct / (C0 * r);
        const double cp = cc / 2.0 / dt;
        const double sg = (fc & 1) ? 1.0 : -1.0;
        // K = -c' + b e^{i w dt} + c' e^{2 i w dt};  L = sg * a * e^{i w dt}
        const double Kr = -cp + b * cw + cp * c2, Ki = b * sw + cp * s2;
        const double Lr = sg * a * cw, Li = sg * a * sw;
        double ph_s, ph_c;
        sincos(-om * (double)(R - F.istart[p]) * dt, &ph_s, &ph_c);
        for (int q = 0; q < 3; q++) {
            const double2 Eh = F.acc[((size_t)f * 6 + q) * F.ns + s];
            const double2 Dh = F.acc[((size_t)f * 6 + 3 + q) * F.ns + s];
            const double tr = Kr * Eh.x - Ki * Eh.y + Lr * Dh.x - Li * Dh.y;
            const double ti = Kr * Eh.y + Ki * Eh.x + Lr * Dh.y + Li * Dh.x;
            acc[2 * q] += area * (ph_c * tr - ph_s * ti);
            acc[2 * q + 1] += area * (ph_c * ti + ph_s * tr);
        }
    }
    // block reduction: warp shuffles then shared memory
    __shared__ double red[32][6];
    for (int q = 0; q < 6; q++)
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int q = 0; q < 6; q++) red[warp][q] = acc[q];
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        for (int q = 0; q < 6; q++) {
            double v = lane < nw ? red[lane][q] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) acc[q] = v;
        }
        if (lane == 0)
            for (int q = 0; q < 3; q++) F.out[((size_t)p * F.nfreq + f) * 3 + q] = make_double2(acc[2 * q], acc[2 * q + 1]);
    }
}

}  // namespace

void launch_aux_step(const DevAux &a, cudaStream_t st) { aux_step_kernel<<<1, 1024, 0, st>>>(a); }

void launch_probe_capture(const DevAux &a, cudaStream_t st) { probe_capture_kernel<<<1, 256, 0, st>>>(a); }

cudaError_t launch_fused_step(const DevPlan &p, int ichunk, bool ade, int npoles, cudaStream_t st)
{
    dim3 grid((p.zr + FDTD_TK - 1) / FDTD_TK, (p.yr + FDTD_TJ - 1) / FDTD_TJ, (p.xr + ichunk - 1) / ichunk);
    dim3 block(FDTD_TK * FDTD_TJ);
    if (!ade)
        fused_step_kernel<false, 0><<<grid, block, 0, st>>>(p, ichunk);
    else if (npoles == 0)
        fused_step_kernel<true, 0><<<grid, block, 0, st>>>(p, ichunk);
    else
        fused_step_kernel<true, 2><<<grid, block, 0, st>>>(p, ichunk);
    return cudaGetLastError();
}

void launch_nfff_accumulate(const DevNfff &n, cudaStream_t st)
{
    if (n.ns <= 0) return;
    nfff_accumulate_kernel<<<(n.ns + 255) / 256, 256, 0, st>>>(n);
}

void launch_farfield_finalize(const DevFarfield &f, cudaStream_t st)
{
    if (f.npoints <= 0 || f.nfreq <= 0) return;
    farfield_finalize_kernel<<<f.npoints * f.nfreq, 256, 0, st>>>(f);
}
