// fdtd_cells.cuh -- the per-cell special path of the Yee step: the CPML
// psi recursions and corrections, the zeroed outer planes, kappa, the ADE
// branch with its embedded CPML, the PEC rule and the TSF corrections.  Shared
// by the slab kernels (fdtd_kernels.cu) and the CPML tiles of the TMA kernel
// (fdtd_bulk.cu); each translation unit gets its own copy.  Templated on the
// storage type T, whose arithmetic type R = real_t<T> is FP32, or FP64 for
// FP64 storage.
#pragma once
#include <cuda_runtime.h>

#include "fdtd_device.cuh"

namespace {

enum { X0 = 0, XN = 1, Y0 = 2, YN = 3, Z0 = 4, ZN = 5 };

// ------------------------------------------------------------ cell updates

// CPML psi_H update and corrections (boundary.c:347-519, face order x0 y0 z0
// xn yn zn), TSF H corrections (source.c:1476-1672) and the outer H planes
// zeroed by boundary_hstep (boundary.c:418-420, 455-457, 490-492), applied to
// H after ystep_h.  `owner` cells write their psi_H.
template <class T, class R = real_t<T>>
__device__ __forceinline__ V3<R> h_special(const DevPlan &P, int i, int j, int k, bool owner, bool tsf, R db, R dey_i, R dez_i,
                                           R dex_j, R dez_j, R dex_k, R dey_k, V3<R> hin)
{
    const uint32_t stp = sr_step<T>(P);
    R hx = hin.x, hy = hin.y, hz = hin.z;
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    const bool il = (i == xr - 1), jl = (j == yr - 1), kl = (k == zr - 1);
    if (tsf && P.tsf_on) tsf_add_h(P, i, j, k, hx, hy, hz);
    const bool jin = (j >= 1 && j < yr - 1), kin = (k >= 1 && k < zr - 1), iin = (i >= 1 && i < xr - 1);
    const R dx = Tab<R>::dx(P);
    const R dbdx = db * dx;
    const R idx_ = R(1) / dx;
    if (P.cp_on[X0] && i < P.cp_d[X0] - 1 && jin && kin) {
        const int64_t q = ((int64_t)i * yr + j) * zr + k;
        const R bh = Tab<R>::ld(P.bh[X0], i), ch = Tab<R>::ld(P.ch[X0], i);
        R pzx = bh * ldgPsi<T>(P, P.psih_in[X0][1], q) + ch * dey_i * idx_;
        R pyx = bh * ldgPsi<T>(P, P.psih_in[X0][0], q) + ch * dez_i * idx_;
        hy += dbdx * pyx;
        hz -= dbdx * pzx;
        if (owner) { stPsi<T>(P, P.psih_out[X0][1], q, pzx, stp, 18 + 2 * X0 + 1); stPsi<T>(P, P.psih_out[X0][0], q, pyx, stp, 18 + 2 * X0 + 0); }
    }
    if (P.cp_on[Y0] && j < P.cp_d[Y0] - 1 && iin && kin) {
        const int64_t q = ((int64_t)i * P.cp_d[Y0] + j) * zr + k;
        const R bh = Tab<R>::ld(P.bh[Y0], j), ch = Tab<R>::ld(P.ch[Y0], j);
        R pxy = bh * ldgPsi<T>(P, P.psih_in[Y0][0], q) + ch * dez_j * idx_;
        R pzy = bh * ldgPsi<T>(P, P.psih_in[Y0][1], q) + ch * dex_j * idx_;
        hx -= dbdx * pxy;
        hz += dbdx * pzy;
        if (owner) { stPsi<T>(P, P.psih_out[Y0][0], q, pxy, stp, 18 + 2 * Y0 + 0); stPsi<T>(P, P.psih_out[Y0][1], q, pzy, stp, 18 + 2 * Y0 + 1); }
    }
    if (P.cp_on[Z0] && k < P.cp_d[Z0] - 1 && iin && jin) {
        const int64_t q = ((int64_t)i * yr + j) * P.cp_d[Z0] + k;
        const R bh = Tab<R>::ld(P.bh[Z0], k), ch = Tab<R>::ld(P.ch[Z0], k);
        R pyz = bh * ldgPsi<T>(P, P.psih_in[Z0][1], q) + ch * dex_k * idx_;
        R pxz = bh * ldgPsi<T>(P, P.psih_in[Z0][0], q) + ch * dey_k * idx_;
        hy -= dbdx * pyz;
        hx += dbdx * pxz;
        if (owner) { stPsi<T>(P, P.psih_out[Z0][1], q, pyz, stp, 18 + 2 * Z0 + 1); stPsi<T>(P, P.psih_out[Z0][0], q, pxz, stp, 18 + 2 * Z0 + 0); }
    }
    if (P.cp_on[XN]) {
        const int d = P.cp_d[XN];
        if (i >= xr - d + 1 && i < xr - 1 && jin && kin) {
            const int ir = i - (xr - d);
            const int64_t q = ((int64_t)ir * yr + j) * zr + k;
            const R bh = Tab<R>::ld(P.bh[XN], ir), ch = Tab<R>::ld(P.ch[XN], ir);
            R pzx = bh * ldgPsi<T>(P, P.psih_in[XN][1], q) + ch * dey_i * idx_;
            R pyx = bh * ldgPsi<T>(P, P.psih_in[XN][0], q) + ch * dez_i * idx_;
            hy += dbdx * pyx;
            hz -= dbdx * pzx;
            if (owner) { stPsi<T>(P, P.psih_out[XN][1], q, pzx, stp, 18 + 2 * XN + 1); stPsi<T>(P, P.psih_out[XN][0], q, pyx, stp, 18 + 2 * XN + 0); }
        }
    }
    if (P.cp_on[YN]) {
        const int d = P.cp_d[YN];
        if (j >= yr - d + 1 && j < yr - 1 && iin && kin) {
            const int jr = j - (yr - d);
            const int64_t q = ((int64_t)i * d + jr) * zr + k;
            const R bh = Tab<R>::ld(P.bh[YN], jr), ch = Tab<R>::ld(P.ch[YN], jr);
            R pxy = bh * ldgPsi<T>(P, P.psih_in[YN][0], q) + ch * dez_j * idx_;
            R pzy = bh * ldgPsi<T>(P, P.psih_in[YN][1], q) + ch * dex_j * idx_;
            hx -= dbdx * pxy;
            hz += dbdx * pzy;
            if (owner) { stPsi<T>(P, P.psih_out[YN][0], q, pxy, stp, 18 + 2 * YN + 0); stPsi<T>(P, P.psih_out[YN][1], q, pzy, stp, 18 + 2 * YN + 1); }
        }
    }
    if (P.cp_on[ZN]) {
        const int d = P.cp_d[ZN];
        if (k >= zr - d + 1 && k < zr - 1 && iin && jin) {
            const int kr = k - (zr - d);
            const int64_t q = ((int64_t)i * yr + j) * d + kr;
            const R bh = Tab<R>::ld(P.bh[ZN], kr), ch = Tab<R>::ld(P.ch[ZN], kr);
            R pyz = bh * ldgPsi<T>(P, P.psih_in[ZN][1], q) + ch * dex_k * idx_;
            R pxz = bh * ldgPsi<T>(P, P.psih_in[ZN][0], q) + ch * dey_k * idx_;
            hy -= dbdx * pyz;
            hx += dbdx * pxz;
            if (owner) { stPsi<T>(P, P.psih_out[ZN][1], q, pyz, stp, 18 + 2 * ZN + 1); stPsi<T>(P, P.psih_out[ZN][0], q, pxz, stp, 18 + 2 * ZN + 0); }
        }
    }
    if ((P.cp_on[XN] && il && jin && kin) || (P.cp_on[YN] && jl && iin && kin) || (P.cp_on[ZN] && kl && iin && jin))
        hx = hy = hz = 0;
    return V3<R>{hx, hy, hz};
}

// H^{n+1/2}(i) at one cell from E^n and the six E differences (ystep_h,
// yee.c:246-256, then h_special where the cell lies in a slab or on a face).
template <class T, class R = real_t<T>>
__device__ __forceinline__ void h_update(const DevPlan &P, const float4 *scls, int cls, int i, int j, int k,
                                         bool special, bool owner, bool tsf, R dey_i, R dez_i, R dex_j, R dez_j,
                                         R dex_k, R dey_k, R h[3])
{
    R da, db;
    Tab<R>::hcoef(P, scls, cls, da, db);
    const bool il = (i == P.xr - 1), jl = (j == P.yr - 1), kl = (k == P.zr - 1);
    R ikx = 1, iky = 1, ikz = 1;
    if (special) { ikx = Tab<R>::ld(P.ikh[0], i); iky = Tab<R>::ld(P.ikh[1], j); ikz = Tab<R>::ld(P.ikh[2], k); }
    if (!(jl || kl)) h[0] = da * h[0] + db * (dey_k * ikz - dez_j * iky);
    if (!(il || kl)) h[1] = da * h[1] + db * (dez_i * ikx - dex_k * ikz);
    if (!(il || jl)) h[2] = da * h[2] + db * (dex_j * iky - dey_i * ikx);
    if (special) {
        const V3<R> o = h_special<T>(P, i, j, k, owner, tsf, db, dey_i, dez_i, dex_j, dez_j, dex_k, dey_k, V3<R>{h[0], h[1], h[2]});
        h[0] = o.x; h[1] = o.y; h[2] = o.z;
    }
}

// E^{n+1}(i) of one cell on the general path: ADE branch with its CPML
// (yee.c:914-1108), ordinary update (yee.c:1113-1128), PEC rule
// (yee.c:1138-1237), boundary_estep zero planes, psi_E and corrections
// (boundary.c:691-884) and TSF E (source.c:547-771).
template <bool ADE, int NPOLES, class T, class R = real_t<T>>
__device__ __noinline__ V3<R> e_special(const DevPlan &P, const float4 *scls, int cls, int i, int j, int k, bool tsf,
                                        V3<R> eo3, V3<R> h3, R hx_jm, R hz_jm, R hx_km, R hy_km, R hy_im, R hz_im)
{
    const uint32_t stp = sr_step<T>(P);
    const R eo[3] = {eo3.x, eo3.y, eo3.z};
    const R h[3] = {h3.x, h3.y, h3.z};
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    R ca[3], cb[3], cba[3];
    unsigned fl;
    int ade_set;
    Tab<R>::ecoef(P, scls, cls, ca, cb, cba, fl, ade_set);
    if (fl & CF_DESIGN) {   // adjoint design region: coefficients per cell
        const int64_t q = ((int64_t)(i - P.dbox[0]) * (P.dbox[3] - P.dbox[2]) + (j - P.dbox[2])) * (P.dbox[5] - P.dbox[4]) + (k - P.dbox[4]);
        for (int a = 0; a < 3; a++) { ca[a] = Tab<R>::ld(P.dcoef, 6 * q + a); cb[a] = Tab<R>::ld(P.dcoef, 6 * q + 3 + a); }
    }
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    const R ikx = Tab<R>::ld(P.ike[0], i), iky = Tab<R>::ld(P.ike[1], j), ikz = Tab<R>::ld(P.ike[2], k);
    const R hx = h[0], hy = h[1], hz = h[2];
    const bool gx = (j > 0 && k > 0), gy = (i > 0 && k > 0), gz = (i > 0 && j > 0);
    const R dhz_i = i > 0 ? hz - hz_im : R(0), dhy_i = i > 0 ? hy - hy_im : R(0);
    const R dhz_j = j > 0 ? hz - hz_jm : R(0), dhx_j = j > 0 ? hx - hx_jm : R(0);
    const R dhx_k = k > 0 ? hx - hx_km : R(0), dhy_k = k > 0 ? hy - hy_km : R(0);
    const R curlx = dhz_j * iky - dhy_k * ikz;
    const R curly = dhx_k * ikz - dhz_i * ikx;
    const R curlz = dhy_i * ikx - dhx_j * iky;
    R nx = eo[0], ny = eo[1], nz = eo[2];
    const R dx = Tab<R>::dx(P);
    const R idx_ = R(1) / dx;
    R px0[2] = {0, 0}, pxn[2] = {0, 0}, py0[2] = {0, 0}, pyn[2] = {0, 0}, pz0[2] = {0, 0}, pzn[2] = {0, 0};
    const bool inx0 = P.cp_on[X0] && i >= 1 && i < P.cp_d[X0];
    const bool iny0 = P.cp_on[Y0] && j >= 1 && j < P.cp_d[Y0];
    const bool inz0 = P.cp_on[Z0] && k >= 1 && k < P.cp_d[Z0];
    const bool inxn = P.cp_on[XN] && i >= xr - P.cp_d[XN] + 1;
    const bool inyn = P.cp_on[YN] && j >= yr - P.cp_d[YN] + 1;
    const bool inzn = P.cp_on[ZN] && k >= zr - P.cp_d[ZN] + 1;
    const bool zero = (P.cp_on[X0] && i == 0) || (P.cp_on[Y0] && j == 0) || (P.cp_on[Z0] && k == 0);
    int64_t qx0 = 0, qxn = 0, qy0 = 0, qyn = 0, qz0 = 0, qzn = 0;
    if (!zero) {
        if (inx0) { qx0 = ((int64_t)i * yr + j) * zr + k; px0[0] = ldPsiE<T>(P, P.psie[X0][0], qx0); px0[1] = ldPsiE<T>(P, P.psie[X0][1], qx0); }
        if (inxn) { qxn = ((int64_t)(i - (xr - P.cp_d[XN])) * yr + j) * zr + k; pxn[0] = ldPsiE<T>(P, P.psie[XN][0], qxn); pxn[1] = ldPsiE<T>(P, P.psie[XN][1], qxn); }
        if (iny0) { qy0 = ((int64_t)i * P.cp_d[Y0] + j) * zr + k; py0[0] = ldPsiE<T>(P, P.psie[Y0][0], qy0); py0[1] = ldPsiE<T>(P, P.psie[Y0][1], qy0); }
        if (inyn) { qyn = ((int64_t)i * P.cp_d[YN] + (j - (yr - P.cp_d[YN]))) * zr + k; pyn[0] = ldPsiE<T>(P, P.psie[YN][0], qyn); pyn[1] = ldPsiE<T>(P, P.psie[YN][1], qyn); }
        if (inz0) { qz0 = ((int64_t)i * yr + j) * P.cp_d[Z0] + k; pz0[0] = ldPsiE<T>(P, P.psie[Z0][0], qz0); pz0[1] = ldPsiE<T>(P, P.psie[Z0][1], qz0); }
        if (inzn) { qzn = ((int64_t)i * yr + j) * P.cp_d[ZN] + (k - (zr - P.cp_d[ZN])); pzn[0] = ldPsiE<T>(P, P.psie[ZN][0], qzn); pzn[1] = ldPsiE<T>(P, P.psie[ZN][1], qzn); }
    }
    if (ADE && (fl & CF_ADE_BRANCH)) {
        const auto &A = Tab<R>::ade(P, ade_set);
        const bool comp[3] = {(fl & CF_ADE_X) != 0, (fl & CF_ADE_Y) != 0, (fl & CF_ADE_Z) != 0};
        // difference-form state (see DevAde); E^{n-1} is the output set before this write
        R qd[3] = {0, 0, 0}, ep[3] = {0, 0, 0}, pc[3][2], qc[3][2];
        for (int a = 0; a < 3; a++) {
            if (!comp[a]) continue;
            qd[a] = Tab<R>::state(P.q[a])[c]; ep[a] = ldE<T>(P.fout[a], c);
            for (int n = 0; n < NPOLES; n++) { pc[a][n] = Tab<R>::state(P.pc[a][n])[c]; qc[a][n] = Tab<R>::state(P.qc[a][n])[c]; }
        }
        const R curl[3] = {curlx, curly, curlz};
        const bool gd[3] = {gx, gy, gz};
        R ne[3] = {nx, ny, nz};
        for (int a = 0; a < 3; a++) {
            if (!(comp[a] && gd[a])) continue;
            R v = A.c0dx * curl[a] + A.qe * qd[a];
            for (int n = 0; n < NPOLES; n++) v += A.qpe[n] * qc[a][n] + A.pe[n] * pc[a][n];
            v += A.c2 * ep[a] + A.c3 * eo[a];
            ne[a] = v;
        }
        if (!zero) {   // CPML inside the ADE branch, first psi_E update
            if (inx0 && i > 1) {   // x0 corrections are scaled by cb == 0 (yee.c:577)
                const R be = Tab<R>::ld(P.be[X0], i), ce = Tab<R>::ld(P.ce[X0], i);
                px0[0] = be * px0[0] + ce * dhz_i * idx_;
                px0[1] = be * px0[1] + ce * dhy_i * idx_;
            }
            if (iny0 && j > 1) {
                const R be = Tab<R>::ld(P.be[Y0], j), ce = Tab<R>::ld(P.ce[Y0], j);
                py0[0] = be * py0[0] + ce * dhz_j * idx_;
                py0[1] = be * py0[1] + ce * dhx_j * idx_;
                if ((i > 0 && k > 0) && comp[0]) ne[0] += dx * cba[0] * py0[0];
                if ((i > 0 && k > 0) && comp[2]) ne[2] -= dx * cba[2] * py0[1];
            }
            if (inz0 && k > 1) {
                const R be = Tab<R>::ld(P.be[Z0], k), ce = Tab<R>::ld(P.ce[Z0], k);
                pz0[1] = be * pz0[1] + ce * dhx_k * idx_;
                pz0[0] = be * pz0[0] + ce * dhy_k * idx_;
                if ((i > 0 && j > 0) && comp[1]) ne[1] += dx * cba[1] * pz0[1];
                if ((i > 0 && j > 0) && comp[0]) ne[0] -= dx * cba[0] * pz0[0];
            }
            if (inxn) {
                const int ir = i - (xr - P.cp_d[XN]);
                const R be = Tab<R>::ld(P.be[XN], ir), ce = Tab<R>::ld(P.ce[XN], ir);
                pxn[0] = be * pxn[0] + ce * dhz_i * idx_;
                pxn[1] = be * pxn[1] + ce * dhy_i * idx_;
                if ((j > 0 && k > 0) && comp[1]) ne[1] -= dx * cba[1] * pxn[0];
                if ((j > 0 && k > 0) && comp[2]) ne[2] += dx * cba[2] * pxn[1];
            }
            if (inyn) {
                const int jr = j - (yr - P.cp_d[YN]);
                const R be = Tab<R>::ld(P.be[YN], jr), ce = Tab<R>::ld(P.ce[YN], jr);
                pyn[0] = be * pyn[0] + ce * dhz_j * idx_;
                pyn[1] = be * pyn[1] + ce * dhx_j * idx_;
                if ((i > 0 && k > 0) && comp[0]) ne[0] += dx * cba[0] * pyn[0];
                if ((i > 0 && k > 0) && comp[2]) ne[2] -= dx * cba[2] * pyn[1];
            }
            if (inzn) {
                const int kr = k - (zr - P.cp_d[ZN]);
                const R be = Tab<R>::ld(P.be[ZN], kr), ce = Tab<R>::ld(P.ce[ZN], kr);
                pzn[1] = be * pzn[1] + ce * dhx_k * idx_;
                pzn[0] = be * pzn[0] + ce * dhy_k * idx_;
                if ((i > 0 && j > 0) && comp[1]) ne[1] += dx * cba[1] * pzn[1];
                if ((i > 0 && j > 0) && comp[0]) ne[0] -= dx * cba[0] * pzn[0];
            }
        }
        for (int a = 0; a < 3; a++) {   // polarisation recursions of the owned components
            if (!comp[a]) continue;
            const R e1 = ne[a];
            Tab<R>::state(P.q[a])[c] = A.ma0 * qd[a] + A.a2 * (ep[a] + R(2) * eo[a] + e1);
            for (int n = 0; n < NPOLES; n++) {
                const R qn = A.rp[n] * pc[a][n] + A.rq[n] * qc[a][n] + A.bp2[n] * ep[a] + A.bp3[n] * eo[a] + A.bp4[n] * e1;
                Tab<R>::state(P.qc[a][n])[c] = qn;
                Tab<R>::state(P.pc[a][n])[c] = pc[a][n] + qn;
            }
        }
        nx = ne[0]; ny = ne[1]; nz = ne[2];
    }
    if (gx && !(ADE && (fl & CF_ADE_X))) nx = ca[0] * eo[0] + cb[0] * curlx;
    if (gy && !(ADE && (fl & CF_ADE_Y))) ny = ca[1] * eo[1] + cb[1] * curly;
    if (gz && !(ADE && (fl & CF_ADE_Z))) nz = ca[2] * eo[2] + cb[2] * curlz;
    if (fl & CF_PEC_X) nx = 0.f;
    if (fl & CF_PEC_Y) ny = 0.f;
    if (fl & CF_PEC_Z) nz = 0.f;
    if (zero) {
        nx = ny = nz = 0.f;
    } else {
        const bool tx = !(fl & CF_ADE_X), ty = !(fl & CF_ADE_Y), tz = !(fl & CF_ADE_Z);
        if (inx0) {
            const R be = Tab<R>::ld(P.be[X0], i), ce = Tab<R>::ld(P.ce[X0], i);
            px0[0] = be * px0[0] + ce * dhz_i * idx_;
            px0[1] = be * px0[1] + ce * dhy_i * idx_;
            if (j > 0 && k > 0) {
                if (ty) ny -= dx * cb[1] * px0[0];
                if (tz) nz += dx * cb[2] * px0[1];
                stPsiE<T>(P, P.psie[X0][0], qx0, px0[0], stp, 6 + 2 * X0 + 0); stPsiE<T>(P, P.psie[X0][1], qx0, px0[1], stp, 6 + 2 * X0 + 1);
            }
        }
        if (iny0) {
            const R be = Tab<R>::ld(P.be[Y0], j), ce = Tab<R>::ld(P.ce[Y0], j);
            py0[0] = be * py0[0] + ce * dhz_j * idx_;
            py0[1] = be * py0[1] + ce * dhx_j * idx_;
            if (i > 0 && k > 0) {
                if (tx) nx += dx * cb[0] * py0[0];
                if (tz) nz -= dx * cb[2] * py0[1];
                stPsiE<T>(P, P.psie[Y0][0], qy0, py0[0], stp, 6 + 2 * Y0 + 0); stPsiE<T>(P, P.psie[Y0][1], qy0, py0[1], stp, 6 + 2 * Y0 + 1);
            }
        }
        if (inz0) {
            const R be = Tab<R>::ld(P.be[Z0], k), ce = Tab<R>::ld(P.ce[Z0], k);
            pz0[1] = be * pz0[1] + ce * dhx_k * idx_;
            pz0[0] = be * pz0[0] + ce * dhy_k * idx_;
            if (i > 0 && j > 0) {
                if (ty) ny += dx * cb[1] * pz0[1];
                if (tz) nx -= dx * cb[0] * pz0[0];     // gated by ztbc in the reference (boundary.c:758-759)
                stPsiE<T>(P, P.psie[Z0][0], qz0, pz0[0], stp, 6 + 2 * Z0 + 0); stPsiE<T>(P, P.psie[Z0][1], qz0, pz0[1], stp, 6 + 2 * Z0 + 1);
            }
        }
        if (inxn) {
            const int ir = i - (xr - P.cp_d[XN]);
            const R be = Tab<R>::ld(P.be[XN], ir), ce = Tab<R>::ld(P.ce[XN], ir);
            pxn[0] = be * pxn[0] + ce * dhz_i * idx_;
            pxn[1] = be * pxn[1] + ce * dhy_i * idx_;
            if (j > 0 && k > 0) {
                if (ty) ny -= dx * cb[1] * pxn[0];
                if (tz) nz += dx * cb[2] * pxn[1];
                stPsiE<T>(P, P.psie[XN][0], qxn, pxn[0], stp, 6 + 2 * XN + 0); stPsiE<T>(P, P.psie[XN][1], qxn, pxn[1], stp, 6 + 2 * XN + 1);
            }
        }
        if (inyn) {
            const int jr = j - (yr - P.cp_d[YN]);
            const R be = Tab<R>::ld(P.be[YN], jr), ce = Tab<R>::ld(P.ce[YN], jr);
            pyn[0] = be * pyn[0] + ce * dhz_j * idx_;
            pyn[1] = be * pyn[1] + ce * dhx_j * idx_;
            if (i > 0 && k > 0) {
                if (tx) nx += dx * cb[0] * pyn[0];
                if (tz) nz -= dx * cb[2] * pyn[1];
                stPsiE<T>(P, P.psie[YN][0], qyn, pyn[0], stp, 6 + 2 * YN + 0); stPsiE<T>(P, P.psie[YN][1], qyn, pyn[1], stp, 6 + 2 * YN + 1);
            }
        }
        if (inzn) {
            const int kr = k - (zr - P.cp_d[ZN]);
            const R be = Tab<R>::ld(P.be[ZN], kr), ce = Tab<R>::ld(P.ce[ZN], kr);
            pzn[1] = be * pzn[1] + ce * dhx_k * idx_;
            pzn[0] = be * pzn[0] + ce * dhy_k * idx_;
            if (i > 0 && j > 0) {
                if (ty) ny += dx * cb[1] * pzn[1];
                if (tx) nx -= dx * cb[0] * pzn[0];
                stPsiE<T>(P, P.psie[ZN][0], qzn, pzn[0], stp, 6 + 2 * ZN + 0); stPsiE<T>(P, P.psie[ZN][1], qzn, pzn[1], stp, 6 + 2 * ZN + 1);
            }
        }
    }
    if (tsf && P.tsf_on) tsf_add_e(P, i, j, k, nx, ny, nz);
    return V3<R>{nx, ny, nz};
}

}  // namespace
