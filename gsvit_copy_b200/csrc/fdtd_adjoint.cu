// fdtd_adjoint.cu -- discrete adjoint of one source-free FDTD step.
//
// No counterpart in the reference.  The forward step of the general path
// (slab kernels; the bulk kernel computes the same expressions) is linear in
// (E, H, psi_E, psi_H): the H half step (ystep_h yee.c:146-265, CPML H
// boundary.c:347-519, zero planes boundary.c:418-492) and the E half step
// (ystep_e yee.c:530-1247 with the dispersive branch in the difference form of
// DevAde and the CPML inside it, yee.c:914-1108, PEC rule, zero planes and CPML
// E boundary.c:691-884).  The TSF corrections are sources that do
// not depend on the fields.  The adjoint applies the transposed half steps in
// reverse order, each in two gathers over the cells, so that no two threads
// write one value:
//   A: per cell, from the adjoint of its updated field: the adjoint of its old
//      field, of its psi (in place) and of the six field differences the
//      update read (the curl and the psi recursions);
//   B: per cell of the other field, the sum of the difference adjoints of the
//      cells whose differences contain it.
// Gates, coefficients and operation order follow e_special / h_special.
#include <cuda_runtime.h>

#include "fdtd_adjoint.cuh"
#include "fdtd_device.cuh"

namespace {

enum { X0 = 0, XN = 1, Y0 = 2, YN = 3, Z0 = 4, ZN = 5 };

__device__ __forceinline__ void cell_ijk(const DevPlan &P, int64_t c, int &i, int &j, int &k)
{
    k = (int)(c % P.zr);
    const int64_t t = c / P.zr;
    j = (int)(t % P.yr);
    i = (int)(t / P.yr);
}

// ---- E half step: A -- adjoint of E^n, psi_E and the H differences, and,
// in cells of the dispersive branch, of the ADE state (E^{n-1}, Q, p, q)
// dd: 0 dhz_j, 1 dhy_k, 2 dhx_k, 3 dhz_i, 4 dhy_i, 5 dhx_j (backward differences)
//
// Forward, per cell (e_special): the ADE value ne of the dispersive components
// (c0dx curl + qe Q + sum(qpe q + pe p) + c2 E^{n-1} + c3 E^n where the curl
// exists, E^n elsewhere), the CPML inside the branch (a first psi_E update,
// psi1 = be psi0 + ce D/dx, and ne +/-= dx cba psi1), the state recursions
// from ne, the ordinary update of the other components, the PEC rule, then
// (off the zeroed planes) the second psi_E update psi2 = be psi1 + ce D/dx
// with corrections of the non-dispersive components, stored where the two
// other indices are > 0.  Reversed here in the opposite order.
struct FaceT {             // one psi_E array of one face at this cell
    bool in, store, first; // cell in the slab; psi2 stored; first update (dispersive branch)
    int64_t q;             // psi index
    float be, ce;
    int dix;               // the difference it reads (dd index)
    int bnd_c;             // the E component of the boundary correction, its sign, its gate component
    float bnd_s;
    int bnd_t;
    int ade_c;             // the E component of the correction in the branch (-1: none), its sign
    float ade_s;
};

template <bool ADE>
__global__ void adj_e_a(const __grid_constant__ DevPlan P, const DevAdj A, int64_t n)
{
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(P, c, i, j, k);
        const int xr = P.xr, yr = P.yr, zr = P.zr;
        const int cls = cls_at(P, i, j, k);
        const float4 *cl = reinterpret_cast<const float4 *>(P.classes);
        const float4 c0 = cl[cls * 4 + 0], c1 = cl[cls * 4 + 1], c2 = cl[cls * 4 + 2], c3 = cl[cls * 4 + 3];
        const unsigned fl = __float_as_uint(c0.w);
        float ca[3] = {c0.x, c0.y, c0.z}, cb[3] = {c1.x, c1.y, c1.z};
        const float cba[3] = {c3.x, c3.y, c3.z};
        if (fl & CF_DESIGN) {
            const int64_t q = ((int64_t)(i - P.dbox[0]) * (P.dbox[3] - P.dbox[2]) + (j - P.dbox[2])) * (P.dbox[5] - P.dbox[4]) + (k - P.dbox[4]);
            for (int a = 0; a < 3; a++) { ca[a] = P.dcoef[6 * q + a]; cb[a] = P.dcoef[6 * q + 3 + a]; }
        }
        const bool ade = ADE && (fl & CF_ADE_BRANCH);
        const bool comp[3] = {ade && (fl & CF_ADE_X), ade && (fl & CF_ADE_Y), ade && (fl & CF_ADE_Z)};
        const bool gd[3] = {j > 0 && k > 0, i > 0 && k > 0, i > 0 && j > 0};
        float e[3] = {A.eb[0][c], A.eb[1][c], A.eb[2][c]};
        float d[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const float dx = P.dx, idx_ = 1.0f / P.dx;
        const bool zero = (P.cp_on[X0] && i == 0) || (P.cp_on[Y0] && j == 0) || (P.cp_on[Z0] && k == 0);
        // the psi_E arrays this cell touches (faces x0 xn y0 yn z0 zn, two each)
        FaceT F[6][2];
        {
            const bool inx0 = P.cp_on[X0] && i >= 1 && i < P.cp_d[X0];
            const bool iny0 = P.cp_on[Y0] && j >= 1 && j < P.cp_d[Y0];
            const bool inz0 = P.cp_on[Z0] && k >= 1 && k < P.cp_d[Z0];
            const bool inxn = P.cp_on[XN] && i >= xr - P.cp_d[XN] + 1;
            const bool inyn = P.cp_on[YN] && j >= yr - P.cp_d[YN] + 1;
            const bool inzn = P.cp_on[ZN] && k >= zr - P.cp_d[ZN] + 1;
            const bool in[6] = {inx0, inxn, iny0, inyn, inz0, inzn};
            const int pos[6] = {i, i - (xr - P.cp_d[XN]), j, j - (yr - P.cp_d[YN]), k, k - (zr - P.cp_d[ZN])};
            const bool first[6] = {inx0 && i > 1, inxn, iny0 && j > 1, inyn, inz0 && k > 1, inzn};
            for (int f = 0; f < 6; f++) {
                const int ax = f / 2;
                int64_t q = 0;
                if (in[f]) {
                    if (f == X0) q = ((int64_t)i * yr + j) * zr + k;
                    else if (f == XN) q = ((int64_t)pos[f] * yr + j) * zr + k;
                    else if (f == Y0) q = ((int64_t)i * P.cp_d[Y0] + j) * zr + k;
                    else if (f == YN) q = ((int64_t)i * P.cp_d[YN] + pos[f]) * zr + k;
                    else if (f == Z0) q = ((int64_t)i * yr + j) * P.cp_d[Z0] + k;
                    else q = ((int64_t)i * yr + j) * P.cp_d[ZN] + pos[f];
                }
                const float be = in[f] ? P.be[f][pos[f]] : 0.f, ce = in[f] ? P.ce[f][pos[f]] : 0.f;
                for (int r = 0; r < 2; r++) {
                    FaceT &t = F[f][r];
                    t.in = in[f] && !zero;
                    t.store = t.in && gd[ax];
                    t.first = t.in && ade && first[f];
                    t.q = q;
                    t.be = be;
                    t.ce = ce;
                    t.ade_c = -1;
                    t.ade_s = 0.f;
                }
                if (ax == 0) {        // psi[0] <- dhz_i: ny -= dx cb1 psi; psi[1] <- dhy_i: nz += dx cb2 psi
                    F[f][0].dix = 3; F[f][0].bnd_c = 1; F[f][0].bnd_s = -1.f; F[f][0].bnd_t = 1;
                    F[f][1].dix = 4; F[f][1].bnd_c = 2; F[f][1].bnd_s = +1.f; F[f][1].bnd_t = 2;
                    if (f == XN) {    // x0 corrections in the branch are scaled by cb == 0 (yee.c:577)
                        F[f][0].ade_c = 1; F[f][0].ade_s = -1.f;
                        F[f][1].ade_c = 2; F[f][1].ade_s = +1.f;
                    }
                } else if (ax == 1) { // psi[0] <- dhz_j: nx += dx cb0 psi; psi[1] <- dhx_j: nz -= dx cb2 psi
                    F[f][0].dix = 0; F[f][0].bnd_c = 0; F[f][0].bnd_s = +1.f; F[f][0].bnd_t = 0;
                    F[f][1].dix = 5; F[f][1].bnd_c = 2; F[f][1].bnd_s = -1.f; F[f][1].bnd_t = 2;
                    F[f][0].ade_c = 0; F[f][0].ade_s = +1.f;
                    F[f][1].ade_c = 2; F[f][1].ade_s = -1.f;
                } else {              // psi[1] <- dhx_k: ny += dx cb1 psi; psi[0] <- dhy_k: nx -= dx cb0 psi
                    F[f][1].dix = 2; F[f][1].bnd_c = 1; F[f][1].bnd_s = +1.f; F[f][1].bnd_t = 1;
                    F[f][0].dix = 1; F[f][0].bnd_c = 0; F[f][0].bnd_s = -1.f;
                    F[f][0].bnd_t = f == Z0 ? 2 : 0;   // the z0 ex correction is gated by ztbc (boundary.c:758-759)
                    F[f][1].ade_c = 1; F[f][1].ade_s = +1.f;
                    F[f][0].ade_c = 0; F[f][0].ade_s = -1.f;
                }
            }
        }
        // second psi_E update and the boundary corrections, reversed
        float lp[6][2], ident[6][2];
        for (int f = 0; f < 6; f++)
            for (int r = 0; r < 2; r++) {
                const FaceT &t = F[f][r];
                lp[f][r] = 0.f;
                ident[f][r] = 0.f;
                if (!t.in) continue;
                const float lam = A.pe[f][r][t.q];
                if (t.store) {
                    const float l2 = lam + (comp[t.bnd_t] ? 0.f : t.bnd_s * dx * cb[t.bnd_c] * e[t.bnd_c]);
                    lp[f][r] = t.be * l2;
                    d[t.dix] += t.ce * idx_ * l2;
                } else {
                    ident[f][r] = lam;   // psi stored unchanged
                }
            }
        if (zero) {
            e[0] = e[1] = e[2] = 0.f;
        } else {
            if (fl & CF_PEC_X) e[0] = 0.f;
            if (fl & CF_PEC_Y) e[1] = 0.f;
            if (fl & CF_PEC_Z) e[2] = 0.f;
        }
        // adjoint of the ADE value of the dispersive components: u = its own
        // adjoint plus what the state recursions read from it
        float u[3] = {0.f, 0.f, 0.f};
        if (ADE && ade) {
            const DevAde &Ad = P.ade[__float_as_int(c2.z)];
            for (int a = 0; a < 3; a++) {
                if (!comp[a]) continue;
                float v = e[a] + Ad.a2 * A.q[a][c];
                for (int m = 0; m < 2; m++)
                    if (A.pc[a][m]) v += Ad.bp4[m] * (A.qc[a][m][c] + A.pc[a][m][c]);
                u[a] = v;
            }
            // the corrections of the CPML inside the branch
            for (int f = 0; f < 6; f++)
                for (int r = 0; r < 2; r++) {
                    const FaceT &t = F[f][r];
                    if (t.first && t.ade_c >= 0 && comp[t.ade_c] && gd[f / 2])
                        lp[f][r] += t.ade_s * dx * cba[t.ade_c] * u[t.ade_c];
                }
        }
        // first psi_E update (dispersive branch) and the psi adjoints
        for (int f = 0; f < 6; f++)
            for (int r = 0; r < 2; r++) {
                const FaceT &t = F[f][r];
                if (!t.in) continue;
                float l0 = ident[f][r];
                if (t.first) {
                    l0 += t.be * lp[f][r];
                    d[t.dix] += t.ce * idx_ * lp[f][r];
                } else {
                    l0 += lp[f][r];
                }
                A.pe[f][r][t.q] = l0;
            }
        const float ikx = P.ike[0][i], iky = P.ike[1][j], ikz = P.ike[2][k];
        // curl x = dhz_j iky - dhy_k ikz, curl y = dhx_k ikz - dhz_i ikx, curl z = dhy_i ikx - dhx_j iky
        float w[3] = {0.f, 0.f, 0.f};
        if (!zero) {
            for (int a = 0; a < 3; a++) {
                if (!gd[a] || comp[a]) continue;   // ordinary update
                w[a] = cb[a] * e[a];
                e[a] = ca[a] * e[a];
            }
        }
        if (ADE && ade) {
            const DevAde &Ad = P.ade[__float_as_int(c2.z)];
            for (int a = 0; a < 3; a++) {
                if (!comp[a]) continue;
                const float ua = u[a], lq1 = A.q[a][c];
                float lqt[2] = {0.f, 0.f}, lp1[2] = {0.f, 0.f};
                for (int m = 0; m < 2; m++)
                    if (A.pc[a][m]) { lp1[m] = A.pc[a][m][c]; lqt[m] = A.qc[a][m][c] + lp1[m]; }
                const float lv = gd[a] ? ua : 0.f;
                float le0 = (gd[a] ? Ad.c3 * ua : ua) + 2.f * Ad.a2 * lq1 + A.ep[a][c];
                float lep = Ad.c2 * lv + Ad.a2 * lq1;
                for (int m = 0; m < 2; m++) {
                    le0 += Ad.bp3[m] * lqt[m];
                    lep += Ad.bp2[m] * lqt[m];
                }
                w[a] = Ad.c0dx * lv;
                e[a] = le0;
                A.ep[a][c] = lep;
                A.q[a][c] = Ad.qe * lv + Ad.ma0 * lq1;
                for (int m = 0; m < 2; m++)
                    if (A.pc[a][m]) {
                        A.qc[a][m][c] = Ad.qpe[m] * lv + Ad.rq[m] * lqt[m];
                        A.pc[a][m][c] = Ad.pe[m] * lv + Ad.rp[m] * lqt[m] + lp1[m];
                    }
            }
        }
        d[0] += w[0] * iky;
        d[1] -= w[0] * ikz;
        d[2] += w[1] * ikz;
        d[3] -= w[1] * ikx;
        d[4] += w[2] * ikx;
        d[5] -= w[2] * iky;
        for (int a = 0; a < 3; a++) A.eb[a][c] = e[a];
        for (int q = 0; q < 6; q++) A.dd[q][c] = d[q];
    }
}

// ---- E half step: B -- H adjoints from the backward-difference adjoints
__global__ void adj_e_b(const __grid_constant__ DevPlan P, const DevAdj A, int64_t n)
{
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(P, c, i, j, k);
        const bool ko = k + 1 < P.zr, jo = j + 1 < P.yr, io = i + 1 < P.xr;
        const int64_t sj = P.sj, si = P.si;
        float hx = A.dd[2][c] + A.dd[5][c], hy = A.dd[1][c] + A.dd[4][c], hz = A.dd[0][c] + A.dd[3][c];
        if (ko) { hx -= A.dd[2][c + 1]; hy -= A.dd[1][c + 1]; }
        if (jo) { hx -= A.dd[5][c + sj]; hz -= A.dd[0][c + sj]; }
        if (io) { hy -= A.dd[4][c + si]; hz -= A.dd[3][c + si]; }
        A.hb[0][c] += hx;
        A.hb[1][c] += hy;
        A.hb[2][c] += hz;
    }
}

// ---- H half step: A -- adjoint of H^{n-1/2}, psi_H and the E differences
// dd: 0 dey_k, 1 dez_j, 2 dez_i, 3 dex_k, 4 dex_j, 5 dey_i (forward differences)
__global__ void adj_h_a(const __grid_constant__ DevPlan P, const DevAdj A, int64_t n)
{
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(P, c, i, j, k);
        const int xr = P.xr, yr = P.yr, zr = P.zr;
        const float4 hc = reinterpret_cast<const float4 *>(P.classes)[cls_at(P, i, j, k) * 4 + 2];
        const float da = hc.x, db = hc.y, dbdx = db * P.dx, idx_ = 1.0f / P.dx;
        const bool il = (i == xr - 1), jl = (j == yr - 1), kl = (k == zr - 1);
        const bool iin = (i >= 1 && i < xr - 1), jin = (j >= 1 && j < yr - 1), kin = (k >= 1 && k < zr - 1);
        float h[3] = {A.hb[0][c], A.hb[1][c], A.hb[2][c]};
        float d[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const bool zero = (P.cp_on[XN] && il && jin && kin) || (P.cp_on[YN] && jl && iin && kin) || (P.cp_on[ZN] && kl && iin && jin);
        if (zero) {
            h[0] = h[1] = h[2] = 0.f;
        } else {
            // x faces: psi[1] <- dey_i (hz -= dbdx psi[1]), psi[0] <- dez_i (hy += dbdx psi[0])
            auto xface = [&](int f, int pos, int64_t q) {
                const float bh = P.bh[f][pos], ch = P.ch[f][pos];
                const float t1 = A.ph[f][1][q] - dbdx * h[2], t0 = A.ph[f][0][q] + dbdx * h[1];
                A.ph[f][1][q] = bh * t1;
                A.ph[f][0][q] = bh * t0;
                d[5] += ch * idx_ * t1;
                d[2] += ch * idx_ * t0;
            };
            // y faces: psi[0] <- dez_j (hx -= dbdx psi[0]), psi[1] <- dex_j (hz += dbdx psi[1])
            auto yface = [&](int f, int pos, int64_t q) {
                const float bh = P.bh[f][pos], ch = P.ch[f][pos];
                const float t0 = A.ph[f][0][q] - dbdx * h[0], t1 = A.ph[f][1][q] + dbdx * h[2];
                A.ph[f][0][q] = bh * t0;
                A.ph[f][1][q] = bh * t1;
                d[1] += ch * idx_ * t0;
                d[4] += ch * idx_ * t1;
            };
            // z faces: psi[1] <- dex_k (hy -= dbdx psi[1]), psi[0] <- dey_k (hx += dbdx psi[0])
            auto zface = [&](int f, int pos, int64_t q) {
                const float bh = P.bh[f][pos], ch = P.ch[f][pos];
                const float t1 = A.ph[f][1][q] - dbdx * h[1], t0 = A.ph[f][0][q] + dbdx * h[0];
                A.ph[f][1][q] = bh * t1;
                A.ph[f][0][q] = bh * t0;
                d[3] += ch * idx_ * t1;
                d[0] += ch * idx_ * t0;
            };
            if (P.cp_on[X0] && i < P.cp_d[X0] - 1 && jin && kin) xface(X0, i, ((int64_t)i * yr + j) * zr + k);
            if (P.cp_on[Y0] && j < P.cp_d[Y0] - 1 && iin && kin) yface(Y0, j, ((int64_t)i * P.cp_d[Y0] + j) * zr + k);
            if (P.cp_on[Z0] && k < P.cp_d[Z0] - 1 && iin && jin) zface(Z0, k, ((int64_t)i * yr + j) * P.cp_d[Z0] + k);
            if (P.cp_on[XN] && i >= xr - P.cp_d[XN] + 1 && i < xr - 1 && jin && kin) {
                const int ir = i - (xr - P.cp_d[XN]);
                xface(XN, ir, ((int64_t)ir * yr + j) * zr + k);
            }
            if (P.cp_on[YN] && j >= yr - P.cp_d[YN] + 1 && j < yr - 1 && iin && kin) {
                const int jr = j - (yr - P.cp_d[YN]);
                yface(YN, jr, ((int64_t)i * P.cp_d[YN] + jr) * zr + k);
            }
            if (P.cp_on[ZN] && k >= zr - P.cp_d[ZN] + 1 && k < zr - 1 && iin && jin) {
                const int kr = k - (zr - P.cp_d[ZN]);
                zface(ZN, kr, ((int64_t)i * yr + j) * P.cp_d[ZN] + kr);
            }
            const float ikx = P.ikh[0][i], iky = P.ikh[1][j], ikz = P.ikh[2][k];
            if (!(jl || kl)) {   // hx += db (dey_k ikz - dez_j iky)
                const float t = db * h[0];
                d[0] += t * ikz;
                d[1] -= t * iky;
                h[0] = da * h[0];
            }
            if (!(il || kl)) {   // hy += db (dez_i ikx - dex_k ikz)
                const float t = db * h[1];
                d[2] += t * ikx;
                d[3] -= t * ikz;
                h[1] = da * h[1];
            }
            if (!(il || jl)) {   // hz += db (dex_j iky - dey_i ikx)
                const float t = db * h[2];
                d[4] += t * iky;
                d[5] -= t * ikx;
                h[2] = da * h[2];
            }
        }
        for (int a = 0; a < 3; a++) A.hb[a][c] = h[a];
        for (int q = 0; q < 6; q++) A.dd[q][c] = d[q];
    }
}

// ---- H half step: B -- E adjoints from the forward-difference adjoints
__global__ void adj_h_b(const __grid_constant__ DevPlan P, const DevAdj A, int64_t n)
{
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(P, c, i, j, k);
        const int64_t sj = P.sj, si = P.si;
        float ex = -(A.dd[3][c] + A.dd[4][c]), ey = -(A.dd[0][c] + A.dd[5][c]), ez = -(A.dd[1][c] + A.dd[2][c]);
        if (k > 0) { ex += A.dd[3][c - 1]; ey += A.dd[0][c - 1]; }
        if (j > 0) { ex += A.dd[4][c - sj]; ez += A.dd[1][c - sj]; }
        if (i > 0) { ey += A.dd[5][c - si]; ez += A.dd[2][c - si]; }
        A.eb[0][c] += ex;
        A.eb[1][c] += ey;
        A.eb[2][c] += ez;
    }
}

// dJ/dE of the step `step` (the E set that step wrote) on the NFFF surface
__global__ void adj_source(const DevObjective O, const DevAdj A, int step)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= O.ns) return;
    double sn, cs;
    sincos(O.omega_dt * (double)step, &sn, &cs);
    const int64_t c = O.cell[s], st = O.nstride[s];
    for (int a = 0; a < 3; a++) {
        const double2 ae = O.ae[(size_t)a * O.ns + s], ad = O.ad[(size_t)a * O.ns + s];
        const double ve = 2.0 * (cs * ae.x + sn * ae.y), vd = 2.0 * (cs * ad.x + sn * ad.y) * O.inv2dx;
        atomicAdd(A.eb[a] + c, (float)ve);
        atomicAdd(A.eb[a] + c + st, (float)vd);
        atomicAdd(A.eb[a] + c - st, (float)(-vd));
    }
}

// curl H^{n+1/2} of the design box cells (the E update's curl; P.fout holds H^{n+1/2})
__global__ void design_curl(const __grid_constant__ DevPlan P, const DevGrad G, int slot)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= G.ncell) return;
    const int nj = G.box[3] - G.box[2], nk = G.box[5] - G.box[4];
    const int k = G.box[4] + (int)(q % nk), j = G.box[2] + (int)((q / nk) % nj), i = G.box[0] + (int)(q / ((int64_t)nk * nj));
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const float *HX = P.fout[3], *HY = P.fout[4], *HZ = P.fout[5];
    const float hx = HX[c], hy = HY[c], hz = HZ[c];
    const float ikx = P.ike[0][i], iky = P.ike[1][j], ikz = P.ike[2][k];
    const float dhz_i = hz - HZ[c - P.si], dhy_i = hy - HY[c - P.si];
    const float dhz_j = hz - HZ[c - P.sj], dhx_j = hx - HX[c - P.sj];
    const float dhx_k = hx - HX[c - 1], dhy_k = hy - HY[c - 1];
    float *out = G.curl + (size_t)slot * 3 * G.ncell + 3 * q;
    out[0] = dhz_j * iky - dhy_k * ikz;
    out[1] = dhx_k * ikz - dhz_i * ikx;
    out[2] = dhy_i * ikx - dhx_j * iky;
}

// dJ/dcb of the design box: the adjoint of E^{n+1} times the curl it was formed with
__global__ void design_accumulate(const DevAdj A, const DevPlan P, const DevGrad G, int slot)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= G.ncell) return;
    const int nj = G.box[3] - G.box[2], nk = G.box[5] - G.box[4];
    const int k = G.box[4] + (int)(q % nk), j = G.box[2] + (int)((q / nk) % nj), i = G.box[0] + (int)(q / ((int64_t)nk * nj));
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const float *cu = G.curl + (size_t)slot * 3 * G.ncell + 3 * q;
    for (int a = 0; a < 3; a++) G.g[3 * q + a] += (double)A.eb[a][c] * (double)cu[a];
}

// A_E(s,c) = sum_p w_p conj(F_pc) alpha_p tw(R_ps) K_ps, A_D likewise with
// L_ps: the far-field map of farfield_partial_kernel and farfield_reduce_kernel
// (alpha_p = dx^2 exp(i w istart_p dt)), transposed for one frequency
__global__ void objective_weights(const DevFarfield F, int freq, int npoints, const int32_t *points, const double *weights,
                                  const double2 *spec, double2 *ae, double2 *ad)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= F.ns) return;
    const double C0 = 299792458.0, PI = 3.14159265358979323846;
    const double dt = F.dt, dx = F.dx, c0dt = C0 * dt, om = F.omega[freq];
    double sw, cw, s2, c2;
    sincos(om * dt, &sw, &cw);
    sincos(2.0 * om * dt, &s2, &c2);
    const int gx = F.cell_ijk[3 * s], gy = F.cell_ijk[3 * s + 1], gz = F.cell_ijk[3 * s + 2], face = F.face[s];
    double AE[3][2] = {{0, 0}, {0, 0}, {0, 0}}, AD[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    for (int t = 0; t < npoints; t++) {
        const int p = points[t];
        const double rx = F.points[3 * p] - gx, ry = F.points[3 * p + 1] - gy, rz = F.points[3 * p + 2] - gz;
        const double rc = sqrt(rx * rx + ry * ry + rz * rz);
        double dot;
        switch (face) {
        case 0: dot = -rx; break;
        case 1: dot = rx; break;
        case 2: dot = -ry; break;
        case 3: dot = ry; break;
        case 4: dot = -rz; break;
        default: dot = rz; break;
        }
        const double ct = dot / rc, r = rc * dx;
        const int R = min((int)(1.0 + r / c0dt), F.ntw - 1);
        const double ir = 1.0 / r, a = ir / (4.0 * PI), b = -ct / (4.0 * PI) * ir * ir, cp = -ct / (4.0 * PI * C0) * ir / (2.0 * dt);
        const double sg = (face & 1) ? 1.0 : -1.0;
        const double Kr = -cp + b * cw + cp * c2, Ki = b * sw + cp * s2, Lr = sg * a * cw, Li = sg * a * sw;
        const double2 w = F.tw[(size_t)freq * F.ntw + R];
        const double wKr = w.x * Kr - w.y * Ki, wKi = w.x * Ki + w.y * Kr, wLr = w.x * Lr - w.y * Li, wLi = w.x * Li + w.y * Lr;
        double sa, ca;
        sincos(om * (double)F.istart[p] * dt, &sa, &ca);
        const double ar = dx * dx * ca, ai = dx * dx * sa;   // alpha_p
        for (int c = 0; c < 3; c++) {
            const double2 f = spec[((size_t)p * F.nfreq + freq) * 3 + c];
            const double gr = weights[t] * f.x, gi = -weights[t] * f.y;   // w_p conj(F)
            const double fr = gr * ar - gi * ai, fi = gr * ai + gi * ar;  // times alpha_p
            AE[c][0] += fr * wKr - fi * wKi;
            AE[c][1] += fr * wKi + fi * wKr;
            AD[c][0] += fr * wLr - fi * wLi;
            AD[c][1] += fr * wLi + fi * wLr;
        }
    }
    for (int c = 0; c < 3; c++) {
        ae[(size_t)c * F.ns + s] = make_double2(AE[c][0], AE[c][1]);
        ad[(size_t)c * F.ns + s] = make_double2(AD[c][0], AD[c][1]);
    }
}

int grid_for(int64_t n)
{
    const int64_t b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

}  // namespace

void launch_adjoint_e(const DevPlan &p, const DevAdj &a, cudaStream_t st)
{
    const int64_t n = (int64_t)p.xr * p.yr * p.zr;
    if (p.nade > 0) adj_e_a<true><<<grid_for(n), 256, 0, st>>>(p, a, n);
    else adj_e_a<false><<<grid_for(n), 256, 0, st>>>(p, a, n);
    adj_e_b<<<grid_for(n), 256, 0, st>>>(p, a, n);
}

void launch_adjoint_h(const DevPlan &p, const DevAdj &a, cudaStream_t st)
{
    const int64_t n = (int64_t)p.xr * p.yr * p.zr;
    adj_h_a<<<grid_for(n), 256, 0, st>>>(p, a, n);
    adj_h_b<<<grid_for(n), 256, 0, st>>>(p, a, n);
}

void launch_adjoint_source(const DevObjective &o, const DevAdj &a, int step, cudaStream_t st)
{
    if (o.ns > 0) adj_source<<<(o.ns + 255) / 256, 256, 0, st>>>(o, a, step);
}

void launch_design_curl(const DevPlan &p, const DevGrad &g, int slot, cudaStream_t st)
{
    if (g.ncell > 0) design_curl<<<(unsigned)((g.ncell + 255) / 256), 256, 0, st>>>(p, g, slot);
}

void launch_design_accumulate(const DevAdj &a, const DevPlan &p, const DevGrad &g, int slot, cudaStream_t st)
{
    if (g.ncell > 0) design_accumulate<<<(unsigned)((g.ncell + 255) / 256), 256, 0, st>>>(a, p, g, slot);
}

void launch_objective_weights(const DevFarfield &f, int freq, int npoints, const int32_t *points, const double *weights,
                              const double2 *spectrum, double2 *ae, double2 *ad, cudaStream_t st)
{
    if (f.ns > 0) objective_weights<<<(f.ns + 127) / 128, 128, 0, st>>>(f, freq, npoints, points, weights, spectrum, ae, ad);
}
