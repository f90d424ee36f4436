// fdtd_adjoint.cu -- discrete adjoint of one source-free FDTD step.
//
// No counterpart in the reference.  The forward step of the general path
// (slab kernels; the bulk kernel computes the same expressions) is linear in
// (E, H, psi_E, psi_H): the H half step (ystep_h yee.c:146-265, CPML H
// boundary.c:347-519, zero planes boundary.c:418-492) and the E half step
// (ystep_e yee.c:530-1247 without the dispersive branch, PEC rule, zero planes
// and CPML E boundary.c:691-884).  The TSF corrections are sources that do
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

// ---- E half step: A -- adjoint of E^n, psi_E and the H differences
// dd: 0 dhz_j, 1 dhy_k, 2 dhx_k, 3 dhz_i, 4 dhy_i, 5 dhx_j (backward differences)
__global__ void adj_e_a(const __grid_constant__ DevPlan P, const DevAdj A, int64_t n)
{
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(P, c, i, j, k);
        const int xr = P.xr, yr = P.yr, zr = P.zr;
        const int cls = cls_at(P, i, j, k);
        const float4 *cl = reinterpret_cast<const float4 *>(P.classes);
        const float4 c0 = cl[cls * 4 + 0], c1 = cl[cls * 4 + 1];
        const unsigned fl = __float_as_uint(c0.w);
        float ca[3] = {c0.x, c0.y, c0.z}, cb[3] = {c1.x, c1.y, c1.z};
        if (fl & CF_DESIGN) {
            const int64_t q = ((int64_t)(i - P.dbox[0]) * (P.dbox[3] - P.dbox[2]) + (j - P.dbox[2])) * (P.dbox[5] - P.dbox[4]) + (k - P.dbox[4]);
            for (int a = 0; a < 3; a++) { ca[a] = P.dcoef[6 * q + a]; cb[a] = P.dcoef[6 * q + 3 + a]; }
        }
        float e[3] = {A.eb[0][c], A.eb[1][c], A.eb[2][c]};
        float d[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const bool zero = (P.cp_on[X0] && i == 0) || (P.cp_on[Y0] && j == 0) || (P.cp_on[Z0] && k == 0);
        if (zero) {
            e[0] = e[1] = e[2] = 0.f;
        } else {
            const float dx = P.dx, idx_ = 1.0f / P.dx;
            const bool inx0 = P.cp_on[X0] && i >= 1 && i < P.cp_d[X0];
            const bool iny0 = P.cp_on[Y0] && j >= 1 && j < P.cp_d[Y0];
            const bool inz0 = P.cp_on[Z0] && k >= 1 && k < P.cp_d[Z0];
            const bool inxn = P.cp_on[XN] && i >= xr - P.cp_d[XN] + 1;
            const bool inyn = P.cp_on[YN] && j >= yr - P.cp_d[YN] + 1;
            const bool inzn = P.cp_on[ZN] && k >= zr - P.cp_d[ZN] + 1;
            // x faces: psi[0] <- dhz_i, psi[1] <- dhy_i; ny -= dx cb1 psi[0], nz += dx cb2 psi[1]
            auto xface = [&](int f, int pos, int64_t q) {
                const float be = P.be[f][pos], ce = P.ce[f][pos];
                const float t0 = A.pe[f][0][q] - dx * cb[1] * e[1], t1 = A.pe[f][1][q] + dx * cb[2] * e[2];
                A.pe[f][0][q] = be * t0;
                A.pe[f][1][q] = be * t1;
                d[3] += ce * idx_ * t0;
                d[4] += ce * idx_ * t1;
            };
            // y faces: psi[0] <- dhz_j, psi[1] <- dhx_j; nx += dx cb0 psi[0], nz -= dx cb2 psi[1]
            auto yface = [&](int f, int pos, int64_t q) {
                const float be = P.be[f][pos], ce = P.ce[f][pos];
                const float t0 = A.pe[f][0][q] + dx * cb[0] * e[0], t1 = A.pe[f][1][q] - dx * cb[2] * e[2];
                A.pe[f][0][q] = be * t0;
                A.pe[f][1][q] = be * t1;
                d[0] += ce * idx_ * t0;
                d[5] += ce * idx_ * t1;
            };
            // z faces: psi[1] <- dhx_k, psi[0] <- dhy_k; ny += dx cb1 psi[1], nx -= dx cb0 psi[0]
            auto zface = [&](int f, int pos, int64_t q) {
                const float be = P.be[f][pos], ce = P.ce[f][pos];
                const float t1 = A.pe[f][1][q] + dx * cb[1] * e[1], t0 = A.pe[f][0][q] - dx * cb[0] * e[0];
                A.pe[f][1][q] = be * t1;
                A.pe[f][0][q] = be * t0;
                d[2] += ce * idx_ * t1;
                d[1] += ce * idx_ * t0;
            };
            if (inx0 && j > 0 && k > 0) xface(X0, i, ((int64_t)i * yr + j) * zr + k);
            if (iny0 && i > 0 && k > 0) yface(Y0, j, ((int64_t)i * P.cp_d[Y0] + j) * zr + k);
            if (inz0 && i > 0 && j > 0) zface(Z0, k, ((int64_t)i * yr + j) * P.cp_d[Z0] + k);
            if (inxn && j > 0 && k > 0) {
                const int ir = i - (xr - P.cp_d[XN]);
                xface(XN, ir, ((int64_t)ir * yr + j) * zr + k);
            }
            if (inyn && i > 0 && k > 0) {
                const int jr = j - (yr - P.cp_d[YN]);
                yface(YN, jr, ((int64_t)i * P.cp_d[YN] + jr) * zr + k);
            }
            if (inzn && i > 0 && j > 0) {
                const int kr = k - (zr - P.cp_d[ZN]);
                zface(ZN, kr, ((int64_t)i * yr + j) * P.cp_d[ZN] + kr);
            }
            if (fl & CF_PEC_X) e[0] = 0.f;
            if (fl & CF_PEC_Y) e[1] = 0.f;
            if (fl & CF_PEC_Z) e[2] = 0.f;
            const float ikx = P.ike[0][i], iky = P.ike[1][j], ikz = P.ike[2][k];
            if (j > 0 && k > 0) {   // curlx = dhz_j iky - dhy_k ikz
                const float t = cb[0] * e[0];
                d[0] += t * iky;
                d[1] -= t * ikz;
                e[0] = ca[0] * e[0];
            }
            if (i > 0 && k > 0) {   // curly = dhx_k ikz - dhz_i ikx
                const float t = cb[1] * e[1];
                d[2] += t * ikz;
                d[3] -= t * ikx;
                e[1] = ca[1] * e[1];
            }
            if (i > 0 && j > 0) {   // curlz = dhy_i ikx - dhx_j iky
                const float t = cb[2] * e[2];
                d[4] += t * ikx;
                d[5] -= t * iky;
                e[2] = ca[2] * e[2];
            }
        }
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
    adj_e_a<<<grid_for(n), 256, 0, st>>>(p, a, n);
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
