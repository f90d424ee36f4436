// fdtd_kernels.cu -- sm_100a kernels of one GSvit FDTD time step.
//
// One step = aux_step (1D TSF grid, 1 CTA) -> bulk kernel (fdtd_bulk.cu,
// fused H+E over the slab-free box) -> slab H -> slab E (the CPML slabs and
// grid edges left outside the bulk box) -> nfff_accumulate (running DFT).
//
// The slab kernels walk a list of boxes (SlabBox) with a flat block index.
// slab_h_kernel updates one cell per thread: ystep_h (yee.c:146-265), then
// h_special -- the CPML psi_H update and corrections (boundary.c:347-519),
// the TSF H corrections (source.c:1464-1672) and the zeroed outer planes.
// slab_h4_kernel is the same update on four consecutive k cells per thread
// with 16-byte loads, used when every box is 4-aligned in k.  slab_e_kernel
// updates one cell per thread: ystep_e with the ADE branch, its embedded CPML,
// the ordinary update and the PEC rule (yee.c:530-1247), then e_special --
// the CPML psi_E update and corrections (boundary.c:691-884) and the TSF E
// corrections (source.c:547-771).  E runs over the runs of k planes that hold a
// dispersive cell with the plan's variant and over the rest with the plain
// variant (SlabLists).  Each half step reads one field set and
// writes the other, so blocks never race on a shared cell.  The *_batch
// forms take a per-box plan index and serve many plans in one launch.
#include <cuda_runtime.h>

#include "../../include/gsvit_b200.h"
#include "fdtd_device.cuh"
#include "fdtd_kernels.cuh"

namespace {

enum { X0 = 0, XN = 1, Y0 = 2, YN = 3, Z0 = 4, ZN = 5 };

// ------------------------------------------------------------ cell updates


#define FULLMASK 0xffffffffu

// CPML psi_H update and corrections (boundary.c:347-519, face order x0 y0 z0
// xn yn zn), TSF H corrections (source.c:1476-1672) and the outer H planes
// zeroed by boundary_hstep (boundary.c:418-420, 455-457, 490-492), applied to
// H after ystep_h.  `owner` cells write their psi_H.
template <class T>
__device__ __forceinline__ float3 h_special(const DevPlan &P, int i, int j, int k, bool owner, bool tsf, float db, float dey_i,
                                         float dez_i, float dex_j, float dez_j, float dex_k, float dey_k, float3 hin)
{
    const uint32_t stp = sr_step<T>(P);
    float hx = hin.x, hy = hin.y, hz = hin.z;
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    const bool il = (i == xr - 1), jl = (j == yr - 1), kl = (k == zr - 1);
    if (tsf && P.tsf_on) tsf_add_h(P, i, j, k, hx, hy, hz);
    const bool jin = (j >= 1 && j < yr - 1), kin = (k >= 1 && k < zr - 1), iin = (i >= 1 && i < xr - 1);
    const float dbdx = db * P.dx;
    const float idx_ = 1.0f / P.dx;
    if (P.cp_on[X0] && i < P.cp_d[X0] - 1 && jin && kin) {
        const int64_t q = ((int64_t)i * yr + j) * zr + k;
        const float bh = __ldg(P.bh[X0] + i), ch = __ldg(P.ch[X0] + i);
        float pzx = bh * ldgPsi<T>(P, P.psih_in[X0][1], q) + ch * dey_i * idx_;
        float pyx = bh * ldgPsi<T>(P, P.psih_in[X0][0], q) + ch * dez_i * idx_;
        hy += dbdx * pyx;
        hz -= dbdx * pzx;
        if (owner) { stPsi<T>(P, P.psih_out[X0][1], q, pzx, stp, 18 + 2 * X0 + 1); stPsi<T>(P, P.psih_out[X0][0], q, pyx, stp, 18 + 2 * X0 + 0); }
    }
    if (P.cp_on[Y0] && j < P.cp_d[Y0] - 1 && iin && kin) {
        const int64_t q = ((int64_t)i * P.cp_d[Y0] + j) * zr + k;
        const float bh = __ldg(P.bh[Y0] + j), ch = __ldg(P.ch[Y0] + j);
        float pxy = bh * ldgPsi<T>(P, P.psih_in[Y0][0], q) + ch * dez_j * idx_;
        float pzy = bh * ldgPsi<T>(P, P.psih_in[Y0][1], q) + ch * dex_j * idx_;
        hx -= dbdx * pxy;
        hz += dbdx * pzy;
        if (owner) { stPsi<T>(P, P.psih_out[Y0][0], q, pxy, stp, 18 + 2 * Y0 + 0); stPsi<T>(P, P.psih_out[Y0][1], q, pzy, stp, 18 + 2 * Y0 + 1); }
    }
    if (P.cp_on[Z0] && k < P.cp_d[Z0] - 1 && iin && jin) {
        const int64_t q = ((int64_t)i * yr + j) * P.cp_d[Z0] + k;
        const float bh = __ldg(P.bh[Z0] + k), ch = __ldg(P.ch[Z0] + k);
        float pyz = bh * ldgPsi<T>(P, P.psih_in[Z0][1], q) + ch * dex_k * idx_;
        float pxz = bh * ldgPsi<T>(P, P.psih_in[Z0][0], q) + ch * dey_k * idx_;
        hy -= dbdx * pyz;
        hx += dbdx * pxz;
        if (owner) { stPsi<T>(P, P.psih_out[Z0][1], q, pyz, stp, 18 + 2 * Z0 + 1); stPsi<T>(P, P.psih_out[Z0][0], q, pxz, stp, 18 + 2 * Z0 + 0); }
    }
    if (P.cp_on[XN]) {
        const int d = P.cp_d[XN];
        if (i >= xr - d + 1 && i < xr - 1 && jin && kin) {
            const int ir = i - (xr - d);
            const int64_t q = ((int64_t)ir * yr + j) * zr + k;
            const float bh = __ldg(P.bh[XN] + ir), ch = __ldg(P.ch[XN] + ir);
            float pzx = bh * ldgPsi<T>(P, P.psih_in[XN][1], q) + ch * dey_i * idx_;
            float pyx = bh * ldgPsi<T>(P, P.psih_in[XN][0], q) + ch * dez_i * idx_;
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
            const float bh = __ldg(P.bh[YN] + jr), ch = __ldg(P.ch[YN] + jr);
            float pxy = bh * ldgPsi<T>(P, P.psih_in[YN][0], q) + ch * dez_j * idx_;
            float pzy = bh * ldgPsi<T>(P, P.psih_in[YN][1], q) + ch * dex_j * idx_;
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
            const float bh = __ldg(P.bh[ZN] + kr), ch = __ldg(P.ch[ZN] + kr);
            float pyz = bh * ldgPsi<T>(P, P.psih_in[ZN][1], q) + ch * dex_k * idx_;
            float pxz = bh * ldgPsi<T>(P, P.psih_in[ZN][0], q) + ch * dey_k * idx_;
            hy -= dbdx * pyz;
            hx += dbdx * pxz;
            if (owner) { stPsi<T>(P, P.psih_out[ZN][1], q, pyz, stp, 18 + 2 * ZN + 1); stPsi<T>(P, P.psih_out[ZN][0], q, pxz, stp, 18 + 2 * ZN + 0); }
        }
    }
    if ((P.cp_on[XN] && il && jin && kin) || (P.cp_on[YN] && jl && iin && kin) || (P.cp_on[ZN] && kl && iin && jin))
        hx = hy = hz = 0.f;
    return make_float3(hx, hy, hz);
}

// H^{n+1/2}(i) at one cell from E^n and the six E differences (ystep_h,
// yee.c:246-256, then h_special where the cell lies in a slab or on a face).
template <class T>
__device__ __forceinline__ void h_update(const DevPlan &P, const float4 *scls, int cls, int i, int j, int k,
                                         bool special, bool owner, bool tsf, float dey_i, float dez_i, float dex_j, float dez_j,
                                         float dex_k, float dey_k, float h[3])
{
    const float4 hc = scls[cls * 4 + 2];     // da, db
    const bool il = (i == P.xr - 1), jl = (j == P.yr - 1), kl = (k == P.zr - 1);
    float ikx = 1.f, iky = 1.f, ikz = 1.f;
    if (special) { ikx = __ldg(P.ikh[0] + i); iky = __ldg(P.ikh[1] + j); ikz = __ldg(P.ikh[2] + k); }
    if (!(jl || kl)) h[0] = hc.x * h[0] + hc.y * (dey_k * ikz - dez_j * iky);
    if (!(il || kl)) h[1] = hc.x * h[1] + hc.y * (dez_i * ikx - dex_k * ikz);
    if (!(il || jl)) h[2] = hc.x * h[2] + hc.y * (dex_j * iky - dey_i * ikx);
    if (special) {
        const float3 o = h_special<T>(P, i, j, k, owner, tsf, hc.y, dey_i, dez_i, dex_j, dez_j, dex_k, dey_k,
                                   make_float3(h[0], h[1], h[2]));
        h[0] = o.x; h[1] = o.y; h[2] = o.z;
    }
}

// E^{n+1}(i) of one cell on the general path: ADE branch with its CPML
// (yee.c:914-1108), ordinary update (yee.c:1113-1128), PEC rule
// (yee.c:1138-1237), boundary_estep zero planes, psi_E and corrections
// (boundary.c:691-884) and TSF E (source.c:547-771).
template <bool ADE, int NPOLES, class T>
__device__ __noinline__ float3 e_special(const DevPlan &P, const float4 *scls, int cls, int i, int j, int k, bool tsf,
                                         float3 eo3, float3 h3, float hx_jm, float hz_jm, float hx_km, float hy_km,
                                         float hy_im, float hz_im)
{
    const uint32_t stp = sr_step<T>(P);
    const float eo[3] = {eo3.x, eo3.y, eo3.z};
    const float h[3] = {h3.x, h3.y, h3.z};
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const float4 c0 = scls[cls * 4 + 0], c1 = scls[cls * 4 + 1], c2 = scls[cls * 4 + 2], c3 = scls[cls * 4 + 3];
    const unsigned fl = __float_as_uint(c0.w);
    float ca[3] = {c0.x, c0.y, c0.z}, cb[3] = {c1.x, c1.y, c1.z};
    const float cba[3] = {c3.x, c3.y, c3.z};
    if (fl & CF_DESIGN) {   // adjoint design region: coefficients per cell
        const int64_t q = ((int64_t)(i - P.dbox[0]) * (P.dbox[3] - P.dbox[2]) + (j - P.dbox[2])) * (P.dbox[5] - P.dbox[4]) + (k - P.dbox[4]);
        for (int a = 0; a < 3; a++) { ca[a] = __ldg(P.dcoef + 6 * q + a); cb[a] = __ldg(P.dcoef + 6 * q + 3 + a); }
    }
    const int ade_set = __float_as_int(c2.z);
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    const float ikx = __ldg(P.ike[0] + i), iky = __ldg(P.ike[1] + j), ikz = __ldg(P.ike[2] + k);
    const float hx = h[0], hy = h[1], hz = h[2];
    const bool gx = (j > 0 && k > 0), gy = (i > 0 && k > 0), gz = (i > 0 && j > 0);
    const float dhz_i = i > 0 ? hz - hz_im : 0.f, dhy_i = i > 0 ? hy - hy_im : 0.f;
    const float dhz_j = j > 0 ? hz - hz_jm : 0.f, dhx_j = j > 0 ? hx - hx_jm : 0.f;
    const float dhx_k = k > 0 ? hx - hx_km : 0.f, dhy_k = k > 0 ? hy - hy_km : 0.f;
    const float curlx = dhz_j * iky - dhy_k * ikz;
    const float curly = dhx_k * ikz - dhz_i * ikx;
    const float curlz = dhy_i * ikx - dhx_j * iky;
    float nx = eo[0], ny = eo[1], nz = eo[2];
    const float idx_ = 1.0f / P.dx;
    float px0[2] = {0, 0}, pxn[2] = {0, 0}, py0[2] = {0, 0}, pyn[2] = {0, 0}, pz0[2] = {0, 0}, pzn[2] = {0, 0};
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
        const DevAde &A = P.ade[ade_set];
        const bool comp[3] = {(fl & CF_ADE_X) != 0, (fl & CF_ADE_Y) != 0, (fl & CF_ADE_Z) != 0};
        // difference-form state (see DevAde); E^{n-1} is the output set before this write
        float qd[3] = {0, 0, 0}, ep[3] = {0, 0, 0}, pc[3][2], qc[3][2];
        for (int a = 0; a < 3; a++) {
            if (!comp[a]) continue;
            qd[a] = P.q[a][c]; ep[a] = ldE<T>(P.fout[a], c);
            for (int n = 0; n < NPOLES; n++) { pc[a][n] = P.pc[a][n][c]; qc[a][n] = P.qc[a][n][c]; }
        }
        const float curl[3] = {curlx, curly, curlz};
        const bool gd[3] = {gx, gy, gz};
        float ne[3] = {nx, ny, nz};
        for (int a = 0; a < 3; a++) {
            if (!(comp[a] && gd[a])) continue;
            float v = A.c0dx * curl[a] + A.qe * qd[a];
            for (int n = 0; n < NPOLES; n++) v += A.qpe[n] * qc[a][n] + A.pe[n] * pc[a][n];
            v += A.c2 * ep[a] + A.c3 * eo[a];
            ne[a] = v;
        }
        if (!zero) {   // CPML inside the ADE branch, first psi_E update
            if (inx0 && i > 1) {   // x0 corrections are scaled by cb == 0 (yee.c:577)
                const float be = __ldg(P.be[X0] + i), ce = __ldg(P.ce[X0] + i);
                px0[0] = be * px0[0] + ce * dhz_i * idx_;
                px0[1] = be * px0[1] + ce * dhy_i * idx_;
            }
            if (iny0 && j > 1) {
                const float be = __ldg(P.be[Y0] + j), ce = __ldg(P.ce[Y0] + j);
                py0[0] = be * py0[0] + ce * dhz_j * idx_;
                py0[1] = be * py0[1] + ce * dhx_j * idx_;
                if ((i > 0 && k > 0) && comp[0]) ne[0] += P.dx * cba[0] * py0[0];
                if ((i > 0 && k > 0) && comp[2]) ne[2] -= P.dx * cba[2] * py0[1];
            }
            if (inz0 && k > 1) {
                const float be = __ldg(P.be[Z0] + k), ce = __ldg(P.ce[Z0] + k);
                pz0[1] = be * pz0[1] + ce * dhx_k * idx_;
                pz0[0] = be * pz0[0] + ce * dhy_k * idx_;
                if ((i > 0 && j > 0) && comp[1]) ne[1] += P.dx * cba[1] * pz0[1];
                if ((i > 0 && j > 0) && comp[0]) ne[0] -= P.dx * cba[0] * pz0[0];
            }
            if (inxn) {
                const int ir = i - (xr - P.cp_d[XN]);
                const float be = __ldg(P.be[XN] + ir), ce = __ldg(P.ce[XN] + ir);
                pxn[0] = be * pxn[0] + ce * dhz_i * idx_;
                pxn[1] = be * pxn[1] + ce * dhy_i * idx_;
                if ((j > 0 && k > 0) && comp[1]) ne[1] -= P.dx * cba[1] * pxn[0];
                if ((j > 0 && k > 0) && comp[2]) ne[2] += P.dx * cba[2] * pxn[1];
            }
            if (inyn) {
                const int jr = j - (yr - P.cp_d[YN]);
                const float be = __ldg(P.be[YN] + jr), ce = __ldg(P.ce[YN] + jr);
                pyn[0] = be * pyn[0] + ce * dhz_j * idx_;
                pyn[1] = be * pyn[1] + ce * dhx_j * idx_;
                if ((i > 0 && k > 0) && comp[0]) ne[0] += P.dx * cba[0] * pyn[0];
                if ((i > 0 && k > 0) && comp[2]) ne[2] -= P.dx * cba[2] * pyn[1];
            }
            if (inzn) {
                const int kr = k - (zr - P.cp_d[ZN]);
                const float be = __ldg(P.be[ZN] + kr), ce = __ldg(P.ce[ZN] + kr);
                pzn[1] = be * pzn[1] + ce * dhx_k * idx_;
                pzn[0] = be * pzn[0] + ce * dhy_k * idx_;
                if ((i > 0 && j > 0) && comp[1]) ne[1] += P.dx * cba[1] * pzn[1];
                if ((i > 0 && j > 0) && comp[0]) ne[0] -= P.dx * cba[0] * pzn[0];
            }
        }
        for (int a = 0; a < 3; a++) {   // polarisation recursions of the owned components
            if (!comp[a]) continue;
            const float e1 = ne[a];
            P.q[a][c] = A.ma0 * qd[a] + A.a2 * (ep[a] + 2.f * eo[a] + e1);
            for (int n = 0; n < NPOLES; n++) {
                const float qn = A.rp[n] * pc[a][n] + A.rq[n] * qc[a][n] + A.bp2[n] * ep[a] + A.bp3[n] * eo[a] + A.bp4[n] * e1;
                P.qc[a][n][c] = qn;
                P.pc[a][n][c] = pc[a][n] + qn;
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
        const float dx = P.dx;
        if (inx0) {
            const float be = __ldg(P.be[X0] + i), ce = __ldg(P.ce[X0] + i);
            px0[0] = be * px0[0] + ce * dhz_i * idx_;
            px0[1] = be * px0[1] + ce * dhy_i * idx_;
            if (j > 0 && k > 0) {
                if (ty) ny -= dx * cb[1] * px0[0];
                if (tz) nz += dx * cb[2] * px0[1];
                stPsiE<T>(P, P.psie[X0][0], qx0, px0[0], stp, 6 + 2 * X0 + 0); stPsiE<T>(P, P.psie[X0][1], qx0, px0[1], stp, 6 + 2 * X0 + 1);
            }
        }
        if (iny0) {
            const float be = __ldg(P.be[Y0] + j), ce = __ldg(P.ce[Y0] + j);
            py0[0] = be * py0[0] + ce * dhz_j * idx_;
            py0[1] = be * py0[1] + ce * dhx_j * idx_;
            if (i > 0 && k > 0) {
                if (tx) nx += dx * cb[0] * py0[0];
                if (tz) nz -= dx * cb[2] * py0[1];
                stPsiE<T>(P, P.psie[Y0][0], qy0, py0[0], stp, 6 + 2 * Y0 + 0); stPsiE<T>(P, P.psie[Y0][1], qy0, py0[1], stp, 6 + 2 * Y0 + 1);
            }
        }
        if (inz0) {
            const float be = __ldg(P.be[Z0] + k), ce = __ldg(P.ce[Z0] + k);
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
            const float be = __ldg(P.be[XN] + ir), ce = __ldg(P.ce[XN] + ir);
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
            const float be = __ldg(P.be[YN] + jr), ce = __ldg(P.ce[YN] + jr);
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
            const float be = __ldg(P.be[ZN] + kr), ce = __ldg(P.ce[ZN] + kr);
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
    return make_float3(nx, ny, nz);
}

// ------------------------------------------------------------ slab kernels

// One thread per cell of the slab boxes (the CPML slabs and every cell the
// bulk kernel does not own).  slab_h forms H^{n+1/2} with the full special
// path; slab_e then forms E^{n+1} from the H^{n+1/2} that slab_h and the bulk
// kernel wrote.  Both read E^n/H^n from the input set only.

// The box of this block: the last one whose first_block is not above
// blockIdx.x (boxes are numbered in ascending first_block; an empty box shares
// its successor's first_block and is skipped).  Binary search: a batch lists
// every instance's boxes, a hundred or more.
__device__ __forceinline__ int box_of_block(const SlabBox *boxes, int nboxes)
{
    const long long bid = blockIdx.x;
    int lo = 0, hi = nboxes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (boxes[mid].first_block <= bid) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ bool box_cell(const SlabBox *boxes, int nboxes, int &i, int &j, int &k, int &inst, bool &tsf)
{
    const SlabBox B = boxes[box_of_block(boxes, nboxes)];
    long long t = ((long long)blockIdx.x - B.first_block) * blockDim.x + threadIdx.x;
    const int nk = B.k1 - B.k0, nj = B.j1 - B.j0;
    if (t >= (long long)(B.i1 - B.i0) * nj * nk) return false;
    k = B.k0 + (int)(t % nk);
    t /= nk;
    j = B.j0 + (int)(t % nj);
    i = B.i0 + (int)(t / nj);
    inst = B.inst;
    tsf = B.tsf != 0;
    return true;
}

// 3 CTAs per SM: the slab kernels are latency-bound, and 24 resident warps
// beat the register spill this costs e_special (1.95 -> 1.60 ms per 512^3 step)
template <class T>
__device__ __forceinline__ void slab_h_cell(const DevPlan &P, int i, int j, int k, bool tsf)
{
    const uint32_t stp = sr_step<T>(P);
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const float *EX = P.fin[0], *EY = P.fin[1], *EZ = P.fin[2];
    const float ex = ldgE<T>(EX, c), ey = ldgE<T>(EY, c), ez = ldgE<T>(EZ, c);
    const bool il = (i == P.xr - 1), jl = (j == P.yr - 1), kl = (k == P.zr - 1);
    const float eyk = kl ? 0.f : ldgE<T>(EY, c + 1), exk = kl ? 0.f : ldgE<T>(EX, c + 1);
    const float ezj = jl ? 0.f : ldgE<T>(EZ, c + P.sj), exj = jl ? 0.f : ldgE<T>(EX, c + P.sj);
    const float ezi = il ? 0.f : ldgE<T>(EZ, c + P.si), eyi = il ? 0.f : ldgE<T>(EY, c + P.si);
    float h[3] = {ldgH<T>(P, P.fin[3], c), ldgH<T>(P, P.fin[4], c), ldgH<T>(P, P.fin[5], c)};
    const float4 *cl = reinterpret_cast<const float4 *>(P.classes);
    h_update<T>(P, cl, cls_at(P, i, j, k), i, j, k, true, true, tsf, eyi - ey, ezi - ez, exj - ex, ezj - ez, exk - ex, eyk - ey, h);
    stH<T>(P, P.fout[3], c, h[0], stp, 3);
    stH<T>(P, P.fout[4], c, h[1], stp, 4);
    stH<T>(P, P.fout[5], c, h[2], stp, 5);
}

// Four consecutive k cells per thread (boxes whose k bounds and row length
// are multiples of 4, as all of them are next to the bulk kernel): 16-byte
// loads of E and H, the same per-cell update as slab_h_cell with the four
// cells' loads in flight together, 16-byte stores.
__device__ __forceinline__ bool box_group4(const SlabBox *boxes, int nboxes, int &i, int &j, int &k, int &inst, bool &tsf)
{
    const SlabBox B = boxes[box_of_block(boxes, nboxes)];
    long long t = ((long long)blockIdx.x - B.first_block) * blockDim.x + threadIdx.x;
    const int nk = (B.k1 - B.k0) / 4, nj = B.j1 - B.j0;
    if (t >= (long long)(B.i1 - B.i0) * nj * nk) return false;
    k = B.k0 + 4 * (int)(t % nk);
    t /= nk;
    j = B.j0 + (int)(t % nj);
    i = B.i0 + (int)(t / nj);
    inst = B.inst;
    tsf = B.tsf != 0;
    return true;
}

template <class T>
__device__ __forceinline__ void slab_h_cell4(const DevPlan &P, int i, int j, int k, bool tsf)
{
    const uint32_t stp = sr_step<T>(P);
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const float *EX = P.fin[0], *EY = P.fin[1], *EZ = P.fin[2];
    const bool il = (i == P.xr - 1), jl = (j == P.yr - 1), kl = (k + 3 == P.zr - 1);
    float ex[4], ey[4], ez[4], exj[4], ezj[4], eyi[4], ezi[4], hx[4], hy[4], hz[4];
    lds4a_f(ex, ldg4_ro<T>(EX, c));
    lds4a_f(ey, ldg4_ro<T>(EY, c));
    lds4a_f(ez, ldg4_ro<T>(EZ, c));
    if (jl) {
        for (int q = 0; q < 4; q++) exj[q] = ezj[q] = 0.f;
    } else {
        lds4a_f(exj, ldg4_ro<T>(EX, c + P.sj));
        lds4a_f(ezj, ldg4_ro<T>(EZ, c + P.sj));
    }
    if (il) {
        for (int q = 0; q < 4; q++) eyi[q] = ezi[q] = 0.f;
    } else {
        lds4a_f(eyi, ldg4_ro<T>(EY, c + P.si));
        lds4a_f(ezi, ldg4_ro<T>(EZ, c + P.si));
    }
    const float exk4 = kl ? 0.f : ldgE<T>(EX, c + 4), eyk4 = kl ? 0.f : ldgE<T>(EY, c + 4);
    lds4a_f(hx, ldg4_ro<T>(P.fin[3], c));
    lds4a_f(hy, ldg4_ro<T>(P.fin[4], c));
    lds4a_f(hz, ldg4_ro<T>(P.fin[5], c));
    const uint32_t cw = __ldg(reinterpret_cast<const uint32_t *>(P.cls + ((int64_t)i * P.yr + j) * P.cpitch + k));
    const float4 *cl = reinterpret_cast<const float4 *>(P.classes);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        float h[3] = {hx[q], hy[q], hz[q]};
        if (Stor<T>::scaled) { h[0] *= P.ihs; h[1] *= P.ihs; h[2] *= P.ihs; }
        const float eyk = q < 3 ? ey[q + 1] : eyk4, exk = q < 3 ? ex[q + 1] : exk4;
        h_update<T>(P, cl, (cw >> (8 * q)) & 0xff, i, j, k + q, true, true, tsf, eyi[q] - ey[q], ezi[q] - ez[q],
                    exj[q] - ex[q], ezj[q] - ez[q], exk - ex[q], eyk - ey[q], h);
        hx[q] = h[0]; hy[q] = h[1]; hz[q] = h[2];
    }
    const float s = Stor<T>::scaled ? P.hs : 1.f;
    stg4<T>(P.fout[3], c, make_float4(hx[0], hx[1], hx[2], hx[3]), s, stp, 3);
    stg4<T>(P.fout[4], c, make_float4(hy[0], hy[1], hy[2], hy[3]), s, stp, 4);
    stg4<T>(P.fout[5], c, make_float4(hz[0], hz[1], hz[2], hz[3]), s, stp, 5);
}

template <class T>
__global__ void __launch_bounds__(256, 2) slab_h4_kernel(const __grid_constant__ DevPlan P, const SlabBox *boxes, int nboxes)
{
    int i, j, k, inst;
    bool tsf;
    if (box_group4(boxes, nboxes, i, j, k, inst, tsf)) slab_h_cell4<T>(P, i, j, k, tsf);
}

template <class T>
__global__ void __launch_bounds__(256, 2) slab_h4_batch(const DevPlan *plans, const SlabBox *boxes, int nboxes)
{
    int i, j, k, inst;
    bool tsf;
    if (box_group4(boxes, nboxes, i, j, k, inst, tsf)) slab_h_cell4<T>(plans[inst], i, j, k, tsf);
}

template <class T>
__global__ void __launch_bounds__(256, 3) slab_h_kernel(const __grid_constant__ DevPlan P, const SlabBox *boxes, int nboxes)
{
    int i, j, k, inst;
    bool tsf;
    if (box_cell(boxes, nboxes, i, j, k, inst, tsf)) slab_h_cell<T>(P, i, j, k, tsf);
}

template <class T>
__global__ void __launch_bounds__(256, 3) slab_h_batch(const DevPlan *plans, const SlabBox *boxes, int nboxes)
{
    int i, j, k, inst;
    bool tsf;
    if (box_cell(boxes, nboxes, i, j, k, inst, tsf)) slab_h_cell<T>(plans[inst], i, j, k, tsf);
}

template <bool ADE, int NPOLES, class T>
__device__ __forceinline__ void slab_e_cell(const DevPlan &P, int i, int j, int k, bool tsf)
{
    const uint32_t stp = sr_step<T>(P);
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const float *HX = P.fout[3], *HY = P.fout[4], *HZ = P.fout[5];   // H^{n+1/2}, written this step
    const float3 eo = make_float3(ldgE<T>(P.fin[0], c), ldgE<T>(P.fin[1], c), ldgE<T>(P.fin[2], c));
    const float3 h = make_float3(ldH<T>(P, HX, c), ldH<T>(P, HY, c), ldH<T>(P, HZ, c));
    const float hx_jm = j > 0 ? ldH<T>(P, HX, c - P.sj) : 0.f, hz_jm = j > 0 ? ldH<T>(P, HZ, c - P.sj) : 0.f;
    const float hx_km = k > 0 ? ldH<T>(P, HX, c - 1) : 0.f, hy_km = k > 0 ? ldH<T>(P, HY, c - 1) : 0.f;
    const float hy_im = i > 0 ? ldH<T>(P, HY, c - P.si) : 0.f, hz_im = i > 0 ? ldH<T>(P, HZ, c - P.si) : 0.f;
    const float4 *cl = reinterpret_cast<const float4 *>(P.classes);
    const float3 en =
        e_special<ADE, NPOLES, T>(P, cl, cls_at(P, i, j, k), i, j, k, tsf, eo, h, hx_jm, hz_jm, hx_km, hy_km, hy_im, hz_im);
    stE<T>(P.fout[0], c, en.x, stp, 0);
    stE<T>(P.fout[1], c, en.y, stp, 1);
    stE<T>(P.fout[2], c, en.z, stp, 2);
}

template <bool ADE, int NPOLES, class T>
__global__ void __launch_bounds__(256, 3) slab_e_kernel(const __grid_constant__ DevPlan P, const SlabBox *boxes, int nboxes)
{
    int i, j, k, inst;
    bool tsf;
    if (box_cell(boxes, nboxes, i, j, k, inst, tsf)) slab_e_cell<ADE, NPOLES, T>(P, i, j, k, tsf);
}

template <bool ADE, int NPOLES, class T>
__global__ void __launch_bounds__(256, 3) slab_e_batch(const DevPlan *plans, const SlabBox *boxes, int nboxes)
{
    int i, j, k, inst;
    bool tsf;
    if (box_cell(boxes, nboxes, i, j, k, inst, tsf)) slab_e_cell<ADE, NPOLES, T>(plans[inst], i, j, k, tsf);
}

// ------------------------------------------------------------ TSF face tables

// This step's TSF corrections for every face cell (source.c:547-771 and
// 1476-1672): the 1D grid value at corr*dcomp(cell) by the cubic
// interpolation of dline.c:89-111 (FP64), projected by gex..ghz, scaled by
// dt/(dx mu0) for H or (dt/dx)/epsilon(cell) for E, gated by TSF_SKIP, the
// source-skip map and (k0 face) the PEC test.  Runs after aux_step.
__device__ __forceinline__ void tsf_face_cell(const DevPlan &P, int t)
{
    const int i0 = P.t0[0], j0 = P.t0[1], k0 = P.t0[2], in = P.t1[0], jn = P.t1[1], kn = P.t1[2];
    const int ni = in - i0 + 1, nj = jn - j0 + 1, nk = kn - k0 + 1;
    const int sz[3] = {nj * nk, ni * nk, ni * nj};
    if (!P.tsf_on || t >= 2 * (sz[0] + sz[1] + sz[2])) return;
    int f = 0, off = t;
    while (f < 6 && off >= sz[f / 2]) { off -= sz[f / 2]; f++; }
    if (f >= 6) return;
    const int a = off / P.tnb[f], b = off % P.tnb[f];
    const uint8_t fl = P.tmap[f][off];
    const double hc = P.hcor;
    float2 dh = make_float2(0.f, 0.f), de = make_float2(0.f, 0.f);
    const float4 *cls4 = reinterpret_cast<const float4 *>(P.classes);
    if (fl & 1) {
        int ei, ej, ek;   // E cell; dH / dE are the dcomp positions of the H and E corrections
        double dH, dE;
        if (f < 2) {
            const int j = j0 + a, k = k0 + b;
            if (f == 0) { ei = i0; dH = tsf_dcomp(P, i0, j, k); dE = tsf_dcomp(P, i0 - 1, j, k); }
            else { ei = in; dH = tsf_dcomp(P, in, j, k); dE = dH; }
            ej = j; ek = k;
        } else if (f < 4) {
            const int i = i0 + a, k = k0 + b;
            if (f == 2) { ej = j0; dH = tsf_dcomp(P, i, j0, k); dE = tsf_dcomp(P, i, j0 - 1, k); }
            else { ej = jn; dH = tsf_dcomp(P, i, jn, k); dE = dH; }
            ei = i; ek = k;
        } else {
            const int i = i0 + a, j = j0 + b;
            if (f == 4) { ek = k0; dH = tsf_dcomp(P, i, j, k0); dE = tsf_dcomp(P, i, j, k0 - 1); }
            else { ek = kn; dH = tsf_dcomp(P, i, j, kn); dE = dH; }
            ei = i; ej = j;
        }
        const double ve = tsf_dval(P.aux_e, P.jres, dH);
        const double vh = tsf_dval(P.aux_h, P.jres, dE);
        const double ce = (double)cls4[cls_at(P, ei, ej, ek) * 4 + 1].w;
        const bool pec = (fl & 2) != 0;
        switch (f) {
        case 0:
            if (ek < kn) dh.x = -(float)(hc * (ve * P.gez));
            if (ej < jn) dh.y = (float)(hc * (ve * P.gey));
            if (ej < jn) de.x = (float)(ce * (vh * P.ghz));
            if (ek < kn) de.y = -(float)(ce * (vh * P.ghy));
            break;
        case 1:
            if (ek < kn) dh.x = (float)(hc * (ve * P.gez));
            if (ej < jn) dh.y = -(float)(hc * (ve * P.gey));
            if (ej < jn) de.x = -(float)(ce * (vh * P.ghz));
            if (ek < kn) de.y = (float)(ce * (vh * P.ghy));
            break;
        case 2:
            if (ek < kn) dh.x = (float)(hc * (ve * P.gez));
            if (ei < in) dh.y = -(float)(hc * (ve * P.gex));
            if (ei < in) de.x = -(float)(ce * (vh * P.ghz));
            if (ek < kn) de.y = (float)(ce * (vh * P.ghx));
            break;
        case 3:
            if (ek < kn) dh.x = -(float)(hc * (ve * P.gez));
            if (ei < in) dh.y = (float)(hc * (ve * P.gex));
            if (ei < in) de.x = (float)(ce * (vh * P.ghz));
            if (ek < kn) de.y = -(float)(ce * (vh * P.ghx));
            break;
        case 4:
            if (ej < jn && !pec) dh.x = -(float)(hc * (ve * P.gey));
            if (ei < in && !pec) dh.y = (float)(hc * (ve * P.gex));
            if (ei < in && !pec) de.x = (float)(ce * (vh * P.ghy));
            if (ej < jn && !pec) de.y = -(float)(ce * (vh * P.ghx));
            break;
        default:
            if (ej < jn) dh.x = (float)(hc * (ve * P.gey));
            if (ei < in) dh.y = -(float)(hc * (ve * P.gex));
            if (ei < in) de.x = -(float)(ce * (vh * P.ghy));
            if (ej < jn) de.y = (float)(ce * (vh * P.ghx));
            break;
        }
    }
    P.tcor_h[f][off] = dh;
    P.tcor_e[f][off] = de;
    (void)a; (void)b;
}

__global__ void tsf_face_kernel(const __grid_constant__ DevPlan P, int total)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < total) tsf_face_cell(P, t);
}

__global__ void tsf_face_batch(const DevPlan *plans)
{
    tsf_face_cell(plans[blockIdx.y], blockIdx.x * blockDim.x + threadIdx.x);
}

// ------------------------------------------------------------ 1D aux grid

// 1D TSF grid step of source.c:1469-1473 over 1dpool.c:84-162, in FP64 with
// the reference's operation order (no contraction); also records the probes
// of the previous step (output.c:341-352).
__device__ __forceinline__ void aux_step_body(const DevAux &A)
{
    const int s = *A.step;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (s > 0 && s - 1 < A.nsteps_planned) {
        for (int q = tid; q < A.nprobes * 6; q += nt) {
            int p = q / 6, comp = q % 6;
            A.probe_out[((size_t)p * A.nsteps_planned + (s - 1)) * 6 + comp] = (double)(ld_any(A.fields[comp], A.probe_cells[p], A.storage) * (comp >= 3 && A.storage ? A.ihs : 1.f));
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

__global__ void aux_step_kernel(const DevAux A) { aux_step_body(A); }

__global__ void aux_step_batch(const DevAux *A) { aux_step_body(A[blockIdx.x]); }

__global__ void probe_capture_kernel(const DevAux A)
{
    const int s = *A.step;     // number of completed steps
    if (s < 1 || s - 1 >= A.nsteps_planned) return;
    for (int q = threadIdx.x; q < A.nprobes * 6; q += blockDim.x) {
        int p = q / 6, comp = q % 6;
        A.probe_out[((size_t)p * A.nsteps_planned + (s - 1)) * 6 + comp] = (double)(ld_any(A.fields[comp], A.probe_cells[p], A.storage) * (comp >= 3 && A.storage ? A.ihs : 1.f));
    }
}

// ------------------------------------------------------------ NFFF running DFT

// Per surface cell s and frequency f:  Ehat += E(step) w,  Dhat += dE/dn(step) w,
// w = exp(-i omega step dt).  FP64 accumulators.  Each step stores the nine
// raw E samples of the cell (E, E(c+st), E(c-st) per component) in ring slot
// step % NFFF_RING; the step that fills the last slot folds the block into the
// accumulators in step order, with the arithmetic of a per-step update, so the
// sums are those of accumulating every step (the accumulators are read and
// written once per NFFF_RING steps instead of every step).
constexpr int NFFF_TW_MAXF = 16;   // frequencies whose twiddles a CTA tabulates in shared memory

// exp(-i omega_f (first_step + j) dt) of the block's steps, computed once per
// CTA: tw[f * nslots + j] = (cos, sin).  All threads of the CTA take part.
__device__ __forceinline__ void nfff_twiddles(const DevNfff &N, int first_step, int nslots, double2 *tw)
{
    for (int t = threadIdx.x; t < nslots * N.nfreq; t += blockDim.x) {
        double sn, cs;
        sincos(N.omega_dt[t / nslots] * (double)(first_step + t % nslots), &sn, &cs);
        tw[t] = make_double2(cs, sn);
    }
    __syncthreads();
}

// tw: the CTA's twiddle table, or nullptr to evaluate them per cell
__device__ __forceinline__ void nfff_fold(const DevNfff &N, int s, int first_step, int nslots, bool clear, const double2 *tw)
{
    const size_t ns = (size_t)N.ns;
    for (int f = 0; f < N.nfreq; f++) {
        double2 A[6];
        for (int q = 0; q < 6; q++) A[q] = N.acc[((size_t)f * 6 + q) * ns + s];
        for (int j = 0; j < nslots; j++) {
            const float *r = N.ring + (size_t)j * 9 * ns + s;
            double v[6];
            for (int a = 0; a < 3; a++) {
                v[a] = (double)r[(3 * a) * ns];
                v[3 + a] = ((double)r[(3 * a + 1) * ns] - (double)r[(3 * a + 2) * ns]) * N.inv2dx;
            }
            double sn, cs;
            if (tw) { cs = tw[f * nslots + j].x; sn = tw[f * nslots + j].y; }
            else sincos(N.omega_dt[f] * (double)(first_step + j), &sn, &cs);
            for (int q = 0; q < 6; q++) {
                A[q].x += v[q] * cs;
                A[q].y -= v[q] * sn;
            }
        }
        for (int q = 0; q < 6; q++) N.acc[((size_t)f * 6 + q) * ns + s] = A[q];
    }
    if (clear)
        for (int j = 0; j < nslots; j++)
            for (int q = 0; q < 9; q++) N.ring[((size_t)j * 9 + q) * ns + s] = 0.f;
}

// the step counter, the slot and the fold decision are the same for every
// thread of a launch (one plan per CTA in a batch), so the CTA-wide twiddle
// table and its barrier are reached by all threads
__device__ __forceinline__ void nfff_accumulate_cell(const DevNfff &N, int s)
{
    if (N.ns <= 0 || N.nfreq <= 0) return;   // a batch instance without a running DFT: zeroed, no step counter
    const int step = *N.step - 1;
    if (step < 0) return;
    const bool live = s < N.ns;
    const int slot = step % NFFF_RING;
    const size_t ns = (size_t)N.ns;
    if (live) {
        const int64_t c = N.cell[s];
        const int64_t st = N.nstride[s];
        float *r = N.ring + (size_t)slot * 9 * ns + s;
        for (int a = 0; a < 3; a++) {
            const float *E = N.e[a];
            r[(3 * a) * ns] = ld_any(E, c, N.storage);
            r[(3 * a + 1) * ns] = ld_any(E, c + st, N.storage);
            r[(3 * a + 2) * ns] = ld_any(E, c - st, N.storage);
        }
    }
    if (slot == NFFF_RING - 1) {
        __shared__ double2 tw[NFFF_RING * NFFF_TW_MAXF];
        const bool table = N.nfreq <= NFFF_TW_MAXF;
        if (table) nfff_twiddles(N, step - (NFFF_RING - 1), NFFF_RING, tw);
        if (live) nfff_fold(N, s, step - (NFFF_RING - 1), NFFF_RING, false, table ? tw : nullptr);
    }
}

// the steps since the last full block (device step counter % NFFF_RING); their
// slots are cleared, so the fold at the end of the block adds zeros for them
__global__ void nfff_fold_pending_kernel(const DevNfff N)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (N.ns <= 0 || N.nfreq <= 0) return;
    const int done = *N.step;
    const int pending = done % NFFF_RING;
    if (pending == 0) return;
    __shared__ double2 tw[NFFF_RING * NFFF_TW_MAXF];
    const bool table = N.nfreq <= NFFF_TW_MAXF;
    if (table) nfff_twiddles(N, done - pending, pending, tw);
    if (s < N.ns) nfff_fold(N, s, done - pending, pending, true, table ? tw : nullptr);
}

__global__ void nfff_accumulate_kernel(const DevNfff N) { nfff_accumulate_cell(N, blockIdx.x * blockDim.x + threadIdx.x); }

__global__ void nfff_accumulate_batch(const DevNfff *N)
{
    nfff_accumulate_cell(N[blockIdx.y], blockIdx.x * blockDim.x + threadIdx.x);
}

// ------------------------------------------------------------ far-field integration

// F_hat_n(omega) = sum_s A_s exp(-i omega (R_ns - istart_n) dt) *
//   [(-c' + b e^{i omega dt} + c' e^{2 i omega dt}) Ehat_s + sgn_f a e^{i omega dt} Dhat_s]
// with r, cos(theta), a, b, c and the retarded index R = (int)(1 + r/(c dt)) of
// farfield.c:175-405: the DFT of the reference time-domain series.
//
// Tiled over (far points x surface-cell groups): a CTA owns 128 far points
// (one per thread) and one group of surface cells, staged 32 at a time in
// shared memory with their accumulators for NF frequencies (read once per
// CTA instead of once per point).  exp(-i omega R dt) comes from a table over
// R; exp(+i omega istart dt), the face area and the sum over groups are
// applied by farfield_reduce_kernel.  FP64 throughout.
template <int NF>
__global__ void __launch_bounds__(128) farfield_partial_kernel(const DevFarfield F, int f0)
{
    constexpr int CH = 32;
    __shared__ double2 sacc[CH][NF][6];
    __shared__ int4 sgeo[CH];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = p < F.npoints;
    const int per = (F.ns + F.groups - 1) / F.groups;
    const int s0 = blockIdx.y * per, s1 = min(F.ns, s0 + per);
    const double C0 = 299792458.0, PI = 3.14159265358979323846;
    const double dt = F.dt, dx = F.dx, c0dt = C0 * dt;
    double x = 0, y = 0, z = 0;
    if (live) { x = F.points[3 * p]; y = F.points[3 * p + 1]; z = F.points[3 * p + 2]; }
    double cw[NF], sw[NF], c2[NF], s2[NF];
    for (int f = 0; f < NF; f++) {
        const double om = F.omega[f0 + f];
        sincos(om * dt, &sw[f], &cw[f]);
        sincos(2.0 * om * dt, &s2[f], &c2[f]);
    }
    double acc[NF][3][2];
    for (int f = 0; f < NF; f++)
        for (int q = 0; q < 3; q++) acc[f][q][0] = acc[f][q][1] = 0.0;
    for (int base = s0; base < s1; base += CH) {
        const int n = min(CH, s1 - base);
        __syncthreads();
        for (int q = threadIdx.x; q < n; q += blockDim.x)
            sgeo[q] = make_int4(F.cell_ijk[3 * (base + q)], F.cell_ijk[3 * (base + q) + 1], F.cell_ijk[3 * (base + q) + 2],
                                F.face[base + q]);
        for (int t = threadIdx.x; t < n * NF * 6; t += blockDim.x) {
            const int q = t % n, fq = t / n;
            sacc[q][fq / 6][fq % 6] = F.acc[((size_t)(f0 + fq / 6) * 6 + fq % 6) * F.ns + base + q];
        }
        __syncthreads();
        if (!live) continue;
        for (int q = 0; q < n; q++) {
            const int4 g = sgeo[q];
            const double rx = x - g.x, ry = y - g.y, rz = z - g.z;
            const double rc = sqrt(rx * rx + ry * ry + rz * rz);
            double dot;   // angle(): normal of the face (farfield.c:44-54)
            switch (g.w) {
            case 0: dot = -rx; break;
            case 1: dot = rx; break;
            case 2: dot = -ry; break;
            case 3: dot = ry; break;
            case 4: dot = -rz; break;
            default: dot = rz; break;
            }
            const double ct = dot / rc;
            const double r = rc * dx;
            const int R = min((int)(1.0 + r / c0dt), F.ntw - 1);
            const double ir = 1.0 / r;
            const double a = ir / (4.0 * PI);
            const double b = -ct / (4.0 * PI) * ir * ir;
            const double cp = -ct / (4.0 * PI * C0) * ir / (2.0 * dt);
            const double sg = (g.w & 1) ? 1.0 : -1.0;
            for (int f = 0; f < NF; f++) {
                const double2 w = F.tw[(size_t)(f0 + f) * F.ntw + R];
                const double Kr = -cp + b * cw[f] + cp * c2[f], Ki = b * sw[f] + cp * s2[f];
                const double Lr = sg * a * cw[f], Li = sg * a * sw[f];
                for (int c = 0; c < 3; c++) {
                    const double2 Eh = sacc[q][f][c], Dh = sacc[q][f][3 + c];
                    const double tr = Kr * Eh.x - Ki * Eh.y + Lr * Dh.x - Li * Dh.y;
                    const double ti = Kr * Eh.y + Ki * Eh.x + Lr * Dh.y + Li * Dh.x;
                    acc[f][c][0] += w.x * tr - w.y * ti;
                    acc[f][c][1] += w.x * ti + w.y * tr;
                }
            }
        }
    }
    if (live)
        for (int f = 0; f < NF; f++)
            for (int c = 0; c < 3; c++)
                F.part[(((size_t)blockIdx.y * F.npoints + p) * F.nfreq + f0 + f) * 3 + c] = make_double2(acc[f][c][0], acc[f][c][1]);
}

// out = area * exp(+i omega istart dt) * sum over groups (fixed order)
__global__ void farfield_reduce_kernel(const DevFarfield F)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= F.npoints * F.nfreq * 3) return;
    const int p = t / (F.nfreq * 3), f = (t / 3) % F.nfreq;
    double re = 0, im = 0;
    for (int g = 0; g < F.groups; g++) {
        const double2 v = F.part[(size_t)g * F.npoints * F.nfreq * 3 + t];
        re += v.x;
        im += v.y;
    }
    double sn, cs;
    sincos(F.omega[f] * (double)F.istart[p] * F.dt, &sn, &cs);
    const double area = F.dx * F.dx;
    F.out[t] = make_double2(area * (cs * re - sn * im), area * (cs * im + sn * re));
}

// The reference's far-field series, farfield.c:207-404, for every (surface
// cell, far point): r and cos(theta) as dist()/angle() (farfield.c:33-56),
// nn = (int)(step + 1 + r/(c dt)) - istart with the reference's operation
// order (the sum can round across an integer, so nn is formed exactly as
// there), three taps per component when 3 <= nn < ndata.  FP64 atomics.
__global__ void nfff_series_kernel(const DevNfffSeries S)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S.ns) return;
    const int step = *S.step - 1;
    const double C0 = 299792458.0, PI = 3.14159265358979323846;
    const double dx = S.dx, dt = S.dt;
    const int fc = S.face[s];
    const double ci = S.cell_ijk[3 * s], cj = S.cell_ijk[3 * s + 1], ck = S.cell_ijk[3 * s + 2];
    const int64_t cc = S.cell[s], st = S.nstride[s];
    double ev[3], dv[3];
    for (int a = 0; a < 3; a++) {
        const float *E = S.e[a];
        ev[a] = (double)ld_any(E, cc, S.storage);
        dv[a] = (double)ld_any(E, cc + st, S.storage) - (double)ld_any(E, cc - st, S.storage);
    }
    const double size = __dmul_rn(dx, dx);
    const double pos = (fc & 1) ? 1.0 : -1.0;
    for (int p = blockIdx.y; p < S.npoints; p += gridDim.y) {
        const double x = S.points[3 * p], y = S.points[3 * p + 1], z = S.points[3 * p + 2];
        const double ux = x - ci, uy = y - cj, uz = z - ck;
        const double rc = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy)), __dmul_rn(uz, uz)));
        double dot;
        switch (fc) {
        case 0: dot = -ux; break;
        case 1: dot = ux; break;
        case 2: dot = -uy; break;
        case 3: dot = uy; break;
        case 4: dot = -uz; break;
        default: dot = uz; break;
        }
        const double ct = dot / rc;
        const double r = __dmul_rn(rc, dx);
        const int nn = (int)__dadd_rn((double)(step + 1), __ddiv_rn(r, __dmul_rn(C0, dt))) - S.istart[p];
        if (nn < 3 || nn >= S.ndata) continue;
        const double a1 = 1.0 / (4.0 * PI * r);
        const double b1 = -1.0 / (4.0 * PI) * ct / (r * r);
        const double c1 = -1.0 / (4.0 * PI) * ct / (C0 * r);
        for (int a = 0; a < 3; a++) {
            double *F = S.series + ((size_t)p * 3 + a) * S.ndata;
            atomicAdd(F + nn, -c1 / 2.0 / dt * ev[a] * size);
            atomicAdd(F + nn - 1, (pos * a1 * dv[a] / 2.0 / dx + b1 * ev[a]) * size);
            atomicAdd(F + nn - 2, c1 / 2.0 / dt * ev[a] * size);
        }
    }
}

}  // namespace

void launch_aux_step(const DevAux &a, cudaStream_t st) { aux_step_kernel<<<1, 1024, 0, st>>>(a); }

void launch_probe_capture(const DevAux &a, cudaStream_t st) { probe_capture_kernel<<<1, 256, 0, st>>>(a); }

void launch_tsf_faces(const DevPlan &p, int total, cudaStream_t st)
{
    if (total > 0) tsf_face_kernel<<<(total + 255) / 256, 256, 0, st>>>(p, total);
}

template <class T>
cudaError_t slab_steps_t(const DevPlan &p, const SlabLists &L, bool ade, int npoles, cudaStream_t st)
{
    if (L.h4blocks > 0)
        slab_h4_kernel<T><<<(unsigned)L.h4blocks, 256, 0, st>>>(p, L.h4, L.nh);
    else
        slab_h_kernel<T><<<(unsigned)L.hblocks, 256, 0, st>>>(p, L.h, L.nh);
    if (L.eblocks > 0) {
        if (!ade)
            slab_e_kernel<false, 0, T><<<(unsigned)L.eblocks, 256, 0, st>>>(p, L.e, L.ne);
        else if (npoles == 0)
            slab_e_kernel<true, 0, T><<<(unsigned)L.eblocks, 256, 0, st>>>(p, L.e, L.ne);
        else
            slab_e_kernel<true, 2, T><<<(unsigned)L.eblocks, 256, 0, st>>>(p, L.e, L.ne);
    }
    if (L.epblocks > 0) slab_e_kernel<false, 0, T><<<(unsigned)L.epblocks, 256, 0, st>>>(p, L.ep, L.nep);
    return cudaGetLastError();
}

cudaError_t launch_slab_steps(const DevPlan &p, const SlabLists &L, bool ade, int npoles, int storage, cudaStream_t st)
{
    if (L.hblocks <= 0) return cudaSuccess;
    if (storage == FDTD_STORE_F16) return slab_steps_t<__half>(p, L, ade, npoles, st);
    if (storage == FDTD_STORE_BF16) return slab_steps_t<__nv_bfloat16>(p, L, ade, npoles, st);
    return slab_steps_t<float>(p, L, ade, npoles, st);
}

void launch_aux_step_batch(const DevAux *a, int nplans, cudaStream_t st)
{
    if (nplans > 0) aux_step_batch<<<nplans, 1024, 0, st>>>(a);
}

void launch_tsf_faces_batch(const DevPlan *p, int nplans, int max_cells, cudaStream_t st)
{
    if (nplans > 0 && max_cells > 0) tsf_face_batch<<<dim3((max_cells + 255) / 256, nplans), 256, 0, st>>>(p);
}

template <class T>
cudaError_t slab_steps_batch_t(const DevPlan *p, const SlabBox *boxes, int nboxes, long long nblocks, const SlabBox *boxes4,
                               long long nblocks4, const SlabBox *eboxes, int neboxes, long long neblocks, bool ade,
                               int npoles, cudaStream_t st)
{
    if (nblocks4 > 0)
        slab_h4_batch<T><<<(unsigned)nblocks4, 256, 0, st>>>(p, boxes4, nboxes);
    else
        slab_h_batch<T><<<(unsigned)nblocks, 256, 0, st>>>(p, boxes, nboxes);
    if (neblocks > 0) {
        if (!ade)
            slab_e_batch<false, 0, T><<<(unsigned)neblocks, 256, 0, st>>>(p, eboxes, neboxes);
        else if (npoles == 0)
            slab_e_batch<true, 0, T><<<(unsigned)neblocks, 256, 0, st>>>(p, eboxes, neboxes);
        else
            slab_e_batch<true, 2, T><<<(unsigned)neblocks, 256, 0, st>>>(p, eboxes, neboxes);
    }
    return cudaGetLastError();
}

cudaError_t launch_slab_steps_batch(const DevPlan *p, const SlabBox *boxes, int nboxes, long long nblocks,
                                    const SlabBox *boxes4, long long nblocks4, const SlabBox *eboxes, int neboxes,
                                    long long neblocks, bool ade, int npoles, int storage, cudaStream_t st)
{
    if (nblocks <= 0) return cudaSuccess;
    if (storage == FDTD_STORE_F16)
        return slab_steps_batch_t<__half>(p, boxes, nboxes, nblocks, boxes4, nblocks4, eboxes, neboxes, neblocks, ade, npoles, st);
    if (storage == FDTD_STORE_BF16)
        return slab_steps_batch_t<__nv_bfloat16>(p, boxes, nboxes, nblocks, boxes4, nblocks4, eboxes, neboxes, neblocks, ade,
                                                 npoles, st);
    return slab_steps_batch_t<float>(p, boxes, nboxes, nblocks, boxes4, nblocks4, eboxes, neboxes, neblocks, ade, npoles, st);
}

cudaError_t launch_slab_e_plain_batch(const DevPlan *p, const SlabBox *boxes, int nboxes, long long nblocks, int storage,
                                      cudaStream_t st)
{
    if (nblocks <= 0) return cudaSuccess;
    if (storage == FDTD_STORE_F16)
        slab_e_batch<false, 0, __half><<<(unsigned)nblocks, 256, 0, st>>>(p, boxes, nboxes);
    else if (storage == FDTD_STORE_BF16)
        slab_e_batch<false, 0, __nv_bfloat16><<<(unsigned)nblocks, 256, 0, st>>>(p, boxes, nboxes);
    else
        slab_e_batch<false, 0, float><<<(unsigned)nblocks, 256, 0, st>>>(p, boxes, nboxes);
    return cudaGetLastError();
}

void launch_nfff_accumulate_batch(const DevNfff *n, int nplans, int max_cells, cudaStream_t st)
{
    if (nplans > 0 && max_cells > 0) nfff_accumulate_batch<<<dim3((max_cells + 255) / 256, nplans), 256, 0, st>>>(n);
}

void launch_nfff_accumulate(const DevNfff &n, cudaStream_t st)
{
    if (n.ns <= 0) return;
    nfff_accumulate_kernel<<<(n.ns + 255) / 256, 256, 0, st>>>(n);
}

void launch_nfff_fold_pending(const DevNfff &n, cudaStream_t st)
{
    if (n.ns <= 0 || n.nfreq <= 0) return;
    nfff_fold_pending_kernel<<<(n.ns + 255) / 256, 256, 0, st>>>(n);
}

void launch_farfield_finalize(const DevFarfield &f, cudaStream_t st)
{
    if (f.npoints <= 0 || f.nfreq <= 0) return;
    const dim3 grid((f.npoints + 127) / 128, f.groups);
    for (int f0 = 0; f0 < f.nfreq; f0 += 4) {
        switch (f.nfreq - f0) {
        case 1: farfield_partial_kernel<1><<<grid, 128, 0, st>>>(f, f0); break;
        case 2: farfield_partial_kernel<2><<<grid, 128, 0, st>>>(f, f0); break;
        case 3: farfield_partial_kernel<3><<<grid, 128, 0, st>>>(f, f0); break;
        default: farfield_partial_kernel<4><<<grid, 128, 0, st>>>(f, f0); break;
        }
    }
    const int nt = f.npoints * f.nfreq * 3;
    farfield_reduce_kernel<<<(nt + 255) / 256, 256, 0, st>>>(f);
}

void launch_nfff_series(const DevNfffSeries &s, cudaStream_t st)
{
    if (s.ns <= 0 || s.npoints <= 0) return;
    const dim3 grid((s.ns + 255) / 256, (unsigned)min(s.npoints, 65535));
    nfff_series_kernel<<<grid, 256, 0, st>>>(s);
}
