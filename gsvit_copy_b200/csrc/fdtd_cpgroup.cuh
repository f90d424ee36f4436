// fdtd_cpgroup.cuh -- the special path of a CPML tile for one 4-cell group
// (four consecutive k cells of row j of plane i, as a thread of the TMA tile
// kernel holds them).
//
// The arithmetic of h_update / e_special (fdtd_cells.cuh) cell by cell, in
// the same operation order, reorganised face by face so that memory moves as
// 4-vectors: one face's psi pair is loaded for the four cells, updated and
// stored before the next face's; the dispersive state of a component is one
// vector per array.  A face of e_special does its first psi update (ADE
// branch, corrections of the components the ADE owns) and its second
// (corrections of the others) together: the two touch disjoint components.
// The z0 correction of Ex, which the reference gates by the z component, is
// the exception: a cell whose ADE owns Ex but not Ez takes it after its
// polarisation recursion and PEC rule, as e_special does.  Faces go x, y, z,
// one per axis (tiles need every grid extent >= both depths + 8); the
// reference's order x0 y0 z0 xn yn zn differs from it only for a corner
// group on faces of both sides, by rounding.  FP32 arithmetic (tiles run
// FP32, FP16 and BF16 storage; no design region).
//
// psi vectors: a face of x or y covers the group whole (its psi rows run over
// all k); a z face is read and written as one vector when its depth is a
// multiple of 4 (the group then lies inside the slab or outside it), else
// cell by cell.  A vector store writes back, for the cells the update skips
// (no psi rule at the cell), the value it loaded: those cells' psi are never
// updated and stay at their initial zero.
#pragma once
#include <cuda_runtime.h>

#include "fdtd_bulk.cuh"
#include "fdtd_cells.cuh"
#include "fdtd_device.cuh"

namespace {

// four psi values at q .. q+3, scaled to FP32 (RO: the read-only path, for
// arrays no thread writes during the launch)
template <class T, bool RO>
__device__ __forceinline__ void psi_ld4(const float *p, int64_t q, bool vec, const bool (&m)[4], float scale, float (&v)[4])
{
    if (vec) {
        const float4 w = RO ? ldg4_ro<T>(p, q) : ldg4<T>(p, q);
        v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
        if constexpr (Stor<T>::scaled) {
#pragma unroll
            for (int c = 0; c < 4; c++) v[c] *= scale;
        }
    } else {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            v[c] = 0.f;
            if (m[c]) v[c] = (RO ? Stor<T>::ldg(p, q + c) : Stor<T>::ld(p, q + c)) * (Stor<T>::scaled ? scale : 1.f);
        }
    }
}

template <class T>
__device__ __forceinline__ void psi_st4(float *p, int64_t q, bool vec, const bool (&m)[4], float scale, const float (&v)[4],
                                        uint32_t stp, uint32_t array)
{
    if (vec) {
        stg4<T>(p, q, make_float4(v[0], v[1], v[2], v[3]), scale, stp, array);
    } else {
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (m[c]) st_any<T>(p, q + c, Stor<T>::scaled ? v[c] * scale : v[c], stp, array);
    }
}

// The psi lines of the faces that hold group (i, j, kq) into L2: psi_E and
// this step's input psi_H, both of which plane i reads.  Issued a plane ahead,
// so that the special path's loads hit L2 rather than DRAM.
template <class T>
__device__ __forceinline__ void cp_prefetch_psi(const DevPlan &P, int i, int j, int kq)
{
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    auto pf = [&](int f, int64_t q) {
        const int64_t b = q * (int64_t)sizeof(T);
        prefetch_l2(reinterpret_cast<const char *>(P.psie[f][0]) + b);
        prefetch_l2(reinterpret_cast<const char *>(P.psie[f][1]) + b);
        prefetch_l2(reinterpret_cast<const char *>(P.psih_in[f][0]) + b);
        prefetch_l2(reinterpret_cast<const char *>(P.psih_in[f][1]) + b);
    };
    if (P.cp_on[X0] && i < P.cp_d[X0]) pf(X0, ((int64_t)i * yr + j) * zr + kq);
    if (P.cp_on[XN] && i >= xr - P.cp_d[XN]) pf(XN, ((int64_t)(i - (xr - P.cp_d[XN])) * yr + j) * zr + kq);
    if (P.cp_on[Y0] && j < P.cp_d[Y0]) pf(Y0, ((int64_t)i * P.cp_d[Y0] + j) * zr + kq);
    if (P.cp_on[YN] && j >= yr - P.cp_d[YN]) pf(YN, ((int64_t)i * P.cp_d[YN] + (j - (yr - P.cp_d[YN]))) * zr + kq);
    if (P.cp_on[Z0] && kq < P.cp_d[Z0]) pf(Z0, ((int64_t)i * yr + j) * P.cp_d[Z0] + kq);
    if (P.cp_on[ZN] && kq + 3 >= zr - P.cp_d[ZN])
        pf(ZN, ((int64_t)i * yr + j) * P.cp_d[ZN] + max(kq - (zr - P.cp_d[ZN]), 0));
}

// H^{n+1/2} of a special group: h_update (special = true) then h_special,
// for the four cells.  d*: the forward E differences of the cells; h: H^n
// (FP32, unscaled) in, H^{n+1/2} out.  `owner` groups write psi_H.
template <int CPF, class T>
__device__ __forceinline__ void cp_h_group(const DevPlan &P, const float4 *scls, uint32_t cw, int i, int j, int kq, bool owner,
                                           bool tsf, const float (&dey_i)[4], const float (&dez_i)[4],
                                           const float (&dex_j)[4], const float (&dez_j)[4], const float (&dex_k)[4],
                                           const float (&dey_k)[4], float (&hx)[4], float (&hy)[4], float (&hz)[4])
{
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    const uint32_t stp = sr_step<T>(P);
    const float ips = P.ips, ps = P.ps;
    const bool il = i == xr - 1, jl = j == yr - 1;
    const bool iin = i >= 1 && i < xr - 1, jin = j >= 1 && j < yr - 1;
    const float ikx = __ldg(P.ikh[0] + i), iky = __ldg(P.ikh[1] + j);
    const float dx = P.dx, idx_ = 1.0f / dx;
    float dbdx[4];
    bool kin[4];
    // 1/kappa of the four cells (kq % 4 == 0, the table is 256-byte aligned)
    const float4 ikz4 = __ldg(reinterpret_cast<const float4 *>(P.ikh[2] + kq));
    const float ikzs[4] = {ikz4.x, ikz4.y, ikz4.z, ikz4.w};
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int k = kq + c;
        const float4 hc = scls[((cw >> (8 * c)) & 0xff) * 4 + 2];
        const float da = hc.x, db = hc.y;
        const float ikz = ikzs[c];
        const bool kl = k == zr - 1;
        kin[c] = k >= 1 && k < zr - 1;
        if (!(jl || kl)) hx[c] = da * hx[c] + db * (dey_k[c] * ikz - dez_j[c] * iky);
        if (!(il || kl)) hy[c] = da * hy[c] + db * (dez_i[c] * ikx - dex_k[c] * ikz);
        if (!(il || jl)) hz[c] = da * hz[c] + db * (dex_j[c] * iky - dey_i[c] * ikx);
        if (tsf && P.tsf_on) tsf_add_h(P, i, j, k, hx[c], hy[c], hz[c]);
        dbdx[c] = db * dx;
    }
    const bool kall = kin[0] && kin[1] && kin[2] && kin[3];
    // x faces: psi[1] <- dey_i (hz -= dbdx psi), psi[0] <- dez_i (hy += dbdx psi)
    auto xface = [&](int f, int pos) {
        const int64_t q = ((int64_t)pos * yr + j) * zr + kq;
        const float bh = __ldg(P.bh[f] + pos), ch = __ldg(P.ch[f] + pos);
        float p0[4], p1[4];
        psi_ld4<T, true>(P.psih_in[f][1], q, true, kin, ips, p1);
        psi_ld4<T, true>(P.psih_in[f][0], q, true, kin, ips, p0);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (!kin[c]) continue;
            const float pzx = bh * p1[c] + ch * dey_i[c] * idx_;
            const float pyx = bh * p0[c] + ch * dez_i[c] * idx_;
            hy[c] += dbdx[c] * pyx;
            hz[c] -= dbdx[c] * pzx;
            p1[c] = pzx;
            p0[c] = pyx;
        }
        if (owner) {
            psi_st4<T>(P.psih_out[f][1], q, kall, kin, ps, p1, stp, 18 + 2 * f + 1);
            psi_st4<T>(P.psih_out[f][0], q, kall, kin, ps, p0, stp, 18 + 2 * f + 0);
        }
    };
    // y faces: psi[0] <- dez_j (hx -= dbdx psi), psi[1] <- dex_j (hz += dbdx psi)
    auto yface = [&](int f, int pos) {
        const int d = P.cp_d[f];
        const int64_t q = ((int64_t)i * d + pos) * zr + kq;
        const float bh = __ldg(P.bh[f] + pos), ch = __ldg(P.ch[f] + pos);
        float p0[4], p1[4];
        psi_ld4<T, true>(P.psih_in[f][0], q, true, kin, ips, p0);
        psi_ld4<T, true>(P.psih_in[f][1], q, true, kin, ips, p1);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (!kin[c]) continue;
            const float pxy = bh * p0[c] + ch * dez_j[c] * idx_;
            const float pzy = bh * p1[c] + ch * dex_j[c] * idx_;
            hx[c] -= dbdx[c] * pxy;
            hz[c] += dbdx[c] * pzy;
            p0[c] = pxy;
            p1[c] = pzy;
        }
        if (owner) {
            psi_st4<T>(P.psih_out[f][0], q, kall, kin, ps, p0, stp, 18 + 2 * f + 0);
            psi_st4<T>(P.psih_out[f][1], q, kall, kin, ps, p1, stp, 18 + 2 * f + 1);
        }
    };
    // z faces: psi[1] <- dex_k (hy -= dbdx psi), psi[0] <- dey_k (hx += dbdx psi);
    // lanes m: the cells of the face's H range, base: the face's first k
    auto zface = [&](int f, int base, const bool (&m)[4]) {
        const int d = P.cp_d[f];
        const bool vec = (d & 3) == 0;
        const int64_t q = ((int64_t)i * yr + j) * d + (kq - base);
        float p0[4], p1[4], bhs[4], chs[4];
        psi_ld4<T, true>(P.psih_in[f][1], q, vec, m, ips, p1);
        psi_ld4<T, true>(P.psih_in[f][0], q, vec, m, ips, p0);
        psi_ld4<float, true>(P.bh[f], kq - base, vec, m, 1.f, bhs);   // profiles of the four cells
        psi_ld4<float, true>(P.ch[f], kq - base, vec, m, 1.f, chs);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (!m[c]) continue;
            const float bh = bhs[c], ch = chs[c];
            const float pyz = bh * p1[c] + ch * dex_k[c] * idx_;
            const float pxz = bh * p0[c] + ch * dey_k[c] * idx_;
            hy[c] -= dbdx[c] * pyz;
            hx[c] += dbdx[c] * pxz;
            p1[c] = pyz;
            p0[c] = pxz;
        }
        if (owner) {
            const bool all = vec && m[0] && m[1] && m[2] && m[3];
            psi_st4<T>(P.psih_out[f][1], q, all, m, ps, p1, stp, 18 + 2 * f + 1);
            psi_st4<T>(P.psih_out[f][0], q, all, m, ps, p0, stp, 18 + 2 * f + 0);
        }
    };
    // one face per axis (tiles need every grid extent >= both depths + 8):
    // x, then y, then z -- boundary_hstep's order x0 y0 z0 xn yn zn except
    // for a corner group on faces of both sides, where the sums differ by
    // rounding only
    bool mz[4], az0 = false, azn = false;
    {
        const int d0 = P.cp_d[Z0], dn = P.cp_d[ZN];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int k = kq + c;
            const bool a0 = P.cp_on[Z0] && k < d0 - 1 && iin && jin;
            const bool an = P.cp_on[ZN] && k >= zr - dn + 1 && k < zr - 1 && iin && jin;
            mz[c] = a0 || an;
            az0 = az0 || a0;
            azn = azn || an;
        }
    }
    if constexpr ((CPF & CPF_X) != 0) {
        if (P.cp_on[X0] && i < P.cp_d[X0] - 1 && jin) xface(X0, i);
        else if (P.cp_on[XN] && i >= xr - P.cp_d[XN] + 1 && i < xr - 1 && jin) xface(XN, i - (xr - P.cp_d[XN]));
    }
    if constexpr ((CPF & CPF_Y) != 0) {
        if (P.cp_on[Y0] && j < P.cp_d[Y0] - 1 && iin) yface(Y0, j);
        else if (P.cp_on[YN] && j >= yr - P.cp_d[YN] + 1 && j < yr - 1 && iin) yface(YN, j - (yr - P.cp_d[YN]));
    }
    if constexpr ((CPF & CPF_Z) != 0) {
        if (az0 || azn) zface(az0 ? Z0 : ZN, az0 ? 0 : zr - P.cp_d[ZN], mz);
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const bool kl = kq + c == zr - 1;
        if ((P.cp_on[XN] && il && jin && kin[c]) || (P.cp_on[YN] && jl && iin && kin[c]) || (P.cp_on[ZN] && kl && iin && jin))
            hx[c] = hy[c] = hz[c] = 0.f;
    }
}

// E^{n+1} of a special group: e_special for the four cells.  e*: E^n; h*:
// H^{n+1/2} of the cells, hxj/hzj of row j-1, hxk0/hyk0 of cell kq-1,
// hyim/hzim of plane i-1.  Writes psi_E and the dispersive state; returns
// the new E in ne (before the store).  adem, aq, aep: the components owned by
// the ADE in some cell of the group and their Q and E^{n-1}, which the caller
// requested before the H phase (the loads then overlap it).
template <int CPF, bool ADE, int NPOLES, class T>
__device__ __forceinline__ void cp_e_group(const DevPlan &P, const float4 *scls, const DevAde *sade, uint32_t cw, int i, int j,
                                           int kq, int64_t c0i, bool tsf, const float (&ex)[4], const float (&ey)[4],
                                           const float (&ez)[4], const float (&hx)[4], const float (&hy)[4],
                                           const float (&hz)[4], const float (&hxj)[4], const float (&hzj)[4], float hxk0,
                                           float hyk0, const float (&hyim)[4], const float (&hzim)[4], uint32_t adem,
                                           float (&aq)[3][4], const float (&aep)[3][4], float (&ne)[3][4])
{
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    const uint32_t stp = sr_step<T>(P);
    const float ipse = P.ipse, pse = P.pse;
    const float dx = P.dx, idx_ = 1.0f / dx;
    const float ikx = __ldg(P.ike[0] + i), iky = __ldg(P.ike[1] + j);
    // backward H differences (the reference's, zero at the lower grid edges)
    auto d_zi = [&](int c) { return i > 0 ? hz[c] - hzim[c] : 0.f; };
    auto d_yi = [&](int c) { return i > 0 ? hy[c] - hyim[c] : 0.f; };
    auto d_zj = [&](int c) { return j > 0 ? hz[c] - hzj[c] : 0.f; };
    auto d_xj = [&](int c) { return j > 0 ? hx[c] - hxj[c] : 0.f; };
    auto d_xk = [&](int c) { return kq + c > 0 ? hx[c] - (c ? hx[c - 1] : hxk0) : 0.f; };
    auto d_yk = [&](int c) { return kq + c > 0 ? hy[c] - (c ? hy[c - 1] : hyk0) : 0.f; };
    auto cls_of = [&](int c) { return (int)((cw >> (8 * c)) & 0xff); };

    bool zero[4];
#pragma unroll
    for (int c = 0; c < 4; c++) zero[c] = (P.cp_on[X0] && i == 0) || (P.cp_on[Y0] && j == 0) || (P.cp_on[Z0] && kq + c == 0);
    // pole state of the owned components (difference form, DevAde)
    float pq[3][2][4], qq[3][2][4];
    if (ADE && NPOLES > 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (!(adem & (1u << a))) continue;
#pragma unroll
            for (int n = 0; n < NPOLES; n++) {
                ldq4a(pq[a][n], P.pc[a][n] + c0i);
                ldq4a(qq[a][n], P.qc[a][n] + c0i);
            }
        }
    }
    // ADE values before the CPML corrections, ordinary update and PEC of the
    // other components
    const float4 ikz4 = __ldg(reinterpret_cast<const float4 *>(P.ike[2] + kq));
    const float ikzs[4] = {ikz4.x, ikz4.y, ikz4.z, ikz4.w};
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int k = kq + c;
        const int cl = cls_of(c);
        const float4 c0 = scls[cl * 4 + 0], c1 = scls[cl * 4 + 1];
        const unsigned fl = __float_as_uint(c0.w);
        const float ikz = ikzs[c];
        const float curl[3] = {d_zj(c) * iky - d_yk(c) * ikz, d_xk(c) * ikz - d_zi(c) * ikx, d_yi(c) * ikx - d_xj(c) * iky};
        const bool gd[3] = {j > 0 && k > 0, i > 0 && k > 0, i > 0 && j > 0};
        const float eo[3] = {ex[c], ey[c], ez[c]};
        const float ca[3] = {c0.x, c0.y, c0.z}, cb[3] = {c1.x, c1.y, c1.z};
        const unsigned cm[3] = {CF_ADE_X, CF_ADE_Y, CF_ADE_Z}, pm[3] = {CF_PEC_X, CF_PEC_Y, CF_PEC_Z};
        const bool branch = ADE && (fl & CF_ADE_BRANCH);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            ne[a][c] = eo[a];
            if (ADE && (fl & cm[a])) {
                if (branch && gd[a]) {
                    const DevAde &A = sade[__float_as_int(scls[cl * 4 + 2].z)];
                    float v = A.c0dx * curl[a] + A.qe * aq[a][c];
#pragma unroll
                    for (int n = 0; n < NPOLES; n++) v += A.qpe[n] * qq[a][n][c] + A.pe[n] * pq[a][n][c];
                    v += A.c2 * aep[a][c] + A.c3 * eo[a];
                    ne[a][c] = v;
                }
            } else {
                if (gd[a]) ne[a][c] = ca[a] * eo[a] + cb[a] * curl[a];
                if (fl & pm[a]) ne[a][c] = 0.f;
            }
        }
    }
    // psi_E face by face (x0 y0 z0 xn yn zn): the first update of the ADE
    // branch with its corrections, then the second with the corrections of
    // the components the ADE does not own (boundary_estep)
    // x faces: psi[0] <- dhz_i, psi[1] <- dhy_i; ny -= dx cb1 psi[0], nz += dx cb2 psi[1]
    auto xface = [&](int f, int pos, bool first_ok) {
        const int64_t q = ((int64_t)pos * yr + j) * zr + kq;
        const float be = __ldg(P.be[f] + pos), ce = __ldg(P.ce[f] + pos);
        bool m[4];
        bool any = false;
#pragma unroll
        for (int c = 0; c < 4; c++) { m[c] = !zero[c] && j > 0 && kq + c > 0; any = any || m[c]; }
        if (!any) return;
        float p0[4], p1[4];
        psi_ld4<T, false>(P.psie[f][0], q, true, m, ipse, p0);
        psi_ld4<T, false>(P.psie[f][1], q, true, m, ipse, p1);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (!m[c]) continue;
            const int cl = cls_of(c);
            const unsigned fl = __float_as_uint(scls[cl * 4].w);
            const float dzi = d_zi(c), dyi = d_yi(c);
            if (ADE && (fl & CF_ADE_BRANCH) && first_ok) {
                p0[c] = be * p0[c] + ce * dzi * idx_;
                p1[c] = be * p1[c] + ce * dyi * idx_;
                if (f == XN) {   // x0 corrections are scaled by cb == 0 (yee.c:577)
                    const float4 c3 = scls[cl * 4 + 3];
                    if (fl & CF_ADE_Y) ne[1][c] -= dx * c3.y * p0[c];
                    if (fl & CF_ADE_Z) ne[2][c] += dx * c3.z * p1[c];
                }
            }
            const float4 c1 = scls[cl * 4 + 1];
            p0[c] = be * p0[c] + ce * dzi * idx_;
            p1[c] = be * p1[c] + ce * dyi * idx_;
            if (!(fl & CF_ADE_Y)) ne[1][c] -= dx * c1.y * p0[c];
            if (!(fl & CF_ADE_Z)) ne[2][c] += dx * c1.z * p1[c];
        }
        psi_st4<T>(P.psie[f][0], q, true, m, pse, p0, stp, 6 + 2 * f + 0);
        psi_st4<T>(P.psie[f][1], q, true, m, pse, p1, stp, 6 + 2 * f + 1);
    };
    // y faces: psi[0] <- dhz_j, psi[1] <- dhx_j; nx += dx cb0 psi[0], nz -= dx cb2 psi[1]
    auto yface = [&](int f, int pos, bool first_ok) {
        const int d = P.cp_d[f];
        const int64_t q = ((int64_t)i * d + pos) * zr + kq;
        const float be = __ldg(P.be[f] + pos), ce = __ldg(P.ce[f] + pos);
        bool m[4];
        bool any = false;
#pragma unroll
        for (int c = 0; c < 4; c++) { m[c] = !zero[c] && i > 0 && kq + c > 0; any = any || m[c]; }
        if (!any) return;
        float p0[4], p1[4];
        psi_ld4<T, false>(P.psie[f][0], q, true, m, ipse, p0);
        psi_ld4<T, false>(P.psie[f][1], q, true, m, ipse, p1);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (!m[c]) continue;
            const int cl = cls_of(c);
            const unsigned fl = __float_as_uint(scls[cl * 4].w);
            const float dzj = d_zj(c), dxj = d_xj(c);
            if (ADE && (fl & CF_ADE_BRANCH) && first_ok) {
                p0[c] = be * p0[c] + ce * dzj * idx_;
                p1[c] = be * p1[c] + ce * dxj * idx_;
                const float4 c3 = scls[cl * 4 + 3];
                if (fl & CF_ADE_X) ne[0][c] += dx * c3.x * p0[c];
                if (fl & CF_ADE_Z) ne[2][c] -= dx * c3.z * p1[c];
            }
            const float4 c1 = scls[cl * 4 + 1];
            p0[c] = be * p0[c] + ce * dzj * idx_;
            p1[c] = be * p1[c] + ce * dxj * idx_;
            if (!(fl & CF_ADE_X)) ne[0][c] += dx * c1.x * p0[c];
            if (!(fl & CF_ADE_Z)) ne[2][c] -= dx * c1.z * p1[c];
        }
        psi_st4<T>(P.psie[f][0], q, true, m, pse, p0, stp, 6 + 2 * f + 0);
        psi_st4<T>(P.psie[f][1], q, true, m, pse, p1, stp, 6 + 2 * f + 1);
    };
    float zdx[4];   // deferred z0 Ex corrections of cells whose ADE owns Ex
    // z faces: psi[1] <- dhx_k, psi[0] <- dhy_k; ny += dx cb1 psi[1], nx -= dx cb0 psi[0]
    // (z0: the nx correction is gated by the z component, as boundary.c:758-759 does);
    // lanes `in`: the cells of the face's E range; base: the face's first k
    auto zface = [&](int f, int base, const bool (&in)[4]) {
        const int d = P.cp_d[f];
        const bool vec = (d & 3) == 0;
        const int64_t q = ((int64_t)i * yr + j) * d + (kq - base);
        bool m[4];
        bool any = false;
#pragma unroll
        for (int c = 0; c < 4; c++) { m[c] = in[c] && !zero[c] && i > 0 && j > 0; any = any || m[c]; }
        if (!any) return;
        float p0[4], p1[4], bes[4], ces[4];
        psi_ld4<T, false>(P.psie[f][1], q, vec, m, ipse, p1);
        psi_ld4<T, false>(P.psie[f][0], q, vec, m, ipse, p0);
        psi_ld4<float, true>(P.be[f], kq - base, vec, m, 1.f, bes);   // profiles of the four cells
        psi_ld4<float, true>(P.ce[f], kq - base, vec, m, 1.f, ces);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (!m[c]) continue;
            const int k = kq + c;
            const int cl = cls_of(c);
            const unsigned fl = __float_as_uint(scls[cl * 4].w);
            const float be = bes[c], ce = ces[c];
            const float dxk = d_xk(c), dyk = d_yk(c);
            if (ADE && (fl & CF_ADE_BRANCH) && (f == ZN || k > 1)) {
                p1[c] = be * p1[c] + ce * dxk * idx_;
                p0[c] = be * p0[c] + ce * dyk * idx_;
                const float4 c3 = scls[cl * 4 + 3];
                if (fl & CF_ADE_Y) ne[1][c] += dx * c3.y * p1[c];
                if (fl & CF_ADE_X) ne[0][c] -= dx * c3.x * p0[c];
            }
            const float4 c1 = scls[cl * 4 + 1];
            p1[c] = be * p1[c] + ce * dxk * idx_;
            p0[c] = be * p0[c] + ce * dyk * idx_;
            if (!(fl & CF_ADE_Y)) ne[1][c] += dx * c1.y * p1[c];
            if (!(fl & (f == Z0 ? CF_ADE_Z : CF_ADE_X))) {
                // z0 gates the Ex correction by the z component: a cell whose
                // ADE owns Ex but not Ez gets it after its recursion and PEC rule
                if (ADE && f == Z0 && (fl & CF_ADE_X)) zdx[c] = dx * c1.x * p0[c];
                else ne[0][c] -= dx * c1.x * p0[c];
            }
        }
        psi_st4<T>(P.psie[f][0], q, vec, m, pse, p0, stp, 6 + 2 * f + 0);
        psi_st4<T>(P.psie[f][1], q, vec, m, pse, p1, stp, 6 + 2 * f + 1);
    };
    // one face per axis, x then y then z (as in cp_h_group)
    bool iz[4], az0 = false, azn = false;
    {
        const int d0 = P.cp_d[Z0], dn = P.cp_d[ZN];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int k = kq + c;
            zdx[c] = 0.f;
            const bool a0 = P.cp_on[Z0] && k >= 1 && k < d0;
            const bool an = P.cp_on[ZN] && k >= zr - dn + 1;
            iz[c] = a0 || an;
            az0 = az0 || a0;
            azn = azn || an;
        }
    }
    if constexpr ((CPF & CPF_X) != 0) {
        if (P.cp_on[X0] && i >= 1 && i < P.cp_d[X0]) xface(X0, i, i > 1);
        else if (P.cp_on[XN] && i >= xr - P.cp_d[XN] + 1) xface(XN, i - (xr - P.cp_d[XN]), true);
    }
    if constexpr ((CPF & CPF_Y) != 0) {
        if (P.cp_on[Y0] && j >= 1 && j < P.cp_d[Y0]) yface(Y0, j, j > 1);
        else if (P.cp_on[YN] && j >= yr - P.cp_d[YN] + 1) yface(YN, j - (yr - P.cp_d[YN]), true);
    }
    if constexpr ((CPF & CPF_Z) != 0) {
        if (az0 || azn) zface(az0 ? Z0 : ZN, az0 ? 0 : zr - P.cp_d[ZN], iz);
    }
    // polarisation recursions of the owned components, their PEC rule
    if (ADE && adem) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int cl = cls_of(c);
            const unsigned fl = __float_as_uint(scls[cl * 4].w);
            if (!(fl & CF_ADE_BRANCH)) continue;
            const DevAde &A = sade[__float_as_int(scls[cl * 4 + 2].z)];
            const float eo[3] = {ex[c], ey[c], ez[c]};
            const unsigned cm[3] = {CF_ADE_X, CF_ADE_Y, CF_ADE_Z}, pm[3] = {CF_PEC_X, CF_PEC_Y, CF_PEC_Z};
#pragma unroll
            for (int a = 0; a < 3; a++) {
                if (!(fl & cm[a])) continue;
                const float e1 = ne[a][c], qd = aq[a][c], ep = aep[a][c];
                aq[a][c] = A.ma0 * qd + A.a2 * (ep + 2.f * eo[a] + e1);
#pragma unroll
                for (int n = 0; n < NPOLES; n++) {
                    const float pc = pq[a][n][c], qc = qq[a][n][c];
                    const float qn = A.rp[n] * pc + A.rq[n] * qc + A.bp2[n] * ep + A.bp3[n] * eo[a] + A.bp4[n] * e1;
                    qq[a][n][c] = qn;
                    pq[a][n][c] = pc + qn;
                }
                if (fl & pm[a]) ne[a][c] = 0.f;
            }
            ne[0][c] -= zdx[c];
        }
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (!(adem & (1u << a))) continue;
            stq4a(P.q[a] + c0i, aq[a]);
#pragma unroll
            for (int n = 0; n < NPOLES; n++) {
                stq4a(P.qc[a][n] + c0i, qq[a][n]);
                stq4a(P.pc[a][n] + c0i, pq[a][n]);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        if (zero[c]) ne[0][c] = ne[1][c] = ne[2][c] = 0.f;
        if (tsf && P.tsf_on) tsf_add_e(P, i, j, kq + c, ne[0][c], ne[1][c], ne[2][c]);
    }
}

}  // namespace
