// fdtd_bulk.cu -- TMA-staged fused step for the bulk of the grid.
//
// The bulk region is every cell outside the CPML slabs and off the grid's
// edge planes (their H/E updates, psi recursions and zeroed planes are done by
// the slab kernels of fdtd_kernels.cu).  Inside it a step is: ystep_h (yee.c:146-265) + TSF H
// (source.c:1464-1672), then ystep_e with the ADE branch and the PEC rule
// (yee.c:530-1247) + TSF E (source.c:547-771).  kappa is 1 everywhere here and
// no edge test of the reference applies.
//
// A CTA owns 15 x 60 (j,k) cells of every plane of its i-chunk.  Thread
// (r, g), r = tid / 16, g = tid % 16, holds the four consecutive k cells
// k0 - 4 + 4g .. k0 - 1 + 4g of row j0 - 1 + r: the 16 x 64 cells on which H
// is computed are the own cells plus the row and the k group the E update
// needs from its neighbours.  Fields move as 4-vectors (16-byte shared and
// global accesses; 8 bytes at 16-bit storage).  The H row above comes through
// a double-buffered exchange, so that one barrier per plane suffices; the k
// neighbour through a shuffle; the plane below stays in registers, and so
// does E(i+1), which becomes the next plane's own E.  Thread 0 streams the
// planes through a 3-stage shared-memory ring with cp.async.bulk.tensor (TMA)
// two planes ahead: E(p) box 17 rows, H(p) box 16 rows, class bytes 16 rows,
// completion on one mbarrier per stage.  Every wait is bounded; a CTA that
// gives up sets the error word and returns after draining its copies.  The
// dispersive state (Q, E^{n-1}; pole state) is read with plain global loads:
// plane i's at the top of plane i, and plane i+1's lines are prefetched into
// L2 at the same time for the components its staged class word marks.
#include <cuda.h>
#include <cuda_runtime.h>

#include "fdtd_bulk.cuh"
#include "../../include/gsvit_b200.h"
#include "fdtd_device.cuh"

namespace {

constexpr int NTH = 256;
constexpr int TROWS = 16;                 // thread rows: j0-1 .. j0+14
constexpr int TGRP = 16;                  // 4-cell groups per row: k0-4 .. k0+59
static_assert(TROWS * TGRP == NTH, "one thread per 4-cell group");
static_assert(BULK_TJ == TROWS - 1 && BULK_TK == 4 * TGRP - 4, "tile of the host work list");
constexpr int ROWS_E = TROWS + 1, ROWS_H = TROWS, BWC = 80;
constexpr int S = 3;
constexpr int CBOX = ROWS_H * BWC;        // 1280 B
constexpr long long WAIT_LIMIT = 1ll << 22;

// Box geometry per storage type T (elements, k innermost).  Boxes start at
// the column ka = (k0 - 4) rounded down to 16 bytes; the E box reaches the
// k + 1 neighbour of the last group (one group further), the class box is
// 80 bytes from (k0 - 4) rounded down to 16.
template <class T>
struct Geo {
    static constexpr int XAL = 16 / (int)sizeof(T);                    // x alignment (elements)
    static constexpr int BWE = sizeof(T) == 4 ? 68 : 72;
    static constexpr int BWH = sizeof(T) == 4 ? 64 : 72;
    static constexpr int EBOX = ROWS_E * BWE * (int)sizeof(T);          // 4624 / 2448 B
    static constexpr int EBOX_PAD = (EBOX + 127) / 128 * 128;           // 4736 / 2560 B
    static constexpr int HBOX = ROWS_H * BWH * (int)sizeof(T);          // 4096 / 2304 B
    static constexpr int HBOX_PAD = (HBOX + 127) / 128 * 128;
    static constexpr int STAGE = 3 * EBOX_PAD + 3 * HBOX_PAD + CBOX;    // 27776 / 15872 B
    static constexpr uint32_t TX = 3 * EBOX + 3 * HBOX + CBOX;          // bytes the TMA delivers per stage
    static_assert(EBOX_PAD % 128 == 0 && HBOX_PAD % 128 == 0 && CBOX % 128 == 0, "TMA boxes must stay 128-B aligned");
    static_assert((BWE * sizeof(T)) % 16 == 0 && (BWH * sizeof(T)) % 16 == 0, "TMA inner extent");
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait: false when the phase did not complete within the limit
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity)
{
    for (long long it = 0; it < WAIT_LIMIT; it++)
        if (bar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load3(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

template <class T>
__device__ __forceinline__ T *ebox(unsigned char *st, int c) { return reinterpret_cast<T *>(st + c * Geo<T>::EBOX_PAD); }
template <class T>
__device__ __forceinline__ T *hbox(unsigned char *st, int c)
{
    return reinterpret_cast<T *>(st + 3 * Geo<T>::EBOX_PAD + c * Geo<T>::HBOX_PAD);
}
template <class T>
__device__ __forceinline__ unsigned char *cbox(unsigned char *st) { return st + 3 * Geo<T>::EBOX_PAD + 3 * Geo<T>::HBOX_PAD; }

// ------------------------------------------------------------- kernel

// Shared-memory layout: the TMA ring, the class table (ncls_layout entries),
// the H row exchange [2 parities][hx, hz][16 rows][16 groups], one mbarrier
// per stage and the ADE table.
struct BulkSmem {
    unsigned char *stages;
    float4 *scls;
    float4 *xch;
    uint64_t *bars;
    DevAde *sade;
};

constexpr int XCH_BYTES = 2 * 2 * TROWS * TGRP * 16;   // 16 KB

template <class T>
__device__ __forceinline__ BulkSmem bulk_smem(unsigned char *smem, int ncls_layout)
{
    constexpr int SS = S * Geo<T>::STAGE;
    BulkSmem m;
    m.stages = smem;
    m.scls = reinterpret_cast<float4 *>(smem + SS);
    m.xch = reinterpret_cast<float4 *>(smem + SS + ncls_layout * 64);
    m.bars = reinterpret_cast<uint64_t *>(smem + SS + ncls_layout * 64 + XCH_BYTES);
    m.sade = reinterpret_cast<DevAde *>(smem + SS + ncls_layout * 64 + XCH_BYTES + S * 8);
    return m;
}

// class and ADE tables of one plan into shared memory (all threads)
template <bool ADE>
__device__ __forceinline__ void bulk_load_tables(const DevPlan &P, const BulkSmem &m)
{
    for (int q = threadIdx.x; q < P.nclasses * 4; q += NTH) m.scls[q] = reinterpret_cast<const float4 *>(P.classes)[q];
    if (ADE)
        for (int q = threadIdx.x; q < P.nade * (int)(sizeof(DevAde) / 4); q += NTH)
            reinterpret_cast<float *>(m.sade)[q] = reinterpret_cast<const float *>(P.ade)[q];
}

// One work item: the i-march over planes [ib, ie) of one (j,k) tile.  The
// ring's stage of plane p is (gplane + p - p0) % S with phase parity
// ((gplane + p - p0) / S) & 1, gplane counting the planes this CTA has
// streamed in earlier items, so that a persistent CTA keeps its mbarriers.
// Returns false when a bounded wait gave up (after draining its copies).
template <bool ADE, int NPOLES, class T>
__device__ __forceinline__ bool bulk_item(const DevPlan &P, const BulkMaps &M, const BulkItem &it, const BulkSmem &m,
                                          uint32_t &gplane, int *err)
{
    unsigned char *stages = m.stages;
    const float4 *scls = m.scls;
    float4 *xch = m.xch;
    uint64_t *bars = m.bars;
    const DevAde *sade = m.sade;

    const int tid = threadIdx.x, tr = tid >> 4, tg = tid & 15;
    const int j0 = it.j0, k0 = it.k0, ib = it.ib, ie = it.ie;
    const int64_t si = P.si, sj = P.sj;
    constexpr int BWE = Geo<T>::BWE, BWH = Geo<T>::BWH, STAGE = Geo<T>::STAGE;
    const int ka = (k0 - 4) & ~(Geo<T>::XAL - 1), ka8 = (k0 - 4) & ~15;   // box origins (16-byte aligned x)
    const int off = (k0 - 4) - ka, off8 = (k0 - 4) - ka8;
    const int p0 = ib - 1;                  // prologue plane: H of plane ib - 1 (ib >= 1 in the bulk)
    const int plast = ie;                   // E(ie) feeds H of plane ie - 1 (ie <= xres - 1)
    const uint32_t g0 = gplane;
    const uint32_t stp = sr_step<T>(P);     // step number of the BF16 rounding dither

    auto issue = [&](int p) {   // thread 0: all boxes of plane p into its stage
        const int s = (int)((g0 + (uint32_t)(p - p0)) % S);
        unsigned char *st = stages + s * STAGE;
        bar_expect_tx(&bars[s], Geo<T>::TX);
        for (int c = 0; c < 3; c++) tma_load3(ebox<T>(st, c), &M.e[c], ka, j0 - 1, p, &bars[s]);
        for (int c = 0; c < 3; c++) tma_load3(hbox<T>(st, c), &M.h[c], ka, j0 - 1, p, &bars[s]);
        tma_load3(cbox<T>(st), &M.cls, ka8, j0 - 1, p, &bars[s]);
    };
    if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int p = p0; p <= plast && p < p0 + S; p++) issue(p);
    }
    gplane = g0 + (uint32_t)(plast - p0 + 1);     // every plane p0..plast is streamed once
    int issued = min(plast, p0 + S - 1);          // last plane issued (uniform over the CTA)

    // this thread's cells: row j = j0 - 1 + tr, k = kq .. kq + 3
    const int j = j0 - 1 + tr, kq = k0 - 4 + 4 * tg;
    const bool own = tr >= 1 && tg >= 1 && j < it.jhi && kq < it.khi;   // groups are whole (khi - k0 % 4 == 0)
    const int eb = tr * BWE + off + 4 * tg, hb = tr * BWH + off + 4 * tg, cb = tr * BWC + off8 + 4 * tg;
    // TSF: does this thread's group touch a face of the TSF box?  Per plane
    // below: faces i = i0-1, i0, in over the box's (j,k) extent; lateral faces
    // j = j0-1, j0, jn and k = k0-1, k0, kn inside [i0, in].  The per-cell tests
    // are those of tsf_add_h/e.
    bool tifc = false, tlat = false;
    const int ti0 = P.t0[0], tin = P.t1[0];
    if (P.tsf_on) {
        const int tj0 = P.t0[1], tjn = P.t1[1], tk0 = P.t0[2], tkn = P.t1[2], kh = kq + 3;
        const bool jin = j >= tj0 - 1 && j <= tjn, kin = kh >= tk0 - 1 && kq <= tkn;
        const bool jf = j == tj0 - 1 || j == tj0 || j == tjn;
        const bool kf = (kq <= tk0 && kh >= tk0 - 1) || (kq <= tkn && kh >= tkn);
        tifc = jin && kin;
        tlat = (jin && kf) || (kin && jf);
    }

    // per-thread state of the march: E^n of plane i (own group), E(i+1) (read
    // for H, carried as the next plane's E), H^{n+1/2} of planes i and i-1
    float ex[4], ey[4], ez[4], eyi[4], ezi[4], hx[4], hy[4], hz[4], hyim[4], hzim[4];
#pragma unroll
    for (int c = 0; c < 4; c++) hyim[c] = hzim[c] = 0.f;
    bool failed = false;
    for (int i = p0; i < ie; i++) {
        const uint32_t gi = g0 + (uint32_t)(i - p0);
        const int s = (int)(gi % S), s1 = (int)((gi + 1) % S);
        bool ok = bar_wait(&bars[s], (gi / S) & 1u);
        ok = ok && bar_wait(&bars[s1], ((gi + 1) / S) & 1u);
        unsigned char *st = stages + s * STAGE, *st1 = stages + s1 * STAGE;
        const bool prologue = (i < ib);
        const bool act = !prologue && own && ok;     // this thread updates and stores its group
        const uint32_t cw = *reinterpret_cast<const uint32_t *>(cbox<T>(st) + cb);
        const int cl0 = cw & 0xff;
        const bool uni = cw == (uint32_t)cl0 * 0x01010101u;   // one class for the four cells
        const bool tsf_plane = (tifc && (i == ti0 - 1 || i == ti0 || i == tin)) || (tlat && i >= ti0 && i <= tin);
        const int64_t c0i = (int64_t)i * si + (int64_t)j * sj + kq;   // global index of this group's first cell
        // dispersive state of this group, requested before the H phase so that
        // the loads overlap it (Drude: Q and E^{n-1}; the pole state follows in
        // the E phase)
        float aq[3][4], aep[3][4];
        uint32_t adem = 0;   // components with at least one dispersive cell in the group
        if (ADE) {
            if (act) {
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int cl = (cw >> (8 * c)) & 0xff;
                    const uint32_t fl = __float_as_uint(scls[cl * 4].w);
                    if (fl & CF_ADE_BRANCH) adem |= fl & (CF_ADE_X | CF_ADE_Y | CF_ADE_Z);
                    if (uni) break;
                }
            }
#pragma unroll
            for (int a = 0; a < 3; a++) {
                if (adem & (1u << a)) {
                    ldq4a(aq[a], P.q[a] + c0i);
                    ldg4a<T>(aep[a], P.fout[a], c0i);
                }
            }
            // the next plane's dispersive state into L2 (its class word is
            // already staged): under full HBM load the H phase alone does not
            // cover a DRAM round trip, an L2 one it does
            if (own && ok && i + 1 < ie) {
                const uint32_t cwn = *reinterpret_cast<const uint32_t *>(cbox<T>(st1) + cb);
                uint32_t mn = 0;
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const uint32_t fl = __float_as_uint(scls[((cwn >> (8 * c)) & 0xff) * 4].w);
                    if (fl & CF_ADE_BRANCH) mn |= fl & (CF_ADE_X | CF_ADE_Y | CF_ADE_Z);
                }
                const int64_t cn = c0i + si;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    if (mn & (1u << a)) {
                        prefetch_l2(P.q[a] + cn);
                        prefetch_l2(reinterpret_cast<const T *>(P.fout[a]) + cn);
#pragma unroll
                        for (int n = 0; n < NPOLES; n++) { prefetch_l2(P.pc[a][n] + cn); prefetch_l2(P.qc[a][n] + cn); }
                    }
                }
            }
        }
        // ---- H phase: four cells per thread
        {
            const T *EX = ebox<T>(st, 0), *EY = ebox<T>(st, 1), *EZ = ebox<T>(st, 2);
            if (i == p0) { lds4a<T>(ey, EY + eb); lds4a<T>(ez, EZ + eb); }   // later planes: carried E(i+1)
            lds4a<T>(ex, EX + eb);
            float exj[4], ezj[4];
            lds4a<T>(exj, EX + eb + BWE);
            lds4a<T>(ezj, EZ + eb + BWE);
            const float exk4 = lds4<T>(EX + eb + 4).x, eyk4 = lds4<T>(EY + eb + 4).x;
            lds4a<T>(eyi, ebox<T>(st1, 1) + eb);
            lds4a<T>(ezi, ebox<T>(st1, 2) + eb);
            lds4a<T>(hx, hbox<T>(st, 0) + hb);
            lds4a<T>(hy, hbox<T>(st, 1) + hb);
            lds4a<T>(hz, hbox<T>(st, 2) + hb);
            float da[4], db[4];
            {
                const float4 hc = scls[cl0 * 4 + 2];
#pragma unroll
                for (int c = 0; c < 4; c++) { da[c] = hc.x; db[c] = hc.y; }
            }
            if (!uni) {
#pragma unroll
                for (int c = 1; c < 4; c++) {
                    const float4 hc = scls[((cw >> (8 * c)) & 0xff) * 4 + 2];
                    da[c] = hc.x; db[c] = hc.y;
                }
            }
#pragma unroll
            for (int c = 0; c < 4; c++) {
                if (Stor<T>::scaled) { hx[c] *= P.ihs; hy[c] *= P.ihs; hz[c] *= P.ihs; }
                const float eyk = c < 3 ? ey[c + 1] : eyk4, exk = c < 3 ? ex[c + 1] : exk4;
                hx[c] = da[c] * hx[c] + db[c] * ((eyk - ey[c]) - (ezj[c] - ez[c]));
                hy[c] = da[c] * hy[c] + db[c] * ((ezi[c] - ez[c]) - (exk - ex[c]));
                hz[c] = da[c] * hz[c] + db[c] * ((exj[c] - ex[c]) - (eyi[c] - ey[c]));
            }
            if (tsf_plane) {
#pragma unroll
                for (int c = 0; c < 4; c++) tsf_add_h(P, i, j, kq + c, hx[c], hy[c], hz[c]);
            }
            if (act) {
                const float q = Stor<T>::scaled ? P.hs : 1.f;
                stg4a<T>(P.fout[3], c0i, hx, q, stp, 3);
                stg4a<T>(P.fout[4], c0i, hy, q, stp, 4);
                stg4a<T>(P.fout[5], c0i, hz, q, stp, 5);
            }
            const int xb = ((int)(i & 1) * 2 * TROWS + tr) * TGRP + tg;
            xch[xb] = make_float4(hx[0], hx[1], hx[2], hx[3]);
            xch[xb + TROWS * TGRP] = make_float4(hz[0], hz[1], hz[2], hz[3]);
        }
        if (__syncthreads_or(!ok)) { failed = true; break; }
        // stage s is free: every thread has read plane i (here and as plane i+1 before)
        if (i + S <= plast) {
            if (tid == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(i + S);
            }
            issued = i + S;
        }
        // ---- E phase on own cells
        const float hyk0 = __shfl_up_sync(0xffffffffu, hy[3], 1), hxk0 = __shfl_up_sync(0xffffffffu, hx[3], 1);
        if (act) {
            const int xb = ((int)(i & 1) * 2 * TROWS + tr - 1) * TGRP + tg;
            const float4 hxj4 = xch[xb], hzj4 = xch[xb + TROWS * TGRP];
            const float hxj[4] = {hxj4.x, hxj4.y, hxj4.z, hxj4.w}, hzj[4] = {hzj4.x, hzj4.y, hzj4.z, hzj4.w};
            float cu[3][4];   // curl H of the four cells
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float hxk = c ? hx[c - 1] : hxk0, hyk = c ? hy[c - 1] : hyk0;
                cu[0][c] = (hz[c] - hzj[c]) - (hy[c] - hyk);
                cu[1][c] = (hx[c] - hxk) - (hz[c] - hzim[c]);
                cu[2][c] = (hy[c] - hyim[c]) - (hx[c] - hxj[c]);
            }
            const float *eo[3] = {ex, ey, ez};
            float ne[3][4];
            float pq[3][2][4], qq[3][2][4];   // critical-point state p, q (NPOLES > 0)
            if (ADE && NPOLES > 0) {
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int n = 0; n < NPOLES; n++)
                        if (adem & (1u << a)) {
                            ldq4a(pq[a][n], P.pc[a][n] + c0i);
                            ldq4a(qq[a][n], P.qc[a][n] + c0i);
                        }
            }
            const unsigned cm[3] = {CF_ADE_X, CF_ADE_Y, CF_ADE_Z};
            if (uni) {
                // one class: coefficients and branches once for the group
                const float4 c0 = scls[cl0 * 4 + 0], c1 = scls[cl0 * 4 + 1];
                const unsigned fl = __float_as_uint(c0.w);
                const float ca[3] = {c0.x, c0.y, c0.z}, cb[3] = {c1.x, c1.y, c1.z};
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int c = 0; c < 4; c++) ne[a][c] = ca[a] * eo[a][c] + cb[a] * cu[a][c];
                if (ADE && (fl & CF_ADE_BRANCH)) {
                    // ADE branch (yee.c:914-1108) without CPML: only the owned components
                    const DevAde &A = sade[__float_as_int(scls[cl0 * 4 + 2].z)];
                    const float c0dx = A.c0dx, qe = A.qe, c2 = A.c2, c3 = A.c3, ma0 = A.ma0, a2 = A.a2;
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        if (!(fl & cm[a])) continue;
#pragma unroll
                        for (int c = 0; c < 4; c++) {
                            // difference-form state (DevAde); E^{n-1} is the output set before this step writes it
                            const float qd = aq[a][c], ep = aep[a][c], e0 = eo[a][c];
                            float v = c0dx * cu[a][c] + qe * qd;
#pragma unroll
                            for (int n = 0; n < NPOLES; n++) v += A.qpe[n] * qq[a][n][c] + A.pe[n] * pq[a][n][c];
                            v += c2 * ep + c3 * e0;
                            ne[a][c] = v;
                            aq[a][c] = ma0 * qd + a2 * (ep + 2.f * e0 + v);
#pragma unroll
                            for (int n = 0; n < NPOLES; n++) {
                                const float pc = pq[a][n][c], qc = qq[a][n][c];
                                const float qn = A.rp[n] * pc + A.rq[n] * qc + A.bp2[n] * ep + A.bp3[n] * e0 + A.bp4[n] * v;
                                qq[a][n][c] = qn;
                                pq[a][n][c] = pc + qn;
                            }
                        }
                    }
                }
                const unsigned pm[3] = {CF_PEC_X, CF_PEC_Y, CF_PEC_Z};
#pragma unroll
                for (int a = 0; a < 3; a++)
                    if (fl & pm[a])
#pragma unroll
                        for (int c = 0; c < 4; c++) ne[a][c] = 0.f;
            } else {
                // material boundary inside the group: cell by cell
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int cl = (cw >> (8 * c)) & 0xff;
                    const float4 c0 = scls[cl * 4 + 0], c1 = scls[cl * 4 + 1];
                    const unsigned fl = __float_as_uint(c0.w);
                    const float ca[3] = {c0.x, c0.y, c0.z}, cb[3] = {c1.x, c1.y, c1.z};
#pragma unroll
                    for (int a = 0; a < 3; a++) ne[a][c] = ca[a] * eo[a][c] + cb[a] * cu[a][c];
                    if (ADE && (fl & CF_ADE_BRANCH)) {
                        const DevAde &A = sade[__float_as_int(scls[cl * 4 + 2].z)];
#pragma unroll
                        for (int a = 0; a < 3; a++) {
                            if (!(fl & cm[a])) continue;
                            const float qd = aq[a][c], ep = aep[a][c], e0 = eo[a][c];
                            float v = A.c0dx * cu[a][c] + A.qe * qd;
#pragma unroll
                            for (int n = 0; n < NPOLES; n++) v += A.qpe[n] * qq[a][n][c] + A.pe[n] * pq[a][n][c];
                            v += A.c2 * ep + A.c3 * e0;
                            ne[a][c] = v;
                            aq[a][c] = A.ma0 * qd + A.a2 * (ep + 2.f * e0 + v);
#pragma unroll
                            for (int n = 0; n < NPOLES; n++) {
                                const float pc = pq[a][n][c], qc = qq[a][n][c];
                                const float qn = A.rp[n] * pc + A.rq[n] * qc + A.bp2[n] * ep + A.bp3[n] * e0 + A.bp4[n] * v;
                                qq[a][n][c] = qn;
                                pq[a][n][c] = pc + qn;
                            }
                        }
                    }
                    if (fl & CF_PEC_X) ne[0][c] = 0.f;
                    if (fl & CF_PEC_Y) ne[1][c] = 0.f;
                    if (fl & CF_PEC_Z) ne[2][c] = 0.f;
                }
            }
            if (tsf_plane) {
#pragma unroll
                for (int c = 0; c < 4; c++) tsf_add_e(P, i, j, kq + c, ne[0][c], ne[1][c], ne[2][c]);
            }
            stg4a<T>(P.fout[0], c0i, ne[0], 1.f, stp, 0);
            stg4a<T>(P.fout[1], c0i, ne[1], 1.f, stp, 1);
            stg4a<T>(P.fout[2], c0i, ne[2], 1.f, stp, 2);
            if (ADE) {
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
        }
#pragma unroll
        for (int c = 0; c < 4; c++) {
            hyim[c] = hy[c]; hzim[c] = hz[c];
            ey[c] = eyi[c]; ez[c] = ezi[c];
        }
    }
    if (failed) {
        if (tid == 0) {
            atomicExch(err, 1);
            // drain: a bounded wait on the last phase issued into every stage
            for (int p = max(p0, issued - S + 1); p <= issued; p++) {
                const uint32_t gp = g0 + (uint32_t)(p - p0);
                bar_wait(&bars[gp % S], (gp / S) & 1u);
            }
        }
        __syncthreads();
        return false;
    }
    __syncthreads();   // the exchange buffer and the stages are free for the next item
    return true;
}

template <bool ADE, int NPOLES, class T>
__global__ void __launch_bounds__(NTH, 2) bulk_kernel(const __grid_constant__ DevPlan P, const __grid_constant__ BulkMaps M,
                                                      const BulkItem *items, int *err)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const BulkSmem m = bulk_smem<T>(smem, P.nclasses);
    bulk_load_tables<ADE>(P, m);
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) bar_init(&m.bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t gplane = 0;
    const BulkItem it = items[blockIdx.x];
    bulk_item<ADE, NPOLES, T>(P, M, it, m, gplane, err);
}

// Many plans in one persistent launch: CTA b takes items b, b + grid, ...;
// each item names its plan (it.inst) in the per-plan tables of this step's
// parity.  Class and ADE tables are reloaded when the plan changes.
template <bool ADE, int NPOLES, class T>
__global__ void __launch_bounds__(NTH, 2) bulk_kernel_batch(const DevPlan *plans, const BulkMaps *maps,
                                                            const BulkItem *items, int nitems, int ncls_layout, int *err)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const BulkSmem m = bulk_smem<T>(smem, ncls_layout);
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) bar_init(&m.bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    uint32_t gplane = 0;
    int cur = -1;
    for (int n = blockIdx.x; n < nitems; n += gridDim.x) {
        const BulkItem it = items[n];
        const DevPlan &P = plans[it.inst];
        if (it.inst != cur) {
            __syncthreads();            // the previous item's readers of the tables are done
            bulk_load_tables<ADE>(P, m);
            cur = it.inst;
        }
        __syncthreads();
        if (!bulk_item<ADE, NPOLES, T>(P, maps[it.inst], it, m, gplane, err)) return;
    }
}

}  // namespace

size_t bulk_smem_bytes(int nclasses, int storage)
{
    const size_t stage = storage == FDTD_STORE_F32 ? (size_t)Geo<float>::STAGE : (size_t)Geo<__half>::STAGE;
    return S * stage + (size_t)nclasses * 64 + XCH_BYTES + S * 8 + FDTD_MAX_ADE * sizeof(DevAde);
}

template <class T>
cudaError_t configure_t()
{
    const int smem = (int)bulk_smem_bytes(256, sizeof(T) == 4 ? FDTD_STORE_F32 : FDTD_STORE_F16);
    const cudaFuncAttribute A = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(bulk_kernel<false, 0, T>, A, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(bulk_kernel<true, 0, T>, A, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(bulk_kernel<true, 2, T>, A, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(bulk_kernel_batch<false, 0, T>, A, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(bulk_kernel_batch<true, 0, T>, A, smem)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(bulk_kernel_batch<true, 2, T>, A, smem);
}

// every variant accepts the largest layout (256 classes), so that any plan or
// batch may launch it
cudaError_t bulk_configure()
{
    cudaError_t e;
    if ((e = configure_t<float>()) != cudaSuccess) return e;
    if ((e = configure_t<__half>()) != cudaSuccess) return e;
    return configure_t<__nv_bfloat16>();
}

template <class T>
void launch_bulk_t(const DevPlan &p, const BulkMaps &m, const BulkItem *items, int nitems, int *err, bool ade, int npoles,
                   size_t smem, cudaStream_t st)
{
    if (!ade)
        bulk_kernel<false, 0, T><<<nitems, NTH, smem, st>>>(p, m, items, err);
    else if (npoles == 0)
        bulk_kernel<true, 0, T><<<nitems, NTH, smem, st>>>(p, m, items, err);
    else
        bulk_kernel<true, 2, T><<<nitems, NTH, smem, st>>>(p, m, items, err);
}

cudaError_t launch_bulk(const DevPlan &p, const BulkMaps &m, const BulkItem *items, int nitems, int *err, bool ade,
                        int npoles, int storage, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    const size_t smem = bulk_smem_bytes(p.nclasses, storage);
    if (storage == FDTD_STORE_F16) launch_bulk_t<__half>(p, m, items, nitems, err, ade, npoles, smem, st);
    else if (storage == FDTD_STORE_BF16) launch_bulk_t<__nv_bfloat16>(p, m, items, nitems, err, ade, npoles, smem, st);
    else launch_bulk_t<float>(p, m, items, nitems, err, ade, npoles, smem, st);
    return cudaGetLastError();
}

template <class T>
void launch_bulk_batch_t(const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems, int grid,
                         int ncls_layout, int *err, bool ade, int npoles, size_t smem, cudaStream_t st)
{
    if (!ade)
        bulk_kernel_batch<false, 0, T><<<grid, NTH, smem, st>>>(plans, maps, items, nitems, ncls_layout, err);
    else if (npoles == 0)
        bulk_kernel_batch<true, 0, T><<<grid, NTH, smem, st>>>(plans, maps, items, nitems, ncls_layout, err);
    else
        bulk_kernel_batch<true, 2, T><<<grid, NTH, smem, st>>>(plans, maps, items, nitems, ncls_layout, err);
}

cudaError_t launch_bulk_batch(const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems, int grid,
                              int ncls_layout, int *err, bool ade, int npoles, int storage, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    const size_t smem = bulk_smem_bytes(ncls_layout, storage);
    grid = min(grid, nitems);
    if (storage == FDTD_STORE_F16)
        launch_bulk_batch_t<__half>(plans, maps, items, nitems, grid, ncls_layout, err, ade, npoles, smem, st);
    else if (storage == FDTD_STORE_BF16)
        launch_bulk_batch_t<__nv_bfloat16>(plans, maps, items, nitems, grid, ncls_layout, err, ade, npoles, smem, st);
    else
        launch_bulk_batch_t<float>(plans, maps, items, nitems, grid, ncls_layout, err, ade, npoles, smem, st);
    return cudaGetLastError();
}

// Tensor maps of one field set: 3D (k, j, i) boxes of BWE x 17 (E) and
// BWH x 16 (H) elements; class bytes 80 x 16 over a row pitch padded to 16 bytes.
int bulk_make_maps(void *encode_fn, const DevPlan &p, float *const f[6], const uint8_t *cls, int cls_pitch, int storage,
                   BulkMaps *out)
{
    auto enc = reinterpret_cast<CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                             const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                             CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                             CUtensorMapFloatOOBfill)>(encode_fn);
    const cuuint64_t dims[3] = {(cuuint64_t)p.zr, (cuuint64_t)p.yr, (cuuint64_t)p.xr};
    const bool f32 = storage == FDTD_STORE_F32;
    const cuuint64_t es = f32 ? 4 : 2;
    const CUtensorMapDataType dtype = storage == FDTD_STORE_F16    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                      : storage == FDTD_STORE_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                                   : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const cuuint32_t bwe = f32 ? Geo<float>::BWE : Geo<__half>::BWE, bwh = f32 ? Geo<float>::BWH : Geo<__half>::BWH;
    const cuuint64_t strides[2] = {(cuuint64_t)p.zr * es, (cuuint64_t)p.zr * es * (cuuint64_t)p.yr};
    const cuuint32_t estr[3] = {1, 1, 1};
    const cuuint32_t boxe[3] = {bwe, ROWS_E, 1}, boxh[3] = {bwh, ROWS_H, 1}, boxc[3] = {BWC, ROWS_H, 1};
    for (int c = 0; c < 3; c++) {
        if (enc(&out->e[c], dtype, 3, f[c], dims, strides, boxe, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return -1;
        if (enc(&out->h[c], dtype, 3, f[3 + c], dims, strides, boxh, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return -1;
    }
    const cuuint64_t cdims[3] = {(cuuint64_t)p.zr, (cuuint64_t)p.yr, (cuuint64_t)p.xr};
    const cuuint64_t cstr[2] = {(cuuint64_t)cls_pitch, (cuuint64_t)cls_pitch * (cuuint64_t)p.yr};
    if (enc(&out->cls, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void *)cls, cdims, cstr, boxc, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return -1;
    return 0;
}
