// fdtd_bulk.cu -- TMA-staged fused step: the bulk of the grid and the CPML tiles.
//
// A step is: ystep_h (yee.c:146-265) + TSF H (source.c:1464-1672), then
// ystep_e with the ADE branch and the PEC rule (yee.c:530-1247) + TSF E
// (source.c:547-771), and, in the CPML tiles, the psi recursions and
// corrections of boundary_hstep / boundary_estep (boundary.c:347-519,
// 691-884), kappa, the zeroed outer planes and the ADE-in-CPML branch
// (yee.c:950-1057).  Every tile does H and E of its cells in one pass over the
// planes: the H values its E update needs from outside the tile (one row, one
// 4-cell group, the plane below) are recomputed from E^n and H^n, so tiles
// never wait for each other and one launch per layout covers its cells.
//
// A CTA owns (TROWS-1) x (4 TGRP-4) (j,k) cells of every plane of its
// i-chunk.  Thread (r, g), r = tid / TGRP, g = tid % TGRP, holds the four
// consecutive k cells k0 - 4 + 4g .. k0 - 1 + 4g of row j0 - 1 + r: the cells
// on which H is computed are the own cells plus the row and the k group the E
// update needs from its neighbours.  Fields move as 4-vectors (16-byte shared
// and global accesses; 8 bytes at 16-bit storage).  The H row above comes
// through a double-buffered exchange, so that one barrier per plane suffices;
// the k neighbour through a shuffle (TGRP divides 32); the plane below stays
// in registers.  Thread 0 streams the planes through a 3-stage shared-memory
// ring with cp.async.bulk.tensor (TMA) two planes ahead: E(p) box TROWS+1
// rows, H(p) box TROWS rows, class bytes TROWS rows, completion on one
// mbarrier per stage; E of planes i and i+1 and H of plane i are read from the
// ring every plane.  Out-of-grid parts of a box (a tile at the grid's edge)
// arrive as zeros.  Every wait is bounded; a CTA that gives up sets the error
// word and returns after draining its copies.  The dispersive state (Q,
// E^{n-1}; pole state) is read with plain global loads: plane i's at the top
// of plane i, and plane i+1's lines are prefetched into L2 at the same time
// for the components its staged class word marks.
//
// In a CPML tile (CP = true) every 4-cell group inside the grid takes the
// special path of fdtd_cpgroup.cuh: h_update with psi_H (written by the owner
// only; halo copies read it) and e_special with psi_E, kappa, ADE-in-CPML,
// PEC and TSF, for the four cells at once with 4-vector psi and state
// traffic.  The CPML kernels carry no plain path: their loop body stays
// small enough for the instruction cache, and on a plain cell the special
// path computes the plain update (kappa 1, no psi, no edge rule).
#include <cuda.h>
#include <cuda_runtime.h>

#include "fdtd_bulk.cuh"
#include "../../include/gsvit_b200.h"
#include "fdtd_cells.cuh"
#include "fdtd_cpgroup.cuh"
#include "fdtd_device.cuh"

namespace {

constexpr int S = 3;                      // TMA ring stages
constexpr long long WAIT_LIMIT = 1ll << 22;

constexpr int rup(int x, int m) { return (x + m - 1) / m * m; }

// thread layout: TR thread rows of TG 4-cell groups
template <int TR, int TG>
struct Lay {
    static constexpr int TROWS = TR, TGRP = TG, NTH = TR * TG;
    static constexpr int ROWS_E = TR + 1, ROWS_H = TR;
    static_assert(32 % TG == 0, "a thread row stays inside one warp");
};
using LBulk = Lay<BULK_TJ + 1, BULK_TK / 4 + 1>;   // 16 x 16
using LXY = Lay<CPXY_TJ + 1, CPXY_TK / 4 + 1>;      // 16 x 16
using LZ = Lay<CPZ_TJ + 1, CPZ_TK / 4 + 1>;         // 32 x 8
// 256 threads each: with two CTAs per SM every thread gets 128 registers
static_assert(LBulk::NTH == 256 && LXY::NTH == 256 && LZ::NTH == 256, "tile layouts");

// Box geometry per storage type T and layout L (elements, k innermost).
// Boxes start at the column ka = (k0 - 4) rounded down to 16 bytes; the E box
// reaches the k + 1 neighbour of the last group, the class box is read as one
// 32-bit word per group from (k0 - 4) rounded down to 16 bytes.
template <class T, class L>
struct Geo {
    static constexpr int XAL = 16 / (int)sizeof(T);                                   // x alignment (elements)
    static constexpr int BWE = sizeof(T) == 4 ? 4 * L::TGRP + 4 : rup(4 * L::TGRP + 5, 8);
    static constexpr int BWH = sizeof(T) == 4 ? 4 * L::TGRP : rup(4 * L::TGRP + 4, 8);
    static constexpr int BWC = rup(4 * L::TGRP + 12, 16);
    static constexpr int EBOX = L::ROWS_E * BWE * (int)sizeof(T);
    static constexpr int EBOX_PAD = rup(EBOX, 128);
    static constexpr int HBOX = L::ROWS_H * BWH * (int)sizeof(T);
    static constexpr int HBOX_PAD = rup(HBOX, 128);
    static constexpr int CBOX = L::ROWS_H * BWC;
    static constexpr int CBOX_PAD = rup(CBOX, 128);
    static constexpr int STAGE = 3 * EBOX_PAD + 3 * HBOX_PAD + CBOX_PAD;
    static constexpr uint32_t TX = 3 * EBOX + 3 * HBOX + CBOX;   // bytes the TMA delivers per stage
    static constexpr int XCH = 2 * 2 * L::NTH * 16;                // H row exchange [parity][hx, hz][thread]
    static_assert((BWE * sizeof(T)) % 16 == 0 && (BWH * sizeof(T)) % 16 == 0 && BWC % 16 == 0, "TMA inner extent");
    static_assert(BWE <= 256 && BWH <= 256 && BWC <= 256 && L::ROWS_E <= 256, "TMA box dimensions");
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

// bounded wait: false when the phase did not complete within `limit` polls
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity, long long limit = WAIT_LIMIT)
{
    for (long long it = 0; it < limit; it++)
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

template <class T, class L>
__device__ __forceinline__ T *ebox(unsigned char *st, int c) { return reinterpret_cast<T *>(st + c * Geo<T, L>::EBOX_PAD); }
template <class T, class L>
__device__ __forceinline__ T *hbox(unsigned char *st, int c)
{
    return reinterpret_cast<T *>(st + 3 * Geo<T, L>::EBOX_PAD + c * Geo<T, L>::HBOX_PAD);
}
template <class T, class L>
__device__ __forceinline__ unsigned char *cbox(unsigned char *st)
{
    return st + 3 * Geo<T, L>::EBOX_PAD + 3 * Geo<T, L>::HBOX_PAD;
}

// ------------------------------------------------------------- kernel

// Shared-memory layout: the TMA ring, the class table (ncls_layout entries),
// the H row exchange [2 parities][hx, hz][threads], S + 1 mbarriers (one per
// stage and one that nothing arrives on, for the stall test) and the ADE table.
struct BulkSmem {
    unsigned char *stages;
    float4 *scls;
    float4 *xch;
    uint64_t *bars;
    DevAde *sade;
};

template <class T, class L>
__device__ __forceinline__ BulkSmem bulk_smem(unsigned char *smem, int ncls_layout)
{
    constexpr int SS = S * Geo<T, L>::STAGE, XCH = Geo<T, L>::XCH;
    BulkSmem m;
    m.stages = smem;
    m.scls = reinterpret_cast<float4 *>(smem + SS);
    m.xch = reinterpret_cast<float4 *>(smem + SS + ncls_layout * 64);
    m.bars = reinterpret_cast<uint64_t *>(smem + SS + ncls_layout * 64 + XCH);
    m.sade = reinterpret_cast<DevAde *>(smem + SS + ncls_layout * 64 + XCH + (S + 1) * 8);
    return m;
}

// class and ADE tables of one plan into shared memory (all threads)
template <bool ADE, class L>
__device__ __forceinline__ void bulk_load_tables(const DevPlan &P, const BulkSmem &m)
{
    for (int q = threadIdx.x; q < P.nclasses * 4; q += L::NTH) m.scls[q] = reinterpret_cast<const float4 *>(P.classes)[q];
    if (ADE)
        for (int q = threadIdx.x; q < P.nade * (int)(sizeof(DevAde) / 4); q += L::NTH)
            reinterpret_cast<float *>(m.sade)[q] = reinterpret_cast<const float *>(P.ade)[q];
}

__device__ __forceinline__ void bulk_init_bars(const BulkSmem &m)
{
    if (threadIdx.x == 0) {
        for (int s = 0; s <= S; s++) bar_init(&m.bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
}

// One work item: the i-march over planes [ib, ie) of one (j,k) tile.  The
// ring's stage of plane p is (gplane + p - p0) % S with phase parity
// ((gplane + p - p0) / S) & 1, gplane counting the planes this CTA has
// streamed in earlier items, so that a persistent CTA keeps its mbarriers.
// Returns false when a bounded wait gave up (after draining its copies).
template <bool ADE, int NPOLES, class T, class L, int CPF>
__device__ __forceinline__ bool bulk_item(const DevPlan &P, const BulkMaps &M, const BulkItem &it, const BulkSmem &m,
                                          uint32_t &gplane, int *err, int stall)
{
    constexpr int TGRP = L::TGRP, TROWS = L::TROWS, NTH = L::NTH;
    constexpr bool CP = CPF != 0;   // a CPML layout; CPF: the faces its tiles can meet (CPF_X | CPF_Y | CPF_Z)
    unsigned char *stages = m.stages;
    const float4 *scls = m.scls;
    float4 *xch = m.xch;
    uint64_t *bars = m.bars;
    const DevAde *sade = m.sade;

    const int tid = threadIdx.x, tr = tid / TGRP, tg = tid % TGRP;
    const int j0 = it.j0, k0 = it.k0, ib = it.ib, ie = it.ie;
    const int64_t si = P.si, sj = P.sj;
    constexpr int BWE = Geo<T, L>::BWE, BWH = Geo<T, L>::BWH, BWC = Geo<T, L>::BWC, STAGE = Geo<T, L>::STAGE;
    const int ka = (k0 - 4) & ~(Geo<T, L>::XAL - 1), ka8 = (k0 - 4) & ~15;   // box origins (16-byte aligned x)
    const int off = (k0 - 4) - ka, off8 = (k0 - 4) - ka8;
    const int p0 = ib - 1;                  // prologue plane: H of plane ib - 1 (out of grid for ib = 0: unused)
    const int plast = ie;                   // E(ie) feeds H of plane ie - 1 (plane xres: zeros)
    const uint32_t g0 = gplane;
    const uint32_t stp = sr_step<T>(P);     // step number of the BF16 rounding dither

    auto issue = [&](int p) {   // thread 0: all boxes of plane p into its stage
        const int s = (int)((g0 + (uint32_t)(p - p0)) % S);
        unsigned char *st = stages + s * STAGE;
        bar_expect_tx(&bars[s], Geo<T, L>::TX);
        for (int c = 0; c < 3; c++) tma_load3(ebox<T, L>(st, c), &M.e[c], ka, j0 - 1, p, &bars[s]);
        for (int c = 0; c < 3; c++) tma_load3(hbox<T, L>(st, c), &M.h[c], ka, j0 - 1, p, &bars[s]);
        tma_load3(cbox<T, L>(st), &M.cls, ka8, j0 - 1, p, &bars[s]);
    };
    if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int p = p0; p <= plast && p < p0 + S; p++) issue(p);
    }
    gplane = g0 + (uint32_t)(plast - p0 + 1);     // every plane p0..plast is streamed once
    int issued = min(plast, p0 + S - 1);          // last plane issued (uniform over the CTA)

    // this thread's cells: row j = j0 - 1 + tr, k = kq .. kq + 3
    const int j = j0 - 1 + tr, kq = k0 - 4 + 4 * tg;
    // groups are whole (klo, khi and k0 are multiples of 4).  A halo row or
    // group that is the grid's first (j = 0, k = 0 .. 3) is owned as well:
    // the E update there reads nothing below it (the backward differences
    // vanish), so a tile starting at j0 = 1 / k0 = 4 also covers row 0 / the
    // first group
    const bool own = (tr >= 1 || j == 0) && (tg >= 1 || kq == 0) && j >= it.jlo && j < it.jhi && kq >= it.klo &&
                     kq < it.khi;
    const int eb = tr * BWE + off + 4 * tg, hb = tr * BWH + off + 4 * tg, cb = tr * BWC + off8 + 4 * tg;
    // CPML tiles: every group inside the grid takes the special path (on a
    // plain cell it computes the plain update: kappa 1, no psi, no edge rule)
    const bool jk_in = j >= 0 && j < P.yr && kq >= 0 && kq < P.zr;
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

    // per-thread state of the march: H^{n+1/2} of plane i-1; E^n of planes i
    // and i+1 and H^n of plane i are read from the staged boxes every plane
    float ex[4], ey[4], ez[4], hx[4], hy[4], hz[4], hyim[4], hzim[4];
#pragma unroll
    for (int c = 0; c < 4; c++) hyim[c] = hzim[c] = 0.f;
    bool failed = false;
    for (int i = p0; i < ie; i++) {
        const uint32_t gi = g0 + (uint32_t)(i - p0);
        const int s = (int)(gi % S), s1 = (int)((gi + 1) % S);
        bool ok = bar_wait(&bars[s], (gi / S) & 1u);
        ok = ok && bar_wait(&bars[s1], ((gi + 1) / S) & 1u);
        if (stall > 0 && i == p0) ok = ok && bar_wait(&bars[S], 0u, stall);   // never completes: the test's expiry
        unsigned char *st = stages + s * STAGE, *st1 = stages + s1 * STAGE;
        const bool prologue = (i < ib);
        const bool act = !prologue && own && ok;     // this thread updates and stores its group
        const bool special = CP && jk_in && i >= 0 && i < P.xr;
        const uint32_t cw = *reinterpret_cast<const uint32_t *>(cbox<T, L>(st) + cb);
        const int cl0 = cw & 0xff;
        // one class for the four cells (and no design cell: those take per-cell
        // coefficients on the cell-by-cell path)
        const bool uni = cw == (uint32_t)cl0 * 0x01010101u && !(P.dcoef && (__float_as_uint(scls[cl0 * 4].w) & CF_DESIGN));
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
                const uint32_t cwn = *reinterpret_cast<const uint32_t *>(cbox<T, L>(st1) + cb);
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
        // the TSF correction entries this group's H and E will take, into L1
        if (tsf_plane && ok) tsf_prefetch_group<float>(P, i, j, kq);
        // CPML tiles: the next plane's psi lines into L2, one request per
        // 128-byte line of a row (the row's first own group and every group
        // on a line boundary)
        if (CP && ok && jk_in && i + 1 < ie && i + 1 < P.xr && i + 1 >= 0 && ((kq & 31) == 0 || tg == 1))
            cp_prefetch_psi<T>(P, i + 1, j, kq);
        // ---- H phase: four cells per thread
        {
            const T *EX = ebox<T, L>(st, 0), *EY = ebox<T, L>(st, 1), *EZ = ebox<T, L>(st, 2);
            lds4a<T>(ex, EX + eb);
            lds4a<T>(ey, EY + eb);
            lds4a<T>(ez, EZ + eb);
            float eyi[4], ezi[4], exj[4], ezj[4];
            lds4a<T>(exj, EX + eb + BWE);
            lds4a<T>(ezj, EZ + eb + BWE);
            const float exk4 = lds4<T>(EX + eb + 4).x, eyk4 = lds4<T>(EY + eb + 4).x;
            lds4a<T>(eyi, ebox<T, L>(st1, 1) + eb);
            lds4a<T>(ezi, ebox<T, L>(st1, 2) + eb);
            lds4a<T>(hx, hbox<T, L>(st, 0) + hb);
            lds4a<T>(hy, hbox<T, L>(st, 1) + hb);
            lds4a<T>(hz, hbox<T, L>(st, 2) + hb);
            if constexpr (!CP) {
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
            } else if (special) {
                // ystep_h with kappa and the edge rules, then psi_H, TSF and the
                // zeroed planes (fdtd_cpgroup.cuh); psi_H is written by the owner
                float dyi[4], dzi[4], dxj[4], dzj[4], dxk[4], dyk[4];
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    if (Stor<T>::scaled) { hx[c] *= P.ihs; hy[c] *= P.ihs; hz[c] *= P.ihs; }
                    const float eyk = c < 3 ? ey[c + 1] : eyk4, exk = c < 3 ? ex[c + 1] : exk4;
                    dyi[c] = eyi[c] - ey[c];
                    dzi[c] = ezi[c] - ez[c];
                    dxj[c] = exj[c] - ex[c];
                    dzj[c] = ezj[c] - ez[c];
                    dxk[c] = exk - ex[c];
                    dyk[c] = eyk - ey[c];
                }
                cp_h_group<CPF, T>(P, scls, cw, i, j, kq, act, tsf_plane, dyi, dzi, dxj, dzj, dxk, dyk, hx, hy, hz);
            }
            if (act) {
                const float q = Stor<T>::scaled ? P.hs : 1.f;
                stg4a<T>(P.fout[3], c0i, hx, q, stp, 3);
                stg4a<T>(P.fout[4], c0i, hy, q, stp, 4);
                stg4a<T>(P.fout[5], c0i, hz, q, stp, 5);
            }
            const int xb = ((int)(i & 1) * 2 * TROWS + tr) * TGRP + tg;
            xch[xb] = make_float4(hx[0], hx[1], hx[2], hx[3]);
            xch[xb + NTH] = make_float4(hz[0], hz[1], hz[2], hz[3]);
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
            // the H row below (a halo row owned at j = 0 reads its own: unused, j - 1 is outside the grid)
            const int xb = ((int)(i & 1) * 2 * TROWS + (tr > 0 ? tr - 1 : 0)) * TGRP + tg;
            const float4 hxj4 = xch[xb], hzj4 = xch[xb + NTH];
            const float hxj[4] = {hxj4.x, hxj4.y, hxj4.z, hxj4.w}, hzj[4] = {hzj4.x, hzj4.y, hzj4.z, hzj4.w};
            const float *eo[3] = {ex, ey, ez};
            float ne[3][4];
            if constexpr (CP) {
                // the general E path (e_special: ADE with its CPML, ordinary
                // update with kappa, PEC, zeroed planes, psi_E, TSF E) by group
                // (an own group lies inside the grid)
                cp_e_group<CPF, ADE, NPOLES, T>(P, scls, sade, cw, i, j, kq, c0i, tsf_plane, ex, ey, ez, hx, hy, hz, hxj, hzj,
                                           hxk0, hyk0, hyim, hzim, adem, aq, aep, ne);
            } else {
                float cu[3][4];   // curl H of the four cells
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const float hxk = c ? hx[c - 1] : hxk0, hyk = c ? hy[c - 1] : hyk0;
                    cu[0][c] = (hz[c] - hzj[c]) - (hy[c] - hyk);
                    cu[1][c] = (hx[c] - hxk) - (hz[c] - hzim[c]);
                    cu[2][c] = (hy[c] - hyim[c]) - (hx[c] - hxj[c]);
                }
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
                    // material boundary inside the group, or a design cell: cell by cell
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const int cl = (cw >> (8 * c)) & 0xff;
                        const float4 c0 = scls[cl * 4 + 0], c1 = scls[cl * 4 + 1];
                        const unsigned fl = __float_as_uint(c0.w);
                        float ca[3] = {c0.x, c0.y, c0.z}, cb[3] = {c1.x, c1.y, c1.z};
                        if (fl & CF_DESIGN) {   // adjoint design region: coefficients per cell (DevPlan::dcoef)
                            const int64_t q = ((int64_t)(i - P.dbox[0]) * (P.dbox[3] - P.dbox[2]) + (j - P.dbox[2])) *
                                                  (P.dbox[5] - P.dbox[4]) + (kq + c - P.dbox[4]);
#pragma unroll
                            for (int a = 0; a < 3; a++) { ca[a] = __ldg(P.dcoef + 6 * q + a); cb[a] = __ldg(P.dcoef + 6 * q + 3 + a); }
                        }
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
            stg4a<T>(P.fout[0], c0i, ne[0], 1.f, stp, 0);
            stg4a<T>(P.fout[1], c0i, ne[1], 1.f, stp, 1);
            stg4a<T>(P.fout[2], c0i, ne[2], 1.f, stp, 2);
        }
#pragma unroll
        for (int c = 0; c < 4; c++) { hyim[c] = hy[c]; hzim[c] = hz[c]; }
    }
    if (failed) {
        if (tid == 0) {
            atomicExch(err, 1);
            // drain: a bounded wait (full limit) on the last phase issued into every stage
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

template <bool ADE, int NPOLES, class T, class L, int CPF>
__global__ void __launch_bounds__(L::NTH, 2) tile_kernel(const __grid_constant__ DevPlan P, const __grid_constant__ BulkMaps M,
                                                         const BulkItem *items, int *err, int stall)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    // an earlier launch of this plan already failed (its fields are void): skip
    if (__syncthreads_or(threadIdx.x == 0 && *(volatile int *)err != 0)) return;
    const BulkSmem m = bulk_smem<T, L>(smem, P.nclasses);
    bulk_load_tables<ADE, L>(P, m);
    bulk_init_bars(m);
    __syncthreads();
    uint32_t gplane = 0;
    const BulkItem it = items[blockIdx.x];
    bulk_item<ADE, NPOLES, T, L, CPF>(P, M, it, m, gplane, err, stall);
}

// The tiles of many plans, one CTA per item: each item names its plan (it.inst)
// in the per-plan tables of this step's parity.
template <bool ADE, int NPOLES, class T, class L, int CPF>
__global__ void __launch_bounds__(L::NTH, 2) tile_kernel_batch(const DevPlan *plans, const BulkMaps *maps,
                                                               const BulkItem *items, int ncls_layout, int *err)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    if (__syncthreads_or(threadIdx.x == 0 && *(volatile int *)err != 0)) return;
    const BulkItem it = items[blockIdx.x];
    const DevPlan &P = plans[it.inst];
    const BulkSmem m = bulk_smem<T, L>(smem, ncls_layout);
    bulk_load_tables<ADE, L>(P, m);
    bulk_init_bars(m);
    __syncthreads();
    uint32_t gplane = 0;
    bulk_item<ADE, NPOLES, T, L, CPF>(P, maps[it.inst], it, m, gplane, err, 0);
}

// Many plans in one persistent launch (bulk layout): CTA b takes items b,
// b + grid, ...; each item names its plan (it.inst) in the per-plan tables of
// this step's parity.  Class and ADE tables are reloaded when the plan changes.
template <bool ADE, int NPOLES, class T>
__global__ void __launch_bounds__(LBulk::NTH, 2) bulk_kernel_batch(const DevPlan *plans, const BulkMaps *maps,
                                                                   const BulkItem *items, int nitems, int ncls_layout, int *err)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const BulkSmem m = bulk_smem<T, LBulk>(smem, ncls_layout);
    bulk_init_bars(m);
    uint32_t gplane = 0;
    int cur = -1;
    for (int n = blockIdx.x; n < nitems; n += gridDim.x) {
        const BulkItem it = items[n];
        const DevPlan &P = plans[it.inst];
        if (it.inst != cur) {
            __syncthreads();            // the previous item's readers of the tables are done
            bulk_load_tables<ADE, LBulk>(P, m);
            cur = it.inst;
        }
        __syncthreads();
        if (!bulk_item<ADE, NPOLES, T, LBulk, 0>(P, maps[it.inst], it, m, gplane, err, 0)) return;
    }
}

template <class T, class L>
constexpr size_t smem_bytes_t(int nclasses)
{
    return (size_t)S * Geo<T, L>::STAGE + (size_t)nclasses * 64 + Geo<T, L>::XCH + (S + 1) * 8 + FDTD_MAX_ADE * sizeof(DevAde);
}

template <class L>
size_t smem_bytes_l(int nclasses, int storage)
{
    return storage == FDTD_STORE_F32 ? smem_bytes_t<float, L>(nclasses) : smem_bytes_t<__half, L>(nclasses);
}

template <class T, class L, int CPF>
cudaError_t configure_tl()
{
    const int smem = (int)smem_bytes_t<T, L>(256);
    const cudaFuncAttribute A = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(tile_kernel<false, 0, T, L, CPF>, A, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(tile_kernel<true, 0, T, L, CPF>, A, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(tile_kernel<true, 2, T, L, CPF>, A, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(tile_kernel_batch<false, 0, T, L, CPF>, A, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(tile_kernel_batch<true, 0, T, L, CPF>, A, smem)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(tile_kernel_batch<true, 2, T, L, CPF>, A, smem);
}

template <class T>
cudaError_t configure_t()
{
    cudaError_t e;
    if ((e = configure_tl<T, LBulk, 0>()) != cudaSuccess) return e;
    if ((e = configure_tl<T, LXY, CPF_X | CPF_Y | CPF_Z>()) != cudaSuccess) return e;
    if ((e = configure_tl<T, LXY, CPF_Y | CPF_Z>()) != cudaSuccess) return e;
    if ((e = configure_tl<T, LZ, CPF_Z>()) != cudaSuccess) return e;
    const int smem = (int)smem_bytes_t<T, LBulk>(256);
    const cudaFuncAttribute A = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if ((e = cudaFuncSetAttribute(bulk_kernel_batch<false, 0, T>, A, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(bulk_kernel_batch<true, 0, T>, A, smem)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(bulk_kernel_batch<true, 2, T>, A, smem);
}

template <class T, class L, int CPF>
void launch_tl(const DevPlan &p, const BulkMaps &m, const BulkItem *items, int nitems, int *err, bool ade, int npoles,
               int stall, cudaStream_t st)
{
    const size_t smem = smem_bytes_t<T, L>(p.nclasses);
    if (!ade)
        tile_kernel<false, 0, T, L, CPF><<<nitems, L::NTH, smem, st>>>(p, m, items, err, stall);
    else if (npoles == 0)
        tile_kernel<true, 0, T, L, CPF><<<nitems, L::NTH, smem, st>>>(p, m, items, err, stall);
    else
        tile_kernel<true, 2, T, L, CPF><<<nitems, L::NTH, smem, st>>>(p, m, items, err, stall);
}

template <class T>
void launch_t(int kind, const DevPlan &p, const BulkMaps &m, const BulkItem *items, int nitems, int *err, bool ade,
              int npoles, int stall, cudaStream_t st)
{
    if (kind == TILE_CPX) launch_tl<T, LXY, CPF_X | CPF_Y | CPF_Z>(p, m, items, nitems, err, ade, npoles, stall, st);
    else if (kind == TILE_CPY) launch_tl<T, LXY, CPF_Y | CPF_Z>(p, m, items, nitems, err, ade, npoles, stall, st);
    else if (kind == TILE_CPZ) launch_tl<T, LZ, CPF_Z>(p, m, items, nitems, err, ade, npoles, stall, st);
    else launch_tl<T, LBulk, 0>(p, m, items, nitems, err, ade, npoles, stall, st);
}

template <class T, class L, int CPF>
void launch_tlb(const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems, int ncls_layout, int *err,
                bool ade, int npoles, cudaStream_t st)
{
    const size_t smem = smem_bytes_t<T, L>(ncls_layout);
    if (!ade)
        tile_kernel_batch<false, 0, T, L, CPF><<<nitems, L::NTH, smem, st>>>(plans, maps, items, ncls_layout, err);
    else if (npoles == 0)
        tile_kernel_batch<true, 0, T, L, CPF><<<nitems, L::NTH, smem, st>>>(plans, maps, items, ncls_layout, err);
    else
        tile_kernel_batch<true, 2, T, L, CPF><<<nitems, L::NTH, smem, st>>>(plans, maps, items, ncls_layout, err);
}

template <class T>
void launch_tb(int kind, const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems, int ncls_layout,
               int *err, bool ade, int npoles, cudaStream_t st)
{
    if (kind == TILE_CPX) launch_tlb<T, LXY, CPF_X | CPF_Y | CPF_Z>(plans, maps, items, nitems, ncls_layout, err, ade, npoles, st);
    else if (kind == TILE_CPY) launch_tlb<T, LXY, CPF_Y | CPF_Z>(plans, maps, items, nitems, ncls_layout, err, ade, npoles, st);
    else if (kind == TILE_CPZ) launch_tlb<T, LZ, CPF_Z>(plans, maps, items, nitems, ncls_layout, err, ade, npoles, st);
    else launch_tlb<T, LBulk, 0>(plans, maps, items, nitems, ncls_layout, err, ade, npoles, st);
}

template <class T>
void launch_bulk_batch_t(const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems, int grid,
                         int ncls_layout, int *err, bool ade, int npoles, size_t smem, cudaStream_t st)
{
    if (!ade)
        bulk_kernel_batch<false, 0, T><<<grid, LBulk::NTH, smem, st>>>(plans, maps, items, nitems, ncls_layout, err);
    else if (npoles == 0)
        bulk_kernel_batch<true, 0, T><<<grid, LBulk::NTH, smem, st>>>(plans, maps, items, nitems, ncls_layout, err);
    else
        bulk_kernel_batch<true, 2, T><<<grid, LBulk::NTH, smem, st>>>(plans, maps, items, nitems, ncls_layout, err);
}

// box shapes (elements) of one layout at one storage type
template <class L>
void box_shape(int storage, cuuint32_t *bwe, cuuint32_t *bwh, cuuint32_t *bwc, cuuint32_t *rows_e, cuuint32_t *rows_h)
{
    if (storage == FDTD_STORE_F32) { *bwe = Geo<float, L>::BWE; *bwh = Geo<float, L>::BWH; *bwc = Geo<float, L>::BWC; }
    else { *bwe = Geo<__half, L>::BWE; *bwh = Geo<__half, L>::BWH; *bwc = Geo<__half, L>::BWC; }
    *rows_e = L::ROWS_E;
    *rows_h = L::ROWS_H;
}

}  // namespace

size_t tile_smem_bytes(int kind, int nclasses, int storage)
{
    if (kind == TILE_CPX || kind == TILE_CPY) return smem_bytes_l<LXY>(nclasses, storage);
    if (kind == TILE_CPZ) return smem_bytes_l<LZ>(nclasses, storage);
    return smem_bytes_l<LBulk>(nclasses, storage);
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

cudaError_t launch_tiles(int kind, const DevPlan &p, const BulkMaps &m, const BulkItem *items, int nitems, int *err,
                         bool ade, int npoles, int storage, int stall, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    if (storage == FDTD_STORE_F16) launch_t<__half>(kind, p, m, items, nitems, err, ade, npoles, stall, st);
    else if (storage == FDTD_STORE_BF16) launch_t<__nv_bfloat16>(kind, p, m, items, nitems, err, ade, npoles, stall, st);
    else launch_t<float>(kind, p, m, items, nitems, err, ade, npoles, stall, st);
    return cudaGetLastError();
}

cudaError_t launch_tiles_batch(int kind, const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems,
                               int ncls_layout, int *err, bool ade, int npoles, int storage, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    if (storage == FDTD_STORE_F16) launch_tb<__half>(kind, plans, maps, items, nitems, ncls_layout, err, ade, npoles, st);
    else if (storage == FDTD_STORE_BF16)
        launch_tb<__nv_bfloat16>(kind, plans, maps, items, nitems, ncls_layout, err, ade, npoles, st);
    else launch_tb<float>(kind, plans, maps, items, nitems, ncls_layout, err, ade, npoles, st);
    return cudaGetLastError();
}

cudaError_t launch_bulk_batch(const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems, int grid,
                              int ncls_layout, int *err, bool ade, int npoles, int storage, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    const size_t smem = tile_smem_bytes(TILE_BULK, ncls_layout, storage);
    grid = min(grid, nitems);
    if (storage == FDTD_STORE_F16)
        launch_bulk_batch_t<__half>(plans, maps, items, nitems, grid, ncls_layout, err, ade, npoles, smem, st);
    else if (storage == FDTD_STORE_BF16)
        launch_bulk_batch_t<__nv_bfloat16>(plans, maps, items, nitems, grid, ncls_layout, err, ade, npoles, smem, st);
    else
        launch_bulk_batch_t<float>(plans, maps, items, nitems, grid, ncls_layout, err, ade, npoles, smem, st);
    return cudaGetLastError();
}

// Tensor maps of one field set for one layout: 3D (k, j, i) boxes of
// BWE x (TROWS+1) (E) and BWH x TROWS (H) elements; class bytes BWC x TROWS
// over a row pitch padded to 16 bytes.
int tile_make_maps(int kind, void *encode_fn, const DevPlan &p, float *const f[6], const uint8_t *cls, int cls_pitch,
                   int storage, BulkMaps *out)
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
    cuuint32_t bwe, bwh, bwc, rows_e, rows_h;
    if (kind == TILE_CPX || kind == TILE_CPY) box_shape<LXY>(storage, &bwe, &bwh, &bwc, &rows_e, &rows_h);
    else if (kind == TILE_CPZ) box_shape<LZ>(storage, &bwe, &bwh, &bwc, &rows_e, &rows_h);
    else box_shape<LBulk>(storage, &bwe, &bwh, &bwc, &rows_e, &rows_h);
    const cuuint64_t strides[2] = {(cuuint64_t)p.zr * es, (cuuint64_t)p.zr * es * (cuuint64_t)p.yr};
    const cuuint32_t estr[3] = {1, 1, 1};
    const cuuint32_t boxe[3] = {bwe, rows_e, 1}, boxh[3] = {bwh, rows_h, 1}, boxc[3] = {bwc, rows_h, 1};
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
