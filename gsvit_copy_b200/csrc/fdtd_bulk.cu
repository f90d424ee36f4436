// fdtd_bulk.cu -- TMA-staged fused step for the bulk of the grid.
//
// The bulk region is every cell outside the CPML slabs (their H/E updates,
// psi recursions and zeroed planes are done by the general kernel).  Inside
// it a step is: ystep_h (yee.c:146-265) + TSF H (source.c:1464-1672), then
// ystep_e with the ADE branch and the PEC rule (yee.c:530-1247) + TSF E
// (source.c:547-771).  kappa is 1 everywhere here.
//
// A CTA owns 31 x 31 (j,k) cells of every plane of its i-chunk.  Its 8 warps
// compute H on the 32 x 32 cells [j0-1, j0+31) x [k0-1, k0+31) -- the own
// cells plus the row and column the E update needs from its neighbours --
// with warp w on rows 4w..4w+3 and lane = column, then E on the own cells.
// Thread 0 streams the planes through a 3-stage shared-memory ring with
// cp.async.bulk.tensor (TMA) two planes ahead: E(p) box 36 x 33, H(p) box
// 36 x 32 (floats, k innermost) and the class byte box 48 x 32, completion
// on one mbarrier per stage.  Every wait is bounded; a CTA that gives up sets
// the error word and returns after draining its copies.
#include <cuda.h>
#include <cuda_runtime.h>

#include "fdtd_bulk.cuh"
#include "../../include/gsvit_b200.h"
#include "fdtd_device.cuh"

namespace {

// Box geometry per storage type T: E boxes BW x 33 and H boxes BW x 32
// elements (k innermost) from the aligned column ka <= k0 - 1, the class byte
// box 48 x 32 from ka8.  TMA needs the box start x and the inner box extent in
// multiples of 16 bytes: 4 floats / 8 16-bit elements.
constexpr int BROWS_E = 33, BROWS_H = 32, BWC = 48;
constexpr int S = 3;
constexpr int CBOX = BROWS_H * BWC;                        // 1536 B
template <class T>
struct Geo {
    static constexpr int XAL = 16 / (int)sizeof(T);                        // x alignment (elements)
    static constexpr int BW = sizeof(T) == 4 ? 36 : 40;                     // box width (elements)
    static constexpr int EBOX = BROWS_E * BW * (int)sizeof(T);              // 4752 / 2640 B
    static constexpr int EBOX_PAD = (EBOX + 127) / 128 * 128;               // 4864 / 2688 B
    static constexpr int HBOX = BROWS_H * BW * (int)sizeof(T);              // 4608 / 2560 B
    static constexpr int STAGE = 3 * EBOX_PAD + 3 * HBOX + CBOX;           // 29952 / 17280 B
    static constexpr uint32_t TX = 3 * EBOX + 3 * HBOX + CBOX;             // bytes the TMA delivers per stage
    static_assert(EBOX_PAD % 128 == 0 && HBOX % 128 == 0 && CBOX % 128 == 0, "TMA boxes must stay 128-B aligned");
};
constexpr int NTH = 256;
constexpr long long WAIT_LIMIT = 1ll << 22;


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
    return reinterpret_cast<T *>(st + 3 * Geo<T>::EBOX_PAD + c * Geo<T>::HBOX);
}
template <class T>
__device__ __forceinline__ unsigned char *cbox(unsigned char *st) { return st + 3 * Geo<T>::EBOX_PAD + 3 * Geo<T>::HBOX; }

// ------------------------------------------------------------- kernel

// Shared-memory layout: the TMA ring, the class table (ncls_layout entries),
// the row exchange of H between warps, one mbarrier per stage and the ADE table.
struct BulkSmem {
    unsigned char *stages;
    float4 *scls;
    float *hrow;        // [8][2][32]
    uint64_t *bars;
    DevAde *sade;
};

template <class T>
__device__ __forceinline__ BulkSmem bulk_smem(unsigned char *smem, int ncls_layout)
{
    constexpr int SS = S * Geo<T>::STAGE;
    BulkSmem m;
    m.stages = smem;
    m.scls = reinterpret_cast<float4 *>(smem + SS);
    m.hrow = reinterpret_cast<float *>(smem + SS + ncls_layout * 64);
    m.bars = reinterpret_cast<uint64_t *>(smem + SS + ncls_layout * 64 + 8 * 2 * 32 * 4);
    m.sade = reinterpret_cast<DevAde *>(smem + SS + ncls_layout * 64 + 8 * 2 * 32 * 4 + S * 8);
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
    float *hrow = m.hrow;
    uint64_t *bars = m.bars;
    const DevAde *sade = m.sade;

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int j0 = it.j0, k0 = it.k0, ib = it.ib, ie = it.ie;
    const int xr = P.xr, yr = P.yr, zr = P.zr;
    const int64_t si = P.si, sj = P.sj;
    constexpr int BW = Geo<T>::BW, STAGE = Geo<T>::STAGE;
    const int ka = (k0 - 1) & ~(Geo<T>::XAL - 1), ka8 = (k0 - 1) & ~15;   // box origins (16-byte aligned x)
    const int off = (k0 - 1) - ka, off8 = (k0 - 1) - ka8;
    const int p0 = (ib > 0) ? ib - 1 : ib;                    // first plane (prologue H when ib > 0)
    const int plast = min(ie, xr - 1);                        // last plane whose data is needed
    const uint32_t g0 = gplane;
    const uint32_t stp = sr_step<T>(P);           // step number of the BF16 rounding dither

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

    // this thread's cells: rows rr = 4w + r (row 0 = j0-1), column lane (k = k0-1+lane)
    const int k = k0 - 1 + lane;
    const int ce = off + lane, ce8 = off8 + lane;
    const bool kown = lane >= 1 && k < it.khi;
    int jr[4];
    bool own[4];
    for (int r = 0; r < 4; r++) {
        jr[r] = j0 - 1 + 4 * w + r;
        own[r] = kown && (4 * w + r) >= 1 && jr[r] < it.jhi;
    }
    // TSF face membership by axis (source.c box faces)
    const bool tsf = P.tsf_on != 0;

    float e[4][3], h[4][3], him[4][2];
    for (int r = 0; r < 4; r++) {
        him[r][0] = him[r][1] = 0.f;
        for (int a = 0; a < 3; a++) { e[r][a] = 0.f; h[r][a] = 0.f; }
    }
    bool failed = false;
    for (int i = p0; i <= plast && i < ie; i++) {
        const uint32_t gi = g0 + (uint32_t)(i - p0);
        const int s = (int)(gi % S);
        const uint32_t par = (gi / S) & 1u;
        const bool have_next = (i + 1 <= plast);
        const int s1 = (int)((gi + 1) % S);
        const uint32_t par1 = ((gi + 1) / S) & 1u;
        bool ok = bar_wait(&bars[s], par);
        if (have_next) ok = ok && bar_wait(&bars[s1], par1);
        if (__syncthreads_or(!ok)) { failed = true; break; }
        unsigned char *st = stages + s * STAGE, *st1 = stages + s1 * STAGE;
        const T *EX = ebox<T>(st, 0), *EY = ebox<T>(st, 1), *EZ = ebox<T>(st, 2);
        const T *HX = hbox<T>(st, 0), *HY = hbox<T>(st, 1), *HZ = hbox<T>(st, 2);
        const unsigned char *CL = cbox<T>(st);
        const T *EY1 = ebox<T>(st1, 1), *EZ1 = ebox<T>(st1, 2);
        auto cv = [](T v) { return Stor<T>::cvt(v); };
        const float ihs = Stor<T>::scaled ? P.ihs : 1.f;
        const bool prologue = (i < ib);
        const bool il = (i == xr - 1);
        // Drude state of this plane's own cells (Q and E^{n-1}), requested before
        // the H phase so that the loads overlap it
        float aq[4][3], aep[4][3];
        if (ADE && NPOLES == 0) {
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const unsigned fl = (!prologue && own[r]) ? __float_as_uint(scls[CL[(4 * w + r) * BWC + ce8] * 4].w) : 0u;
                const int64_t c = (int64_t)i * si + (int64_t)jr[r] * sj + k;
                const unsigned cm[3] = {CF_ADE_X, CF_ADE_Y, CF_ADE_Z};
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const bool need = (fl & CF_ADE_BRANCH) && (fl & cm[a]);
                    aq[r][a] = need ? P.q[a][c] : 0.f;
                    aep[r][a] = need ? ldE<T>(P.fout[a], c) : 0.f;
                }
            }
        }
        // ---- H phase: 4 cells per thread
        for (int r = 0; r < 4; r++) {
            const int rr = 4 * w + r, j = jr[r];
            const int b = rr * BW + ce;
            const float ex = cv(EX[b]), ey = cv(EY[b]), ez = cv(EZ[b]);
            e[r][0] = ex; e[r][1] = ey; e[r][2] = ez;
            const float exj = cv(EX[b + BW]), ezj = cv(EZ[b + BW]);
            const float exk = cv(EX[b + 1]), eyk = cv(EY[b + 1]);
            const float eyi = have_next ? cv(EY1[b]) : 0.f, ezi = have_next ? cv(EZ1[b]) : 0.f;
            const int cl = CL[rr * BWC + ce8];
            const float4 hc = scls[cl * 4 + 2];
            float hx = cv(HX[b]), hy = cv(HY[b]), hz = cv(HZ[b]);
            if (Stor<T>::scaled) { hx *= ihs; hy *= ihs; hz *= ihs; }
            const bool jl = (j == yr - 1), kl = (k == zr - 1);
            if (!(jl || kl)) hx = hc.x * hx + hc.y * ((eyk - ey) - (ezj - ez));
            if (!(il || kl)) hy = hc.x * hy + hc.y * ((ezi - ez) - (exk - ex));
            if (!(il || jl)) hz = hc.x * hz + hc.y * ((exj - ex) - (eyi - ey));
            if (tsf) tsf_add_h(P, i, j, k, hx, hy, hz);
            h[r][0] = hx; h[r][1] = hy; h[r][2] = hz;
            if (!prologue && own[r]) {
                const int64_t c = (int64_t)i * si + (int64_t)j * sj + k;
                stH<T>(P, P.fout[3], c, hx, stp, 3);
                stH<T>(P, P.fout[4], c, hy, stp, 4);
                stH<T>(P, P.fout[5], c, hz, stp, 5);
            }
        }
        if (!prologue) {
            hrow[(w * 2 + 0) * 32 + lane] = h[3][2];
            hrow[(w * 2 + 1) * 32 + lane] = h[3][0];
        }
        __syncthreads();
        // ---- E phase on own cells
        if (!prologue) {
            float hyk[4], hxk[4];
            for (int r = 0; r < 4; r++) {
                hyk[r] = __shfl_up_sync(0xffffffffu, h[r][1], 1);
                hxk[r] = __shfl_up_sync(0xffffffffu, h[r][0], 1);
            }
            for (int r = 0; r < 4; r++) {
                if (!own[r]) continue;
                const int rr = 4 * w + r, j = jr[r];
                const float hzj = r ? h[r - 1][2] : hrow[((w - 1) * 2 + 0) * 32 + lane];
                const float hxj = r ? h[r - 1][0] : hrow[((w - 1) * 2 + 1) * 32 + lane];
                const int cl = CL[rr * BWC + ce8];
                const float4 c0 = scls[cl * 4 + 0], c1 = scls[cl * 4 + 1];
                const unsigned fl = __float_as_uint(c0.w);
                const float curlx = (h[r][2] - hzj) - (h[r][1] - hyk[r]);
                const float curly = (h[r][0] - hxk[r]) - (h[r][2] - him[r][1]);
                const float curlz = (h[r][1] - him[r][0]) - (h[r][0] - hxj);
                const bool gx = (j > 0 && k > 0), gy = (i > 0 && k > 0), gz = (i > 0 && j > 0);
                float nx = e[r][0], ny = e[r][1], nz = e[r][2];
                const int64_t c = (int64_t)i * si + (int64_t)j * sj + k;
                if (ADE && (fl & CF_ADE_BRANCH)) {
                    // ADE branch (yee.c:914-1108) without CPML: only the owned components
                    const DevAde &A = sade[__float_as_int(scls[cl * 4 + 2].z)];
                    const float curl[3] = {curlx, curly, curlz};
                    const bool gd[3] = {gx, gy, gz};
                    const unsigned cm[3] = {CF_ADE_X, CF_ADE_Y, CF_ADE_Z};
                    float ne[3] = {nx, ny, nz};
                    for (int a = 0; a < 3; a++) {
                        if (!(fl & cm[a])) continue;
                        const float eo = e[r][a];
                        // difference-form state (DevAde); E^{n-1} is the output set before this step writes it
                        const float qd = (NPOLES == 0) ? aq[r][a] : P.q[a][c], ep = (NPOLES == 0) ? aep[r][a] : ldE<T>(P.fout[a], c);
                        float pc[2] = {0.f, 0.f}, qc[2] = {0.f, 0.f};
                        for (int n = 0; n < NPOLES; n++) { pc[n] = P.pc[a][n][c]; qc[n] = P.qc[a][n][c]; }
                        float v = eo;
                        if (gd[a]) {
                            v = A.c0dx * curl[a] + A.qe * qd;
                            for (int n = 0; n < NPOLES; n++) v += A.qpe[n] * qc[n] + A.pe[n] * pc[n];
                            v += A.c2 * ep + A.c3 * eo;
                        }
                        ne[a] = v;
                        P.q[a][c] = A.ma0 * qd + A.a2 * (ep + 2.f * eo + v);
                        for (int n = 0; n < NPOLES; n++) {
                            const float qn = A.rp[n] * pc[n] + A.rq[n] * qc[n] + A.bp2[n] * ep + A.bp3[n] * eo + A.bp4[n] * v;
                            P.qc[a][n][c] = qn;
                            P.pc[a][n][c] = pc[n] + qn;
                        }
                    }
                    if (gx && !(fl & CF_ADE_X)) ne[0] = c0.x * nx + c1.x * curlx;
                    if (gy && !(fl & CF_ADE_Y)) ne[1] = c0.y * ny + c1.y * curly;
                    if (gz && !(fl & CF_ADE_Z)) ne[2] = c0.z * nz + c1.z * curlz;
                    nx = ne[0]; ny = ne[1]; nz = ne[2];
                } else {
                    if (gx) nx = c0.x * nx + c1.x * curlx;
                    if (gy) ny = c0.y * ny + c1.y * curly;
                    if (gz) nz = c0.z * nz + c1.z * curlz;
                }
                if (fl & CF_PEC_X) nx = 0.f;
                if (fl & CF_PEC_Y) ny = 0.f;
                if (fl & CF_PEC_Z) nz = 0.f;
                if (tsf) tsf_add_e(P, i, j, k, nx, ny, nz);
                stE<T>(P.fout[0], c, nx, stp, 0);
                stE<T>(P.fout[1], c, ny, stp, 1);
                stE<T>(P.fout[2], c, nz, stp, 2);
            }
        }
        for (int r = 0; r < 4; r++) { him[r][0] = h[r][1]; him[r][1] = h[r][2]; }
        __syncthreads();   // stage s is free
        if (i + S <= plast) {
            if (tid == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(i + S);
            }
            issued = i + S;
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
    return S * stage + (size_t)nclasses * 64 + 8 * 2 * 32 * 4 + S * 8 + FDTD_MAX_ADE * sizeof(DevAde);
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

// Tensor maps of one field set: 3D (k, j, i) float boxes of 36 x 33 (E) and
// 36 x 32 (H); class bytes 48 x 32 over a row pitch padded to 16 bytes.
int bulk_make_maps(void *encode_fn, const DevPlan &p, float *const f[6], const uint8_t *cls, int cls_pitch, int storage, BulkMaps *out)
{
    auto enc = reinterpret_cast<CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                             const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                             CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                             CUtensorMapFloatOOBfill)>(encode_fn);
    const cuuint64_t dims[3] = {(cuuint64_t)p.zr, (cuuint64_t)p.yr, (cuuint64_t)p.xr};
    const cuuint64_t es = storage == FDTD_STORE_F32 ? 4 : 2;
    const CUtensorMapDataType dtype = storage == FDTD_STORE_F16    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                      : storage == FDTD_STORE_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                                   : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const cuuint32_t BW = storage == FDTD_STORE_F32 ? Geo<float>::BW : Geo<__half>::BW;
    const cuuint64_t strides[2] = {(cuuint64_t)p.zr * es, (cuuint64_t)p.zr * es * (cuuint64_t)p.yr};
    const cuuint32_t estr[3] = {1, 1, 1};
    const cuuint32_t boxe[3] = {BW, BROWS_E, 1}, boxh[3] = {BW, BROWS_H, 1}, boxc[3] = {BWC, BROWS_H, 1};
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
