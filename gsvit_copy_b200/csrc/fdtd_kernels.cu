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

#include "fdtd_cells.cuh"

namespace {

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
    using R = real_t<T>;
    const uint32_t stp = sr_step<T>(P);
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const float *EX = P.fin[0], *EY = P.fin[1], *EZ = P.fin[2];
    const R ex = ldgE<T>(EX, c), ey = ldgE<T>(EY, c), ez = ldgE<T>(EZ, c);
    const bool il = (i == P.xr - 1), jl = (j == P.yr - 1), kl = (k == P.zr - 1);
    const R eyk = kl ? R(0) : ldgE<T>(EY, c + 1), exk = kl ? R(0) : ldgE<T>(EX, c + 1);
    const R ezj = jl ? R(0) : ldgE<T>(EZ, c + P.sj), exj = jl ? R(0) : ldgE<T>(EX, c + P.sj);
    const R ezi = il ? R(0) : ldgE<T>(EZ, c + P.si), eyi = il ? R(0) : ldgE<T>(EY, c + P.si);
    R h[3] = {ldgH<T>(P, P.fin[3], c), ldgH<T>(P, P.fin[4], c), ldgH<T>(P, P.fin[5], c)};
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
    using R = real_t<T>;
    const uint32_t stp = sr_step<T>(P);
    const int64_t c = (int64_t)i * P.si + (int64_t)j * P.sj + k;
    const float *HX = P.fout[3], *HY = P.fout[4], *HZ = P.fout[5];   // H^{n+1/2}, written this step
    const V3<R> eo{ldgE<T>(P.fin[0], c), ldgE<T>(P.fin[1], c), ldgE<T>(P.fin[2], c)};
    const V3<R> h{ldH<T>(P, HX, c), ldH<T>(P, HY, c), ldH<T>(P, HZ, c)};
    const R hx_jm = j > 0 ? ldH<T>(P, HX, c - P.sj) : R(0), hz_jm = j > 0 ? ldH<T>(P, HZ, c - P.sj) : R(0);
    const R hx_km = k > 0 ? ldH<T>(P, HX, c - 1) : R(0), hy_km = k > 0 ? ldH<T>(P, HY, c - 1) : R(0);
    const R hy_im = i > 0 ? ldH<T>(P, HY, c - P.si) : R(0), hz_im = i > 0 ? ldH<T>(P, HZ, c - P.si) : R(0);
    const float4 *cl = reinterpret_cast<const float4 *>(P.classes);
    const V3<R> en =
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
template <class R>
__device__ __forceinline__ void tsf_face_cell(const DevPlan &P, int t)
{
    using V2 = typename Tab<R>::V2;
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
    V2 dh{0, 0}, de{0, 0};
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
        const double ce = (double)Tab<R>::tsfe(P, cls4, cls_at(P, ei, ej, ek));
        const bool pec = (fl & 2) != 0;
        switch (f) {
        case 0:
            if (ek < kn) dh.x = -(R)(hc * (ve * P.gez));
            if (ej < jn) dh.y = (R)(hc * (ve * P.gey));
            if (ej < jn) de.x = (R)(ce * (vh * P.ghz));
            if (ek < kn) de.y = -(R)(ce * (vh * P.ghy));
            break;
        case 1:
            if (ek < kn) dh.x = (R)(hc * (ve * P.gez));
            if (ej < jn) dh.y = -(R)(hc * (ve * P.gey));
            if (ej < jn) de.x = -(R)(ce * (vh * P.ghz));
            if (ek < kn) de.y = (R)(ce * (vh * P.ghy));
            break;
        case 2:
            if (ek < kn) dh.x = (R)(hc * (ve * P.gez));
            if (ei < in) dh.y = -(R)(hc * (ve * P.gex));
            if (ei < in) de.x = -(R)(ce * (vh * P.ghz));
            if (ek < kn) de.y = (R)(ce * (vh * P.ghx));
            break;
        case 3:
            if (ek < kn) dh.x = -(R)(hc * (ve * P.gez));
            if (ei < in) dh.y = (R)(hc * (ve * P.gex));
            if (ei < in) de.x = (R)(ce * (vh * P.ghz));
            if (ek < kn) de.y = -(R)(ce * (vh * P.ghx));
            break;
        case 4:
            if (ej < jn && !pec) dh.x = -(R)(hc * (ve * P.gey));
            if (ei < in && !pec) dh.y = (R)(hc * (ve * P.gex));
            if (ei < in && !pec) de.x = (R)(ce * (vh * P.ghy));
            if (ej < jn && !pec) de.y = -(R)(ce * (vh * P.ghx));
            break;
        default:
            if (ej < jn) dh.x = (R)(hc * (ve * P.gey));
            if (ei < in) dh.y = -(R)(hc * (ve * P.gex));
            if (ei < in) de.x = -(R)(ce * (vh * P.ghy));
            if (ej < jn) de.y = (R)(ce * (vh * P.ghx));
            break;
        }
    }
    reinterpret_cast<V2 *>(P.tcor_h[f])[off] = dh;
    reinterpret_cast<V2 *>(P.tcor_e[f])[off] = de;
    (void)a; (void)b;
}

__global__ void tsf_face_kernel(const __grid_constant__ DevPlan P, int total)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < total) {
        if (P.real64) tsf_face_cell<double>(P, t);
        else tsf_face_cell<float>(P, t);
    }
}

__global__ void tsf_face_batch(const DevPlan *plans)
{
    tsf_face_cell<float>(plans[blockIdx.y], blockIdx.x * blockDim.x + threadIdx.x);
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
            A.probe_out[((size_t)p * A.nsteps_planned + (s - 1)) * 6 + comp] = ld_any(A.fields[comp], A.probe_cells[p], A.storage) * (comp >= 3 ? (double)A.ihs : 1.0);
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
        A.probe_out[((size_t)p * A.nsteps_planned + (s - 1)) * 6 + comp] = ld_any(A.fields[comp], A.probe_cells[p], A.storage) * (comp >= 3 ? (double)A.ihs : 1.0);
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

// tw: the CTA's twiddle table, or nullptr to evaluate them per cell.  S: the
// element type of the sample ring (FP32; FP64 for FP64-storage plans)
// STAGE (FP32 samples only): the cell's ring (8 x 9 values) is read once into
// registers instead of once per frequency (the ring is far larger than L2),
// at 144 registers a thread; the same arithmetic in the same order.
template <class S, bool STAGE = false>
__device__ __forceinline__ void nfff_fold(const DevNfff &N, int s, int first_step, int nslots, bool clear, const double2 *tw)
{
    const size_t ns = (size_t)N.ns;
    S *ring = reinterpret_cast<S *>(N.ring);
    if constexpr (STAGE && sizeof(S) == 4) {
        float rv[NFFF_RING][9];
#pragma unroll
        for (int j = 0; j < NFFF_RING; j++)
#pragma unroll
            for (int q = 0; q < 9; q++) rv[j][q] = j < nslots ? ring[((size_t)j * 9 + q) * ns + s] : 0.f;
        for (int f = 0; f < N.nfreq; f++) {
            double2 A[6];
            for (int q = 0; q < 6; q++) A[q] = N.acc[((size_t)f * 6 + q) * ns + s];
#pragma unroll
            for (int j = 0; j < NFFF_RING; j++) {
                if (j >= nslots) break;
                double v[6];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    v[a] = (double)rv[j][3 * a];
                    v[3 + a] = ((double)rv[j][3 * a + 1] - (double)rv[j][3 * a + 2]) * N.inv2dx;
                }
                double sn, cs;
                if (tw) { cs = tw[f * nslots + j].x; sn = tw[f * nslots + j].y; }
                else sincos(N.omega_dt[f] * (double)(first_step + j), &sn, &cs);
#pragma unroll
                for (int q = 0; q < 6; q++) {
                    A[q].x += v[q] * cs;
                    A[q].y -= v[q] * sn;
                }
            }
            for (int q = 0; q < 6; q++) N.acc[((size_t)f * 6 + q) * ns + s] = A[q];
        }
        if (clear)
            for (int j = 0; j < nslots; j++)
                for (int q = 0; q < 9; q++) ring[((size_t)j * 9 + q) * ns + s] = 0;
        return;
    }
    for (int f = 0; f < N.nfreq; f++) {
        double2 A[6];
        for (int q = 0; q < 6; q++) A[q] = N.acc[((size_t)f * 6 + q) * ns + s];
        for (int j = 0; j < nslots; j++) {
            const S *r = ring + (size_t)j * 9 * ns + s;
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
            for (int q = 0; q < 9; q++) ring[((size_t)j * 9 + q) * ns + s] = 0;
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
    if (s < N.ns) {
        if (N.storage == FDTD_STORE_F64) nfff_fold<double>(N, s, done - pending, pending, true, table ? tw : nullptr);
        else nfff_fold<float>(N, s, done - pending, pending, true, table ? tw : nullptr);
    }
}

// The NFFF step in two launches (single plans and batches): the sampling, which every step
// does, in a light kernel (few registers, full occupancy: its nine gathered
// loads a cell want many in flight), and the fold, which only the step that
// fills the ring does, in a kernel that every other step leaves at once.
// Both launch every step, so a captured graph is right at any step offset.
template <class S>
__device__ __forceinline__ void nfff_sample_cell(const DevNfff &N, int s)
{
    if (N.ns <= 0 || N.nfreq <= 0 || s >= N.ns) return;
    const int step = *N.step - 1;
    if (step < 0) return;
    const size_t ns = (size_t)N.ns;
    const int64_t c = N.cell[s];
    const int64_t st = N.nstride[s];
    S *r = reinterpret_cast<S *>(N.ring) + (size_t)(step % NFFF_RING) * 9 * ns + s;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float *E = N.e[a];
        r[(3 * a) * ns] = (S)ld_any(E, c, N.storage);
        r[(3 * a + 1) * ns] = (S)ld_any(E, c + st, N.storage);
        r[(3 * a + 2) * ns] = (S)ld_any(E, c - st, N.storage);
    }
}

__global__ void nfff_sample_kernel(const DevNfff N)
{
    if (N.storage == FDTD_STORE_F64) nfff_sample_cell<double>(N, blockIdx.x * blockDim.x + threadIdx.x);
    else nfff_sample_cell<float>(N, blockIdx.x * blockDim.x + threadIdx.x);
}

// the step counter is the same for every thread of the launch: a CTA either
// leaves at once or reaches the twiddle table's barrier with all its threads
template <class S>
__device__ __forceinline__ void nfff_fold_full_ring(const DevNfff &N, int s)
{
    if (N.ns <= 0 || N.nfreq <= 0) return;
    const int step = *N.step - 1;
    if (step < 0 || step % NFFF_RING != NFFF_RING - 1) return;
    __shared__ double2 tw[NFFF_RING * NFFF_TW_MAXF];
    const bool table = N.nfreq <= NFFF_TW_MAXF;
    if (table) nfff_twiddles(N, step - (NFFF_RING - 1), NFFF_RING, tw);
    if (s < N.ns) nfff_fold<S, true>(N, s, step - (NFFF_RING - 1), NFFF_RING, false, table ? tw : nullptr);
}

__global__ void __launch_bounds__(128, 3) nfff_fold_kernel(const DevNfff N)
{
    if (N.storage == FDTD_STORE_F64) nfff_fold_full_ring<double>(N, blockIdx.x * blockDim.x + threadIdx.x);
    else nfff_fold_full_ring<float>(N, blockIdx.x * blockDim.x + threadIdx.x);
}

// batches: one plan per CTA row (blockIdx.y), so the step counter and the fold
// decision are the same for every thread of a CTA
__global__ void nfff_sample_batch(const DevNfff *N)
{
    nfff_sample_cell<float>(N[blockIdx.y], blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(128, 3) nfff_fold_batch(const DevNfff *N)
{
    nfff_fold_full_ring<float>(N[blockIdx.y], blockIdx.x * blockDim.x + threadIdx.x);
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
// applied by farfield_reduce_kernel.  FP64 throughout.  The pair geometry
// takes one reciprocal (1/rc) and the retarded index its exact division;
// the other factors are products with constants.  A thread owns a far point
// so that each staged surface cell serves the CTA's 128 points (the pair
// loop is FP64-arithmetic bound; a warp per point would stage every cell 16
// times as often).
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
    const double idx = 1.0 / dx, k4 = 1.0 / (4.0 * PI), kc = 1.0 / (4.0 * PI * C0 * 2.0 * dt);
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
            // one reciprocal for the geometry; the retarded index keeps the
            // reference's division (it must round as there)
            const double irc = 1.0 / rc;
            const double ct = dot * irc;
            const double r = rc * dx;
            const int R = min((int)(1.0 + r / c0dt), F.ntw - 1);
            const double ir = irc * idx;
            const double a = ir * k4;
            const double b = -ct * k4 * ir * ir;
            const double cp = -ct * kc * ir;
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
cudaError_t slab_steps_t(const DevPlan &p, const SlabLists &L, bool ade, int npoles, cudaStream_t st, int part)
{
    bool h4 = false;
    if (part & 1) {
        if constexpr (sizeof(T) <= 4) {   // 4-cell groups: FP32 and 16-bit storage
            if (L.h4blocks > 0) {
                slab_h4_kernel<T><<<(unsigned)L.h4blocks, 256, 0, st>>>(p, L.h4, L.nh);
                h4 = true;
            }
        }
        if (!h4) slab_h_kernel<T><<<(unsigned)L.hblocks, 256, 0, st>>>(p, L.h, L.nh);
    }
    if (!(part & 2)) return cudaGetLastError();
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

cudaError_t launch_slab_steps(const DevPlan &p, const SlabLists &L, bool ade, int npoles, int storage, cudaStream_t st,
                              int part)
{
    if (L.hblocks <= 0) return cudaSuccess;
    if (storage == FDTD_STORE_F64) return slab_steps_t<double>(p, L, ade, npoles, st, part);
    if (storage == FDTD_STORE_F16) return slab_steps_t<__half>(p, L, ade, npoles, st, part);
    if (storage == FDTD_STORE_BF16) return slab_steps_t<__nv_bfloat16>(p, L, ade, npoles, st, part);
    return slab_steps_t<float>(p, L, ade, npoles, st, part);
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
                               int npoles, cudaStream_t st, int part)
{
    if (part & 1) {
        if (nblocks4 > 0)
            slab_h4_batch<T><<<(unsigned)nblocks4, 256, 0, st>>>(p, boxes4, nboxes);
        else
            slab_h_batch<T><<<(unsigned)nblocks, 256, 0, st>>>(p, boxes, nboxes);
    }
    if ((part & 2) && neblocks > 0) {
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
                                    long long neblocks, bool ade, int npoles, int storage, cudaStream_t st, int part)
{
    if (nblocks <= 0) return cudaSuccess;
    if (storage == FDTD_STORE_F16)
        return slab_steps_batch_t<__half>(p, boxes, nboxes, nblocks, boxes4, nblocks4, eboxes, neboxes, neblocks, ade, npoles, st,
                                          part);
    if (storage == FDTD_STORE_BF16)
        return slab_steps_batch_t<__nv_bfloat16>(p, boxes, nboxes, nblocks, boxes4, nblocks4, eboxes, neboxes, neblocks, ade,
                                                 npoles, st, part);
    return slab_steps_batch_t<float>(p, boxes, nboxes, nblocks, boxes4, nblocks4, eboxes, neboxes, neblocks, ade, npoles, st,
                                     part);
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
    if (nplans <= 0 || max_cells <= 0) return;
    nfff_sample_batch<<<dim3((max_cells + 255) / 256, nplans), 256, 0, st>>>(n);
    nfff_fold_batch<<<dim3((max_cells + 127) / 128, nplans), 128, 0, st>>>(n);
}

void launch_nfff_accumulate(const DevNfff &n, cudaStream_t st)
{
    if (n.ns <= 0) return;
    nfff_sample_kernel<<<(n.ns + 255) / 256, 256, 0, st>>>(n);
    nfff_fold_kernel<<<(n.ns + 127) / 128, 128, 0, st>>>(n);
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
