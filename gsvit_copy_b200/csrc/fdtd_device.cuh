// fdtd_device.cuh -- device helpers shared by the step kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd_internal.h"

__device__ __forceinline__ int cls_at(const DevPlan &P, int i, int j, int k)
{
    return __ldg(P.cls + ((int64_t)i * P.yr + j) * P.cpitch + k);
}

// dcomp of source.c:54-107 with the reference call (i0=0, i1=xres, ...): the
// corner offsets and the rx = 0 branch are resolved on the host; FP64 with
// the reference's operation order (no contraction).
__device__ __forceinline__ double tsf_dcomp(const DevPlan &P, int i, int j, int k)
{
    double rx = P.trx_zero ? 0.0 : (double)(i - P.trx_origin);
    double ry = (double)(j - P.try_origin);
    double rz = (double)(k - P.trz_origin);
    double s = __dadd_rn(__dadd_rn(__dmul_rn(P.tax, rx), __dmul_rn(P.tay, ry)), __dmul_rn(P.taz, rz));
    return __dmul_rn(P.corr, __dadd_rn(10.0, s));
}

// sv_dline_get_dval, dline.c:89-111 (4-point cubic, linear near the ends)
__device__ __forceinline__ double tsf_dval(const double *data, int res, double x)
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

// Add the precomputed TSF corrections of this step to the H cell (i,j,k).
// Face order as the reference applies them: i0, in, j0, jn, k0, kn
// (source.c:1476-1672); components (hy,hz) on i faces, (hx,hz) on j faces,
// (hx,hy) on k faces.
__device__ __forceinline__ void tsf_add_h(const DevPlan &P, int i, int j, int k, float &hx, float &hy, float &hz)
{
    const int i0 = P.t0[0], j0 = P.t0[1], k0 = P.t0[2], in = P.t1[0], jn = P.t1[1], kn = P.t1[2];
    const bool ji = j >= j0 && j <= jn, ki = k >= k0 && k <= kn, ii = i >= i0 && i <= in;
    if (ji && ki) {
        if (i == i0 - 1) { const float2 d = P.tcor_h[0][(j - j0) * P.tnb[0] + (k - k0)]; hy += d.x; hz += d.y; }
        if (i == in) { const float2 d = P.tcor_h[1][(j - j0) * P.tnb[1] + (k - k0)]; hy += d.x; hz += d.y; }
    }
    if (ii && ki) {
        if (j == j0 - 1) { const float2 d = P.tcor_h[2][(i - i0) * P.tnb[2] + (k - k0)]; hx += d.x; hz += d.y; }
        if (j == jn) { const float2 d = P.tcor_h[3][(i - i0) * P.tnb[3] + (k - k0)]; hx += d.x; hz += d.y; }
    }
    if (ii && ji) {
        if (k == k0 - 1) { const float2 d = P.tcor_h[4][(i - i0) * P.tnb[4] + (j - j0)]; hx += d.x; hy += d.y; }
        if (k == kn) { const float2 d = P.tcor_h[5][(i - i0) * P.tnb[5] + (j - j0)]; hx += d.x; hy += d.y; }
    }
}

// Same for the E cell (source.c:547-771): (ey,ez) on i faces, (ex,ez) on j
// faces, (ex,ey) on k faces.
__device__ __forceinline__ void tsf_add_e(const DevPlan &P, int i, int j, int k, float &ex, float &ey, float &ez)
{
    const int i0 = P.t0[0], j0 = P.t0[1], k0 = P.t0[2], in = P.t1[0], jn = P.t1[1], kn = P.t1[2];
    const bool ji = j >= j0 && j <= jn, ki = k >= k0 && k <= kn, ii = i >= i0 && i <= in;
    if (ji && ki) {
        if (i == i0) { const float2 d = P.tcor_e[0][(j - j0) * P.tnb[0] + (k - k0)]; ey += d.x; ez += d.y; }
        if (i == in) { const float2 d = P.tcor_e[1][(j - j0) * P.tnb[1] + (k - k0)]; ey += d.x; ez += d.y; }
    }
    if (ii && ki) {
        if (j == j0) { const float2 d = P.tcor_e[2][(i - i0) * P.tnb[2] + (k - k0)]; ex += d.x; ez += d.y; }
        if (j == jn) { const float2 d = P.tcor_e[3][(i - i0) * P.tnb[3] + (k - k0)]; ex += d.x; ez += d.y; }
    }
    if (ii && ji) {
        if (k == k0) { const float2 d = P.tcor_e[4][(i - i0) * P.tnb[4] + (j - j0)]; ex += d.x; ey += d.y; }
        if (k == kn) { const float2 d = P.tcor_e[5][(i - i0) * P.tnb[5] + (j - j0)]; ex += d.x; ey += d.y; }
    }
}
