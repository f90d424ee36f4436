// fdtd_device.cuh -- device helpers shared by the step kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fdtd_internal.h"

// ---- field storage: FP32, FP16, BF16 or FP64 elements behind the float
// pointers of DevPlan.  Arithmetic is FP32 (Stor<T>::real) for the first three
// and FP64 for FP64 storage (the reference-precision mode).  Stor<T>::scaled
// tells whether H and psi carry the power-of-two scales of DevPlan (16-bit
// storage only).
template <class T>
struct Stor;

// murmur3's 32-bit finaliser: a bijection with full avalanche, used as the
// random source of stochastic rounding (deterministic given cell, step and array)
__device__ __forceinline__ uint32_t sr_mix(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

// per-step, per-array seed of the rounding dither (array: 0-5 the field
// components, 6-17 psi_E, 18-29 psi_H)
__device__ __forceinline__ uint32_t sr_seed(uint32_t step, uint32_t array)
{
    return sr_mix(step * 0x9e3779b9u ^ (array + 1u) * 0x27d4eb2fu);
}

template <>
struct Stor<float> {
    using real = float;
    static constexpr bool scaled = false;
    static constexpr bool stochastic = false;
    __device__ static float ld(const float *p, int64_t i) { return p[i]; }
    __device__ static float ldg(const float *p, int64_t i) { return __ldg(p + i); }
    __device__ static void st(float *p, int64_t i, float v) { p[i] = v; }
    __device__ static float cvt(float v) { return v; }
};
template <>
struct Stor<__half> {
    using real = float;
    static constexpr bool scaled = true;
    static constexpr bool stochastic = false;
    __device__ static float ld(const float *p, int64_t i) { return __half2float(reinterpret_cast<const __half *>(p)[i]); }
    __device__ static float ldg(const float *p, int64_t i) { return __half2float(__ldg(reinterpret_cast<const __half *>(p) + i)); }
    __device__ static void st(float *p, int64_t i, float v) { reinterpret_cast<__half *>(p)[i] = __float2half_rn(v); }
    __device__ static float cvt(__half v) { return __half2float(v); }
};
template <>
struct Stor<__nv_bfloat16> {
    // BF16 keeps 8 significant bits: round to nearest would drop every
    // per-step increment below half an ulp (a wave resolved by hundreds of
    // steps per period stalls), so stores round stochastically -- the 16
    // dropped bits are compared against a uniform random number, which makes
    // the stored value an unbiased estimate of the FP32 result.
    using real = float;
    static constexpr bool scaled = true;
    static constexpr bool stochastic = true;
    __device__ static float ld(const float *p, int64_t i)
    {
        return __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(p)[i]);
    }
    __device__ static float ldg(const float *p, int64_t i)
    {
        return __bfloat162float(__ldg(reinterpret_cast<const __nv_bfloat16 *>(p) + i));
    }
    __device__ static void st(float *p, int64_t i, float v) { reinterpret_cast<__nv_bfloat16 *>(p)[i] = __float2bfloat16_rn(v); }
    __device__ static void st_sr(float *p, int64_t i, float v, uint32_t seed)
    {
        uint32_t u = __float_as_uint(v);
        if ((u & 0x7f800000u) != 0x7f800000u) u += sr_mix((uint32_t)i ^ seed) & 0xffffu;   // finite values only
        reinterpret_cast<uint16_t *>(p)[i] = (uint16_t)(u >> 16);
    }
    __device__ static float cvt(__nv_bfloat16 v) { return __bfloat162float(v); }
};

template <>
struct Stor<double> {
    using real = double;
    static constexpr bool scaled = false;
    static constexpr bool stochastic = false;
    __device__ static double ld(const float *p, int64_t i) { return reinterpret_cast<const double *>(p)[i]; }
    __device__ static double ldg(const float *p, int64_t i) { return __ldg(reinterpret_cast<const double *>(p) + i); }
    __device__ static void st(float *p, int64_t i, double v) { reinterpret_cast<double *>(p)[i] = v; }
};

// one element of a field stored as FDTD_STORE_* `storage` (small kernels
// that read a few values per thread branch on it at run time)
__device__ __forceinline__ double ld_any(const float *p, int64_t i, int storage)
{
    if (storage == 1) return Stor<__half>::ld(p, i);
    if (storage == 2) return Stor<__nv_bfloat16>::ld(p, i);
    if (storage == 3) return Stor<double>::ld(p, i);
    return p[i];
}

// three components of the arithmetic type R (float3 / double3)
template <class R>
struct V3t;
template <>
struct V3t<float> { using type = float3; };
template <>
struct V3t<double> { using type = double3; };
template <class R>
using V3 = typename V3t<R>::type;

// ---- coefficient tables of the arithmetic type R.  R = float reads the
// FP32 tables of DevPlan; R = double (FDTD_STORE_F64 plans) reads the FP64
// tables the same pointers then hold.
template <class R>
struct Tab;
template <>
struct Tab<float> {
    using Ade = DevAde;
    using V2 = float2;
    __device__ static float dx(const DevPlan &P) { return P.dx; }
    __device__ static float ld(const float *p, int64_t q) { return __ldg(p + q); }
    __device__ static float *state(float *p) { return p; }
    // da, db of class c (scls: the class table as float4, shared or global)
    __device__ static void hcoef(const DevPlan &, const float4 *scls, int c, float &da, float &db)
    {
        const float4 hc = scls[c * 4 + 2];
        da = hc.x;
        db = hc.y;
    }
    __device__ static void ecoef(const DevPlan &, const float4 *scls, int c, float ca[3], float cb[3], float cba[3],
                                 unsigned &flags, int &ade)
    {
        const float4 c0 = scls[c * 4 + 0], c1 = scls[c * 4 + 1], c2 = scls[c * 4 + 2], c3 = scls[c * 4 + 3];
        ca[0] = c0.x; ca[1] = c0.y; ca[2] = c0.z;
        cb[0] = c1.x; cb[1] = c1.y; cb[2] = c1.z;
        cba[0] = c3.x; cba[1] = c3.y; cba[2] = c3.z;
        flags = __float_as_uint(c0.w);
        ade = __float_as_int(c2.z);
    }
    __device__ static float tsfe(const DevPlan &, const float4 *scls, int c) { return scls[c * 4 + 1].w; }
    __device__ static const DevAde &ade(const DevPlan &P, int a) { return P.ade[a]; }
};
template <>
struct Tab<double> {
    using Ade = DevAde64;
    using V2 = double2;
    __device__ static double dx(const DevPlan &P) { return P.dxd; }
    __device__ static double ld(const float *p, int64_t q) { return __ldg(reinterpret_cast<const double *>(p) + q); }
    __device__ static double *state(float *p) { return reinterpret_cast<double *>(p); }
    __device__ static const DevClass64 &cls(const DevPlan &P, int c) { return reinterpret_cast<const DevClass64 *>(P.classes)[c]; }
    __device__ static void hcoef(const DevPlan &P, const float4 *, int c, double &da, double &db)
    {
        da = cls(P, c).da;
        db = cls(P, c).db;
    }
    __device__ static void ecoef(const DevPlan &P, const float4 *, int c, double ca[3], double cb[3], double cba[3],
                                 unsigned &flags, int &ade)
    {
        const DevClass64 &k = cls(P, c);
        for (int a = 0; a < 3; a++) { ca[a] = k.ca[a]; cb[a] = k.cb[a]; cba[a] = k.cba[a]; }
        flags = k.flags;
        ade = k.ade;
    }
    __device__ static double tsfe(const DevPlan &P, const float4 *, int c) { return cls(P, c).tsfe; }
    __device__ static const DevAde64 &ade(const DevPlan &P, int a) { return reinterpret_cast<const DevAde64 *>(P.ade)[a]; }
};

// E (unscaled), H (times hs), psi_H (times ps) and psi_E (times pse) element
// access.  Stores take the step number `stp` (sr_step) and the array index of
// sr_seed, which only stochastic rounding uses.
template <class T>
__device__ __forceinline__ uint32_t sr_step(const DevPlan &P)
{
    if constexpr (Stor<T>::stochastic) return (uint32_t)__ldg(P.stepc);
    else return 0u;
}
template <class T>
__device__ __forceinline__ void st_any(float *p, int64_t i, typename Stor<T>::real v, uint32_t stp, uint32_t array)
{
    if constexpr (Stor<T>::stochastic) Stor<T>::st_sr(p, i, v, sr_seed(stp, array));
    else Stor<T>::st(p, i, v);
}
template <class T>
using real_t = typename Stor<T>::real;
template <class T>
__device__ __forceinline__ real_t<T> ldE(const float *p, int64_t i) { return Stor<T>::ld(p, i); }
template <class T>
__device__ __forceinline__ real_t<T> ldgE(const float *p, int64_t i) { return Stor<T>::ldg(p, i); }
template <class T>
__device__ __forceinline__ void stE(float *p, int64_t i, real_t<T> v, uint32_t stp, uint32_t array)
{
    st_any<T>(p, i, v, stp, array);
}
template <class T>
__device__ __forceinline__ real_t<T> ldH(const DevPlan &P, const float *p, int64_t i)
{
    if constexpr (Stor<T>::scaled) return Stor<T>::ld(p, i) * P.ihs;
    else return Stor<T>::ld(p, i);
}
template <class T>
__device__ __forceinline__ real_t<T> ldgH(const DevPlan &P, const float *p, int64_t i)
{
    if constexpr (Stor<T>::scaled) return Stor<T>::ldg(p, i) * P.ihs;
    else return Stor<T>::ldg(p, i);
}
template <class T>
__device__ __forceinline__ void stH(const DevPlan &P, float *p, int64_t i, real_t<T> v, uint32_t stp, uint32_t array)
{
    if constexpr (Stor<T>::scaled) st_any<T>(p, i, v * P.hs, stp, array);
    else st_any<T>(p, i, v, stp, array);
}
template <class T>
__device__ __forceinline__ real_t<T> ldPsi(const DevPlan &P, const float *p, int64_t i)
{
    if constexpr (Stor<T>::scaled) return Stor<T>::ld(p, i) * P.ips;
    else return Stor<T>::ld(p, i);
}
template <class T>
__device__ __forceinline__ real_t<T> ldgPsi(const DevPlan &P, const float *p, int64_t i)
{
    if constexpr (Stor<T>::scaled) return Stor<T>::ldg(p, i) * P.ips;
    else return Stor<T>::ldg(p, i);
}
template <class T>
__device__ __forceinline__ void stPsi(const DevPlan &P, float *p, int64_t i, real_t<T> v, uint32_t stp, uint32_t array)
{
    if constexpr (Stor<T>::scaled) st_any<T>(p, i, v * P.ps, stp, array);
    else st_any<T>(p, i, v, stp, array);
}
template <class T>
__device__ __forceinline__ real_t<T> ldPsiE(const DevPlan &P, const float *p, int64_t i)
{
    if constexpr (Stor<T>::scaled) return Stor<T>::ld(p, i) * P.ipse;
    else return Stor<T>::ld(p, i);
}
template <class T>
__device__ __forceinline__ void stPsiE(const DevPlan &P, float *p, int64_t i, real_t<T> v, uint32_t stp, uint32_t array)
{
    if constexpr (Stor<T>::scaled) st_any<T>(p, i, v * P.pse, stp, array);
    else st_any<T>(p, i, v, stp, array);
}

// a hint that moves the line holding p into L2; no register, no wait
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// ---- 4-vectors of the storage type

// four consecutive elements from shared memory (16- or 8-byte aligned)
template <class T>
__device__ __forceinline__ float4 lds4(const T *p);
template <>
__device__ __forceinline__ float4 lds4<float>(const float *p) { return *reinterpret_cast<const float4 *>(p); }
template <>
__device__ __forceinline__ float4 lds4<__half>(const __half *p)
{
    const uint2 u = *reinterpret_cast<const uint2 *>(p);
    const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
}
template <>
__device__ __forceinline__ float4 lds4<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    const uint2 u = *reinterpret_cast<const uint2 *>(p);
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
}

// four consecutive elements of a global field array (element index c, c % 4 == 0)
template <class T>
__device__ __forceinline__ float4 ldg4(const float *base, int64_t c)
{
    if constexpr (sizeof(T) == 4) return *reinterpret_cast<const float4 *>(base + c);
    else return lds4<T>(reinterpret_cast<const T *>(base) + c);
}
// the same through the read-only data path (arrays no thread writes during the kernel)
template <class T>
__device__ __forceinline__ float4 ldg4_ro(const float *base, int64_t c)
{
    if constexpr (sizeof(T) == 4) return __ldg(reinterpret_cast<const float4 *>(base + c));
    else {
        const uint2 u = __ldg(reinterpret_cast<const uint2 *>(reinterpret_cast<const T *>(base) + c));
        return lds4<T>(reinterpret_cast<const T *>(&u));
    }
}

// round one FP32 value to the 16-bit storage type (bits), as Stor<T>::st does
template <class T>
__device__ __forceinline__ uint32_t bits16(float v, int64_t i, uint32_t seed)
{
    if constexpr (Stor<T>::stochastic) {
        uint32_t u = __float_as_uint(v);
        if ((u & 0x7f800000u) != 0x7f800000u) u += sr_mix((uint32_t)i ^ seed) & 0xffffu;
        return u >> 16;
    } else {
        const __half h = __float2half_rn(v);
        return (uint32_t)*reinterpret_cast<const unsigned short *>(&h);
    }
}

// store four values (times `scale` at 16-bit storage) at element c, c % 4 == 0
template <class T>
__device__ __forceinline__ void stg4(float *base, int64_t c, float4 v, float scale, uint32_t stp, uint32_t array)
{
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4 *>(base + c) = v;
    } else {
        const uint32_t seed = Stor<T>::stochastic ? sr_seed(stp, array) : 0u;
        const uint32_t a = bits16<T>(v.x * scale, c, seed), b = bits16<T>(v.y * scale, c + 1, seed);
        const uint32_t d = bits16<T>(v.z * scale, c + 2, seed), e = bits16<T>(v.w * scale, c + 3, seed);
        *reinterpret_cast<uint2 *>(reinterpret_cast<T *>(base) + c) = make_uint2(a | (b << 16), d | (e << 16));
    }
}

// the same as arrays of four floats
template <class T>
__device__ __forceinline__ void lds4a(float (&d)[4], const T *p)
{
    const float4 v = lds4<T>(p);
    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
}
template <class T>
__device__ __forceinline__ void ldg4a(float (&d)[4], const float *base, int64_t c)
{
    const float4 v = ldg4<T>(base, c);
    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
}
template <class T>
__device__ __forceinline__ void stg4a(float *base, int64_t c, const float (&v)[4], float scale, uint32_t stp, uint32_t array)
{
    stg4<T>(base, c, make_float4(v[0], v[1], v[2], v[3]), scale, stp, array);
}
__device__ __forceinline__ void lds4a_f(float (&d)[4], const float4 v)
{
    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
}
// FP32 state arrays (ADE)
__device__ __forceinline__ void ldq4a(float (&d)[4], const float *p)
{
    const float4 v = *reinterpret_cast<const float4 *>(p);
    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
}
__device__ __forceinline__ void stq4a(float *p, const float (&v)[4]) { *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]); }

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
template <class R>
__device__ __forceinline__ void tsf_add_h(const DevPlan &P, int i, int j, int k, R &hx, R &hy, R &hz)
{
    using V2 = typename Tab<R>::V2;
    const V2 *const *tc = reinterpret_cast<const V2 *const *>(P.tcor_h);
    const int i0 = P.t0[0], j0 = P.t0[1], k0 = P.t0[2], in = P.t1[0], jn = P.t1[1], kn = P.t1[2];
    const bool ji = j >= j0 && j <= jn, ki = k >= k0 && k <= kn, ii = i >= i0 && i <= in;
    if (ji && ki) {
        if (i == i0 - 1) { const V2 d = tc[0][(j - j0) * P.tnb[0] + (k - k0)]; hy += d.x; hz += d.y; }
        if (i == in) { const V2 d = tc[1][(j - j0) * P.tnb[1] + (k - k0)]; hy += d.x; hz += d.y; }
    }
    if (ii && ki) {
        if (j == j0 - 1) { const V2 d = tc[2][(i - i0) * P.tnb[2] + (k - k0)]; hx += d.x; hz += d.y; }
        if (j == jn) { const V2 d = tc[3][(i - i0) * P.tnb[3] + (k - k0)]; hx += d.x; hz += d.y; }
    }
    if (ii && ji) {
        if (k == k0 - 1) { const V2 d = tc[4][(i - i0) * P.tnb[4] + (j - j0)]; hx += d.x; hy += d.y; }
        if (k == kn) { const V2 d = tc[5][(i - i0) * P.tnb[5] + (j - j0)]; hx += d.x; hy += d.y; }
    }
}

// Same for the E cell (source.c:547-771): (ey,ez) on i faces, (ex,ez) on j
// faces, (ex,ey) on k faces.
template <class R>
__device__ __forceinline__ void tsf_add_e(const DevPlan &P, int i, int j, int k, R &ex, R &ey, R &ez)
{
    using V2 = typename Tab<R>::V2;
    const V2 *const *tc = reinterpret_cast<const V2 *const *>(P.tcor_e);
    const int i0 = P.t0[0], j0 = P.t0[1], k0 = P.t0[2], in = P.t1[0], jn = P.t1[1], kn = P.t1[2];
    const bool ji = j >= j0 && j <= jn, ki = k >= k0 && k <= kn, ii = i >= i0 && i <= in;
    if (ji && ki) {
        if (i == i0) { const V2 d = tc[0][(j - j0) * P.tnb[0] + (k - k0)]; ey += d.x; ez += d.y; }
        if (i == in) { const V2 d = tc[1][(j - j0) * P.tnb[1] + (k - k0)]; ey += d.x; ez += d.y; }
    }
    if (ii && ki) {
        if (j == j0) { const V2 d = tc[2][(i - i0) * P.tnb[2] + (k - k0)]; ex += d.x; ez += d.y; }
        if (j == jn) { const V2 d = tc[3][(i - i0) * P.tnb[3] + (k - k0)]; ex += d.x; ez += d.y; }
    }
    if (ii && ji) {
        if (k == k0) { const V2 d = tc[4][(i - i0) * P.tnb[4] + (j - j0)]; ex += d.x; ey += d.y; }
        if (k == kn) { const V2 d = tc[5][(i - i0) * P.tnb[5] + (j - j0)]; ex += d.x; ey += d.y; }
    }
}

// L1 prefetch of the entries tsf_add_h and tsf_add_e read for the cells
// (i, j, kq .. kq+3) of a 4-cell group, under the same tests (every address
// is one those calls read).  Issued at the top of a plane: their reads come
// at the end of the H and E phases, where an L2 round trip of the warp that
// holds a face group would hold the whole CTA at the plane's barrier.
template <class R>
__device__ __forceinline__ void tsf_prefetch_group(const DevPlan &P, int i, int j, int kq)
{
    using V2 = typename Tab<R>::V2;
    const V2 *const *th = reinterpret_cast<const V2 *const *>(P.tcor_h);
    const V2 *const *te = reinterpret_cast<const V2 *const *>(P.tcor_e);
    const int i0 = P.t0[0], j0 = P.t0[1], k0 = P.t0[2], in = P.t1[0], jn = P.t1[1], kn = P.t1[2];
    const int kh = kq + 3;
    const bool ji = j >= j0 && j <= jn, ii = i >= i0 && i <= in;
    const bool kany = kh >= k0 && kq <= kn;               // some cell of the group has k0 <= k <= kn
    const int kk = (kq > k0 ? kq : k0) - k0;              // its first such cell, from k0
    if (ii && ji) {   // k faces: one entry per (i, j)
        const int q4 = (i - i0) * P.tnb[4] + (j - j0), q5 = (i - i0) * P.tnb[5] + (j - j0);
        if (kq <= k0 - 1 && kh >= k0 - 1) prefetch_l1(th[4] + q4);
        if (kq <= k0 && kh >= k0) prefetch_l1(te[4] + q4);
        if (kq <= kn && kh >= kn) { prefetch_l1(th[5] + q5); prefetch_l1(te[5] + q5); }
    }
    if (ii && kany) {   // j faces: the group's entries are consecutive in k
        if (j == j0 - 1) prefetch_l1(th[2] + (i - i0) * P.tnb[2] + kk);
        if (j == j0) prefetch_l1(te[2] + (i - i0) * P.tnb[2] + kk);
        if (j == jn) { prefetch_l1(th[3] + (i - i0) * P.tnb[3] + kk); prefetch_l1(te[3] + (i - i0) * P.tnb[3] + kk); }
    }
    if (ji && kany) {   // i faces
        if (i == i0 - 1) prefetch_l1(th[0] + (j - j0) * P.tnb[0] + kk);
        if (i == i0) prefetch_l1(te[0] + (j - j0) * P.tnb[0] + kk);
        if (i == in) { prefetch_l1(th[1] + (j - j0) * P.tnb[1] + kk); prefetch_l1(te[1] + (j - j0) * P.tnb[1] + kk); }
    }
}
