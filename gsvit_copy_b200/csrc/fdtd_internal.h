// fdtd_internal.h -- shared host/device definitions of the B200 FDTD library.
//
// Device data layout (HBM):
//   fields      six float arrays E/H x,y,z in the reference order (i slowest,
//               k fastest), ping-pong pairs: every step reads one set and
//               writes the other, so that CTAs may recompute a neighbour's H
//               row without racing with its owner;
//   class map   one byte per cell: index of a coefficient class (DevClass)
//               derived on the host from the material table, the interface
//               map, the dispersive-neighbour rule and the PEC rule;
//   CPML        psi slabs per face in the reference layout (boundary.c:102-280),
//               psi_H ping-pong like the fields, psi_E in place;
//   ADE state   E^{n-1}, P_D^n, P_D^{n-1} (+ 2 CP poles) per component, full
//               grid arrays touched only by dispersive cells.
#pragma once
#include <stdint.h>
#include <vector_types.h>

#define FDTD_MAX_CLASSES 256
#define FDTD_MAX_ADE 8

// class flag bits
#define CF_ADE_X      0x001u   // Ex taken by the ADE branch (tbc == 0)
#define CF_ADE_Y      0x002u
#define CF_ADE_Z      0x004u
#define CF_ADE_BRANCH 0x008u   // the cell enters the dispersive branch
#define CF_PEC_X      0x010u   // PEC rule zeroes Ex (yee.c:1138-1237)
#define CF_PEC_Y      0x020u
#define CF_PEC_Z      0x040u
#define CF_DESIGN     0x080u   // E coefficients per cell (DevPlan::dcoef), adjoint design region

struct alignas(16) DevClass {
    // float4 0: ordinary update E = ca*E + cb*curl (get_cabs, yee.c:1397-1493)
    float ca[3];
    uint32_t flags;
    // float4 1: cb, also used by the boundary_estep CPML corrections; TSF-E factor
    float cb[3];
    float tsfe;     // (dt/dx)/epsilon(cell) of the TSF-E correction (source.c:548,566)
    // float4 2: H update (yee.c:219-243) and CPML-H db (get_db, yee.c:1620-1647)
    float da, db;
    int32_t ade;    // ADE coefficient set
    float pad0;
    // float4 3: CPML cb inside the ADE branch (yee.c:950-1057), from the ADE material
    float cba[3];
    float pad1;
};

// The same class in FP64 (FDTD_STORE_F64 plans: DevPlan::classes then points
// to these).
struct alignas(16) DevClass64 {
    double ca[3], cb[3];
    double da, db;
    double cba[3];
    double tsfe;
    uint32_t flags;
    int32_t ade;
};

// ADE coefficients of calculate_ade_a/bp/c (plan.c:2737-2763), recast for the
// difference form of the polarisation state: per component the kernels keep
// Q = P_D^n - P_D^{n-1} and, per critical-point pole, p = P_cp^n and
// q = P_cp^n - P_cp^{n-1}; E^{n-1} is the output field set before it is
// overwritten.  The reference's
//   E^{n+1} = c0 curl + c1 (-a0 P^{n-1} + (1-a1) P^n) + ... + c2 E^{n-1} + c3 E^n,
//   P^{n+1} = a0 P^{n-1} + a1 P^n + a2 (E^{n-1} + 2 E^n + E^{n+1})
// becomes, with a0 + a1 = 1 exactly,
//   E^{n+1} = c0 curl + c1 a0 Q + sum_p [c1 bp0 q + c1 (1 - bp0 - bp1) p] + c2 E^{n-1} + c3 E^n,
//   Q' = -a0 Q + a2 (E^{n-1} + 2 E^n + E^{n+1}),
//   q' = (bp0 + bp1 - 1) p - bp0 q + bp2 E^{n-1} + bp3 E^n + bp4 E^{n+1},  p' = p + q'.
// The same recursion, but FP32 no longer subtracts two nearly equal P values
// (P grows like the time integral of Q), so it tracks the FP64 reference.
struct DevAde {
    float c0dx;          // ade_c0 / dx
    float c2, c3;
    float qe;            // c1 * a0
    float ma0, a2;       // Q recursion
    float pe[2], qpe[2]; // c1 (1 - bp0 - bp1), c1 bp0
    float rp[2], rq[2];  // q recursion: bp0 + bp1 - 1, -bp0
    float bp2[2], bp3[2], bp4[2];
};

// The same set in FP64 (FDTD_STORE_F64 plans: DevPlan::ade then points to these).
struct DevAde64 {
    double c0dx;
    double c2, c3;
    double qe;
    double ma0, a2;
    double pe[2], qpe[2];
    double rp[2], rq[2];
    double bp2[2], bp3[2], bp4[2];
};

struct DevPlan {
    int xr, yr, zr;
    int64_t si, sj;                 // strides of i and j (k stride is 1)
    // plain range per axis: a cell with every index in [plo, phi) takes the
    // plain update (no CPML psi, kappa 1, no edge or zeroed-plane rule)
    int plo[3], phi[3];
    // FDTD_STORE_F64 plan: fields, psi and ADE state are doubles, and every
    // table below (classes, ADE sets, CPML profiles, 1/kappa, TSF corrections,
    // design coefficients) holds doubles behind its float-typed pointer
    int real64;
    float dx;                       // cell size (cubic cells)
    double dxd;                     // the same in FP64
    // 16-bit field storage (FDTD_STORE_F16 / _BF16): H is stored times hs,
    // psi_H times ps and psi_E times pse (powers of two, so the scaling is
    // exact); FP32 storage uses none of them.  The field and psi pointers
    // below then point to 16-bit elements.
    float hs, ihs, ps, ips, pse, ipse;
    const int *stepc;               // device step counter (seeds the BF16 stochastic rounding)
    // fields: [0..2] = E x,y,z, [3..5] = H x,y,z
    const float *fin[6];
    float *fout[6];
    const uint8_t *cls;             // class map, rows padded to cpitch bytes
    int cpitch;
    const DevClass *classes;
    int nclasses;
    // design region: ca[3], cb[3] per cell of the box dbox (i0 i1 j0 j1 k0 k1)
    const float *dcoef;
    int dbox[6];
    // ADE
    int nade;
    const DevAde *ade;
    float *q[3];                    // Drude current Q per component
    float *pc[3][2], *qc[3][2];     // critical-point poles: p and q per component
    // CPML: face order x0 xn y0 yn z0 zn
    int cp_on[6], cp_d[6];
    const float *be[6], *ce[6], *bh[6], *ch[6];
    const float *ike[3], *ikh[3];   // 1/kappa per axis (E and H), length xr / yr / zr
    float *psie[6][2];              // x: {peyx, pezx} y: {pexy, pezy} z: {pexz, peyz}
    const float *psih_in[6][2];     // x: {phyx, phzx} y: {phxy, phzy} z: {phxz, phyz}
    float *psih_out[6][2];
    // TSF
    int tsf_on;
    int t0[3], t1[3];               // box corners i0 j0 k0 / in jn kn
    int tskip[6];
    const uint8_t *tmap[6];         // per face cell: bit0 apply (mat_too_close_check), bit1 PEC at the face cell
    float2 *tcor_h[6], *tcor_e[6];  // this step's TSF corrections per face cell (two components each)
    int tnb[6];                     // inner extent of the face tables
    double corr, hcor;
    double tax, tay, taz;           // propagation direction sin(t)cos(p), sin(t)sin(p), cos(t)
    int trx_origin, try_origin, trz_origin;  // dcomp corner (source.c:54-107), or flags for the rx=0 quirk
    int trx_zero;                   // dcomp leaves rx = 0 (theta > pi/2, phi in (pi/2, pi])
    double gex, gey, gez, ghx, ghy, ghz;     // projections gex..ghz of a unit field (source.c:131-165)
    const double *aux_e, *aux_h;
    int jres;
};
