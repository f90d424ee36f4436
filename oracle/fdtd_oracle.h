/*
 * fdtd_oracle.h -- CPU restatement of GSvit's FP64 stepping loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests, smoke()
 * and the CPU-baseline leg of bench.py compare the CUDA path against.  The
 * product (gsvit_copy_b200/) never links, loads or calls it.
 *
 * It consumes the same flat descriptor as the CUDA library (include/gsvit_b200.h)
 * and restates, in double precision and in the reference's own order, the
 * CPU step sequence of src3d/svit.c:217-237:
 *   ystep_h (yee.c:146-265) -> TSF H (source.c:1421-1672 incl. 1dpool.c)
 *   -> CPML H (boundary.c:283-519) -> ystep_e (yee.c:530-1247)
 *   -> CPML E (boundary.c:522-884) -> TSF E (source.c:547-771)
 *   -> far field (farfield.c:175-405) -> probes (output.c:341-352).
 */
#ifndef FDTD_ORACLE_H
#define FDTD_ORACLE_H

#include "../include/gsvit_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_state oracle_state;

/* Build the state (derived maps, CPML profiles, TSF aux grid, far-field
 * geometry).  Returns NULL and fills err (if non-NULL, 256 bytes) on error. */
oracle_state *oracle_create(const fdtd_desc *desc, char *err);
void oracle_destroy(oracle_state *s);

/* Run nsteps full steps. */
int oracle_step(oracle_state *s, int nsteps);

/* Copy the six field arrays (N doubles each, [i][j][k]); NULL entries skipped. */
int oracle_get_fields(const oracle_state *s, double *ex, double *ey, double *ez,
                      double *hx, double *hy, double *hz);
int oracle_set_fields(oracle_state *s, const double *ex, const double *ey, const double *ez,
                      const double *hx, const double *hy, const double *hz);

/* Derived maps (FDTD_MAP_MAT / BNDS / SOURCESKIP) as N int32. */
int oracle_get_map(const oracle_state *s, int which, int32_t *out);

/* Probe series, layout out[(p*nsteps_planned + step)*6 + c]. */
int oracle_get_probes(const oracle_state *s, double *out);

/* Reference time-domain far-field series: out[(p*3 + c)*ndata + m]. */
int oracle_nfff_ndata(const oracle_state *s);
int oracle_get_nfff_series(const oracle_state *s, double *out);
/* istart per far point as the reference derives it (farfield.c:57-102). */
int oracle_get_nfff_istart(const oracle_state *s, int32_t *out);

/* 1D auxiliary grid state (e then h, res doubles each). */
int oracle_aux_res(const oracle_state *s);
int oracle_get_aux(const oracle_state *s, double *e, double *h);

int oracle_get_step(const oracle_state *s);

/* Coefficients of the source-free linear step (for the FP64 adjoint):
 * ca, cb: 3*N component-major; da, db: N; flags: N (bits 0-2 tbc, 3-5 PEC
 * zeroed components, 6 dispersive cell). */
int oracle_get_coeffs(const oracle_state *s, double *ca, double *cb, double *da, double *db, int32_t *flags);
int oracle_get_ade_mat(const oracle_state *s, int32_t *out);
/* Transpose of the far-field series of one step (the step index its
 * far-field call saw): out[a*N + c] += sum over the far points pts of the tap
 * coefficients that read E[a][c] times lam[(p*3 + a)*ndata + m]. */
int oracle_farfield_transpose(const oracle_state *s, int step, int npts, const int32_t *pts, const double *lam, double *out);
/* CPML profiles of a face; returns its depth (0 when disabled). */
int oracle_get_cpml(const oracle_state *s, int face, double *be, double *ce, double *bh, double *ch, double *ke, double *kh);

#ifdef __cplusplus
}
#endif
#endif
