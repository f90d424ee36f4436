// fdtd_adjoint.cuh -- discrete adjoint of the source-free step (fdtd_adjoint.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd_internal.h"
#include "fdtd_kernels.cuh"

// Adjoint state and scratch of one plan (FP32, the layouts of DevPlan).
struct DevAdj {
    float *eb[3], *hb[3];      // adjoints of E and H
    float *dd[6];              // adjoints of the six field differences of a half step
    float *pe[6][2];           // adjoints of psi_E (DevPlan::psie layout)
    float *ph[6][2];           // adjoints of psi_H (DevPlan::psih_in layout)
    // plans with dispersive cells: adjoints of the ADE state (the difference
    // form of DevAde), of E^{n-1} as the next step reads it, of Q, and of the
    // critical-point p and q (NULL without poles)
    float *ep[3], *q[3];
    float *pc[3][2], *qc[3][2];
};

// far-field objective: per surface cell and component the complex weights
// A_E, A_D of dJ/dv = 2 Re(exp(-i w n dt) A) (v = E and its normal difference)
struct DevObjective {
    int ns;
    const int32_t *cell, *nstride;
    double inv2dx, omega_dt;
    const double2 *ae, *ad;    // [c * ns + s]
};

// design box: per cell and component the accumulated dJ/dcb (FP64), the
// curl of H^{n+1/2} of the steps of one segment (FP32)
struct DevGrad {
    int box[6];
    int64_t ncell;
    double *g;                 // 3 per cell
    float *curl;               // [step][3 * ncell]
};

void launch_adjoint_e(const DevPlan &p, const DevAdj &a, cudaStream_t st);
void launch_adjoint_h(const DevPlan &p, const DevAdj &a, cudaStream_t st);
void launch_adjoint_source(const DevObjective &o, const DevAdj &a, int step, cudaStream_t st);
void launch_design_curl(const DevPlan &p, const DevGrad &g, int slot, cudaStream_t st);
void launch_design_accumulate(const DevAdj &a, const DevPlan &p, const DevGrad &g, int slot, cudaStream_t st);
// A_E, A_D of the objective from the final spectrum (DevFarfield geometry)
void launch_objective_weights(const DevFarfield &f, int freq, int npoints, const int32_t *points, const double *weights,
                              const double2 *spectrum, double2 *ae, double2 *ad, cudaStream_t st);
