// fdtd_kernels.cuh -- launch interface of the device kernels (fdtd_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd_internal.h"


struct DevAux {                 // 1D auxiliary grid of the TSF source (1dpool.c)
    double *e, *h;              // res values each
    double *bnd;                // 8 saved boundary values (Sv1DPool fbnx*)
    const double *wave;
    int nwave;
    int res;
    double ce, chh;             // (1/eps)*dt/(EPS0*dx1) and (1/mu)*dt/(MU0*dx1)
    double lc;                  // Liao factor (dt*c - dx1)/(dt*c + dx1)
    int *step;                  // device step counter
    // probes of the previous step
    int nprobes;
    const int64_t *probe_cells;
    const float *const *fields; // 6 pointers to the field set that holds the previous step
    double *probe_out;          // [p][nsteps][6]
    int nsteps_planned;
    int storage;                // FDTD_STORE_* of the fields
    float ihs;                  // 1 / H storage scale
};

// steps of E samples buffered per surface cell before they are folded into
// the FP64 accumulators (one accumulator read/write per NFFF_RING steps)
constexpr int NFFF_RING = 8;

struct DevNfff {
    int ns;                     // surface cells
    int nfreq;
    const int32_t *cell;        // linear index of the surface cell
    const int32_t *nstride;     // +/- stride along the face normal
    const float *const *e;      // 3 E field pointers (the set written by this step)
    double2 *acc;               // [(f*6 + q)*ns + s], q = Ex,Ey,Ez, dEx,dEy,dEz
    float *ring;                // NFFF_RING steps of raw samples [(slot*9 + 3a + r)*ns + s], r: E(c), E(c+st), E(c-st);
                                // FP32 elements (FP64 for FDTD_STORE_F64 plans)
    const double *omega_dt;     // nfreq
    const int *step;            // device step counter (already advanced)
    double inv2dx;
    int storage;                // FDTD_STORE_* of the fields
};

// a box of cells; its blocks are [first_block, next box's first_block), one cell
// (or one 4-cell group in a 4-cell list) per thread
struct SlabBox {
    int i0, i1, j0, j1, k0, k1;
    long long first_block;
    int inst;                   // plan of the box in a batched launch
    int tsf;                    // 1 if the box meets the TSF correction region [t0 - 1, t1] on every axis;
                                // the cells of other boxes skip the TSF test
};

void launch_aux_step(const DevAux &a, cudaStream_t st);

// Batched forms: one launch covers many plans whose per-plan parameters are
// device tables (of this step's parity), indexed by the plan number.
void launch_aux_step_batch(const DevAux *a, int nplans, cudaStream_t st);
void launch_tsf_faces_batch(const DevPlan *p, int nplans, int max_cells, cudaStream_t st);
// H over boxes (or boxes4 in 4-cell groups, nblocks4 > 0) and E over eboxes,
// the instances' runs of k planes with a dispersive cell (SlabLists::e)
// part: 1 the H kernel, 2 the E kernel over the dispersive runs, 3 both
cudaError_t launch_slab_steps_batch(const DevPlan *p, const SlabBox *boxes, int nboxes, long long nblocks,
                                    const SlabBox *boxes4, long long nblocks4, const SlabBox *eboxes, int neboxes,
                                    long long neblocks, bool ade, int npoles, int storage, cudaStream_t st, int part = 3);
// E over every instance's runs without a dispersive cell (SlabLists::ep)
cudaError_t launch_slab_e_plain_batch(const DevPlan *p, const SlabBox *boxes, int nboxes, long long nblocks, int storage,
                                      cudaStream_t st);
void launch_nfff_accumulate_batch(const DevNfff *n, int nplans, int max_cells, cudaStream_t st);
void launch_probe_capture(const DevAux &a, cudaStream_t st);
void launch_tsf_faces(const DevPlan &p, int total, cudaStream_t st);
// The slab work lists of a plan.  H runs over every slab box, in 4-cell
// groups when h4blocks > 0 (every k bound and the row length multiples of 4).
// E runs over the same cells split along k: `e` holds the runs of k planes
// with a dispersive cell (the plan's E variant), `ep` the runs without one
// (the plain E variant, fewer registers); without a split `e` is every box.
struct SlabLists {
    const SlabBox *h;
    int nh;
    long long hblocks;
    const SlabBox *h4;
    long long h4blocks;
    const SlabBox *e;
    int ne;
    long long eblocks;
    const SlabBox *ep;
    int nep;
    long long epblocks;
};
// part: 1 the H kernel, 2 the E kernels, 3 both (in that order)
cudaError_t launch_slab_steps(const DevPlan &p, const SlabLists &L, bool ade, int npoles, int storage, cudaStream_t st,
                              int part = 3);
void launch_nfff_accumulate(const DevNfff &n, cudaStream_t st);
// folds the samples of the steps since the last multiple of NFFF_RING into the
// accumulators and clears their ring slots; due before the accumulators are read
void launch_nfff_fold_pending(const DevNfff &n, cudaStream_t st);

struct DevFarfield {
    int npoints, nfreq, ns;
    const int32_t *points;      // 3*npoints
    const int32_t *istart;
    const int32_t *cell_ijk;    // 3*ns  (i,j,k of each surface cell)
    const int8_t *face;         // ns, 0..5 = x0 xn y0 yn z0 zn
    const double2 *acc;
    const double *omega;        // nfreq
    double dt, dx;
    double2 *out;               // [(p*nfreq + f)*3 + c]
    // tiled finalize
    int ntw;                    // twiddle entries per frequency
    const double2 *tw;          // [f*ntw + R] = exp(-i omega R dt)
    int groups;                 // surface-cell groups of the partial sums
    double2 *part;              // [((g*npoints + p)*nfreq + f)*3 + c] (scratch)
};

// The reference's own time-domain far-field series (farfield.c:175-405),
// accumulated exactly: three taps per (surface cell, far point) and step.
struct DevNfffSeries {
    int ns, npoints, ndata;
    const int32_t *cell;        // linear index of the surface cell
    const int32_t *nstride;     // +/- stride along the face normal
    const int32_t *cell_ijk;    // 3*ns
    const int8_t *face;         // ns
    const int32_t *points;      // 3*npoints
    const int32_t *istart;      // npoints
    const float *const *e;      // 3 E field pointers (the set written by this step)
    double *series;             // [(p*3 + c)*ndata + m]
    const int *step;            // device step counter (already advanced)
    double dx, dt;
    int storage;                // FDTD_STORE_* of the fields
};
void launch_nfff_series(const DevNfffSeries &s, cudaStream_t st);

void launch_farfield_finalize(const DevFarfield &f, cudaStream_t st);
