/*
 * gsvit_b200.h -- C ABI of the B200-native GSvit 3D FDTD stepping library.
 *
 * The library replaces the GPU side of GSvit's stepping loop: the worker-thread
 * driver src3d/gpu.c and the kernels of src3d/gpu_kernels.cu, whose own C
 * interface is the family of `cudaError_t wrap_*(SvGpuPlan*)` calls declared in
 * src3d/gpu_kernels.h:476-523 over the POD plan src3d/gpu_kernels.h:110-474.
 *
 * Everything here is plain C: fixed-width integers, doubles/floats, host
 * pointers and sizes.  The library owns all device memory.  Every call returns
 * an int status (FDTD_OK = 0, negative = error class) and never aborts; the
 * text of the last error of the calling thread is available from
 * fdtd_last_error().
 *
 * Data layout of every 3D host array crossing this boundary is the reference's
 * `data[i][j][k]` order with k (z) fastest (src3d/dcube.c:31-53), stored
 * contiguously: element (i,j,k) is at ((i*yres + j)*zres + k).
 *
 * The descriptor `fdtd_desc` is a flat copy of what GSvit's planner leaves in
 * SvSet/SvPool after init_and_make_plan() (src3d/plan.c:5442): grid and time
 * step, the material table (SvMatProp, src3d/settings.h:920-964, after the
 * epsilon/mu scaling of src3d/plan.c:4669-4698), the material index map and
 * voxel arrays (SvYeeData, src3d/yee.h:45-101), the CPML settings of
 * SvSetBoundary, the TSF source (SvSourceTSF + the waveform of
 * src3d/plan.c:1522-1597), the NFFF box and far points, and the probe list.
 */
#ifndef GSVIT_B200_H
#define GSVIT_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
#define FDTD_OK              0
#define FDTD_E_INVALID      -1   /* bad descriptor / argument */
#define FDTD_E_UNSUPPORTED  -2   /* feature outside the implemented path */
#define FDTD_E_CUDA         -3   /* CUDA runtime / driver error */
#define FDTD_E_NOMEM        -4   /* host or device allocation failed */
#define FDTD_E_STATE        -5   /* call out of order (e.g. not initialised) */
#define FDTD_E_TIMEOUT      -6   /* a bounded device wait gave up: that step's
                                  * fields are incomplete.  fdtd_sync and every
                                  * call that reads results back (fields, probes,
                                  * far field, snapshot, objective) report it;
                                  * the plan then refuses to step
                                  * (FDTD_E_STATE) and must be destroyed */

/* ---- material / mode codes (values of src3d/settings.h:103-123) -------- */
#define FDTD_MAT_LINEAR   0
#define FDTD_MAT_LINTAB   1
#define FDTD_MAT_DRUDE    2
#define FDTD_MAT_CP3      3
#define FDTD_MAT_CP       4
#define FDTD_MAT_ADE      5
#define FDTD_MAT_PLRC     6
#define FDTD_MAT_PEC     10

#define FDTD_MATMODE_NONE      0
#define FDTD_MATMODE_ELECTRIC  1
#define FDTD_MATMODE_MAGNETIC  2
#define FDTD_MATMODE_FULL      3

/* faces, in the order used by every per-face array below */
#define FDTD_FACE_X0 0
#define FDTD_FACE_XN 1
#define FDTD_FACE_Y0 2
#define FDTD_FACE_YN 3
#define FDTD_FACE_Z0 4
#define FDTD_FACE_ZN 5

/* field storage precision of the device copy (arithmetic is always FP32).
 * F16 / BF16 hold the six field components and the CPML psi slabs as 16-bit
 * numbers (H times 2^9, psi_H times the power of two nearest dx, psi_E times
 * that and 2^9); the Drude/critical-point state and the far-field
 * accumulators stay FP32/FP64.  BF16 stores round stochastically (a
 * deterministic hash of cell, array and step), F16 stores to nearest.  The
 * bulk kernel needs z rows of a multiple of 16 bytes (zres a multiple of 8
 * at 16 bits).  No counterpart in the reference, which stores FP32 on the GPU
 * (gpu.c:805-1172). */
#define FDTD_STORE_F32   0
#define FDTD_STORE_F16   1
#define FDTD_STORE_BF16  2
/* Reference precision: fields, psi slabs and the Drude/critical-point state
 * stored in FP64 and every update computed in FP64 from FP64 coefficient
 * tables, one thread per cell on the general kernels (the arithmetic of
 * GSvit's CPU path, yee.c:145-1247, boundary.c, source.c).  Meant for
 * pinning the FP32 and 16-bit runs at sizes the CPU oracle cannot reach; no
 * batches, no adjoint.  No counterpart in the reference's GPU path. */
#define FDTD_STORE_F64   3

/* field component bit mask (copy-in / copy-out), cf. SvGpuSync pool.h:49-54 */
#define FDTD_EX 0x01
#define FDTD_EY 0x02
#define FDTD_EZ 0x04
#define FDTD_HX 0x08
#define FDTD_HY 0x10
#define FDTD_HZ 0x20
#define FDTD_E   (FDTD_EX | FDTD_EY | FDTD_EZ)
#define FDTD_H   (FDTD_HX | FDTD_HY | FDTD_HZ)
#define FDTD_EH  (FDTD_E | FDTD_H)

/* derived integer maps that can be read back for bit-exact checks */
#define FDTD_MAP_MAT         0   /* material index  (SvYeeData.mat)        */
#define FDTD_MAP_BNDS        1   /* interface flag  (plan.c:5387-5416)     */
#define FDTD_MAP_SOURCESKIP  2   /* TSF skip flag   (plan.c:5298-5326)     */
#define FDTD_MAP_CLASS       3   /* per-cell coefficient class of the kernel */

/* One material, the post-plan SvMatProp (settings.h:920-964).  epsilon and mu
 * are absolute (already multiplied by EPSILON_0 / MU_0 as plan.c:4669-4698
 * does); the ade_* coefficients are those of calculate_ade_a/bp/c
 * (plan.c:2737-2763).  Only the types LINTAB, ADE and PEC are stepped by the
 * library; the other codes are rejected with FDTD_E_UNSUPPORTED. */
typedef struct fdtd_material {
    int32_t type;
    int32_t reserved;
    double epsilon, mu, sigma, sigast;
    double drude_omega_p, drude_nu;
    double cp_a[2], cp_phi[2], cp_omega[2], cp_gamma[2];
    double ade_a0, ade_a1, ade_a2;
    double ade_bp0[2], ade_bp1[2], ade_bp2[2], ade_bp3[2], ade_bp4[2];
    double ade_c0, ade_c1, ade_c2, ade_c3;
} fdtd_material;

/* CPML on one outer face (SvSetBoundary, settings.h; grading of
 * boundary.c:34-99).  sigma is sigma_max in S/m (the parser's automatic value
 * 0.8*(m+1)/(377*dx) must already be resolved), kappa is kappa_max, a is the
 * CFS alpha maximum. */
typedef struct fdtd_cpml_face {
    int32_t enabled;
    int32_t depth;
    int32_t m;
    int32_t reserved;
    double sigma, kappa, a;
} fdtd_cpml_face;

/* Total/scattered-field plane-wave source (SvSourceTSF, source.h;
 * set-up plan.c:1522-1597).  Angles in radians as the parser stores them. */
typedef struct fdtd_tsf {
    int32_t enabled;
    int32_t i0, j0, k0, in, jn, kn;     /* box corners, inclusive            */
    int32_t skip[6];                    /* TSF_SKIP per face (FDTD_FACE_*)   */
    int32_t skipdepth;                  /* TSF_SKIP depth; -1 = no skip map  */
    double theta, phi, psi;
    double layered_epsilon, layered_mu; /* relative, of the 1D aux grid      */
    int32_t nwave;                      /* number of waveform samples        */
    int32_t reserved;
    const double *wave;                 /* e[step] of the waveform file      */
} fdtd_tsf;

/* Near-to-far-field box and far points (settings.c:5621-5705, farfield.c).
 * The library accumulates, per surface cell and frequency, FP64 running DFTs
 * of E and dE/dn and integrates them to the far points at the end.  The
 * reference time-domain series (farfield.c:175-405) is the DFT of the same
 * sums; see fdtd_nfff_spectrum(). */
typedef struct fdtd_nfff {
    int32_t enabled;
    int32_t i0, j0, k0, in, jn, kn;     /* integration box                   */
    int32_t skip[6];                    /* NFFF_SKIP per face                */
    int32_t skip_lo[6][2];              /* per face: min of the 2 tangential indices */
    int32_t skip_hi[6][2];              /* per face: max of the 2 tangential indices */
    int32_t npoints;
    int32_t nfreq;                      /* running-DFT frequencies (0 = none)  */
    int32_t series;                     /* 1 = also accumulate the reference's
                                         * time-domain series (farfield.c:175-405)
                                         * exactly: cost O(npoints x surface) per
                                         * step, meant for few far points      */
    int32_t reserved;
    const int32_t *points;              /* 3*npoints far-point cells (ri,rj,rk) */
    const int32_t *istart;              /* npoints; NULL = farfield.c:76-91 rule */
    const double *omega;                /* nfreq angular frequencies (rad/s)  */
} fdtd_nfff;

/* Design region of the adjoint (no counterpart in the reference, which takes
 * per-cell permittivity only through voxel arrays or one material per cell):
 * the relative permittivity of every cell of a box of lossless, non-magnetic
 * dielectric cells, in double precision.  The cells keep their material
 * index (vacuum or a LINTAB material, whose epsilon is then ignored).  The
 * E coefficients of the box and of the cells one step above it on each axis
 * (which average epsilon over the cells sharing an edge, yee.c:1397-1493)
 * are held per cell; that box must lie outside every CPML slab and strictly
 * inside the TSF box, and the bulk kernel stays off for such plans. */
typedef struct fdtd_design {
    int32_t enabled;
    int32_t i0, i1, j0, j1, k0, k1;     /* half-open cell ranges            */
    int32_t reserved;
    const double *eps_r;                /* (i1-i0)*(j1-j0)*(k1-k0), k fastest */
} fdtd_design;

typedef struct fdtd_desc {
    int32_t abi_version;                /* FDTD_ABI_VERSION                  */
    int32_t xres, yres, zres;
    double dx, dy, dz, dt;
    int32_t nsteps;                     /* planned steps (probe storage)     */
    int32_t matmode;                    /* FDTD_MATMODE_*                    */
    int32_t nmat;                       /* 0 = no material table              */
    int32_t storage;                    /* FDTD_STORE_*                      */
    const fdtd_material *mats;          /* nmat entries, mats[0] = vacuum    */
    const int32_t *mat;                 /* N material indices or NULL        */
    const float *epsilon, *sigma;       /* N voxel values or NULL (matmode)  */
    const float *mu, *sigast;           /* N voxel values or NULL (matmode)  */
    fdtd_cpml_face cpml[6];
    fdtd_tsf tsf;
    fdtd_nfff nfff;
    int32_t nprobes;
    int32_t reserved;
    const int32_t *probes;              /* 3*nprobes cells (i,j,k)           */
    fdtd_design design;                 /* adjoint design region (optional)  */
} fdtd_desc;

typedef struct fdtd_plan fdtd_plan;

/* ---- lifetime ---------------------------------------------------------- */

/* Build the device plan: derived maps, coefficient classes, CPML profiles,
 * TSF/NFFF tables, device allocation and zeroed fields.  Replaces
 * sv_gpu_new (gpu.c:1960-2712) + sv_pool_gpu_init (gpu.c:46-57, device
 * allocation gpu.c:805-1172).  `device` is the CUDA ordinal. */
int fdtd_plan_create(const fdtd_desc *desc, int device, fdtd_plan **out);

/* Free everything the plan holds.  The reference has no counterpart. */
int fdtd_plan_destroy(fdtd_plan *plan);

/* Run subsequent work on a caller-supplied cudaStream_t (NULL = the plan's
 * own stream).  The reference synchronises after every launch
 * (gpu_kernels.cu:6063-6068); this library never synchronises implicitly. */
int fdtd_set_stream(fdtd_plan *plan, void *cuda_stream);

/* Block until the plan's queued work is finished (sv_pool_sync gpu.c:787-801). */
int fdtd_sync(fdtd_plan *plan);

/* ---- fields ------------------------------------------------------------ */

/* Host -> device copy of the selected components (mask of FDTD_EX..FDTD_HZ),
 * each a contiguous double array of N values; the double->float conversion of
 * sv_pool_gpu_copyto (gpu.c:629-685).  comps[c] may be NULL for unselected c. */
int fdtd_set_fields(fdtd_plan *plan, int mask, const double *const comps[6]);

/* Device -> host copy (sv_pool_gpu_copyfrom, gpu.c:687-785). */
int fdtd_get_fields(fdtd_plan *plan, int mask, double *const comps[6]);

/* Same as fdtd_get_fields but without widening: FP32 output. */
int fdtd_get_fields_f32(fdtd_plan *plan, int mask, float *const comps[6]);

/* Host -> device copy from FP32 arrays (used by end-to-end timing with
 * pinned host buffers). */
/* New relative permittivities of the design region's cells (dbox order, k
 * fastest); takes effect from the next step.  No counterpart in the reference. */
int fdtd_set_design_eps(fdtd_plan *plan, const double *eps_r);

int fdtd_set_fields_f32(fdtd_plan *plan, int mask, const float *const comps[6]);

/* ---- stepping ------------------------------------------------------------ */

/* Advance nsteps full time steps (H half-step, TSF, CPML, E half-step, probes,
 * NFFF accumulation), i.e. nsteps iterations of the GPU branch of the loop in
 * svit.c:240-256 (wrap_hKernel ... wrap_cpml_estep, farfield, outpoint). */
int fdtd_step(fdtd_plan *plan, int nsteps);

/* Same, captured once into a CUDA graph of `chunk` steps and replayed
 * (chunk rounded down to an even number >= 2; one graph per field-set
 * parity, kept until a call with another chunk or the plan's destruction;
 * the steps past the last whole chunk run as fdtd_step).  Bitwise equal to
 * fdtd_step and the faster of the two for long runs: 2.69 against 2.75 ms
 * a step on the 512^3 rough surface.  */
int fdtd_step_graph(fdtd_plan *plan, int nsteps, int chunk);

/* Same as fdtd_step, with its scratch in static device memory.  No
 * counterpart in the reference.  It is meant for callers that cannot call
 * cudaMalloc where they step: applications whose device memory belongs to
 * another allocator (a framework's caching allocator or a fixed budget), and
 * loops where cudaMalloc's implicit device-wide synchronisation would stall
 * other streams.  The only scratch of a step is the pair of TSF face
 * correction tables per face (written by one kernel of the step and read by
 * the Yee kernels of the same step); this entry point places them in one
 * file-scope static device array of FDTD_STATIC_SCRATCH_BYTES instead of
 * plan-owned buffers, and calls no allocator.  The caller still owns the plan
 * (inputs and outputs); every GPU that loads the library holds the 32 MiB
 * array until the process exits.
 *  - The first call on a device does set-up: it looks up the array's device
 *    address (with that device current) and keeps it for the life of the
 *    process.  Make that first call before any stream capture.  The kept
 *    address assumes the device is not reset (cudaDeviceReset) while the
 *    library stays loaded.
 *  - A plan whose tables need more than FDTD_STATIC_SCRATCH_BYTES (2 x 8 bytes
 *    per TSF face cell, each table rounded up to 256 bytes) is rejected with
 *    FDTD_E_UNSUPPORTED; the fields are left untouched.
 *  - The array keeps whatever the last call left in it.  Nothing in it has to
 *    start at zero: every entry a step reads was written earlier in that step.
 *  - There is one array per device.  Calls that overlap in time on the same
 *    device (plans on different streams or host threads) race on it. */
#define FDTD_STATIC_SCRATCH_BYTES (32u * 1024u * 1024u)
int fdtd_step_static_scratch(fdtd_plan *plan, int nsteps);

/* Current step counter (set->sc.step_act). */
int fdtd_get_step(const fdtd_plan *plan, int *step);

/* Run nsteps with CUDA events around every launch of the fused Yee kernel
 * only, and return their summed device time in milliseconds (profiling aid
 * for the roofline of the dominant kernel). */
int fdtd_step_timed(fdtd_plan *plan, int nsteps, double *fused_ms, int *fused_launches);

/* Per-kernel profile of nsteps steps (CUDA events around every launch):
 * out[0..1] = bulk kernel total ms / algorithmic bytes per launch,
 * out[2..3] = slab kernels (H+E) total ms / algorithmic bytes per launch,
 * out[4] = 1D aux grid + TSF face tables total ms, out[5] = NFFF running DFT
 * total ms, out[6] = all kernels of the steps total ms, out[7] = kernel
 * launches per step. */
int fdtd_step_profile(fdtd_plan *plan, int nsteps, double out[8]);

/* ---- outputs ------------------------------------------------------------- */

/* Probe series: out[(p*nsteps + step)*6 + c], c = Ex,Ey,Ez,Hx,Hy,Hz, for the
 * steps run so far (outpointdata layout of output.c:341-352, doubles). */
int fdtd_get_probes(fdtd_plan *plan, double *out, size_t out_len);

/* Far-field spectrum: for each far point p and frequency f the complex FP64
 * DFT  F_c(omega) = sum_m F_c[m] exp(-i omega m dt)  of the reference
 * time-domain far-field series F_c of farfield.c:175-405 (c = x,y,z),
 * out[((p*nfreq + f)*3 + c)*2 + {0,1}] = {re, im}. */
int fdtd_nfff_spectrum(fdtd_plan *plan, double *out, size_t out_len);

/* Length of the time-domain far-field series of a plan created with
 * nfff.series = 1: ndata = 2000 + 2*nsteps + |res|/(c dt/dx) (farfield.c:63-64). */
int fdtd_nfff_ndata(const fdtd_plan *plan, int *ndata);

/* The time-domain far-field series itself (rpoints[n].ex/ey/ez->data of
 * farfield.c), FP64: out[(p*3 + c)*ndata + m]. */
int fdtd_nfff_series(fdtd_plan *plan, double *out, size_t out_len);

/* Read back a derived integer map (FDTD_MAP_*) as N int32 values. */
int fdtd_get_map(fdtd_plan *plan, int which, int32_t *out, size_t out_len);

/* Number of distinct coefficient classes the plan derived. */
int fdtd_get_nclasses(const fdtd_plan *plan, int *nclasses);

/* ---- batches ---------------------------------------------------------------
 * No counterpart in the reference (GSvit steps one domain per process).  Many
 * independent plans -- instances of uneven size, material and source -- are
 * stepped in lockstep: each kernel of a step is one launch over all of them,
 * with per-instance parameter tables on the device (one launch per kernel
 * variant in use: no ADE, Drude, critical-point poles).  Each instance runs
 * the kernels it runs alone: the TMA tiles over its whole grid, one CTA per
 * tile of every such instance, or else a persistent bulk kernel that walks
 * the concatenated bulk work list, and the slab kernels.  Results are
 * bit-identical to the same plans stepped one by one. */
typedef struct fdtd_batch fdtd_batch;

/* Create nplans plans from descs[0..nplans) on one device and stream.  The
 * time-domain far-field series (nfff.series) is not available in a batch. */
int fdtd_batch_create(const fdtd_desc *descs, int nplans, int device, fdtd_batch **out);
int fdtd_batch_destroy(fdtd_batch *batch);
int fdtd_batch_size(const fdtd_batch *batch, int *nplans);
/* The plan of instance `index`, for fields, probes, far fields, maps and
 * snapshots; it is stepped only through the batch. */
int fdtd_batch_plan(fdtd_batch *batch, int index, fdtd_plan **plan);
/* Advance every instance by nsteps (eager launches / CUDA graph of `chunk`
 * steps, as fdtd_step and fdtd_step_graph). */
int fdtd_batch_step(fdtd_batch *batch, int nsteps);
int fdtd_batch_step_graph(fdtd_batch *batch, int nsteps, int chunk);
/* Wait for the batch; reports an expired bounded wait as FDTD_E_TIMEOUT. */
int fdtd_batch_sync(fdtd_batch *batch);
/* Autotuner: times trial_steps steps for each candidate work list of the
 * bulk kernel (planes per bulk item 8 / 16 / 32 / 64 / whole, persistent grid
 * or one CTA per item; it steps the instances without TMA tiles), keeps the
 * fastest and restores every instance's state.  report (if not NULL)
 * receives up to report_len/3 rows {planes (0 = whole), persistent, ms per
 * step}; *ncand the number of rows. */
int fdtd_batch_tune(fdtd_batch *batch, int trial_steps, double *report, int report_len, int *ncand);
/* The bulk work list in use: planes per item (0 = whole), persistent launch,
 * grid size and number of items. */
int fdtd_batch_config(const fdtd_batch *batch, int *planes_per_item, int *persistent, int *grid, int *items);
/* The CUDA stream (cudaStream_t) every launch of the batch goes to, so that a
 * caller can record events around its steps or order work after them. */
int fdtd_batch_get_stream(const fdtd_batch *batch, void **stream);

/* ---- checkpoint (forward snapshots) ---------------------------------------- */

/* Bytes needed for one snapshot of the complete stepping state (fields, CPML
 * psi slabs, ADE state, 1D aux grid, NFFF accumulators and the up to 8 steps
 * of surface samples not yet folded into them, step counter). */
int fdtd_snapshot_size(const fdtd_plan *plan, size_t *bytes);
/* Save / restore the state into / from a caller buffer (host memory). */
int fdtd_snapshot_save(fdtd_plan *plan, void *host_buf, size_t bytes);
int fdtd_snapshot_restore(fdtd_plan *plan, const void *host_buf, size_t bytes);

/* ---- diagnostics ----------------------------------------------------------- */

/* Last error text of the calling thread ("" if none). */
const char *fdtd_last_error(void);

/* Algorithmic HBM bytes of one full time step of this plan (fields, class
 * map, CPML slabs, ADE state, NFFF accumulators) -- the numerator of the
 * roofline figure. */
int fdtd_step_bytes(const fdtd_plan *plan, double *bytes);

/* ---- adjoint (no counterpart in the reference) --------------------------
 * Objective: far-field power at one running-DFT frequency over selected far
 * points, J = sum_t w_t (|F_x(p_t)|^2 + |F_y(p_t)|^2 + |F_z(p_t)|^2), with F
 * the spectrum of fdtd_nfff_spectrum(). */
typedef struct fdtd_objective {
    int32_t freq;                       /* index into nfff.omega             */
    int32_t npoints;
    const int32_t *points;              /* indices into nfff.points          */
    const double *weights;              /* npoints weights (e.g. solid angle) */
} fdtd_objective;

/* J of the far field accumulated so far. */
int fdtd_objective_value(fdtd_plan *plan, const fdtd_objective *obj, double *J);

/* Runs nsteps forward steps from the plan's current state, keeping a device
 * checkpoint of the full stepping state every `checkpoint` steps, evaluates
 * J, then the discrete adjoint of those steps backwards, recomputing each
 * segment of the forward run from its checkpoint (the lossy CPML makes the
 * step irreversible).  grad[c] = dJ/d eps_r of every design cell (dbox
 * order, k fastest).  Needs a design region, FP32 storage and the
 * running-DFT far field; Drude / critical-point materials outside the design
 * region are transposed with their polarisation state.  On return the plan holds the
 * forward state after nsteps.  Device memory: (nsteps/checkpoint + 1) copies
 * of the stepping state (fdtd_snapshot_size) plus checkpoint x 12 bytes per
 * cell of the design box. */
int fdtd_adjoint_gradient(fdtd_plan *plan, const fdtd_objective *obj, int nsteps, int checkpoint,
                          double *J, double *grad);

/* The transposed step applied nsteps times to an adjoint state (E then H
 * components, N values each, in place; psi adjoints start at zero): the
 * operator the gradient runs, exposed for checking against an independent
 * transpose. */
int fdtd_adjoint_transpose(fdtd_plan *plan, int nsteps, double *const comps[6]);

#ifdef __cplusplus
}
#endif

#endif /* GSVIT_B200_H */
