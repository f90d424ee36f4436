// fdtd_api.cu -- the C ABI of include/gsvit_b200.h.
//
// Owns the device state of one plan and sequences the kernels of a step on a
// single CUDA stream.  The reference's GPU driver (gpu.c) keeps a worker
// thread per GPU, pushes one token per stage and spins on the host after
// every launch (gpu.c:787-801, gpu_kernels.cu:6063-6068); here a step is
// three stream-ordered launches with no host synchronisation, and
// fdtd_step_graph replays them from a CUDA graph.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gsvit_b200.h"
#include "fdtd_internal.h"
#include "fdtd_bulk.cuh"
#include "fdtd_kernels.cuh"
#include "fdtd_adjoint.cuh"
#include "plan_host.h"

namespace {

constexpr double C0 = 299792458.0;
constexpr double MU0 = 1.256637061435917295e-6;
constexpr double EPS0 = 8.854187817620389850e-12;
constexpr double PI_D = 3.1415926535897932384626433832795028841971693993751;

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define CK(x)                                                                                                   \
    do {                                                                                                        \
        cudaError_t e_ = (x);                                                                                   \
        if (e_ != cudaSuccess) return fail(FDTD_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));      \
    } while (0)

struct DevBuf {        // a list of device allocations freed with the plan
    std::vector<void *> ptrs;
    size_t bytes = 0;
    template <class T>
    cudaError_t alloc(T **p, size_t count)
    {
        void *q = nullptr;
        size_t b = count * sizeof(T);
        if (b == 0) b = 16;
        cudaError_t e = cudaMalloc(&q, b);
        if (e != cudaSuccess) return e;
        e = cudaMemset(q, 0, b);
        if (e != cudaSuccess) { cudaFree(q); return e; }
        ptrs.push_back(q);
        bytes += b;
        *p = (T *)q;
        return cudaSuccess;
    }
    void free_all()
    {
        for (void *p : ptrs) cudaFree(p);
        ptrs.clear();
    }
};

struct SnapItem {      // one contiguous device range that is part of the stepping state
    void *ptr;
    size_t bytes;
};

}  // namespace

struct fdtd_plan {
    HostPlan hp;
    int device = 0;
    int storage = FDTD_STORE_F32;  // element type of the fields and psi slabs
    size_t esz = 4;                // its size in bytes
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    DevBuf mem;
    float *fields[2][6] = {};      // ping-pong field sets
    float *psih[2][6][2] = {};     // ping-pong psi_H slabs
    int cur = 0;                   // set holding the latest state
    DevPlan dp;                    // template; fin/fout/psih set per launch
    DevAux aux;
    const float **d_fieldptrs[2] = {nullptr, nullptr};   // device copies of fields[s]
    int *d_step = nullptr;
    int host_step = 0;
    // work decomposition: slab kernels (CPML slabs, grid edges) and TMA bulk kernel
    SlabBox *d_boxes = nullptr;     // slab boxes (numbered one cell per thread)
    int nboxes = 0;
    long long nslab_blocks = 0;
    SlabBox *d_boxes4 = nullptr;    // the same numbered in 4-cell groups (H kernel), when all are 4-aligned
    long long nslab_blocks4 = 0;
    SlabLists slabs{};              // the lists above plus the E split (runs with / without dispersive cells)
    BulkItem *d_bulk = nullptr;
    int nbulk = 0;
    bool bulk_on = false;
    BulkMaps bmaps[2];
    // TMA tiles of the whole grid (single plans): bulk items of the interior
    // box and the CPML tiles around it (TILE_BULK / TILE_CPX / TILE_CPY / TILE_CPZ)
    bool tiles_on = false;
    BulkItem *d_tiles[NTILE] = {};
    int ntiles[NTILE] = {};
    BulkMaps tmaps[NTILE][2];
    std::vector<BulkItem> h_tiles[NTILE];   // host copies of the tile lists (batched launches)
    int stall = 0;                        // tests: expire every CTA's first wait after this many polls
    // the CPML tile kinds run beside the bulk kind: forked from the plan's
    // stream by an event, joined back before the NFFF step
    cudaStream_t side[NTILE] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[NTILE] = {};
    double tile_bytes[NTILE] = {};         // algorithmic HBM bytes per launch of each tile kind
    int *d_err = nullptr;                 // set by a bulk CTA whose bounded wait expired
    const int *batch_err = nullptr;       // the batch's error word, for an instance of a batch
    bool failed = false;                  // an expired wait was reported: the plan only accepts destroy
    int region[6] = {0, 0, 0, 0, 0, 0};   // bulk box Xlo Xhi Ylo Yhi Zlo Zhi
    std::vector<SlabBox> h_boxes;         // host copies of the work lists (batched launches)
    std::vector<SlabBox> h_eboxes;        // E runs with a dispersive cell (every box when unsplit)
    std::vector<SlabBox> h_epboxes;       // E runs without one
    std::vector<BulkItem> h_bulk;
    int bulk_len = 0;                     // planes per bulk item
    int tsf_cells = 0;                    // face cells of the TSF correction tables
    double bulk_bytes = 0, slab_bytes = 0; // algorithmic HBM bytes per launch
    // NFFF
    bool nfff = false;
    int nfff_npoints = 0, nfff_nfreq = 0, nfff_ns = 0;
    DevNfff nf;
    const float **d_efieldptrs[2] = {nullptr, nullptr};
    DevFarfield ff;
    std::vector<double> omega;
    bool nfff_series = false;             // time-domain series of farfield.c, exact
    DevNfffSeries ns;
    int nfff_ndata = 0;
    // graphs per parity
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_steps = 0;
    cudaStream_t graph_stream[2] = {nullptr, nullptr};
    std::vector<SnapItem> snap;
    double step_bytes = 0;
};

namespace {

// The device error words of a plan, read after its stream is synchronised.  A
// bulk CTA whose bounded wait expired left its cells of that step unwritten,
// so every later readback would return corrupt values: the readback reports
// FDTD_E_TIMEOUT instead and the plan refuses further steps.
int device_error(fdtd_plan *P)
{
    int err = 0;
    CK(cudaMemcpy(&err, P->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!err && P->batch_err) CK(cudaMemcpy(&err, P->batch_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        P->failed = true;
        return fail(FDTD_E_TIMEOUT, "a bounded wait of the bulk kernel expired; the fields are incomplete and the plan "
                                    "must be destroyed");
    }
    return FDTD_OK;
}

int refuse_failed(const fdtd_plan *P)
{
    return fail(FDTD_E_STATE, "a bounded device wait of this plan expired earlier; destroy the plan");
}

DevPlan plan_for(const fdtd_plan *P, int in)
{
    DevPlan d = P->dp;
    int out = 1 - in;
    for (int c = 0; c < 6; c++) {
        d.fin[c] = P->fields[in][c];
        d.fout[c] = P->fields[out][c];
    }
    for (int f = 0; f < 6; f++)
        for (int q = 0; q < 2; q++) {
            d.psih_in[f][q] = P->psih[in][f][q];
            d.psih_out[f][q] = P->psih[out][f][q];
        }
    return d;
}

// one launch of the tile kernel of `kind` (TILE_*) for this step's parity
int launch_tile_kind(fdtd_plan *P, const DevPlan &d, int in, int kind, cudaStream_t st)
{
    const cudaError_t e = launch_tiles(kind, d, P->tmaps[kind][in], P->d_tiles[kind], P->ntiles[kind], P->d_err,
                                       P->hp.has_ade, P->hp.maxpoles, P->storage, P->stall, st);
    if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("tile step launch: ") + cudaGetErrorString(e));
    return FDTD_OK;
}

// the Yee/CPML/TSF/ADE part of one step: the TMA tiles (bulk, then the CPML
// tiles; they touch disjoint cells and read only the input set), or, for
// plans without them, the bulk box and the slab kernels
int launch_fused(fdtd_plan *P, int in, cudaStream_t st)
{
    DevPlan d = plan_for(P, in);
    cudaError_t e;
    if (P->tiles_on) {
        // the four kinds touch disjoint cells and read only the input set:
        // the CPML kinds on side streams, so that each kind's last partial
        // wave of CTAs overlaps the others
        cudaError_t e = cudaEventRecord(P->ev_fork, st);
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("tile fork: ") + cudaGetErrorString(e));
        for (int kind = TILE_CPX; kind < NTILE; kind++) {
            if (!P->ntiles[kind]) continue;
            if ((e = cudaStreamWaitEvent(P->side[kind], P->ev_fork, 0)) != cudaSuccess)
                return fail(FDTD_E_CUDA, std::string("tile fork: ") + cudaGetErrorString(e));
            const int rc = launch_tile_kind(P, d, in, kind, P->side[kind]);
            if (rc != FDTD_OK) return rc;
            if ((e = cudaEventRecord(P->ev_join[kind], P->side[kind])) != cudaSuccess)
                return fail(FDTD_E_CUDA, std::string("tile join: ") + cudaGetErrorString(e));
        }
        const int rc = launch_tile_kind(P, d, in, TILE_BULK, st);
        if (rc != FDTD_OK) return rc;
        for (int kind = TILE_CPX; kind < NTILE; kind++) {
            if (!P->ntiles[kind]) continue;
            if ((e = cudaStreamWaitEvent(st, P->ev_join[kind], 0)) != cudaSuccess)
                return fail(FDTD_E_CUDA, std::string("tile join: ") + cudaGetErrorString(e));
        }
        return FDTD_OK;
    }
    if (P->bulk_on && P->side[TILE_CPX] && P->slabs.hblocks > 0) {
        // the slab H kernel beside the bulk kernel (disjoint cells, input set
        // only); the slab E kernels after both: they read H^{n+1/2} the bulk
        // kernel wrote next to the slabs
        if ((e = cudaEventRecord(P->ev_fork, st)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(P->side[TILE_CPX], P->ev_fork, 0)) != cudaSuccess)
            return fail(FDTD_E_CUDA, std::string("slab fork: ") + cudaGetErrorString(e));
        e = launch_slab_steps(d, P->slabs, P->hp.has_ade, P->hp.maxpoles, P->storage, P->side[TILE_CPX], 1);
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("slab step launch: ") + cudaGetErrorString(e));
        if ((e = cudaEventRecord(P->ev_join[TILE_CPX], P->side[TILE_CPX])) != cudaSuccess)
            return fail(FDTD_E_CUDA, std::string("slab join: ") + cudaGetErrorString(e));
        e = launch_tiles(TILE_BULK, d, P->bmaps[in], P->d_bulk, P->nbulk, P->d_err, P->hp.has_ade, P->hp.maxpoles,
                         P->storage, 0, st);
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("bulk step launch: ") + cudaGetErrorString(e));
        if ((e = cudaStreamWaitEvent(st, P->ev_join[TILE_CPX], 0)) != cudaSuccess)
            return fail(FDTD_E_CUDA, std::string("slab join: ") + cudaGetErrorString(e));
        e = launch_slab_steps(d, P->slabs, P->hp.has_ade, P->hp.maxpoles, P->storage, st, 2);
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("slab step launch: ") + cudaGetErrorString(e));
        return FDTD_OK;
    }
    if (P->bulk_on) {   // first: the slab E update reads H^{n+1/2} the bulk kernel wrote next to the slabs
        e = launch_tiles(TILE_BULK, d, P->bmaps[in], P->d_bulk, P->nbulk, P->d_err, P->hp.has_ade, P->hp.maxpoles,
                         P->storage, 0, st);
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("bulk step launch: ") + cudaGetErrorString(e));
    }
    e = launch_slab_steps(d, P->slabs, P->hp.has_ade, P->hp.maxpoles, P->storage, st);
    if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("slab step launch: ") + cudaGetErrorString(e));
    return FDTD_OK;
}

// NFFF work of a step: running DFT and/or the exact time-domain series,
// both reading the E set this step wrote
void launch_nfff(fdtd_plan *P, int in, cudaStream_t st)
{
    if (!P->nfff) return;
    if (P->nfff_nfreq > 0) {
        DevNfff n = P->nf;
        n.e = P->d_efieldptrs[1 - in];
        launch_nfff_accumulate(n, st);
    }
    if (P->nfff_series) {
        DevNfffSeries q = P->ns;
        q.e = P->d_efieldptrs[1 - in];
        launch_nfff_series(q, st);
    }
}

int launch_step(fdtd_plan *P, cudaStream_t st)
{
    const int in = P->cur;
    DevAux a = P->aux;
    a.fields = P->d_fieldptrs[in];
    launch_aux_step(a, st);
    if (P->tsf_cells) launch_tsf_faces(P->dp, P->tsf_cells, st);
    int rc = launch_fused(P, in, st);
    if (rc != FDTD_OK) return rc;
    launch_nfff(P, in, st);
    P->cur = 1 - in;
    return FDTD_OK;
}

int final_probes(fdtd_plan *P, cudaStream_t st)
{
    if (P->hp.probes.empty()) return FDTD_OK;
    DevAux a = P->aux;
    a.fields = P->d_fieldptrs[P->cur];
    launch_probe_capture(a, st);
    return FDTD_OK;
}

// Bulk work items of a plan: (j,k) tiles of the bulk box, planes cut into
// chunks of `len`, chunk-major so that CTAs that run together share planes in
// L2 (the halo rows/columns of neighbouring tiles are then served from L2).
std::vector<BulkItem> bulk_items(const int lo[3], const int hi[3], int len, int inst)
{
    std::vector<BulkItem> blk;
    for (int ib = lo[0]; ib < hi[0]; ib += len)
        for (int j0 = lo[1]; j0 < hi[1]; j0 += BULK_TJ)
            for (int k0 = lo[2]; k0 < hi[2]; k0 += BULK_TK)
                blk.push_back({j0, k0, ib, std::min(hi[0], ib + len), lo[1], hi[1], lo[2], hi[2], inst, 0});
    return blk;
}


int plan_create_impl(const fdtd_desc *desc, int device, fdtd_plan **out, bool pole_arrays);

// The largest run [a, b) of indices along one axis whose cells take the plain
// update (hp.ike/ikh of 1, outside the CPML psi ranges of boundary.c:347-519
// and 691-884, off the edge planes).  H is special below depth - 1 and from
// res - depth + 1 up, E below depth and from res - depth + 1 up; both at the
// first and last index.
void plain_run(const HostPlan &hp, int ax, int R, int *a, int *b, bool *hplain_below)
{
    const fdtd_cpml_face &lo = hp.cp[2 * ax], &hi = hp.cp[2 * ax + 1];
    auto hpl = [&](int q) {
        if (q < 0 || q >= R - 1) return false;
        if (lo.enabled && q < lo.depth - 1) return false;
        if (hi.enabled && q >= R - hi.depth + 1) return false;
        return hp.ikh[ax][q] == 1.0f;
    };
    auto epl = [&](int q) {
        if (q <= 0 || q >= R - 1) return false;
        if (lo.enabled && q < lo.depth) return false;
        if (hi.enabled && q >= R - hi.depth + 1) return false;
        return hp.ike[ax][q] == 1.0f;
    };
    int ba = 0, bb = 0;
    for (int q = 0; q < R;) {
        if (!(hpl(q) && epl(q))) { q++; continue; }
        int e = q;
        while (e < R && hpl(e) && epl(e)) e++;
        if (e - q > bb - ba) { ba = q; bb = e; }
        q = e;
    }
    *a = ba;
    *b = bb;
    *hplain_below = ba > 0 && hpl(ba - 1);
}

// planes [a0, a1) cut into chunks of about `target` planes
std::vector<std::pair<int, int>> plane_chunks(int a0, int a1, int target)
{
    std::vector<std::pair<int, int>> out;
    if (a1 <= a0) return out;
    const int nch = std::max(1, (a1 - a0 + target - 1) / target);
    const int len = (a1 - a0 + nch - 1) / nch;
    for (int i = a0; i < a1; i += len) out.push_back({i, std::min(a1, i + len)});
    return out;
}

// (j,k) tiles of [jlo, jhi) x [klo, khi) with tj x tk own cells, over the
// plane chunks.  jend / kend: the tiles end at jhi / khi, so that the first
// one may start below jlo / klo (its rows or groups there supply halo values
// only); otherwise they start at jlo / klo and the last one ends past jhi / khi.
void push_tiles(std::vector<BulkItem> &v, const std::vector<std::pair<int, int>> &ch, int jlo, int jhi, int klo, int khi,
                int tj, int tk, bool jend = false, bool kend = false)
{
    if (jlo >= jhi || klo >= khi) return;
    // a region starting at the grid's first row (group) needs own rows from
    // row 1 (k 4) only: the tile starting there owns its halo row 0 (group 0)
    const int j1 = jlo == 0 ? 1 : jlo, k1 = klo == 0 ? 4 : klo;
    const int js = jend ? jhi - std::max(1, (jhi - j1 + tj - 1) / tj) * tj : jlo;
    const int ks = kend ? khi - std::max(1, (khi - k1 + tk - 1) / tk) * tk : klo;
    for (const auto &c : ch)
        for (int j0 = js; j0 < jhi; j0 += tj)
            for (int k0 = ks; k0 < khi; k0 += tk) v.push_back({j0, k0, c.first, c.second, jlo, jhi, klo, khi, 0, 0});
}

template <class T>
cudaError_t upload(DevBuf &m, T **dst, const T *src, size_t count)
{
    cudaError_t e = m.alloc(dst, count);
    if (e != cudaSuccess || count == 0) return e;
    return cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice);
}

}  // namespace

extern "C" {

const char *fdtd_last_error(void) { return g_err.c_str(); }

int fdtd_plan_create(const fdtd_desc *desc, int device, fdtd_plan **out) { return plan_create_impl(desc, device, out, false); }

}  // extern "C"

namespace {

// pole_arrays: allocate the critical-point state even for a Drude-only plan,
// so that a batched launch may run it with the two-pole kernel variant
// Work lists of the TMA tile kernels for a single plan.  The interior box
// (every index plain on every axis, the bulk tile's halo row, group and plane
// plain for H) goes to the bulk layout, its last tiles partial; the rest of
// the grid to the CPML layouts: whole planes of the x slabs and rows of the y
// slabs in 15 x 60 tiles, the z slabs between the y slabs in 31 x 28 tiles.
// The CPML tiles below the box end at its first row / k cell, so that the
// part of them past the grid's low edge is the idle one.  Sets
// DevPlan::plo/phi, uploads the lists and encodes the tensor maps of the
// three layouts.
int build_tiles(fdtd_plan *P, const HostPlan &hp, DevPlan &d, const uint8_t *cls)
{
    const int X = hp.xr, Y = hp.yr, Z = hp.zr;
    const int R[3] = {X, Y, Z};
    int a[3], b[3];
    bool below[3];
    for (int ax = 0; ax < 3; ax++) {
        plain_run(hp, ax, R[ax], &a[ax], &b[ax], &below[ax]);
        d.plo[ax] = a[ax];
        d.phi[ax] = b[ax];
    }
    // bulk box: H of the plane / row below its first one must be plain too; k
    // bounds multiples of 4 with a plain 4-cell halo group below
    int lo[3], hi[3];
    for (int ax = 0; ax < 3; ax++) {
        lo[ax] = below[ax] ? a[ax] : a[ax] + 1;
        hi[ax] = b[ax];
    }
    lo[2] = (lo[2] + 3) / 4 * 4;
    while (lo[2] < hi[2] && !(lo[2] - 4 >= a[2] - (below[2] ? 1 : 0))) lo[2] += 4;
    hi[2] = hi[2] / 4 * 4;
    int bi0 = lo[0], bi1 = hi[0], bj0 = lo[1], bj1 = hi[1], bk0 = lo[2], bk1 = hi[2];
    // the z slabs in whole z tiles: the first starts at k0 = 4 and owns the
    // group at k = 0 (CPZ_TK + 4 cells), the last ends at the grid's edge; the
    // plain cells they take from the interior box fill lanes that would idle
    // (only while the box keeps at least one bulk tile's width of k).  At
    // 512^3 with 16-cell CPML this also keeps the TSF box's z faces (k = 24,
    // 488) out of the bulk tiles, whose per-cell path they would take in
    // every column: 34 x 20 z tiles (box from k = 24) ran the z kind in 0.48
    // instead of 0.64 ms but the bulk kind in 1.67 instead of 1.45 ms.
    {
        const int a0 = bk0 > 0 ? 4 + (bk0 - 4 + CPZ_TK - 1) / CPZ_TK * CPZ_TK : bk0;
        const int a1 = bk1 < Z ? Z - (Z - bk1 + CPZ_TK - 1) / CPZ_TK * CPZ_TK : bk1;
        if (a1 - a0 >= BULK_TK) { bk0 = a0; bk1 = a1; }
    }
    const bool bulk = bi0 < bi1 && bj0 < bj1 && bk0 < bk1;
    // design cells (per-cell E coefficients) are handled by the bulk layout
    // only: a plan whose design cells reach outside the interior box keeps the
    // slab kernels
    if (hp.design && !(bulk && hp.abox[0] >= bi0 && hp.abox[1] <= bi1 && hp.abox[2] >= bj0 && hp.abox[3] <= bj1 &&
                       hp.abox[4] >= bk0 && hp.abox[5] <= bk1)) {
        P->tiles_on = false;
        return FDTD_OK;
    }
    std::vector<BulkItem> it[NTILE];
    // planes per item: about 10 in the bulk (neighbouring tiles then share
    // their halo rows in L2; 512^3 rough surface, bulk kernel 2.24 ms at 96
    // planes, 1.72 ms at 8-12, 1.79 ms at 4), whole x slabs, 16 in the y and z
    // CPML tiles
    if (bulk) {
        push_tiles(it[TILE_BULK], plane_chunks(bi0, bi1, 10), bj0, bj1, bk0, bk1, BULK_TJ, BULK_TK);
        const auto xs0 = plane_chunks(0, bi0, 1 << 30), xs1 = plane_chunks(bi1, X, 1 << 30);
        push_tiles(it[TILE_CPX], xs0, 0, Y, 0, Z, CPXY_TJ, CPXY_TK);
        push_tiles(it[TILE_CPX], xs1, 0, Y, 0, Z, CPXY_TJ, CPXY_TK);
        const auto mid = plane_chunks(bi0, bi1, 16);
        push_tiles(it[TILE_CPY], mid, 0, bj0, 0, Z, CPXY_TJ, CPXY_TK, true, false);
        push_tiles(it[TILE_CPY], mid, bj1, Y, 0, Z, CPXY_TJ, CPXY_TK);
        push_tiles(it[TILE_CPZ], mid, bj0, bj1, 0, bk0, CPZ_TJ, CPZ_TK, false, true);
        push_tiles(it[TILE_CPZ], mid, bj0, bj1, bk1, Z, CPZ_TJ, CPZ_TK);
    } else {
        bi0 = bi1 = bj0 = bj1 = bk0 = bk1 = 0;
        push_tiles(it[TILE_CPX], plane_chunks(0, X, 16), 0, Y, 0, Z, CPXY_TJ, CPXY_TK);
    }
    // algorithmic bytes per launch: fields 12 x esz + class byte per cell, the
    // dispersive state of dispersive components, 4 psi values read and written
    // per CPML cell (psi arrays, charged to the CPML tiles)
    const double esz = (double)P->esz;
    auto box_bytes = [&](int i0, int i1, int j0, int j1, int k0, int k1) {
        double bsum = 0;
        if (i0 >= i1 || j0 >= j1 || k0 >= k1) return bsum;
#pragma omp parallel for reduction(+ : bsum) schedule(static)
        for (int i = i0; i < i1; i++)
            for (int j = j0; j < j1; j++)
                for (int k = k0; k < k1; k++) {
                    const DevClass &c = hp.classes[hp.cls[((size_t)i * Y + j) * Z + k]];
                    bsum += 12.0 * esz + 1.0;
                    if (c.flags & CF_ADE_BRANCH)
                        bsum += (((c.flags & CF_ADE_X) ? 1 : 0) + ((c.flags & CF_ADE_Y) ? 1 : 0) + ((c.flags & CF_ADE_Z) ? 1 : 0)) *
                                (8.0 + esz + 16.0 * hp.maxpoles);
                }
        return bsum;
    };
    const double all = box_bytes(0, X, 0, Y, 0, Z);
    P->tile_bytes[TILE_BULK] = box_bytes(bi0, bi1, bj0, bj1, bk0, bk1);
    P->tile_bytes[TILE_CPZ] = box_bytes(bi0, bi1, bj0, bj1, 0, bk0) + box_bytes(bi0, bi1, bj0, bj1, bk1, Z);
    P->tile_bytes[TILE_CPY] = box_bytes(bi0, bi1, 0, bj0, 0, Z) + box_bytes(bi0, bi1, bj1, Y, 0, Z);
    P->tile_bytes[TILE_CPX] = all - P->tile_bytes[TILE_BULK] - P->tile_bytes[TILE_CPZ] - P->tile_bytes[TILE_CPY];
    // psi values: charged to the CPML kinds by the cells of each slab they hold
    for (int f = 0; f < 6; f++)
        if (hp.cp[f].enabled) {
            const int dep = hp.cp[f].depth;
            const double per = 4 * 2.0 * esz;
            if (f < 2) P->tile_bytes[TILE_CPX] += (double)dep * Y * Z * per;
            else if (f < 4) {   // y slabs: the x-slab planes belong to CPX
                P->tile_bytes[TILE_CPX] += (double)(X - (bi1 - bi0)) * dep * Z * per;
                P->tile_bytes[TILE_CPY] += (double)(bi1 - bi0) * dep * Z * per;
            } else {   // z slabs: CPX planes, CPY rows, CPZ the rest
                P->tile_bytes[TILE_CPX] += (double)(X - (bi1 - bi0)) * Y * dep * per;
                P->tile_bytes[TILE_CPY] += (double)(bi1 - bi0) * (Y - (bj1 - bj0)) * dep * per;
                P->tile_bytes[TILE_CPZ] += (double)(bi1 - bi0) * (bj1 - bj0) * dep * per;
            }
        }
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || !fn || q != cudaDriverEntryPointSuccess) return fail(FDTD_E_CUDA, "cuTensorMapEncodeTiled entry point");
    for (int kind = 0; kind < NTILE; kind++) {
        P->ntiles[kind] = (int)it[kind].size();
        P->h_tiles[kind] = it[kind];
        if (it[kind].empty()) continue;
        e = upload(P->mem, &P->d_tiles[kind], it[kind].data(), it[kind].size());
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("tile work lists: ") + cudaGetErrorString(e));
        for (int sset = 0; sset < 2; sset++)
            if (tile_make_maps(kind, fn, d, P->fields[sset], cls, d.cpitch, P->storage, &P->tmaps[kind][sset]) != 0)
                return fail(FDTD_E_CUDA, "tensor map encoding");
    }
    e = bulk_configure();
    if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("tile kernel shared memory: ") + cudaGetErrorString(e));
    return FDTD_OK;
}

int plan_create_impl(const fdtd_desc *desc, int device, fdtd_plan **out, bool pole_arrays)
{
    if (!out) return fail(FDTD_E_INVALID, "out is NULL");
    *out = nullptr;
    if (!desc) return fail(FDTD_E_INVALID, "desc is NULL");
    fdtd_plan *P = new (std::nothrow) fdtd_plan();
    if (!P) return fail(FDTD_E_NOMEM, "host allocation failed");
    std::string err;
    int rc = build_host_plan(desc, &P->hp, &err);
    if (rc != FDTD_OK) {
        delete P;
        return fail(rc, err);
    }
    HostPlan &hp = P->hp;
    if (pole_arrays && hp.has_ade) hp.maxpoles = 2;
    P->storage = desc->storage;
    P->esz = desc->storage == FDTD_STORE_F32 ? 4 : desc->storage == FDTD_STORE_F64 ? 8 : 2;
    const size_t esz = P->esz;
    P->device = device;
    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) { delete P; return fail(FDTD_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce)); }
    auto release = [&]() {
        for (int k = 0; k < NTILE; k++) {
            if (P->side[k]) cudaStreamDestroy(P->side[k]);
            if (P->ev_join[k]) cudaEventDestroy(P->ev_join[k]);
        }
        if (P->ev_fork) cudaEventDestroy(P->ev_fork);
        P->mem.free_all();
        if (P->own_stream) cudaStreamDestroy(P->own_stream);
        delete P;
    };
    auto bail = [&](cudaError_t e, const char *what) {
        release();
        return fail(e == cudaErrorMemoryAllocation ? FDTD_E_NOMEM : FDTD_E_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
    };
    auto bail_rc = [&](int rc) {   // the error text is already set
        release();
        return rc;
    };
#define CA(x, what) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return bail(e_, what); } while (0)
    CA(cudaStreamCreateWithFlags(&P->own_stream, cudaStreamNonBlocking), "stream");
    P->stream = P->own_stream;
    const size_t n = hp.n;
    DevPlan &d = P->dp;
    std::memset(&d, 0, sizeof(d));
    d.xr = hp.xr; d.yr = hp.yr; d.zr = hp.zr;
    d.sj = hp.zr;
    d.si = (int64_t)hp.yr * hp.zr;
    d.dx = (float)hp.dx;
    d.dxd = hp.dx;
    const bool r64 = P->storage == FDTD_STORE_F64;   // FP64 fields, state, tables and arithmetic
    d.real64 = r64 ? 1 : 0;
    const size_t rsz = r64 ? 8 : 4;                  // element size of the ADE state and the tables
    // an FP64 table (r64) or its FP32 twin, uploaded behind a float pointer
    auto upload_tab = [&](float **dst, const std::vector<float> &f32, const std::vector<double> &f64) {
        if (!r64) return upload(P->mem, dst, f32.data(), f32.size());
        double *q = nullptr;
        cudaError_t e = upload(P->mem, &q, f64.data(), f64.size());
        *dst = reinterpret_cast<float *>(q);
        return e;
    };
    // 16-bit storage scales, chosen so that every stored value of a field of
    // unit amplitude is of order one: H ~ E / Z0 (Z0 = 377 ohm) is stored
    // times 2^9; psi_H accumulates dE/dx ~ E / dx and is stored times the
    // power of two nearest dx; psi_E accumulates dH/dx and is stored times
    // that and 2^9.  Powers of two make scaling and unscaling exact.
    d.hs = 1.f; d.ihs = 1.f; d.ps = 1.f; d.ips = 1.f; d.pse = 1.f; d.ipse = 1.f;
    if (P->storage == FDTD_STORE_F16 || P->storage == FDTD_STORE_BF16) {
        const int e2 = std::max(-100, std::min(100, (int)std::lround(std::log2(hp.dx))));
        d.hs = 512.f;
        d.ihs = 1.f / 512.f;
        d.ps = std::ldexp(1.f, e2);
        d.ips = std::ldexp(1.f, -e2);
        d.pse = std::ldexp(1.f, e2 + 9);
        d.ipse = std::ldexp(1.f, -e2 - 9);
    }
    // a field or psi array of `cnt` elements of the storage type, in float units
    auto store_alloc = [&](float **ptr, size_t cnt) { return P->mem.alloc(ptr, (cnt * esz + 3) / 4); };
    for (int s = 0; s < 2; s++)
        for (int c = 0; c < 6; c++) {
            CA(store_alloc(&P->fields[s][c], n), "field allocation");
            P->snap.push_back({P->fields[s][c], n * esz});
        }
    uint8_t *cls;
    {
        const int pitch = (hp.zr + 15) / 16 * 16;   // TMA row pitch must be a multiple of 16 bytes
        std::vector<uint8_t> padded((size_t)hp.xr * hp.yr * pitch, 0);
        for (size_t row = 0; row < (size_t)hp.xr * hp.yr; row++)
            std::memcpy(&padded[row * pitch], &hp.cls[row * hp.zr], hp.zr);
        CA(upload(P->mem, &cls, padded.data(), padded.size()), "class map");
        d.cpitch = pitch;
    }
    d.cls = cls;
    if (r64) {
        DevClass64 *classes;
        CA(upload(P->mem, &classes, hp.classes64.data(), hp.classes64.size()), "class table");
        d.classes = reinterpret_cast<const DevClass *>(classes);
    } else {
        DevClass *classes;
        CA(upload(P->mem, &classes, hp.classes.data(), hp.classes.size()), "class table");
        d.classes = classes;
    }
    d.nclasses = (int)hp.classes.size();
    if (hp.design) {
        float *dc;
        CA(upload_tab(&dc, hp.dcoef, hp.dcoef64), "design coefficients");
        d.dcoef = dc;
        for (int q = 0; q < 6; q++) d.dbox[q] = hp.abox[q];
    }
    double bytes = (12.0 * esz + 1.0) * (double)n;   // 6 field reads + 6 writes + class byte
    if (hp.has_ade) {
        if (r64) {
            DevAde64 *ade;
            CA(upload(P->mem, &ade, hp.ades64.data(), hp.ades64.size()), "ADE table");
            d.ade = reinterpret_cast<const DevAde *>(ade);
        } else {
            DevAde *ade;
            CA(upload(P->mem, &ade, hp.ades.data(), hp.ades.size()), "ADE table");
            d.ade = ade;
        }
        d.nade = (int)hp.ades.size();
        const size_t nst = n * rsz / 4;   // state array in float units
        for (int a = 0; a < 3; a++) {
            CA(P->mem.alloc(&d.q[a], nst), "ADE state");
            P->snap.push_back({d.q[a], n * rsz});
            for (int q = 0; q < hp.maxpoles; q++) {
                CA(P->mem.alloc(&d.pc[a][q], nst), "ADE state");
                CA(P->mem.alloc(&d.qc[a][q], nst), "ADE state");
                P->snap.push_back({d.pc[a][q], n * rsz}); P->snap.push_back({d.qc[a][q], n * rsz});
            }
        }
        size_t nd = 0;   // dispersive components: Q read + written (8 B), E^{n-1} read, + 16 B per pole (p, q)
        for (size_t c = 0; c < n; c++) {
            const DevClass &k = hp.classes[hp.cls[c]];
            if (k.flags & CF_ADE_BRANCH)
                nd += ((k.flags & CF_ADE_X) ? 1 : 0) + ((k.flags & CF_ADE_Y) ? 1 : 0) + ((k.flags & CF_ADE_Z) ? 1 : 0);
        }
        bytes += (double)nd * (2.0 * rsz + esz + 4.0 * rsz * hp.maxpoles);
    }
    // CPML
    for (int f = 0; f < 6; f++) {
        d.cp_on[f] = hp.cp[f].enabled;
        d.cp_d[f] = hp.cp[f].depth;
        if (!hp.cp[f].enabled) continue;
        const int dep = hp.cp[f].depth;
        float *be, *ce, *bh, *ch;
        CA(upload_tab(&be, hp.be[f], hp.be64[f]), "cpml");
        CA(upload_tab(&ce, hp.ce[f], hp.ce64[f]), "cpml");
        CA(upload_tab(&bh, hp.bh[f], hp.bh64[f]), "cpml");
        CA(upload_tab(&ch, hp.ch[f], hp.ch64[f]), "cpml");
        d.be[f] = be; d.ce[f] = ce; d.bh[f] = bh; d.ch[f] = ch;
        size_t cnt = (f < 2) ? (size_t)dep * hp.yr * hp.zr : (f < 4) ? (size_t)hp.xr * dep * hp.zr : (size_t)hp.xr * hp.yr * dep;
        for (int q = 0; q < 2; q++) {
            CA(store_alloc(&d.psie[f][q], cnt), "cpml psi");
            P->snap.push_back({d.psie[f][q], cnt * esz});
            for (int s = 0; s < 2; s++) {
                CA(store_alloc(&P->psih[s][f][q], cnt), "cpml psi");
                P->snap.push_back({P->psih[s][f][q], cnt * esz});
            }
        }
        bytes += (double)cnt * esz * 2 * 4;   // 4 psi arrays read + written
    }
    for (int ax = 0; ax < 3; ax++) {
        float *a, *b;
        CA(upload_tab(&a, hp.ike[ax], hp.ike64[ax]), "kappa");
        CA(upload_tab(&b, hp.ikh[ax], hp.ikh64[ax]), "kappa");
        d.ike[ax] = a;
        d.ikh[ax] = b;
    }
    // TSF
    std::memset(&P->aux, 0, sizeof(P->aux));
    CA(P->mem.alloc(&P->d_step, 1), "step counter");
    P->snap.push_back({P->d_step, sizeof(int)});
    P->aux.step = P->d_step;
    d.stepc = P->d_step;
    P->aux.storage = P->storage;
    P->aux.ihs = d.ihs;
    d.tsf_on = hp.tsf;
    if (hp.tsf) {
        const fdtd_tsf &t = desc->tsf;
        d.t0[0] = t.i0; d.t0[1] = t.j0; d.t0[2] = t.k0;
        d.t1[0] = t.in; d.t1[1] = t.jn; d.t1[2] = t.kn;
        for (int f = 0; f < 6; f++) {
            d.tskip[f] = t.skip[f];
            uint8_t *m;
            CA(upload(P->mem, &m, hp.tmap[f].data(), hp.tmap[f].size()), "tsf map");
            d.tmap[f] = m;
            CA(P->mem.alloc(&d.tcor_h[f], hp.tmap[f].size() * rsz / 4), "tsf corrections");   // float2 / double2
            CA(P->mem.alloc(&d.tcor_e[f], hp.tmap[f].size() * rsz / 4), "tsf corrections");
            d.tnb[f] = hp.tmap_dims[f][1];
            P->tsf_cells += (int)hp.tmap[f].size();
        }
        d.corr = hp.corr;
        d.hcor = hp.dt / hp.dx / MU0;
        const double th = t.theta, ph = t.phi, ps = t.psi;
        d.tax = std::sin(th) * std::cos(ph);
        d.tay = std::sin(th) * std::sin(ph);
        d.taz = std::cos(th);
        // corner selection of dcomp, source.c:63-102
        int ox = 0, oy = 0, oz = 0, rxz = 0;
        const int X = hp.xr, Y = hp.yr, Z = hp.zr;
        if (th >= 0 && th <= PI_D / 2.0) {
            oz = 0;
            if (ph >= 0 && ph <= PI_D / 2.0) { ox = 0; oy = 0; }
            else if (ph > PI_D / 2.0 && ph <= PI_D) { ox = X; oy = 0; }
            else if (ph > PI_D && ph <= 3.0 * PI_D / 2.0) { ox = X; oy = Y; }
            else { ox = 0; oy = Y; }
        } else {
            oz = Z;
            if (ph >= 0 && ph <= PI_D / 2.0) { ox = 0; oy = 0; }
            else if (ph > PI_D / 2.0 && ph <= PI_D) { rxz = 1; oy = 0; }
            else if (ph > PI_D && ph <= 3.0 * PI_D / 2.0) { ox = X; oy = Y; }
            else { ox = 0; oy = Y; }
        }
        d.trx_origin = ox; d.try_origin = oy; d.trz_origin = oz; d.trx_zero = rxz;
        // projections of source.c:131-165 for a unit field
        d.gex = (std::cos(ps) * std::sin(ph) - std::sin(ps) * std::cos(th) * std::cos(ph));
        d.gey = (-std::cos(ps) * std::cos(ph) - std::sin(ps) * std::cos(th) * std::sin(ph));
        d.gez = (std::sin(ps) * std::sin(th));
        d.ghx = (std::sin(ps) * std::sin(ph) + std::cos(ps) * std::cos(th) * std::cos(ph));
        d.ghy = (-std::sin(ps) * std::cos(ph) + std::cos(ps) * std::cos(th) * std::sin(ph));
        d.ghz = (-std::cos(ps) * std::sin(th));
        double *ae, *ah, *bnd, *wave;
        CA(P->mem.alloc(&ae, (size_t)hp.jres + 4), "aux");   /* dval may touch data[res] (dline.c:104) */
        CA(P->mem.alloc(&ah, (size_t)hp.jres + 4), "aux");
        CA(P->mem.alloc(&bnd, 8), "aux");
        CA(upload(P->mem, &wave, hp.wave.data(), hp.wave.size()), "wave");
        P->snap.push_back({ae, (size_t)hp.jres * 8}); P->snap.push_back({ah, (size_t)hp.jres * 8}); P->snap.push_back({bnd, (size_t)64});
        d.aux_e = ae; d.aux_h = ah; d.jres = hp.jres;
        P->aux.e = ae; P->aux.h = ah; P->aux.bnd = bnd; P->aux.wave = wave;
        P->aux.nwave = (int)hp.wave.size();
        P->aux.res = hp.jres;
        const double multe = hp.dt / (EPS0 * hp.jdx) / 1;
        const double multh = hp.dt / (MU0 * hp.jdx) / 1;
        P->aux.ce = 1.0 / t.layered_epsilon * multe;
        P->aux.chh = 1.0 / t.layered_mu * multh;
        P->aux.lc = (hp.dt * C0 - hp.jdx) / (hp.dt * C0 + hp.jdx);
    }
    // probes
    P->aux.nsteps_planned = hp.nsteps;
    if (!hp.probes.empty()) {
        int64_t *pc;
        double *po;
        CA(upload(P->mem, &pc, hp.probes.data(), hp.probes.size()), "probes");
        CA(P->mem.alloc(&po, hp.probes.size() * 6 * (size_t)std::max(hp.nsteps, 1)), "probe output");
        P->aux.nprobes = (int)hp.probes.size();
        P->aux.probe_cells = pc;
        P->aux.probe_out = po;
    }
    for (int s = 0; s < 2; s++) {
        const float **fp;
        CA(P->mem.alloc(&fp, 6), "field pointer table");
        CA(cudaMemcpy(fp, P->fields[s], sizeof(float *) * 6, cudaMemcpyHostToDevice), "field pointer table");
        P->d_fieldptrs[s] = fp;
    }
    // NFFF running DFT over the box faces (farfield.c:207-404 loops), skip rules included
    if (desc->nfff.enabled && desc->nfff.npoints > 0 && (desc->nfff.nfreq > 0 || desc->nfff.series)) {
        const fdtd_nfff &f = desc->nfff;
        if (f.i0 < 1 || f.j0 < 1 || f.k0 < 1 || f.in > hp.xr - 2 || f.jn > hp.yr - 2 || f.kn > hp.zr - 2 || f.in <= f.i0 ||
            f.jn <= f.j0 || f.kn <= f.k0)
            return bail(cudaErrorInvalidValue, "NFFF box must lie inside [1, res-2]");
        std::vector<int32_t> cell, nstr, ijk;
        std::vector<int8_t> face;
        auto skipped = [&](int fc, int a, int b) {
            return f.skip[fc] && a >= f.skip_lo[fc][0] && b >= f.skip_lo[fc][1] && a <= f.skip_hi[fc][0] && b <= f.skip_hi[fc][1];
        };
        auto add = [&](int fc, int i, int j, int k, int64_t st) {
            cell.push_back((int32_t)(((int64_t)i * hp.yr + j) * hp.zr + k));
            nstr.push_back((int32_t)st);
            ijk.push_back(i); ijk.push_back(j); ijk.push_back(k);
            face.push_back((int8_t)fc);
        };
        if ((double)hp.n > 2.0e9) return bail(cudaErrorInvalidValue, "grid too large for 32-bit NFFF cell indices");
        for (int j = f.j0; j < f.jn; j++)
            for (int k = f.k0; k < f.kn; k++) {
                if (!skipped(0, j, k)) add(0, f.i0, j, k, d.si);
                if (!skipped(1, j, k)) add(1, f.in, j, k, d.si);
            }
        for (int i = f.i0; i < f.in; i++)
            for (int k = f.k0; k < f.kn; k++) {
                if (!skipped(2, i, k)) add(2, i, f.j0, k, d.sj);
                if (!skipped(3, i, k)) add(3, i, f.jn, k, d.sj);
            }
        for (int i = f.i0; i < f.in; i++)
            for (int j = f.j0; j < f.jn; j++) {
                if (!skipped(4, i, j)) add(4, i, j, f.k0, 1);
                if (!skipped(5, i, j)) add(5, i, j, f.kn, 1);
            }
        P->nfff = true;
        P->nfff_npoints = f.npoints;
        P->nfff_nfreq = f.nfreq;
        P->nfff_ns = (int)cell.size();
        if (f.nfreq > 0) P->omega.assign(f.omega, f.omega + f.nfreq);
        int32_t *dcell, *dnstr, *dijk, *dpts, *dist;
        int8_t *dface;
        CA(upload(P->mem, &dcell, cell.data(), cell.size()), "nfff");
        CA(upload(P->mem, &dnstr, nstr.data(), nstr.size()), "nfff");
        CA(upload(P->mem, &dijk, ijk.data(), ijk.size()), "nfff");
        CA(upload(P->mem, &dface, face.data(), face.size()), "nfff");
        CA(upload(P->mem, &dpts, f.points, (size_t)3 * f.npoints), "nfff");
        std::vector<int32_t> ist(f.npoints);
        {
            const double div = C0 * hp.dt / hp.dx;   // farfield.c:72-91 (per point)
            for (int q = 0; q < f.npoints; q++) {
                if (f.istart) { ist[q] = f.istart[q]; continue; }
                double ri = f.points[3 * q], rj = f.points[3 * q + 1], rk = f.points[3 * q + 2];
                double v = std::sqrt((ri / div) * (ri / div) + (rj / div) * (rj / div) + (rk / div) * (rk / div)) - 500;
                ist[q] = (int)(v > 0 ? v : 0);
            }
        }
        CA(upload(P->mem, &dist, ist.data(), ist.size()), "nfff");
        for (int s = 0; s < 2; s++) {
            const float **fp;
            CA(P->mem.alloc(&fp, 3), "field pointer table");
            CA(cudaMemcpy(fp, P->fields[s], sizeof(float *) * 3, cudaMemcpyHostToDevice), "field pointer table");
            P->d_efieldptrs[s] = fp;
        }
        if (f.nfreq > 0) {
            std::vector<double> odt(f.nfreq);
            for (int q = 0; q < f.nfreq; q++) odt[q] = f.omega[q] * hp.dt;
            double *dodt, *dom;
            double2 *acc, *outp;
            CA(upload(P->mem, &dodt, odt.data(), odt.size()), "nfff");
            CA(upload(P->mem, &dom, f.omega, (size_t)f.nfreq), "nfff");
            const size_t nacc = (size_t)f.nfreq * 6 * cell.size();
            CA(P->mem.alloc(&acc, nacc), "nfff accumulators");
            P->snap.push_back({acc, nacc * sizeof(double2)});
            float *ring;   // samples not yet folded into acc: part of the state (FP64 for r64 plans)
            const size_t nring = (size_t)NFFF_RING * 9 * cell.size();
            CA(P->mem.alloc(&ring, nring * rsz / 4), "nfff sample ring");
            P->snap.push_back({ring, nring * rsz});
            P->nf.ring = ring;
            CA(P->mem.alloc(&outp, (size_t)f.npoints * f.nfreq * 3), "nfff output");
            // exp(-i omega R dt) over every retarded index R the box can produce:
            // R <= 1 + (largest point-to-box-corner distance) / (c dt)
            double dmax = 0;
            for (int q = 0; q < f.npoints; q++)
                for (int corner = 0; corner < 8; corner++) {
                    const double cx = (corner & 1) ? f.in : f.i0, cy = (corner & 2) ? f.jn : f.j0, cz = (corner & 4) ? f.kn : f.k0;
                    const double ux = f.points[3 * q] - cx, uy = f.points[3 * q + 1] - cy, uz = f.points[3 * q + 2] - cz;
                    dmax = std::max(dmax, std::sqrt(ux * ux + uy * uy + uz * uz));
                }
            const int ntw = (int)(1.0 + dmax * hp.dx / (C0 * hp.dt)) + 2;
            std::vector<double2> tw((size_t)f.nfreq * ntw);
            for (int q = 0; q < f.nfreq; q++)
                for (int R = 0; R < ntw; R++) {
                    const double ph = f.omega[q] * (double)R * hp.dt;
                    tw[(size_t)q * ntw + R] = make_double2(std::cos(ph), -std::sin(ph));
                }
            double2 *dtw, *part;
            CA(upload(P->mem, &dtw, tw.data(), tw.size()), "far-field twiddles");
            int nsm = 148;
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
            const int ptiles = (f.npoints + 127) / 128;
            int groups = (4 * nsm + ptiles - 1) / ptiles;
            groups = std::max(1, std::min(groups, std::max(1, (int)cell.size() / 256)));
            CA(P->mem.alloc(&part, (size_t)groups * f.npoints * f.nfreq * 3), "far-field partial sums");
            P->nf.ns = (int)cell.size();
            P->nf.nfreq = f.nfreq;
            P->nf.cell = dcell;
            P->nf.nstride = dnstr;
            P->nf.acc = acc;
            P->nf.omega_dt = dodt;
            P->nf.step = P->d_step;
            P->nf.storage = P->storage;
            P->nf.inv2dx = 1.0 / (2.0 * hp.dx);
            P->ff.npoints = f.npoints;
            P->ff.nfreq = f.nfreq;
            P->ff.ns = (int)cell.size();
            P->ff.points = dpts;
            P->ff.istart = dist;
            P->ff.cell_ijk = dijk;
            P->ff.face = dface;
            P->ff.acc = acc;
            P->ff.omega = dom;
            P->ff.dt = hp.dt;
            P->ff.dx = hp.dx;
            P->ff.out = outp;
            P->ff.ntw = ntw;
            P->ff.tw = dtw;
            P->ff.groups = groups;
            P->ff.part = part;
        }
        if (f.series) {
            // farfield.c:63-64
            P->nfff_ndata = (int)(2000 + 2 * desc->nsteps +
                                  std::sqrt((double)(hp.xr * hp.xr + hp.yr * hp.yr + hp.zr * hp.zr)) / (C0 * hp.dt / hp.dx));
            const size_t nser = (size_t)f.npoints * 3 * P->nfff_ndata;
            double *ser;
            CA(P->mem.alloc(&ser, nser), "far-field series");
            CA(cudaMemset(ser, 0, nser * sizeof(double)), "far-field series");
            P->snap.push_back({ser, nser * sizeof(double)});
            P->nfff_series = true;
            P->ns.ns = (int)cell.size();
            P->ns.npoints = f.npoints;
            P->ns.ndata = P->nfff_ndata;
            P->ns.cell = dcell;
            P->ns.nstride = dnstr;
            P->ns.cell_ijk = dijk;
            P->ns.face = dface;
            P->ns.points = dpts;
            P->ns.istart = dist;
            P->ns.series = ser;
            P->ns.step = P->d_step;
            P->ns.storage = P->storage;
            P->ns.dx = hp.dx;
            P->ns.dt = hp.dt;
        }
        if (f.nfreq > 0) bytes += (double)cell.size() * (9.0 * esz + (double)f.nfreq * 6 * 16 * 2);
    }
    // work decomposition: the bulk box (outside every CPML slab, one extra
    // plane on the low sides so that its halo row/column/plane is slab-free,
    // off the grid's edge planes, k bounds multiples of 4) goes to the TMA
    // kernel when the k rows are 16-byte multiples; the rest (slabs, edge
    // planes) to the slab kernels
    {
        const int X = hp.xr, Y = hp.yr, Z = hp.zr;
        int lo[3], hi[3];
        const int res[3] = {X, Y, Z};
        for (int ax = 0; ax < 3; ax++) {
            lo[ax] = std::max(1, hp.cp[2 * ax].enabled ? hp.cp[2 * ax].depth + 1 : 0);
            hi[ax] = std::min(res[ax] - 1, hp.cp[2 * ax + 1].enabled ? res[ax] - hp.cp[2 * ax + 1].depth : res[ax]);
        }
        lo[2] = std::max(4, (lo[2] + 3) / 4 * 4);   // the k halo group k0-4..k0-1 stays in the grid
        hi[2] = hi[2] / 4 * 4;
        const char *nob = getenv("GSVIT_B200_NO_BULK");
        // (design cells take the bulk kernel's per-cell coefficient path; those
        // outside the box take e_special's)
        P->bulk_on = !r64 && ((size_t)Z * esz % 16 == 0) && lo[0] < hi[0] && lo[1] < hi[1] && lo[2] < hi[2] && !(nob && nob[0] == '1');
        std::vector<SlabBox> boxes;
        std::vector<BulkItem> blk;
        long long nblk = 0;
        auto add_box = [&](int i0, int i1, int j0, int j1, int k0, int k1) {
            if (i0 >= i1 || j0 >= j1 || k0 >= k1) return;
            // TSF corrections touch cells in [t0 - 1, t1] on every axis (tsf_add_h/e)
            const bool meets = d.tsf_on && i0 <= d.t1[0] && i1 >= d.t0[0] && j0 <= d.t1[1] && j1 >= d.t0[1] &&
                               k0 <= d.t1[2] && k1 >= d.t0[2];
            boxes.push_back({i0, i1, j0, j1, k0, k1, nblk, 0, meets ? 1 : 0});
            nblk += ((long long)(i1 - i0) * (j1 - j0) * (k1 - k0) + 255) / 256;
        };
        // planes per work item: about 10.  CTAs of neighbouring tiles then stay
        // within a few planes of each other, so that the halo rows and columns
        // one reads are still in L2 when the other reads them (the tiles of the
        // Drude-metal half run about 2x slower than the vacuum half: with 96
        // planes per item their drift evicted the halos; 512^3 rough surface,
        // bulk kernel 2.24 ms at 96 planes, 1.72 ms at 8-12, 1.79 ms at 4)
        auto chunks = [&](int a0, int a1, int *len) {
            const int planes = a1 - a0;
            const int nch = std::max(1, (planes + 9) / 10);
            *len = (planes + nch - 1) / nch;
        };
        if (P->bulk_on) {
            add_box(0, lo[0], 0, Y, 0, Z);
            add_box(hi[0], X, 0, Y, 0, Z);
            add_box(lo[0], hi[0], 0, lo[1], 0, Z);
            add_box(lo[0], hi[0], hi[1], Y, 0, Z);
            add_box(lo[0], hi[0], lo[1], hi[1], 0, lo[2]);
            add_box(lo[0], hi[0], lo[1], hi[1], hi[2], Z);
            int len;
            chunks(lo[0], hi[0], &len);
            blk = bulk_items(lo, hi, len, 0);
            P->bulk_len = len;
            for (int ax = 0; ax < 3; ax++) { P->region[2 * ax] = lo[ax]; P->region[2 * ax + 1] = hi[ax]; }
        } else {
            add_box(0, X, 0, Y, 0, Z);
        }
        if (nblk > 0x7fffffffLL) return bail(cudaErrorInvalidValue, "grid too large for the slab kernels");
        {   // algorithmic bytes per launch: 24 B field reads + 24 B writes + 1 class byte per cell;
            // 12 B (Q read + write, E^{n-1} read) + 16 B per pole per dispersive field component;
            // 4 psi arrays x (4 B read + 4 B write) per CPML cell (slab kernels only)
            auto cell_bytes = [&](int i0, int i1, int j0, int j1, int k0, int k1) {
                double b = 0;
#pragma omp parallel for reduction(+ : b) schedule(static)
                for (int i = i0; i < i1; i++)
                    for (int j = j0; j < j1; j++)
                        for (int k = k0; k < k1; k++) {
                            const DevClass &c = hp.classes[hp.cls[((size_t)i * Y + j) * Z + k]];
                            b += 12.0 * esz + 1.0;
                            if (c.flags & CF_ADE_BRANCH)
                                b += (((c.flags & CF_ADE_X) ? 1 : 0) + ((c.flags & CF_ADE_Y) ? 1 : 0) + ((c.flags & CF_ADE_Z) ? 1 : 0)) *
                                     (8.0 + esz + 16.0 * hp.maxpoles);
                        }
                return b;
            };
            double total = 0;
            for (auto &b : boxes) total += cell_bytes(b.i0, b.i1, b.j0, b.j1, b.k0, b.k1);
            double psi = 0;
            for (int f = 0; f < 6; f++)
                if (hp.cp[f].enabled) {
                    const int dep = hp.cp[f].depth;
                    psi += ((f < 2) ? (double)dep * Y * Z : (f < 4) ? (double)X * dep * Z : (double)X * Y * dep) * 4 * 2.0 * esz;
                }
            P->slab_bytes = total + psi;
            P->bulk_bytes = P->bulk_on ? cell_bytes(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]) : 0;
        }
        CA(upload(P->mem, &P->d_boxes, boxes.data(), boxes.size()), "slab boxes");
        {   // 4-cell groups for the H kernel when every box's k bounds and the row length allow
            bool w4 = (Z % 4 == 0);
            for (auto &b : boxes) w4 = w4 && b.k0 % 4 == 0 && b.k1 % 4 == 0;
            if (w4 && !boxes.empty()) {
                std::vector<SlabBox> b4 = boxes;
                long long nb = 0;
                for (auto &b : b4) {
                    b.first_block = nb;
                    nb += ((long long)(b.i1 - b.i0) * (b.j1 - b.j0) * ((b.k1 - b.k0) / 4) + 255) / 256;
                }
                CA(upload(P->mem, &P->d_boxes4, b4.data(), b4.size()), "slab boxes");
                P->nslab_blocks4 = nb;
            }
        }
        P->h_boxes = boxes;
        P->h_bulk = blk;
        P->nboxes = (int)boxes.size();
        P->nslab_blocks = nblk;
        {   // E lists: each box split along k into runs of planes that hold a
            // dispersive cell and runs that hold none; plain runs shorter than
            // 8 planes stay with the dispersive list (its kernel handles plain
            // cells the same way), so the split adds few boxes
            std::vector<SlabBox> eb, pb;
            long long neb = 0, npb = 0;
            auto push = [&](const SlabBox &b0, int k0, int k1, bool disp) {
                SlabBox b = b0;
                b.k0 = k0;
                b.k1 = k1;
                long long &n = disp ? neb : npb;
                b.first_block = n;
                n += ((long long)(b.i1 - b.i0) * (b.j1 - b.j0) * (k1 - k0) + 255) / 256;
                (disp ? eb : pb).push_back(b);
            };
            for (const SlabBox &b : boxes) {
                if (!hp.has_ade) { push(b, b.k0, b.k1, true); continue; }
                std::vector<char> dk(b.k1 - b.k0, 0);
#pragma omp parallel for schedule(static)
                for (int k = b.k0; k < b.k1; k++) {
                    char any = 0;
                    for (int i = b.i0; i < b.i1 && !any; i++)
                        for (int j = b.j0; j < b.j1; j++)
                            if (hp.classes[hp.cls[((size_t)i * Y + j) * Z + k]].flags & CF_ADE_BRANCH) { any = 1; break; }
                    dk[k - b.k0] = any;
                }
                for (int k = b.k0; k < b.k1;) {   // short plain runs count as dispersive
                    int e = k;
                    while (e < b.k1 && dk[e - b.k0] == dk[k - b.k0]) e++;
                    if (!dk[k - b.k0] && e - k < 8)
                        for (int q = k; q < e; q++) dk[q - b.k0] = 1;
                    k = e;
                }
                for (int k = b.k0; k < b.k1;) {
                    int e = k;
                    while (e < b.k1 && dk[e - b.k0] == dk[k - b.k0]) e++;
                    push(b, k, e, dk[k - b.k0] != 0);
                    k = e;
                }
            }
            P->h_eboxes = pb.empty() ? boxes : eb;
            P->h_epboxes = pb;
            SlabLists &L = P->slabs;
            L.h = P->d_boxes;
            L.nh = P->nboxes;
            L.hblocks = nblk;
            L.h4 = P->d_boxes4;
            L.h4blocks = P->nslab_blocks4;
            if (pb.empty()) {
                L.e = P->d_boxes;
                L.ne = P->nboxes;
                L.eblocks = nblk;
            } else {
                SlabBox *de = nullptr, *dp = nullptr;
                if (!eb.empty()) CA(upload(P->mem, &de, eb.data(), eb.size()), "slab boxes");
                CA(upload(P->mem, &dp, pb.data(), pb.size()), "slab boxes");
                L.e = de;
                L.ne = (int)eb.size();
                L.eblocks = neb;
                L.ep = dp;
                L.nep = (int)pb.size();
                L.epblocks = npb;
            }
        }
        CA(P->mem.alloc(&P->d_err, 1), "error word");
        if (P->bulk_on) {
            CA(upload(P->mem, &P->d_bulk, blk.data(), blk.size()), "work table");
            P->nbulk = (int)blk.size();
            void *fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            CA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q), "driver entry point");
            if (!fn || q != cudaDriverEntryPointSuccess) return bail(cudaErrorNotSupported, "cuTensorMapEncodeTiled");
            for (int sset = 0; sset < 2; sset++)
                if (tile_make_maps(TILE_BULK, fn, d, P->fields[sset], cls, d.cpitch, P->storage, &P->bmaps[sset]) != 0)
                    return bail(cudaErrorInvalidValue, "tensor map encoding");
            // the largest layout (256 classes), so that any plan or batch may launch
            CA(bulk_configure(), "bulk kernel shared memory");
        }
        // TMA tiles over the whole grid (single plans; batches may use them too)
        // the CPML tiles take one face per axis: every extent at least both depths + 8
        bool roomy = true;
        int dmin = 1 << 30;
        for (int ax = 0; ax < 3; ax++) {
            const int ext = ax == 0 ? X : ax == 1 ? Y : Z;
            const int dd = (hp.cp[2 * ax].enabled ? hp.cp[2 * ax].depth : 0) + (hp.cp[2 * ax + 1].enabled ? hp.cp[2 * ax + 1].depth : 0);
            roomy = roomy && ext >= dd + 8;
            for (int f = 2 * ax; f < 2 * ax + 2; f++)
                if (hp.cp[f].enabled) dmin = std::min(dmin, hp.cp[f].depth);
        }
        const bool can_tile = !r64 && roomy && ((size_t)Z * esz % 16 == 0) && !(nob && nob[0] == '1');
        // Default: tiles for grids of at least 2^24 cells with CPML of depth
        // >= 12.  Rough-surface steps, ms, slab kernels / tiles (the CPML kinds
        // concurrent with the bulk): 512^3 d16 3.11 / 2.74, 384^3 d16 1.56 /
        // 1.39, 256^3 d16 0.62 / 0.58, 256^3 d12 0.59 / 0.59; smaller grids
        // and thinner slabs fill the CPML tiles poorly and the slab kernels
        // win: 256x256x128 d12 0.42 / 0.44, 192^3 d16 0.36 / 0.40, 128^3 d8
        // 0.16 / 0.21.  GSVIT_B200_TILES=1 / 0 at plan creation forces them
        // on / off.
        const char *tv = getenv("GSVIT_B200_TILES");
        const bool want = tv ? tv[0] == '1' : (dmin >= 12 && (double)hp.n >= 16777216.0);
        P->tiles_on = can_tile && want;
        // test hook of the bounded-wait error path: every tile CTA of this plan
        // also waits, at most this many polls, on an mbarrier nothing arrives on
        if (const char *stv = getenv("GSVIT_B200_STALL_TEST")) P->stall = std::max(0, atoi(stv));
        if (P->tiles_on) {
            int rc = build_tiles(P, hp, d, cls);
            if (rc != FDTD_OK) return bail_rc(rc);
        }
        if (P->tiles_on || P->bulk_on) {   // side streams and events of the concurrent CPML kinds / slab H
            CA(cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming), "tile events");
            for (int k = TILE_CPX; k < NTILE; k++) {
                CA(cudaStreamCreateWithFlags(&P->side[k], cudaStreamNonBlocking), "tile streams");
                CA(cudaEventCreateWithFlags(&P->ev_join[k], cudaEventDisableTiming), "tile events");
            }
        }
    }
    P->step_bytes = bytes;
    CA(cudaDeviceSynchronize(), "plan set-up");
#undef CA
    *out = P;
    return FDTD_OK;
}

// FP32 <-> storage element conversion on the host (H components carry hs)
void pack_storage(int storage, float scale, const float *src, size_t n, uint16_t *dst)
{
    for (size_t q = 0; q < n; q++) {
        const float v = src[q] * scale;
        if (storage == FDTD_STORE_F16) {
            __half h = __float2half_rn(v);
            std::memcpy(&dst[q], &h, 2);
        } else {
            __nv_bfloat16 h = __float2bfloat16_rn(v);
            std::memcpy(&dst[q], &h, 2);
        }
    }
}

void unpack_storage(int storage, float scale, const uint16_t *src, size_t n, float *dst)
{
    for (size_t q = 0; q < n; q++) {
        if (storage == FDTD_STORE_F16) {
            __half h;
            std::memcpy(&h, &src[q], 2);
            dst[q] = __half2float(h) * scale;
        } else {
            __nv_bfloat16 h;
            std::memcpy(&h, &src[q], 2);
            dst[q] = __bfloat162float(h) * scale;
        }
    }
}

// component c of the current set from FP32 host values; `sync` makes the
// copy complete before returning (FP32 storage copies asynchronously
// otherwise, 16-bit storage always completes, its staging buffer is local)
int upload_comp(fdtd_plan *P, int c, const float *src, bool sync)
{
    const size_t n = P->hp.n;
    if (P->storage == FDTD_STORE_F32) {
        CK(cudaMemcpyAsync(P->fields[P->cur][c], src, n * 4, cudaMemcpyHostToDevice, P->stream));
        if (sync) CK(cudaStreamSynchronize(P->stream));
        return FDTD_OK;
    }
    if (P->storage == FDTD_STORE_F64) {
        std::vector<double> w(src, src + n);
        CK(cudaMemcpyAsync(P->fields[P->cur][c], w.data(), n * 8, cudaMemcpyHostToDevice, P->stream));
        CK(cudaStreamSynchronize(P->stream));
        return FDTD_OK;
    }
    std::vector<uint16_t> tmp(n);
    pack_storage(P->storage, c >= 3 ? P->dp.hs : 1.f, src, n, tmp.data());
    CK(cudaMemcpyAsync(P->fields[P->cur][c], tmp.data(), n * 2, cudaMemcpyHostToDevice, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    return FDTD_OK;
}

// component c of the current set as FP32 host values (FP32 storage: an
// asynchronous copy the caller synchronises)
int download_comp(fdtd_plan *P, int c, float *dst)
{
    const size_t n = P->hp.n;
    if (P->storage == FDTD_STORE_F32) {
        CK(cudaMemcpyAsync(dst, P->fields[P->cur][c], n * 4, cudaMemcpyDeviceToHost, P->stream));
        return FDTD_OK;
    }
    if (P->storage == FDTD_STORE_F64) {
        std::vector<double> w(n);
        CK(cudaMemcpyAsync(w.data(), P->fields[P->cur][c], n * 8, cudaMemcpyDeviceToHost, P->stream));
        CK(cudaStreamSynchronize(P->stream));
        for (size_t q = 0; q < n; q++) dst[q] = (float)w[q];
        return FDTD_OK;
    }
    std::vector<uint16_t> tmp(n);
    CK(cudaMemcpyAsync(tmp.data(), P->fields[P->cur][c], n * 2, cudaMemcpyDeviceToHost, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    unpack_storage(P->storage, c >= 3 ? P->dp.ihs : 1.f, tmp.data(), n, dst);
    return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_plan_destroy(fdtd_plan *P)
{
    if (!P) return FDTD_OK;
    cudaSetDevice(P->device);
    if (P->stream) cudaStreamSynchronize(P->stream);
    for (int s = 0; s < 2; s++)
        if (P->graph[s]) cudaGraphExecDestroy(P->graph[s]);
    for (int k = 0; k < NTILE; k++) {
        if (P->side[k]) { cudaStreamSynchronize(P->side[k]); cudaStreamDestroy(P->side[k]); }
        if (P->ev_join[k]) cudaEventDestroy(P->ev_join[k]);
    }
    if (P->ev_fork) cudaEventDestroy(P->ev_fork);
    P->mem.free_all();
    if (P->own_stream) cudaStreamDestroy(P->own_stream);
    delete P;
    return FDTD_OK;
}

int fdtd_set_stream(fdtd_plan *P, void *stream)
{
    if (!P) return fail(FDTD_E_INVALID, "plan is NULL");
    P->stream = stream ? (cudaStream_t)stream : P->own_stream;
    return FDTD_OK;
}

int fdtd_sync(fdtd_plan *P)
{
    if (!P) return fail(FDTD_E_INVALID, "plan is NULL");
    CK(cudaSetDevice(P->device));
    CK(cudaStreamSynchronize(P->stream));
    return device_error(P);
}

int fdtd_set_fields(fdtd_plan *P, int mask, const double *const comps[6])
{
    if (!P || !comps) return fail(FDTD_E_INVALID, "NULL argument");
    CK(cudaSetDevice(P->device));
    if (P->storage == FDTD_STORE_F64) {   // no rounding: the doubles as they are
        for (int c = 0; c < 6; c++) {
            if (!(mask & (1 << c))) continue;
            if (!comps[c]) return fail(FDTD_E_INVALID, "selected component pointer is NULL");
            CK(cudaMemcpyAsync(P->fields[P->cur][c], comps[c], P->hp.n * 8, cudaMemcpyHostToDevice, P->stream));
        }
        CK(cudaStreamSynchronize(P->stream));
        return FDTD_OK;
    }
    std::vector<float> tmp(P->hp.n);
    for (int c = 0; c < 6; c++) {
        if (!(mask & (1 << c))) continue;
        if (!comps[c]) return fail(FDTD_E_INVALID, "selected component pointer is NULL");
        for (size_t q = 0; q < P->hp.n; q++) tmp[q] = (float)comps[c][q];
        int rc = upload_comp(P, c, tmp.data(), true);
        if (rc != FDTD_OK) return rc;
    }
    return FDTD_OK;
}

int fdtd_set_design_eps(fdtd_plan *P, const double *eps_r)
{
    if (!P || !eps_r) return fail(FDTD_E_INVALID, "NULL argument");
    if (!P->hp.design) return fail(FDTD_E_INVALID, "the plan has no design region");
    const int *b = P->hp.dbox;
    const size_t nd = (size_t)(b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]);
    for (size_t q = 0; q < nd; q++)
        if (!(eps_r[q] >= 1e-3 && eps_r[q] < 1e6)) return fail(FDTD_E_INVALID, "design eps_r must be positive and finite");
    CK(cudaSetDevice(P->device));
    CK(cudaStreamSynchronize(P->stream));
    design_coefficients(&P->hp, eps_r);
    if (P->storage == FDTD_STORE_F64)
        CK(cudaMemcpy(const_cast<float *>(P->dp.dcoef), P->hp.dcoef64.data(), P->hp.dcoef64.size() * sizeof(double),
                      cudaMemcpyHostToDevice));
    else
        CK(cudaMemcpy(const_cast<float *>(P->dp.dcoef), P->hp.dcoef.data(), P->hp.dcoef.size() * sizeof(float),
                      cudaMemcpyHostToDevice));
    return FDTD_OK;
}

int fdtd_set_fields_f32(fdtd_plan *P, int mask, const float *const comps[6])
{
    if (!P || !comps) return fail(FDTD_E_INVALID, "NULL argument");
    CK(cudaSetDevice(P->device));
    for (int c = 0; c < 6; c++) {
        if (!(mask & (1 << c))) continue;
        if (!comps[c]) return fail(FDTD_E_INVALID, "selected component pointer is NULL");
        int rc = upload_comp(P, c, comps[c], false);
        if (rc != FDTD_OK) return rc;
    }
    return FDTD_OK;
}

int fdtd_get_fields_f32(fdtd_plan *P, int mask, float *const comps[6])
{
    if (!P || !comps) return fail(FDTD_E_INVALID, "NULL argument");
    CK(cudaSetDevice(P->device));
    for (int c = 0; c < 6; c++) {
        if (!(mask & (1 << c))) continue;
        if (!comps[c]) return fail(FDTD_E_INVALID, "selected component pointer is NULL");
        int rc = download_comp(P, c, comps[c]);
        if (rc != FDTD_OK) return rc;
    }
    CK(cudaStreamSynchronize(P->stream));
    return device_error(P);
}

int fdtd_get_fields(fdtd_plan *P, int mask, double *const comps[6])
{
    if (!P || !comps) return fail(FDTD_E_INVALID, "NULL argument");
    CK(cudaSetDevice(P->device));
    if (P->storage == FDTD_STORE_F64) {
        for (int c = 0; c < 6; c++) {
            if (!(mask & (1 << c))) continue;
            if (!comps[c]) return fail(FDTD_E_INVALID, "selected component pointer is NULL");
            CK(cudaMemcpyAsync(comps[c], P->fields[P->cur][c], P->hp.n * 8, cudaMemcpyDeviceToHost, P->stream));
        }
        CK(cudaStreamSynchronize(P->stream));
        return device_error(P);
    }
    std::vector<float> tmp(P->hp.n);
    for (int c = 0; c < 6; c++) {
        if (!(mask & (1 << c))) continue;
        if (!comps[c]) return fail(FDTD_E_INVALID, "selected component pointer is NULL");
        int rc = download_comp(P, c, tmp.data());
        if (rc != FDTD_OK) return rc;
        CK(cudaStreamSynchronize(P->stream));
        for (size_t q = 0; q < P->hp.n; q++) comps[c][q] = (double)tmp[q];
    }
    CK(cudaStreamSynchronize(P->stream));
    return device_error(P);
}

int fdtd_step(fdtd_plan *P, int nsteps)
{
    if (!P || nsteps < 0) return fail(FDTD_E_INVALID, "bad argument");
    if (P->failed) return refuse_failed(P);
    CK(cudaSetDevice(P->device));
    for (int s = 0; s < nsteps; s++) {
        int rc = launch_step(P, P->stream);
        if (rc != FDTD_OK) return rc;
        P->host_step++;
    }
    final_probes(P, P->stream);
    CK(cudaGetLastError());
    return FDTD_OK;
}

}  // extern "C"

// Scratch of fdtd_step_static_scratch: this step's TSF face correction tables,
// one per device (the module's copy on each device), never allocated.
static __device__ __align__(256) unsigned char g_static_scratch[FDTD_STATIC_SCRATCH_BYTES];

namespace {

constexpr int kStaticDevices = 64;
std::mutex g_static_mu;
// the array's device address per device, looked up once and kept for the
// life of the process: valid as long as the device is not reset
// (cudaDeviceReset) while the library stays loaded
void *g_static_addr[kStaticDevices] = {};

// Device address of g_static_scratch on `device` (current), looked up once.
int static_scratch_addr(int device, unsigned char **out)
{
    if (device < 0 || device >= kStaticDevices) return fail(FDTD_E_UNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(FDTD_E_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
        g_static_addr[device] = p;
    }
    *out = static_cast<unsigned char *>(g_static_addr[device]);
    return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_step_static_scratch(fdtd_plan *P, int nsteps)
{
    if (!P || nsteps < 0) return fail(FDTD_E_INVALID, "bad argument");
    if (P->failed) return refuse_failed(P);
    CK(cudaSetDevice(P->device));
    unsigned char *base = nullptr;
    int rc = static_scratch_addr(P->device, &base);
    if (rc != FDTD_OK) return rc;
    // carve the twelve tables (H and E corrections of six faces) out of the array
    float2 *th[6] = {}, *te[6] = {};
    size_t used = 0;
    if (P->tsf_cells) {
        for (int f = 0; f < 6; f++) {
            const size_t esz2 = P->storage == FDTD_STORE_F64 ? sizeof(double2) : sizeof(float2);
            const size_t bytes = (P->hp.tmap[f].size() * esz2 + 255) & ~(size_t)255;
            if (used + 2 * bytes > FDTD_STATIC_SCRATCH_BYTES)
                return fail(FDTD_E_UNSUPPORTED, "the TSF face tables of this plan need more than the "
                                                "FDTD_STATIC_SCRATCH_BYTES (32 MiB) of static scratch");
            th[f] = reinterpret_cast<float2 *>(base + used);
            te[f] = reinterpret_cast<float2 *>(base + used + bytes);
            used += 2 * bytes;
        }
    }
    float2 *keep_h[6], *keep_e[6];
    for (int f = 0; f < 6; f++) {
        keep_h[f] = P->dp.tcor_h[f];
        keep_e[f] = P->dp.tcor_e[f];
        if (P->tsf_cells) {
            P->dp.tcor_h[f] = th[f];
            P->dp.tcor_e[f] = te[f];
        }
    }
    rc = FDTD_OK;
    for (int s = 0; s < nsteps && rc == FDTD_OK; s++) {
        rc = launch_step(P, P->stream);
        if (rc == FDTD_OK) P->host_step++;
    }
    for (int f = 0; f < 6; f++) {
        P->dp.tcor_h[f] = keep_h[f];
        P->dp.tcor_e[f] = keep_e[f];
    }
    if (rc != FDTD_OK) return rc;
    final_probes(P, P->stream);
    CK(cudaGetLastError());
    return FDTD_OK;
}

int fdtd_step_graph(fdtd_plan *P, int nsteps, int chunk)
{
    if (!P || nsteps < 0) return fail(FDTD_E_INVALID, "bad argument");
    if (P->failed) return refuse_failed(P);
    CK(cudaSetDevice(P->device));
    if (chunk < 2) chunk = 2;
    chunk &= ~1;   // an even number of steps returns the ping-pong parity
    if (P->graph_steps != chunk) {
        for (int s = 0; s < 2; s++)
            if (P->graph[s]) { cudaGraphExecDestroy(P->graph[s]); P->graph[s] = nullptr; }
        P->graph_steps = chunk;
    }
    int done = 0;
    while (nsteps - done >= chunk) {
        const int par = P->cur;
        if (!P->graph[par]) {
            cudaGraph_t g;
            cudaStream_t cs = P->stream;
            CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            for (int s = 0; s < chunk; s++) {
                int rc = launch_step(P, cs);
                if (rc != FDTD_OK) {
                    cudaStreamEndCapture(cs, &g);
                    return rc;
                }
            }
            CK(cudaStreamEndCapture(cs, &g));
            cudaGraphExec_t ge;
            cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            P->graph[par] = ge;
            P->cur = par;   // capture advanced cur by chunk (even): unchanged
        }
        CK(cudaGraphLaunch(P->graph[par], P->stream));
        done += chunk;
        P->host_step += chunk;
    }
    for (; done < nsteps; done++) {
        int rc = launch_step(P, P->stream);
        if (rc != FDTD_OK) return rc;
        P->host_step++;
    }
    final_probes(P, P->stream);
    CK(cudaGetLastError());
    return FDTD_OK;
}

int fdtd_get_step(const fdtd_plan *P, int *step)
{
    if (!P || !step) return fail(FDTD_E_INVALID, "NULL argument");
    *step = P->host_step;
    return FDTD_OK;
}

int fdtd_step_timed(fdtd_plan *P, int nsteps, double *fused_ms, int *fused_launches)
{
    if (!P || nsteps < 0) return fail(FDTD_E_INVALID, "bad argument");
    if (P->failed) return refuse_failed(P);
    CK(cudaSetDevice(P->device));
    std::vector<cudaEvent_t> ev(2 * (size_t)nsteps);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    for (int s = 0; s < nsteps; s++) {
        const int in = P->cur;
        DevAux a = P->aux;
        a.fields = P->d_fieldptrs[in];
        launch_aux_step(a, P->stream);
        if (P->tsf_cells) launch_tsf_faces(P->dp, P->tsf_cells, P->stream);
        CK(cudaEventRecord(ev[2 * s], P->stream));
        int rc = launch_fused(P, in, P->stream);
        CK(cudaEventRecord(ev[2 * s + 1], P->stream));
        if (rc != FDTD_OK) return rc;
        launch_nfff(P, in, P->stream);
        P->cur = 1 - in;
        P->host_step++;
    }
    final_probes(P, P->stream);
    CK(cudaStreamSynchronize(P->stream));
    double tot = 0;
    for (int s = 0; s < nsteps; s++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[2 * s], ev[2 * s + 1]));
        tot += ms;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (fused_ms) *fused_ms = tot;
    if (fused_launches) *fused_launches = nsteps;
    return FDTD_OK;
}

int fdtd_step_profile(fdtd_plan *P, int nsteps, double out[8])
{
    if (!P || nsteps < 1 || !out) return fail(FDTD_E_INVALID, "bad argument");
    if (P->failed) return refuse_failed(P);
    CK(cudaSetDevice(P->device));
    const int NE = 6;
    std::vector<cudaEvent_t> ev((size_t)NE * nsteps);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    cudaStream_t st = P->stream;
    for (int s = 0; s < nsteps; s++) {
        cudaEvent_t *E = &ev[(size_t)NE * s];
        const int in = P->cur;
        DevAux a = P->aux;
        a.fields = P->d_fieldptrs[in];
        CK(cudaEventRecord(E[0], st));
        launch_aux_step(a, st);
        if (P->tsf_cells) launch_tsf_faces(P->dp, P->tsf_cells, st);
        CK(cudaEventRecord(E[1], st));
        DevPlan d = plan_for(P, in);
        if (P->tiles_on) {
            int rc = launch_tile_kind(P, d, in, TILE_BULK, st);
            if (rc != FDTD_OK) return rc;
            CK(cudaEventRecord(E[2], st));
            for (int kind = TILE_CPX; kind < NTILE && rc == FDTD_OK; kind++) rc = launch_tile_kind(P, d, in, kind, st);
            if (rc != FDTD_OK) return rc;
        } else {
            if (P->bulk_on) {
                cudaError_t e = launch_tiles(TILE_BULK, d, P->bmaps[in], P->d_bulk, P->nbulk, P->d_err, P->hp.has_ade,
                                             P->hp.maxpoles, P->storage, 0, st);
                if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("bulk step launch: ") + cudaGetErrorString(e));
            }
            CK(cudaEventRecord(E[2], st));
            cudaError_t e = launch_slab_steps(d, P->slabs, P->hp.has_ade, P->hp.maxpoles, P->storage, st);
            if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("slab step launch: ") + cudaGetErrorString(e));
        }
        CK(cudaEventRecord(E[3], st));
        launch_nfff(P, in, st);
        CK(cudaEventRecord(E[4], st));
        P->cur = 1 - in;
        P->host_step++;
    }
    final_probes(P, st);
    CK(cudaStreamSynchronize(st));
    double aux = 0, bulk = 0, slab = 0, nf = 0, tot = 0;
    for (int s = 0; s < nsteps; s++) {
        cudaEvent_t *E = &ev[(size_t)NE * s];
        float t01, t12, t23, t34, t04;
        CK(cudaEventElapsedTime(&t01, E[0], E[1]));
        CK(cudaEventElapsedTime(&t12, E[1], E[2]));
        CK(cudaEventElapsedTime(&t23, E[2], E[3]));
        CK(cudaEventElapsedTime(&t34, E[3], E[4]));
        CK(cudaEventElapsedTime(&t04, E[0], E[4]));
        aux += t01; bulk += t12; slab += t23; nf += t34; tot += t04;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    out[0] = bulk;
    out[2] = slab;
    out[4] = aux;
    out[5] = nf;
    out[6] = tot;
    int nyee;
    if (P->tiles_on) {
        out[1] = P->tile_bytes[TILE_BULK];
        out[3] = P->tile_bytes[TILE_CPX] + P->tile_bytes[TILE_CPY] + P->tile_bytes[TILE_CPZ];
        nyee = 0;
        for (int kind = 0; kind < NTILE; kind++) nyee += P->ntiles[kind] > 0;
    } else {
        out[1] = P->bulk_bytes;
        out[3] = P->slab_bytes;
        const SlabLists &L = P->slabs;   // slab H, then E over the dispersive and the plain runs
        nyee = (P->bulk_on ? 1 : 0) + (L.hblocks > 0 ? 1 + (L.eblocks > 0 ? 1 : 0) + (L.epblocks > 0 ? 1 : 0) : 0);
    }
    out[7] = 1 + (P->tsf_cells ? 1 : 0) + nyee + (P->nfff_nfreq > 0 ? 2 : 0) + (P->nfff_series ? 1 : 0);
    return FDTD_OK;
}

int fdtd_get_probes(fdtd_plan *P, double *out, size_t out_len)
{
    if (!P || (!out && out_len)) return fail(FDTD_E_INVALID, "NULL argument");
    size_t need = P->hp.probes.size() * 6 * (size_t)std::max(P->hp.nsteps, 1);
    if (P->hp.probes.empty()) return FDTD_OK;
    if (out_len < need) return fail(FDTD_E_INVALID, "probe buffer too small");
    CK(cudaSetDevice(P->device));
    CK(cudaMemcpyAsync(out, P->aux.probe_out, need * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    return device_error(P);
}

int fdtd_nfff_spectrum(fdtd_plan *P, double *out, size_t out_len)
{
    if (!P || !out) return fail(FDTD_E_INVALID, "NULL argument");
    if (!P->nfff || P->nfff_nfreq <= 0) return fail(FDTD_E_STATE, "the plan has no NFFF box / frequencies");
    size_t need = (size_t)P->nfff_npoints * P->nfff_nfreq * 3 * 2;
    if (out_len < need) return fail(FDTD_E_INVALID, "spectrum buffer too small");
    CK(cudaSetDevice(P->device));
    launch_nfff_fold_pending(P->nf, P->stream);
    launch_farfield_finalize(P->ff, P->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, P->ff.out, need * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    return device_error(P);
}

int fdtd_nfff_ndata(const fdtd_plan *P, int *ndata)
{
    if (!P || !ndata) return fail(FDTD_E_INVALID, "NULL argument");
    if (!P->nfff_series) return fail(FDTD_E_STATE, "the plan was created without nfff.series");
    *ndata = P->nfff_ndata;
    return FDTD_OK;
}

int fdtd_nfff_series(fdtd_plan *P, double *out, size_t out_len)
{
    if (!P || !out) return fail(FDTD_E_INVALID, "NULL argument");
    if (!P->nfff_series) return fail(FDTD_E_STATE, "the plan was created without nfff.series");
    const size_t need = (size_t)P->nfff_npoints * 3 * P->nfff_ndata;
    if (out_len < need) return fail(FDTD_E_INVALID, "series buffer too small");
    CK(cudaSetDevice(P->device));
    CK(cudaMemcpyAsync(out, P->ns.series, need * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    return device_error(P);
}

int fdtd_get_map(fdtd_plan *P, int which, int32_t *out, size_t out_len)
{
    if (!P || !out) return fail(FDTD_E_INVALID, "NULL argument");
    if (out_len < P->hp.n) return fail(FDTD_E_INVALID, "map buffer too small");
    const size_t n = P->hp.n;
    switch (which) {
    case FDTD_MAP_BNDS: for (size_t c = 0; c < n; c++) out[c] = P->hp.bnds[c]; break;
    case FDTD_MAP_SOURCESKIP: for (size_t c = 0; c < n; c++) out[c] = P->hp.sskip[c]; break;
    case FDTD_MAP_CLASS: {
        std::vector<uint8_t> tmp(n);
        CK(cudaSetDevice(P->device));
        // rows of zres bytes at a pitch of cpitch bytes on the device
        CK(cudaMemcpy2D(tmp.data(), P->hp.zr, P->dp.cls, P->dp.cpitch, P->hp.zr, (size_t)P->hp.xr * P->hp.yr,
                        cudaMemcpyDeviceToHost));
        for (size_t c = 0; c < n; c++) out[c] = tmp[c];
        break;
    }
    default: return fail(FDTD_E_INVALID, "unknown map");
    }
    return FDTD_OK;
}

int fdtd_get_nclasses(const fdtd_plan *P, int *nclasses)
{
    if (!P || !nclasses) return fail(FDTD_E_INVALID, "NULL argument");
    *nclasses = (int)P->hp.classes.size();
    return FDTD_OK;
}

int fdtd_snapshot_size(const fdtd_plan *P, size_t *bytes)
{
    if (!P || !bytes) return fail(FDTD_E_INVALID, "NULL argument");
    size_t b = sizeof(int) * 2;
    for (auto &s : P->snap) b += s.bytes;
    *bytes = b;
    return FDTD_OK;
}

int fdtd_snapshot_save(fdtd_plan *P, void *host_buf, size_t bytes)
{
    size_t need = 0;
    int rc = fdtd_snapshot_size(P, &need);
    if (rc != FDTD_OK) return rc;
    if (!host_buf || bytes < need) return fail(FDTD_E_INVALID, "snapshot buffer too small");
    CK(cudaSetDevice(P->device));
    char *p = (char *)host_buf;
    std::memcpy(p, &P->cur, sizeof(int)); p += sizeof(int);
    std::memcpy(p, &P->host_step, sizeof(int)); p += sizeof(int);
    for (auto &s : P->snap) {
        CK(cudaMemcpyAsync(p, s.ptr, s.bytes, cudaMemcpyDeviceToHost, P->stream));
        p += s.bytes;
    }
    CK(cudaStreamSynchronize(P->stream));
    return device_error(P);
}

int fdtd_snapshot_restore(fdtd_plan *P, const void *host_buf, size_t bytes)
{
    size_t need = 0;
    int rc = fdtd_snapshot_size(P, &need);
    if (rc != FDTD_OK) return rc;
    if (!host_buf || bytes < need) return fail(FDTD_E_INVALID, "snapshot buffer too small");
    CK(cudaSetDevice(P->device));
    const char *p = (const char *)host_buf;
    std::memcpy(&P->cur, p, sizeof(int)); p += sizeof(int);
    std::memcpy(&P->host_step, p, sizeof(int)); p += sizeof(int);
    for (auto &s : P->snap) {
        CK(cudaMemcpyAsync(s.ptr, p, s.bytes, cudaMemcpyHostToDevice, P->stream));
        p += s.bytes;
    }
    CK(cudaStreamSynchronize(P->stream));
    return FDTD_OK;
}

int fdtd_step_bytes(const fdtd_plan *P, double *bytes)
{
    if (!P || !bytes) return fail(FDTD_E_INVALID, "NULL argument");
    *bytes = P->step_bytes;
    return FDTD_OK;
}

}  // extern "C"

// ============================================================== batches
//
// Many independent plans (instances of uneven size and material) stepped in
// lockstep: each kernel of a step is ONE launch over all instances, with the
// per-instance parameters in device tables (per ping-pong parity) and every
// work item naming its instance.  The bulk kernel runs persistently: a grid
// of resident CTAs walks the concatenated item list.  The instance plans keep
// their own state and remain the handles for fields, probes and far fields.

struct fdtd_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<fdtd_plan *> plans;
    DevBuf mem;
    int ncls = 0, sms = 148;
    int cur = 0;
    int storage = FDTD_STORE_F32;   // one field storage type for every instance
    // instances are grouped by kernel variant -- 0: no ADE, 1: Drude, 2: with
    // critical-point poles -- so that each runs the variant it runs alone and
    // gives the same bits; a step launches each kernel once per group in use
    std::vector<int> group;
    DevPlan *d_plans[2] = {nullptr, nullptr};
    BulkMaps *d_maps[2] = {nullptr, nullptr};
    DevAux *d_aux[2] = {nullptr, nullptr};
    DevNfff *d_nfff[2] = {nullptr, nullptr};
    BulkItem *d_items[3] = {nullptr, nullptr, nullptr};
    size_t items_cap[3] = {0, 0, 0};
    int nitems[3] = {0, 0, 0}, bulk_grid[3] = {0, 0, 0}, chunk_len = 0;
    bool persistent = true;
    SlabBox *d_boxes[3] = {nullptr, nullptr, nullptr};
    SlabBox *d_boxes4[3] = {nullptr, nullptr, nullptr};   // 4-cell groups when every box of the group is 4-aligned
    int nboxes[3] = {0, 0, 0};
    long long nslab_blocks[3] = {0, 0, 0};
    long long nslab_blocks4[3] = {0, 0, 0};
    SlabBox *d_eboxes[3] = {nullptr, nullptr, nullptr};   // E: the instances' dispersive runs, per variant
    int neboxes[3] = {0, 0, 0};
    long long neblocks[3] = {0, 0, 0};
    SlabBox *d_epboxes = nullptr;                         // E: every instance's plain runs, one launch
    int nepboxes = 0;
    long long nepblocks = 0;
    int max_tsf = 0, max_nfff = 0;
    int *d_err = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_steps = 0;
    // Each instance runs the path it runs alone: the TMA tiles over its whole
    // grid (fdtd_plan::tiles_on; their lists concatenated per kernel variant
    // and tile kind, one CTA per item) or the bulk box and slab kernels (the
    // lists above hold only these instances).
    int ntiled = 0;
    BulkItem *d_titems[3][NTILE] = {};   // [variant group][tile kind]
    int ntitems[3][NTILE] = {};
    BulkMaps *d_tmaps[NTILE][2] = {};    // [tile kind][parity], indexed by instance
};

namespace {

void batch_free(fdtd_batch *B)
{
    if (!B) return;
    cudaSetDevice(B->device);
    if (B->stream) cudaStreamSynchronize(B->stream);
    for (int s = 0; s < 2; s++)
        if (B->graph[s]) cudaGraphExecDestroy(B->graph[s]);
    for (auto *p : B->plans) fdtd_plan_destroy(p);
    B->mem.free_all();
    if (B->stream) cudaStreamDestroy(B->stream);
    delete B;
}

// bulk work list of every instance with `len` planes per item (0 = each
// plan's own choice); grid: resident CTAs of the persistent launch
cudaError_t batch_set_items(fdtd_batch *B, int len, bool persistent)
{
    for (int g = 0; g < 3; g++) {
        std::vector<BulkItem> all;
        for (size_t q = 0; q < B->plans.size(); q++) {
            fdtd_plan *P = B->plans[q];
            if (!P->bulk_on || P->tiles_on || B->group[q] != g) continue;
            const int lo[3] = {P->region[0], P->region[2], P->region[4]}, hi[3] = {P->region[1], P->region[3], P->region[5]};
            const auto it = bulk_items(lo, hi, len > 0 ? len : P->bulk_len, (int)q);
            all.insert(all.end(), it.begin(), it.end());
        }
        if (all.size() > B->items_cap[g]) {
            BulkItem *d;
            cudaError_t e = B->mem.alloc(&d, all.size());
            if (e != cudaSuccess) return e;
            B->d_items[g] = d;
            B->items_cap[g] = all.size();
        }
        if (!all.empty()) {
            cudaError_t e = cudaMemcpy(B->d_items[g], all.data(), all.size() * sizeof(BulkItem), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return e;
        }
        B->nitems[g] = (int)all.size();
        B->bulk_grid[g] = persistent ? 2 * B->sms : std::max(1, B->nitems[g]);
    }
    B->chunk_len = len;
    B->persistent = persistent;
    for (int s = 0; s < 2; s++)
        if (B->graph[s]) { cudaGraphExecDestroy(B->graph[s]); B->graph[s] = nullptr; }
    return cudaSuccess;
}

int batch_launch_step(fdtd_batch *B, cudaStream_t st)
{
    const int in = B->cur, n = (int)B->plans.size();
    launch_aux_step_batch(B->d_aux[in], n, st);
    if (B->max_tsf) launch_tsf_faces_batch(B->d_plans[in], n, B->max_tsf, st);
    for (int g = 0; g < 3; g++)   // instances with TMA tiles
        for (int kind = 0; kind < NTILE; kind++) {
            if (!B->ntitems[g][kind]) continue;
            cudaError_t e = launch_tiles_batch(kind, B->d_plans[in], B->d_tmaps[kind][in], B->d_titems[g][kind],
                                               B->ntitems[g][kind], B->ncls, B->d_err, g > 0, g == 2 ? 2 : 0, B->storage, st);
            if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("batched tile launch: ") + cudaGetErrorString(e));
        }
    // the others: bulk box and slab kernels, variant by variant (a side
    // stream for the slab H kernels, as single plans have, measured slower on
    // the 48-instance batch: 11.3 against 13.9 Gcell/s)
    for (int g = 0; g < 3; g++) {
        if (!B->nitems[g] && !B->nboxes[g] && !B->neboxes[g]) continue;
        const bool ade = g > 0;
        const int npoles = g == 2 ? 2 : 0;
        cudaError_t e = launch_bulk_batch(B->d_plans[in], B->d_maps[in], B->d_items[g], B->nitems[g], B->bulk_grid[g], B->ncls,
                                          B->d_err, ade, npoles, B->storage, st);
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("batched bulk launch: ") + cudaGetErrorString(e));
        e = launch_slab_steps_batch(B->d_plans[in], B->d_boxes[g], B->nboxes[g], B->nslab_blocks[g], B->d_boxes4[g],
                                    B->nslab_blocks4[g], B->d_eboxes[g], B->neboxes[g], B->neblocks[g], ade, npoles,
                                    B->storage, st);
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("batched slab launch: ") + cudaGetErrorString(e));
    }
    if (B->nepboxes) {   // E of every instance's plain runs (after all H half steps)
        cudaError_t e = launch_slab_e_plain_batch(B->d_plans[in], B->d_epboxes, B->nepboxes, B->nepblocks, B->storage, st);
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("batched slab launch: ") + cudaGetErrorString(e));
    }
    if (B->max_nfff) launch_nfff_accumulate_batch(B->d_nfff[in], n, B->max_nfff, st);
    B->cur = 1 - in;
    return FDTD_OK;
}

// the instance plans follow the batch: parity, step count, last probes
int batch_after_steps(fdtd_batch *B, int nsteps)
{
    for (auto *P : B->plans) {
        P->cur = B->cur;
        P->host_step += nsteps;
        final_probes(P, B->stream);
    }
    CK(cudaGetLastError());
    return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_batch_create(const fdtd_desc *descs, int nplans, int device, fdtd_batch **out)
{
    if (!out) return fail(FDTD_E_INVALID, "out is NULL");
    *out = nullptr;
    if (!descs || nplans < 1) return fail(FDTD_E_INVALID, "no plans");
    for (int q = 0; q < nplans; q++)
        if (descs[q].nfff.enabled && descs[q].nfff.series)
            return fail(FDTD_E_UNSUPPORTED, "the time-domain far-field series is not available in a batch");
    for (int q = 1; q < nplans; q++)
        if (descs[q].storage != descs[0].storage)
            return fail(FDTD_E_UNSUPPORTED, "the instances of a batch must share one field storage type");
    if (nplans > 0 && descs[0].storage == FDTD_STORE_F64)
        return fail(FDTD_E_UNSUPPORTED, "FP64 storage is not available in a batch");
    fdtd_batch *B = new (std::nothrow) fdtd_batch();
    if (!B) return fail(FDTD_E_NOMEM, "host allocation failed");
    B->device = device;
    B->storage = descs[0].storage;
    auto bail = [&](int rc) { batch_free(B); return rc; };
    if (cudaSetDevice(device) != cudaSuccess) { delete B; return fail(FDTD_E_CUDA, "cudaSetDevice"); }
    cudaDeviceGetAttribute(&B->sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess) { delete B; return fail(FDTD_E_CUDA, "stream"); }
    for (int q = 0; q < nplans; q++) {
        fdtd_plan *P = nullptr;
        const int rc = plan_create_impl(&descs[q], device, &P, false);
        if (rc != FDTD_OK) {
            const std::string m = fdtd_last_error();
            batch_free(B);
            return fail(rc, "batch plan " + std::to_string(q) + ": " + m);
        }
        P->stream = B->stream;
        B->plans.push_back(P);
        B->group.push_back(!P->hp.has_ade ? 0 : P->hp.maxpoles > 0 ? 2 : 1);
        B->ncls = std::max(B->ncls, (int)P->hp.classes.size());
        B->max_tsf = std::max(B->max_tsf, P->tsf_cells);
        if (P->nfff && P->nfff_nfreq > 0) B->max_nfff = std::max(B->max_nfff, P->nfff_ns);
    }
#define BA(x, what) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { fail(FDTD_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); return bail(FDTD_E_CUDA); } } while (0)
    // per-instance parameter tables of both parities
    for (int in = 0; in < 2; in++) {
        std::vector<DevPlan> dp;
        std::vector<BulkMaps> bm(nplans);
        std::vector<DevAux> ax;
        std::vector<DevNfff> nf(nplans);
        std::memset(bm.data(), 0, sizeof(BulkMaps) * nplans);
        std::memset(nf.data(), 0, sizeof(DevNfff) * nplans);
        for (int q = 0; q < nplans; q++) {
            fdtd_plan *P = B->plans[q];
            dp.push_back(plan_for(P, in));
            if (P->bulk_on) bm[q] = P->bmaps[in];
            DevAux a = P->aux;
            a.fields = P->d_fieldptrs[in];
            ax.push_back(a);
            if (P->nfff && P->nfff_nfreq > 0) {
                nf[q] = P->nf;
                nf[q].e = P->d_efieldptrs[1 - in];
            }
        }
        BA(upload(B->mem, &B->d_plans[in], dp.data(), dp.size()), "batch tables");
        BA(upload(B->mem, &B->d_maps[in], bm.data(), bm.size()), "batch tables");
        BA(upload(B->mem, &B->d_aux[in], ax.data(), ax.size()), "batch tables");
        BA(upload(B->mem, &B->d_nfff[in], nf.data(), nf.size()), "batch tables");
    }
    // slab boxes of every instance (numbered one cell per thread), per kernel variant
    for (int g = 0; g < 3; g++) {
        std::vector<SlabBox> boxes;
        for (int q = 0; q < nplans; q++) {
            if (B->group[q] != g || B->plans[q]->tiles_on) continue;
            for (SlabBox b : B->plans[q]->h_boxes) {
                b.first_block = B->nslab_blocks[g];
                b.inst = q;
                boxes.push_back(b);
                B->nslab_blocks[g] += ((long long)(b.i1 - b.i0) * (b.j1 - b.j0) * (b.k1 - b.k0) + 255) / 256;
            }
        }
        if (B->nslab_blocks[g] > 0x7fffffffLL) { fail(FDTD_E_UNSUPPORTED, "too many slab cells for one launch"); return bail(FDTD_E_UNSUPPORTED); }
        BA(upload(B->mem, &B->d_boxes[g], boxes.data(), boxes.size()), "batch slab boxes");
        B->nboxes[g] = (int)boxes.size();
        // E runs with a dispersive cell, numbered for this variant's launch
        std::vector<SlabBox> ebx;
        for (int q = 0; q < nplans; q++) {
            if (B->group[q] != g || B->plans[q]->tiles_on) continue;
            for (SlabBox b : B->plans[q]->h_eboxes) {
                b.first_block = B->neblocks[g];
                b.inst = q;
                ebx.push_back(b);
                B->neblocks[g] += ((long long)(b.i1 - b.i0) * (b.j1 - b.j0) * (b.k1 - b.k0) + 255) / 256;
            }
        }
        if (B->neblocks[g] > 0x7fffffffLL) { fail(FDTD_E_UNSUPPORTED, "too many slab cells for one launch"); return bail(FDTD_E_UNSUPPORTED); }
        if (!ebx.empty()) BA(upload(B->mem, &B->d_eboxes[g], ebx.data(), ebx.size()), "batch slab boxes");
        B->neboxes[g] = (int)ebx.size();
        bool w4 = !boxes.empty();
        for (auto &b : boxes) w4 = w4 && B->plans[b.inst]->hp.zr % 4 == 0 && b.k0 % 4 == 0 && b.k1 % 4 == 0;
        if (w4) {
            for (auto &b : boxes) {
                b.first_block = B->nslab_blocks4[g];
                B->nslab_blocks4[g] += ((long long)(b.i1 - b.i0) * (b.j1 - b.j0) * ((b.k1 - b.k0) / 4) + 255) / 256;
            }
            BA(upload(B->mem, &B->d_boxes4[g], boxes.data(), boxes.size()), "batch slab boxes");
        }
    }
    {   // E runs without a dispersive cell, every instance in one launch
        std::vector<SlabBox> pbx;
        for (int q = 0; q < nplans; q++) {
            if (B->plans[q]->tiles_on) continue;
            for (SlabBox b : B->plans[q]->h_epboxes) {
                b.first_block = B->nepblocks;
                b.inst = q;
                pbx.push_back(b);
                B->nepblocks += ((long long)(b.i1 - b.i0) * (b.j1 - b.j0) * (b.k1 - b.k0) + 255) / 256;
            }
        }
        if (B->nepblocks > 0x7fffffffLL) { fail(FDTD_E_UNSUPPORTED, "too many slab cells for one launch"); return bail(FDTD_E_UNSUPPORTED); }
        if (!pbx.empty()) BA(upload(B->mem, &B->d_epboxes, pbx.data(), pbx.size()), "batch slab boxes");
        B->nepboxes = (int)pbx.size();
    }
    BA(B->mem.alloc(&B->d_err, 1), "error word");
    for (auto *P : B->plans) P->batch_err = B->d_err;   // the instances' readbacks check the batch's word too
    for (auto *P : B->plans) B->ntiled += P->tiles_on ? 1 : 0;
    if (B->ntiled) {
        for (int kind = 0; kind < NTILE; kind++) {
            for (int in = 0; in < 2; in++) {
                std::vector<BulkMaps> tm(nplans);
                std::memset(tm.data(), 0, sizeof(BulkMaps) * nplans);
                for (int q = 0; q < nplans; q++)
                    if (B->plans[q]->ntiles[kind]) tm[q] = B->plans[q]->tmaps[kind][in];
                BA(upload(B->mem, &B->d_tmaps[kind][in], tm.data(), tm.size()), "batch tile maps");
            }
            for (int g = 0; g < 3; g++) {
                std::vector<BulkItem> all;
                for (int q = 0; q < nplans; q++) {
                    if (B->group[q] != g || !B->plans[q]->tiles_on) continue;
                    for (BulkItem it : B->plans[q]->h_tiles[kind]) {
                        it.inst = q;
                        all.push_back(it);
                    }
                }
                if (!all.empty()) BA(upload(B->mem, &B->d_titems[g][kind], all.data(), all.size()), "batch tile lists");
                B->ntitems[g][kind] = (int)all.size();
            }
        }
    }
    BA(batch_set_items(B, 0, true), "batch work list");
    BA(cudaDeviceSynchronize(), "batch set-up");
#undef BA
    *out = B;
    return FDTD_OK;
}

int fdtd_batch_destroy(fdtd_batch *B)
{
    batch_free(B);
    return FDTD_OK;
}

int fdtd_batch_get_stream(const fdtd_batch *B, void **stream)
{
    if (!B || !stream) return fail(FDTD_E_INVALID, "NULL argument");
    *stream = (void *)B->stream;
    return FDTD_OK;
}

int fdtd_batch_size(const fdtd_batch *B, int *nplans)
{
    if (!B || !nplans) return fail(FDTD_E_INVALID, "NULL argument");
    *nplans = (int)B->plans.size();
    return FDTD_OK;
}

int fdtd_batch_plan(fdtd_batch *B, int index, fdtd_plan **plan)
{
    if (!B || !plan || index < 0 || index >= (int)B->plans.size()) return fail(FDTD_E_INVALID, "bad argument");
    *plan = B->plans[index];
    return FDTD_OK;
}

int fdtd_batch_step(fdtd_batch *B, int nsteps)
{
    if (!B || nsteps < 0) return fail(FDTD_E_INVALID, "bad argument");
    CK(cudaSetDevice(B->device));
    for (int s = 0; s < nsteps; s++) {
        const int rc = batch_launch_step(B, B->stream);
        if (rc != FDTD_OK) return rc;
    }
    return batch_after_steps(B, nsteps);
}

int fdtd_batch_step_graph(fdtd_batch *B, int nsteps, int chunk)
{
    if (!B || nsteps < 0) return fail(FDTD_E_INVALID, "bad argument");
    CK(cudaSetDevice(B->device));
    if (chunk < 2) chunk = 2;
    chunk &= ~1;   // an even number of steps returns the ping-pong parity
    if (B->graph_steps != chunk) {
        for (int s = 0; s < 2; s++)
            if (B->graph[s]) { cudaGraphExecDestroy(B->graph[s]); B->graph[s] = nullptr; }
        B->graph_steps = chunk;
    }
    int done = 0;
    while (nsteps - done >= chunk) {
        const int par = B->cur;
        if (!B->graph[par]) {
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
            for (int s = 0; s < chunk; s++) {
                const int rc = batch_launch_step(B, B->stream);
                if (rc != FDTD_OK) { cudaStreamEndCapture(B->stream, &g); B->cur = par; return rc; }
            }
            CK(cudaStreamEndCapture(B->stream, &g));
            cudaGraphExec_t ge;
            const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            B->graph[par] = ge;
            B->cur = par;   // capture advanced cur by chunk (even): unchanged
        }
        CK(cudaGraphLaunch(B->graph[par], B->stream));
        done += chunk;
    }
    for (int s = done; s < nsteps; s++) {
        const int rc = batch_launch_step(B, B->stream);
        if (rc != FDTD_OK) return rc;
    }
    return batch_after_steps(B, nsteps);
}

int fdtd_batch_sync(fdtd_batch *B)
{
    if (!B) return fail(FDTD_E_INVALID, "batch is NULL");
    CK(cudaSetDevice(B->device));
    CK(cudaStreamSynchronize(B->stream));
    int err = 0;
    CK(cudaMemcpy(&err, B->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(FDTD_E_TIMEOUT, "a bounded wait of the batched bulk kernel expired");
    for (auto *P : B->plans) {
        const int rc = fdtd_sync(P);
        if (rc != FDTD_OK) return rc;
    }
    return FDTD_OK;
}

int fdtd_batch_tune(fdtd_batch *B, int trial_steps, double *report, int report_len, int *ncand)
{
    if (!B || trial_steps < 1) return fail(FDTD_E_INVALID, "bad argument");
    CK(cudaSetDevice(B->device));
    CK(cudaStreamSynchronize(B->stream));
    // keep the state: every plan's stepping state into one device backup
    size_t total = 0;
    for (auto *P : B->plans)
        for (auto &it : P->snap) total += it.bytes;
    char *backup = nullptr;
    CK(cudaMalloc(&backup, std::max<size_t>(total, 16)));
    auto copy_state = [&](bool save) -> cudaError_t {
        char *q = backup;
        for (auto *P : B->plans)
            for (auto &it : P->snap) {
                cudaError_t e = save ? cudaMemcpyAsync(q, it.ptr, it.bytes, cudaMemcpyDeviceToDevice, B->stream)
                                     : cudaMemcpyAsync(it.ptr, q, it.bytes, cudaMemcpyDeviceToDevice, B->stream);
                if (e != cudaSuccess) return e;
                q += it.bytes;
            }
        return cudaSuccess;
    };
    const int cur0 = B->cur;
    std::vector<int> steps0;
    for (auto *P : B->plans) steps0.push_back(P->host_step);
    cudaError_t e = copy_state(true);
    // candidates: planes per item x (persistent grid | one CTA per item)
    const int lens[] = {8, 16, 32, 64, 1 << 20};
    int best_len = 0;
    bool best_pers = true;
    double best = 1e300;
    int n = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    for (int li = 0; li < 5 && e == cudaSuccess; li++)
        for (int pi = 0; pi < 2 && e == cudaSuccess; pi++) {
            const bool pers = (pi == 0);
            e = batch_set_items(B, lens[li], pers);
            if (e != cudaSuccess) break;
            int rc = batch_launch_step(B, B->stream);   // warm-up
            if (rc == FDTD_OK) e = cudaEventRecord(e0, B->stream);
            for (int s = 0; s < trial_steps && rc == FDTD_OK && e == cudaSuccess; s++) rc = batch_launch_step(B, B->stream);
            if (rc != FDTD_OK) { e = cudaErrorLaunchFailure; break; }
            if (e == cudaSuccess) e = cudaEventRecord(e1, B->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) break;
            if (report && 3 * n + 2 < report_len) {
                report[3 * n] = lens[li] == (1 << 20) ? 0 : lens[li];
                report[3 * n + 1] = pers ? 1 : 0;
                report[3 * n + 2] = ms / trial_steps;
            }
            n++;
            if (ms < best) { best = ms; best_len = lens[li]; best_pers = pers; }
        }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    // restore the state and keep the fastest work list
    B->cur = cur0;
    cudaError_t e2 = copy_state(false);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
    cudaFree(backup);
    for (size_t q = 0; q < B->plans.size(); q++) {
        B->plans[q]->cur = cur0;
        B->plans[q]->host_step = steps0[q];
    }
    if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("batch tuning: ") + cudaGetErrorString(e));
    if (ncand) *ncand = n;
    CK(batch_set_items(B, best_len, best_pers));
    return FDTD_OK;
}

int fdtd_batch_config(const fdtd_batch *B, int *planes_per_item, int *persistent, int *grid, int *items)
{
    if (!B) return fail(FDTD_E_INVALID, "batch is NULL");
    if (planes_per_item) *planes_per_item = B->chunk_len == (1 << 20) ? 0 : B->chunk_len;
    if (persistent) *persistent = B->persistent ? 1 : 0;
    if (grid) *grid = std::max(B->bulk_grid[0], std::max(B->bulk_grid[1], B->bulk_grid[2]));
    if (items) *items = B->nitems[0] + B->nitems[1] + B->nitems[2];
    return FDTD_OK;
}

}  // extern "C"

// ------------------------------------------------------------ adjoint
// (no counterpart in the reference)

namespace {

struct AdjBufs {             // adjoint state of one plan, zero-initialised
    DevBuf mem;
    DevAdj a;
    ~AdjBufs() { mem.free_all(); }
};

cudaError_t adj_alloc(fdtd_plan *P, AdjBufs &B)
{
    std::memset(&B.a, 0, sizeof(B.a));
    const size_t n = P->hp.n;
    cudaError_t e;
    for (int c = 0; c < 3; c++) {
        if ((e = B.mem.alloc(&B.a.eb[c], n)) != cudaSuccess) return e;
        if ((e = B.mem.alloc(&B.a.hb[c], n)) != cudaSuccess) return e;
    }
    for (int q = 0; q < 6; q++)
        if ((e = B.mem.alloc(&B.a.dd[q], n)) != cudaSuccess) return e;
    const HostPlan &hp = P->hp;
    for (int f = 0; f < 6; f++) {
        if (!hp.cp[f].enabled) continue;
        const int dep = hp.cp[f].depth;
        const size_t cnt = (f < 2) ? (size_t)dep * hp.yr * hp.zr : (f < 4) ? (size_t)hp.xr * dep * hp.zr : (size_t)hp.xr * hp.yr * dep;
        for (int q = 0; q < 2; q++) {
            if ((e = B.mem.alloc(&B.a.pe[f][q], cnt)) != cudaSuccess) return e;
            if ((e = B.mem.alloc(&B.a.ph[f][q], cnt)) != cudaSuccess) return e;
        }
    }
    if (hp.has_ade)
        for (int c = 0; c < 3; c++) {
            if ((e = B.mem.alloc(&B.a.ep[c], n)) != cudaSuccess) return e;
            if ((e = B.mem.alloc(&B.a.q[c], n)) != cudaSuccess) return e;
            for (int m = 0; m < hp.maxpoles; m++) {
                if ((e = B.mem.alloc(&B.a.pc[c][m], n)) != cudaSuccess) return e;
                if ((e = B.mem.alloc(&B.a.qc[c][m], n)) != cudaSuccess) return e;
            }
        }
    return cudaSuccess;
}

// transpose of the step with index `step`: the objective's dJ/dE of that step,
// the design accumulation, then the E and H half steps in reverse order
void adj_step_back(fdtd_plan *P, AdjBufs &B, const DevObjective *obj, int step, const DevGrad *g, int slot)
{
    if (obj) launch_adjoint_source(*obj, B.a, step, P->stream);
    if (g) launch_design_accumulate(B.a, P->dp, *g, slot, P->stream);
    launch_adjoint_e(P->dp, B.a, P->stream);
    launch_adjoint_h(P->dp, B.a, P->stream);
}

struct DevCheckpoints {      // device copies of the stepping state
    DevBuf mem;
    size_t bytes = 0;
    std::vector<unsigned char *> slot;
    std::vector<int> cur, step;
    ~DevCheckpoints() { mem.free_all(); }
};

cudaError_t ckpt_alloc(fdtd_plan *P, DevCheckpoints &K, int nslots)
{
    for (auto &s : P->snap) K.bytes += (s.bytes + 255) / 256 * 256;
    for (int q = 0; q < nslots; q++) {
        unsigned char *p;
        cudaError_t e = K.mem.alloc(&p, K.bytes);
        if (e != cudaSuccess) return e;
        K.slot.push_back(p);
    }
    K.cur.assign(nslots, 0);
    K.step.assign(nslots, 0);
    return cudaSuccess;
}

cudaError_t ckpt_save(fdtd_plan *P, DevCheckpoints &K, int q)
{
    size_t off = 0;
    for (auto &s : P->snap) {
        cudaError_t e = cudaMemcpyAsync(K.slot[q] + off, s.ptr, s.bytes, cudaMemcpyDeviceToDevice, P->stream);
        if (e != cudaSuccess) return e;
        off += (s.bytes + 255) / 256 * 256;
    }
    K.cur[q] = P->cur;
    K.step[q] = P->host_step;
    return cudaSuccess;
}

cudaError_t ckpt_restore(fdtd_plan *P, DevCheckpoints &K, int q)
{
    size_t off = 0;
    for (auto &s : P->snap) {
        cudaError_t e = cudaMemcpyAsync(s.ptr, K.slot[q] + off, s.bytes, cudaMemcpyDeviceToDevice, P->stream);
        if (e != cudaSuccess) return e;
        off += (s.bytes + 255) / 256 * 256;
    }
    P->cur = K.cur[q];
    P->host_step = K.step[q];
    return cudaSuccess;
}

int check_objective(const fdtd_plan *P, const fdtd_objective *obj)
{
    if (!obj) return fail(FDTD_E_INVALID, "objective is NULL");
    if (!P->nfff || P->nfff_nfreq <= 0) return fail(FDTD_E_STATE, "the objective needs the running-DFT far field (nfff.nfreq > 0)");
    if (obj->freq < 0 || obj->freq >= P->nfff_nfreq) return fail(FDTD_E_INVALID, "objective frequency index out of range");
    if (obj->npoints < 1 || !obj->points || !obj->weights) return fail(FDTD_E_INVALID, "objective without far points");
    for (int t = 0; t < obj->npoints; t++) {
        if (obj->points[t] < 0 || obj->points[t] >= P->nfff_npoints) return fail(FDTD_E_INVALID, "objective far point out of range");
        if (!std::isfinite(obj->weights[t])) return fail(FDTD_E_INVALID, "objective weight not finite");
    }
    return FDTD_OK;
}

// J of the spectrum now in P->ff.out (host copy of the objective's points)
int objective_from_spectrum(fdtd_plan *P, const fdtd_objective *obj, double *J)
{
    const size_t n = (size_t)P->nfff_npoints * P->nfff_nfreq * 3;
    std::vector<double2> spec(n);
    CK(cudaMemcpyAsync(spec.data(), P->ff.out, n * sizeof(double2), cudaMemcpyDeviceToHost, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    const int rc = device_error(P);
    if (rc != FDTD_OK) return rc;
    double j = 0;
    for (int t = 0; t < obj->npoints; t++)
        for (int c = 0; c < 3; c++) {
            const double2 f = spec[((size_t)obj->points[t] * P->nfff_nfreq + obj->freq) * 3 + c];
            j += obj->weights[t] * (f.x * f.x + f.y * f.y);
        }
    *J = j;
    return FDTD_OK;
}

int check_adjoint_plan(const fdtd_plan *P)
{
    if (P->storage != FDTD_STORE_F32) return fail(FDTD_E_UNSUPPORTED, "the adjoint needs FP32 field storage");
    return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_objective_value(fdtd_plan *P, const fdtd_objective *obj, double *J)
{
    if (!P || !J) return fail(FDTD_E_INVALID, "NULL argument");
    int rc = check_objective(P, obj);
    if (rc != FDTD_OK) return rc;
    CK(cudaSetDevice(P->device));
    launch_nfff_fold_pending(P->nf, P->stream);
    launch_farfield_finalize(P->ff, P->stream);
    CK(cudaGetLastError());
    return objective_from_spectrum(P, obj, J);
}

int fdtd_adjoint_transpose(fdtd_plan *P, int nsteps, double *const comps[6])
{
    if (!P || !comps || nsteps < 0) return fail(FDTD_E_INVALID, "bad argument");
    for (int c = 0; c < 6; c++)
        if (!comps[c]) return fail(FDTD_E_INVALID, "component pointer is NULL");
    int rc = check_adjoint_plan(P);
    if (rc != FDTD_OK) return rc;
    CK(cudaSetDevice(P->device));
    AdjBufs B;
    CK(adj_alloc(P, B));
    const size_t n = P->hp.n;
    std::vector<float> tmp(n);
    for (int c = 0; c < 6; c++) {
        for (size_t q = 0; q < n; q++) tmp[q] = (float)comps[c][q];
        CK(cudaMemcpy(c < 3 ? B.a.eb[c] : B.a.hb[c - 3], tmp.data(), n * 4, cudaMemcpyHostToDevice));
    }
    for (int s = 0; s < nsteps; s++) adj_step_back(P, B, nullptr, 0, nullptr, 0);
    CK(cudaGetLastError());
    for (int c = 0; c < 6; c++) {
        CK(cudaMemcpyAsync(tmp.data(), c < 3 ? B.a.eb[c] : B.a.hb[c - 3], n * 4, cudaMemcpyDeviceToHost, P->stream));
        CK(cudaStreamSynchronize(P->stream));
        for (size_t q = 0; q < n; q++) comps[c][q] = (double)tmp[q];
    }
    return FDTD_OK;
}

int fdtd_adjoint_gradient(fdtd_plan *P, const fdtd_objective *obj, int nsteps, int checkpoint, double *J, double *grad)
{
    if (!P || !J || !grad || nsteps < 1 || checkpoint < 1) return fail(FDTD_E_INVALID, "bad argument");
    if (!P->hp.design) return fail(FDTD_E_STATE, "the plan has no design region");
    if (P->failed) return refuse_failed(P);
    int rc = check_objective(P, obj);
    if (rc == FDTD_OK) rc = check_adjoint_plan(P);
    if (rc != FDTD_OK) return rc;
    CK(cudaSetDevice(P->device));
    const int K = std::min(checkpoint, nsteps), nseg = (nsteps + K - 1) / K;
    DevCheckpoints ck;
    {
        cudaError_t e = ckpt_alloc(P, ck, nseg + 1);
        if (e != cudaSuccess) return fail(FDTD_E_NOMEM, std::string("adjoint checkpoints: ") + cudaGetErrorString(e));
    }
    // forward pass with a checkpoint at the start of every segment
    for (int m = 0; m < nsteps; m++) {
        if (m % K == 0) CK(ckpt_save(P, ck, m / K));
        rc = launch_step(P, P->stream);
        if (rc != FDTD_OK) return rc;
        P->host_step++;
    }
    final_probes(P, P->stream);
    CK(ckpt_save(P, ck, nseg));
    launch_nfff_fold_pending(P->nf, P->stream);
    launch_farfield_finalize(P->ff, P->stream);
    CK(cudaGetLastError());
    rc = objective_from_spectrum(P, obj, J);
    if (rc != FDTD_OK) return rc;
    // objective weights, adjoint state, design accumulators
    DevBuf mem;
    struct Free { DevBuf &m; ~Free() { m.free_all(); } } guard{mem};
    int32_t *dpts;
    double *dw;
    double2 *ae, *ad;
    const int ns = P->nf.ns;
    CK(upload(mem, &dpts, obj->points, (size_t)obj->npoints));
    CK(upload(mem, &dw, obj->weights, (size_t)obj->npoints));
    CK(mem.alloc(&ae, (size_t)3 * ns));
    CK(mem.alloc(&ad, (size_t)3 * ns));
    launch_objective_weights(P->ff, obj->freq, obj->npoints, dpts, dw, P->ff.out, ae, ad, P->stream);
    DevObjective o;
    o.ns = ns;
    o.cell = P->nf.cell;
    o.nstride = P->nf.nstride;
    o.inv2dx = P->nf.inv2dx;
    o.omega_dt = P->omega[obj->freq] * P->hp.dt;
    o.ae = ae;
    o.ad = ad;
    DevGrad g;
    for (int q = 0; q < 6; q++) g.box[q] = P->hp.abox[q];
    g.ncell = (int64_t)(g.box[1] - g.box[0]) * (g.box[3] - g.box[2]) * (g.box[5] - g.box[4]);
    CK(mem.alloc(&g.g, (size_t)3 * g.ncell));
    {
        cudaError_t e = mem.alloc(&g.curl, (size_t)K * 3 * g.ncell);
        if (e != cudaSuccess) return fail(FDTD_E_NOMEM, std::string("adjoint curl buffer: ") + cudaGetErrorString(e));
    }
    AdjBufs B;
    CK(adj_alloc(P, B));
    // backward: recompute each segment from its checkpoint, then its steps in reverse
    for (int seg = nseg - 1; seg >= 0; seg--) {
        const int m0 = seg * K, m1 = std::min(nsteps, m0 + K);
        CK(ckpt_restore(P, ck, seg));
        for (int m = m0; m < m1; m++) {
            rc = launch_step(P, P->stream);
            if (rc != FDTD_OK) return rc;
            P->host_step++;
            launch_design_curl(plan_for(P, 1 - P->cur), g, m - m0, P->stream);
        }
        for (int m = m1 - 1; m >= m0; m--) adj_step_back(P, B, &o, m, &g, m - m0);
        CK(cudaGetLastError());
    }
    CK(ckpt_restore(P, ck, nseg));
    std::vector<double> dcb((size_t)3 * g.ncell);
    CK(cudaMemcpyAsync(dcb.data(), g.g, dcb.size() * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    design_gradient(&P->hp, dcb.data(), grad);
    return FDTD_OK;
}

}  // extern "C"

