// fdtd_api.cu -- the C ABI of include/gsvit_b200.h.
//
// Owns the device state of one plan and sequences the kernels of a step on a
// single CUDA stream.  The reference's GPU driver (gpu.c) keeps a worker
// thread per GPU, pushes one token per stage and spins on the host after
// every launch (gpu.c:787-801, gpu_kernels.cu:6063-6068); here a step is
// three stream-ordered launches with no host synchronisation, and
// fdtd_step_graph replays them from a CUDA graph.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gsvit_b200.h"
#include "fdtd_internal.h"
#include "fdtd_kernels.cuh"
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
    int ichunk = 0;
    // NFFF
    bool nfff = false;
    int nfff_npoints = 0, nfff_nfreq = 0, nfff_ns = 0;
    DevNfff nf;
    const float **d_efieldptrs[2] = {nullptr, nullptr};
    DevFarfield ff;
    std::vector<double> omega;
    // graphs per parity
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_steps = 0;
    cudaStream_t graph_stream[2] = {nullptr, nullptr};
    std::vector<SnapItem> snap;
    double step_bytes = 0;
};

namespace {

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

int launch_step(fdtd_plan *P, cudaStream_t st)
{
    const int in = P->cur;
    DevAux a = P->aux;
    a.fields = P->d_fieldptrs[in];
    launch_aux_step(a, st);
    DevPlan d = plan_for(P, in);
    cudaError_t e = launch_fused_step(d, P->ichunk, P->hp.has_ade, P->hp.maxpoles, st);
    if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("fused step launch: ") + cudaGetErrorString(e));
    if (P->nfff) {
        DevNfff n = P->nf;
        n.e = P->d_efieldptrs[1 - in];
        launch_nfff_accumulate(n, st);
    }
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

int fdtd_plan_create(const fdtd_desc *desc, int device, fdtd_plan **out)
{
    if (!out) return fail(FDTD_E_INVALID, "out is NULL");
    *out = nullptr;
    if (!desc) return fail(FDTD_E_INVALID, "desc is NULL");
    if (desc->storage != FDTD_STORE_F32)
        return fail(FDTD_E_UNSUPPORTED, "reduced-precision field storage is not available in this build");
    fdtd_plan *P = new (std::nothrow) fdtd_plan();
    if (!P) return fail(FDTD_E_NOMEM, "host allocation failed");
    std::string err;
    int rc = build_host_plan(desc, &P->hp, &err);
    if (rc != FDTD_OK) {
        delete P;
        return fail(rc, err);
    }
    HostPlan &hp = P->hp;
    P->device = device;
    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) { delete P; return fail(FDTD_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce)); }
    auto bail = [&](cudaError_t e, const char *what) {
        P->mem.free_all();
        if (P->own_stream) cudaStreamDestroy(P->own_stream);
        delete P;
        return fail(e == cudaErrorMemoryAllocation ? FDTD_E_NOMEM : FDTD_E_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
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
    for (int s = 0; s < 2; s++)
        for (int c = 0; c < 6; c++) {
            CA(P->mem.alloc(&P->fields[s][c], n), "field allocation");
            P->snap.push_back({P->fields[s][c], n * sizeof(float)});
        }
    uint8_t *cls;
    CA(upload(P->mem, &cls, hp.cls.data(), n), "class map");
    d.cls = cls;
    DevClass *classes;
    CA(upload(P->mem, &classes, hp.classes.data(), hp.classes.size()), "class table");
    d.classes = classes;
    d.nclasses = (int)hp.classes.size();
    double bytes = 49.0 * (double)n;   // 6 field reads + 6 writes + class byte
    if (hp.has_ade) {
        DevAde *ade;
        CA(upload(P->mem, &ade, hp.ades.data(), hp.ades.size()), "ADE table");
        d.ade = ade;
        d.nade = (int)hp.ades.size();
        for (int a = 0; a < 3; a++) {
            CA(P->mem.alloc(&d.ep[a], n), "ADE state");
            CA(P->mem.alloc(&d.dp[a], n), "ADE state");
            CA(P->mem.alloc(&d.dpp[a], n), "ADE state");
            P->snap.push_back({d.ep[a], n * 4}); P->snap.push_back({d.dp[a], n * 4}); P->snap.push_back({d.dpp[a], n * 4});
            for (int q = 0; q < hp.maxpoles; q++) {
                CA(P->mem.alloc(&d.p_[a][q], n), "ADE state");
                CA(P->mem.alloc(&d.pp_[a][q], n), "ADE state");
                P->snap.push_back({d.p_[a][q], n * 4}); P->snap.push_back({d.pp_[a][q], n * 4});
            }
        }
        size_t nd = 0;   // dispersive cells: per owned component E^{n-1}, P_D, P_D^{n-1} (+4 per pole) read+written
        for (size_t c = 0; c < n; c++) {
            const DevClass &k = hp.classes[hp.cls[c]];
            if (k.flags & CF_ADE_BRANCH)
                nd += ((k.flags & CF_ADE_X) ? 1 : 0) + ((k.flags & CF_ADE_Y) ? 1 : 0) + ((k.flags & CF_ADE_Z) ? 1 : 0);
        }
        bytes += (double)nd * (3 + 4 * hp.maxpoles) * 8.0;
    }
    // CPML
    for (int f = 0; f < 6; f++) {
        d.cp_on[f] = hp.cp[f].enabled;
        d.cp_d[f] = hp.cp[f].depth;
        if (!hp.cp[f].enabled) continue;
        const int dep = hp.cp[f].depth;
        float *be, *ce, *bh, *ch;
        CA(upload(P->mem, &be, hp.be[f].data(), dep), "cpml");
        CA(upload(P->mem, &ce, hp.ce[f].data(), dep), "cpml");
        CA(upload(P->mem, &bh, hp.bh[f].data(), dep), "cpml");
        CA(upload(P->mem, &ch, hp.ch[f].data(), dep), "cpml");
        d.be[f] = be; d.ce[f] = ce; d.bh[f] = bh; d.ch[f] = ch;
        size_t cnt = (f < 2) ? (size_t)dep * hp.yr * hp.zr : (f < 4) ? (size_t)hp.xr * dep * hp.zr : (size_t)hp.xr * hp.yr * dep;
        for (int q = 0; q < 2; q++) {
            CA(P->mem.alloc(&d.psie[f][q], cnt), "cpml psi");
            P->snap.push_back({d.psie[f][q], cnt * 4});
            for (int s = 0; s < 2; s++) {
                CA(P->mem.alloc(&P->psih[s][f][q], cnt), "cpml psi");
                P->snap.push_back({P->psih[s][f][q], cnt * 4});
            }
        }
        bytes += (double)cnt * 4 * 2 * 4;   // 4 psi arrays read + written
    }
    for (int ax = 0; ax < 3; ax++) {
        float *a, *b;
        CA(upload(P->mem, &a, hp.ike[ax].data(), hp.ike[ax].size()), "kappa");
        CA(upload(P->mem, &b, hp.ikh[ax].data(), hp.ikh[ax].size()), "kappa");
        d.ike[ax] = a;
        d.ikh[ax] = b;
    }
    // TSF
    std::memset(&P->aux, 0, sizeof(P->aux));
    CA(P->mem.alloc(&P->d_step, 1), "step counter");
    P->snap.push_back({P->d_step, sizeof(int)});
    P->aux.step = P->d_step;
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
    if (desc->nfff.enabled && desc->nfff.npoints > 0 && desc->nfff.nfreq > 0) {
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
        P->omega.assign(f.omega, f.omega + f.nfreq);
        std::vector<double> odt(f.nfreq);
        for (int q = 0; q < f.nfreq; q++) odt[q] = f.omega[q] * hp.dt;
        int32_t *dcell, *dnstr, *dijk, *dpts, *dist;
        int8_t *dface;
        double *dodt, *dom;
        double2 *acc, *outp;
        CA(upload(P->mem, &dcell, cell.data(), cell.size()), "nfff");
        CA(upload(P->mem, &dnstr, nstr.data(), nstr.size()), "nfff");
        CA(upload(P->mem, &dijk, ijk.data(), ijk.size()), "nfff");
        CA(upload(P->mem, &dface, face.data(), face.size()), "nfff");
        CA(upload(P->mem, &dodt, odt.data(), odt.size()), "nfff");
        CA(upload(P->mem, &dom, f.omega, (size_t)f.nfreq), "nfff");
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
        const size_t nacc = (size_t)f.nfreq * 6 * cell.size();
        CA(P->mem.alloc(&acc, nacc), "nfff accumulators");
        P->snap.push_back({acc, nacc * sizeof(double2)});
        CA(P->mem.alloc(&outp, (size_t)f.npoints * f.nfreq * 3), "nfff output");
        for (int s = 0; s < 2; s++) {
            const float **fp;
            CA(P->mem.alloc(&fp, 3), "field pointer table");
            CA(cudaMemcpy(fp, P->fields[s], sizeof(float *) * 3, cudaMemcpyHostToDevice), "field pointer table");
            P->d_efieldptrs[s] = fp;
        }
        P->nf.ns = (int)cell.size();
        P->nf.nfreq = f.nfreq;
        P->nf.cell = dcell;
        P->nf.nstride = dnstr;
        P->nf.acc = acc;
        P->nf.omega_dt = dodt;
        P->nf.step = P->d_step;
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
        bytes += (double)cell.size() * (9 * 4 + (double)f.nfreq * 6 * 16 * 2);
    }
    // i-chunking: enough CTAs to fill the SMs a few times over
    {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int tiles = ((hp.zr + FDTD_TK - 1) / FDTD_TK) * ((hp.yr + FDTD_TJ - 1) / FDTD_TJ);
        int want = (4 * sms + tiles - 1) / tiles;
        int chunks = std::max(1, std::min(want, hp.xr / 16));
        P->ichunk = (hp.xr + chunks - 1) / chunks;
    }
    P->step_bytes = bytes;
    CA(cudaDeviceSynchronize(), "plan set-up");
#undef CA
    *out = P;
    return FDTD_OK;
}

int fdtd_plan_destroy(fdtd_plan *P)
{
    if (!P) return FDTD_OK;
    cudaSetDevice(P->device);
    if (P->stream) cudaStreamSynchronize(P->stream);
    for (int s = 0; s < 2; s++)
        if (P->graph[s]) cudaGraphExecDestroy(P->graph[s]);
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
    return FDTD_OK;
}

int fdtd_set_fields(fdtd_plan *P, int mask, const double *const comps[6])
{
    if (!P || !comps) return fail(FDTD_E_INVALID, "NULL argument");
    CK(cudaSetDevice(P->device));
    std::vector<float> tmp(P->hp.n);
    for (int c = 0; c < 6; c++) {
        if (!(mask & (1 << c))) continue;
        if (!comps[c]) return fail(FDTD_E_INVALID, "selected component pointer is NULL");
        for (size_t q = 0; q < P->hp.n; q++) tmp[q] = (float)comps[c][q];
        CK(cudaMemcpyAsync(P->fields[P->cur][c], tmp.data(), P->hp.n * 4, cudaMemcpyHostToDevice, P->stream));
        CK(cudaStreamSynchronize(P->stream));
    }
    return FDTD_OK;
}

int fdtd_set_fields_f32(fdtd_plan *P, int mask, const float *const comps[6])
{
    if (!P || !comps) return fail(FDTD_E_INVALID, "NULL argument");
    CK(cudaSetDevice(P->device));
    for (int c = 0; c < 6; c++) {
        if (!(mask & (1 << c))) continue;
        if (!comps[c]) return fail(FDTD_E_INVALID, "selected component pointer is NULL");
        CK(cudaMemcpyAsync(P->fields[P->cur][c], comps[c], P->hp.n * 4, cudaMemcpyHostToDevice, P->stream));
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
        CK(cudaMemcpyAsync(comps[c], P->fields[P->cur][c], P->hp.n * 4, cudaMemcpyDeviceToHost, P->stream));
    }
    CK(cudaStreamSynchronize(P->stream));
    return FDTD_OK;
}

int fdtd_get_fields(fdtd_plan *P, int mask, double *const comps[6])
{
    if (!P || !comps) return fail(FDTD_E_INVALID, "NULL argument");
    CK(cudaSetDevice(P->device));
    std::vector<float> tmp(P->hp.n);
    for (int c = 0; c < 6; c++) {
        if (!(mask & (1 << c))) continue;
        if (!comps[c]) return fail(FDTD_E_INVALID, "selected component pointer is NULL");
        CK(cudaMemcpyAsync(tmp.data(), P->fields[P->cur][c], P->hp.n * 4, cudaMemcpyDeviceToHost, P->stream));
        CK(cudaStreamSynchronize(P->stream));
        for (size_t q = 0; q < P->hp.n; q++) comps[c][q] = (double)tmp[q];
    }
    return FDTD_OK;
}

int fdtd_step(fdtd_plan *P, int nsteps)
{
    if (!P || nsteps < 0) return fail(FDTD_E_INVALID, "bad argument");
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

int fdtd_step_graph(fdtd_plan *P, int nsteps, int chunk)
{
    if (!P || nsteps < 0) return fail(FDTD_E_INVALID, "bad argument");
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
    CK(cudaSetDevice(P->device));
    std::vector<cudaEvent_t> ev(2 * (size_t)nsteps);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    for (int s = 0; s < nsteps; s++) {
        const int in = P->cur;
        DevAux a = P->aux;
        a.fields = P->d_fieldptrs[in];
        launch_aux_step(a, P->stream);
        DevPlan d = plan_for(P, in);
        CK(cudaEventRecord(ev[2 * s], P->stream));
        cudaError_t e = launch_fused_step(d, P->ichunk, P->hp.has_ade, P->hp.maxpoles, P->stream);
        CK(cudaEventRecord(ev[2 * s + 1], P->stream));
        if (e != cudaSuccess) return fail(FDTD_E_CUDA, std::string("fused step launch: ") + cudaGetErrorString(e));
        if (P->nfff) {
            DevNfff n = P->nf;
            n.e = P->d_efieldptrs[1 - in];
            launch_nfff_accumulate(n, P->stream);
        }
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

int fdtd_get_probes(fdtd_plan *P, double *out, size_t out_len)
{
    if (!P || (!out && out_len)) return fail(FDTD_E_INVALID, "NULL argument");
    size_t need = P->hp.probes.size() * 6 * (size_t)std::max(P->hp.nsteps, 1);
    if (P->hp.probes.empty()) return FDTD_OK;
    if (out_len < need) return fail(FDTD_E_INVALID, "probe buffer too small");
    CK(cudaSetDevice(P->device));
    CK(cudaMemcpyAsync(out, P->aux.probe_out, need * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    return FDTD_OK;
}

int fdtd_nfff_spectrum(fdtd_plan *P, double *out, size_t out_len)
{
    if (!P || !out) return fail(FDTD_E_INVALID, "NULL argument");
    if (!P->nfff) return fail(FDTD_E_STATE, "the plan has no NFFF box / frequencies");
    size_t need = (size_t)P->nfff_npoints * P->nfff_nfreq * 3 * 2;
    if (out_len < need) return fail(FDTD_E_INVALID, "spectrum buffer too small");
    CK(cudaSetDevice(P->device));
    launch_farfield_finalize(P->ff, P->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, P->ff.out, need * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    return FDTD_OK;
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
        CK(cudaMemcpy(tmp.data(), P->dp.cls, n, cudaMemcpyDeviceToHost));
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
    return FDTD_OK;
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
