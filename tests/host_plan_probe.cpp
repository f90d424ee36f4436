// host_plan_probe.cpp -- test infrastructure: a C entry point over the
// library's host planner (gsvit_copy_b200/csrc/plan_host.cpp), built with g++
// by tests/test_host_plan.py, so that the CPU suite checks the planner's
// integer maps and coefficient classes without a GPU.  Not part of the library.
#include <cstdio>
#include <cstring>
#include <string>

#include "../gsvit_copy_b200/csrc/plan_host.h"

// which: FDTD_MAP_BNDS, FDTD_MAP_SOURCESKIP or FDTD_MAP_CLASS (per-cell class
// index); *nclasses receives the number of coefficient classes.  Returns 0, the
// planner's status, or -1 when out_len is short; err receives its message.
extern "C" int host_plan_map(const fdtd_desc *d, int which, int32_t *out, size_t out_len, int *nclasses, char *err,
                             size_t err_len)
{
    HostPlan hp;
    std::string e;
    const int rc = build_host_plan(d, &hp, &e);
    if (rc != 0) {
        std::snprintf(err, err_len, "%s", e.c_str());
        return rc;
    }
    if (out_len < hp.n) return -1;
    for (size_t c = 0; c < hp.n; c++)
        out[c] = which == FDTD_MAP_BNDS ? hp.bnds[c] : which == FDTD_MAP_SOURCESKIP ? hp.sskip[c] : hp.cls[c];
    *nclasses = (int)hp.classes.size();
    return 0;
}

// The planner's coefficient class table: up to max_classes DevClass records
// (64 bytes each, layout of fdtd_internal.h) into out; returns the number of
// classes, or a negative status.
extern "C" int host_plan_classes(const fdtd_desc *d, void *out, int max_classes, char *err, size_t err_len)
{
    HostPlan hp;
    std::string e;
    const int rc = build_host_plan(d, &hp, &e);
    if (rc != 0) {
        std::snprintf(err, err_len, "%s", e.c_str());
        return rc < 0 ? rc : -rc;
    }
    const int n = (int)hp.classes.size();
    if (n > max_classes) return -1;
    std::memcpy(out, hp.classes.data(), sizeof(DevClass) * n);
    return n;
}

// CPML profiles of one face (0..5: x0 xn y0 yn z0 zn) as the planner holds
// them: be, ce, bh, ch (FP32) and kappa_e, kappa_h (FP64), `cap` entries at
// most each; returns the face depth (0 for a disabled face) or a negative status.
extern "C" int host_plan_cpml(const fdtd_desc *d, int face, float *be, float *ce, float *bh, float *ch, double *ke,
                              double *kh, int cap)
{
    HostPlan hp;
    std::string e;
    if (build_host_plan(d, &hp, &e) != 0 || face < 0 || face > 5) return -1;
    if (!hp.cp[face].enabled) return 0;
    const int n = (int)hp.be[face].size();
    if (n > cap) return -1;
    for (int q = 0; q < n; q++) {
        be[q] = hp.be[face][q];
        ce[q] = hp.ce[face][q];
        bh[q] = hp.bh[face][q];
        ch[q] = hp.ch[face][q];
        ke[q] = q < (int)hp.ke[face].size() ? hp.ke[face][q] : 0.0;
        kh[q] = q < (int)hp.kh[face].size() ? hp.kh[face][q] : 0.0;
    }
    return n;
}

// Scalars of the plan: aux-grid resolution (0 without TSF), whether an ADE
// material exists, the critical-point pole count of the kernels.
extern "C" int host_plan_scalars(const fdtd_desc *d, int *jres, int *has_ade, int *maxpoles)
{
    HostPlan hp;
    std::string e;
    if (build_host_plan(d, &hp, &e) != 0) return -1;
    *jres = hp.tsf ? hp.jres : 0;
    *has_ade = hp.has_ade ? 1 : 0;
    *maxpoles = hp.maxpoles;
    return 0;
}

// Design region of the plan: the affected box (abox, i0 i1 j0 j1 k0 k1) and
// its per-cell E coefficients (ca[3], cb[3] per cell, abox order, k fastest),
// recomputed for eps_r (dbox order) first when eps_r is not NULL; returns the
// number of cells, 0 without a design region, or -1.
extern "C" long long host_plan_design(const fdtd_desc *d, const double *eps_r, int abox[6], float *dcoef, size_t cap)
{
    HostPlan hp;
    std::string e;
    if (build_host_plan(d, &hp, &e) != 0) return -1;
    if (!hp.design) return 0;
    if (eps_r) design_coefficients(&hp, eps_r);
    for (int q = 0; q < 6; q++) abox[q] = hp.abox[q];
    if (hp.dcoef.size() > cap) return -1;
    std::memcpy(dcoef, hp.dcoef.data(), sizeof(float) * hp.dcoef.size());
    return (long long)(hp.dcoef.size() / 6);
}

// The chain rule of the design region at permittivities eps_r: grad (dbox
// order) = dJ/d eps_r for dJ/dcb = dcb (3 per affected cell, abox order).
extern "C" int host_plan_design_gradient(const fdtd_desc *d, const double *eps_r, const double *dcb, double *grad)
{
    HostPlan hp;
    std::string e;
    if (build_host_plan(d, &hp, &e) != 0 || !hp.design) return -1;
    design_coefficients(&hp, eps_r);
    design_gradient(&hp, dcb, grad);
    return 0;
}

// The planner's ADE coefficient sets (DevAde, in the order of the ADE
// materials); *record receives sizeof(DevAde).  Returns the number of sets or -1.
extern "C" int host_plan_ades(const fdtd_desc *d, void *out, int max_sets, int *record)
{
    HostPlan hp;
    std::string e;
    if (build_host_plan(d, &hp, &e) != 0) return -1;
    *record = (int)sizeof(DevAde);
    const int n = (int)hp.ades.size();
    if (n > max_sets) return -1;
    std::memcpy(out, hp.ades.data(), sizeof(DevAde) * n);
    return n;
}
