// plan_host.h -- host plan produced from an fdtd_desc (see plan_host.cpp).
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/gsvit_b200.h"
#include "fdtd_internal.h"

struct HostPlan {
    int xr = 0, yr = 0, zr = 0;
    size_t n = 0;
    double dx = 0, dt = 0;
    int nsteps = 0;
    std::vector<uint8_t> cls;            // per-cell class index
    std::vector<DevClass> classes;
    std::vector<DevAde> ades;
    // FDTD_STORE_F64 plans: the same tables in FP64 (classes then deduplicated
    // on the FP64 coefficients, so classes64[c] rounds to classes[c])
    bool real64 = false;
    std::vector<DevClass64> classes64;
    std::vector<DevAde64> ades64;
    std::vector<double> be64[6], ce64[6], bh64[6], ch64[6];
    std::vector<double> ike64[3], ikh64[3];
    std::vector<double> dcoef64;
    bool has_ade = false;
    int maxpoles = 0;
    std::vector<int8_t> bnds, sskip;     // derived maps (plan.c:5387-5416, 5298-5326)
    fdtd_cpml_face cp[6];
    std::vector<float> be[6], ce[6], bh[6], ch[6];
    std::vector<double> ke[6], kh[6];
    std::vector<float> ike[3], ikh[3];
    bool tsf = false;
    double corr = 1, jdx = 0;
    int jres = 0;
    std::vector<double> wave;
    std::vector<uint8_t> tmap[6];
    int tmap_dims[6][2];
    std::vector<int64_t> probes;         // linear cell indices
    // adjoint design region: per-cell epsilon of the box dbox; the E
    // coefficients of the affected box abox (dbox plus one cell above on each
    // axis) are per cell, 6 floats (ca[3], cb[3]) each, from the epsilon and
    // sigma of the context box (abox plus one cell below on each axis)
    bool design = false;
    int dbox[6] = {0, 0, 0, 0, 0, 0}, abox[6] = {0, 0, 0, 0, 0, 0}, cbox[6] = {0, 0, 0, 0, 0, 0};
    std::vector<double> ctx_eps, ctx_sig;
    std::vector<float> dcoef;
};

// recompute the per-cell coefficients of the design region for new relative
// permittivities of its cells (eps_r, dbox order, k fastest)
void design_coefficients(HostPlan *hp, const double *eps_r);

// dJ/d eps_r of every design cell (dbox order) from dJ/dcb of the affected
// cells (3 per cell, abox order): the chain rule through the edge averaging
// of get_cabs (yee.c:1397-1493) of lossless cells, cb = dt / (eps dx)
void design_gradient(const HostPlan *hp, const double *dcb, double *grad);

int build_host_plan(const fdtd_desc *d, HostPlan *hp, std::string *err);
