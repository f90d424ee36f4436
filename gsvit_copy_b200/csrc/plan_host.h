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
};

int build_host_plan(const fdtd_desc *d, HostPlan *hp, std::string *err);
