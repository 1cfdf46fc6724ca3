// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// POD scalar bundle and reduction record that cross the host/device seam.
//
// Layout-compatible with the reference's include/lpbf_step_const.hpp:19-33
// (StepConst: 216 bytes, `radiation` at offset 176; Partial: 24 bytes), so a
// caller built against the reference passes the same bytes to this library.
// make_const follows lpbf_step_const.hpp:36-54.
//
// Plain C++17, no CUDA tokens: included by g++ host code and nvcc alike.
// ---------------------------------------------------------------------------
#pragma once
#include <cmath>
#include "params.hpp"

struct StepConst {
    int    nx, ny;
    double dx, dy, inv_dx2, inv_dy2, inv_r0_sq;
    double alpha, K, rho, cp, rho_cp, inv_h, h, dt;
    double peak_S, eta, P;
    double hConv, Tamb, Tsub, dSub, eps;
    bool   radiation;
    double kmult;
    double x_l, y_l;   // laser centre for the step being launched [m]
    double q_scale;    // source multiplier (0 = beam off)
};

// Peak temperature with its flat index (ties -> smallest index) and the
// extent of molten rows (ymax < 0 means nothing is molten).
struct Partial { double tmax; long long arg; int ymin; int ymax; };

static_assert(sizeof(StepConst) == 216, "StepConst ABI");
static_assert(sizeof(Partial) == 24, "Partial ABI");

inline StepConst make_const(lpbf::Material const& mat, lpbf::Process const& pr,
                            lpbf::Domain const& dom, double dt) {
    StepConst k{};
    k.nx = dom.nx;
    k.ny = dom.ny;
    k.dx = dom.dx();
    k.dy = dom.dy();
    k.inv_dx2   = 1.0 / (k.dx * k.dx);
    k.inv_dy2   = 1.0 / (k.dy * k.dy);
    k.inv_r0_sq = 1.0 / (pr.r0 * pr.r0);
    k.alpha  = mat.alpha();
    k.K      = mat.k;
    k.rho    = mat.rho;
    k.cp     = mat.cp;
    k.rho_cp = mat.rho * mat.cp;
    k.inv_h  = 1.0 / pr.h;
    k.h      = pr.h;
    k.dt     = dt;
    k.peak_S = (2.0 * mat.eta * pr.P) / (M_PI * pr.r0 * pr.r0);
    k.eta    = mat.eta;
    k.P      = pr.P;
    k.hConv  = pr.hConv;
    k.Tamb   = pr.Tamb;
    k.Tsub   = pr.Tsub;
    k.dSub   = pr.dSub;
    k.eps    = mat.eps;
    k.radiation = pr.radiation;
    k.kmult   = 1.0;
    k.q_scale = 1.0;
    k.x_l = 0.0;
    k.y_l = 0.0;
    return k;
}
