// SPDX-License-Identifier: 0BSD
// ===========================================================================
// ORACLE -- test/baseline infrastructure only.  Builds into
// oracle/_ref/libref_hh.so.
//
// Drives the reference's own CPU step task, lpbf::StepTileTask
// (include/step_task.hpp:37-223, included unmodified from the read-only
// reference tree), through the hh-compat task graph with n worker threads
// over row-strip tiles -- the reference's Hedgehog CPU path.  The per-step
// driver work follows src/main.cpp:316-402: build tiles with halo rows
// (main.cpp:115-155), push, collect, stitch, advance the laser, then the
// single-threaded global measure() (main.cpp:164-211).  Unlike main.cpp the
// grid, time step and laser plan are parameters (main.cpp hard-wires a
// 240x120 domain, the CFL time step and a single +x track).
// ===========================================================================
#include <hedgehog.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <memory>
#include <vector>

#include "params.hpp"
#include "tile.hpp"
#include "step_task.hpp"

using namespace lpbf;

namespace {

std::shared_ptr<HaloTile> build_tile(int idx, int y0, int y1, int nx, int ny,
                                     const std::vector<double>& T, int step,
                                     double t, double xl, double yl, double q) {
    auto tile = std::make_shared<HaloTile>();
    tile->idx = idx; tile->y0 = y0; tile->y1 = y1; tile->nx = nx;
    tile->step = step; tile->t = t;
    tile->x_laser = xl; tile->y_laser = yl; tile->q_scale = q;
    const int rows = tile->total_rows();
    tile->data.resize(static_cast<std::size_t>(rows) * nx);
    const int top = (y0 == 0) ? y0 : y0 - 1;          // mirror at the domain edge
    const int bot = (y1 == ny - 1) ? y1 : y1 + 1;
    std::copy_n(&T[(std::size_t)top * nx], nx, &tile->at(0, 0));
    std::copy_n(&T[(std::size_t)y0 * nx], (std::size_t)(y1 - y0 + 1) * nx, &tile->at(1, 0));
    std::copy_n(&T[(std::size_t)bot * nx], nx, &tile->at(rows - 1, 0));
    return tile;
}

double global_peak(const std::vector<double>& T, int nx, int ny, double Tm,
                   int* ymin_out, int* ymax_out) {
    double Tmax = 0.0;
    int ymin = ny, ymax = -1;
    for (int y = 0; y < ny; ++y) {
        const double* row = &T[(std::size_t)y * nx];
        bool any = false;
        for (int x = 0; x < nx; ++x) {
            const double v = row[x];
            if (v > Tmax) Tmax = v;
            if (v > Tm) any = true;
        }
        if (any) { ymin = std::min(ymin, y); ymax = std::max(ymax, y); }
    }
    *ymin_out = ymin; *ymax_out = ymax;
    return Tmax;
}

}  // namespace

extern "C" {

// Advance T (nx*ny, row-major, in/out) by n_steps along plan_xyq (x_l, y_l,
// q_scale per step) with `n_threads` StepTileTask workers over `n_tiles` row
// strips.  peak_trace (nullable) receives measure()'s peak T after each step.
// Returns the wall time of the stepping loop in seconds.
double ref_hh_run(double* T_io, int nx, int ny, double Lx, double Ly,
                  const double* mat6, const double* pr8, int radiation,
                  double dt, const double* plan_xyq, int n_steps,
                  int n_threads, int n_tiles, int phys, double kmult,
                  double Tm, double* peak_trace) {
    Material mat;
    mat.k = mat6[0]; mat.rho = mat6[1]; mat.cp = mat6[2];
    mat.Tm = mat6[3]; mat.eps = mat6[4]; mat.eta = mat6[5];
    Process pr;
    pr.P = pr8[0]; pr.V = pr8[1]; pr.r0 = pr8[2]; pr.h = pr8[3];
    pr.hConv = pr8[4]; pr.dSub = pr8[5]; pr.Tamb = pr8[6]; pr.Tsub = pr8[7];
    pr.radiation = radiation != 0;
    Domain dom;
    dom.nx = nx; dom.ny = ny; dom.Lx = Lx; dom.Ly = Ly;
    if (n_tiles > ny) n_tiles = ny;
    if (n_tiles < 1) n_tiles = 1;

    std::vector<double> T(T_io, T_io + (std::size_t)nx * ny);
    std::vector<int> y0(n_tiles), y1(n_tiles);
    for (int i = 0; i < n_tiles; ++i) {
        y0[i] = (i * ny) / n_tiles;
        y1[i] = ((i + 1) * ny) / n_tiles - 1;
    }

    auto prof = std::make_shared<StepProfile>();
    double wall = 0.0;
    {
        hh::Graph<1, HaloTile, HaloTile> graph("LPBF-2D");
        auto task = std::make_shared<StepTileTask>(
            "Step", (std::size_t)std::max(1, n_threads), mat, pr, dom, dt, prof,
            phys ? Physics::Extended : Physics::Baseline, kmult);
        graph.inputs(task);
        graph.outputs(task);
        graph.executeGraph();

        const auto t0 = std::chrono::steady_clock::now();
        for (int s = 0; s < n_steps; ++s) {
            const double xl = plan_xyq[3 * s], yl = plan_xyq[3 * s + 1], q = plan_xyq[3 * s + 2];
            for (int i = 0; i < n_tiles; ++i)
                graph.pushData(build_tile(i, y0[i], y1[i], nx, ny, T, s, s * dt, xl, yl, q));
            for (int got = 0; got < n_tiles; ++got) {
                auto r = graph.getBlockingResult();
                if (!r) break;
                auto tile = std::get<std::shared_ptr<HaloTile>>(*r);
                std::copy_n(&tile->at(1, 0), (std::size_t)tile->owned_rows() * nx,
                            &T[(std::size_t)tile->y0 * nx]);
            }
            int ymin, ymax;
            const double pk = global_peak(T, nx, ny, Tm, &ymin, &ymax);
            if (peak_trace) peak_trace[s] = pk;
        }
        wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        graph.finishPushingData();
        graph.waitForTermination();
    }
    std::copy(T.begin(), T.end(), T_io);
    return wall;
}

}  // extern "C"
