// SPDX-License-Identifier: 0BSD
// Drop-in test driver: the reference's case-0 single-track run (240 x 120,
// IN718 defaults, CFL time step, 1.5 ms) through the GpuStepTask /
// MetricsTask / SnapshotWriterTask graph of include/gpu_step_task.hpp on
// liblpbf_b200.  Usage:
//   gpu_task_demo OUTDIR MODE FUSED PINNED BATCH [DEPTH]
// Writes OUTDIR/metrics.csv, OUTDIR/T_step_*.bin (every 200 steps and the
// last) and OUTDIR/summary.txt (peak_T peak_W steady_W_sub n_steps).
#include <hedgehog.h>

#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <memory>
#include <string>
#include <vector>

#include "gpu_step_task.hpp"

using namespace lpbf;

// The reference's single-track law: start at 0.2 Lx on the centre line, the
// kernel uses the position before the advance, wrap back past 0.9 Lx.
static std::vector<Tick> single_track(const Process& pr, const Domain& dom, double dt,
                                      int n, int snap_every) {
    std::vector<Tick> plan(n);
    const double x0 = 0.20 * dom.Lx, y = 0.50 * dom.Ly;
    double x = x0;
    bool wrapped = false;
    for (int s = 0; s < n; ++s) {
        Tick& t = plan[s];
        t.step = s;
        t.t = s * dt;
        t.x_l = x;
        t.y_l = y;
        t.q_scale = 1.0;
        x += pr.V * dt;
        if (x > 0.90 * dom.Lx) { x = x0; wrapped = true; }
        t.x_laser_csv = x;
        t.wrapped = wrapped;
        t.dump = (snap_every > 0 && s % snap_every == 0) || s == n - 1;
    }
    return plan;
}

int main(int argc, char** argv) {
    if (argc < 6) {
        std::fprintf(stderr, "usage: %s OUTDIR MODE FUSED PINNED BATCH [DEPTH]\n", argv[0]);
        return 2;
    }
    const std::string out = argv[1];
    const int mode = std::atoi(argv[2]), fused = std::atoi(argv[3]), pinned = std::atoi(argv[4]);
    const int batch = std::atoi(argv[5]);
    const int depth = argc > 6 ? std::atoi(argv[6]) : 0;
    std::filesystem::create_directories(out);

    Material mat;
    Process pr;
    Domain dom;
    const double dt = dt_cfl(mat, dom);
    const int n = static_cast<int>(1.5e-3 / dt);
    const std::vector<Tick> plan = single_track(pr, dom, dt, n, 200);
    StepConst k = make_const(mat, pr, dom, dt);

    auto acc = std::make_shared<RunAccum>();
    {
        hh::Graph<1, Tick, StepResult> graph("drop-in");
        auto gpu = std::make_shared<GpuStepTask>(dom, k, 0, mat.Tm, n, plan, pr.Tamb, true, batch,
                                                 mode, fused != 0, pinned != 0);
        gpu->depth(depth);
        auto metrics = std::make_shared<MetricsTask>(dom, mat.Tm, acc, true, out);
        auto snap = std::make_shared<SnapshotWriterTask>(2, out);
        graph.inputs(gpu);
        graph.edges(gpu, gpu);
        graph.edges(gpu, metrics);
        graph.edges(gpu, snap);
        graph.outputs(metrics);
        graph.outputs(snap);
        graph.executeGraph();
        graph.pushData(std::make_shared<Tick>(plan[0]));
        graph.finishPushingData();
        while (auto r = graph.getBlockingResult()) { (void)r; }
        graph.waitForTermination();
    }
    FILE* f = std::fopen((out + "/summary.txt").c_str(), "w");
    std::fprintf(f, "%.17g %.17g %.17g %d\n", acc->peak_T, acc->peak_W, acc->steady_W_sub, n);
    std::fclose(f);
    return 0;
}
