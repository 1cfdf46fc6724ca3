// SPDX-License-Identifier: 0BSD
// ===========================================================================
// ORACLE -- test infrastructure only.  Builds into oracle/_ref/libref_plan.so.
//
// Compiles the reference's Hedgehog+CUDA driver translation unit
// (src/gpu/hh_gpu_main.cpp, from the read-only reference tree, `main`
// renamed) against the hh-compat header so that its laser planner
// build_plan (hh_gpu_main.cpp:141-157) can be called directly, and so that
// the reference's own GPU task graph can be timed as the GPU baseline
// (ref_gpu_task_run below; its kernels are the reference's kernels.cu built
// for sm_100a, linked in by oracle/Makefile).
// ===========================================================================
#define main lpbf_reference_hhcuda_main
#include "src/gpu/hh_gpu_main.cpp"
#undef main

extern "C" int ref_build_plan(double P, double V, double r0, double Lx, double Ly,
                              int nx, int ny, double dt, int n_steps, int snap_every,
                              lpbf::Tick* out) {
    lpbf::Process pr; pr.P = P; pr.V = V; pr.r0 = r0;
    lpbf::Domain dom; dom.Lx = Lx; dom.Ly = Ly; dom.nx = nx; dom.ny = ny;
    std::vector<lpbf::Tick> plan = build_plan(pr, dom, dt, n_steps, snap_every);
    std::copy(plan.begin(), plan.end(), out);
    return (int)plan.size();
}

// The reference's own GPU step task graph of one run (run_one_row,
// hh_gpu_main.cpp:171-207: GpuStepTask -> MetricsTask/SnapshotWriterTask,
// the task recirculating its Tick), on a caller-given grid, constants and
// per-step plan, with no disk output; its GpuStepTask and kernels are the
// reference's own (include/gpu_step_task.hpp, src/gpu/kernels.cu built for
// sm_100a).  Returns the wall milliseconds from the first pushed Tick to the
// graph's end (the task's device set-up included, as in run_one_row); peak_T
// receives the run's accumulated peak temperature.
extern "C" double ref_gpu_task_run(int nx, int ny, double Lx, double Ly, const StepConst* k,
                                   double Tm, double Tamb, const lpbf::Tick* ticks,
                                   int n_steps, int batch, int mode, int fused, int pinned,
                                   double* peak_T) {
    lpbf::Domain dom; dom.Lx = Lx; dom.Ly = Ly; dom.nx = nx; dom.ny = ny;
    std::vector<lpbf::Tick> plan(ticks, ticks + n_steps);
    auto acc = std::make_shared<RunAccum>();
    hh::Graph<1, Tick, StepResult> graph("LPBF-2D-HHCUDA");
    auto gpu = std::make_shared<GpuStepTask>(dom, *k, 0, Tm, n_steps, plan, Tamb,
                                             /*write_outputs=*/false, batch, mode,
                                             fused != 0, pinned != 0);
    auto metrics = std::make_shared<MetricsTask>(dom, Tm, acc, false, std::string());
    auto snap = std::make_shared<SnapshotWriterTask>(1, std::string());
    graph.inputs(gpu);
    graph.edges(gpu, gpu);
    graph.edges(gpu, metrics);
    graph.edges(gpu, snap);
    graph.outputs(metrics);
    graph.outputs(snap);
    graph.executeGraph();
    const auto wall0 = std::chrono::steady_clock::now();
    graph.pushData(std::make_shared<Tick>(plan[0]));
    graph.finishPushingData();
    while (auto res = graph.getBlockingResult()) { (void)res; }
    graph.waitForTermination();
    const double wall_ms = std::chrono::duration<double, std::milli>(
        std::chrono::steady_clock::now() - wall0).count();
    *peak_T = acc->peak_T;
    return wall_ms;
}
