// SPDX-License-Identifier: 0BSD
// ===========================================================================
// ORACLE -- test infrastructure only.  Builds into oracle/_ref/libref_plan.so.
//
// Compiles the reference's Hedgehog+CUDA driver translation unit
// (src/gpu/hh_gpu_main.cpp, from the read-only reference tree, `main`
// renamed) against the hh-compat header so that its laser planner
// build_plan (hh_gpu_main.cpp:141-157) can be called directly.  Nothing here
// launches a kernel.
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
