// SPDX-License-Identifier: 0BSD
// ===========================================================================
// ORACLE -- test infrastructure only.  Builds into oracle/_ref/libref.so.
//
// Compiles the reference's own standalone GPU driver translation unit
// (src/gpu/lpbf_cuda.cu, included from the read-only reference tree with its
// `main` renamed) so that its host-side CPU stepper `cpu_step`
// (lpbf_cuda.cu:154-210), `measure_host` (:225-253) and `run_cpu` (:423-448)
// can be called directly, with no code of ours in their arithmetic.  The
// reference's kernels.cu is linked in only because lpbf_cuda.cu references
// its launch wrappers; the CPU entry points below never launch anything.
// ===========================================================================
#define main lpbf_reference_cuda_main
#include "src/gpu/lpbf_cuda.cu"
#undef main

extern "C" {

// One reference cpu_step over the full grid (copies through std::vector).
void ref_cpu_step(const double* Tin, double* Tout, const StepConst* k, int phys) {
    const std::size_t N = (std::size_t)k->nx * k->ny;
    std::vector<double> a(Tin, Tin + N), b(N);
    cpu_step(a, b, *k, phys ? Physics::Extended : Physics::Baseline);
    std::copy(b.begin(), b.end(), Tout);
}

// n reference cpu_steps along an explicit laser plan (x_l, y_l, q_scale per
// step).  T holds the initial field and receives the final one.
void ref_cpu_run_plan(double* T, const StepConst* k0, const double* plan_xyq,
                      int n_steps, int phys) {
    const std::size_t N = (std::size_t)k0->nx * k0->ny;
    std::vector<double> a(T, T + N), b(N);
    StepConst k = *k0;
    const Physics ph = phys ? Physics::Extended : Physics::Baseline;
    for (int s = 0; s < n_steps; ++s) {
        k.x_l = plan_xyq[3 * s + 0];
        k.y_l = plan_xyq[3 * s + 1];
        k.q_scale = plan_xyq[3 * s + 2];
        cpu_step(a, b, k, ph);
        a.swap(b);
    }
    std::copy(a.begin(), a.end(), T);
}

// The reference measure_host() on one field.
void ref_measure_host(const double* T, int nx, int ny, double Lx, double Ly,
                      double Tm, double* peak_T, double* W_um, double* W_sub_um,
                      int* x_hot) {
    Domain dom;
    dom.nx = nx; dom.ny = ny; dom.Lx = Lx; dom.Ly = Ly;
    std::vector<double> v(T, T + (std::size_t)nx * ny);
    const StepMetrics m = measure_host(v, dom, Tm);
    *peak_T = m.peak_T; *W_um = m.W_um; *W_sub_um = m.W_sub_um; *x_hot = m.x_hot;
}

// The reference run_cpu(): the full CPU solver with its built-in single-track
// laser law and per-step measure_host.  Material/Process/Domain are given
// field by field.  Returns wall ms; T receives the final field.
double ref_run_cpu(double* T, int nx, int ny, double Lx, double Ly,
                   const double* mat6 /*k,rho,cp,Tm,eps,eta*/,
                   const double* pr8 /*P,V,r0,h,hConv,dSub,Tamb,Tsub*/,
                   int radiation, double dt, int n_steps, int phys, double kmult,
                   double* peak_T, double* peak_W, double* steady_W_sub) {
    Material mat;
    mat.k = mat6[0]; mat.rho = mat6[1]; mat.cp = mat6[2];
    mat.Tm = mat6[3]; mat.eps = mat6[4]; mat.eta = mat6[5];
    Process pr;
    pr.P = pr8[0]; pr.V = pr8[1]; pr.r0 = pr8[2]; pr.h = pr8[3];
    pr.hConv = pr8[4]; pr.dSub = pr8[5]; pr.Tamb = pr8[6]; pr.Tsub = pr8[7];
    pr.radiation = radiation != 0;
    Domain dom;
    dom.nx = nx; dom.ny = ny; dom.Lx = Lx; dom.Ly = Ly;
    RunResult rr = run_cpu(mat, pr, dom, dt, n_steps,
                           phys ? Physics::Extended : Physics::Baseline, kmult);
    std::copy(rr.Tfinal.begin(), rr.Tfinal.end(), T);
    *peak_T = rr.peak_T; *peak_W = rr.peak_W; *steady_W_sub = rr.steady_W_sub;
    return rr.wall_ms;
}

}  // extern "C"

extern "C" {
// The reference make_const (include/lpbf_step_const.hpp:36-54), field by field.
void ref_make_const(int nx, int ny, double Lx, double Ly, const double* mat6,
                    const double* pr8, int radiation, double dt, StepConst* out) {
    Material mat;
    mat.k = mat6[0]; mat.rho = mat6[1]; mat.cp = mat6[2];
    mat.Tm = mat6[3]; mat.eps = mat6[4]; mat.eta = mat6[5];
    Process pr;
    pr.P = pr8[0]; pr.V = pr8[1]; pr.r0 = pr8[2]; pr.h = pr8[3];
    pr.hConv = pr8[4]; pr.dSub = pr8[5]; pr.Tamb = pr8[6]; pr.Tsub = pr8[7];
    pr.radiation = radiation != 0;
    Domain dom;
    dom.nx = nx; dom.ny = ny; dom.Lx = Lx; dom.Ly = Ly;
    *out = make_const(mat, pr, dom, dt);
}
// The reference dt_cfl / dt_cfl_ext (include/params.hpp:44-47,128-132).
double ref_dt_cfl(int nx, int ny, double Lx, double Ly, double k, double rho,
                  double cp, int ext, double kmult) {
    Material mat; mat.k = k; mat.rho = rho; mat.cp = cp;
    Domain dom; dom.nx = nx; dom.ny = ny; dom.Lx = Lx; dom.Ly = Ly;
    return ext ? dt_cfl_ext(mat, dom, kmult) : dt_cfl(mat, dom);
}
}  // extern "C"
