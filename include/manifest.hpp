// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Manifest ensembles on the batched process-map kernel.
//
// Replaces the reference's --manifest mode (src/gpu/hh_gpu_main.cpp:162-270),
// which builds and runs one GpuStepTask graph per CSV row, one after another:
// here every baseline-physics row with the same step count advances in one
// batch (lpbf_b200_batch_*), one step per launch with the sub-grid melt width
// computed on the device after each step (lpbf_b200_batch_run_wsub);
// extended-physics rows run one by one through lpbf_b200_advance.  Rows,
// columns, per-row constants, plans and the RESULT line are the reference's:
//   * columns matched by header name: run_id, cond_id, draw_id, config, P_W,
//     V_mps, r0_m, eta, dsub_m, kmult, physics (hh_gpu_main.cpp:244-251);
//   * per row: default Material/Process/Domain with P, V, r0, eta, dSub
//     overridden, dt = dt_cfl (or dt_cfl_ext with kmult), n_steps =
//     int(t_end / dt), the single-track plan, make_const with kmult
//     (hh_gpu_main.cpp:171-183);
//   * steady W_sub = largest sub-grid melt width over cruise steps, peak T =
//     largest per-step peak (the RunAccum of MetricsTask,
//     include/gpu_step_task.hpp:380-405);
//   * RESULT line format of emit_result_line (hh_gpu_main.cpp:209-216).
// wall_ms of a batched row is its batch's wall time divided by its rows.
// ---------------------------------------------------------------------------
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "gpu_messages.hpp"
#include "lpbf_b200.h"
#include "lpbf_kernels.hpp"
#include "lpbf_step_const.hpp"
#include "params.hpp"

namespace lpbf {
namespace manifest {

struct RunSpec {
    std::string run_id, cond_id, draw_id, config, physics;
    double P = 0, V = 0, r0 = 0, eta = 0, dsub_m = 0, kmult = 1.0;
};
struct RowResult { double steady_W = 0, peak_T = 0, wall_ms = 0; long n_steps = 0; };

// Commas only, no quoting; '\r' dropped (the reference's split).
inline std::vector<std::string> split_csv(const std::string& line) {
    std::vector<std::string> out;
    std::string cur;
    for (char ch : line) {
        if (ch == ',') { out.push_back(cur); cur.clear(); }
        else if (ch != '\r') cur.push_back(ch);
    }
    out.push_back(cur);
    return out;
}

// Rows of a manifest file; false with *err set on a missing file, an empty
// file or a missing column (the reference exits with status 4 on those).
inline bool read_manifest(const std::string& path, std::vector<RunSpec>* rows, std::string* err) {
    std::ifstream f(path);
    if (!f) { *err = "cannot open manifest '" + path + "'"; return false; }
    std::string header;
    if (!std::getline(f, header)) { *err = "empty manifest"; return false; }
    const std::vector<std::string> cols = split_csv(header);
    static const char* names[] = {"run_id", "cond_id", "draw_id", "config", "P_W", "V_mps",
                                  "r0_m", "eta", "dsub_m", "kmult", "physics"};
    int idx[11];
    for (int c = 0; c < 11; ++c) {
        idx[c] = -1;
        for (size_t i = 0; i < cols.size(); ++i)
            if (cols[i] == names[c]) { idx[c] = (int)i; break; }
        if (idx[c] < 0) { *err = std::string("manifest missing column '") + names[c] + "'"; return false; }
    }
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty()) continue;
        const std::vector<std::string> v = split_csv(line);
        auto at = [&](int c) -> std::string { return idx[c] < (int)v.size() ? v[idx[c]] : std::string(); };
        RunSpec r;
        r.run_id = at(0); r.cond_id = at(1); r.draw_id = at(2); r.config = at(3);
        r.P = std::atof(at(4).c_str()); r.V = std::atof(at(5).c_str());
        r.r0 = std::atof(at(6).c_str()); r.eta = std::atof(at(7).c_str());
        r.dsub_m = std::atof(at(8).c_str()); r.kmult = std::atof(at(9).c_str());
        r.physics = at(10);
        rows->push_back(r);
    }
    return true;
}

// The single-track laser law (hh_gpu_main.cpp:141-157): start at 0.2 Lx on
// the centre line, advance V dt per step, wrap back once past 0.9 Lx; the
// step uses the pre-advance position, x_laser_csv/wrapped the post-advance.
inline std::vector<Tick> single_track_plan(const Process& pr, const Domain& dom, double dt,
                                           int n_steps) {
    std::vector<Tick> plan(std::max(n_steps, 0));
    double x = 0.20 * dom.Lx;
    const double y = 0.50 * dom.Ly, x0 = x;
    bool wrapped = false;
    for (int s = 0; s < n_steps; ++s) {
        Tick& t = plan[s];
        t.step = s; t.t = s * dt;
        t.x_l = x; t.y_l = y; t.q_scale = 1.0;
        x += pr.V * dt;
        if (x > 0.90 * dom.Lx) { x = x0; wrapped = true; }
        t.x_laser_csv = x; t.wrapped = wrapped;
        t.dump = (s == n_steps - 1);
    }
    return plan;
}

inline bool cruise(const Tick& t, double Lx) {
    return !t.wrapped && t.x_laser_csv >= 0.45 * Lx && t.x_laser_csv <= 0.85 * Lx;
}

inline double sub_grid_width_um(const double* col, int n, double dy, double Tm) {
    int a = -1, b = -1;
    for (int y = 0; y < n; ++y)
        if (col[y] > Tm) { if (a < 0) a = y; b = y; }
    if (a < 0) return 0.0;
    double lo = a * dy, hi = b * dy;
    if (a > 0) lo = ((a - 1) + (Tm - col[a - 1]) / (col[a] - col[a - 1])) * dy;
    if (b < n - 1) hi = (b + (Tm - col[b]) / (col[b + 1] - col[b])) * dy;
    return (hi - lo) * 1e6;
}

struct Prepared {
    Material mat; Process pr; Domain dom;
    StepConst k{};
    int n_steps = 0, phys = 0;
    std::vector<Tick> plan;
};

inline Prepared prepare(const RunSpec& rs, double t_end) {
    Prepared p;
    p.pr.P = rs.P; p.pr.V = rs.V; p.pr.r0 = rs.r0;
    p.mat.eta = rs.eta; p.pr.dSub = rs.dsub_m;
    p.phys = rs.physics == "ext" ? 1 : 0;
    const double dt = p.phys ? dt_cfl_ext(p.mat, p.dom, rs.kmult) : dt_cfl(p.mat, p.dom);
    p.n_steps = static_cast<int>(t_end / dt);
    p.plan = single_track_plan(p.pr, p.dom, dt, p.n_steps);
    p.k = make_const(p.mat, p.pr, p.dom, dt);
    p.k.kmult = rs.kmult;
    return p;
}

namespace detail {
inline bool ok(cudaError_t e) { return e == cudaSuccess; }

// Baseline rows sharing a step count, as one batch.
inline bool run_batch(std::vector<Prepared>& ps, const std::vector<int>& ids,
                      std::vector<RowResult>& out, cudaStream_t s) {
    const int n = (int)ids.size();
    const int steps = ps[ids[0]].n_steps;
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<double*> A(n), B(n);
    std::vector<Partial*> ring(n);
    std::vector<lpbf_b200_scenario> sc(n);
    std::vector<unsigned char> cr((size_t)steps * n);
    bool good = true;
    for (int i = 0; i < n && good; ++i) {
        Prepared& p = ps[ids[i]];
        const size_t N = (size_t)p.k.nx * p.k.ny;
        good = ok(cudaMalloc(&A[i], N * 8)) && ok(cudaMalloc(&B[i], N * 8)) &&
               ok(cudaMalloc(&ring[i], sizeof(Partial) * std::max(steps, 1)));
        if (!good) break;
        std::vector<double> T0(N, p.pr.Tamb);
        good = ok(cudaMemcpyAsync(A[i], T0.data(), N * 8, cudaMemcpyHostToDevice, s)) &&
               ok(cudaStreamSynchronize(s));
        sc[i] = lpbf_b200_scenario{&p.k, p.plan.data(), A[i], B[i], ring[i], 0, p.pr.Tamb,
                                   p.mat.Tm};
        for (int t = 0; t < steps; ++t) cr[(size_t)t * n + i] = cruise(p.plan[t], p.dom.Lx) ? 1 : 0;
    }
    unsigned char* d_cr = nullptr;
    double* d_w = nullptr;
    void* work = nullptr;
    lpbf_b200_batch* b = nullptr;
    std::vector<double> w((size_t)steps * n);
    if (good) {
        lpbf_b200_batch_opts o{};
        const size_t wb = lpbf_b200_batch_workspace_bytes(sc.data(), n, steps, &o);
        good = wb > 0 && ok(cudaMalloc(&work, wb)) && ok(cudaMalloc(&d_cr, cr.size())) &&
               ok(cudaMalloc(&d_w, w.size() * 8)) &&
               ok(cudaMemcpyAsync(d_cr, cr.data(), cr.size(), cudaMemcpyHostToDevice, s)) &&
               lpbf_b200_batch_create(sc.data(), n, steps, &o, work, wb, s, &b) == LPBF_OK &&
               lpbf_b200_batch_run_wsub(b, 0, steps, d_cr, d_w, s) == LPBF_OK &&
               ok(cudaMemcpyAsync(w.data(), d_w, w.size() * 8, cudaMemcpyDeviceToHost, s)) &&
               ok(cudaStreamSynchronize(s));
    }
    const double ms = std::chrono::duration<double, std::milli>(
        std::chrono::steady_clock::now() - t0).count();
    for (int i = 0; i < n && good; ++i) {
        std::vector<Partial> r(steps);
        good = ok(cudaMemcpy(r.data(), ring[i], sizeof(Partial) * steps, cudaMemcpyDeviceToHost));
        RowResult& o = out[ids[i]];
        o.n_steps = steps;
        o.wall_ms = ms / n;
        for (int t = 0; t < steps; ++t) {
            o.peak_T = std::max(o.peak_T, r[t].tmax);
            if (cr[(size_t)t * n + i]) o.steady_W = std::max(o.steady_W, w[(size_t)t * n + i]);
        }
    }
    if (b) lpbf_b200_batch_destroy(b);
    cudaFree(work); cudaFree(d_cr); cudaFree(d_w);
    for (int i = 0; i < n; ++i) { cudaFree(A[i]); cudaFree(B[i]); cudaFree(ring[i]); }
    return good;
}

// One extended-physics row: a step per call, the hot column on cruise steps.
inline bool run_ext(Prepared& p, RowResult& o, cudaStream_t s) {
    const auto t0 = std::chrono::steady_clock::now();
    const int nx = p.k.nx, ny = p.k.ny;
    const size_t N = (size_t)nx * ny;
    double *A = nullptr, *B = nullptr, *col = nullptr;
    Partial* ring = nullptr;
    void* work = nullptr;
    const size_t wb = lpbf_b200_workspace_bytes();
    bool good = ok(cudaMalloc(&A, N * 8)) && ok(cudaMalloc(&B, N * 8)) &&
                ok(cudaMalloc(&col, ny * 8)) && ok(cudaMalloc(&ring, sizeof(Partial))) &&
                ok(cudaMalloc(&work, wb)) && lpbf_b200_workspace_init(work, wb, s) == LPBF_OK;
    if (good) {
        std::vector<double> T0(N, p.pr.Tamb);
        good = ok(cudaMemcpy(A, T0.data(), N * 8, cudaMemcpyHostToDevice));
    }
    lpbf_b200_opts opt{1, 0, p.pr.Tamb, p.mat.Tm, 1, 0};
    std::vector<double> h(ny);
    for (int t = 0; t < p.n_steps && good; ++t) {
        int in_b = 0;
        good = lpbf_b200_advance(A, B, &p.k, &p.plan[t], 1, &opt, ring, work, wb, s, &in_b) ==
               LPBF_OK;
        if (in_b) std::swap(A, B);
        Partial r{};
        good = good && ok(cudaMemcpyAsync(&r, ring, sizeof(Partial), cudaMemcpyDeviceToHost, s)) &&
               ok(cudaStreamSynchronize(s));
        if (!good) break;
        o.peak_T = std::max(o.peak_T, r.tmax);
        if (r.tmax > p.mat.Tm && cruise(p.plan[t], p.dom.Lx)) {
            lpbf_launch_extract_col(A, nx, ny, ring, col, s);
            good = ok(cudaMemcpyAsync(h.data(), col, ny * 8, cudaMemcpyDeviceToHost, s)) &&
                   ok(cudaStreamSynchronize(s));
            o.steady_W = std::max(o.steady_W, sub_grid_width_um(h.data(), ny, p.dom.dy(), p.mat.Tm));
        }
    }
    o.n_steps = p.n_steps;
    o.wall_ms = std::chrono::duration<double, std::milli>(
        std::chrono::steady_clock::now() - t0).count();
    cudaFree(A); cudaFree(B); cudaFree(col); cudaFree(ring); cudaFree(work);
    return good;
}
}  // namespace detail

// Results in row order; false if a CUDA call or launch failed.
inline bool run_rows(const std::vector<RunSpec>& rows, double t_end, std::vector<RowResult>* out,
                     cudaStream_t s = nullptr) {
    std::vector<Prepared> ps;
    ps.reserve(rows.size());
    for (const RunSpec& r : rows) ps.push_back(prepare(r, t_end));
    out->assign(rows.size(), RowResult{});
    std::map<int, std::vector<int>> groups;            // baseline rows by step count
    bool good = true;
    for (size_t i = 0; i < ps.size(); ++i) {
        if (ps[i].phys == 0 && ps[i].n_steps > 0) groups[ps[i].n_steps].push_back((int)i);
        else if (ps[i].phys == 1) good = detail::run_ext(ps[i], (*out)[i], s) && good;
    }
    for (auto& g : groups) good = detail::run_batch(ps, g.second, *out, s) && good;
    return good;
}

inline void print_header(FILE* f) {
    std::fprintf(f, "# RESULT,run_id,cond_id,draw_id,config,physics,P_W,V_mps,r0_m,eta,"
                    "dsub_m,kmult,steady_W_sub_um,peak_T_K,wall_ms,n_steps\n");
}
inline void print_result(FILE* f, const RunSpec& rs, const RowResult& r) {
    std::fprintf(f, "RESULT,%s,%s,%s,%s,%s,%.6g,%.6g,%.6g,%.6g,%.6g,%.6g,%.6g,%.6g,%.3f,%ld\n",
                 rs.run_id.c_str(), rs.cond_id.c_str(), rs.draw_id.c_str(), rs.config.c_str(),
                 rs.physics.c_str(), rs.P, rs.V, rs.r0, rs.eta, rs.dsub_m, rs.kmult, r.steady_W,
                 r.peak_T, r.wall_ms, r.n_steps);
}

}  // namespace manifest
}  // namespace lpbf
