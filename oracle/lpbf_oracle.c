/* SPDX-License-Identifier: 0BSD
 * ===========================================================================
 * ORACLE -- test infrastructure only.  Nothing in the product links this file;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it
 * (through oracle/oracle.py), and only as the checker.
 *
 * A plain-C, single-threaded restatement of the reference's CPU arithmetic for
 * the 2D z-averaged explicit heat step of hedgehog_lpbf.  Every expression
 * keeps the reference's evaluation order; the file is compiled with
 * -ffp-contract=off so no multiply-add is fused, which makes the results
 * bit-identical to the reference's own cpu_step built with g++ on x86-64
 * (checked by tests/test_oracle.py against oracle/_ref and the golden case0).
 *
 *   oracle_step      src/gpu/lpbf_cuda.cu:154-210 (cpu_step), baseline branch
 *                    = include/step_task.hpp:87-131, extended branch
 *                    = include/step_task.hpp:132-187.  bc=1 adds fixed-value
 *                    (Dirichlet) edges, which the reference cannot express.
 *   oracle_reduce    src/gpu/kernels.cu:205-262 (reduce + finalize semantics:
 *                    tmax init -1, arg init N, ties -> smallest flat index).
 *   oracle_measure   src/main.cpp:164-211 (measure(): Tmax init 0, W, W_sub).
 *   oracle_run       src/gpu/lpbf_cuda.cu:423-448 (run_cpu loop) driven by an
 *                    explicit per-step laser plan instead of the built-in law.
 * ===========================================================================
 */
#include <math.h>
#include <stdbool.h>
#include <stddef.h>
#include <string.h>

#include "lpbf_oracle.h"

static const double SIGMA_SB = 5.670374419e-8;  /* params.hpp:11 */

/* ---- IN718 Mills tables and property model (params.hpp:61-111) -------- */
#define N_PTS 9
static const double T_SOL = 1533.0, T_LIQ = 1609.0, LF = 210.0e3;
static const double T_PTS[N_PTS]  = {298, 473, 673, 873, 1073, 1273, 1473, 1533, 1609};
static const double K_PTS[N_PTS]  = {8.9, 12.9, 15.8, 18.7, 21.9, 25.6, 28.6, 29.3, 29.6};
static const double CP_PTS[N_PTS] = {435, 479, 515, 558, 580, 628, 670, 685, 720};

static double interp(double T, const double* xs, const double* ys, int n) {
    if (T <= xs[0]) return ys[0];
    if (T >= xs[n - 1]) return ys[n - 1];
    int i = 1;
    while (T > xs[i]) ++i;
    const double f = (T - xs[i - 1]) / (xs[i] - xs[i - 1]);
    return ys[i - 1] + f * (ys[i] - ys[i - 1]);
}
double oracle_k_of(double T)  { return interp(T, T_PTS, K_PTS, N_PTS); }
double oracle_cp_of(double T) { return interp(T, T_PTS, CP_PTS, N_PTS); }
double oracle_k_enh(double T, double kmult) {
    if (kmult <= 1.0) return 1.0;
    double s;
    if (T <= T_SOL) s = 0.0;
    else if (T >= T_LIQ) s = 1.0;
    else s = (T - T_SOL) / (T_LIQ - T_SOL);
    return 1.0 + (kmult - 1.0) * s;
}
double oracle_k_eff(double T, double kmult) { return oracle_k_of(T) * oracle_k_enh(T, kmult); }
double oracle_cp_eff(double T) {
    double c = oracle_cp_of(T);
    if (T >= T_SOL && T <= T_LIQ) c += LF / (T_LIQ - T_SOL);
    return c;
}

/* ---- one explicit-Euler step over the whole grid ---------------------- */
void oracle_step(const double* Tin, double* Tout, const OracleStepConst* k,
                 int phys, int bc, double T_D) {
    const int nx = k->nx, ny = k->ny;
    for (int y = 0; y < ny; ++y) {
        const double ypos = (double)y * k->dy;
        for (int x = 0; x < nx; ++x) {
            const size_t c = (size_t)y * nx + x;
            if (bc == 1 && (x == 0 || y == 0 || x == nx - 1 || y == ny - 1)) {
                Tout[c] = T_D;
                continue;
            }
            const double T = Tin[c];
            const double xpos = (double)x * k->dx;
            const double r2 = (xpos - k->x_l) * (xpos - k->x_l)
                            + (ypos - k->y_l) * (ypos - k->y_l);
            if (phys == 0) {
                double lap_x;
                if (x == 0)           lap_x = (Tin[c + 1] - T) * k->inv_dx2;
                else if (x == nx - 1) lap_x = (Tin[c - 1] - T) * k->inv_dx2;
                else lap_x = (Tin[c + 1] - 2.0 * T + Tin[c - 1]) * k->inv_dx2;
                const double Tym = (y == 0) ? T : Tin[c - nx];
                const double Typ = (y == ny - 1) ? T : Tin[c + nx];
                const double lap_y = (Typ - 2.0 * T + Tym) * k->inv_dy2;
                const double S = k->q_scale * k->peak_S
                               * exp(-2.0 * r2 * k->inv_r0_sq) / (k->rho_cp * k->h);
                double q_top = k->hConv * (T - k->Tamb);
                if (k->radiation) {
                    const double T4 = T * T * T * T;
                    const double Ta4 = k->Tamb * k->Tamb * k->Tamb * k->Tamb;
                    q_top += k->eps * SIGMA_SB * (T4 - Ta4);
                }
                const double q_bot = (k->K / k->dSub) * (T - k->Tsub);
                const double loss = (q_top + q_bot) * k->inv_h / k->rho_cp;
                const double dTdt = k->alpha * (lap_x + lap_y) + S - loss;
                Tout[c] = T + k->dt * dTdt;
            } else {
                const double Txm = (x == 0) ? T : Tin[c - 1];
                const double Txp = (x == nx - 1) ? T : Tin[c + 1];
                const double Tym = (y == 0) ? T : Tin[c - nx];
                const double Typ = (y == ny - 1) ? T : Tin[c + nx];
                const double kCe = oracle_k_eff(T, k->kmult);
                const double kxm = 0.5 * (kCe + oracle_k_eff(Txm, k->kmult));
                const double kxp = 0.5 * (kCe + oracle_k_eff(Txp, k->kmult));
                const double kym = 0.5 * (kCe + oracle_k_eff(Tym, k->kmult));
                const double kyp = 0.5 * (kCe + oracle_k_eff(Typ, k->kmult));
                const double div_k_grad = (kxp * (Txp - T) - kxm * (T - Txm)) * k->inv_dx2
                                        + (kyp * (Typ - T) - kym * (T - Tym)) * k->inv_dy2;
                const double q_in = k->q_scale * k->peak_S * exp(-2.0 * r2 * k->inv_r0_sq);
                double q_top = k->hConv * (T - k->Tamb);
                if (k->radiation) {
                    const double T4 = T * T * T * T;
                    const double Ta4 = k->Tamb * k->Tamb * k->Tamb * k->Tamb;
                    q_top += k->eps * SIGMA_SB * (T4 - Ta4);
                }
                const double q_bot = (oracle_k_of(T) / k->dSub) * (T - k->Tsub);
                const double rhs = div_k_grad + (q_in - q_top - q_bot) * k->inv_h;
                Tout[c] = T + k->dt * rhs / (k->rho * oracle_cp_eff(T));
            }
        }
    }
}

/* ---- peak T / argmax / molten-row extent (GPU reduce semantics) ------- */
void oracle_reduce(const double* T, int nx, int ny, double Tm, OraclePartial* out) {
    const long long N = (long long)nx * ny;
    double tmax = -1.0;
    long long arg = N;
    int ymin = ny, ymax = -1;
    for (long long i = 0; i < N; ++i) {
        const double v = T[i];
        if (v > tmax) { tmax = v; arg = i; }
        if (v > Tm) {
            const int yy = (int)(i / nx);
            if (yy < ymin) ymin = yy;
            if (yy > ymax) ymax = yy;
        }
    }
    out->tmax = tmax;
    out->arg = arg;
    out->ymin = ymin;
    out->ymax = ymax;
}

/* ---- measure(): peak T, row-count width, sub-grid width --------------- */
void oracle_measure(const double* T, int nx, int ny, double dy, double Tm,
                    OracleMeasure* m) {
    int y_min = ny, y_max = -1, x_hot = 0;
    double Tmax = 0.0;
    for (int y = 0; y < ny; ++y) {
        const double* row = T + (size_t)y * nx;
        bool any = false;
        for (int x = 0; x < nx; ++x) {
            const double v = row[x];
            if (v > Tmax) { Tmax = v; x_hot = x; }
            if (v > Tm) any = true;
        }
        if (any) {
            if (y < y_min) y_min = y;
            if (y > y_max) y_max = y;
        }
    }
    m->peak_T = Tmax;
    m->x_hot = x_hot;
    m->W_um = (y_max < 0) ? 0.0 : (y_max - y_min + 1) * dy * 1e6;
    m->W_sub_um = 0.0;
    if (Tmax > Tm) {
        int a = -1, b = -1;
        for (int y = 0; y < ny; ++y)
            if (T[(size_t)y * nx + x_hot] > Tm) { if (a < 0) a = y; b = y; }
        if (a >= 0) {
            double y_lo = a * dy, y_hi = b * dy;
            if (a > 0) {
                const double T0 = T[(size_t)(a - 1) * nx + x_hot];
                const double T1 = T[(size_t)a * nx + x_hot];
                y_lo = ((a - 1) + (Tm - T0) / (T1 - T0)) * dy;
            }
            if (b < ny - 1) {
                const double T0 = T[(size_t)b * nx + x_hot];
                const double T1 = T[(size_t)(b + 1) * nx + x_hot];
                y_hi = (b + (Tm - T0) / (T1 - T0)) * dy;
            }
            m->W_sub_um = (y_hi - y_lo) * 1e6;
        }
    }
}

/* Sub-grid melt width from one column (gpu_step_task.hpp:380-395). */
double oracle_w_sub(const double* col, int ny, double dy, double Tm) {
    int a = -1, b = -1;
    for (int y = 0; y < ny; ++y)
        if (col[y] > Tm) { if (a < 0) a = y; b = y; }
    if (a < 0) return 0.0;
    double y_lo = a * dy, y_hi = b * dy;
    if (a > 0) y_lo = ((a - 1) + (Tm - col[a - 1]) / (col[a] - col[a - 1])) * dy;
    if (b < ny - 1) y_hi = (b + (Tm - col[b]) / (col[b + 1] - col[b])) * dy;
    return (y_hi - y_lo) * 1e6;
}

/* ---- n steps along an explicit laser plan ----------------------------- */
int oracle_run(double* T_a, double* T_b, const OracleStepConst* k0,
               const OracleLaser* plan, int n_steps, int phys, int bc,
               double T_D, double Tm, OraclePartial* ring) {
    OracleStepConst k = *k0;
    double* cur = T_a;
    double* nxt = T_b;
    int which = 0;
    for (int s = 0; s < n_steps; ++s) {
        k.x_l = plan[s].x_l;
        k.y_l = plan[s].y_l;
        k.q_scale = plan[s].q_scale;
        oracle_step(cur, nxt, &k, phys, bc, T_D);
        double* t = cur; cur = nxt; nxt = t;
        which ^= 1;
        if (ring) oracle_reduce(cur, k.nx, k.ny, Tm, &ring[s]);
    }
    return which;   /* 0: result in T_a, 1: result in T_b */
}
