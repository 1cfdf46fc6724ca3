/* SPDX-License-Identifier: 0BSD
 * ORACLE -- test infrastructure only (see lpbf_oracle.c).
 * C mirrors of the reference's POD types (include/lpbf_step_const.hpp:19-33). */
#pragma once
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny;
    double dx, dy, inv_dx2, inv_dy2, inv_r0_sq;
    double alpha, K, rho, cp, rho_cp, inv_h, h, dt;
    double peak_S, eta, P;
    double hConv, Tamb, Tsub, dSub, eps;
    bool radiation;
    double kmult;
    double x_l, y_l;
    double q_scale;
} OracleStepConst;

typedef struct { double tmax; long long arg; int ymin; int ymax; } OraclePartial;
typedef struct { double x_l, y_l, q_scale; } OracleLaser;
typedef struct { double peak_T; int x_hot; double W_um; double W_sub_um; } OracleMeasure;

double oracle_k_of(double T);
double oracle_cp_of(double T);
double oracle_k_enh(double T, double kmult);
double oracle_k_eff(double T, double kmult);
double oracle_cp_eff(double T);
void oracle_step(const double* Tin, double* Tout, const OracleStepConst* k,
                 int phys, int bc, double T_D);
void oracle_reduce(const double* T, int nx, int ny, double Tm, OraclePartial* out);
void oracle_measure(const double* T, int nx, int ny, double dy, double Tm,
                    OracleMeasure* m);
double oracle_w_sub(const double* col, int ny, double dy, double Tm);
int oracle_run(double* T_a, double* T_b, const OracleStepConst* k0,
               const OracleLaser* plan, int n_steps, int phys, int bc,
               double T_D, double Tm, OraclePartial* ring);
int oracle_run_quiet(double* T_a, double* T_b, const OracleStepConst* k0,
                     const OracleLaser* plan, int n_steps, int bc, double T_D, double Tm,
                     OraclePartial* ring, int n_threads, const long long* probe_idx,
                     double* probe_val);

#ifdef __cplusplus
}
#endif
