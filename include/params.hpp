// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Physical parameters of the 2D z-averaged LPBF heat step.
//
// Source-compatible with the reference's include/params.hpp: the same
// namespace, struct names, field names, field order and default values
// (IN718), so host code written against the reference compiles unchanged.
//
//   Material / Process / Domain      params.hpp:13-40
//   dt_cfl                           params.hpp:44-47
//   in718::{interp, k_of, cp_of, k_enh, k_eff, cp_eff, alpha_eff_max}
//                                    params.hpp:61-123
//   dt_cfl_ext                       params.hpp:128-132
//
// The Mills property table values are physical data and must be identical to
// the reference's for parity of the extended physics.
// ---------------------------------------------------------------------------
#pragma once
#include <algorithm>
#include <cmath>

namespace lpbf {

enum class Physics { Baseline, Extended };

inline constexpr double SIGMA_SB = 5.670374419e-8;   // W/m^2/K^4

struct Material {
    double k   = 25.0;      // conductivity           W/m/K
    double rho = 8190.0;    // density                kg/m^3
    double cp  = 565.0;     // heat capacity          J/kg/K
    double Tm  = 1609.0;    // melt threshold         K
    double eps = 0.40;      // emissivity
    double eta = 0.35;      // absorptivity
    constexpr double alpha() const noexcept { return k / (rho * cp); }
};

struct Process {
    double P     = 285.0;     // laser power           W
    double V     = 0.96;      // scan speed            m/s
    double r0    = 33.5e-6;   // 1/e^2 beam radius     m
    double h     = 40.0e-6;   // layer thickness       m
    double hConv = 100.0;     // convection coeff.     W/m^2/K
    double dSub  = 30.0e-6;   // substrate distance    m
    double Tamb  = 298.15;    // ambient               K
    double Tsub  = 298.15;    // substrate             K
    bool   radiation = true;
};

struct Domain {
    double Lx = 1.6e-3, Ly = 0.6e-3;
    int    nx = 240, ny = 120;
    constexpr double dx() const noexcept { return Lx / (nx - 1); }
    constexpr double dy() const noexcept { return Ly / (ny - 1); }
};

// Explicit-Euler stability limit with the reference's 0.35 safety factor.
inline double dt_cfl(Material const& m, Domain const& d) noexcept {
    const double sx = 1.0 / (d.dx() * d.dx());
    const double sy = 1.0 / (d.dy() * d.dy());
    return 0.35 / (m.alpha() * (sx + sy));
}

// Temperature-dependent IN718 properties (Mills), piecewise linear, with the
// latent heat folded into an apparent heat capacity over [T_SOL, T_LIQ].
namespace in718 {

inline constexpr double T_SOL = 1533.0;
inline constexpr double T_LIQ = 1609.0;
inline constexpr double LF    = 210.0e3;

inline constexpr int    N_PTS = 9;
inline constexpr double T_PTS [N_PTS] = { 298,  473,  673,  873, 1073,
                                         1273, 1473, 1533, 1609 };
inline constexpr double K_PTS [N_PTS] = { 8.9, 12.9, 15.8, 18.7, 21.9,
                                         25.6, 28.6, 29.3, 29.6 };
inline constexpr double CP_PTS[N_PTS] = { 435,  479,  515,  558,  580,
                                          628,  670,  685,  720 };

// Clamped piecewise-linear lookup; the segment is found by a forward scan.
inline double interp(double T, double const* xs, double const* ys, int n)
    noexcept {
    if (T <= xs[0])     return ys[0];
    if (T >= xs[n - 1]) return ys[n - 1];
    int i = 1;
    while (T > xs[i]) ++i;
    const double f = (T - xs[i - 1]) / (xs[i] - xs[i - 1]);
    return ys[i - 1] + f * (ys[i] - ys[i - 1]);
}

inline double k_of (double T) noexcept { return interp(T, T_PTS, K_PTS,  N_PTS); }
inline double cp_of(double T) noexcept { return interp(T, T_PTS, CP_PTS, N_PTS); }

// Melt-pool conductivity multiplier: 1 below the solidus, kmult above the
// liquidus, linear in between; kmult <= 1 disables it.
inline double k_enh(double T, double kmult) noexcept {
    if (kmult <= 1.0) return 1.0;
    const double s = (T <= T_SOL) ? 0.0
                   : (T >= T_LIQ) ? 1.0
                   : (T - T_SOL) / (T_LIQ - T_SOL);
    return 1.0 + (kmult - 1.0) * s;
}
inline double k_eff(double T, double kmult) noexcept {
    return k_of(T) * k_enh(T, kmult);
}
inline double cp_eff(double T) noexcept {
    double c = cp_of(T);
    if (T >= T_SOL && T <= T_LIQ) c += LF / (T_LIQ - T_SOL);
    return c;
}
inline double alpha_eff_max(double rho, double kmult) noexcept {
    double m = 0.0;
    for (double T = 298.0; T <= 2200.0; T += 5.0)
        m = std::max(m, k_eff(T, kmult) / (rho * cp_of(T)));
    return m;
}

}  // namespace in718

inline double dt_cfl_ext(Material const& m, Domain const& d,
                         double kmult = 1.0) noexcept {
    const double a  = in718::alpha_eff_max(m.rho, kmult);
    const double sx = 1.0 / (d.dx() * d.dx());
    const double sy = 1.0 / (d.dy() * d.dy());
    return 0.35 / (a * (sx + sy));
}

}  // namespace lpbf
