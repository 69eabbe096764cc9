// ORACLE — test infrastructure only (see refelem.hpp header).
// Exact Riemann solution for the Euler equations (Toro, "Riemann Solvers and
// Numerical Methods for Fluid Dynamics", ch. 4), restating the reference's
// src/sod_exact_riemann.mojo: f_K pressure functions (:1-35), the Newton star
// pressure solve seeded with the two-rarefaction guess (:38-85) and the wave
// sampling of sod_exact_rho (:88-120), extended to sample u and p and both
// wave families (shock or rarefaction on either side) as Toro's sampler does.
#pragma once
#include <cmath>
#include <stdexcept>

namespace orc {

inline double sod_fK(double p, double rK, double pK, double aK, double g) {  // sod_exact_riemann.mojo f_K
  if (p > pK) {
    double A = 2.0 / ((g + 1.0) * rK), B = (g - 1.0) / (g + 1.0) * pK;
    return (p - pK) * std::sqrt(A / (p + B));
  }
  double e = (g - 1.0) / (2.0 * g);
  return (2.0 * aK / (g - 1.0)) * (std::pow(p / pK, e) - 1.0);
}
inline double sod_dfK(double p, double rK, double pK, double aK, double g) {
  if (p > pK) {
    double A = 2.0 / ((g + 1.0) * rK), B = (g - 1.0) / (g + 1.0) * pK;
    double s = std::sqrt(A / (p + B));
    return s * (1.0 - 0.5 * (p - pK) / (p + B));
  }
  return (1.0 / (rK * aK)) * std::pow(p / pK, -(g + 1.0) / (2.0 * g));
}
inline double sod_pstar(double rL, double uL, double pL, double aL, double rR, double uR, double pR, double aR, double g) {
  double e = (g - 1.0) / (2.0 * g);
  double ptr = std::pow((aL + aR - 0.5 * (g - 1.0) * (uR - uL)) / (aL / std::pow(pL, e) + aR / std::pow(pR, e)), 1.0 / e);
  double p = ptr > 0.0 ? ptr : 0.5 * (pL + pR);
  for (int it = 0; it < 50; ++it) {
    double res = sod_fK(p, rL, pL, aL, g) + sod_fK(p, rR, pR, aR, g) + (uR - uL);
    double dp = -res / (sod_dfK(p, rL, pL, aL, g) + sod_dfK(p, rR, pR, aR, g));
    double pn = p + dp;
    if (pn <= 0.0) pn = 0.5 * p;
    double rel = std::fabs(2.0 * (pn - p) / (pn + p));
    p = pn;
    if (rel < 1.0e-10) return p;
  }
  throw std::runtime_error("Sod Newton did not converge");
}
// out4 = {p_star, u_star, rho_star_L, rho_star_R}
inline void sod_star(double rL, double uL, double pL, double rR, double uR, double pR, double g, double* out) {
  double aL = std::sqrt(g * pL / rL), aR = std::sqrt(g * pR / rR);
  double ps = sod_pstar(rL, uL, pL, aL, rR, uR, pR, aR, g);
  double us = 0.5 * (uL + uR) + 0.5 * (sod_fK(ps, rR, pR, aR, g) - sod_fK(ps, rL, pL, aL, g));
  double gm = (g - 1.0) / (g + 1.0);
  double rsl = ps > pL ? rL * ((ps / pL + gm) / (gm * ps / pL + 1.0)) : rL * std::pow(ps / pL, 1.0 / g);
  double rsr = ps > pR ? rR * ((ps / pR + gm) / (gm * ps / pR + 1.0)) : rR * std::pow(ps / pR, 1.0 / g);
  out[0] = ps;
  out[1] = us;
  out[2] = rsl;
  out[3] = rsr;
}
inline void sod_sample(double rL, double uL, double pL, double rR, double uR, double pR, double g, double x0, double t,
                       const double* x, int n, double* rho, double* u, double* p) {
  double st[4];
  sod_star(rL, uL, pL, rR, uR, pR, g, st);
  const double ps = st[0], us = st[1];
  const double aL = std::sqrt(g * pL / rL), aR = std::sqrt(g * pR / rR);
  for (int k = 0; k < n; ++k) {
    double xi = (x[k] - x0) / t, r, v, pp;
    if (xi <= us) {  // left of contact
      if (ps > pL) {  // left shock
        double SL = uL - aL * std::sqrt((g + 1.0) / (2.0 * g) * ps / pL + (g - 1.0) / (2.0 * g));
        if (xi <= SL) { r = rL; v = uL; pp = pL; }
        else { r = st[2]; v = us; pp = ps; }
      } else {  // left rarefaction
        double asL = aL * std::pow(ps / pL, (g - 1.0) / (2.0 * g));
        double hd = uL - aL, tl = us - asL;
        if (xi <= hd) { r = rL; v = uL; pp = pL; }
        else if (xi > tl) { r = st[2]; v = us; pp = ps; }
        else {
          double c = 2.0 / (g + 1.0) + (g - 1.0) / ((g + 1.0) * aL) * (uL - xi);
          r = rL * std::pow(c, 2.0 / (g - 1.0));
          v = 2.0 / (g + 1.0) * (aL + 0.5 * (g - 1.0) * uL + xi);
          pp = pL * std::pow(c, 2.0 * g / (g - 1.0));
        }
      }
    } else {  // right of contact
      if (ps > pR) {  // right shock
        double SR = uR + aR * std::sqrt((g + 1.0) / (2.0 * g) * ps / pR + (g - 1.0) / (2.0 * g));
        if (xi >= SR) { r = rR; v = uR; pp = pR; }
        else { r = st[3]; v = us; pp = ps; }
      } else {  // right rarefaction
        double asR = aR * std::pow(ps / pR, (g - 1.0) / (2.0 * g));
        double hd = uR + aR, tl = us + asR;
        if (xi >= hd) { r = rR; v = uR; pp = pR; }
        else if (xi < tl) { r = st[3]; v = us; pp = ps; }
        else {
          double c = 2.0 / (g + 1.0) - (g - 1.0) / ((g + 1.0) * aR) * (uR - xi);
          r = rR * std::pow(c, 2.0 / (g - 1.0));
          v = 2.0 / (g + 1.0) * (-aR + 0.5 * (g - 1.0) * uR + xi);
          pp = pR * std::pow(c, 2.0 * g / (g - 1.0));
        }
      }
    }
    rho[k] = r;
    u[k] = v;
    p[k] = pp;
  }
}

}  // namespace orc
