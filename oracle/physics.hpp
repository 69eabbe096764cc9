// ORACLE — test infrastructure only (see refelem.hpp header).
// CPU restatement of mojoxm's `Physics` implementations used by the 3D
// solver: Advection (src/advection.mojo), Euler with Rusanov / Roe / HLLE /
// HLLEC and the Harten-Hyman entropy fix (src/euler.mojo), vacuum Maxwell
// (src/maxwell.mojo), shallow water embedded in 3D (src/shallow_water.mojo)
// ideal MHD with GLM divergence cleaning (src/mhd.mojo) and the five-moment
// two-fluid plasma model (src/two_fluid.mojo).
// Templated on the arithmetic type so the same code runs in FP64 (the oracle
// proper) and in FP32 (mimicking the reference's all-Float32 GPU path).
#pragma once
#include <algorithm>
#include <cmath>

#include "mesh3d.hpp"

namespace orc {

// PHYS_MHD: 3D IdealMHD (9 components); in 2D the GLM stack (7 components).
// PHYS_MHD_PLAIN: the 2D stack without divergence cleaning (6 components).
enum { PHYS_ADVECTION = 0, PHYS_EULER = 1, PHYS_MAXWELL = 2, PHYS_SW = 3, PHYS_MHD = 4, PHYS_MHD_PLAIN = 5,
       PHYS_TWO_FLUID = 6 };
enum { FLUX_RUSANOV = 0, FLUX_ROE = 1, FLUX_HLLE = 2, FLUX_HLLEC = 3, FLUX_HLLC = 4, FLUX_HLL = 5 };

template <typename R>
inline R rmax(R a, R b) { return a > b ? a : b; }
template <typename R>
inline R rmin(R a, R b) { return a < b ? a : b; }
template <typename R>
inline R rabs(R a) { return a >= R(0) ? a : -a; }

// ---------------------------------------------------------------- Advection
template <typename R>
struct Advection {  // advection.mojo:187-286
  static constexpr int NC = 1;
  R vx, vy, vz, inflow_q;
  void internal_flux(const R* q, R* f) const {  // :227-233
    f[0] = vx * q[0];
    f[1] = vy * q[0];
    f[2] = vz * q[0];
  }
  R numerical_flux(const R* ql, const R* qr, R nx, R ny, R nz, R* f) const {  // :241-253
    R nc = vx * nx + vy * ny + vz * nz;
    R a = rabs(nc);
    f[0] = R(0.5) * ((nc + a) * ql[0] + (nc - a) * qr[0]);
    return a;
  }
  R boundary_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {  // :265-279
    R nc = vx * nx + vy * ny + vz * nz;
    R a = rabs(nc);
    R g = (bc == BC_INFLOW) ? inflow_q : R(0);
    f[0] = R(0.5) * ((nc + a) * q[0] + (nc - a) * g);
    return a;
  }
  void source_term(const R*, R* s) const { s[0] = R(0); }
  void limit_state(R*) const {}
};

// -------------------------------------------------------------------- Euler
template <typename R>
struct Euler {  // euler.mojo:531-792
  static constexpr int NC = 5;
  R gamma, min_density, min_pressure;
  int flux_type;
  bool entropy_fix;
  R gx, gy, gz;
  R inflow[5];

  R rho_f(const R* q) const { return q[0] > min_density ? q[0] : min_density; }  // :44-46
  R p_f(const R* q) const {                                                        // :49-56
    R rho = rho_f(q);
    R ke = R(0.5) * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) / rho;
    R p = (gamma - R(1)) * (q[4] - ke);
    return p > min_pressure ? p : min_pressure;
  }
  void flux_1d(const R* q, R* f) const {  // :64-72
    R rho = rho_f(q), p = p_f(q);
    R u = q[1] / rho;
    f[0] = q[1];
    f[1] = q[1] * u + p;
    f[2] = q[2] * u;
    f[3] = q[3] * u;
    f[4] = u * (q[4] + p);
  }
  void internal_flux(const R* q, R* f) const {  // :597-621
    R rho = rho_f(q), p = p_f(q);
    R u = q[1] / rho, v = q[2] / rho, w = q[3] / rho;
    f[0] = q[1]; f[1] = q[1] * u + p; f[2] = q[1] * v; f[3] = q[1] * w; f[4] = u * (q[4] + p);
    f[5] = q[2]; f[6] = q[2] * u; f[7] = q[2] * v + p; f[8] = q[2] * w; f[9] = v * (q[4] + p);
    f[10] = q[3]; f[11] = q[3] * u; f[12] = q[3] * v; f[13] = q[3] * w + p; f[14] = w * (q[4] + p);
  }
  struct TB { R tx, ty, tz, bx, by, bz; };
  static TB construct_tb(R nx, R ny, R nz) {  // :94-118
    R ax = nx, ay = ny, az = nz;
    R anx = ax >= R(0) ? ax : -ax;
    if (anx >= R(0.9)) ay += R(1); else ax += R(1);
    R pro = nx * ax + ny * ay + nz * az;
    ax -= nx * pro; ay -= ny * pro; az -= nz * pro;
    R mag = std::sqrt(ax * ax + ay * ay + az * az);
    TB t;
    t.tx = ax / mag; t.ty = ay / mag; t.tz = az / mag;
    t.bx = ny * t.tz - nz * t.ty;
    t.by = nz * t.tx - nx * t.tz;
    t.bz = nx * t.ty - ny * t.tx;
    return t;
  }
  void roe_avg(const R* ql, const R* qr, R pl, R pr, R& u, R& v, R& w, R& enth, R& a) const {  // :161-176
    R g1 = gamma - R(1);
    R rl = rho_f(ql), rr = rho_f(qr);
    R sl = std::sqrt(rl), sr = std::sqrt(rr), s = sl + sr;
    u = (ql[1] / sl + qr[1] / sr) / s;
    v = (ql[2] / sl + qr[2] / sr) / s;
    w = (ql[3] / sl + qr[3] / sr) / s;
    enth = ((ql[4] + pl) / sl + (qr[4] + pr) / sr) / s;
    R q2 = u * u + v * v + w * w;
    R aa2 = rmax(g1 * (enth - R(0.5) * q2), R(0));
    a = std::sqrt(aa2);
  }
  static void fluctuations(const R* s, const R* wave, R* amdq, R* apdq) {  // :184-199
    for (int m = 0; m < 5; ++m) {
      amdq[m] = R(0); apdq[m] = R(0);
      for (int mw = 0; mw < 3; ++mw) {
        R sm = s[mw], wm = wave[m * 3 + mw];
        if (sm < R(0)) amdq[m] += sm * wm; else apdq[m] += sm * wm;
      }
    }
  }
  void hh_fix(const R* ql, const R* qr, const R* s, const R* wave, R* amdq, R* apdq) const {  // :207-288
    R rho_l = rho_f(ql), p_l = p_f(ql);
    R c_l = std::sqrt(gamma * p_l / rho_l);
    R s0 = ql[1] / rho_l - c_l;
    for (int m = 0; m < 5; ++m) amdq[m] = R(0);
    bool apdq_only = s0 > R(0) && s[0] > R(0);
    if (!apdq_only) {
      R q10 = rmax(ql[0] + wave[0], min_density);
      R q11 = ql[1] + wave[3], q12 = ql[2] + wave[6], q13 = ql[3] + wave[9], q14 = ql[4] + wave[12];
      R ke1 = R(0.5) * (q11 * q11 + q12 * q12 + q13 * q13) / q10;
      R p1 = rmax((gamma - R(1)) * (q14 - ke1), min_pressure);
      R c1 = std::sqrt(gamma * p1 / q10);
      R s1 = q11 / q10 - c1;
      R sf;
      if (s0 < R(0) && s1 > R(0)) sf = s0 * (s1 - s[0]) / (s1 - s0);
      else if (s[0] < R(0)) sf = s[0];
      else sf = R(0);
      for (int m = 0; m < 5; ++m) amdq[m] = sf * wave[m * 3 + 0];
      if (s[1] < R(0)) {
        for (int m = 0; m < 5; ++m) amdq[m] += s[1] * wave[m * 3 + 1];
        R rho_r = rho_f(qr), p_r = p_f(qr);
        R c_r = std::sqrt(gamma * p_r / rho_r);
        R s3 = qr[1] / rho_r + c_r;
        R q20 = rmax(qr[0] - wave[2], min_density);
        R q21 = qr[1] - wave[5], q22 = qr[2] - wave[8], q23 = qr[3] - wave[11], q24 = qr[4] - wave[14];
        R ke2 = R(0.5) * (q21 * q21 + q22 * q22 + q23 * q23) / q20;
        R p2 = rmax((gamma - R(1)) * (q24 - ke2), min_pressure);
        R c2 = std::sqrt(gamma * p2 / q20);
        R s2 = q21 / q20 + c2;
        R sf2;
        if (s2 < R(0) && s3 > R(0)) sf2 = s2 * (s3 - s[2]) / (s3 - s2);
        else if (s[2] < R(0)) sf2 = s[2];
        else sf2 = R(0);
        for (int m = 0; m < 5; ++m) amdq[m] += sf2 * wave[m * 3 + 2];
      }
    }
    for (int m = 0; m < 5; ++m) {
      R ddf = R(0);
      for (int mw = 0; mw < 3; ++mw) ddf += s[mw] * wave[m * 3 + mw];
      apdq[m] = ddf - amdq[m];
    }
  }
  void roe(const R* ql, const R* qr, R* s, R* wave, R* amdq, R* apdq) const {  // :296-361
    R g1 = gamma - R(1);
    R d0 = qr[0] - ql[0], d1 = qr[1] - ql[1], d2 = qr[2] - ql[2], d3 = qr[3] - ql[3], d4 = qr[4] - ql[4];
    R pl = p_f(ql), pr = p_f(qr);
    R u, v, w, enth, a;
    roe_avg(ql, qr, pl, pr, u, v, w, enth, a);
    R q2 = u * u + v * v + w * w;
    R g1a2 = g1 / (a * a);
    R euv = enth - q2;
    R a4 = g1a2 * (euv * d0 + u * d1 + v * d2 + w * d3 - d4);
    R a2 = d2 - v * d0;
    R a3 = d3 - w * d0;
    R a5 = (d1 + (a - u) * d0 - a * a4) / (R(2) * a);
    R a1 = d0 - a4 - a5;
    wave[0] = a1; wave[3] = a1 * (u - a); wave[6] = a1 * v; wave[9] = a1 * w; wave[12] = a1 * (enth - u * a);
    s[0] = u - a;
    wave[1] = a4; wave[4] = a4 * u; wave[7] = a4 * v + a2; wave[10] = a4 * w + a3;
    wave[13] = a4 * R(0.5) * q2 + a2 * v + a3 * w;
    s[1] = u;
    wave[2] = a5; wave[5] = a5 * (u + a); wave[8] = a5 * v; wave[11] = a5 * w; wave[14] = a5 * (enth + u * a);
    s[2] = u + a;
    if (entropy_fix) hh_fix(ql, qr, s, wave, amdq, apdq); else fluctuations(s, wave, amdq, apdq);
  }
  void hlle(const R* ql, const R* qr, R* s, R* wave, R* amdq, R* apdq) const {  // :364-412
    R pl = p_f(ql), pr = p_f(qr);
    R u, v, w, enth, a;
    roe_avg(ql, qr, pl, pr, u, v, w, enth, a);
    R rl = rho_f(ql), al = std::sqrt(gamma * pl / rl), ul = ql[1] / rl;
    R rr = rho_f(qr), ar = std::sqrt(gamma * pr / rr), ur = qr[1] / rr;
    s[0] = rmin(ul - al, u - a);
    s[2] = rmax(ur + ar, u + a);
    s[1] = R(0);
    R fl[5], fr[5];
    flux_1d(ql, fl);
    flux_1d(qr, fr);
    R den = s[0] - s[2];
    for (int m = 0; m < 5; ++m) {
      R qh = (fr[m] - fl[m] - s[2] * qr[m] + s[0] * ql[m]) / den;
      wave[m * 3 + 0] = qh - ql[m];
      wave[m * 3 + 1] = R(0);
      wave[m * 3 + 2] = qr[m] - qh;
    }
    if (entropy_fix) hh_fix(ql, qr, s, wave, amdq, apdq); else fluctuations(s, wave, amdq, apdq);
  }
  void hllec(const R* ql, const R* qr, R* s, R* wave, R* amdq, R* apdq) const {  // :415-485
    R pl = p_f(ql), pr = p_f(qr);
    R u, v, w, enth, a;
    roe_avg(ql, qr, pl, pr, u, v, w, enth, a);
    R rl = rho_f(ql), al = std::sqrt(gamma * pl / rl), ul = ql[1] / rl;
    R rr = rho_f(qr), ar = std::sqrt(gamma * pr / rr), ur = qr[1] / rr;
    s[0] = rmin(ul - al, u - a);
    s[2] = rmax(ur + ar, u + a);
    s[1] = (pr - pl + rl * ul * (s[0] - ul) - rr * ur * (s[2] - ur)) / (rl * (s[0] - ul) - rr * (s[2] - ur));
    R lm = rl * (s[0] - ul) / (s[0] - s[1]);
    R hL[5] = {lm, lm * s[1], lm * ql[2] / rl, lm * ql[3] / rl,
               lm * (ql[4] / rl + (s[1] - ul) * (s[1] + pl / (rl * (s[0] - ul))))};
    R rm = rr * (s[2] - ur) / (s[2] - s[1]);
    R hR[5] = {rm, rm * s[1], rm * qr[2] / rr, rm * qr[3] / rr,
               rm * (qr[4] / rr + (s[1] - ur) * (s[1] + pr / (rr * (s[2] - ur))))};
    for (int m = 0; m < 5; ++m) {
      wave[m * 3 + 0] = hL[m] - ql[m];
      wave[m * 3 + 1] = hR[m] - hL[m];
      wave[m * 3 + 2] = qr[m] - hR[m];
    }
    if (entropy_fix) hh_fix(ql, qr, s, wave, amdq, apdq); else fluctuations(s, wave, amdq, apdq);
  }
  R numerical_flux(const R* q_l, const R* q_r, R nx, R ny, R nz, R* flux) const {  // :626-691
    TB tb = construct_tb(nx, ny, nz);
    R ql[5], qr[5], rf[5];
    ql[0] = q_l[0]; ql[4] = q_l[4];
    ql[1] = nx * q_l[1] + ny * q_l[2] + nz * q_l[3];
    ql[2] = tb.tx * q_l[1] + tb.ty * q_l[2] + tb.tz * q_l[3];
    ql[3] = tb.bx * q_l[1] + tb.by * q_l[2] + tb.bz * q_l[3];
    qr[0] = q_r[0]; qr[4] = q_r[4];
    qr[1] = nx * q_r[1] + ny * q_r[2] + nz * q_r[3];
    qr[2] = tb.tx * q_r[1] + tb.ty * q_r[2] + tb.tz * q_r[3];
    qr[3] = tb.bx * q_r[1] + tb.by * q_r[2] + tb.bz * q_r[3];
    R vmax;
    if (flux_type == FLUX_RUSANOV) {  // :649-668
      R rhol = rho_f(ql), rhor = rho_f(qr), pl = p_f(ql), pr = p_f(qr);
      R cl = std::sqrt(gamma * pl / rhol), cr = std::sqrt(gamma * pr / rhor);
      R uxl = ql[1] / rhol, uxr = qr[1] / rhor;
      R cmax = rmax(rabs(uxl) + cl, rabs(uxr) + cr);
      rf[0] = R(0.5) * (ql[1] + qr[1] + cmax * (rhol - rhor));
      rf[1] = R(0.5) * (ql[1] * uxl + pl + qr[1] * uxr + pr + cmax * (ql[1] - qr[1]));
      rf[2] = R(0.5) * (ql[2] * uxl + qr[2] * uxr + cmax * (ql[2] - qr[2]));
      rf[3] = R(0.5) * (ql[3] * uxl + qr[3] * uxr + cmax * (ql[3] - qr[3]));
      rf[4] = R(0.5) * ((ql[4] + pl) * uxl + (qr[4] + pr) * uxr + cmax * (ql[4] - qr[4]));
      vmax = cmax;
    } else {
      R s[3], wave[15], amdq[5], apdq[5];
      if (flux_type == FLUX_ROE) roe(ql, qr, s, wave, amdq, apdq);
      else if (flux_type == FLUX_HLLE) hlle(ql, qr, s, wave, amdq, apdq);
      else hllec(ql, qr, s, wave, amdq, apdq);
      R fl[5], fr[5];  // euler_flux_from_fluctuations :495-520
      flux_1d(ql, fl);
      flux_1d(qr, fr);
      for (int m = 0; m < 5; ++m) rf[m] = R(0.5) * (fl[m] + fr[m]) - R(0.5) * (apdq[m] - amdq[m]);
      vmax = rmax(rmax(rabs(s[0]), rabs(s[1])), rabs(s[2]));
    }
    flux[0] = rf[0]; flux[4] = rf[4];  // euler_antirotate :137-143
    flux[1] = nx * rf[1] + tb.tx * rf[2] + tb.bx * rf[3];
    flux[2] = ny * rf[1] + tb.ty * rf[2] + tb.by * rf[3];
    flux[3] = nz * rf[1] + tb.tz * rf[2] + tb.bz * rf[3];
    return vmax;
  }
  R boundary_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {  // :705-730
    R g[5];
    if (bc == BC_WALL) {
      g[0] = q[0]; g[4] = q[4];
      R mn = q[1] * nx + q[2] * ny + q[3] * nz;
      g[1] = q[1] - R(2) * mn * nx;
      g[2] = q[2] - R(2) * mn * ny;
      g[3] = q[3] - R(2) * mn * nz;
    } else if (bc == BC_INFLOW) {
      for (int c = 0; c < 5; ++c) g[c] = inflow[c];
    } else {
      for (int c = 0; c < 5; ++c) g[c] = q[c];
    }
    return numerical_flux(q, g, nx, ny, nz, f);
  }
  void source_term(const R* q, R* s) const {  // :738-747
    s[0] = R(0);
    s[1] = q[0] * gx;
    s[2] = q[0] * gy;
    s[3] = q[0] * gz;
    s[4] = q[1] * gx + q[2] * gy + q[3] * gz;
  }
  void limit_state(R* q) const {  // :758-792
    R rho = q[0];
    if (!(rho > min_density)) {
      q[0] = min_density; q[1] = R(0); q[2] = R(0); q[3] = R(0);
      q[4] = min_pressure / (gamma - R(1));
      return;
    }
    R m2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (!(m2 >= R(0))) {
      q[1] = R(0); q[2] = R(0); q[3] = R(0);
      q[4] = min_pressure / (gamma - R(1));
      return;
    }
    R ke = R(0.5) * m2 / rho;
    R p = (gamma - R(1)) * (q[4] - ke);
    if (!(p > min_pressure)) q[4] = ke + min_pressure / (gamma - R(1));
  }
};

// ------------------------------------------------------------------ Maxwell
template <typename R>
struct Maxwell {  // maxwell.mojo:48-255
  static constexpr int NC = 6;
  R c, J[3], M[3], inflow[6];
  void internal_flux(const R* q, R* f) const {  // :127-156
    R c2 = c * c;
    R Ex = q[0], Ey = q[1], Ez = q[2], Bx = q[3], By = q[4], Bz = q[5];
    f[0] = R(0); f[1] = c2 * Bz; f[2] = -c2 * By; f[3] = R(0); f[4] = -Ez; f[5] = Ey;
    f[6] = -c2 * Bz; f[7] = R(0); f[8] = c2 * Bx; f[9] = Ez; f[10] = R(0); f[11] = -Ex;
    f[12] = c2 * By; f[13] = -c2 * Bx; f[14] = R(0); f[15] = -Ey; f[16] = Ex; f[17] = R(0);
  }
  R numerical_flux(const R* l, const R* r, R nx, R ny, R nz, R* f) const {  // :161-207
    R c2 = c * c;
    R FElx = c2 * (l[4] * nz - l[5] * ny), FEly = c2 * (l[5] * nx - l[3] * nz), FElz = c2 * (l[3] * ny - l[4] * nx);
    R FErx = c2 * (r[4] * nz - r[5] * ny), FEry = c2 * (r[5] * nx - r[3] * nz), FErz = c2 * (r[3] * ny - r[4] * nx);
    R FBlx = ny * l[2] - nz * l[1], FBly = nz * l[0] - nx * l[2], FBlz = nx * l[1] - ny * l[0];
    R FBrx = ny * r[2] - nz * r[1], FBry = nz * r[0] - nx * r[2], FBrz = nx * r[1] - ny * r[0];
    R h = R(0.5), al = c;
    f[0] = h * (FElx + FErx) - h * al * (r[0] - l[0]);
    f[1] = h * (FEly + FEry) - h * al * (r[1] - l[1]);
    f[2] = h * (FElz + FErz) - h * al * (r[2] - l[2]);
    f[3] = h * (FBlx + FBrx) - h * al * (r[3] - l[3]);
    f[4] = h * (FBly + FBry) - h * al * (r[4] - l[4]);
    f[5] = h * (FBlz + FBrz) - h * al * (r[5] - l[5]);
    return c;
  }
  R boundary_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {  // :213-240
    R g[6];
    if (bc == BC_WALL) {
      R En = q[0] * nx + q[1] * ny + q[2] * nz;
      R Bn = q[3] * nx + q[4] * ny + q[5] * nz;
      g[0] = R(2) * En * nx - q[0]; g[1] = R(2) * En * ny - q[1]; g[2] = R(2) * En * nz - q[2];
      g[3] = q[3] - R(2) * Bn * nx; g[4] = q[4] - R(2) * Bn * ny; g[5] = q[5] - R(2) * Bn * nz;
    } else if (bc == BC_INFLOW) {
      for (int k = 0; k < 6; ++k) g[k] = inflow[k];
    } else {
      for (int k = 0; k < 6; ++k) g[k] = q[k];
    }
    return numerical_flux(q, g, nx, ny, nz, f);
  }
  void source_term(const R*, R* s) const {  // :245-252
    R c2 = c * c;
    s[0] = -c2 * J[0]; s[1] = -c2 * J[1]; s[2] = -c2 * J[2];
    s[3] = -M[0]; s[4] = -M[1]; s[5] = -M[2];
  }
  void limit_state(R*) const {}
};

// ------------------------------------------------------------ ShallowWater
template <typename R>
struct ShallowWater {  // shallow_water.mojo:31-167
  static constexpr int NC = 3;
  R g, h_min, inflow[3];
  void internal_flux(const R* q, R* f) const {  // :63-86
    R h = q[0] > h_min ? q[0] : h_min;
    R hu = q[1], hv = q[2], u = hu / h, v = hv / h;
    R gh = R(0.5) * g * h * h;
    f[0] = hu; f[1] = hu * u + gh; f[2] = hu * v;
    f[3] = hv; f[4] = hu * v; f[5] = hv * v + gh;
    f[6] = R(0); f[7] = R(0); f[8] = R(0);
  }
  R numerical_flux(const R* l, const R* r, R nx, R ny, R, R* f) const {  // :90-134
    R hl = l[0] > h_min ? l[0] : h_min;
    R ul = l[1] / hl, vl = l[2] / hl, unl = ul * nx + vl * ny, cl = std::sqrt(g * hl), gl = R(0.5) * g * hl * hl;
    R hr = r[0] > h_min ? r[0] : h_min;
    R ur = r[1] / hr, vr = r[2] / hr, unr = ur * nx + vr * ny, cr = std::sqrt(g * hr), gr = R(0.5) * g * hr * hr;
    R Fl0 = l[1] * nx + l[2] * ny, Fl1 = l[1] * unl + gl * nx, Fl2 = l[2] * unl + gl * ny;
    R Fr0 = r[1] * nx + r[2] * ny, Fr1 = r[1] * unr + gr * nx, Fr2 = r[2] * unr + gr * ny;
    R al = rmax(rabs(unl) + cl, rabs(unr) + cr);
    R h = R(0.5);
    f[0] = h * (Fl0 + Fr0) - h * al * (r[0] - l[0]);
    f[1] = h * (Fl1 + Fr1) - h * al * (r[1] - l[1]);
    f[2] = h * (Fl2 + Fr2) - h * al * (r[2] - l[2]);
    return al;
  }
  R boundary_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {  // :138-156
    R gs[3];
    if (bc == BC_WALL) {
      gs[0] = q[0];
      R mn = q[1] * nx + q[2] * ny;
      gs[1] = q[1] - R(2) * mn * nx;
      gs[2] = q[2] - R(2) * mn * ny;
    } else if (bc == BC_INFLOW) {
      gs[0] = inflow[0]; gs[1] = inflow[1]; gs[2] = inflow[2];
    } else {
      gs[0] = q[0]; gs[1] = q[1]; gs[2] = q[2];
    }
    return numerical_flux(q, gs, nx, ny, nz, f);
  }
  void source_term(const R*, R* s) const { s[0] = R(0); s[1] = R(0); s[2] = R(0); }
  void limit_state(R*) const {}
};

// ------------------------------------------------------------------ IdealMHD
// q = [rho, rho u, rho v, rho w, E, Bx, By, Bz, psi]
template <typename R>
struct IdealMHD {  // mhd.mojo:199-367
  static constexpr int NC = 9;
  R gamma, min_density, min_pressure, c_h, alpha_d, inflow[9];
  R rho_f(const R* q) const { return q[0] > min_density ? q[0] : min_density; }  // :46-48
  R gas_pressure(const R* q) const {  // :51-62
    R rho = rho_f(q);
    R ke = R(0.5) * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) / rho;
    R me = R(0.5) * (q[5] * q[5] + q[6] * q[6] + q[7] * q[7]);
    R p = (gamma - R(1)) * (q[4] - ke - me);
    return p > min_pressure ? p : min_pressure;
  }
  R fast_speed(const R* q, R nx, R ny, R nz) const {  // :71-85
    R rho = rho_f(q), p = gas_pressure(q);
    R bx = q[5], by = q[6], bz = q[7], bn = bx * nx + by * ny + bz * nz;
    R cs2 = gamma * p / rho, ca2 = (bx * bx + by * by + bz * bz) / rho, can2 = (bn * bn) / rho;
    R disc = (cs2 + ca2) * (cs2 + ca2) - R(4) * cs2 * can2;
    if (disc < R(0)) disc = R(0);
    return std::sqrt(R(0.5) * (cs2 + ca2 + std::sqrt(disc)));
  }
  void internal_flux(const R* q, R* f) const {  // :92-146
    R rho = rho_f(q), mx = q[1], my = q[2], mz = q[3], u = mx / rho, v = my / rho, w = mz / rho;
    R E = q[4], bx = q[5], by = q[6], bz = q[7], psi = q[8];
    R pt = gas_pressure(q) + R(0.5) * (bx * bx + by * by + bz * bz);
    R ub = u * bx + v * by + w * bz, ch2 = c_h * c_h;
    f[0] = mx; f[1] = mx * u + pt - bx * bx; f[2] = mx * v - bx * by; f[3] = mx * w - bx * bz;
    f[4] = u * (E + pt) - bx * ub; f[5] = psi; f[6] = u * by - v * bx; f[7] = u * bz - w * bx; f[8] = ch2 * bx;
    f[9] = my; f[10] = my * u - by * bx; f[11] = my * v + pt - by * by; f[12] = my * w - by * bz;
    f[13] = v * (E + pt) - by * ub; f[14] = v * bx - u * by; f[15] = psi; f[16] = v * bz - w * by; f[17] = ch2 * by;
    f[18] = mz; f[19] = mz * u - bz * bx; f[20] = mz * v - bz * by; f[21] = mz * w + pt - bz * bz;
    f[22] = w * (E + pt) - bz * ub; f[23] = w * bx - u * bz; f[24] = w * by - v * bz; f[25] = psi; f[26] = ch2 * bz;
  }
  void normal_flux(const R* q, R nx, R ny, R nz, R* F) const {  // :151-194
    R rho = rho_f(q), u = q[1] / rho, v = q[2] / rho, w = q[3] / rho;
    R E = q[4], bx = q[5], by = q[6], bz = q[7], psi = q[8];
    R pt = gas_pressure(q) + R(0.5) * (bx * bx + by * by + bz * bz);
    R ub = u * bx + v * by + w * bz, un = u * nx + v * ny + w * nz, bn = bx * nx + by * ny + bz * nz;
    F[0] = rho * un;
    F[1] = rho * u * un + pt * nx - bn * bx;
    F[2] = rho * v * un + pt * ny - bn * by;
    F[3] = rho * w * un + pt * nz - bn * bz;
    F[4] = un * (E + pt) - bn * ub;
    F[5] = un * bx - u * bn + psi * nx;
    F[6] = un * by - v * bn + psi * ny;
    F[7] = un * bz - w * bn + psi * nz;
    F[8] = c_h * c_h * bn;
  }
  R numerical_flux(const R* l, const R* r, R nx, R ny, R nz, R* f) const {  // :280-307
    R Fl[9], Fr[9];
    normal_flux(l, nx, ny, nz, Fl);
    normal_flux(r, nx, ny, nz, Fr);
    R cfl = fast_speed(l, nx, ny, nz), cfr = fast_speed(r, nx, ny, nz);
    R unl = (l[1] * nx + l[2] * ny + l[3] * nz) / rho_f(l), unr = (r[1] * nx + r[2] * ny + r[3] * nz) / rho_f(r);
    R al = rmax(rmax(rabs(unl) + cfl, rabs(unr) + cfr), c_h);
    R h = R(0.5);
    for (int c = 0; c < 9; ++c) f[c] = h * (Fl[c] + Fr[c]) - h * al * (r[c] - l[c]);
    return al;
  }
  R boundary_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {  // :312-353
    R g[9];
    if (bc == BC_WALL) {  // conducting wall: reflect u_n and B_n
      g[0] = q[0]; g[4] = q[4]; g[8] = q[8];
      R mn = q[1] * nx + q[2] * ny + q[3] * nz;
      g[1] = q[1] - R(2) * mn * nx; g[2] = q[2] - R(2) * mn * ny; g[3] = q[3] - R(2) * mn * nz;
      R bn = q[5] * nx + q[6] * ny + q[7] * nz;
      g[5] = q[5] - R(2) * bn * nx; g[6] = q[6] - R(2) * bn * ny; g[7] = q[7] - R(2) * bn * nz;
    } else if (bc == BC_INFLOW) {
      for (int k = 0; k < 9; ++k) g[k] = inflow[k];
    } else {
      for (int k = 0; k < 9; ++k) g[k] = q[k];
    }
    return numerical_flux(q, g, nx, ny, nz, f);
  }
  void source_term(const R* q, R* s) const {  // :357-361 (GLM damping)
    for (int c = 0; c < 8; ++c) s[c] = R(0);
    s[8] = -alpha_d * q[8];
  }
  void limit_state(R*) const {}
};

// --------------------------------------------------------- FiveMomentTwoFluid
// q[0..4] electrons, q[5..9] ions, q[10..15] (E, B), q[16] psi
template <typename R>
struct TwoFluid {  // two_fluid.mojo:139-513
  static constexpr int NC = 17;
  R gamma_e, gamma_i, q_e, m_e, q_i, m_i, eps0, c_light, c_h, alpha_d, min_density, min_pressure, inflow[17];
  R rho_f(const R* s) const { return s[0] > min_density ? s[0] : min_density; }  // :52-54
  R pressure(const R* s, R g) const {  // :57-65
    R rho = rho_f(s);
    R ke = R(0.5) * (s[1] * s[1] + s[2] * s[2] + s[3] * s[3]) / rho;
    R p = (g - R(1)) * (s[4] - ke);
    return p > min_pressure ? p : min_pressure;
  }
  R sound(const R* s, R g) const { return std::sqrt(g * pressure(s, g) / rho_f(s)); }  // :68-71
  void species_flux_dir(const R* s, R g, int d, R* f) const {  // :76-101
    R rho = rho_f(s), mx = s[1], my = s[2], mz = s[3], u = mx / rho, v = my / rho, w = mz / rho, E = s[4];
    R p = pressure(s, g);
    if (d == 0) { f[0] = mx; f[1] = mx * u + p; f[2] = mx * v; f[3] = mx * w; f[4] = u * (E + p); }
    else if (d == 1) { f[0] = my; f[1] = my * u; f[2] = my * v + p; f[3] = my * w; f[4] = v * (E + p); }
    else { f[0] = mz; f[1] = mz * u; f[2] = mz * v; f[3] = mz * w + p; f[4] = w * (E + p); }
  }
  void species_normal(const R* s, R g, R nx, R ny, R nz, R* f) const {  // :107-132
    R rho = rho_f(s), u = s[1] / rho, v = s[2] / rho, w = s[3] / rho, E = s[4], p = pressure(s, g);
    R un = u * nx + v * ny + w * nz;
    f[0] = rho * un; f[1] = rho * u * un + p * nx; f[2] = rho * v * un + p * ny; f[3] = rho * w * un + p * nz;
    f[4] = un * (E + p);
  }
  void internal_flux(const R* q, R* f) const {  // :258-305
    R c2 = c_light * c_light, ch2 = c_h * c_h;
    R Ex = q[10], Ey = q[11], Ez = q[12], Bx = q[13], By = q[14], Bz = q[15], psi = q[16];
    for (int d = 0; d < 3; ++d) {
      species_flux_dir(q, gamma_e, d, f + d * 17);
      species_flux_dir(q + 5, gamma_i, d, f + d * 17 + 5);
      R* F = f + d * 17;
      if (d == 0) { F[10] = R(0); F[11] = c2 * Bz; F[12] = -c2 * By; F[13] = psi; F[14] = -Ez; F[15] = Ey; F[16] = ch2 * Bx; }
      else if (d == 1) { F[10] = -c2 * Bz; F[11] = R(0); F[12] = c2 * Bx; F[13] = Ez; F[14] = psi; F[15] = -Ex; F[16] = ch2 * By; }
      else { F[10] = c2 * By; F[11] = -c2 * Bx; F[12] = R(0); F[13] = -Ey; F[14] = Ex; F[15] = psi; F[16] = ch2 * Bz; }
    }
  }
  R numerical_flux(const R* l, const R* r, R nx, R ny, R nz, R* f) const {  // :307-374
    R Fl[17], Fr[17];
    species_normal(l, gamma_e, nx, ny, nz, Fl);
    species_normal(r, gamma_e, nx, ny, nz, Fr);
    species_normal(l + 5, gamma_i, nx, ny, nz, Fl + 5);
    species_normal(r + 5, gamma_i, nx, ny, nz, Fr + 5);
    R c2 = c_light * c_light, ch2 = c_h * c_h;
    for (int side = 0; side < 2; ++side) {
      const R* q = side == 0 ? l : r;
      R* F = side == 0 ? Fl : Fr;
      R Ex = q[10], Ey = q[11], Ez = q[12], Bx = q[13], By = q[14], Bz = q[15], psi = q[16];
      R bn = Bx * nx + By * ny + Bz * nz;
      F[10] = c2 * (By * nz - Bz * ny); F[11] = c2 * (Bz * nx - Bx * nz); F[12] = c2 * (Bx * ny - By * nx);
      F[13] = (ny * Ez - nz * Ey) + psi * nx; F[14] = (nz * Ex - nx * Ez) + psi * ny;
      F[15] = (nx * Ey - ny * Ex) + psi * nz; F[16] = ch2 * bn;
    }
    R un_el = (l[1] * nx + l[2] * ny + l[3] * nz) / rho_f(l), un_er = (r[1] * nx + r[2] * ny + r[3] * nz) / rho_f(r);
    R un_il = (l[6] * nx + l[7] * ny + l[8] * nz) / rho_f(l + 5), un_ir = (r[6] * nx + r[7] * ny + r[8] * nz) / rho_f(r + 5);
    R ae = rmax(rabs(un_el) + sound(l, gamma_e), rabs(un_er) + sound(r, gamma_e));
    R ai = rmax(rabs(un_il) + sound(l + 5, gamma_i), rabs(un_ir) + sound(r + 5, gamma_i));
    R al = rmax(rmax(ae, ai), rmax(c_light, c_h)), h = R(0.5);
    for (int c = 0; c < 17; ++c) f[c] = h * (Fl[c] + Fr[c]) - h * al * (r[c] - l[c]);
    return al;
  }
  R boundary_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {  // :376-446
    R g[17];
    for (int k = 0; k < 17; ++k) g[k] = q[k];
    if (bc == BC_WALL) {
      R me = q[1] * nx + q[2] * ny + q[3] * nz, mi = q[6] * nx + q[7] * ny + q[8] * nz;
      g[1] = q[1] - R(2) * me * nx; g[2] = q[2] - R(2) * me * ny; g[3] = q[3] - R(2) * me * nz;
      g[6] = q[6] - R(2) * mi * nx; g[7] = q[7] - R(2) * mi * ny; g[8] = q[8] - R(2) * mi * nz;
      R En = q[10] * nx + q[11] * ny + q[12] * nz, Bn = q[13] * nx + q[14] * ny + q[15] * nz;
      g[10] = R(2) * En * nx - q[10]; g[11] = R(2) * En * ny - q[11]; g[12] = R(2) * En * nz - q[12];
      g[13] = q[13] - R(2) * Bn * nx; g[14] = q[14] - R(2) * Bn * ny; g[15] = q[15] - R(2) * Bn * nz;
    } else if (bc == BC_INFLOW) {
      for (int k = 0; k < 17; ++k) g[k] = inflow[k];
    }
    return numerical_flux(q, g, nx, ny, nz, f);
  }
  void source_term(const R* q, R* s) const {  // :448-510
    R rho_e = rho_f(q), ue = q[1] / rho_e, ve = q[2] / rho_e, we = q[3] / rho_e;
    R rho_i = rho_f(q + 5), ui = q[6] / rho_i, vi = q[7] / rho_i, wi = q[8] / rho_i;
    R Ex = q[10], Ey = q[11], Ez = q[12], Bx = q[13], By = q[14], Bz = q[15], psi = q[16];
    R qme = q_e / m_e, qmi = q_i / m_i;
    s[0] = R(0);
    s[1] = qme * rho_e * (Ex + (ve * Bz - we * By));
    s[2] = qme * rho_e * (Ey + (we * Bx - ue * Bz));
    s[3] = qme * rho_e * (Ez + (ue * By - ve * Bx));
    s[4] = qme * rho_e * (ue * Ex + ve * Ey + we * Ez);
    s[5] = R(0);
    s[6] = qmi * rho_i * (Ex + (vi * Bz - wi * By));
    s[7] = qmi * rho_i * (Ey + (wi * Bx - ui * Bz));
    s[8] = qmi * rho_i * (Ez + (ui * By - vi * Bx));
    s[9] = qmi * rho_i * (ui * Ex + vi * Ey + wi * Ez);
    R Jx = qme * rho_e * ue + qmi * rho_i * ui, Jy = qme * rho_e * ve + qmi * rho_i * vi;
    R Jz = qme * rho_e * we + qmi * rho_i * wi, inv_eps0 = R(1) / eps0;
    s[10] = -Jx * inv_eps0; s[11] = -Jy * inv_eps0; s[12] = -Jz * inv_eps0;
    s[13] = R(0); s[14] = R(0); s[15] = R(0);
    s[16] = -alpha_d * psi;
  }
  void limit_state(R*) const {}
};

}  // namespace orc
