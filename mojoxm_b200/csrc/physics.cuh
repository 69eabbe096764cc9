// Device physics for the 3D stage kernel: pointwise flux, numerical flux,
// boundary flux (ghost-state), source and positivity floor of mojoxm's
// `Physics` implementations (trait: src/solver.mojo:97-145).
//   Advection     src/advection.mojo:187-286
//   Euler         src/euler.mojo:44-792 (Rusanov/Roe/HLLE/HLLEC, Harten-Hyman fix)
//   Maxwell       src/maxwell.mojo:48-255
//   ShallowWater  src/shallow_water.mojo:31-167
//   IdealMHD      src/mhd.mojo:1-367 (GLM divergence cleaning)
//   TwoFluid      src/two_fluid.mojo:1-513 (five-moment electrons + ions + Maxwell + GLM)
// Each formula keeps the reference's operation order, except that divisions
// by positive quantities (floored densities, square roots of them, the HLLE
// wave-speed span) are taken as one reciprocal and products, which in FP32
// use the hardware reciprocal / reciprocal square root (a few ulp apart from
// the reference's quotients); comparisons that the reference writes as
// `not (x > floor)` stay NaN-catching.
#pragma once
#include "dg_common.cuh"

namespace mxm {

template <class R>
__device__ __forceinline__ R rmax(R a, R b) { return a > b ? a : b; }
template <class R>
__device__ __forceinline__ R rmin(R a, R b) { return a < b ? a : b; }
template <class R>
__device__ __forceinline__ R rabs(R a) { return a >= R(0) ? a : -a; }

// Reciprocal and square root of a positive, floored quantity (density,
// pressure ratio).  FP64 keeps the correctly rounded operations; FP32 uses
// the hardware approximations (within 2 ulp), which the FP32 state carries
// anyway.  Arguments are > 0 and finite wherever these are used.
template <class R>
__device__ __forceinline__ R pos_rcp(R x) { return R(1) / x; }
template <>
__device__ __forceinline__ float pos_rcp<float>(float x) { return __fdividef(1.0f, x); }
template <class R>
__device__ __forceinline__ R pos_sqrt(R x) { return sqrt(x); }
template <>
__device__ __forceinline__ float pos_sqrt<float>(float x) { return x * rsqrtf(x); }

// ------------------------------------------------------------------ advection
template <class R>
struct AdvectionD {
  static constexpr int NC = 1;
  static constexpr bool kSource = false, kLimit = false;
  static constexpr bool kLightFlux = true;
  R vx, vy, vz, inflow_q;
  __device__ void flux(const R* q, R* F) const {  // F[d*NC + c]
    F[0] = vx * q[0];
    F[1] = vy * q[0];
    F[2] = vz * q[0];
  }
  __device__ R num_flux(const R* ql, const R* qr, R nx, R ny, R nz, R* f) const {
    R nc = vx * nx + vy * ny + vz * nz;
    R a = rabs(nc);
    f[0] = R(0.5) * ((nc + a) * ql[0] + (nc - a) * qr[0]);
    return a;
  }
  // ghost state of a boundary face: the BC flux is num_flux(q, ghost)
  __device__ void ghost(const R*, int bc, R, R, R, R* g) const { g[0] = (bc == BC_INFLOW) ? inflow_q : R(0); }
  __device__ R bnd_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {
    R g[1];
    ghost(q, bc, nx, ny, nz, g);
    return num_flux(q, g, nx, ny, nz, f);
  }
  __device__ void source(const R*, R* s) const { s[0] = R(0); }
  __device__ void limit(R*) const {}
};

// ---------------------------------------------------------------------- euler
template <class R, int FLUX>
struct EulerD {
  static constexpr int NC = 5;
  static constexpr bool kSource = true, kLimit = true;
  // register-light numerical flux (the tensor-core stage kernel may then
  // run as many blocks per SM as fit in shared memory, up to three)
  static constexpr bool kLightFlux = FLUX == FLUX_RUSANOV;
  R gamma, rho_min, p_min, gx, gy, gz;
  R inflow[5];
  int entropy_fix;

  __device__ __forceinline__ R rho_f(const R* q) const { return q[0] > rho_min ? q[0] : rho_min; }
  __device__ __forceinline__ R p_f(const R* q, R rho) const {
    R ke = R(0.5) * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) * pos_rcp(rho);
    R p = (gamma - R(1)) * (q[4] - ke);
    return p > p_min ? p : p_min;
  }
  // pressure from the reciprocal density ri = 1/rho and the velocity
  __device__ __forceinline__ R p_fi(const R* q, R u, R v, R w) const {
    R p = (gamma - R(1)) * (q[4] - R(0.5) * (q[1] * u + q[2] * v + q[3] * w));
    return p > p_min ? p : p_min;
  }
  __device__ void flux(const R* q, R* F) const {  // euler.mojo:597-621
    const R ri = pos_rcp(rho_f(q));
    const R u = q[1] * ri, v = q[2] * ri, w = q[3] * ri;
    const R p = p_fi(q, u, v, w);
    F[0] = q[1]; F[1] = q[1] * u + p; F[2] = q[1] * v; F[3] = q[1] * w; F[4] = u * (q[4] + p);
    F[5] = q[2]; F[6] = q[2] * u; F[7] = q[2] * v + p; F[8] = q[2] * w; F[9] = v * (q[4] + p);
    F[10] = q[3]; F[11] = q[3] * u; F[12] = q[3] * v; F[13] = q[3] * w + p; F[14] = w * (q[4] + p);
  }
  __device__ void flux1d(const R* q, R* f) const {  // euler.mojo:64-72
    R rho = rho_f(q), p = p_f(q, rho);
    R u = q[1] * pos_rcp(rho);
    f[0] = q[1]; f[1] = q[1] * u + p; f[2] = q[2] * u; f[3] = q[3] * u; f[4] = u * (q[4] + p);
  }
  __device__ void roe_avg(const R* ql, const R* qr, R pl, R pr, R& u, R& v, R& w, R& enth, R& a) const {
    R sl = pos_sqrt(rho_f(ql)), sr = pos_sqrt(rho_f(qr));  // euler.mojo:161-176
    const R il = pos_rcp(sl), ir = pos_rcp(sr), is = pos_rcp(sl + sr);
    u = (ql[1] * il + qr[1] * ir) * is;
    v = (ql[2] * il + qr[2] * ir) * is;
    w = (ql[3] * il + qr[3] * ir) * is;
    enth = ((ql[4] + pl) * il + (qr[4] + pr) * ir) * is;
    R aa2 = rmax((gamma - R(1)) * (enth - R(0.5) * (u * u + v * v + w * w)), R(0));
    a = sqrt(aa2);
  }
  __device__ void fluct(const R* s, const R* wv, R* amdq, R* apdq) const {  // euler.mojo:184-199
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      R am = R(0), ap = R(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        R t = s[k] * wv[m * 3 + k];
        if (s[k] < R(0)) am += t; else ap += t;
      }
      amdq[m] = am;
      apdq[m] = ap;
    }
  }
  __device__ void hh_fix(const R* ql, const R* qr, const R* s, const R* wv, R* amdq, R* apdq) const {  // euler.mojo:207-288
    R rl = rho_f(ql), pl = p_f(ql, rl);
    R s0 = ql[1] / rl - sqrt(gamma * pl / rl);
#pragma unroll
    for (int m = 0; m < 5; ++m) amdq[m] = R(0);
    if (!(s0 > R(0) && s[0] > R(0))) {
      R q10 = rmax(ql[0] + wv[0], rho_min);
      R q11 = ql[1] + wv[3], q12 = ql[2] + wv[6], q13 = ql[3] + wv[9], q14 = ql[4] + wv[12];
      R ke1 = R(0.5) * (q11 * q11 + q12 * q12 + q13 * q13) / q10;
      R p1 = rmax((gamma - R(1)) * (q14 - ke1), p_min);
      R s1 = q11 / q10 - sqrt(gamma * p1 / q10);
      R sf = (s0 < R(0) && s1 > R(0)) ? s0 * (s1 - s[0]) / (s1 - s0) : (s[0] < R(0) ? s[0] : R(0));
#pragma unroll
      for (int m = 0; m < 5; ++m) amdq[m] = sf * wv[m * 3 + 0];
      if (s[1] < R(0)) {
#pragma unroll
        for (int m = 0; m < 5; ++m) amdq[m] += s[1] * wv[m * 3 + 1];
        R rr = rho_f(qr), pr = p_f(qr, rr);
        R s3 = qr[1] / rr + sqrt(gamma * pr / rr);
        R q20 = rmax(qr[0] - wv[2], rho_min);
        R q21 = qr[1] - wv[5], q22 = qr[2] - wv[8], q23 = qr[3] - wv[11], q24 = qr[4] - wv[14];
        R ke2 = R(0.5) * (q21 * q21 + q22 * q22 + q23 * q23) / q20;
        R p2 = rmax((gamma - R(1)) * (q24 - ke2), p_min);
        R s2 = q21 / q20 + sqrt(gamma * p2 / q20);
        R sf2 = (s2 < R(0) && s3 > R(0)) ? s2 * (s3 - s[2]) / (s3 - s2) : (s[2] < R(0) ? s[2] : R(0));
#pragma unroll
        for (int m = 0; m < 5; ++m) amdq[m] += sf2 * wv[m * 3 + 2];
      }
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      R d = R(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) d += s[k] * wv[m * 3 + k];
      apdq[m] = d - amdq[m];
    }
  }
  // 1D Riemann problem in the face frame (rotated states): numerical flux rf.
  __device__ R solve1d(const R* ql, const R* qr, R* rf) const {
    if (FLUX == FLUX_RUSANOV) {  // euler.mojo:649-668
      R rhol = rho_f(ql), rhor = rho_f(qr), pl = p_f(ql, rhol), pr = p_f(qr, rhor);
      R cl = sqrt(gamma * pl / rhol), cr = sqrt(gamma * pr / rhor);
      R uxl = ql[1] / rhol, uxr = qr[1] / rhor;
      R cmax = rmax(rabs(uxl) + cl, rabs(uxr) + cr);
      rf[0] = R(0.5) * (ql[1] + qr[1] + cmax * (rhol - rhor));
      rf[1] = R(0.5) * (ql[1] * uxl + pl + qr[1] * uxr + pr + cmax * (ql[1] - qr[1]));
      rf[2] = R(0.5) * (ql[2] * uxl + qr[2] * uxr + cmax * (ql[2] - qr[2]));
      rf[3] = R(0.5) * (ql[3] * uxl + qr[3] * uxr + cmax * (ql[3] - qr[3]));
      rf[4] = R(0.5) * ((ql[4] + pl) * uxl + (qr[4] + pr) * uxr + cmax * (ql[4] - qr[4]));
      return cmax;
    } else {
      R s[3], wv[15], amdq[5], apdq[5];
      R pl = p_f(ql, rho_f(ql)), pr = p_f(qr, rho_f(qr));
      R u, v, w, enth, a;
      roe_avg(ql, qr, pl, pr, u, v, w, enth, a);
      if (FLUX == FLUX_ROE) {  // euler.mojo:296-361
        R g1 = gamma - R(1);
        R d0 = qr[0] - ql[0], d1 = qr[1] - ql[1], d2 = qr[2] - ql[2], d3 = qr[3] - ql[3], d4 = qr[4] - ql[4];
        R q2 = u * u + v * v + w * w;
        R g1a2 = g1 / (a * a);
        R euv = enth - q2;
        R a4 = g1a2 * (euv * d0 + u * d1 + v * d2 + w * d3 - d4);
        R a2 = d2 - v * d0, a3 = d3 - w * d0;
        R a5 = (d1 + (a - u) * d0 - a * a4) / (R(2) * a);
        R a1 = d0 - a4 - a5;
        wv[0] = a1; wv[3] = a1 * (u - a); wv[6] = a1 * v; wv[9] = a1 * w; wv[12] = a1 * (enth - u * a);
        wv[1] = a4; wv[4] = a4 * u; wv[7] = a4 * v + a2; wv[10] = a4 * w + a3;
        wv[13] = a4 * R(0.5) * q2 + a2 * v + a3 * w;
        wv[2] = a5; wv[5] = a5 * (u + a); wv[8] = a5 * v; wv[11] = a5 * w; wv[14] = a5 * (enth + u * a);
        s[0] = u - a; s[1] = u; s[2] = u + a;
      } else {
        R rl = rho_f(ql), irl = pos_rcp(rl), al = pos_sqrt(gamma * pl * irl), ul = ql[1] * irl;
        R rr = rho_f(qr), irr = pos_rcp(rr), ar = pos_sqrt(gamma * pr * irr), ur = qr[1] * irr;
        s[0] = rmin(ul - al, u - a);
        s[2] = rmax(ur + ar, u + a);
        if (FLUX == FLUX_HLLE) {  // euler.mojo:364-412
          s[1] = R(0);
          R fl[5], fr[5];
          flux1d(ql, fl);
          flux1d(qr, fr);
          const R iden = -pos_rcp(s[2] - s[0]);  // s[2] > s[0]: 1 / (s[0] - s[2])
#pragma unroll
          for (int m = 0; m < 5; ++m) {
            R qh = (fr[m] - fl[m] - s[2] * qr[m] + s[0] * ql[m]) * iden;
            wv[m * 3 + 0] = qh - ql[m];
            wv[m * 3 + 1] = R(0);
            wv[m * 3 + 2] = qr[m] - qh;
          }
        } else {  // HLLEC  euler.mojo:415-485
          s[1] = (pr - pl + rl * ul * (s[0] - ul) - rr * ur * (s[2] - ur)) / (rl * (s[0] - ul) - rr * (s[2] - ur));
          R lm = rl * (s[0] - ul) / (s[0] - s[1]);
          R hL[5] = {lm, lm * s[1], lm * ql[2] / rl, lm * ql[3] / rl,
                     lm * (ql[4] / rl + (s[1] - ul) * (s[1] + pl / (rl * (s[0] - ul))))};
          R rm = rr * (s[2] - ur) / (s[2] - s[1]);
          R hR[5] = {rm, rm * s[1], rm * qr[2] / rr, rm * qr[3] / rr,
                     rm * (qr[4] / rr + (s[1] - ur) * (s[1] + pr / (rr * (s[2] - ur))))};
#pragma unroll
          for (int m = 0; m < 5; ++m) {
            wv[m * 3 + 0] = hL[m] - ql[m];
            wv[m * 3 + 1] = hR[m] - hL[m];
            wv[m * 3 + 2] = qr[m] - hR[m];
          }
        }
      }
      if (entropy_fix) hh_fix(ql, qr, s, wv, amdq, apdq);
      else fluct(s, wv, amdq, apdq);
      R fl[5], fr[5];  // euler_flux_from_fluctuations  euler.mojo:495-520
      flux1d(ql, fl);
      flux1d(qr, fr);
#pragma unroll
      for (int m = 0; m < 5; ++m) rf[m] = R(0.5) * (fl[m] + fr[m]) - R(0.5) * (apdq[m] - amdq[m]);
      return rmax(rmax(rabs(s[0]), rabs(s[1])), rabs(s[2]));
    }
  }
  __device__ R num_flux(const R* q_l, const R* q_r, R nx, R ny, R nz, R* flux) const {  // euler.mojo:626-691
    if (FLUX == FLUX_RUSANOV) {
      // euler.mojo:649-668 evaluated in the world frame: with the orthonormal
      // frame (n, t, b), anti-rotating the face-frame Rusanov flux gives
      // 0.5 (m_L un_L + m_R un_R + (p_L + p_R) n + cmax (m_L - m_R)) for the
      // momentum, so the rotation pair and the tangent construction drop out.
      const R rl = rho_f(q_l), rr = rho_f(q_r), il = pos_rcp(rl), ir = pos_rcp(rr);
      const R pl = p_fi(q_l, q_l[1] * il, q_l[2] * il, q_l[3] * il);
      const R pr = p_fi(q_r, q_r[1] * ir, q_r[2] * ir, q_r[3] * ir);
      const R mnl = nx * q_l[1] + ny * q_l[2] + nz * q_l[3], mnr = nx * q_r[1] + ny * q_r[2] + nz * q_r[3];
      const R ul = mnl * il, ur = mnr * ir;
      const R cmax = rmax(rabs(ul) + pos_sqrt(gamma * pl * il), rabs(ur) + pos_sqrt(gamma * pr * ir));
      const R h = R(0.5), ps = pl + pr;
      flux[0] = h * (mnl + mnr + cmax * (rl - rr));
      flux[1] = h * (q_l[1] * ul + q_r[1] * ur + ps * nx + cmax * (q_l[1] - q_r[1]));
      flux[2] = h * (q_l[2] * ul + q_r[2] * ur + ps * ny + cmax * (q_l[2] - q_r[2]));
      flux[3] = h * (q_l[3] * ul + q_r[3] * ur + ps * nz + cmax * (q_l[3] - q_r[3]));
      flux[4] = h * ((q_l[4] + pl) * ul + (q_r[4] + pr) * ur + cmax * (q_l[4] - q_r[4]));
      return cmax;
    }
    // tangent/binormal (euler.mojo:94-118)
    R ax = nx, ay = ny, az = nz;
    if (rabs(nx) >= R(0.9)) ay += R(1); else ax += R(1);
    R pro = nx * ax + ny * ay + nz * az;
    ax -= nx * pro; ay -= ny * pro; az -= nz * pro;
    R mag = sqrt(ax * ax + ay * ay + az * az);
    R tx = ax / mag, ty = ay / mag, tz = az / mag;
    R bx = ny * tz - nz * ty, by = nz * tx - nx * tz, bz = nx * ty - ny * tx;
    R ql[5], qr[5], rf[5];
    ql[0] = q_l[0]; ql[4] = q_l[4];
    ql[1] = nx * q_l[1] + ny * q_l[2] + nz * q_l[3];
    ql[2] = tx * q_l[1] + ty * q_l[2] + tz * q_l[3];
    ql[3] = bx * q_l[1] + by * q_l[2] + bz * q_l[3];
    qr[0] = q_r[0]; qr[4] = q_r[4];
    qr[1] = nx * q_r[1] + ny * q_r[2] + nz * q_r[3];
    qr[2] = tx * q_r[1] + ty * q_r[2] + tz * q_r[3];
    qr[3] = bx * q_r[1] + by * q_r[2] + bz * q_r[3];
    R vmax = solve1d(ql, qr, rf);
    flux[0] = rf[0]; flux[4] = rf[4];
    flux[1] = nx * rf[1] + tx * rf[2] + bx * rf[3];
    flux[2] = ny * rf[1] + ty * rf[2] + by * rf[3];
    flux[3] = nz * rf[1] + tz * rf[2] + bz * rf[3];
    return vmax;
  }
  __device__ R bnd_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {  // euler.mojo:705-730
    R g[5];
    ghost(q, bc, nx, ny, nz, g);
    return num_flux(q, g, nx, ny, nz, f);
  }
  __device__ void ghost(const R* q, int bc, R nx, R ny, R nz, R* g) const {
    if (bc == BC_WALL) {
      R mn = q[1] * nx + q[2] * ny + q[3] * nz;
      g[0] = q[0]; g[4] = q[4];
      g[1] = q[1] - R(2) * mn * nx; g[2] = q[2] - R(2) * mn * ny; g[3] = q[3] - R(2) * mn * nz;
    } else if (bc == BC_INFLOW) {
#pragma unroll
      for (int c = 0; c < 5; ++c) g[c] = inflow[c];
    } else {
#pragma unroll
      for (int c = 0; c < 5; ++c) g[c] = q[c];
    }
  }
  __device__ void source(const R* q, R* s) const {  // euler.mojo:738-747
    s[0] = R(0);
    s[1] = q[0] * gx;
    s[2] = q[0] * gy;
    s[3] = q[0] * gz;
    s[4] = q[1] * gx + q[2] * gy + q[3] * gz;
  }
  // Positivity floor after the RK write.  The pressure recovery
  // p = (gamma - 1)(E - |m|^2 / 2 rho) runs in FP64 for every state type:
  // near vacuum E and the kinetic energy cancel, and an FP32 difference
  // would decide the floor on rounding noise.
  __device__ void limit(R* q) const {  // euler.mojo:758-792
    if constexpr (sizeof(R) == 4) {
      // Fast accept in FP32 for the common case far from the floors: with
      // rho above rho_min, a = E rho and b = |m|^2 / 2 rounded in FP32 (each
      // within a few ulps, b a sum of non-negative terms) and d = a - b,
      // |d - (E rho - |m|^2 / 2)| <= 4 * 2^-24 (a + b); when (gamma - 1) d
      // clears p_min rho by (gamma - 1) 1e-6 (a + b) plus 0.1 % of p_min rho
      // (the products' own rounding), the FP64 test below passes and would
      // leave q unchanged.  NaNs fail the comparisons and take the FP64 path.
      const float r = q[0];
      if (r > rho_min) {
        const float a = q[4] * r, bb = 0.5f * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        const float g1 = gamma - 1.0f;
        if (g1 * (a - bb) > 1.001f * (p_min * r) + 1.0e-6f * g1 * (a + bb)) return;
      }
    }
    const double rho = double(q[0]), g1 = double(gamma) - 1.0, pm = double(p_min);
    if (!(rho > double(rho_min))) {
      q[0] = rho_min; q[1] = R(0); q[2] = R(0); q[3] = R(0);
      q[4] = R(pm / g1);
      return;
    }
    const double m1 = double(q[1]), m2_ = double(q[2]), m3 = double(q[3]);
    const double m2 = m1 * m1 + m2_ * m2_ + m3 * m3;
    if (!(m2 >= 0.0)) {
      q[1] = R(0); q[2] = R(0); q[3] = R(0);
      q[4] = R(pm / g1);
      return;
    }
    // p > pm  <=>  g1 (E rho - m2 / 2) > pm rho  (rho > 0): the test needs no
    // FP64 division; the floored energy is formed as before
    if (!(g1 * (double(q[4]) * rho - 0.5 * m2) > pm * rho)) q[4] = R(0.5 * m2 * (1.0 / rho) + pm / g1);
  }
};

// -------------------------------------------------------------------- maxwell
template <class R>
struct MaxwellD {
  static constexpr int NC = 6;
  static constexpr bool kSource = true, kLimit = false;
  static constexpr bool kLightFlux = true;
  R c, J[3], M[3], inflow[6];
  __device__ void flux(const R* q, R* F) const {  // maxwell.mojo:127-156
    R c2 = c * c;
    F[0] = R(0); F[1] = c2 * q[5]; F[2] = -c2 * q[4]; F[3] = R(0); F[4] = -q[2]; F[5] = q[1];
    F[6] = -c2 * q[5]; F[7] = R(0); F[8] = c2 * q[3]; F[9] = q[2]; F[10] = R(0); F[11] = -q[0];
    F[12] = c2 * q[4]; F[13] = -c2 * q[3]; F[14] = R(0); F[15] = -q[1]; F[16] = q[0]; F[17] = R(0);
  }
  __device__ R num_flux(const R* l, const R* r, R nx, R ny, R nz, R* f) const {  // maxwell.mojo:161-207
    R c2 = c * c, h = R(0.5);
    f[0] = h * (c2 * (l[4] * nz - l[5] * ny) + c2 * (r[4] * nz - r[5] * ny)) - h * c * (r[0] - l[0]);
    f[1] = h * (c2 * (l[5] * nx - l[3] * nz) + c2 * (r[5] * nx - r[3] * nz)) - h * c * (r[1] - l[1]);
    f[2] = h * (c2 * (l[3] * ny - l[4] * nx) + c2 * (r[3] * ny - r[4] * nx)) - h * c * (r[2] - l[2]);
    f[3] = h * ((ny * l[2] - nz * l[1]) + (ny * r[2] - nz * r[1])) - h * c * (r[3] - l[3]);
    f[4] = h * ((nz * l[0] - nx * l[2]) + (nz * r[0] - nx * r[2])) - h * c * (r[4] - l[4]);
    f[5] = h * ((nx * l[1] - ny * l[0]) + (nx * r[1] - ny * r[0])) - h * c * (r[5] - l[5]);
    return c;
  }
  __device__ R bnd_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {  // maxwell.mojo:213-240
    R g[6];
    ghost(q, bc, nx, ny, nz, g);
    return num_flux(q, g, nx, ny, nz, f);
  }
  __device__ void ghost(const R* q, int bc, R nx, R ny, R nz, R* g) const {
    if (bc == BC_WALL) {
      R En = q[0] * nx + q[1] * ny + q[2] * nz, Bn = q[3] * nx + q[4] * ny + q[5] * nz;
      g[0] = R(2) * En * nx - q[0]; g[1] = R(2) * En * ny - q[1]; g[2] = R(2) * En * nz - q[2];
      g[3] = q[3] - R(2) * Bn * nx; g[4] = q[4] - R(2) * Bn * ny; g[5] = q[5] - R(2) * Bn * nz;
    } else if (bc == BC_INFLOW) {
#pragma unroll
      for (int k = 0; k < 6; ++k) g[k] = inflow[k];
    } else {
#pragma unroll
      for (int k = 0; k < 6; ++k) g[k] = q[k];
    }
  }
  __device__ void source(const R*, R* s) const {  // maxwell.mojo:245-252
    R c2 = c * c;
    s[0] = -c2 * J[0]; s[1] = -c2 * J[1]; s[2] = -c2 * J[2];
    s[3] = -M[0]; s[4] = -M[1]; s[5] = -M[2];
  }
  __device__ void limit(R*) const {}
};

// -------------------------------------------------------------- shallow water
template <class R>
struct ShallowWaterD {
  static constexpr int NC = 3;
  static constexpr bool kSource = false, kLimit = false;
  static constexpr bool kLightFlux = true;
  R g, h_min, inflow[3];
  __device__ void flux(const R* q, R* F) const {  // shallow_water.mojo:63-86
    R h = q[0] > h_min ? q[0] : h_min;
    R u = q[1] / h, v = q[2] / h, gh = R(0.5) * g * h * h;
    F[0] = q[1]; F[1] = q[1] * u + gh; F[2] = q[1] * v;
    F[3] = q[2]; F[4] = q[1] * v; F[5] = q[2] * v + gh;
    F[6] = R(0); F[7] = R(0); F[8] = R(0);
  }
  __device__ R num_flux(const R* l, const R* r, R nx, R ny, R, R* f) const {  // shallow_water.mojo:90-134
    R hl = l[0] > h_min ? l[0] : h_min, hr = r[0] > h_min ? r[0] : h_min;
    R ul = l[1] / hl, vl = l[2] / hl, ur = r[1] / hr, vr = r[2] / hr;
    R unl = ul * nx + vl * ny, unr = ur * nx + vr * ny;
    R cl = sqrt(g * hl), cr = sqrt(g * hr);
    R gl = R(0.5) * g * hl * hl, gr = R(0.5) * g * hr * hr;
    R al = rmax(rabs(unl) + cl, rabs(unr) + cr), h = R(0.5);
    f[0] = h * ((l[1] * nx + l[2] * ny) + (r[1] * nx + r[2] * ny)) - h * al * (r[0] - l[0]);
    f[1] = h * ((l[1] * unl + gl * nx) + (r[1] * unr + gr * nx)) - h * al * (r[1] - l[1]);
    f[2] = h * ((l[2] * unl + gl * ny) + (r[2] * unr + gr * ny)) - h * al * (r[2] - l[2]);
    return al;
  }
  __device__ R bnd_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {  // shallow_water.mojo:138-156
    R gs[3];
    ghost(q, bc, nx, ny, nz, gs);
    return num_flux(q, gs, nx, ny, nz, f);
  }
  __device__ void ghost(const R* q, int bc, R nx, R ny, R, R* gs) const {
    if (bc == BC_WALL) {
      R mn = q[1] * nx + q[2] * ny;
      gs[0] = q[0]; gs[1] = q[1] - R(2) * mn * nx; gs[2] = q[2] - R(2) * mn * ny;
    } else if (bc == BC_INFLOW) {
      gs[0] = inflow[0]; gs[1] = inflow[1]; gs[2] = inflow[2];
    } else {
      gs[0] = q[0]; gs[1] = q[1]; gs[2] = q[2];
    }
  }
  __device__ void source(const R*, R* s) const { s[0] = s[1] = s[2] = R(0); }
  __device__ void limit(R*) const {}
};

// ------------------------------------------------------------------ ideal MHD
// q = [rho, rho u, rho v, rho w, E, Bx, By, Bz, psi]; Dedner GLM cleaning
// (psi carries div B at speed c_h and decays at rate alpha_d).
template <class R>
struct MhdD {
  static constexpr int NC = 9;
  static constexpr bool kSource = true, kLimit = false;
  static constexpr bool kLightFlux = true;
  R gamma, rho_min, p_min, c_h, alpha_d, inflow[9];

  __device__ __forceinline__ R rho_f(const R* q) const { return q[0] > rho_min ? q[0] : rho_min; }  // mhd.mojo:46-48
  // floored gas pressure from ri = 1 / rho (mhd.mojo:51-62)
  __device__ __forceinline__ R p_gas(const R* q, R ri) const {
    const R ke = R(0.5) * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) * ri;
    const R me = R(0.5) * (q[5] * q[5] + q[6] * q[6] + q[7] * q[7]);
    const R p = (gamma - R(1)) * (q[4] - ke - me);
    return p > p_min ? p : p_min;
  }
  // fast magnetosonic speed along n (mhd.mojo:71-85)
  __device__ __forceinline__ R fast_speed(const R* q, R ri, R p, R nx, R ny, R nz) const {
    const R bx = q[5], by = q[6], bz = q[7], bn = bx * nx + by * ny + bz * nz;
    const R cs2 = gamma * p * ri, ca2 = (bx * bx + by * by + bz * bz) * ri, can2 = (bn * bn) * ri;
    R disc = (cs2 + ca2) * (cs2 + ca2) - R(4) * cs2 * can2;
    if (disc < R(0)) disc = R(0);
    return sqrt(R(0.5) * (cs2 + ca2 + sqrt(disc)));
  }
  __device__ void flux(const R* q, R* F) const {  // mhd.mojo:92-146
    const R ri = pos_rcp(rho_f(q));
    const R mx = q[1], my = q[2], mz = q[3], u = mx * ri, v = my * ri, w = mz * ri;
    const R E = q[4], bx = q[5], by = q[6], bz = q[7], psi = q[8];
    const R pt = p_gas(q, ri) + R(0.5) * (bx * bx + by * by + bz * bz);
    const R ub = u * bx + v * by + w * bz, ch2 = c_h * c_h;
    F[0] = mx; F[1] = mx * u + pt - bx * bx; F[2] = mx * v - bx * by; F[3] = mx * w - bx * bz;
    F[4] = u * (E + pt) - bx * ub; F[5] = psi; F[6] = u * by - v * bx; F[7] = u * bz - w * bx; F[8] = ch2 * bx;
    F[9] = my; F[10] = my * u - by * bx; F[11] = my * v + pt - by * by; F[12] = my * w - by * bz;
    F[13] = v * (E + pt) - by * ub; F[14] = v * bx - u * by; F[15] = psi; F[16] = v * bz - w * by; F[17] = ch2 * by;
    F[18] = mz; F[19] = mz * u - bz * bx; F[20] = mz * v - bz * by; F[21] = mz * w + pt - bz * bz;
    F[22] = w * (E + pt) - bz * ub; F[23] = w * bx - u * bz; F[24] = w * by - v * bz; F[25] = psi; F[26] = ch2 * bz;
  }
  // F . n of one state (mhd.mojo:151-194)
  __device__ __forceinline__ void normal_flux(const R* q, R ri, R p, R nx, R ny, R nz, R* F) const {
    const R rho = rho_f(q), u = q[1] * ri, v = q[2] * ri, w = q[3] * ri;
    const R E = q[4], bx = q[5], by = q[6], bz = q[7], psi = q[8];
    const R pt = p + R(0.5) * (bx * bx + by * by + bz * bz);
    const R ub = u * bx + v * by + w * bz, un = u * nx + v * ny + w * nz, bn = bx * nx + by * ny + bz * nz;
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
  // Rusanov with alpha = max(|u_n| + c_f, c_h) (mhd.mojo:280-307)
  __device__ R num_flux(const R* l, const R* r, R nx, R ny, R nz, R* f) const {
    const R il = pos_rcp(rho_f(l)), ir = pos_rcp(rho_f(r));
    const R pl = p_gas(l, il), pr = p_gas(r, ir);
    R Fl[9], Fr[9];
    normal_flux(l, il, pl, nx, ny, nz, Fl);
    normal_flux(r, ir, pr, nx, ny, nz, Fr);
    const R cfl = fast_speed(l, il, pl, nx, ny, nz), cfr = fast_speed(r, ir, pr, nx, ny, nz);
    const R unl = (l[1] * nx + l[2] * ny + l[3] * nz) * il, unr = (r[1] * nx + r[2] * ny + r[3] * nz) * ir;
    const R al = rmax(rmax(rabs(unl) + cfl, rabs(unr) + cfr), c_h), h = R(0.5);
#pragma unroll
    for (int c = 0; c < 9; ++c) f[c] = h * (Fl[c] + Fr[c]) - h * al * (r[c] - l[c]);
    return al;
  }
  // ghost state: conducting wall reflects u_n and B_n; inflow; outflow copies (mhd.mojo:312-353)
  __device__ void ghost(const R* q, int bc, R nx, R ny, R nz, R* g) const {
    if (bc == BC_WALL) {
      const R mn = q[1] * nx + q[2] * ny + q[3] * nz, bn = q[5] * nx + q[6] * ny + q[7] * nz;
      g[0] = q[0]; g[4] = q[4]; g[8] = q[8];
      g[1] = q[1] - R(2) * mn * nx; g[2] = q[2] - R(2) * mn * ny; g[3] = q[3] - R(2) * mn * nz;
      g[5] = q[5] - R(2) * bn * nx; g[6] = q[6] - R(2) * bn * ny; g[7] = q[7] - R(2) * bn * nz;
    } else if (bc == BC_INFLOW) {
#pragma unroll
      for (int k = 0; k < 9; ++k) g[k] = inflow[k];
    } else {
#pragma unroll
      for (int k = 0; k < 9; ++k) g[k] = q[k];
    }
  }
  __device__ R bnd_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {
    R g[9];
    ghost(q, bc, nx, ny, nz, g);
    return num_flux(q, g, nx, ny, nz, f);
  }
  __device__ void source(const R* q, R* s) const {  // mhd.mojo:357-361: GLM damping of psi
#pragma unroll
    for (int c = 0; c < 8; ++c) s[c] = R(0);
    s[8] = -alpha_d * q[8];
  }
  __device__ void limit(R*) const {}
};

// ----------------------------------------------------------- five-moment two-fluid
// q[0..4] electrons (rho, m, E), q[5..9] ions, q[10..15] (E, B), q[16] psi;
// fluids couple to the field only through the source (Lorentz force, work,
// Ampere current), the GLM psi cleans div B.
template <class R>
struct TwoFluidD {
  static constexpr int NC = 17;
  static constexpr bool kSource = true, kLimit = false;
  static constexpr bool kLightFlux = true;
  R gamma_e, gamma_i, q_e, m_e, q_i, m_i, eps0, c_light, c_h, alpha_d, rho_min, p_min, inflow[17];

  __device__ __forceinline__ R rho_f(const R* s) const { return s[0] > rho_min ? s[0] : rho_min; }  // two_fluid.mojo:52-54
  // floored species pressure from ri = 1 / rho (two_fluid.mojo:57-65)
  __device__ __forceinline__ R p_s(const R* s, R g, R ri) const {
    const R p = (g - R(1)) * (s[4] - R(0.5) * (s[1] * s[1] + s[2] * s[2] + s[3] * s[3]) * ri);
    return p > p_min ? p : p_min;
  }
  __device__ __forceinline__ void species_flux(const R* s, R g, R* F) const {  // two_fluid.mojo:76-101 (F[d*NC + c])
    const R ri = pos_rcp(rho_f(s)), u = s[1] * ri, v = s[2] * ri, w = s[3] * ri, p = p_s(s, g, ri);
    F[0] = s[1]; F[1] = s[1] * u + p; F[2] = s[1] * v; F[3] = s[1] * w; F[4] = u * (s[4] + p);
    F[NC + 0] = s[2]; F[NC + 1] = s[2] * u; F[NC + 2] = s[2] * v + p; F[NC + 3] = s[2] * w; F[NC + 4] = v * (s[4] + p);
    F[2 * NC + 0] = s[3]; F[2 * NC + 1] = s[3] * u; F[2 * NC + 2] = s[3] * v; F[2 * NC + 3] = s[3] * w + p;
    F[2 * NC + 4] = w * (s[4] + p);
  }
  __device__ void flux(const R* q, R* F) const {  // two_fluid.mojo:258-305
    species_flux(q, gamma_e, F);
    species_flux(q + 5, gamma_i, F + 5);
    const R c2 = c_light * c_light, ch2 = c_h * c_h;
    const R Ex = q[10], Ey = q[11], Ez = q[12], Bx = q[13], By = q[14], Bz = q[15], psi = q[16];
    F[10] = R(0); F[11] = c2 * Bz; F[12] = -c2 * By; F[13] = psi; F[14] = -Ez; F[15] = Ey; F[16] = ch2 * Bx;
    F[NC + 10] = -c2 * Bz; F[NC + 11] = R(0); F[NC + 12] = c2 * Bx; F[NC + 13] = Ez; F[NC + 14] = psi;
    F[NC + 15] = -Ex; F[NC + 16] = ch2 * By;
    F[2 * NC + 10] = c2 * By; F[2 * NC + 11] = -c2 * Bx; F[2 * NC + 12] = R(0); F[2 * NC + 13] = -Ey;
    F[2 * NC + 14] = Ex; F[2 * NC + 15] = psi; F[2 * NC + 16] = ch2 * Bz;
  }
  // species F.n and Rusanov speed |u.n| + c_s (two_fluid.mojo:107-132, :349-366)
  __device__ __forceinline__ R species_normal(const R* s, R g, R nx, R ny, R nz, R* F) const {
    const R rho = rho_f(s), ri = pos_rcp(rho), u = s[1] * ri, v = s[2] * ri, w = s[3] * ri, p = p_s(s, g, ri);
    const R un = u * nx + v * ny + w * nz;
    F[0] = rho * un; F[1] = rho * u * un + p * nx; F[2] = rho * v * un + p * ny; F[3] = rho * w * un + p * nz;
    F[4] = un * (s[4] + p);
    const R unm = (s[1] * nx + s[2] * ny + s[3] * nz) * ri;
    return rabs(unm) + sqrt(g * p * ri);
  }
  __device__ __forceinline__ void field_normal(const R* q, R nx, R ny, R nz, R* F) const {  // :329-347
    const R c2 = c_light * c_light, ch2 = c_h * c_h;
    const R Ex = q[10], Ey = q[11], Ez = q[12], Bx = q[13], By = q[14], Bz = q[15], psi = q[16];
    F[10] = c2 * (By * nz - Bz * ny); F[11] = c2 * (Bz * nx - Bx * nz); F[12] = c2 * (Bx * ny - By * nx);
    F[13] = (ny * Ez - nz * Ey) + psi * nx; F[14] = (nz * Ex - nx * Ez) + psi * ny;
    F[15] = (nx * Ey - ny * Ex) + psi * nz; F[16] = ch2 * (Bx * nx + By * ny + Bz * nz);
  }
  // Rusanov: alpha = max(fluid speeds of both sides, c, c_h) (two_fluid.mojo:307-374)
  __device__ R num_flux(const R* l, const R* r, R nx, R ny, R nz, R* f) const {
    R Fl[17], Fr[17];
    const R ael = species_normal(l, gamma_e, nx, ny, nz, Fl), aer = species_normal(r, gamma_e, nx, ny, nz, Fr);
    const R ail = species_normal(l + 5, gamma_i, nx, ny, nz, Fl + 5), air = species_normal(r + 5, gamma_i, nx, ny, nz, Fr + 5);
    field_normal(l, nx, ny, nz, Fl);
    field_normal(r, nx, ny, nz, Fr);
    const R al = rmax(rmax(rmax(ael, aer), rmax(ail, air)), rmax(c_light, c_h)), h = R(0.5);
#pragma unroll
    for (int c = 0; c < 17; ++c) f[c] = h * (Fl[c] + Fr[c]) - h * al * (r[c] - l[c]);
    return al;
  }
  // wall: slip for both fluids, PEC for the field (two_fluid.mojo:376-428)
  __device__ void ghost(const R* q, int bc, R nx, R ny, R nz, R* g) const {
    if (bc == BC_INFLOW) {
#pragma unroll
      for (int k = 0; k < 17; ++k) g[k] = inflow[k];
      return;
    }
#pragma unroll
    for (int k = 0; k < 17; ++k) g[k] = q[k];
    if (bc == BC_WALL) {
      const R me = q[1] * nx + q[2] * ny + q[3] * nz, mi = q[6] * nx + q[7] * ny + q[8] * nz;
      g[1] = q[1] - R(2) * me * nx; g[2] = q[2] - R(2) * me * ny; g[3] = q[3] - R(2) * me * nz;
      g[6] = q[6] - R(2) * mi * nx; g[7] = q[7] - R(2) * mi * ny; g[8] = q[8] - R(2) * mi * nz;
      const R En = q[10] * nx + q[11] * ny + q[12] * nz, Bn = q[13] * nx + q[14] * ny + q[15] * nz;
      g[10] = R(2) * En * nx - q[10]; g[11] = R(2) * En * ny - q[11]; g[12] = R(2) * En * nz - q[12];
      g[13] = q[13] - R(2) * Bn * nx; g[14] = q[14] - R(2) * Bn * ny; g[15] = q[15] - R(2) * Bn * nz;
    }
  }
  __device__ R bnd_flux(const R* q, int bc, R nx, R ny, R nz, R* f) const {
    R g[17];
    ghost(q, bc, nx, ny, nz, g);
    return num_flux(q, g, nx, ny, nz, f);
  }
  __device__ void source(const R* q, R* s) const {  // two_fluid.mojo:430-510
    const R ie = pos_rcp(rho_f(q)), ii = pos_rcp(rho_f(q + 5));
    const R rho_e = rho_f(q), rho_i = rho_f(q + 5);
    const R ue = q[1] * ie, ve = q[2] * ie, we = q[3] * ie, ui = q[6] * ii, vi = q[7] * ii, wi = q[8] * ii;
    const R Ex = q[10], Ey = q[11], Ez = q[12], Bx = q[13], By = q[14], Bz = q[15];
    const R qme = q_e / m_e, qmi = q_i / m_i;
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
    const R ie0 = R(1) / eps0;
    s[10] = -(qme * rho_e * ue + qmi * rho_i * ui) * ie0;
    s[11] = -(qme * rho_e * ve + qmi * rho_i * vi) * ie0;
    s[12] = -(qme * rho_e * we + qmi * rho_i * wi) * ie0;
    s[13] = R(0); s[14] = R(0); s[15] = R(0);
    s[16] = -alpha_d * q[16];
  }
  __device__ void limit(R*) const {}
};

}  // namespace mxm
