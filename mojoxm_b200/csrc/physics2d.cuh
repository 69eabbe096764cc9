// Device physics of mojoxm's 2D triangle kernels.  Unlike 3D these are not
// routed through the Physics trait: each has its own volume-flux floors and
// face-flux formula (ghost states built inside the face kernel).
//   Euler   src/local_mesh_2d_gpu_euler.mojo:33-144 (vol), :220-337 (Rusanov,
//           alpha = |v| + c), :392-545 (HLLC); HLLE = the 3D euler_hlle_solver on
//           the state embedded with w = 0, n_z = 0 (src/euler.mojo:364-412)
//   SW      src/local_mesh_2d_gpu_sw.mojo:27-176 (vol), :178-306 (Rusanov), :308-450 (HLL)
//   Maxwell src/local_mesh_2d_gpu_maxwell.mojo:31-218 (vol), :219-377 (Rusanov + PEC)
//   Advect. src/local_mesh_2d_gpu_advection.mojo:117-182 (vol), :249-300 (upwind)
//   MHD     src/local_mesh_2d_gpu_mhd.mojo (6 components, no cleaning) and
//           src/local_mesh_2d_gpu_mhd_glm.mojo (7, GLM psi; psi damping is
//           operator-split per SSPRK3 step, outside the stage)
#pragma once
#include "physics.cuh"

namespace mxm {

template <class R>
struct Advection2D {
  static constexpr int NC = 1;
  static constexpr bool kSource = false;
  R vx, vy, inflow_q;
  __device__ void flux(const R* q, R* Fx, R* Fy) const {
    Fx[0] = vx * q[0];
    Fy[0] = vy * q[0];
  }
  __device__ void face(const R* qL, const R* qR, int bc, R nx, R ny, R* f) const {
    R vn = vx * nx + vy * ny;
    if (vn >= R(0)) f[0] = vn * qL[0];
    else if (bc == BC_INTERIOR) f[0] = vn * qR[0];
    else if (bc == BC_INFLOW) f[0] = vn * inflow_q;
    else f[0] = R(0);
  }
  __device__ void source(const R*, R* s) const { s[0] = R(0); }
  __device__ R speed(const R*) const { return sqrt(vx * vx + vy * vy); }
};

template <class R, int FLUX>
struct Euler2D {
  static constexpr int NC = 4;
  static constexpr bool kSource = true;
  R gamma, rho_min, p_min, gx, gy;
  R inflow[4];
  int entropy_fix;
  __device__ void flux(const R* q, R* Fx, R* Fy) const {
    R rho = q[0];
    if (rho < rho_min) rho = rho_min;
    R u = q[1] / rho, v = q[2] / rho;
    R p = (gamma - R(1)) * (q[3] - R(0.5) * rho * (u * u + v * v));
    if (p < p_min) p = p_min;
    Fx[0] = q[1]; Fx[1] = q[1] * u + p; Fx[2] = q[1] * v; Fx[3] = u * (q[3] + p);
    Fy[0] = q[2]; Fy[1] = q[2] * u; Fy[2] = q[2] * v + p; Fy[3] = v * (q[3] + p);
  }
  __device__ void ghost(const R* qL, int bc, R nx, R ny, R* g) const {
    if (bc == BC_WALL) {
      R mn = qL[1] * nx + qL[2] * ny;
      g[0] = qL[0]; g[1] = qL[1] - R(2) * mn * nx; g[2] = qL[2] - R(2) * mn * ny; g[3] = qL[3];
    } else if (bc == BC_INFLOW) {
      g[0] = inflow[0]; g[1] = inflow[1]; g[2] = inflow[2]; g[3] = inflow[3];
    } else {
      g[0] = qL[0]; g[1] = qL[1]; g[2] = qL[2]; g[3] = qL[3];
    }
  }
  __device__ void face(const R* qL, const R* qRin, int bc, R nx, R ny, R* f) const {
    R qR[4];
    if (bc == BC_INTERIOR) { qR[0] = qRin[0]; qR[1] = qRin[1]; qR[2] = qRin[2]; qR[3] = qRin[3]; }
    else ghost(qL, bc, nx, ny, qR);
    if (FLUX == FLUX_HLLE) {
      EulerD<R, FLUX_HLLE> e3;
      e3.gamma = gamma; e3.rho_min = rho_min; e3.p_min = p_min; e3.entropy_fix = entropy_fix;
      e3.gx = e3.gy = e3.gz = R(0);
      R l3[5] = {qL[0], qL[1], qL[2], R(0), qL[3]}, r3[5] = {qR[0], qR[1], qR[2], R(0), qR[3]}, f3[5];
      e3.num_flux(l3, r3, nx, ny, R(0), f3);
      f[0] = f3[0]; f[1] = f3[1]; f[2] = f3[2]; f[3] = f3[4];
      return;
    }
    R rL = qL[0] < rho_min ? rho_min : qL[0];
    R rR = qR[0] < rho_min ? rho_min : qR[0];
    R uL = qL[1] / rL, vL = qL[2] / rL, uR = qR[1] / rR, vR = qR[2] / rR;
    R pL = (gamma - R(1)) * (qL[3] - R(0.5) * rL * (uL * uL + vL * vL));
    if (pL < p_min) pL = p_min;
    R pR = (gamma - R(1)) * (qR[3] - R(0.5) * rR * (uR * uR + vR * vR));
    if (pR < p_min) pR = p_min;
    if (FLUX == FLUX_HLLC) {
      R aL = sqrt(gamma * pL / rL), aR = sqrt(gamma * pR / rR);
      R unL = uL * nx + vL * ny, unR = uR * nx + vR * ny;
      R FnL[4] = {qL[1] * nx + qL[2] * ny, (qL[1] * uL + pL) * nx + (qL[1] * vL) * ny,
                  (qL[1] * vL) * nx + (qL[2] * vL + pL) * ny, (uL * (qL[3] + pL)) * nx + (vL * (qL[3] + pL)) * ny};
      R FnR[4] = {qR[1] * nx + qR[2] * ny, (qR[1] * uR + pR) * nx + (qR[1] * vR) * ny,
                  (qR[1] * vR) * nx + (qR[2] * vR + pR) * ny, (uR * (qR[3] + pR)) * nx + (vR * (qR[3] + pR)) * ny};
      R SL = unL - aL, tt = unR - aR;
      if (tt < SL) SL = tt;
      R SR = unL + aL;
      tt = unR + aR;
      if (tt > SR) SR = tt;
      R Ss = (pR - pL + rL * unL * (SL - unL) - rR * unR * (SR - unR)) / (rL * (SL - unL) - rR * (SR - unR));
      if (SL >= R(0)) {
#pragma unroll
        for (int k = 0; k < 4; ++k) f[k] = FnL[k];
      } else if (SR <= R(0)) {
#pragma unroll
        for (int k = 0; k < 4; ++k) f[k] = FnR[k];
      } else if (Ss >= R(0)) {
        R co = (SL - unL) / (SL - Ss), rs = rL * co;
        R us = uL + (Ss - unL) * nx, vs = vL + (Ss - unL) * ny;
        R Es = qL[3] / rL + (Ss - unL) * (Ss + pL / (rL * (SL - unL)));
        f[0] = FnL[0] + SL * (rs - qL[0]);
        f[1] = FnL[1] + SL * (rs * us - qL[1]);
        f[2] = FnL[2] + SL * (rs * vs - qL[2]);
        f[3] = FnL[3] + SL * (rs * Es - qL[3]);
      } else {
        R co = (SR - unR) / (SR - Ss), rs = rR * co;
        R us = uR + (Ss - unR) * nx, vs = vR + (Ss - unR) * ny;
        R Es = qR[3] / rR + (Ss - unR) * (Ss + pR / (rR * (SR - unR)));
        f[0] = FnR[0] + SR * (rs - qR[0]);
        f[1] = FnR[1] + SR * (rs * us - qR[1]);
        f[2] = FnR[2] + SR * (rs * vs - qR[2]);
        f[3] = FnR[3] + SR * (rs * Es - qR[3]);
      }
      return;
    }
    // Rusanov with alpha = max(|v| + c)
    R sL = sqrt(uL * uL + vL * vL) + sqrt(gamma * pL / rL);
    R sR = sqrt(uR * uR + vR * vR) + sqrt(gamma * pR / rR);
    R FxL[4] = {qL[1], qL[1] * uL + pL, qL[1] * vL, uL * (qL[3] + pL)};
    R FyL[4] = {qL[2], qL[2] * uL, qL[2] * vL + pL, vL * (qL[3] + pL)};
    R FxR[4] = {qR[1], qR[1] * uR + pR, qR[1] * vR, uR * (qR[3] + pR)};
    R FyR[4] = {qR[2], qR[2] * uR, qR[2] * vR + pR, vR * (qR[3] + pR)};
    R al = sL > sR ? sL : sR, h = R(0.5);
#pragma unroll
    for (int k = 0; k < 4; ++k) f[k] = h * ((FxL[k] + FxR[k]) * nx + (FyL[k] + FyR[k]) * ny) - h * al * (qR[k] - qL[k]);
  }
  __device__ void source(const R* q, R* s) const {
    R rho = q[0];
    if (rho < rho_min) rho = rho_min;
    s[0] = R(0);
    s[1] = rho * gx;
    s[2] = rho * gy;
    s[3] = q[1] * gx + q[2] * gy;
  }
  // nodal signal speed |v| + c with the volume-kernel floors
  __device__ R speed(const R* q) const {
    R rho = q[0] < rho_min ? rho_min : q[0];
    R u = q[1] / rho, v = q[2] / rho;
    R p = (gamma - R(1)) * (q[3] - R(0.5) * rho * (u * u + v * v));
    if (p < p_min) p = p_min;
    return sqrt(u * u + v * v) + sqrt(gamma * p / rho);
  }
};

template <class R, int FLUX>
struct ShallowWater2D {
  static constexpr int NC = 3;
  static constexpr bool kSource = false;
  R g, h_min, inflow[3];
  __device__ void flux(const R* q, R* Fx, R* Fy) const {
    R h = q[0];
    if (h < h_min) h = h_min;
    R u = q[1] / h, v = q[2] / h, p = R(0.5) * g * h * h;
    Fx[0] = q[1]; Fx[1] = q[1] * u + p; Fx[2] = q[1] * v;
    Fy[0] = q[2]; Fy[1] = q[2] * u; Fy[2] = q[2] * v + p;
  }
  __device__ void face(const R* qL, const R* qRin, int bc, R nx, R ny, R* f) const {
    R qR[3];
    if (bc == BC_INTERIOR) { qR[0] = qRin[0]; qR[1] = qRin[1]; qR[2] = qRin[2]; }
    else if (bc == BC_WALL) {
      R mn = qL[1] * nx + qL[2] * ny;
      qR[0] = qL[0]; qR[1] = qL[1] - R(2) * mn * nx; qR[2] = qL[2] - R(2) * mn * ny;
    } else if (bc == BC_INFLOW) { qR[0] = inflow[0]; qR[1] = inflow[1]; qR[2] = inflow[2]; }
    else { qR[0] = qL[0]; qR[1] = qL[1]; qR[2] = qL[2]; }
    R hL = qL[0] < h_min ? h_min : qL[0], hR = qR[0] < h_min ? h_min : qR[0];
    R uL = qL[1] / hL, vL = qL[2] / hL, uR = qR[1] / hR, vR = qR[2] / hR;
    R pL = R(0.5) * g * hL * hL, pR = R(0.5) * g * hR * hR;
    R cL = sqrt(g * hL), cR = sqrt(g * hR);
    R FxL[3] = {qL[1], qL[1] * uL + pL, qL[1] * vL}, FyL[3] = {qL[2], qL[2] * uL, qL[2] * vL + pL};
    R FxR[3] = {qR[1], qR[1] * uR + pR, qR[1] * vR}, FyR[3] = {qR[2], qR[2] * uR, qR[2] * vR + pR};
    if (FLUX == FLUX_HLL) {
      R unL = uL * nx + vL * ny, unR = uR * nx + vR * ny;
      R SL = unL - cL, tt = unR - cR;
      if (tt < SL) SL = tt;
      R SR = unL + cL;
      tt = unR + cR;
      if (tt > SR) SR = tt;
      R FnL[3], FnR[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        FnL[k] = FxL[k] * nx + FyL[k] * ny;
        FnR[k] = FxR[k] * nx + FyR[k] * ny;
      }
      if (SL >= R(0)) {
#pragma unroll
        for (int k = 0; k < 3; ++k) f[k] = FnL[k];
      } else if (SR <= R(0)) {
#pragma unroll
        for (int k = 0; k < 3; ++k) f[k] = FnR[k];
      } else {
        R inv = R(1) / (SR - SL);
#pragma unroll
        for (int k = 0; k < 3; ++k) f[k] = (SR * FnL[k] - SL * FnR[k] + SL * SR * (qR[k] - qL[k])) * inv;
      }
      return;
    }
    R sL = sqrt(uL * uL + vL * vL) + cL, sR = sqrt(uR * uR + vR * vR) + cR;
    R al = sL > sR ? sL : sR, h = R(0.5);
#pragma unroll
    for (int k = 0; k < 3; ++k) f[k] = h * ((FxL[k] + FxR[k]) * nx + (FyL[k] + FyR[k]) * ny) - h * al * (qR[k] - qL[k]);
  }
  __device__ void source(const R*, R* s) const { s[0] = s[1] = s[2] = R(0); }
  __device__ R speed(const R* q) const {
    R h = q[0] < h_min ? h_min : q[0];
    R u = q[1] / h, v = q[2] / h;
    return sqrt(u * u + v * v) + sqrt(g * h);
  }
};

template <class R>
struct Maxwell2D {
  static constexpr int NC = 6;
  static constexpr bool kSource = true;
  R c, J[3], M[3], inflow[6];
  __device__ void flux(const R* q, R* Fx, R* Fy) const {
    R c2 = c * c;
    Fx[0] = R(0); Fx[1] = c2 * q[5]; Fx[2] = -c2 * q[4]; Fx[3] = R(0); Fx[4] = -q[2]; Fx[5] = q[1];
    Fy[0] = -c2 * q[5]; Fy[1] = R(0); Fy[2] = c2 * q[3]; Fy[3] = q[2]; Fy[4] = R(0); Fy[5] = -q[0];
  }
  __device__ void face(const R* qL, const R* qRin, int bc, R nx, R ny, R* f) const {
    R qR[6];
    if (bc == BC_INTERIOR) {
#pragma unroll
      for (int k = 0; k < 6; ++k) qR[k] = qRin[k];
    } else if (bc == BC_WALL) {
      R En = qL[0] * nx + qL[1] * ny, Bn = qL[3] * nx + qL[4] * ny;
      qR[0] = R(2) * En * nx - qL[0]; qR[1] = R(2) * En * ny - qL[1]; qR[2] = -qL[2];
      qR[3] = qL[3] - R(2) * Bn * nx; qR[4] = qL[4] - R(2) * Bn * ny; qR[5] = qL[5];
    } else if (bc == BC_INFLOW) {
#pragma unroll
      for (int k = 0; k < 6; ++k) qR[k] = inflow[k];
    } else {
#pragma unroll
      for (int k = 0; k < 6; ++k) qR[k] = qL[k];
    }
    R c2 = c * c, h = R(0.5);
    f[0] = h * (c2 * (-qL[5] * ny) + c2 * (-qR[5] * ny)) - h * c * (qR[0] - qL[0]);
    f[1] = h * (c2 * (qL[5] * nx) + c2 * (qR[5] * nx)) - h * c * (qR[1] - qL[1]);
    f[2] = h * (c2 * (qL[3] * ny - qL[4] * nx) + c2 * (qR[3] * ny - qR[4] * nx)) - h * c * (qR[2] - qL[2]);
    f[3] = h * (ny * qL[2] + ny * qR[2]) - h * c * (qR[3] - qL[3]);
    f[4] = h * (-nx * qL[2] + -nx * qR[2]) - h * c * (qR[4] - qL[4]);
    f[5] = h * ((nx * qL[1] - ny * qL[0]) + (nx * qR[1] - ny * qR[0])) - h * c * (qR[5] - qL[5]);
  }
  __device__ void source(const R*, R* s) const {
    R c2 = c * c;
    s[0] = -c2 * J[0]; s[1] = -c2 * J[1]; s[2] = -c2 * J[2];
    s[3] = -M[0]; s[4] = -M[1]; s[5] = -M[2];
  }
  __device__ R speed(const R*) const { return c; }
};

// 2D ideal MHD, state (rho, mx, my, Bx, By, E[, psi]).  Rusanov against
// |v| + c_f (c_f from Bx^2, as the reference writes it) and, with GLM, c_h.
template <class R, bool GLM>
struct Mhd2D {
  static constexpr int NC = GLM ? 7 : 6;
  static constexpr bool kSource = false;
  R gamma, rho_min, p_min, c_h, inflow[7];
  // physical fluxes and the Rusanov speed of one state
  // (local_mesh_2d_gpu_mhd.mojo:73-102 / _glm.mojo:89-124; speeds :321-331 / :355-363)
  __device__ R flux_speed(const R* q, R* Fx, R* Fy) const {
    R rho = q[0];
    if (rho < rho_min) rho = rho_min;
    const R ri = pos_rcp(rho);
    const R mx = q[1], my = q[2], Bx = q[3], By = q[4], E = q[5];
    const R u = mx * ri, v = my * ri, BB = Bx * Bx + By * By;
    const R ke = R(0.5) * (mx * mx + my * my) * ri;
    R p = (gamma - R(1)) * (E - ke - R(0.5) * BB);
    if (p < p_min) p = p_min;
    const R ps = p + R(0.5) * BB, ub = u * Bx + v * By;
    const R psi = GLM ? q[NC - 1] : R(0);
    Fx[0] = mx; Fx[1] = mx * u + ps - Bx * Bx; Fx[2] = mx * v - Bx * By; Fx[3] = psi;
    Fx[4] = u * By - v * Bx; Fx[5] = (E + ps) * u - Bx * ub;
    Fy[0] = my; Fy[1] = my * u - By * Bx; Fy[2] = my * v + ps - By * By; Fy[3] = v * Bx - u * By;
    Fy[4] = psi; Fy[5] = (E + ps) * v - By * ub;
    if (GLM) {
      const R ch2 = c_h * c_h;
      Fx[NC - 1] = ch2 * Bx;
      Fy[NC - 1] = ch2 * By;
    }
    const R cs2 = gamma * p * ri, ca2 = BB * ri, sm = cs2 + ca2;
    R disc = sm * sm - R(4) * cs2 * (Bx * Bx) * ri;
    if (disc < R(0)) disc = R(0);
    R sp = sqrt(u * u + v * v) + sqrt(R(0.5) * (sm + sqrt(disc)));
    if (GLM && c_h > sp) sp = c_h;
    return sp;
  }
  __device__ void flux(const R* q, R* Fx, R* Fy) const { (void)flux_speed(q, Fx, Fy); }
  __device__ void face(const R* qL, const R* qRin, int bc, R nx, R ny, R* f) const {
    R qR[NC];
    if (bc == BC_INTERIOR) {
#pragma unroll
      for (int k = 0; k < NC; ++k) qR[k] = qRin[k];
    } else if (bc == BC_WALL) {  // conducting slip wall: reflect m_n and B_n (GLM: psi too)
      const R mn = qL[1] * nx + qL[2] * ny, bn = qL[3] * nx + qL[4] * ny;
      qR[0] = qL[0]; qR[1] = qL[1] - R(2) * mn * nx; qR[2] = qL[2] - R(2) * mn * ny;
      qR[3] = qL[3] - R(2) * bn * nx; qR[4] = qL[4] - R(2) * bn * ny; qR[5] = qL[5];
      if (GLM) qR[NC - 1] = -qL[NC - 1];
    } else if (bc == BC_INFLOW) {
#pragma unroll
      for (int k = 0; k < NC; ++k) qR[k] = inflow[k];
    } else {
#pragma unroll
      for (int k = 0; k < NC; ++k) qR[k] = qL[k];
    }
    R FxL[NC], FyL[NC], FxR[NC], FyR[NC];
    const R sL = flux_speed(qL, FxL, FyL), sR = flux_speed(qR, FxR, FyR);
    const R al = sL > sR ? sL : sR, h = R(0.5);
#pragma unroll
    for (int k = 0; k < NC; ++k) f[k] = h * ((FxL[k] + FxR[k]) * nx + (FyL[k] + FyR[k]) * ny) - h * al * (qR[k] - qL[k]);
  }
  __device__ void source(const R*, R* s) const {
#pragma unroll
    for (int k = 0; k < NC; ++k) s[k] = R(0);
  }
  __device__ R speed(const R* q) const {
    R Fx[NC], Fy[NC];
    return flux_speed(q, Fx, Fy);
  }
};

}  // namespace mxm
