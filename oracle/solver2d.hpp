// ORACLE — test infrastructure only (see refelem.hpp header).
// CPU restatement of mojoxm's 2D triangle path:
//   LocalMesh2D (host Kuhn-triangle mesh + BC overlay)  src/local_mesh_2d.mojo:106-395
//   per-physics face-flux kernels + fused vol/lift/RK   src/local_mesh_2d_gpu_{euler,sw,maxwell,advection}.mojo
//   cell mean + BJ limiter (component 0 only)           src/local_mesh_2d_gpu.mojo:180-198,
//                                                       src/local_mesh_2d_gpu_limiter.mojo:74-210
//   SSPRK3 stage plans                                   src/ssprk3.mojo:56-78
// 2D HLLE has no reference kernel: it is the 3D euler_hlle_solver applied to
// the state embedded with w = 0 and n_z = 0 (src/euler.mojo:364-412,626-691).
#pragma once
#include <vector>

#include "physics.hpp"

namespace orc {

template <typename R>
struct Mesh2D {  // LocalMesh2D  local_mesh_2d.mojo:73-395 (geometry FP64 host, stored as R)
  int P, NP, NFP, Nx, Ny;
  int64_t Ne, Nf;
  std::vector<R> elem_node_xy, elem_invJ, elem_inv_2A, face_normal, face_length;
  std::vector<int32_t> elem_faces, elem_face_side, elem_canon_to_ref, face_elem, face_elem_node, face_bc_type;
  Mesh2D(int P_, int nx, int ny, double Lx, double Ly, const int bc[4])
      : P(P_), NP(num_tri_nodes(P_)), NFP(P_ + 1), Nx(nx), Ny(ny) {
    const double dx = Lx / double(Nx), dy = Ly / double(Ny);
    Ne = int64_t(Nx) * Ny * 2;
    const int64_t nfp = int64_t(Nx) * Ny * 3;
    const int64_t exm = bc[0] ? Ny : 0, eym = bc[2] ? Nx : 0;
    Nf = nfp + exm + eym;
    RefElem2D re(P);
    elem_node_xy.assign(Ne * NP * 2, R(0));
    elem_invJ.assign(Ne * 4, R(0));
    elem_inv_2A.assign(Ne, R(0));
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i) {
        double bx = double(i) * dx, by = double(j) * dy;
        for (int t = 0; t < 2; ++t) {
          int64_t e = (int64_t(j) * Nx + i) * 2 + t;
          double v0x = bx, v0y = by, v1x, v1y, v2x, v2y;
          if (t == 0) { v1x = bx + dx; v1y = by; v2x = bx + dx; v2y = by + dy; }
          else { v1x = bx + dx; v1y = by + dy; v2x = bx; v2y = by + dy; }
          for (int n = 0; n < NP; ++n) {
            double r = re.node_pos[n * 2], s = re.node_pos[n * 2 + 1], l0 = 1.0 - r - s;
            elem_node_xy[(e * NP + n) * 2 + 0] = R(l0 * v0x + r * v1x + s * v2x);
            elem_node_xy[(e * NP + n) * 2 + 1] = R(l0 * v0y + r * v1y + s * v2y);
          }
          double J00 = v1x - v0x, J01 = v2x - v0x, J10 = v1y - v0y, J11 = v2y - v0y;
          double det = J00 * J11 - J01 * J10;
          if (!(det > 0.0)) throw std::runtime_error("LocalMesh2D: non-positive area");
          double id = 1.0 / det;
          elem_invJ[e * 4 + 0] = R(J11 * id);
          elem_invJ[e * 4 + 1] = R(-J01 * id);
          elem_invJ[e * 4 + 2] = R(-J10 * id);
          elem_invJ[e * 4 + 3] = R(J00 * id);
          elem_inv_2A[e] = R(id);
        }
      }
    face_elem.assign(Nf * 2, 0);
    face_elem_node.assign(Nf * 2 * NFP, 0);
    face_normal.assign(Nf * 2, R(0));
    face_length.assign(Nf, R(0));
    face_bc_type.assign(Nf, 0);
    elem_faces.assign(Ne * 3, 0);
    elem_face_side.assign(Ne * 3, 0);
    elem_canon_to_ref.assign(Ne * 3 * NFP, 0);
    const int s0t[3] = {0, 0, 1}, s0e[3] = {2, 1, 1}, s1t[3] = {1, 1, 0}, s1e[3] = {0, 2, 0}, fdi[3] = {0, 1, 0},
              fdj[3] = {0, 0, 1};
    const double dl = std::sqrt(dx * dx + dy * dy);
    const double fnx[3] = {-dy / dl, 1.0, 0.0}, fny[3] = {dx / dl, 0.0, 1.0}, fln[3] = {dl, dy, dx};
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i) {
        int64_t cell = int64_t(j) * Nx + i;
        for (int ft = 0; ft < 3; ++ft) {
          int64_t fid = cell * 3 + ft;
          int64_t e0 = cell * 2 + s0t[ft];
          int ni = (i + fdi[ft] + Nx) % Nx, nj = (j + fdj[ft] + Ny) % Ny;
          int64_t e1 = (int64_t(nj) * Nx + ni) * 2 + s1t[ft];
          face_elem[fid * 2] = int32_t(e0);
          face_elem[fid * 2 + 1] = int32_t(e1);
          face_normal[fid * 2] = R(fnx[ft]);
          face_normal[fid * 2 + 1] = R(fny[ft]);
          face_length[fid] = R(fln[ft]);
          int l0 = s0e[ft], l1 = s1e[ft];
          elem_faces[e0 * 3 + l0] = int32_t(fid);
          elem_face_side[e0 * 3 + l0] = 0;
          elem_faces[e1 * 3 + l1] = int32_t(fid);
          elem_face_side[e1 * 3 + l1] = 1;
          for (int m = 0; m < NFP; ++m) {
            face_elem_node[(fid * 2) * NFP + m] = re.edge_to_elem[l0 * NFP + m];
            face_elem_node[(fid * 2 + 1) * NFP + m] = re.edge_to_elem[l1 * NFP + (NFP - 1 - m)];
            elem_canon_to_ref[(e0 * 3 + l0) * NFP + m] = m;
            elem_canon_to_ref[(e1 * 3 + l1) * NFP + m] = NFP - 1 - m;
          }
        }
      }
    if (bc[1])
      for (int j = 0; j < Ny; ++j) {
        int64_t fid = (int64_t(j) * Nx + (Nx - 1)) * 3 + 1;
        face_elem[fid * 2 + 1] = face_elem[fid * 2];
        face_bc_type[fid] = bc[1];
      }
    if (bc[3])
      for (int i = 0; i < Nx; ++i) {
        int64_t fid = (int64_t(Ny - 1) * Nx + i) * 3 + 2;
        face_elem[fid * 2 + 1] = face_elem[fid * 2];
        face_bc_type[fid] = bc[3];
      }
    auto minus = [&](int64_t nf, int64_t e, int lf, R nx, R ny, R len, int v) {
      face_elem[nf * 2] = int32_t(e);
      face_elem[nf * 2 + 1] = int32_t(e);
      face_normal[nf * 2] = nx;
      face_normal[nf * 2 + 1] = ny;
      face_length[nf] = len;
      face_bc_type[nf] = v;
      elem_faces[e * 3 + lf] = int32_t(nf);
      elem_face_side[e * 3 + lf] = 0;
      for (int m = 0; m < NFP; ++m) {
        int nn = re.edge_to_elem[lf * NFP + m];
        face_elem_node[(nf * 2) * NFP + m] = nn;
        face_elem_node[(nf * 2 + 1) * NFP + m] = nn;
        elem_canon_to_ref[(e * 3 + lf) * NFP + m] = m;
      }
    };
    if (bc[0])
      for (int j = 0; j < Ny; ++j) minus(nfp + j, (int64_t(j) * Nx) * 2 + 1, 2, R(-1), R(0), R(dy), bc[0]);
    if (bc[2])
      for (int i = 0; i < Nx; ++i) minus(nfp + exm + i, int64_t(i) * 2 + 0, 0, R(0), R(-1), R(dx), bc[2]);
  }
};

// Per-physics 2D kernels (face flux into fstar[fid, m, c]; vol+lift+RK).
template <typename R>
struct Phys2D {
  int kind, flux;
  R gamma = R(1.4), min_density = R(0), min_pressure = R(0), gx = R(0), gy = R(0);
  R inflow[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
  R c_h = R(0), alpha_d = R(0);              // 2D MHD (GLM)
  R vx = R(0), vy = R(0), inflow_q = R(0);  // advection
  R g = R(9.81), h_min = R(0);              // shallow water
  R c = R(1), J[3] = {R(0), R(0), R(0)}, M[3] = {R(0), R(0), R(0)};
  bool entropy_fix = false;
  int nc() const {
    return kind == PHYS_ADVECTION ? 1 : kind == PHYS_EULER ? 4 : kind == PHYS_MAXWELL ? 6
         : kind == PHYS_MHD ? 7 : kind == PHYS_MHD_PLAIN ? 6 : 3;
  }

  // Ghost state for BC faces; identical plumbing in every 2D face kernel.
  void ghost(const R* qL, int bc, R nx, R ny, R* qR) const {
    const int n = nc();
    if (bc == BC_WALL) {
      if (kind == PHYS_EULER) {  // euler.mojo 2D :288-293
        R mn = qL[1] * nx + qL[2] * ny;
        qR[0] = qL[0]; qR[1] = qL[1] - R(2) * mn * nx; qR[2] = qL[2] - R(2) * mn * ny; qR[3] = qL[3];
      } else if (kind == PHYS_SW) {
        R mn = qL[1] * nx + qL[2] * ny;
        qR[0] = qL[0]; qR[1] = qL[1] - R(2) * mn * nx; qR[2] = qL[2] - R(2) * mn * ny;
      } else if (kind == PHYS_MAXWELL) {  // local_mesh_2d_gpu_maxwell.mojo face kernel
        R En = qL[0] * nx + qL[1] * ny, Bn = qL[3] * nx + qL[4] * ny;
        qR[0] = R(2) * En * nx - qL[0]; qR[1] = R(2) * En * ny - qL[1]; qR[2] = -qL[2];
        qR[3] = qL[3] - R(2) * Bn * nx; qR[4] = qL[4] - R(2) * Bn * ny; qR[5] = qL[5];
      } else if (kind == PHYS_MHD || kind == PHYS_MHD_PLAIN) {
        // local_mesh_2d_gpu_mhd.mojo:276-284, _mhd_glm.mojo:296-305 (psi reflects)
        R mn = qL[1] * nx + qL[2] * ny, bn = qL[3] * nx + qL[4] * ny;
        qR[0] = qL[0]; qR[1] = qL[1] - R(2) * mn * nx; qR[2] = qL[2] - R(2) * mn * ny;
        qR[3] = qL[3] - R(2) * bn * nx; qR[4] = qL[4] - R(2) * bn * ny; qR[5] = qL[5];
        if (kind == PHYS_MHD) qR[6] = -qL[6];
      }
    } else if (bc == BC_INFLOW) {
      for (int k = 0; k < n; ++k) qR[k] = inflow[k];
    } else {
      for (int k = 0; k < n; ++k) qR[k] = qL[k];
    }
  }

  void face_flux(const R* qL, const R* qRin, int bc, R nx, R ny, R* f) const {
    const int n = nc();
    R qR[8];
    if (kind == PHYS_ADVECTION) {  // local_mesh_2d_gpu_advection.mojo:249-300
      R vn = vx * nx + vy * ny;
      if (bc == BC_INTERIOR) f[0] = vn >= R(0) ? vn * qL[0] : vn * qRin[0];
      else if (bc == BC_INFLOW) f[0] = vn >= R(0) ? vn * qL[0] : vn * inflow_q;
      else f[0] = vn >= R(0) ? vn * qL[0] : R(0);
      return;
    }
    if (bc == BC_INTERIOR) for (int k = 0; k < n; ++k) qR[k] = qRin[k];
    else ghost(qL, bc, nx, ny, qR);
    const R h = R(0.5);
    if (kind == PHYS_EULER && flux == FLUX_RUSANOV) {  // local_mesh_2d_gpu_euler.mojo:220-337
      R rL = qL[0] < min_density ? min_density : qL[0];
      R uL = qL[1] / rL, vL = qL[2] / rL;
      R pL = (gamma - R(1)) * (qL[3] - R(0.5) * rL * (uL * uL + vL * vL));
      if (pL < min_pressure) pL = min_pressure;
      R sL = std::sqrt(uL * uL + vL * vL) + std::sqrt(gamma * pL / rL);
      R rR = qR[0] < min_density ? min_density : qR[0];
      R uR = qR[1] / rR, vR = qR[2] / rR;
      R pR = (gamma - R(1)) * (qR[3] - R(0.5) * rR * (uR * uR + vR * vR));
      if (pR < min_pressure) pR = min_pressure;
      R sR = std::sqrt(uR * uR + vR * vR) + std::sqrt(gamma * pR / rR);
      R FxL[4] = {qL[1], qL[1] * uL + pL, qL[1] * vL, uL * (qL[3] + pL)};
      R FyL[4] = {qL[2], qL[2] * uL, qL[2] * vL + pL, vL * (qL[3] + pL)};
      R FxR[4] = {qR[1], qR[1] * uR + pR, qR[1] * vR, uR * (qR[3] + pR)};
      R FyR[4] = {qR[2], qR[2] * uR, qR[2] * vR + pR, vR * (qR[3] + pR)};
      R al = sL > sR ? sL : sR;
      for (int k = 0; k < 4; ++k) f[k] = h * ((FxL[k] + FxR[k]) * nx + (FyL[k] + FyR[k]) * ny) - h * al * (qR[k] - qL[k]);
      return;
    }
    if (kind == PHYS_EULER && flux == FLUX_HLLC) {  // local_mesh_2d_gpu_euler.mojo:392-545
      R rL = qL[0] < min_density ? min_density : qL[0];
      R rR = qR[0] < min_density ? min_density : qR[0];
      R uL = qL[1] / rL, vL = qL[2] / rL, uR = qR[1] / rR, vR = qR[2] / rR;
      R pL = (gamma - R(1)) * (qL[3] - R(0.5) * rL * (uL * uL + vL * vL));
      if (pL < min_pressure) pL = min_pressure;
      R pR = (gamma - R(1)) * (qR[3] - R(0.5) * rR * (uR * uR + vR * vR));
      if (pR < min_pressure) pR = min_pressure;
      R aL = std::sqrt(gamma * pL / rL), aR = std::sqrt(gamma * pR / rR);
      R unL = uL * nx + vL * ny, unR = uR * nx + vR * ny;
      R FnL[4] = {qL[1] * nx + qL[2] * ny, (qL[1] * uL + pL) * nx + (qL[1] * vL) * ny,
                  (qL[1] * vL) * nx + (qL[2] * vL + pL) * ny, (uL * (qL[3] + pL)) * nx + (vL * (qL[3] + pL)) * ny};
      R FnR[4] = {qR[1] * nx + qR[2] * ny, (qR[1] * uR + pR) * nx + (qR[1] * vR) * ny,
                  (qR[1] * vR) * nx + (qR[2] * vR + pR) * ny, (uR * (qR[3] + pR)) * nx + (vR * (qR[3] + pR)) * ny};
      R SL = unL - aL, t = unR - aR;
      if (t < SL) SL = t;
      R SR = unL + aL;
      t = unR + aR;
      if (t > SR) SR = t;
      R num = pR - pL + rL * unL * (SL - unL) - rR * unR * (SR - unR);
      R den = rL * (SL - unL) - rR * (SR - unR);
      R Ss = num / den;
      if (SL >= R(0)) { for (int k = 0; k < 4; ++k) f[k] = FnL[k]; }
      else if (SR <= R(0)) { for (int k = 0; k < 4; ++k) f[k] = FnR[k]; }
      else if (Ss >= R(0)) {
        R co = (SL - unL) / (SL - Ss), rs = rL * co;
        R us = uL + (Ss - unL) * nx, vs = vL + (Ss - unL) * ny;
        R Es = qL[3] / rL + (Ss - unL) * (Ss + pL / (rL * (SL - unL)));
        R qs[4] = {rs, rs * us, rs * vs, rs * Es};
        for (int k = 0; k < 4; ++k) f[k] = FnL[k] + SL * (qs[k] - qL[k]);
      } else {
        R co = (SR - unR) / (SR - Ss), rs = rR * co;
        R us = uR + (Ss - unR) * nx, vs = vR + (Ss - unR) * ny;
        R Es = qR[3] / rR + (Ss - unR) * (Ss + pR / (rR * (SR - unR)));
        R qs[4] = {rs, rs * us, rs * vs, rs * Es};
        for (int k = 0; k < 4; ++k) f[k] = FnR[k] + SR * (qs[k] - qR[k]);
      }
      return;
    }
    if (kind == PHYS_EULER) {  // HLLE: the 3D solver on the embedded state
      Euler<R> e3;
      e3.gamma = gamma; e3.min_density = min_density; e3.min_pressure = min_pressure;
      e3.flux_type = FLUX_HLLE; e3.entropy_fix = entropy_fix;
      e3.gx = e3.gy = e3.gz = R(0);
      R l3[5] = {qL[0], qL[1], qL[2], R(0), qL[3]}, r3[5] = {qR[0], qR[1], qR[2], R(0), qR[3]}, f3[5];
      e3.numerical_flux(l3, r3, nx, ny, R(0), f3);
      f[0] = f3[0]; f[1] = f3[1]; f[2] = f3[2]; f[3] = f3[4];
      return;
    }
    if (kind == PHYS_MHD || kind == PHYS_MHD_PLAIN) {
      // Rusanov against |v| + c_f (c_f with Bx^2), and c_h for GLM:
      // local_mesh_2d_gpu_mhd.mojo:301-378, local_mesh_2d_gpu_mhd_glm.mojo:325-413
      const bool glm = kind == PHYS_MHD;
      R FxL[7], FyL[7], FxR[7], FyR[7];
      vol_flux(qL, FxL, FyL);
      vol_flux(qR, FxR, FyR);
      auto speed = [&](const R* q) {
        R rho = q[0];
        if (rho < min_density) rho = min_density;
        R u = q[1] / rho, v = q[2] / rho, BB = q[3] * q[3] + q[4] * q[4];
        R ke = R(0.5) * (q[1] * q[1] + q[2] * q[2]) / rho;
        R pr = (gamma - R(1)) * (q[5] - ke - R(0.5) * BB);
        if (pr < min_pressure) pr = min_pressure;
        R cs2 = gamma * pr / rho, ca2 = BB / rho, sm = cs2 + ca2;
        R disc = sm * sm - R(4) * cs2 * (q[3] * q[3]) / rho;
        if (disc < R(0)) disc = R(0);
        R cf = std::sqrt(R(0.5) * (sm + std::sqrt(disc)));
        R sp = std::sqrt(u * u + v * v) + cf;
        if (glm && c_h > sp) sp = c_h;
        return sp;
      };
      R sL = speed(qL), sR = speed(qR);
      R al = sL > sR ? sL : sR;
      for (int k = 0; k < n; ++k) f[k] = h * ((FxL[k] + FxR[k]) * nx + (FyL[k] + FyR[k]) * ny) - h * al * (qR[k] - qL[k]);
      return;
    }
    if (kind == PHYS_SW) {
      R hL = qL[0] < h_min ? h_min : qL[0], hR = qR[0] < h_min ? h_min : qR[0];
      R uL = qL[1] / hL, vL = qL[2] / hL, uR = qR[1] / hR, vR = qR[2] / hR;
      R pL = R(0.5) * g * hL * hL, pR = R(0.5) * g * hR * hR;
      R cL = std::sqrt(g * hL), cR = std::sqrt(g * hR);
      R FxL[3] = {qL[1], qL[1] * uL + pL, qL[1] * vL}, FyL[3] = {qL[2], qL[2] * uL, qL[2] * vL + pL};
      R FxR[3] = {qR[1], qR[1] * uR + pR, qR[1] * vR}, FyR[3] = {qR[2], qR[2] * uR, qR[2] * vR + pR};
      if (flux == FLUX_HLL) {  // local_mesh_2d_gpu_sw.mojo:308-450
        R unL = uL * nx + vL * ny, unR = uR * nx + vR * ny;
        R SL = unL - cL, t = unR - cR;
        if (t < SL) SL = t;
        R SR = unL + cL;
        t = unR + cR;
        if (t > SR) SR = t;
        R FnL[3], FnR[3];
        for (int k = 0; k < 3; ++k) { FnL[k] = FxL[k] * nx + FyL[k] * ny; FnR[k] = FxR[k] * nx + FyR[k] * ny; }
        if (SL >= R(0)) { for (int k = 0; k < 3; ++k) f[k] = FnL[k]; }
        else if (SR <= R(0)) { for (int k = 0; k < 3; ++k) f[k] = FnR[k]; }
        else {
          R inv = R(1) / (SR - SL);
          for (int k = 0; k < 3; ++k) f[k] = (SR * FnL[k] - SL * FnR[k] + SL * SR * (qR[k] - qL[k])) * inv;
        }
        return;
      }
      // Rusanov  local_mesh_2d_gpu_sw.mojo:178-306
      R sL = std::sqrt(uL * uL + vL * vL) + cL, sR = std::sqrt(uR * uR + vR * vR) + cR;
      R al = sL > sR ? sL : sR;
      for (int k = 0; k < 3; ++k) f[k] = h * ((FxL[k] + FxR[k]) * nx + (FyL[k] + FyR[k]) * ny) - h * al * (qR[k] - qL[k]);
      return;
    }
    // Maxwell Rusanov  local_mesh_2d_gpu_maxwell.mojo:219-377
    R c2 = c * c;
    R FEl[3] = {c2 * (-qL[5] * ny), c2 * (qL[5] * nx), c2 * (qL[3] * ny - qL[4] * nx)};
    R FBl[3] = {ny * qL[2], -nx * qL[2], nx * qL[1] - ny * qL[0]};
    R FEr[3] = {c2 * (-qR[5] * ny), c2 * (qR[5] * nx), c2 * (qR[3] * ny - qR[4] * nx)};
    R FBr[3] = {ny * qR[2], -nx * qR[2], nx * qR[1] - ny * qR[0]};
    for (int k = 0; k < 3; ++k) {
      f[k] = h * (FEl[k] + FEr[k]) - h * c * (qR[k] - qL[k]);
      f[3 + k] = h * (FBl[k] + FBr[k]) - h * c * (qR[3 + k] - qL[3 + k]);
    }
  }

  // Physical fluxes (x, y) at a node as the vol kernels compute them.
  void vol_flux(const R* q, R* Fx, R* Fy) const {
    if (kind == PHYS_ADVECTION) { Fx[0] = vx * q[0]; Fy[0] = vy * q[0]; return; }
    if (kind == PHYS_EULER) {  // euler 2D vol  :33-144
      R rho = q[0];
      if (rho < min_density) rho = min_density;
      R u = q[1] / rho, v = q[2] / rho;
      R p = (gamma - R(1)) * (q[3] - R(0.5) * rho * (u * u + v * v));
      if (p < min_pressure) p = min_pressure;
      Fx[0] = q[1]; Fx[1] = q[1] * u + p; Fx[2] = q[1] * v; Fx[3] = u * (q[3] + p);
      Fy[0] = q[2]; Fy[1] = q[2] * u; Fy[2] = q[2] * v + p; Fy[3] = v * (q[3] + p);
      return;
    }
    if (kind == PHYS_SW) {  // sw 2D vol  local_mesh_2d_gpu_sw.mojo:27-176
      R hh = q[0];
      if (hh < h_min) hh = h_min;
      R u = q[1] / hh, v = q[2] / hh, p = R(0.5) * g * hh * hh;
      Fx[0] = q[1]; Fx[1] = q[1] * u + p; Fx[2] = q[1] * v;
      Fy[0] = q[2]; Fy[1] = q[2] * u; Fy[2] = q[2] * v + p;
      return;
    }
    if (kind == PHYS_MHD || kind == PHYS_MHD_PLAIN) {
      // (rho, mx, my, Bx, By, E[, psi]): local_mesh_2d_gpu_mhd.mojo:73-102, _mhd_glm.mojo:89-124
      R rho = q[0];
      if (rho < min_density) rho = min_density;
      R mx = q[1], my = q[2], Bx = q[3], By = q[4], E = q[5];
      R u = mx / rho, v = my / rho, BB = Bx * Bx + By * By;
      R ke = R(0.5) * (mx * mx + my * my) / rho, mp = R(0.5) * BB;
      R pr = (gamma - R(1)) * (E - ke - mp);
      if (pr < min_pressure) pr = min_pressure;
      R ps = pr + R(0.5) * BB;
      const bool glm = kind == PHYS_MHD;
      R psi = glm ? q[6] : R(0), ch2 = c_h * c_h;
      Fx[0] = mx; Fx[1] = mx * u + ps - Bx * Bx; Fx[2] = mx * v - Bx * By; Fx[3] = glm ? psi : R(0);
      Fx[4] = u * By - v * Bx; Fx[5] = (E + ps) * u - Bx * (u * Bx + v * By);
      Fy[0] = my; Fy[1] = my * u - By * Bx; Fy[2] = my * v + ps - By * By; Fy[3] = v * Bx - u * By;
      Fy[4] = glm ? psi : R(0); Fy[5] = (E + ps) * v - By * (u * Bx + v * By);
      if (glm) { Fx[6] = ch2 * Bx; Fy[6] = ch2 * By; }
      return;
    }
    R c2 = c * c;  // maxwell 2D vol  local_mesh_2d_gpu_maxwell.mojo:31-218
    Fx[0] = R(0); Fx[1] = c2 * q[5]; Fx[2] = -c2 * q[4]; Fx[3] = R(0); Fx[4] = -q[2]; Fx[5] = q[1];
    Fy[0] = -c2 * q[5]; Fy[1] = R(0); Fy[2] = c2 * q[3]; Fy[3] = q[2]; Fy[4] = R(0); Fy[5] = -q[0];
  }
  void source(const R* q, R* s) const {
    for (int k = 0; k < 8; ++k) s[k] = R(0);
    if (kind == PHYS_EULER) {
      R rho = q[0] < min_density ? min_density : q[0];
      s[1] = rho * gx;
      s[2] = rho * gy;
      s[3] = q[1] * gx + q[2] * gy;
    } else if (kind == PHYS_MAXWELL) {
      R c2 = c * c;
      s[0] = -c2 * J[0]; s[1] = -c2 * J[1]; s[2] = -c2 * J[2]; s[3] = -M[0]; s[4] = -M[1]; s[5] = -M[2];
    }
  }
};

struct Solver2DBase {
  virtual ~Solver2DBase() {}
  int P, NP, NFP, NC;
  int64_t Ne;
  virtual void set_buf(int which, const double* src) = 0;
  virtual void get_buf(int which, double* dst) const = 0;
  virtual void eval_rhs(const double* q, double* rhs) = 0;
  virtual void stage(int s, double dt) = 0;
  virtual void step(double dt) = 0;
  virtual void enable_limiter(bool on, double eps) = 0;
  virtual void limit(int which) = 0;
  virtual void node_xy(double* out) const = 0;
};

template <typename R>
struct Solver2D : Solver2DBase {
  Mesh2D<R> mesh;
  Phys2D<R> ph;
  std::vector<R> Dr, Ds, Lift, w, fstar, cmean, theta;
  std::vector<R> q[3];
  bool lim_on = false;
  R lim_eps = R(0.1);
  Solver2D(int P_, int nx, int ny, double Lx, double Ly, const int bc[4], const Phys2D<R>& p)
      : mesh(P_, nx, ny, Lx, Ly, bc), ph(p) {
    P = P_;
    NP = mesh.NP;
    NFP = mesh.NFP;
    NC = ph.nc();
    Ne = mesh.Ne;
    RefElem2D re(P);
    for (double v : re.Dr) Dr.push_back(R(v));
    for (double v : re.Ds) Ds.push_back(R(v));
    for (double v : re.Lift) Lift.push_back(R(v));
    for (double v : re.w) w.push_back(R(v));
    for (auto& b : q) b.assign(size_t(Ne) * NP * NC, R(0));
    fstar.assign(size_t(mesh.Nf) * NFP * NC, R(0));
    cmean.assign(size_t(Ne) * NC, R(0));
    theta.assign(size_t(Ne), R(1));
  }
  void set_buf(int which, const double* src) override {
    for (size_t k = 0; k < q[which].size(); ++k) q[which][k] = R(src[k]);
  }
  void get_buf(int which, double* dst) const override {
    for (size_t k = 0; k < q[which].size(); ++k) dst[k] = double(q[which][k]);
  }
  void node_xy(double* out) const override {
    for (size_t k = 0; k < mesh.elem_node_xy.size(); ++k) out[k] = double(mesh.elem_node_xy[k]);
  }
  void faces(const R* qi) {
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < mesh.Nf * NFP; ++t) {
      int64_t fid = t / NFP;
      int m = int(t % NFP);
      R nx = mesh.face_normal[fid * 2], ny = mesh.face_normal[fid * 2 + 1];
      int bc = mesh.face_bc_type[fid];
      int64_t el = mesh.face_elem[fid * 2], er = mesh.face_elem[fid * 2 + 1];
      int nl = mesh.face_elem_node[(fid * 2) * NFP + m], nr = mesh.face_elem_node[(fid * 2 + 1) * NFP + m];
      ph.face_flux(qi + (el * NP + nl) * NC, qi + (er * NP + nr) * NC, bc, nx, ny, &fstar[(fid * NFP + m) * NC]);
    }
  }
  void vol_lift(const R* qi, const R* qa, const R* qb, R* qo, R a, R b, R cc, R dt, bool rhs_only) {
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < Ne * NP; ++t) {
      int64_t e = t / NP;
      int i = int(t % NP);
      const R* iJ = &mesh.elem_invJ[e * 4];
      R acc[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
      R fc[8] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};
      for (int j = 0; j < NP; ++j) {
        R Fx[8], Fy[8];
        ph.vol_flux(qi + (e * NP + j) * NC, Fx, Fy);
        R dr = Dr[i * NP + j], ds = Ds[i * NP + j];
        for (int c = 0; c < NC; ++c)
          acc[c] += (iJ[0] * Fx[c] + iJ[1] * Fy[c]) * dr + (iJ[2] * Fx[c] + iJ[3] * Fy[c]) * ds;
      }
      for (int lf = 0; lf < 3; ++lf) {
        int64_t fid = mesh.elem_faces[e * 3 + lf];
        R sign = mesh.elem_face_side[e * 3 + lf] == 0 ? R(1) : R(-1);
        R flen = mesh.face_length[fid];
        for (int m = 0; m < NFP; ++m) {
          int r = mesh.elem_canon_to_ref[(e * 3 + lf) * NFP + m];
          R sLf = sign * flen * Lift[lf * NP * NFP + i * NFP + r];
          for (int c = 0; c < NC; ++c) fc[c] += sLf * fstar[(fid * NFP + m) * NC + c];
        }
      }
      R src[8];
      ph.source(qi + (e * NP + i) * NC, src);
      R i2A = mesh.elem_inv_2A[e];
      for (int c = 0; c < NC; ++c) {
        R rhs = acc[c] - i2A * fc[c] + src[c];
        int64_t idx = (e * NP + i) * NC + c;
        qo[idx] = rhs_only ? rhs : a * qa[idx] + b * qb[idx] + cc * dt * rhs;
      }
    }
  }
  void eval_rhs(const double* qd, double* rhs) override {
    std::vector<R> qi(size_t(Ne) * NP * NC), ro(qi.size());
    for (size_t k = 0; k < qi.size(); ++k) qi[k] = R(qd[k]);
    faces(qi.data());
    vol_lift(qi.data(), nullptr, nullptr, ro.data(), R(0), R(0), R(0), R(0), true);
    for (size_t k = 0; k < ro.size(); ++k) rhs[k] = double(ro[k]);
  }
  void limit_buf(R* qq) {  // bj_limit_full_2d  local_mesh_2d_gpu_limiter.mojo:196-210
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; ++e)
      for (int c = 0; c < NC; ++c) {
        R s = R(0);
        for (int n = 0; n < NP; ++n) s += qq[(e * NP + n) * NC + c] * w[n];
        cmean[e * NC + c] = s;
      }
    const R eps2 = lim_eps * lim_eps;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; ++e) {
      R own = cmean[e * NC], mn = own, mx = own;
      for (int lf = 0; lf < 3; ++lf) {
        int64_t fid = mesh.elem_faces[e * 3 + lf];
        int64_t el = mesh.face_elem[fid * 2], er = mesh.face_elem[fid * 2 + 1];
        int64_t nb = (el == e) ? er : el;
        if (nb == e) continue;
        R a = cmean[nb * NC];
        if (a < mn) mn = a;
        if (a > mx) mx = a;
      }
      R pD = mx - own, nD = own - mn;
      if (pD < R(0)) pD = R(0);
      if (nD < R(0)) nD = R(0);
      R th = R(1);
      for (int n = 0; n < NP; ++n) {
        R dl = qq[(e * NP + n) * NC] - own;
        R da = dl >= R(0) ? dl : -dl;
        if (da <= R(1.0e-30)) continue;
        R D = dl > R(0) ? pD : nD;
        R num = D * D + R(2) * D * da + eps2;
        R den = D * D + R(2) * da * da + D * da + eps2;
        R al = num / den;
        if (al < th) th = al;
      }
      theta[e] = th;
    }
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < Ne * NP * NC; ++t) {
      int64_t e = t / (int64_t(NP) * NC);
      R th = theta[e];
      if (!(th < R(1))) continue;
      int c = int(t % NC);
      R bm = cmean[e * NC + c];
      qq[t] = bm + th * (qq[t] - bm);
    }
  }
  void limit(int which) override { limit_buf(q[which].data()); }
  void enable_limiter(bool on, double eps) override {
    lim_on = on;
    lim_eps = R(eps);
  }
  void stage(int s, double dtd) override {  // ssprk3_stage_plans  ssprk3.mojo:56-78
    R dt = R(dtd);
    R *p0 = q[0].data(), *p1 = q[1].data(), *p2 = q[2].data();
    R *qi, *qa, *qb, *qo, a, b, c;
    if (s == 0) { qi = p0; qa = p0; qb = p0; qo = p1; a = R(1); b = R(0); c = R(1); }
    else if (s == 1) { qi = p1; qa = p0; qb = p1; qo = p2; a = R(0.75); b = R(0.25); c = R(0.25); }
    else { qi = p2; qa = p0; qb = p2; qo = p0; a = R(1.0 / 3.0); b = R(2.0 / 3.0); c = R(2.0 / 3.0); }
    faces(qi);
    vol_lift(qi, qa, qb, qo, a, b, c, dt, false);
    if (lim_on) limit_buf(qo);
  }
  void step(double dt) override {
    for (int s = 0; s < 3; ++s) stage(s, dt);
    // GLM psi damping, operator-split once per step: psi *= exp(-alpha_d dt)
    // (local_mesh_2d_gpu_mhd_glm.mojo:464-485, examples/mhd_alfven_glm_2d_gpu.mojo:240-241)
    if (ph.kind == PHYS_MHD && ph.alpha_d > R(0)) {
      const R decay = R(std::exp(-double(ph.alpha_d) * double(R(dt))));
      R* q0 = q[0].data();
      for (int64_t t = 0; t < Ne * NP; ++t) q0[t * 7 + 6] = q0[t * 7 + 6] * decay;
    }
  }
};

template <typename R>
Solver2DBase* make2(int P, int nx, int ny, double Lx, double Ly, const int* bcs, int kind, int flux, int efix,
                    const double* p) {
  Phys2D<R> ph;
  ph.kind = kind;
  ph.flux = flux;
  ph.entropy_fix = efix != 0;
  if (kind == PHYS_ADVECTION) {
    ph.vx = R(p[0]); ph.vy = R(p[1]); ph.inflow_q = R(p[3]);
  } else if (kind == PHYS_EULER) {
    ph.gamma = R(p[0]); ph.min_density = R(p[1]); ph.min_pressure = R(p[2]);
    ph.gx = R(p[3]); ph.gy = R(p[4]);
    // inflow (rho, rhou, rhov, E): the 3D layout's rhow slot (p[9]) is skipped
    ph.inflow[0] = R(p[6]); ph.inflow[1] = R(p[7]); ph.inflow[2] = R(p[8]); ph.inflow[3] = R(p[10]);
  } else if (kind == PHYS_MAXWELL) {
    ph.c = R(p[0]);
    for (int k = 0; k < 3; ++k) { ph.J[k] = R(p[1 + k]); ph.M[k] = R(p[4 + k]); }
    for (int k = 0; k < 6; ++k) ph.inflow[k] = R(p[7 + k]);
  } else if (kind == PHYS_SW) {
    ph.g = R(p[0]); ph.h_min = R(p[1]);
    for (int k = 0; k < 3; ++k) ph.inflow[k] = R(p[2 + k]);
  } else if (kind == PHYS_MHD || kind == PHYS_MHD_PLAIN) {
    // the 3D IdealMHD parameter layout {gamma, rho_min, p_min, c_h, alpha_d,
    // inflow rho, rhou, rhov, rhow, E, Bx, By, Bz, psi}; 2D state order
    // (rho, mx, my, Bx, By, E[, psi])
    ph.gamma = R(p[0]); ph.min_density = R(p[1]); ph.min_pressure = R(p[2]);
    ph.c_h = R(p[3]); ph.alpha_d = R(p[4]);
    ph.inflow[0] = R(p[5]); ph.inflow[1] = R(p[6]); ph.inflow[2] = R(p[7]); ph.inflow[3] = R(p[10]);
    ph.inflow[4] = R(p[11]); ph.inflow[5] = R(p[9]); ph.inflow[6] = R(p[13]);
  } else {
    throw std::runtime_error("unknown physics kind");
  }
  return new Solver2D<R>(P, nx, ny, Lx, Ly, bcs, ph);
}

}  // namespace orc
