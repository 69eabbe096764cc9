// ORACLE — test infrastructure only (see refelem.hpp header).
// CPU restatement of mojoxm's periodic Kuhn-tetrahedron mesh builder with the
// boundary-condition overlay, producing the same device arrays the reference
// kernels read (elem_faces, face_elem, face_elem_node, elem_canon_to_ref,
// face normals/areas, per-element invJ and 1/(6V)).
// Follows src/local_mesh.mojo:64-769 (tables), :777-898 (element/face build
// kernels), :946-1187 (BC overlays), :1241-1485 (LocalMesh); np=1 identity
// ordering from src/mesh.mojo:362-408; BC codes from src/boundary.mojo:310-313.
#pragma once
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "refelem.hpp"

namespace orc {

enum { BC_INTERIOR = 0, BC_WALL = 1, BC_OUTFLOW = 2, BC_INFLOW = 3 };

inline int kuhn_vertex(int t, int k) {  // local_mesh.mojo:64-114
  static const int tab[6][4] = {{0, 1, 3, 7}, {0, 3, 2, 7}, {0, 2, 6, 7}, {0, 6, 4, 7}, {0, 4, 5, 7}, {0, 5, 1, 7}};
  return tab[t][k];
}
inline int corner_dx(int c) { return (c == 1 || c == 3 || c == 5 || c == 7) ? 1 : 0; }  // :117-120
inline int corner_dy(int c) { return (c == 2 || c == 3 || c == 6 || c == 7) ? 1 : 0; }  // :123-126
inline int corner_dz(int c) { return c >= 4 ? 1 : 0; }                                  // :129-132

struct TetFaceInfo {
  int face_type, di, dj, dk, side;
};
inline TetFaceInfo tet_face_info(int t, int f) {  // local_mesh.mojo:168-217
  static const TetFaceInfo tab[6][4] = {
      {{6, 0, 0, 0, 0}, {1, 0, 0, 0, 0}, {0, 0, 0, 0, 0}, {11, 0, 0, -1, 1}},
      {{8, 0, 0, 0, 0}, {2, 0, 0, 0, 0}, {1, 0, 0, 0, 1}, {10, 0, 0, -1, 1}},
      {{9, 0, 0, 0, 0}, {3, 0, 0, 0, 0}, {2, 0, 0, 0, 1}, {6, -1, 0, 0, 1}},
      {{10, 0, 0, 0, 0}, {4, 0, 0, 0, 0}, {3, 0, 0, 0, 1}, {7, -1, 0, 0, 1}},
      {{11, 0, 0, 0, 0}, {5, 0, 0, 0, 0}, {4, 0, 0, 0, 1}, {9, 0, -1, 0, 1}},
      {{7, 0, 0, 0, 0}, {0, 0, 0, 0, 1}, {5, 0, 0, 0, 1}, {8, 0, -1, 0, 1}},
  };
  return tab[t][f];
}
inline int face_type_corner(int ft, int idx) {  // local_mesh.mojo:220-292
  static const int tab[12][3] = {{0, 1, 7}, {0, 3, 7}, {0, 2, 7}, {0, 6, 7}, {0, 4, 7}, {0, 5, 7},
                                 {1, 3, 7}, {1, 5, 7}, {2, 3, 7}, {2, 6, 7}, {4, 6, 7}, {4, 5, 7}};
  return tab[ft][idx];
}

// Face-canonical barycentric weights of canon index m.  local_mesh.mojo:401-455
inline void canon_face_barycentric(int m, int P, int b[3]) {
  if (m < 3) {
    b[0] = b[1] = b[2] = 0;
    b[m] = P;
    return;
  }
  const int el = P - 1;
  if (m < 3 + 3 * el) {
    int which = (m - 3) / el, k = (m - 3) % el + 1;
    if (which == 0) { b[0] = P - k; b[1] = k; b[2] = 0; }
    else if (which == 1) { b[0] = 0; b[1] = P - k; b[2] = k; }
    else { b[0] = k; b[1] = 0; b[2] = P - k; }
    return;
  }
  int idx = 3 + 3 * el;
  for (int b0 = P - 2; b0 > 0; --b0)
    for (int b1 = P - b0 - 1; b1 > 0; --b1) {
      if (idx == m) {
        b[0] = b0; b[1] = b1; b[2] = P - b0 - b1;
        return;
      }
      ++idx;
    }
  throw std::runtime_error("canon_face_barycentric: index out of range");
}

template <typename Real>
struct MeshTables {  // local_mesh.mojo:481-495
  std::vector<Real> tet_invJ, tet_inv_6V, tet_node_rel_xyz;
  std::vector<int32_t> tet_face_type, tet_face_off, tet_face_side, tet_canon_to_ref;
  std::vector<int32_t> ft_side0_tet, ft_side1_tet, ft_side1_off, ft_elem_node;
  std::vector<Real> ft_normal, ft_area;
};

// local_mesh.mojo:498-769
template <typename Real>
MeshTables<Real> compute_tables(Real dx, Real dy, Real dz, int P) {
  const int NP = num_tet_nodes(P), NFP = num_tri_nodes(P);
  RefElem3D re(P);
  const auto& rfn = re.face_to_elem;
  auto tne = tet_node_exponents(P);
  MeshTables<Real> T;
  T.tet_invJ.assign(54, Real(0));
  T.tet_inv_6V.assign(6, Real(0));
  T.tet_node_rel_xyz.assign(6 * NP * 3, Real(0));
  for (int t = 0; t < 6; ++t) {
    Real vx[4], vy[4], vz[4];
    for (int k = 0; k < 4; ++k) {
      int c = kuhn_vertex(t, k);
      vx[k] = Real(corner_dx(c));
      vy[k] = Real(corner_dy(c));
      vz[k] = Real(corner_dz(c));
    }
    Real J[9];
    J[0] = (vx[1] - vx[0]) * dx; J[1] = (vx[2] - vx[0]) * dx; J[2] = (vx[3] - vx[0]) * dx;
    J[3] = (vy[1] - vy[0]) * dy; J[4] = (vy[2] - vy[0]) * dy; J[5] = (vy[3] - vy[0]) * dy;
    J[6] = (vz[1] - vz[0]) * dz; J[7] = (vz[2] - vz[0]) * dz; J[8] = (vz[3] - vz[0]) * dz;
    Real det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) + J[2] * (J[3] * J[7] - J[4] * J[6]);
    if (!(det > Real(0))) throw std::runtime_error("non-positive Jacobian in tet template");
    Real V = det / Real(6);
    T.tet_inv_6V[t] = Real(1) / (Real(6) * V);
    Real* iJ = &T.tet_invJ[t * 9];
    iJ[0] = (J[4] * J[8] - J[5] * J[7]) / det;
    iJ[1] = (J[2] * J[7] - J[1] * J[8]) / det;
    iJ[2] = (J[1] * J[5] - J[2] * J[4]) / det;
    iJ[3] = (J[5] * J[6] - J[3] * J[8]) / det;
    iJ[4] = (J[0] * J[8] - J[2] * J[6]) / det;
    iJ[5] = (J[2] * J[3] - J[0] * J[5]) / det;
    iJ[6] = (J[3] * J[7] - J[4] * J[6]) / det;
    iJ[7] = (J[1] * J[6] - J[0] * J[7]) / det;
    iJ[8] = (J[0] * J[4] - J[1] * J[3]) / det;
    const Real Pf = Real(P);
    for (int n = 0; n < NP; ++n) {
      Real w0 = Real(tne[n].a0) / Pf, w1 = Real(tne[n].a1) / Pf, w2 = Real(tne[n].a2) / Pf, w3 = Real(tne[n].a3) / Pf;
      T.tet_node_rel_xyz[(t * NP + n) * 3 + 0] = w0 * vx[0] + w1 * vx[1] + w2 * vx[2] + w3 * vx[3];
      T.tet_node_rel_xyz[(t * NP + n) * 3 + 1] = w0 * vy[0] + w1 * vy[1] + w2 * vy[2] + w3 * vy[3];
      T.tet_node_rel_xyz[(t * NP + n) * 3 + 2] = w0 * vz[0] + w1 * vz[1] + w2 * vz[2] + w3 * vz[3];
    }
  }
  T.tet_face_type.assign(24, 0);
  T.tet_face_off.assign(72, 0);
  T.tet_face_side.assign(24, 0);
  T.tet_canon_to_ref.assign(24 * NFP, 0);
  std::vector<int32_t> cnode(24 * NFP, 0);
  for (int t = 0; t < 6; ++t)
    for (int f = 0; f < 4; ++f) {
      TetFaceInfo info = tet_face_info(t, f);
      const int ft = info.face_type;
      T.tet_face_type[t * 4 + f] = ft;
      T.tet_face_off[(t * 4 + f) * 3 + 0] = info.di;
      T.tet_face_off[(t * 4 + f) * 3 + 1] = info.dj;
      T.tet_face_off[(t * 4 + f) * 3 + 2] = info.dk;
      T.tet_face_side[t * 4 + f] = info.side;
      int fv[3], n = 0;
      for (int k = 0; k < 4; ++k)
        if (k != f) fv[n++] = k;
      int owner_cube[3];
      for (int kk = 0; kk < 3; ++kk) {
        int cc = kuhn_vertex(t, fv[kk]);
        if (info.di == -1) cc ^= 1;
        if (info.dj == -1) cc ^= 2;
        if (info.dk == -1) cc ^= 4;
        owner_cube[kk] = cc;
      }
      int canon[3] = {face_type_corner(ft, 0), face_type_corner(ft, 1), face_type_corner(ft, 2)};
      int c2r_vertex[3] = {-1, -1, -1};
      for (int k = 0; k < 3; ++k)
        for (int ii = 0; ii < 3; ++ii)
          if (owner_cube[ii] == canon[k]) {
            c2r_vertex[k] = ii;
            break;
          }
      for (int m = 0; m < NFP; ++m) {
        int b[3];
        canon_face_barycentric(m, P, b);
        int w_at_fv[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k) w_at_fv[c2r_vertex[k]] = b[k];
        int a[4] = {0, 0, 0, 0};
        for (int ii = 0; ii < 3; ++ii) a[fv[ii]] = w_at_fv[ii];
        int tn = lookup_node(tne, a[0], a[1], a[2], a[3]);
        if (tn < 0) throw std::runtime_error("find_tet_node failed");
        cnode[(t * 4 + f) * NFP + m] = tn;
        int ref_m = -1;
        for (int mm = 0; mm < NFP; ++mm)
          if (rfn[f * NFP + mm] == tn) {
            ref_m = mm;
            break;
          }
        if (ref_m < 0) throw std::runtime_error("canon-to-ref lookup failed");
        T.tet_canon_to_ref[(t * 4 + f) * NFP + m] = ref_m;
      }
    }
  T.ft_side0_tet.assign(12, 0);
  T.ft_side1_tet.assign(12, 0);
  T.ft_side1_off.assign(36, 0);
  std::vector<int> s0lf(12, 0), s1lf(12, 0);
  for (int t = 0; t < 6; ++t)
    for (int f = 0; f < 4; ++f) {
      TetFaceInfo info = tet_face_info(t, f);
      if (info.side == 0) {
        T.ft_side0_tet[info.face_type] = t;
        s0lf[info.face_type] = f;
      } else {
        T.ft_side1_tet[info.face_type] = t;
        s1lf[info.face_type] = f;
        T.ft_side1_off[info.face_type * 3 + 0] = -info.di;
        T.ft_side1_off[info.face_type * 3 + 1] = -info.dj;
        T.ft_side1_off[info.face_type * 3 + 2] = -info.dk;
      }
    }
  T.ft_normal.assign(36, Real(0));
  T.ft_area.assign(12, Real(0));
  for (int ft = 0; ft < 12; ++ft) {
    int c0 = face_type_corner(ft, 0), c1 = face_type_corner(ft, 1), c2 = face_type_corner(ft, 2);
    Real p0x = Real(corner_dx(c0)) * dx, p0y = Real(corner_dy(c0)) * dy, p0z = Real(corner_dz(c0)) * dz;
    Real p1x = Real(corner_dx(c1)) * dx, p1y = Real(corner_dy(c1)) * dy, p1z = Real(corner_dz(c1)) * dz;
    Real p2x = Real(corner_dx(c2)) * dx, p2y = Real(corner_dy(c2)) * dy, p2z = Real(corner_dz(c2)) * dz;
    Real e1x = p1x - p0x, e1y = p1y - p0y, e1z = p1z - p0z;
    Real e2x = p2x - p0x, e2y = p2y - p0y, e2z = p2z - p0z;
    Real nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    Real nl = std::sqrt(nx * nx + ny * ny + nz * nz);
    Real area = Real(0.5) * nl;
    nx = nx / nl; ny = ny / nl; nz = nz / nl;
    int t0 = T.ft_side0_tet[ft], f0 = s0lf[ft];
    int v4 = kuhn_vertex(t0, f0);
    Real v4x = Real(corner_dx(v4)) * dx, v4y = Real(corner_dy(v4)) * dy, v4z = Real(corner_dz(v4)) * dz;
    Real dn = (v4x - p0x) * nx + (v4y - p0y) * ny + (v4z - p0z) * nz;
    if (dn > Real(0)) { nx = -nx; ny = -ny; nz = -nz; }
    T.ft_normal[ft * 3 + 0] = nx;
    T.ft_normal[ft * 3 + 1] = ny;
    T.ft_normal[ft * 3 + 2] = nz;
    T.ft_area[ft] = area;
  }
  T.ft_elem_node.assign(24 * NFP, 0);
  for (int ft = 0; ft < 12; ++ft) {
    int t0 = T.ft_side0_tet[ft], f0 = s0lf[ft], t1 = T.ft_side1_tet[ft], f1 = s1lf[ft];
    for (int m = 0; m < NFP; ++m) {
      T.ft_elem_node[(ft * 2 + 0) * NFP + m] = cnode[(t0 * 4 + f0) * NFP + m];
      T.ft_elem_node[(ft * 2 + 1) * NFP + m] = cnode[(t1 * 4 + f1) * NFP + m];
    }
  }
  return T;
}

// LocalMesh + BC overlay, single patch (bnd_off = 0).
template <typename Real>
struct Mesh3D {
  int P, NP, NFP, Nx, Ny, Nz;
  int bc[6];  // -x, +x, -y, +y, -z, +z   (boundary.mojo:328-333)
  int64_t Ne, Nf;
  Real dx, dy, dz;
  std::vector<Real> elem_node_xyz, elem_invJ, elem_inv_6V, face_normal, face_area;
  std::vector<int32_t> elem_faces, elem_face_side, elem_canon_to_ref, face_elem, face_elem_node, face_bc_type;

  Mesh3D(int P_, int nx, int ny, int nz, double Lx, double Ly, double Lz, const int bcs[6])
      : P(P_), NP(num_tet_nodes(P_)), NFP(num_tri_nodes(P_)), Nx(nx), Ny(ny), Nz(nz) {
    for (int i = 0; i < 6; ++i) bc[i] = bcs[i];
    Ne = int64_t(Nx) * Ny * Nz * 6;
    const int64_t nf_per = int64_t(Nx) * Ny * Nz * 12;
    const int64_t ex_mx = bc[0] ? 2LL * Ny * Nz : 0, ex_my = bc[2] ? 2LL * Nx * Nz : 0, ex_mz = bc[4] ? 2LL * Nx * Ny : 0;
    Nf = nf_per + ex_mx + ex_my + ex_mz;
    dx = Real(Lx / double(Nx));
    dy = Real(Ly / double(Ny));
    dz = Real(Lz / double(Nz));
    auto T = compute_tables<Real>(dx, dy, dz, P);
    elem_node_xyz.assign(Ne * NP * 3, Real(0));
    elem_invJ.assign(Ne * 9, Real(0));
    elem_inv_6V.assign(Ne, Real(0));
    elem_faces.assign(Ne * 4, 0);
    elem_face_side.assign(Ne * 4, 0);
    elem_canon_to_ref.assign(Ne * 4 * NFP, 0);
    face_elem.assign(Nf * 2, 0);
    face_elem_node.assign(Nf * 2 * NFP, 0);
    face_normal.assign(Nf * 3, Real(0));
    face_area.assign(Nf, Real(0));
    face_bc_type.assign(Nf, 0);
    // build_elements_kernel  local_mesh.mojo:777-845
    for (int64_t e = 0; e < Ne; ++e) {
      int t = int(e % 6);
      int64_t cell = e / 6;
      int k = int(cell / (int64_t(Nx) * Ny));
      int64_t rem = cell - int64_t(k) * Nx * Ny;
      int j = int(rem / Nx), i = int(rem - int64_t(j) * Nx);
      Real ox = Real(i) * dx, oy = Real(j) * dy, oz = Real(k) * dz;
      for (int n = 0; n < NP; ++n) {
        elem_node_xyz[(e * NP + n) * 3 + 0] = ox + T.tet_node_rel_xyz[(t * NP + n) * 3 + 0] * dx;
        elem_node_xyz[(e * NP + n) * 3 + 1] = oy + T.tet_node_rel_xyz[(t * NP + n) * 3 + 1] * dy;
        elem_node_xyz[(e * NP + n) * 3 + 2] = oz + T.tet_node_rel_xyz[(t * NP + n) * 3 + 2] * dz;
      }
      for (int q = 0; q < 9; ++q) elem_invJ[e * 9 + q] = T.tet_invJ[t * 9 + q];
      elem_inv_6V[e] = T.tet_inv_6V[t];
      for (int lf = 0; lf < 4; ++lf) {
        int ft = T.tet_face_type[t * 4 + lf];
        int oi = (i + T.tet_face_off[(t * 4 + lf) * 3 + 0] + Nx) % Nx;
        int oj = (j + T.tet_face_off[(t * 4 + lf) * 3 + 1] + Ny) % Ny;
        int ok = (k + T.tet_face_off[(t * 4 + lf) * 3 + 2] + Nz) % Nz;
        int64_t owner = oi + int64_t(Nx) * (oj + int64_t(Ny) * ok);
        elem_faces[e * 4 + lf] = int32_t(owner * 12 + ft);
        elem_face_side[e * 4 + lf] = T.tet_face_side[t * 4 + lf];
        for (int m = 0; m < NFP; ++m) elem_canon_to_ref[(e * 4 + lf) * NFP + m] = T.tet_canon_to_ref[(t * 4 + lf) * NFP + m];
      }
    }
    // build_faces_kernel  local_mesh.mojo:848-898
    for (int64_t f = 0; f < nf_per; ++f) {
      int ft = int(f % 12);
      int64_t cell = f / 12;
      int k = int(cell / (int64_t(Nx) * Ny));
      int64_t rem = cell - int64_t(k) * Nx * Ny;
      int j = int(rem / Nx), i = int(rem - int64_t(j) * Nx);
      face_elem[f * 2 + 0] = int32_t(cell * 6 + T.ft_side0_tet[ft]);
      int si = (i + T.ft_side1_off[ft * 3 + 0] + Nx) % Nx;
      int sj = (j + T.ft_side1_off[ft * 3 + 1] + Ny) % Ny;
      int sk = (k + T.ft_side1_off[ft * 3 + 2] + Nz) % Nz;
      int64_t s1 = si + int64_t(Nx) * (sj + int64_t(Ny) * sk);
      face_elem[f * 2 + 1] = int32_t(s1 * 6 + T.ft_side1_tet[ft]);
      for (int d = 0; d < 3; ++d) face_normal[f * 3 + d] = T.ft_normal[ft * 3 + d];
      face_area[f] = T.ft_area[ft];
      for (int m = 0; m < NFP; ++m) {
        face_elem_node[(f * 2 + 0) * NFP + m] = T.ft_elem_node[(ft * 2 + 0) * NFP + m];
        face_elem_node[(f * 2 + 1) * NFP + m] = T.ft_elem_node[(ft * 2 + 1) * NFP + m];
      }
    }
    // BC overlay, order as LocalMesh.__init__  local_mesh.mojo:1363-1473
    bool all_periodic = true;
    for (int q = 0; q < 6; ++q) all_periodic &= (bc[q] == BC_INTERIOR);
    if (all_periodic) return;
    const int64_t mx_base = nf_per, my_base = mx_base + ex_mx, mz_base = my_base + ex_my;
    auto plus = [&](int64_t fid, int v) {  // apply_plus_*_bc_kernel  :946-1007
      face_elem[fid * 2 + 1] = face_elem[fid * 2 + 0];
      face_bc_type[fid] = v;
    };
    if (bc[1])
      for (int tid = 0; tid < 2 * Ny * Nz; ++tid) {
        int fo = tid % 2, jk = tid / 2, kk = jk % Nz, jj = jk / Nz;
        int64_t cube = (Nx - 1) + int64_t(Nx) * (jj + int64_t(Ny) * kk);
        plus(cube * 12 + 6 + fo, bc[1]);
      }
    if (bc[3])
      for (int tid = 0; tid < 2 * Nx * Nz; ++tid) {
        int fo = tid % 2, ik = tid / 2, kk = ik % Nz, ii = ik / Nz;
        int64_t cube = ii + int64_t(Nx) * ((Ny - 1) + int64_t(Ny) * kk);
        plus(cube * 12 + 8 + fo, bc[3]);
      }
    if (bc[5])
      for (int tid = 0; tid < 2 * Nx * Ny; ++tid) {
        int fo = tid % 2, ij = tid / 2, jj = ij % Ny, ii = ij / Ny;
        int64_t cube = ii + int64_t(Nx) * (jj + int64_t(Ny) * (Nz - 1));
        plus(cube * 12 + 10 + fo, bc[5]);
      }
    auto minus = [&](int64_t new_fid, int64_t elem, int ft, int v) {  // apply_minus_*_bc_kernel  :1022-1187
      face_elem[new_fid * 2 + 0] = int32_t(elem);
      face_elem[new_fid * 2 + 1] = int32_t(elem);
      for (int m = 0; m < NFP; ++m) {
        int pat = T.ft_elem_node[(ft * 2 + 1) * NFP + m];
        face_elem_node[(new_fid * 2 + 0) * NFP + m] = pat;
        face_elem_node[(new_fid * 2 + 1) * NFP + m] = pat;
      }
      for (int d = 0; d < 3; ++d) face_normal[new_fid * 3 + d] = -T.ft_normal[ft * 3 + d];
      face_area[new_fid] = T.ft_area[ft];
      face_bc_type[new_fid] = v;
      elem_faces[elem * 4 + 3] = int32_t(new_fid);
      elem_face_side[elem * 4 + 3] = 0;
    };
    if (bc[0])
      for (int tid = 0; tid < 2 * Ny * Nz; ++tid) {
        int fo = tid % 2, jk = tid / 2, kk = jk % Nz, jj = jk / Nz;
        int64_t cube = 0 + int64_t(Nx) * (jj + int64_t(Ny) * kk);
        minus(mx_base + tid, cube * 6 + 2 + fo, 6 + fo, bc[0]);
      }
    if (bc[2])
      for (int tid = 0; tid < 2 * Nx * Nz; ++tid) {
        int fo = tid % 2, ik = tid / 2, kk = ik % Nz, ii = ik / Nz;
        int64_t cube = ii + int64_t(Nx) * (0 + int64_t(Ny) * kk);
        minus(my_base + tid, cube * 6 + 5 - fo, 8 + fo, bc[2]);
      }
    if (bc[4])
      for (int tid = 0; tid < 2 * Nx * Ny; ++tid) {
        int fo = tid % 2, ij = tid / 2, jj = ij % Ny, ii = ij / Ny;
        int64_t cube = ii + int64_t(Nx) * (jj + int64_t(Ny) * 0);
        minus(mz_base + tid, cube * 6 + 1 - fo, 10 + fo, bc[4]);
      }
  }
};

}  // namespace orc
