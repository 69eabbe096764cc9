// Kuhn mesh topology tables and fused per-type operators (see refops.hpp).
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "refops.hpp"

namespace mxm {

std::vector<int> reference_face_order(int dim, int P, const RefOps& r) {
  // Element node of each reference face-local slot, then its position in
  // our ascending face order.
  const int NFP = r.NFP;
  std::vector<int> out(r.NF * NFP, -1);
  auto find = [&](const int a[4]) {
    for (int i = 0; i < r.NP; ++i)
      if (r.nodes[i].a[0] == a[0] && r.nodes[i].a[1] == a[1] && r.nodes[i].a[2] == a[2] && r.nodes[i].a[3] == a[3])
        return i;
    return -1;
  };
  for (int f = 0; f < r.NF; ++f) {
    std::vector<int> ref;
    if (dim == 2) {
      const int va = f, vb = (f + 1) % 3;  // edges (0,1) (1,2) (2,0), endpoints included
      for (int k = 0; k <= P; ++k) {
        int a[4] = {0, 0, 0, 0};
        a[va] = P - k;
        a[vb] = k;
        ref.push_back(find(a));
      }
    } else {
      int v[3], c = 0;
      for (int k = 0; k < 4; ++k)
        if (k != f) v[c++] = k;
      for (int l = 0; l < 3; ++l) {
        int a[4] = {0, 0, 0, 0};
        a[v[l]] = P;
        ref.push_back(find(a));
      }
      const int ea[3] = {v[0], v[1], v[2]}, eb[3] = {v[1], v[2], v[0]};
      for (int e = 0; e < 3; ++e)
        for (int k = 1; k < P; ++k) {
          int a[4] = {0, 0, 0, 0};
          a[ea[e]] = P - k;
          a[eb[e]] = k;
          ref.push_back(find(a));
        }
      for (int x = P - 2; x > 0; --x)
        for (int y = P - x - 1; y > 0; --y) {
          int a[4] = {0, 0, 0, 0};
          a[v[0]] = x;
          a[v[1]] = y;
          a[v[2]] = P - x - y;
          ref.push_back(find(a));
        }
    }
    // Reference 2D edge f joins vertices (f, f+1): RefOps face (f+2)%3.
    const int fo = dim == 2 ? (f + 2) % 3 : f;
    for (int m = 0; m < NFP; ++m) {
      int en = ref[m];
      for (int mm = 0; mm < NFP; ++mm)
        if (r.face_nodes[fo * NFP + mm] == en) out[f * NFP + m] = mm;
    }
  }
  return out;
}

namespace {
// Kuhn subdivision of the unit cube into 6 tets around the 0-7 diagonal; the
// tet-type numbering and vertex order fix the element and node layout of the
// state (src/local_mesh.mojo:64-114).  Corner c = x + 2y + 4z.
const int kKuhnCorners[6][4] = {{0, 1, 3, 7}, {0, 3, 2, 7}, {0, 2, 6, 7}, {0, 6, 4, 7}, {0, 4, 5, 7}, {0, 5, 1, 7}};
}  // namespace

Kuhn3D build_kuhn3d(const RefOps& r, double dx, double dy, double dz) {
  Kuhn3D k;
  const int P = r.P, NP = r.NP, NFP = r.NFP;
  for (int t = 0; t < 6; ++t)
    for (int v = 0; v < 4; ++v) {
      int c = kKuhnCorners[t][v];
      k.vert[t][v][0] = c & 1;
      k.vert[t][v][1] = (c >> 1) & 1;
      k.vert[t][v][2] = (c >> 2) & 1;
    }
  // integer node positions scaled by P, in cell units
  auto npos = [&](int t, int n, int o[3]) {
    for (int d = 0; d < 3; ++d) {
      int s = 0;
      for (int v = 0; v < 4; ++v) s += r.nodes[n].a[v] * k.vert[t][v][d];
      o[d] = s;
    }
  };
  const double h[3] = {dx, dy, dz};
  k.rel_xyz.assign(6 * NP * 3, 0.0);
  for (int t = 0; t < 6; ++t)
    for (int n = 0; n < NP; ++n) {
      int o[3];
      npos(t, n, o);
      for (int d = 0; d < 3; ++d) k.rel_xyz[(t * NP + n) * 3 + d] = double(o[d]) / P;
    }
  k.nb_node.assign(6 * 4 * NFP, -1);
  for (int t = 0; t < 6; ++t) {
    // Jacobian columns v1-v0, v2-v0, v3-v0 in physical units
    double J[3][3];
    for (int d = 0; d < 3; ++d)
      for (int c = 0; c < 3; ++c) J[d][c] = (k.vert[t][c + 1][d] - k.vert[t][0][d]) * h[d];
    double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                 J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    if (!(det > 0.0)) throw std::runtime_error("non-positive Kuhn tet Jacobian");
    k.inv6V[t] = 1.0 / det;
    // inverse via adjugate: invJ[k][d] = d r_k / d x_d
    double A[3][3];
    A[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    A[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
    A[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    A[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    A[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
    A[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
    A[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    A[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
    A[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) k.invJ[t][a * 3 + b] = A[a][b] / det;
    for (int lf = 0; lf < 4; ++lf) {
      int fv[3][3], c = 0;
      for (int v = 0; v < 4; ++v)
        if (v != lf) {
          for (int d = 0; d < 3; ++d) fv[c][d] = k.vert[t][v][d];
          ++c;
        }
      // outward normal of this tet's face, area
      double p[3][3];
      for (int a = 0; a < 3; ++a)
        for (int d = 0; d < 3; ++d) p[a][d] = fv[a][d] * h[d];
      double e1[3], e2[3], n[3];
      for (int d = 0; d < 3; ++d) {
        e1[d] = p[1][d] - p[0][d];
        e2[d] = p[2][d] - p[0][d];
      }
      n[0] = e1[1] * e2[2] - e1[2] * e2[1];
      n[1] = e1[2] * e2[0] - e1[0] * e2[2];
      n[2] = e1[0] * e2[1] - e1[1] * e2[0];
      double nl = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      k.area[t][lf] = 0.5 * nl;
      double opp = 0.0;
      for (int d = 0; d < 3; ++d) {
        n[d] /= nl;
        opp += (k.vert[t][lf][d] * h[d] - p[0][d]) * n[d];
      }
      if (opp > 0.0)
        for (int d = 0; d < 3; ++d) n[d] = -n[d];
      // neighbour: the tet of a neighbouring (or the same) cell sharing the face
      bool found = false;
      for (int ox = -1; ox <= 1 && !found; ++ox)
        for (int oy = -1; oy <= 1 && !found; ++oy)
          for (int oz = -1; oz <= 1 && !found; ++oz)
            for (int t2 = 0; t2 < 6 && !found; ++t2) {
              if (ox == 0 && oy == 0 && oz == 0 && t2 == t) continue;
              const int o[3] = {ox, oy, oz};
              for (int lf2 = 0; lf2 < 4 && !found; ++lf2) {
                int hit = 0;
                for (int v = 0; v < 4; ++v) {
                  if (v == lf2) continue;
                  for (int a = 0; a < 3; ++a)
                    if (k.vert[t2][v][0] + o[0] == fv[a][0] && k.vert[t2][v][1] + o[1] == fv[a][1] &&
                        k.vert[t2][v][2] + o[2] == fv[a][2])
                      ++hit;
                }
                if (hit == 3) {
                  found = true;
                  k.nb_t[t][lf] = t2;
                  k.nb_lf[t][lf] = lf2;
                  for (int d = 0; d < 3; ++d) k.off[t][lf][d] = o[d];
                }
              }
            }
      if (!found) throw std::runtime_error("Kuhn face neighbour not found");
      const int* o = k.off[t][lf];
      int ax = -1, dir = 0;
      for (int d = 0; d < 3; ++d)
        if (o[d] != 0) {
          ax = d;
          dir = o[d];
        }
      k.axis[t][lf] = ax;
      k.dir[t][lf] = dir;
      // side: internal faces belong to the lower tet index, cube faces to the lower cell
      k.side[t][lf] = (ax < 0) ? (t < k.nb_t[t][lf] ? 0 : 1) : (dir > 0 ? 0 : 1);
      for (int d = 0; d < 3; ++d) k.normal[t][lf][d] = k.side[t][lf] == 0 ? n[d] : -n[d];
      // node pairing by integer position
      const int t2 = k.nb_t[t][lf];
      for (int m = 0; m < NFP; ++m) {
        int own = r.face_nodes[lf * NFP + m], po[3];
        npos(t, own, po);
        for (int n2 = 0; n2 < NP; ++n2) {
          int p2[3];
          npos(t2, n2, p2);
          if (p2[0] + P * o[0] == po[0] && p2[1] + P * o[1] == po[1] && p2[2] + P * o[2] == po[2]) {
            k.nb_node[(t * 4 + lf) * NFP + m] = n2;
            break;
          }
        }
        if (k.nb_node[(t * 4 + lf) * NFP + m] < 0) throw std::runtime_error("Kuhn face node pairing failed");
      }
    }
  }
  return k;
}

Kuhn2D build_kuhn2d(const RefOps& r, double dx, double dy) {
  // Kuhn split of the unit square along the (0,0)-(1,1) diagonal:
  // T0 = (0,0),(1,0),(1,1); T1 = (0,0),(1,1),(0,1)  (local_mesh_2d.mojo:125-160).
  static const int V[2][3][2] = {{{0, 0}, {1, 0}, {1, 1}}, {{0, 0}, {1, 1}, {0, 1}}};
  Kuhn2D k;
  const int P = r.P, NP = r.NP, NFP = r.NFP;
  for (int t = 0; t < 2; ++t)
    for (int v = 0; v < 3; ++v)
      for (int d = 0; d < 2; ++d) k.vert[t][v][d] = V[t][v][d];
  auto npos = [&](int t, int n, int o[2]) {
    for (int d = 0; d < 2; ++d) {
      int s = 0;
      for (int v = 0; v < 3; ++v) s += r.nodes[n].a[v] * k.vert[t][v][d];
      o[d] = s;
    }
  };
  const double h[2] = {dx, dy};
  k.rel_xy.assign(2 * NP * 2, 0.0);
  for (int t = 0; t < 2; ++t)
    for (int n = 0; n < NP; ++n) {
      int o[2];
      npos(t, n, o);
      for (int d = 0; d < 2; ++d) k.rel_xy[(t * NP + n) * 2 + d] = double(o[d]) / P;
    }
  k.nb_node.assign(2 * 3 * NFP, -1);
  // 2D face numbering: local edge lf joins vertices (lf, lf+1); the face
  // opposite vertex f in RefOps is edge (f+1, f+2).  Map edge -> opposite vertex.
  for (int t = 0; t < 2; ++t) {
    double J00 = (k.vert[t][1][0] - k.vert[t][0][0]) * dx, J01 = (k.vert[t][2][0] - k.vert[t][0][0]) * dx;
    double J10 = (k.vert[t][1][1] - k.vert[t][0][1]) * dy, J11 = (k.vert[t][2][1] - k.vert[t][0][1]) * dy;
    double det = J00 * J11 - J01 * J10;
    if (!(det > 0.0)) throw std::runtime_error("non-positive Kuhn triangle Jacobian");
    k.inv2A[t] = 1.0 / det;
    k.invJ[t][0] = J11 / det;
    k.invJ[t][1] = -J01 / det;
    k.invJ[t][2] = -J10 / det;
    k.invJ[t][3] = J00 / det;
    for (int lf = 0; lf < 3; ++lf) {
      const int va = lf, vb = (lf + 1) % 3, vo = (lf + 2) % 3;
      double ex = (k.vert[t][vb][0] - k.vert[t][va][0]) * dx, ey = (k.vert[t][vb][1] - k.vert[t][va][1]) * dy;
      double len = std::sqrt(ex * ex + ey * ey);
      k.length[t][lf] = len;
      double nx = ey / len, ny = -ex / len;
      double ox = (k.vert[t][vo][0] - k.vert[t][va][0]) * dx, oy = (k.vert[t][vo][1] - k.vert[t][va][1]) * dy;
      if (ox * nx + oy * ny > 0.0) {
        nx = -nx;
        ny = -ny;
      }
      bool found = false;
      for (int ox2 = -1; ox2 <= 1 && !found; ++ox2)
        for (int oy2 = -1; oy2 <= 1 && !found; ++oy2)
          for (int t2 = 0; t2 < 2 && !found; ++t2) {
            if (ox2 == 0 && oy2 == 0 && t2 == t) continue;
            for (int lf2 = 0; lf2 < 3 && !found; ++lf2) {
              const int a2 = lf2, b2 = (lf2 + 1) % 3;
              auto eq = [&](int v2, int v) {
                return k.vert[t2][v2][0] + ox2 == k.vert[t][v][0] && k.vert[t2][v2][1] + oy2 == k.vert[t][v][1];
              };
              if ((eq(a2, va) && eq(b2, vb)) || (eq(a2, vb) && eq(b2, va))) {
                found = true;
                k.nb_t[t][lf] = t2;
                k.nb_lf[t][lf] = lf2;
                k.off[t][lf][0] = ox2;
                k.off[t][lf][1] = oy2;
              }
            }
          }
      if (!found) throw std::runtime_error("Kuhn edge neighbour not found");
      int ax = -1, dir = 0;
      for (int d = 0; d < 2; ++d)
        if (k.off[t][lf][d] != 0) {
          ax = d;
          dir = k.off[t][lf][d];
        }
      k.axis[t][lf] = ax;
      k.dir[t][lf] = dir;
      k.side[t][lf] = (ax < 0) ? (t < k.nb_t[t][lf] ? 0 : 1) : (dir > 0 ? 0 : 1);
      k.normal[t][lf][0] = k.side[t][lf] == 0 ? nx : -nx;
      k.normal[t][lf][1] = k.side[t][lf] == 0 ? ny : -ny;
      const int t2 = k.nb_t[t][lf];
      const int fo = vo;  // RefOps face index = vertex opposite the edge
      for (int m = 0; m < NFP; ++m) {
        int own = r.face_nodes[fo * NFP + m], po[2];
        npos(t, own, po);
        for (int n2 = 0; n2 < NP; ++n2) {
          int p2[2];
          npos(t2, n2, p2);
          if (p2[0] + P * k.off[t][lf][0] == po[0] && p2[1] + P * k.off[t][lf][1] == po[1]) {
            k.nb_node[(t * 3 + lf) * NFP + m] = n2;
            break;
          }
        }
        if (k.nb_node[(t * 3 + lf) * NFP + m] < 0) throw std::runtime_error("Kuhn edge node pairing failed");
      }
    }
  }
  return k;
}

std::vector<double> shared_operator(const RefOps& r) {
  // [D_0 | .. | D_{dim-1} | -Lift_0 | .. | -Lift_{nf-1}]  (NP x K), one
  // operator for every element type.  2D local edge lf joins vertices
  // (lf, lf+1), i.e. RefOps face (lf+2)%3.
  const int NP = r.NP, NFP = r.NFP, dim = r.dim, nf = r.NF, K = dim * NP + nf * NFP;
  std::vector<double> A(size_t(NP) * K, 0.0);
  for (int i = 0; i < NP; ++i) {
    double* row = &A[size_t(i) * K];
    for (int d = 0; d < dim; ++d)
      for (int j = 0; j < NP; ++j) row[d * NP + j] = r.D[(d * NP + i) * NP + j];
    for (int lf = 0; lf < nf; ++lf) {
      const int fo = dim == 2 ? (lf + 2) % 3 : lf;
      for (int m = 0; m < NFP; ++m) row[dim * NP + lf * NFP + m] = -r.Lift[(fo * NP + i) * NFP + m];
    }
  }
  return A;
}

}  // namespace mxm
