// ORACLE — test infrastructure only.  CPU restatement of mojoxm's reference
// elements (3D equispaced Lagrange tetrahedron, 2D triangle) used as the
// parity checker for the CUDA path.  Only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline leg may load it; the product library never does.
//
// Follows src/reference.mojo (3D) and src/reference_2d.mojo (2D) of the
// reference step by step: homogeneous-monomial basis, Vandermonde inverse by
// Gauss-Jordan with partial pivoting, exact Dirichlet-formula integrals.
#pragma once
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <vector>

namespace orc {

inline int num_tet_nodes(int P) { return (P + 1) * (P + 2) * (P + 3) / 6; }  // reference.mojo:60-61
inline int num_tri_nodes(int P) { return (P + 1) * (P + 2) / 2; }            // reference.mojo:64-65

struct Mono {  // reference.mojo:75-81
  int a0, a1, a2, a3;
  double c;
};
using Poly = std::vector<Mono>;

inline Poly poly_mul(const Poly& a, const Poly& b) {  // reference.mojo:84-90
  Poly out;
  out.reserve(a.size() * b.size());
  for (auto& x : a)
    for (auto& y : b) out.push_back({x.a0 + y.a0, x.a1 + y.a1, x.a2 + y.a2, x.a3 + y.a3, x.c * y.c});
  return out;
}

inline double factorial(int n) {  // reference.mojo:93-97
  double f = 1.0;
  for (int k = 2; k <= n; ++k) f *= double(k);
  return f;
}

inline double integrate_ref_tet(const Poly& p) {  // reference.mojo:101-108
  double s = 0.0;
  for (auto& m : p) {
    int dn = m.a0 + m.a1 + m.a2 + m.a3 + 3;
    double num = factorial(m.a0) * factorial(m.a1) * factorial(m.a2) * factorial(m.a3);
    s += m.c * num / factorial(dn);
  }
  return s;
}

inline double integrate_ref_tri(const Poly& p) {  // reference.mojo:113-120
  double s = 0.0;
  for (auto& m : p) {
    int dn = m.a0 + m.a1 + m.a2 + 2;
    double num = factorial(m.a0) * factorial(m.a1) * factorial(m.a2);
    s += m.c * num / factorial(dn);
  }
  return s;
}

// Canonical tet node order: vertices, edges (0,1)(1,2)(2,0)(0,3)(1,3)(2,3),
// face interiors (faces opposite v0..v3), volume interior.
// reference.mojo:136-200
inline std::vector<Mono> tet_node_exponents(int P) {
  const int ea[6] = {0, 1, 2, 0, 1, 2}, eb[6] = {1, 2, 0, 3, 3, 3};
  std::vector<Mono> out;
  out.push_back({P, 0, 0, 0, 0});
  out.push_back({0, P, 0, 0, 0});
  out.push_back({0, 0, P, 0, 0});
  out.push_back({0, 0, 0, P, 0});
  if (P < 2) return out;
  for (int e = 0; e < 6; ++e)
    for (int k = 1; k < P; ++k) {
      int ex[4];
      for (int v = 0; v < 4; ++v) ex[v] = (ea[e] == v) ? P - k : ((eb[e] == v) ? k : 0);
      out.push_back({ex[0], ex[1], ex[2], ex[3], 0});
    }
  if (P < 3) return out;
  for (int f = 0; f < 4; ++f) {
    int ni[3], n = 0;
    for (int i = 0; i < 4; ++i)
      if (i != f) ni[n++] = i;
    for (int a0 = P - 2; a0 > 0; --a0)
      for (int a1 = P - a0 - 1; a1 > 0; --a1) {
        int a2 = P - a0 - a1;
        int ex[4] = {0, 0, 0, 0};
        ex[ni[0]] = a0;
        ex[ni[1]] = a1;
        ex[ni[2]] = a2;
        out.push_back({ex[0], ex[1], ex[2], ex[3], 0});
      }
  }
  if (P < 4) return out;
  for (int a0 = P - 2; a0 > 0; --a0)
    for (int a1 = P - a0 - 1; a1 > 0; --a1)
      for (int a2 = P - a0 - a1 - 1; a2 > 0; --a2) out.push_back({a0, a1, a2, P - a0 - a1 - a2, 0});
  return out;
}

// reference.mojo:203-237
inline std::vector<Mono> tri_node_exponents(int P) {
  std::vector<Mono> out;
  out.push_back({P, 0, 0, 0, 0});
  out.push_back({0, P, 0, 0, 0});
  out.push_back({0, 0, P, 0, 0});
  if (P < 2) return out;
  const int ea[3] = {0, 1, 2}, eb[3] = {1, 2, 0};
  for (int e = 0; e < 3; ++e)
    for (int k = 1; k < P; ++k) {
      int ex[3];
      for (int v = 0; v < 3; ++v) ex[v] = (ea[e] == v) ? P - k : ((eb[e] == v) ? k : 0);
      out.push_back({ex[0], ex[1], ex[2], 0, 0});
    }
  if (P < 3) return out;
  for (int a0 = P - 2; a0 > 0; --a0)
    for (int a1 = P - a0 - 1; a1 > 0; --a1) out.push_back({a0, a1, P - a0 - a1, 0, 0});
  return out;
}

inline std::vector<Mono> tet_degP_monomials(int P) {  // reference.mojo:250-257
  std::vector<Mono> out;
  for (int a0 = 0; a0 <= P; ++a0)
    for (int a1 = 0; a1 <= P - a0; ++a1)
      for (int a2 = 0; a2 <= P - a0 - a1; ++a2) out.push_back({a0, a1, a2, P - a0 - a1 - a2, 1.0});
  return out;
}

inline std::vector<Mono> tri_degP_monomials(int P) {  // reference.mojo:260-266
  std::vector<Mono> out;
  for (int a0 = 0; a0 <= P; ++a0)
    for (int a1 = 0; a1 <= P - a0; ++a1) out.push_back({a0, a1, P - a0 - a1, 0, 1.0});
  return out;
}

// Gauss-Jordan inversion with partial pivoting.  reference.mojo:289-331
inline std::vector<double> mat_inv(const std::vector<double>& m, int n) {
  const int cols = 2 * n;
  std::vector<double> a(size_t(n) * cols);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) a[i * cols + j] = m[i * n + j];
    for (int j = 0; j < n; ++j) a[i * cols + n + j] = (i == j) ? 1.0 : 0.0;
  }
  for (int i = 0; i < n; ++i) {
    int pivot = i;
    double best = 0.0;
    for (int r = i; r < n; ++r) {
      double v = std::fabs(a[r * cols + i]);
      if (v > best) {
        best = v;
        pivot = r;
      }
    }
    if (best == 0.0) throw std::runtime_error("mat_inv: singular matrix");
    if (pivot != i)
      for (int c = 0; c < cols; ++c) std::swap(a[i * cols + c], a[pivot * cols + c]);
    double pv = a[i * cols + i];
    for (int c = 0; c < cols; ++c) a[i * cols + c] /= pv;
    for (int r = 0; r < n; ++r) {
      if (r == i) continue;
      double f = a[r * cols + i];
      if (f == 0.0) continue;
      for (int c = 0; c < cols; ++c) a[r * cols + c] -= f * a[i * cols + c];
    }
  }
  std::vector<double> inv(size_t(n) * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) inv[i * n + j] = a[i * cols + n + j];
  return inv;
}

// C[i,k] with phi_i = sum_k C[i,k] m_k.  reference.mojo:349-387
inline std::vector<double> build_basis_coefs(const std::vector<Mono>& nodes, const std::vector<Mono>& monos, int P) {
  const int N = int(nodes.size());
  if (N != int(monos.size())) throw std::runtime_error("node/monomial count mismatch");
  std::vector<double> V(size_t(N) * N);
  const double Pf = double(P);
  for (int j = 0; j < N; ++j) {
    double l[4] = {nodes[j].a0 / Pf, nodes[j].a1 / Pf, nodes[j].a2 / Pf, nodes[j].a3 / Pf};
    for (int k = 0; k < N; ++k) {
      const Mono& mk = monos[k];
      double v = 1.0;
      for (int t = 0; t < mk.a0; ++t) v *= l[0];
      for (int t = 0; t < mk.a1; ++t) v *= l[1];
      for (int t = 0; t < mk.a2; ++t) v *= l[2];
      for (int t = 0; t < mk.a3; ++t) v *= l[3];
      V[j * N + k] = v;
    }
  }
  auto Vinv = mat_inv(V, N);
  std::vector<double> C(size_t(N) * N);
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < N; ++k) C[i * N + k] = Vinv[k * N + i];
  return C;
}

inline Poly coefs_to_poly(const std::vector<double>& coefs, int i, const std::vector<Mono>& monos) {  // reference.mojo:390-400
  const int N = int(monos.size());
  Poly out;
  for (int k = 0; k < N; ++k) {
    double c = coefs[i * N + k];
    if (c == 0.0) continue;
    out.push_back({monos[k].a0, monos[k].a1, monos[k].a2, monos[k].a3, c});
  }
  return out;
}

// d/dr_k with l0 = 1 - r - s - t.  reference.mojo:411-427
inline Poly poly_drdx(const Poly& p, int k) {
  const double dl0 = -1.0, dl1 = (k == 0) ? 1.0 : 0.0, dl2 = (k == 1) ? 1.0 : 0.0, dl3 = (k == 2) ? 1.0 : 0.0;
  Poly out;
  for (auto& m : p) {
    if (m.a0 > 0) out.push_back({m.a0 - 1, m.a1, m.a2, m.a3, m.c * double(m.a0) * dl0});
    if (m.a1 > 0 && dl1 != 0.0) out.push_back({m.a0, m.a1 - 1, m.a2, m.a3, m.c * double(m.a1) * dl1});
    if (m.a2 > 0 && dl2 != 0.0) out.push_back({m.a0, m.a1, m.a2 - 1, m.a3, m.c * double(m.a2) * dl2});
    if (m.a3 > 0 && dl3 != 0.0) out.push_back({m.a0, m.a1, m.a2, m.a3 - 1, m.c * double(m.a3) * dl3});
  }
  return out;
}

inline int lookup_node(const std::vector<Mono>& nodes, int a0, int a1, int a2, int a3) {  // reference.mojo:444-450
  for (size_t i = 0; i < nodes.size(); ++i)
    if (nodes[i].a0 == a0 && nodes[i].a1 == a1 && nodes[i].a2 == a2 && nodes[i].a3 == a3) return int(i);
  return -1;
}

// face_to_elem[f*NFP + l]: element node of face-local node l on face f.
// reference.mojo:453-511
inline std::vector<int32_t> face_to_element_node(int P, const std::vector<Mono>& tet) {
  const int NFP = num_tri_nodes(P);
  std::vector<int32_t> out(4 * NFP, -1);
  for (int f = 0; f < 4; ++f) {
    const int vA = (f == 0) ? 1 : 0, vB = (f <= 1) ? 2 : 1, vC = (f <= 2) ? 3 : 2;
    const int vv[3] = {vA, vB, vC};
    for (int l = 0; l < 3; ++l) {
      int ex[4] = {0, 0, 0, 0};
      ex[vv[l]] = P;
      out[f * NFP + l] = lookup_node(tet, ex[0], ex[1], ex[2], ex[3]);
    }
    if (P < 2) continue;
    int pos = 3;
    const int ea[3] = {vA, vB, vC}, eb[3] = {vB, vC, vA};
    for (int e = 0; e < 3; ++e)
      for (int k = 1; k < P; ++k) {
        int ex[4];
        for (int v = 0; v < 4; ++v) ex[v] = (ea[e] == v) ? P - k : ((eb[e] == v) ? k : 0);
        out[f * NFP + pos++] = lookup_node(tet, ex[0], ex[1], ex[2], ex[3]);
      }
    if (P < 3) continue;
    for (int a0 = P - 2; a0 > 0; --a0)
      for (int a1 = P - a0 - 1; a1 > 0; --a1) {
        int a2 = P - a0 - a1;
        int ex[4] = {0, 0, 0, 0};
        ex[vA] = a0;
        ex[vB] = a1;
        ex[vC] = a2;
        out[f * NFP + pos++] = lookup_node(tet, ex[0], ex[1], ex[2], ex[3]);
      }
  }
  return out;
}

// ReferenceElement[P].__init__  reference.mojo:519-659
struct RefElem3D {
  int P, NP, NFP;
  std::vector<double> node_pos;      // [NP*3] (r,s,t)
  std::vector<double> D;             // [3*NP*NP]
  std::vector<double> Lift;          // [4*NP*NFP]
  std::vector<double> Minv;          // [NP*NP]
  std::vector<int32_t> face_to_elem; // [4*NFP]
  std::vector<double> w;             // [NP]
  std::vector<double> M, M_tri;
  explicit RefElem3D(int P_) : P(P_), NP(num_tet_nodes(P_)), NFP(num_tri_nodes(P_)) {
    auto tet = tet_node_exponents(P);
    auto tri = tri_node_exponents(P);
    if (int(tet.size()) != NP || int(tri.size()) != NFP) throw std::runtime_error("node count mismatch");
    const double Pf = double(P);
    for (auto& n : tet) {
      node_pos.push_back(n.a1 / Pf);
      node_pos.push_back(n.a2 / Pf);
      node_pos.push_back(n.a3 / Pf);
    }
    auto tet_m = tet_degP_monomials(P), tri_m = tri_degP_monomials(P);
    auto tc = build_basis_coefs(tet, tet_m, P), trc = build_basis_coefs(tri, tri_m, P);
    std::vector<Poly> phi, tphi;
    for (int i = 0; i < NP; ++i) phi.push_back(coefs_to_poly(tc, i, tet_m));
    for (int i = 0; i < NFP; ++i) tphi.push_back(coefs_to_poly(trc, i, tri_m));
    M.assign(size_t(NP) * NP, 0.0);
    for (int i = 0; i < NP; ++i)
      for (int j = 0; j < NP; ++j) M[i * NP + j] = integrate_ref_tet(poly_mul(phi[i], phi[j]));
    Minv = mat_inv(M, NP);
    std::vector<double> S(size_t(3) * NP * NP);
    for (int k = 0; k < 3; ++k)
      for (int i = 0; i < NP; ++i) {
        auto dpi = poly_drdx(phi[i], k);
        for (int j = 0; j < NP; ++j) S[k * NP * NP + i * NP + j] = integrate_ref_tet(poly_mul(dpi, phi[j]));
      }
    D.assign(size_t(3) * NP * NP, 0.0);
    for (int k = 0; k < 3; ++k)
      for (int i = 0; i < NP; ++i)
        for (int j = 0; j < NP; ++j) {
          double s = 0.0;
          for (int ip = 0; ip < NP; ++ip) s += Minv[i * NP + ip] * S[k * NP * NP + ip * NP + j];
          D[k * NP * NP + i * NP + j] = s;
        }
    M_tri.assign(size_t(NFP) * NFP, 0.0);
    for (int i = 0; i < NFP; ++i)
      for (int j = 0; j < NFP; ++j) M_tri[i * NFP + j] = integrate_ref_tri(poly_mul(tphi[i], tphi[j]));
    face_to_elem = face_to_element_node(P, tet);
    std::vector<double> Lraw(size_t(4) * NP * NFP, 0.0);
    for (int f = 0; f < 4; ++f)
      for (int l = 0; l < NFP; ++l) {
        int i = face_to_elem[f * NFP + l];
        if (i < 0) throw std::runtime_error("face_to_elem lookup failed");
        for (int m = 0; m < NFP; ++m) Lraw[f * NP * NFP + i * NFP + m] = 2.0 * M_tri[l * NFP + m];
      }
    Lift.assign(size_t(4) * NP * NFP, 0.0);
    for (int f = 0; f < 4; ++f)
      for (int i = 0; i < NP; ++i)
        for (int m = 0; m < NFP; ++m) {
          double s = 0.0;
          for (int ip = 0; ip < NP; ++ip) s += Minv[i * NP + ip] * Lraw[f * NP * NFP + ip * NFP + m];
          Lift[f * NP * NFP + i * NFP + m] = s;
        }
    for (int i = 0; i < NP; ++i) w.push_back(integrate_ref_tet(phi[i]) / (1.0 / 6.0));
  }
};

}  // namespace orc

namespace orc {

// 2D triangle reference element.  src/reference_2d.mojo:87-306
inline std::vector<int32_t> edge_to_element_node(int P, const std::vector<Mono>& tri) {  // reference_2d.mojo:87-127
  const int NE = P + 1;
  std::vector<int32_t> out(3 * NE, -1);
  const int va[3] = {0, 1, 2}, vb[3] = {1, 2, 0};
  for (int e = 0; e < 3; ++e)
    for (int k = 0; k < NE; ++k) {
      int ex[3];
      for (int v = 0; v < 3; ++v) ex[v] = (va[e] == v) ? (P - k) : ((vb[e] == v) ? k : 0);
      int i = lookup_node(tri, ex[0], ex[1], ex[2], 0);
      if (i < 0) throw std::runtime_error("edge_to_element_node lookup failed");
      out[e * NE + k] = i;
    }
  return out;
}

inline std::vector<double> edge_mass_matrix(int P) {  // reference_2d.mojo:278-306
  const int NE = P + 1;
  std::vector<double> V(NE * NE);
  for (int k = 0; k < NE; ++k) {
    double xik = double(k) / double(P), pw = 1.0;
    for (int j = 0; j < NE; ++j) {
      V[k * NE + j] = pw;
      pw *= xik;
    }
  }
  auto C = mat_inv(V, NE);
  std::vector<double> M(NE * NE);
  for (int k = 0; k < NE; ++k)
    for (int l = 0; l < NE; ++l) {
      double s = 0.0;
      for (int i = 0; i < NE; ++i)
        for (int j = 0; j < NE; ++j) s += C[i * NE + k] * C[j * NE + l] / double(i + j + 1);
      M[k * NE + l] = s;
    }
  return M;
}

struct RefElem2D {  // ReferenceElement2D[P].__init__  reference_2d.mojo:157-275
  int P, NP, NFP;
  std::vector<double> node_pos, Dr, Ds, Lift, Minv, w;
  std::vector<int32_t> edge_to_elem;
  explicit RefElem2D(int P_) : P(P_), NP(num_tri_nodes(P_)), NFP(P_ + 1) {
    auto tri = tri_node_exponents(P);
    const double Pf = double(P);
    for (auto& n : tri) {
      node_pos.push_back(n.a1 / Pf);
      node_pos.push_back(n.a2 / Pf);
    }
    auto mon = tri_degP_monomials(P);
    auto co = build_basis_coefs(tri, mon, P);
    std::vector<Poly> phi;
    for (int i = 0; i < NP; ++i) phi.push_back(coefs_to_poly(co, i, mon));
    std::vector<double> M(NP * NP);
    for (int i = 0; i < NP; ++i)
      for (int j = 0; j < NP; ++j) M[i * NP + j] = integrate_ref_tri(poly_mul(phi[i], phi[j]));
    Minv = mat_inv(M, NP);
    for (int i = 0; i < NP; ++i) w.push_back(2.0 * integrate_ref_tri(phi[i]));
    std::vector<double> S(2 * NP * NP);
    for (int k = 0; k < 2; ++k)
      for (int i = 0; i < NP; ++i) {
        auto dpi = poly_drdx(phi[i], k);
        for (int j = 0; j < NP; ++j) S[k * NP * NP + i * NP + j] = integrate_ref_tri(poly_mul(dpi, phi[j]));
      }
    Dr.assign(NP * NP, 0.0);
    Ds.assign(NP * NP, 0.0);
    for (int k = 0; k < 2; ++k)
      for (int i = 0; i < NP; ++i)
        for (int j = 0; j < NP; ++j) {
          double s = 0.0;
          for (int ip = 0; ip < NP; ++ip) s += Minv[i * NP + ip] * S[k * NP * NP + ip * NP + j];
          (k == 0 ? Dr : Ds)[i * NP + j] = s;
        }
    auto Me = edge_mass_matrix(P);
    edge_to_elem = edge_to_element_node(P, tri);
    std::vector<double> Lraw(3 * NP * NFP, 0.0);
    for (int e = 0; e < 3; ++e)
      for (int l = 0; l < NFP; ++l) {
        int i = edge_to_elem[e * NFP + l];
        for (int m = 0; m < NFP; ++m) Lraw[e * NP * NFP + i * NFP + m] = Me[l * NFP + m];
      }
    Lift.assign(3 * NP * NFP, 0.0);
    for (int e = 0; e < 3; ++e)
      for (int i = 0; i < NP; ++i)
        for (int m = 0; m < NFP; ++m) {
          double s = 0.0;
          for (int ip = 0; ip < NP; ++ip) s += Minv[i * NP + ip] * Lraw[e * NP * NFP + ip * NFP + m];
          Lift[e * NP * NFP + i * NFP + m] = s;
        }
  }
};

}  // namespace orc
