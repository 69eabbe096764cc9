// Host reference operators (see refops.hpp), computed in binary128
// (__float128) and rounded once to FP64.
//
// The monomial/Vandermonde route on equispaced simplex nodes loses about
// log10(cond) digits (~7 at P = 5 in FP64); carrying 113-bit mantissas keeps
// the rounded FP64 operators at full precision for every P in 1..5.  This
// file is compiled by the host compiler (not nvcc) because of __float128.
#include <map>
#include <mutex>
#include <stdexcept>
#include <utility>

#include "refops.hpp"

namespace mxm {
namespace {

using Q = __float128;

Q qabs(Q x) { return x < 0 ? -x : x; }

Q qfact(int n) {
  Q f = 1;
  for (int k = 2; k <= n; ++k) f *= k;
  return f;
}

Q qpow(Q x, int e) {
  Q r = 1;
  for (int k = 0; k < e; ++k) r *= x;
  return r;
}

// LU with partial pivoting: A X = B, B is n x m, solved in place.
void lu_solve(std::vector<Q> A, int n, std::vector<Q>& B, int m) {
  for (int c = 0; c < n; ++c) {
    int p = c;
    Q best = qabs(A[c * n + c]);
    for (int r = c + 1; r < n; ++r)
      if (qabs(A[r * n + c]) > best) {
        best = qabs(A[r * n + c]);
        p = r;
      }
    if (best == 0) throw std::runtime_error("singular operator matrix");
    if (p != c) {
      for (int k = 0; k < n; ++k) std::swap(A[c * n + k], A[p * n + k]);
      for (int k = 0; k < m; ++k) std::swap(B[c * m + k], B[p * m + k]);
    }
    for (int r = c + 1; r < n; ++r) {
      Q f = A[r * n + c] / A[c * n + c];
      if (f == 0) continue;
      for (int k = c; k < n; ++k) A[r * n + k] -= f * A[c * n + k];
      for (int k = 0; k < m; ++k) B[r * m + k] -= f * B[c * m + k];
    }
  }
  for (int r = n - 1; r >= 0; --r)
    for (int k = 0; k < m; ++k) {
      Q s = B[r * m + k];
      for (int j = r + 1; j < n; ++j) s -= A[r * n + j] * B[j * m + k];
      B[r * m + k] = s / A[r * n + r];
    }
}

// mojoxm's equispaced node order (part of the state layout): vertices, edges
// (0,1)(1,2)(2,0)(0,3)(1,3)(2,3), face interiors (faces opposite v0..v3,
// remaining vertices ascending, points in descending lexicographic order of
// the first two weights), volume interior.
std::vector<NodeExp> simplex_nodes(int dim, int P) {
  std::vector<NodeExp> out;
  const int nv = dim + 1;
  for (int v = 0; v < nv; ++v) {
    NodeExp n{{0, 0, 0, 0}};
    n.a[v] = P;
    out.push_back(n);
  }
  if (P < 2) return out;
  static const int e3[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
  const int ne = dim == 3 ? 6 : 3;
  for (int e = 0; e < ne; ++e)
    for (int k = 1; k < P; ++k) {
      NodeExp n{{0, 0, 0, 0}};
      n.a[e3[e][0]] = P - k;
      n.a[e3[e][1]] = k;
      out.push_back(n);
    }
  if (P < 3) return out;
  auto tri_interior = [&](const int v[3]) {
    for (int x = P - 2; x > 0; --x)
      for (int y = P - x - 1; y > 0; --y) {
        NodeExp n{{0, 0, 0, 0}};
        n.a[v[0]] = x;
        n.a[v[1]] = y;
        n.a[v[2]] = P - x - y;
        out.push_back(n);
      }
  };
  if (dim == 2) {
    const int v[3] = {0, 1, 2};
    tri_interior(v);
    return out;
  }
  for (int f = 0; f < 4; ++f) {
    int v[3], c = 0;
    for (int k = 0; k < 4; ++k)
      if (k != f) v[c++] = k;
    tri_interior(v);
  }
  if (P < 4) return out;
  for (int x = P - 2; x > 0; --x)
    for (int y = P - x - 1; y > 0; --y)
      for (int z = P - x - y - 1; z > 0; --z) {
        NodeExp n{{x, y, z, P - x - y - z}};
        out.push_back(n);
      }
  return out;
}

struct Mono {
  int e[3];
};
// total-degree <= P monomials in dim variables
std::vector<Mono> monomials(int dim, int P) {
  std::vector<Mono> m;
  for (int t = 0; t <= (dim == 3 ? P : 0); ++t)
    for (int s = 0; s <= (dim >= 2 ? P - t : 0); ++s)
      for (int r = 0; r <= P - t - s; ++r) m.push_back({{r, s, t}});
  return m;
}
// exact integral of x^a y^b z^c over the unit simplex of dimension dim
Q simplex_int(int dim, int a, int b, int c) {
  if (dim == 3) return qfact(a) * qfact(b) * qfact(c) / qfact(a + b + c + 3);
  if (dim == 2) return qfact(a) * qfact(b) / qfact(a + b + 2);
  return Q(1) / Q(a + 1);
}

// Lagrange coefficients C[i][k] (phi_i = sum_k C[i][k] m_k) at points X.
std::vector<Q> lagrange_coefs(int dim, const std::vector<Mono>& mon, const std::vector<Q>& X) {
  const int n = int(mon.size());
  std::vector<Q> V(n * n), I(n * n, Q(0));
  for (int j = 0; j < n; ++j) {
    for (int k = 0; k < n; ++k) {
      Q v = 1;
      for (int d = 0; d < dim; ++d) v *= qpow(X[j * dim + d], mon[k].e[d]);
      V[j * n + k] = v;
    }
    I[j * n + j] = 1;
  }
  lu_solve(V, n, I, n);  // V^-1 = C^T
  std::vector<Q> C(n * n);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) C[i * n + k] = I[k * n + i];
  return C;
}

// C G C^T for a Gram matrix G of the monomials
std::vector<Q> congruence(const std::vector<Q>& C, const std::vector<Q>& G, int n) {
  std::vector<Q> T(n * n, Q(0)), R(n * n, Q(0));
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) {
      const Q c = C[i * n + k];
      if (c == 0) continue;
      for (int l = 0; l < n; ++l) T[i * n + l] += c * G[k * n + l];
    }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      Q s = 0;
      for (int l = 0; l < n; ++l) s += T[i * n + l] * C[j * n + l];
      R[i * n + j] = s;
    }
  return R;
}

RefOps build_uncached(int dim, int P) {
  RefOps r;
  r.dim = dim;
  r.P = P;
  r.nodes = simplex_nodes(dim, P);
  r.NP = int(r.nodes.size());
  r.NF = dim + 1;
  auto mon = monomials(dim, P);
  if (int(mon.size()) != r.NP) throw std::runtime_error("node count mismatch");
  const int NP = r.NP;
  std::vector<Q> X(NP * dim);
  for (int j = 0; j < NP; ++j)
    for (int d = 0; d < dim; ++d) X[j * dim + d] = Q(r.nodes[j].a[d + 1]) / Q(P);
  const auto C = lagrange_coefs(dim, mon, X);
  std::vector<Q> G(NP * NP);
  for (int k = 0; k < NP; ++k)
    for (int l = 0; l < NP; ++l)
      G[k * NP + l] = simplex_int(dim, mon[k].e[0] + mon[l].e[0], mon[k].e[1] + mon[l].e[1], mon[k].e[2] + mon[l].e[2]);
  const auto M = congruence(C, G, NP);
  // weak derivative operators D_d = M^-1 S_d, S_d[i][j] = int (d phi_i/dx_d) phi_j
  r.D.assign(dim * NP * NP, 0.0);
  for (int d = 0; d < dim; ++d) {
    std::vector<Q> Gd(NP * NP, Q(0));
    for (int k = 0; k < NP; ++k) {
      if (mon[k].e[d] == 0) continue;
      int e[3] = {mon[k].e[0], mon[k].e[1], mon[k].e[2]};
      const Q fac = e[d];
      e[d] -= 1;
      for (int l = 0; l < NP; ++l)
        Gd[k * NP + l] = fac * simplex_int(dim, e[0] + mon[l].e[0], e[1] + mon[l].e[1], e[2] + mon[l].e[2]);
    }
    auto S = congruence(C, Gd, NP);
    lu_solve(M, NP, S, NP);
    for (int k = 0; k < NP * NP; ++k) r.D[d * NP * NP + k] = double(S[k]);
  }
  // cell-mean weights w_i = int phi_i / |reference simplex|
  const Q vol = dim == 3 ? Q(1) / Q(6) : Q(1) / Q(2);
  for (int i = 0; i < NP; ++i) {
    Q s = 0;
    for (int k = 0; k < NP; ++k) s += C[i * NP + k] * simplex_int(dim, mon[k].e[0], mon[k].e[1], mon[k].e[2]);
    r.w.push_back(double(s / vol));
  }
  // faces (opposite vertex f: nodes with a_f = 0, ascending element index)
  r.NFP = dim == 3 ? (P + 1) * (P + 2) / 2 : P + 1;
  const int NFP = r.NFP;
  r.face_nodes.assign(r.NF * NFP, -1);
  std::vector<Q> Minv(NP * NP, Q(0));
  for (int i = 0; i < NP; ++i) Minv[i * NP + i] = 1;
  lu_solve(M, NP, Minv, NP);
  r.Lift.assign(r.NF * NP * NFP, 0.0);
  const int fdim = dim - 1;
  const auto fm = monomials(fdim, P);
  for (int f = 0; f < r.NF; ++f) {
    std::vector<int> fn;
    for (int i = 0; i < NP; ++i)
      if (r.nodes[i].a[f] == 0) fn.push_back(i);
    if (int(fn.size()) != NFP || int(fm.size()) != NFP) throw std::runtime_error("face node count mismatch");
    for (int m = 0; m < NFP; ++m) r.face_nodes[f * NFP + m] = fn[m];
    int v[3], c = 0;
    for (int k = 0; k <= dim; ++k)
      if (k != f) v[c++] = k;
    // face coordinates: barycentrics of the 2nd (and 3rd) face vertex,
    // an affine map onto the unit simplex of dimension fdim
    std::vector<Q> FX(NFP * fdim);
    for (int m = 0; m < NFP; ++m)
      for (int d = 0; d < fdim; ++d) FX[m * fdim + d] = Q(r.nodes[fn[m]].a[v[d + 1]]) / Q(P);
    const auto FC = lagrange_coefs(fdim, fm, FX);
    std::vector<Q> FG(NFP * NFP);
    for (int k = 0; k < NFP; ++k)
      for (int l = 0; l < NFP; ++l)
        FG[k * NFP + l] = simplex_int(fdim, fm[k].e[0] + fm[l].e[0], fm[k].e[1] + fm[l].e[1], 0);
    auto Mf = congruence(FC, FG, NFP);
    // 3D: per unit area (reference triangle has area 1/2); 2D: edge [0,1]
    if (dim == 3)
      for (auto& x : Mf) x *= 2;
    for (int i = 0; i < NP; ++i)
      for (int m = 0; m < NFP; ++m) {
        Q s = 0;
        for (int l = 0; l < NFP; ++l) s += Minv[i * NP + fn[l]] * Mf[l * NFP + m];
        r.Lift[(f * NP + i) * NFP + m] = double(s);
      }
  }
  return r;
}

}  // namespace

RefOps build_refops(int dim, int P) {
  if (P < 1 || P > 5 || (dim != 2 && dim != 3)) throw std::runtime_error("unsupported order/dimension");
  static std::mutex mu;
  static std::map<std::pair<int, int>, RefOps> cache;
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_pair(dim, P);
  auto it = cache.find(key);
  if (it == cache.end()) it = cache.emplace(key, build_uncached(dim, P)).first;
  return it->second;
}

}  // namespace mxm
