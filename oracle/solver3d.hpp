// ORACLE — test infrastructure only (see refelem.hpp header).
// CPU restatement of mojoxm's 3D fused RK-stage kernel, Barth-Jespersen /
// Venkatakrishnan cell limiter and SSPRK3 stepping:
//   rk_stage_kernel                    src/solver.mojo:161-337
//   compute_cell_averages_kernel       src/solver.mojo:384-407
//   bj_limiter_compute_theta_kernel    src/solver.mojo:410-500
//   bj_limiter_apply_kernel            src/solver.mojo:503-530
//   Solver.step_ssprk3 / _step_stage   src/solver.mojo:1015-1092
// The element loop is OpenMP-parallel; each element reproduces the kernel's
// phases (physical flux, face numerical/boundary flux, volume + lift sums,
// source, RK combine, limit_state) in the same order.
#pragma once
#include <vector>

#include "physics.hpp"

namespace orc {

struct SolverBase {
  virtual ~SolverBase() {}
  int P, NP, NFP, NC;
  int64_t Ne;
  virtual void set_buf(int which, const double* src) = 0;
  virtual void get_buf(int which, double* dst) const = 0;
  virtual void eval_rhs(const double* q, double* rhs) = 0;
  virtual void stage(int s, double dt) = 0;
  virtual void step(double dt) = 0;
  virtual void enable_limiter(bool on, double eps) = 0;
  virtual void limit(int which) = 0;
  virtual void get_theta(double* out) const = 0;
  virtual double max_face_speed() = 0;
  virtual void node_xyz(double* out) const = 0;
  virtual void mesh_arrays(int32_t* elem_faces, int32_t* elem_face_side, int32_t* face_elem, int32_t* face_bc,
                           double* face_normal, double* face_area) const = 0;
  virtual int64_t num_faces() const = 0;
};

template <typename R, typename Phys>
struct Solver3D : SolverBase {
  static constexpr int NCc = Phys::NC;
  Mesh3D<R> mesh;
  Phys phys;
  std::vector<R> D, Lift, w;
  std::vector<R> q[3];  // d_q, d_q1, d_q2
  std::vector<R> cell_avg, theta;
  bool lim_on = false;
  R lim_eps = R(0.1);

  Solver3D(int P_, int nx, int ny, int nz, double Lx, double Ly, double Lz, const int bcs[6], const Phys& ph)
      : mesh(P_, nx, ny, nz, Lx, Ly, Lz, bcs), phys(ph) {
    P = P_;
    NP = mesh.NP;
    NFP = mesh.NFP;
    NC = NCc;
    Ne = mesh.Ne;
    RefElem3D re(P);  // operators FP64 on the host, then cast like to_float32 (reference.mojo:667-671)
    for (double v : re.D) D.push_back(R(v));
    for (double v : re.Lift) Lift.push_back(R(v));
    for (double v : re.w) w.push_back(R(v));
    for (auto& b : q) b.assign(size_t(Ne) * NP * NC, R(0));
    cell_avg.assign(size_t(Ne) * NC, R(0));
    theta.assign(size_t(Ne), R(1));
  }

  void set_buf(int which, const double* src) override {
    for (size_t k = 0; k < q[which].size(); ++k) q[which][k] = R(src[k]);
  }
  void get_buf(int which, double* dst) const override {
    for (size_t k = 0; k < q[which].size(); ++k) dst[k] = double(q[which][k]);
  }
  void node_xyz(double* out) const override {
    for (size_t k = 0; k < mesh.elem_node_xyz.size(); ++k) out[k] = double(mesh.elem_node_xyz[k]);
  }
  int64_t num_faces() const override { return mesh.Nf; }
  void mesh_arrays(int32_t* ef, int32_t* efs, int32_t* fe, int32_t* fbc, double* fn, double* fa) const override {
    for (size_t k = 0; k < mesh.elem_faces.size(); ++k) ef[k] = mesh.elem_faces[k];
    for (size_t k = 0; k < mesh.elem_face_side.size(); ++k) efs[k] = mesh.elem_face_side[k];
    for (size_t k = 0; k < mesh.face_elem.size(); ++k) fe[k] = mesh.face_elem[k];
    for (size_t k = 0; k < mesh.face_bc_type.size(); ++k) fbc[k] = mesh.face_bc_type[k];
    for (size_t k = 0; k < mesh.face_normal.size(); ++k) fn[k] = double(mesh.face_normal[k]);
    for (size_t k = 0; k < mesh.face_area.size(); ++k) fa[k] = double(mesh.face_area[k]);
  }

  // One element of rk_stage_kernel.  With rhs_only the RK combine and
  // limit_state are skipped and the raw semi-discrete RHS is stored.
  void stage_elem(int64_t e, const R* q_in, const R* q_a, const R* q_b, R* q_out, R a, R b, R cc, R dt, bool rhs_only,
                  std::vector<R>& vol, std::vector<R>& fac) const {
    const int NF = 4;
    // Phase 1  solver.mojo:224-232
    for (int i = 0; i < NP; ++i) phys.internal_flux(q_in + (e * NP + i) * NC, &vol[size_t(i) * 3 * NC]);
    // Phase 2  solver.mojo:234-271
    for (int lf = 0; lf < NF; ++lf)
      for (int m = 0; m < NFP; ++m) {
        int64_t fid = mesh.elem_faces[e * NF + lf];
        R nx = mesh.face_normal[fid * 3 + 0], ny = mesh.face_normal[fid * 3 + 1], nz = mesh.face_normal[fid * 3 + 2];
        int64_t el = mesh.face_elem[fid * 2 + 0], er = mesh.face_elem[fid * 2 + 1];
        int nl = mesh.face_elem_node[fid * 2 * NFP + m], nr = mesh.face_elem_node[fid * 2 * NFP + NFP + m];
        const R* ql = q_in + (el * NP + nl) * NC;
        const R* qr = q_in + (er * NP + nr) * NC;
        R* fs = &fac[(size_t(lf) * NFP + m) * NC];
        int bct = mesh.face_bc_type[fid];
        if (bct != 0) phys.boundary_flux(ql, bct, nx, ny, nz, fs);
        else phys.numerical_flux(ql, qr, nx, ny, nz, fs);
      }
    // Phase 3 + 4  solver.mojo:277-337
    const R* iJ = &mesh.elem_invJ[e * 9];
    const R inv6V = mesh.elem_inv_6V[e];
    for (int i = 0; i < NP; ++i) {
      const int64_t ob = (e * NP + i) * NC;
      R src[NCc];
      phys.source_term(q_in + ob, src);
      for (int c = 0; c < NC; ++c) {
        R vc = R(0);
        for (int j = 0; j < NP; ++j) {
          const R* F = &vol[size_t(j) * 3 * NC];
          R fx = F[0 * NC + c], fy = F[1 * NC + c], fz = F[2 * NC + c];
          R fr0 = iJ[0] * fx + iJ[1] * fy + iJ[2] * fz;
          R fr1 = iJ[3] * fx + iJ[4] * fy + iJ[5] * fz;
          R fr2 = iJ[6] * fx + iJ[7] * fy + iJ[8] * fz;
          vc += fr0 * D[0 * NP * NP + i * NP + j] + fr1 * D[1 * NP * NP + i * NP + j] + fr2 * D[2 * NP * NP + i * NP + j];
        }
        R fc = R(0);
        for (int lf = 0; lf < NF; ++lf) {
          R sign = mesh.elem_face_side[e * NF + lf] == 0 ? R(1) : R(-1);
          int64_t fid = mesh.elem_faces[e * NF + lf];
          R area = mesh.face_area[fid];
          for (int m = 0; m < NFP; ++m) {
            int r = mesh.elem_canon_to_ref[(e * NF + lf) * NFP + m];
            R Lim = Lift[lf * NP * NFP + i * NFP + r];
            fc += sign * area * Lim * fac[(size_t(lf) * NFP + m) * NC + c];
          }
        }
        R rhs = vc - inv6V * fc + src[c];
        if (rhs_only) q_out[ob + c] = rhs;
        else q_out[ob + c] = a * q_a[ob + c] + b * q_b[ob + c] + cc * dt * rhs;
      }
      if (!rhs_only) phys.limit_state(q_out + ob);
    }
  }

  void rk_stage(const R* q_in, const R* q_a, const R* q_b, R* q_out, R a, R b, R cc, R dt, bool rhs_only) {
#pragma omp parallel
    {
      std::vector<R> vol(size_t(NP) * 3 * NC), fac(size_t(4) * NFP * NC);
#pragma omp for schedule(static)
      for (int64_t e = 0; e < Ne; ++e) stage_elem(e, q_in, q_a, q_b, q_out, a, b, cc, dt, rhs_only, vol, fac);
    }
  }

  // Max over all face nodes of the speed numerical_flux / boundary_flux
  // return (the value solver.mojo:266-268 discards), evaluated on d_q.
  double max_face_speed() override {
    double best = 0.0;
    const R* qi = q[0].data();
    R fs[NCc];
    for (int64_t e = 0; e < Ne; ++e)
      for (int lf = 0; lf < 4; ++lf)
        for (int m = 0; m < NFP; ++m) {
          int64_t fid = mesh.elem_faces[e * 4 + lf];
          R nx = mesh.face_normal[fid * 3 + 0], ny = mesh.face_normal[fid * 3 + 1], nz = mesh.face_normal[fid * 3 + 2];
          int64_t el = mesh.face_elem[fid * 2 + 0], er = mesh.face_elem[fid * 2 + 1];
          int nl = mesh.face_elem_node[fid * 2 * NFP + m], nr = mesh.face_elem_node[fid * 2 * NFP + NFP + m];
          const R* ql = qi + (el * NP + nl) * NC;
          const R* qr = qi + (er * NP + nr) * NC;
          int bct = mesh.face_bc_type[fid];
          R s = (bct != 0) ? phys.boundary_flux(ql, bct, nx, ny, nz, fs) : phys.numerical_flux(ql, qr, nx, ny, nz, fs);
          if (double(s) > best) best = double(s);
        }
    return best;
  }

  void eval_rhs(const double* qd, double* rhs) override {
    std::vector<R> qi(size_t(Ne) * NP * NC), ro(size_t(Ne) * NP * NC);
    for (size_t k = 0; k < qi.size(); ++k) qi[k] = R(qd[k]);
    rk_stage(qi.data(), nullptr, nullptr, ro.data(), R(0), R(0), R(0), R(0), true);
    for (size_t k = 0; k < ro.size(); ++k) rhs[k] = double(ro[k]);
  }

  // Limiter  solver.mojo:384-530 (np=1: owned_elem_ids is the identity)
  void limit_buf(R* qq) {
    const int64_t n = Ne;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e)
      for (int c = 0; c < NC; ++c) {
        R s = R(0);
        for (int nn = 0; nn < NP; ++nn) s += w[nn] * qq[(e * NP + nn) * NC + c];
        cell_avg[e * NC + c] = s;
      }
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
      R own[NCc], mn[NCc], mx[NCc], pD[NCc], nD[NCc];
      for (int c = 0; c < NC; ++c) own[c] = mn[c] = mx[c] = cell_avg[e * NC + c];
      for (int lf = 0; lf < 4; ++lf) {
        int64_t fid = mesh.elem_faces[e * 4 + lf];
        int64_t el = mesh.face_elem[fid * 2], er = mesh.face_elem[fid * 2 + 1];
        int64_t nb = (el == e) ? er : el;
        for (int c = 0; c < NC; ++c) {
          R av = cell_avg[nb * NC + c];
          if (av < mn[c]) mn[c] = av;
          if (av > mx[c]) mx[c] = av;
        }
      }
      R eps2 = lim_eps * lim_eps;
      for (int c = 0; c < NC; ++c) {
        R p = mx[c] - own[c];
        pD[c] = p < R(0) ? R(0) : p;
        R m = own[c] - mn[c];
        nD[c] = m < R(0) ? R(0) : m;
      }
      R th = R(1);
      const R tiny = R(1.0e-30);
      for (int nn = 0; nn < NP; ++nn)
        for (int c = 0; c < NC; ++c) {
          R dl = qq[(e * NP + nn) * NC + c] - own[c];
          R da = dl >= R(0) ? dl : -dl;
          if (da <= tiny) continue;
          R Dd = dl > R(0) ? pD[c] : nD[c];
          R D2 = Dd * Dd, d2 = da * da, Dda = Dd * da;
          R num = D2 + R(2) * Dda + eps2;
          R den = D2 + R(2) * d2 + Dda + eps2;
          R al = num / den;
          if (al < th) th = al;
        }
      theta[e] = th;
    }
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
      R th = theta[e];
      if (!(th < R(1))) continue;
      for (int nn = 0; nn < NP; ++nn)
        for (int c = 0; c < NC; ++c) {
          R bm = cell_avg[e * NC + c];
          R v = qq[(e * NP + nn) * NC + c];
          qq[(e * NP + nn) * NC + c] = bm + th * (v - bm);
        }
    }
  }
  void limit(int which) override { limit_buf(q[which].data()); }
  void get_theta(double* out) const override {
    for (int64_t e = 0; e < Ne; ++e) out[e] = double(theta[e]);
  }
  void enable_limiter(bool on, double eps) override {
    lim_on = on;
    lim_eps = R(eps);
  }

  // solver.mojo:1071-1092 (Float32 coefficients as literal in the reference)
  void stage(int s, double dtd) override {
    R dt = R(dtd);
    R* p0 = q[0].data();
    R* p1 = q[1].data();
    R* p2 = q[2].data();
    if (s == 0) rk_stage(p0, p0, p0, p1, R(1), R(0), R(1), dt, false);
    else if (s == 1) rk_stage(p1, p0, p1, p2, R(0.75), R(0.25), R(0.25), dt, false);
    else rk_stage(p2, p0, p2, p0, R(1.0 / 3.0), R(2.0 / 3.0), R(2.0 / 3.0), dt, false);
    if (lim_on) limit_buf(s == 0 ? p1 : (s == 1 ? p2 : p0));
  }
  void step(double dt) override {
    for (int s = 0; s < 3; ++s) stage(s, dt);
  }
};

}  // namespace orc
