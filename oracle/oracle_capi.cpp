// ORACLE — test infrastructure only (see refelem.hpp header).
// Plain C entry points so Python tests (ctypes) and bench.py's CPU-baseline
// leg can drive the CPU restatement.  Physics parameters use the same flat
// layout as the product's `mxm_dg_physics_desc.p[]` (field order of the Mojo
// structs: src/euler.mojo:534-554, src/maxwell.mojo:55-74,
// src/shallow_water.mojo:34-40, src/advection.mojo:192-199).
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>

#include "solver2d.hpp"
#include "solver3d.hpp"
#include "sod_exact.hpp"

using namespace orc;

static thread_local std::string g_err;

template <typename R>
static SolverBase* make3(int P, int nx, int ny, int nz, double Lx, double Ly, double Lz, const int* bcs, int kind, int flux,
                         int efix, const double* p) {
  if (kind == PHYS_ADVECTION) {
    Advection<R> ph{R(p[0]), R(p[1]), R(p[2]), R(p[3])};
    return new Solver3D<R, Advection<R>>(P, nx, ny, nz, Lx, Ly, Lz, bcs, ph);
  }
  if (kind == PHYS_EULER) {
    Euler<R> ph;
    ph.gamma = R(p[0]); ph.min_density = R(p[1]); ph.min_pressure = R(p[2]);
    ph.flux_type = flux; ph.entropy_fix = efix != 0;
    ph.gx = R(p[3]); ph.gy = R(p[4]); ph.gz = R(p[5]);
    for (int c = 0; c < 5; ++c) ph.inflow[c] = R(p[6 + c]);
    return new Solver3D<R, Euler<R>>(P, nx, ny, nz, Lx, Ly, Lz, bcs, ph);
  }
  if (kind == PHYS_MAXWELL) {
    Maxwell<R> ph;
    ph.c = R(p[0]);
    for (int k = 0; k < 3; ++k) { ph.J[k] = R(p[1 + k]); ph.M[k] = R(p[4 + k]); }
    for (int k = 0; k < 6; ++k) ph.inflow[k] = R(p[7 + k]);
    return new Solver3D<R, Maxwell<R>>(P, nx, ny, nz, Lx, Ly, Lz, bcs, ph);
  }
  if (kind == PHYS_SW) {
    ShallowWater<R> ph;
    ph.g = R(p[0]); ph.h_min = R(p[1]);
    for (int k = 0; k < 3; ++k) ph.inflow[k] = R(p[2 + k]);
    return new Solver3D<R, ShallowWater<R>>(P, nx, ny, nz, Lx, Ly, Lz, bcs, ph);
  }
  if (kind == PHYS_MHD) {
    IdealMHD<R> ph;
    ph.gamma = R(p[0]); ph.min_density = R(p[1]); ph.min_pressure = R(p[2]); ph.c_h = R(p[3]); ph.alpha_d = R(p[4]);
    for (int k = 0; k < 9; ++k) ph.inflow[k] = R(p[5 + k]);
    return new Solver3D<R, IdealMHD<R>>(P, nx, ny, nz, Lx, Ly, Lz, bcs, ph);
  }
  if (kind == PHYS_TWO_FLUID) {
    TwoFluid<R> ph;
    ph.gamma_e = R(p[0]); ph.gamma_i = R(p[1]); ph.q_e = R(p[2]); ph.m_e = R(p[3]); ph.q_i = R(p[4]);
    ph.m_i = R(p[5]); ph.eps0 = R(p[6]); ph.c_light = R(p[7]); ph.c_h = R(p[8]); ph.alpha_d = R(p[9]);
    ph.min_density = R(p[10]); ph.min_pressure = R(p[11]);
    for (int k = 0; k < 17; ++k) ph.inflow[k] = R(p[12 + k]);
    return new Solver3D<R, TwoFluid<R>>(P, nx, ny, nz, Lx, Ly, Lz, bcs, ph);
  }
  throw std::runtime_error("unknown physics kind");
}

#define GUARD(expr)                 \
  try {                             \
    expr;                           \
    return 0;                       \
  } catch (std::exception & ex) {   \
    g_err = ex.what();              \
    return -1;                      \
  }

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

// ---- reference elements (golden-vector checks) ----
int orc_refelem3d(int P, double* D, double* Lift, double* w, int32_t* face_to_elem, double* Minv, double* node_pos) {
  GUARD({
    RefElem3D re(P);
    std::memcpy(D, re.D.data(), re.D.size() * 8);
    std::memcpy(Lift, re.Lift.data(), re.Lift.size() * 8);
    std::memcpy(w, re.w.data(), re.w.size() * 8);
    std::memcpy(face_to_elem, re.face_to_elem.data(), re.face_to_elem.size() * 4);
    std::memcpy(Minv, re.Minv.data(), re.Minv.size() * 8);
    std::memcpy(node_pos, re.node_pos.data(), re.node_pos.size() * 8);
  })
}
int orc_mat_inv(const double* m, int n, double* out) {
  GUARD({
    std::vector<double> a(m, m + n * n);
    auto r = mat_inv(a, n);
    std::memcpy(out, r.data(), r.size() * 8);
  })
}
int orc_refelem2d(int P, double* Dr, double* Ds, double* Lift, double* w, int32_t* edge_to_elem, double* Minv,
                  double* node_pos) {
  GUARD({
    RefElem2D re(P);
    std::memcpy(Dr, re.Dr.data(), re.Dr.size() * 8);
    std::memcpy(Ds, re.Ds.data(), re.Ds.size() * 8);
    std::memcpy(Lift, re.Lift.data(), re.Lift.size() * 8);
    std::memcpy(w, re.w.data(), re.w.size() * 8);
    std::memcpy(edge_to_elem, re.edge_to_elem.data(), re.edge_to_elem.size() * 4);
    std::memcpy(Minv, re.Minv.data(), re.Minv.size() * 8);
    std::memcpy(node_pos, re.node_pos.data(), re.node_pos.size() * 8);
  })
}

// ---- 3D solver ----
int orc3_create(int real_kind, int P, int nx, int ny, int nz, double Lx, double Ly, double Lz, const int* bcs, int kind,
                int flux, int efix, const double* p, void** out) {
  GUARD({
    *out = real_kind == 0 ? (void*)make3<double>(P, nx, ny, nz, Lx, Ly, Lz, bcs, kind, flux, efix, p)
                          : (void*)make3<float>(P, nx, ny, nz, Lx, Ly, Lz, bcs, kind, flux, efix, p);
  })
}
void orc3_destroy(void* h) { delete (SolverBase*)h; }
int64_t orc3_num_elements(void* h) { return ((SolverBase*)h)->Ne; }
int64_t orc3_num_faces(void* h) { return ((SolverBase*)h)->num_faces(); }
int orc3_np(void* h) { return ((SolverBase*)h)->NP; }
int orc3_nfp(void* h) { return ((SolverBase*)h)->NFP; }
int orc3_nc(void* h) { return ((SolverBase*)h)->NC; }
int orc3_set_buf(void* h, int which, const double* src) { GUARD(((SolverBase*)h)->set_buf(which, src)) }
int orc3_get_buf(void* h, int which, double* dst) { GUARD(((SolverBase*)h)->get_buf(which, dst)) }
int orc3_eval_rhs(void* h, const double* q, double* rhs) { GUARD(((SolverBase*)h)->eval_rhs(q, rhs)) }
int orc3_stage(void* h, int s, double dt) { GUARD(((SolverBase*)h)->stage(s, dt)) }
int orc3_step(void* h, double dt, int nsteps) {
  GUARD(for (int k = 0; k < nsteps; ++k)((SolverBase*)h)->step(dt))
}
int orc3_enable_limiter(void* h, int on, double eps) { GUARD(((SolverBase*)h)->enable_limiter(on != 0, eps)) }
int orc3_limit(void* h, int which) { GUARD(((SolverBase*)h)->limit(which)) }
int orc3_theta(void* h, double* out) { GUARD(((SolverBase*)h)->get_theta(out)) }
int orc3_node_xyz(void* h, double* out) { GUARD(((SolverBase*)h)->node_xyz(out)) }
double orc3_max_face_speed(void* h) { return ((SolverBase*)h)->max_face_speed(); }
int orc3_mesh_arrays(void* h, int32_t* ef, int32_t* efs, int32_t* fe, int32_t* fbc, double* fn, double* fa) {
  GUARD(((SolverBase*)h)->mesh_arrays(ef, efs, fe, fbc, fn, fa))
}

// ---- 2D solver ----
int orc2_create(int real_kind, int P, int nx, int ny, double Lx, double Ly, const int* bcs, int kind, int flux,
                int efix, const double* p, void** out) {
  GUARD({
    *out = real_kind == 0 ? (void*)make2<double>(P, nx, ny, Lx, Ly, bcs, kind, flux, efix, p)
                          : (void*)make2<float>(P, nx, ny, Lx, Ly, bcs, kind, flux, efix, p);
  })
}
void orc2_destroy(void* h) { delete (Solver2DBase*)h; }
int64_t orc2_num_elements(void* h) { return ((Solver2DBase*)h)->Ne; }
int orc2_np(void* h) { return ((Solver2DBase*)h)->NP; }
int orc2_nc(void* h) { return ((Solver2DBase*)h)->NC; }
int orc2_set_buf(void* h, int which, const double* src) { GUARD(((Solver2DBase*)h)->set_buf(which, src)) }
int orc2_get_buf(void* h, int which, double* dst) { GUARD(((Solver2DBase*)h)->get_buf(which, dst)) }
int orc2_eval_rhs(void* h, const double* q, double* rhs) { GUARD(((Solver2DBase*)h)->eval_rhs(q, rhs)) }
int orc2_stage(void* h, int s, double dt) { GUARD(((Solver2DBase*)h)->stage(s, dt)) }
int orc2_step(void* h, double dt, int nsteps) {
  GUARD(for (int k = 0; k < nsteps; ++k)((Solver2DBase*)h)->step(dt))
}
int orc2_enable_limiter(void* h, int on, double eps) { GUARD(((Solver2DBase*)h)->enable_limiter(on != 0, eps)) }
int orc2_limit(void* h, int which) { GUARD(((Solver2DBase*)h)->limit(which)) }
int orc2_node_xy(void* h, double* out) { GUARD(((Solver2DBase*)h)->node_xy(out)) }

// ---- Sod exact Riemann solution ----
int orc_sod_exact(double rhoL, double uL, double pL, double rhoR, double uR, double pR, double gamma, double x0, double t,
                  const double* x, int n, double* rho, double* u, double* p) {
  GUARD(sod_sample(rhoL, uL, pL, rhoR, uR, pR, gamma, x0, t, x, n, rho, u, p))
}
int orc_sod_star(double rhoL, double uL, double pL, double rhoR, double uR, double pR, double gamma, double* out4) {
  GUARD(sod_star(rhoL, uL, pL, rhoR, uR, pR, gamma, out4))
}
}
