// Host FP64 construction of the nodal DG reference operators and the Kuhn
// mesh topology tables the device kernels consume.
//
// Reference elements: equispaced Lagrange nodes on the unit tetrahedron /
// triangle in mojoxm's node order (src/reference.mojo:136-237 -- the state
// layout is shared with the Mojo driver, so the order is part of the ABI).
// Operators are built from the monomial basis r^a s^b t^c with exact simplex
// integrals and LU solves; they equal the reference's
// D_ref = M^-1 S, Lift_ref = M^-1 (2 M_tri) (src/reference.mojo:580-650) and
// the 2D edge lift (src/reference_2d.mojo:196-255) to FP64 round-off.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace mxm {

struct NodeExp {
  int a[4];  // barycentric exponents, sum = P (a[3] = 0 on triangles)
};

// Tetrahedron (dim 3) or triangle (dim 2) reference element of order P.
struct RefOps {
  int dim = 3, P = 1, NP = 0, NF = 0, NFP = 0;
  std::vector<NodeExp> nodes;
  std::vector<double> D;       // [dim][NP][NP]   weak-form derivative operators M^-1 S_k
  std::vector<double> Lift;    // [NF][NP][NFP]   face lift, columns in face_nodes order
  std::vector<double> w;       // [NP]            cell-mean weights, sum 1
  std::vector<int> face_nodes; // [NF][NFP]       element node of each face-local index
  // Face-local order: ascending element-node index (not the reference's
  // canonical order; the product keeps one consistent order end to end).
};

RefOps build_refops(int dim, int P);

// Reference's canonical face-local order (src/reference.mojo:453-511 and
// reference_2d.mojo:87-127), used only to export operators for comparison.
std::vector<int> reference_face_order(int dim, int P, const RefOps& r);

// ---------------------------------------------------------------- Kuhn 3D
// Per (tet type t, local face lf): neighbour type/face/cell offset, the
// side convention of mojoxm's face numbering (lower tet index owns internal
// faces, the lower cell owns cube faces), and node pairing.
struct Kuhn3D {
  int vert[6][4][3];      // cube-corner coords of tet-local vertices (local_mesh.mojo:64-114)
  int nb_t[6][4], nb_lf[6][4], off[6][4][3], side[6][4];
  int axis[6][4], dir[6][4];      // cube-face axis (0/1/2) and direction (+1/-1), axis -1 if internal
  std::vector<int> nb_node;       // [6][4][NFP] neighbour element node paired with face node m
  double normal[6][4][3];         // unit normal, side 0 -> side 1
  double area[6][4];
  double invJ[6][9];              // d(r,s,t)/d(x,y,z), row-major [k][d]
  double inv6V[6];
  std::vector<double> rel_xyz;    // [6][NP][3] node position in cell-unit coordinates
};
Kuhn3D build_kuhn3d(const RefOps& r, double dx, double dy, double dz);

// ---------------------------------------------------------------- Kuhn 2D
struct Kuhn2D {
  int vert[2][3][2];
  int nb_t[2][3], nb_lf[2][3], off[2][3][2], side[2][3];
  int axis[2][3], dir[2][3];
  std::vector<int> nb_node;  // [2][3][NFP]
  double normal[2][3][2];
  double length[2][3];
  double invJ[2][4];
  double inv2A[2];
  std::vector<double> rel_xy;  // [2][NP][2]
};
Kuhn2D build_kuhn2d(const RefOps& r, double dx, double dy);

// Operator shared by every element type, row-major NP x K:
// A = [D_r | D_s (| D_t) | -Lift_0 | ... ] with lift columns in face_nodes
// order (2D: local edge lf = RefOps face (lf+2)%3).  The kernels apply the
// per-type invJ to nodal fluxes and side*area/(6V) (3D) or
// side*length/(2A) (2D) to f*.
std::vector<double> shared_operator(const RefOps& r);

}  // namespace mxm
