"""ORACLE — test infrastructure only.

ctypes front end for the CPU restatement of mojoxm's DG path (liboracle.so,
built from the headers in this directory by its Makefile).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module;
the product package never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

PHYS_ADVECTION, PHYS_EULER, PHYS_MAXWELL, PHYS_SW = 0, 1, 2, 3
FLUX_RUSANOV, FLUX_ROE, FLUX_HLLE, FLUX_HLLEC, FLUX_HLLC, FLUX_HLL = 0, 1, 2, 3, 4, 5
BC_INTERIOR, BC_WALL, BC_OUTFLOW, BC_INFLOW = 0, 1, 2, 3

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


def build() -> str:
    """Compile liboracle.so in place (make) and return its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_last_error.restype = ctypes.c_char_p
        for n in ("orc3_num_elements", "orc3_num_faces", "orc2_num_elements"):
            getattr(L, n).restype = ctypes.c_int64
        L.orc3_max_face_speed.restype = ctypes.c_double
        _LIB = L
    return _LIB


def _chk(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def ntet(P):
    return (P + 1) * (P + 2) * (P + 3) // 6


def ntri(P):
    return (P + 1) * (P + 2) // 2


def refelem3d(P):
    NP, NFP = ntet(P), ntri(P)
    D = np.zeros(3 * NP * NP)
    Lift = np.zeros(4 * NP * NFP)
    w = np.zeros(NP)
    f2e = np.zeros(4 * NFP, np.int32)
    Minv = np.zeros(NP * NP)
    pos = np.zeros(NP * 3)
    _chk(lib().orc_refelem3d(P, _d(D), _d(Lift), _d(w), _i(f2e), _d(Minv), _d(pos)))
    return dict(D=D.reshape(3, NP, NP), Lift=Lift.reshape(4, NP, NFP), w=w, face_to_elem=f2e.reshape(4, NFP),
                Minv=Minv.reshape(NP, NP), node_pos=pos.reshape(NP, 3))


def refelem2d(P):
    NP, NE = ntri(P), P + 1
    Dr = np.zeros(NP * NP)
    Ds = np.zeros(NP * NP)
    Lift = np.zeros(3 * NP * NE)
    w = np.zeros(NP)
    e2e = np.zeros(3 * NE, np.int32)
    Minv = np.zeros(NP * NP)
    pos = np.zeros(NP * 2)
    _chk(lib().orc_refelem2d(P, _d(Dr), _d(Ds), _d(Lift), _d(w), _i(e2e), _d(Minv), _d(pos)))
    return dict(Dr=Dr.reshape(NP, NP), Ds=Ds.reshape(NP, NP), Lift=Lift.reshape(3, NP, NE), w=w,
                edge_to_elem=e2e.reshape(3, NE), Minv=Minv.reshape(NP, NP), node_pos=pos.reshape(NP, 2))


def mat_inv(m):
    m = np.ascontiguousarray(m, dtype=np.float64)
    n = m.shape[0]
    out = np.zeros_like(m)
    _chk(lib().orc_mat_inv(_d(m), n, _d(out)))
    return out


def sod_star(rhoL, uL, pL, rhoR, uR, pR, gamma=1.4):
    out = np.zeros(4)
    _chk(lib().orc_sod_star(*(ctypes.c_double(v) for v in (rhoL, uL, pL, rhoR, uR, pR, gamma)), _d(out)))
    return out


def sod_exact(x, t, rhoL, uL, pL, rhoR, uR, pR, gamma=1.4, x0=0.5):
    x = np.ascontiguousarray(x, dtype=np.float64)
    r, u, p = np.zeros_like(x), np.zeros_like(x), np.zeros_like(x)
    _chk(lib().orc_sod_exact(*(ctypes.c_double(v) for v in (rhoL, uL, pL, rhoR, uR, pR, gamma, x0, t)), _d(x),
                             ctypes.c_int(len(x)), _d(r), _d(u), _d(p)))
    return r, u, p


class Oracle3D:
    """CPU restatement of Solver[PhysT, P] (3D Kuhn tets).  real='f64'|'f32'."""

    def __init__(self, P, n, L, physics, bcs=(0,) * 6, real="f64"):
        nx, ny, nz = (n, n, n) if np.isscalar(n) else n
        Lx, Ly, Lz = (L, L, L) if np.isscalar(L) else L
        p = np.zeros(32)
        p[: len(physics["p"])] = physics["p"]
        b = np.array(bcs, np.int32)
        h = ctypes.c_void_p()
        _chk(lib().orc3_create(0 if real == "f64" else 1, P, nx, ny, nz, ctypes.c_double(Lx), ctypes.c_double(Ly),
                               ctypes.c_double(Lz), _i(b), physics["kind"], physics.get("flux", 0),
                               int(physics.get("entropy_fix", 0)), _d(p), ctypes.byref(h)))
        self.h = h
        L_ = lib()
        self.P, self.Ne, self.NP, self.NFP, self.NC = P, L_.orc3_num_elements(h), L_.orc3_np(h), L_.orc3_nfp(h), L_.orc3_nc(h)
        self.shape = (self.Ne, self.NP, self.NC)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc3_destroy(self.h)
            self.h = None

    def set(self, q, which=0):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
        assert q.size == self.Ne * self.NP * self.NC
        _chk(lib().orc3_set_buf(self.h, which, _d(q)))

    def get(self, which=0):
        out = np.zeros(self.shape)
        _chk(lib().orc3_get_buf(self.h, which, _d(out)))
        return out

    def rhs(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.shape)
        out = np.zeros(self.shape)
        _chk(lib().orc3_eval_rhs(self.h, _d(q), _d(out)))
        return out

    def stage(self, s, dt):
        _chk(lib().orc3_stage(self.h, s, ctypes.c_double(dt)))

    def step(self, dt, nsteps=1):
        _chk(lib().orc3_step(self.h, ctypes.c_double(dt), nsteps))

    def enable_limiter(self, on=True, eps=0.1):
        _chk(lib().orc3_enable_limiter(self.h, int(on), ctypes.c_double(eps)))

    def limit(self, which=0):
        _chk(lib().orc3_limit(self.h, which))

    def theta(self):
        out = np.zeros(self.Ne)
        _chk(lib().orc3_theta(self.h, _d(out)))
        return out

    def node_xyz(self):
        out = np.zeros((self.Ne, self.NP, 3))
        _chk(lib().orc3_node_xyz(self.h, _d(out)))
        return out

    def max_face_speed(self):
        return lib().orc3_max_face_speed(self.h)

    def mesh_arrays(self):
        Nf = lib().orc3_num_faces(self.h)
        ef = np.zeros(self.Ne * 4, np.int32)
        efs = np.zeros(self.Ne * 4, np.int32)
        fe = np.zeros(Nf * 2, np.int32)
        fbc = np.zeros(Nf, np.int32)
        fn = np.zeros(Nf * 3)
        fa = np.zeros(Nf)
        _chk(lib().orc3_mesh_arrays(self.h, _i(ef), _i(efs), _i(fe), _i(fbc), _d(fn), _d(fa)))
        return dict(elem_faces=ef.reshape(-1, 4), elem_face_side=efs.reshape(-1, 4), face_elem=fe.reshape(-1, 2),
                    face_bc_type=fbc, face_normal=fn.reshape(-1, 3), face_area=fa)


class Oracle2D:
    """CPU restatement of the 2D per-physics stage kernels + 2D limiter."""

    def __init__(self, P, n, L, physics, bcs=(0,) * 4, real="f64"):
        nx, ny = (n, n) if np.isscalar(n) else n
        Lx, Ly = (L, L) if np.isscalar(L) else L
        p = np.zeros(32)
        p[: len(physics["p"])] = physics["p"]
        b = np.array(bcs, np.int32)
        h = ctypes.c_void_p()
        _chk(lib().orc2_create(0 if real == "f64" else 1, P, nx, ny, ctypes.c_double(Lx), ctypes.c_double(Ly), _i(b),
                               physics["kind"], physics.get("flux", 0), int(physics.get("entropy_fix", 0)), _d(p),
                               ctypes.byref(h)))
        self.h = h
        L_ = lib()
        self.P, self.Ne, self.NP, self.NC = P, L_.orc2_num_elements(h), L_.orc2_np(h), L_.orc2_nc(h)
        self.shape = (self.Ne, self.NP, self.NC)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc2_destroy(self.h)
            self.h = None

    def set(self, q, which=0):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
        _chk(lib().orc2_set_buf(self.h, which, _d(q)))

    def get(self, which=0):
        out = np.zeros(self.shape)
        _chk(lib().orc2_get_buf(self.h, which, _d(out)))
        return out

    def rhs(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.shape)
        out = np.zeros(self.shape)
        _chk(lib().orc2_eval_rhs(self.h, _d(q), _d(out)))
        return out

    def stage(self, s, dt):
        _chk(lib().orc2_stage(self.h, s, ctypes.c_double(dt)))

    def step(self, dt, nsteps=1):
        _chk(lib().orc2_step(self.h, ctypes.c_double(dt), nsteps))

    def enable_limiter(self, on=True, eps=0.1):
        _chk(lib().orc2_enable_limiter(self.h, int(on), ctypes.c_double(eps)))

    def limit(self, which=0):
        _chk(lib().orc2_limit(self.h, which))

    def node_xy(self):
        out = np.zeros((self.Ne, self.NP, 2))
        _chk(lib().orc2_node_xy(self.h, _d(out)))
        return out
