"""mojoxm_b200 -- B200 (sm_100a) nodal DG right-hand side, SSPRK3 stage and
slope limiter for Kuhn tetrahedral (3D) and triangular (2D) meshes.

Python front end over the C ABI in include/mxm_dg.h (libmxm_dg.so, built in
this directory by build.py).  The names mirror mojoxm's host API:

    physics = Euler(gamma=1.4, min_density=1e-6, min_pressure=1e-6,
                    flux_type=FLUX_HLLEC, entropy_fix=True)
    solver = Solver(Mesh(nx, ny, nz, L, BoundaryConditions.periodic()),
                    physics, P=2, precision="f64")
    solver.upload_state(q0)                    # or write solver.d_q on the device
    solver.step_ssprk3(dt)
    rho = solver.download_owned_component(0)

(src/solver.mojo:538-1092, src/euler.mojo:556-584, src/boundary.mojo:326-362).
There is no CPU execution path: constructing a Solver without the CUDA
library or without a GPU raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmxm_dg.so")

# include/mxm_dg.h constants
OK, EINVAL, ENOMEM, ECUDA, ENONFINITE, ETIMEDOUT, ENOTREADY = 0, -1, -2, -3, -4, -5, -6
PHYS_ADVECTION, PHYS_EULER, PHYS_MAXWELL, PHYS_SHALLOW_WATER, PHYS_MHD, PHYS_MHD_PLAIN, PHYS_TWO_FLUID = range(7)
FLUX_RUSANOV, FLUX_ROE, FLUX_HLLE, FLUX_HLLEC, FLUX_HLLC, FLUX_HLL = 0, 1, 2, 3, 4, 5
BC_INTERIOR, BC_WALL, BC_OUTFLOW, BC_INFLOW = 0, 1, 2, 3
PREC = {"f64": 0, "f32": 1, "mixed": 2, "tf32": 3}

EXPORTED = [
    "mxm_dg_slab_plan", "mxm_dg_slab_exchange_ops", "mxm_dg_create_slab", "mxm_dg_slab_info", "mxm_dg_slab_layout", "mxm_dg_slab_stage",
    "mxm_dg_nccl_unique_id", "mxm_dg_slab_connect_nccl", "mxm_dg_group_create", "mxm_dg_group_step_n",
    "mxm_dg_group_synchronize", "mxm_dg_group_last_error", "mxm_dg_group_destroy", "mxm_dg_group_time_steps",
    "mxm_dg_version", "mxm_dg_node_xyz_f32", "mxm_dg_advance_host_async", "mxm_dg_create", "mxm_dg_destroy", "mxm_dg_sizes", "mxm_dg_dof_count",
    "mxm_dg_state_bytes_per_step", "mxm_dg_state_ptr", "mxm_dg_node_xyz_ptr", "mxm_dg_node_xyz",
    "mxm_dg_upload_state", "mxm_dg_download_state", "mxm_dg_download_component", "mxm_dg_download_component_f64",
    "mxm_dg_enable_limiter", "mxm_dg_step_ssprk3", "mxm_dg_step_n", "mxm_dg_rk_stage", "mxm_dg_eval_rhs",
    "mxm_dg_limit", "mxm_dg_advance_host", "mxm_dg_max_wavespeed", "mxm_dg_reduce_conserved",
    "mxm_dg_synchronize", "mxm_dg_time_steps", "mxm_dg_launches_per_step", "mxm_dg_last_error",
    "mxm_dg_operator", "mxm_dg_reference_operators", "mxm_dg_set_device", "mxm_dg_host_alloc", "mxm_dg_host_free",
    "mxm_dg_reduce_conserved_noalloc",
    "mxm_dg_batch_create", "mxm_dg_batch_destroy", "mxm_dg_batch_add", "mxm_dg_batch_autotune",
    "mxm_dg_batch_tile_cells", "mxm_dg_batch_step", "mxm_dg_batch_time_steps", "mxm_dg_batch_synchronize",
    "mxm_dg_batch_dof_count", "mxm_dg_batch_launches_per_step", "mxm_dg_batch_last_error",
    "mxm_dg_fill_ic", "mxm_dg_selftest_wait_timeout",
    "mxm_dg_server_create", "mxm_dg_server_destroy", "mxm_dg_server_submit", "mxm_dg_server_poll",
    "mxm_dg_server_wait", "mxm_dg_server_stats", "mxm_dg_server_last_error",
]

IC_CONSTANT, IC_SINE_WAVE, IC_VORTEX, IC_SOD, IC_DAM_BREAK, IC_CAVITY, IC_PLANE_WAVE, IC_ALFVEN = range(8)


class DGError(RuntimeError):
    def __init__(self, rc, msg):
        super().__init__(f"mxm_dg error {rc}: {msg}")
        self.rc = rc


class _PhysDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("flux_type", ctypes.c_int32), ("entropy_fix", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("p", ctypes.c_double * 32)]


class _MeshDesc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
                ("bc", ctypes.c_int32 * 6)]


_lib = None


def lib():
    """Load libmxm_dg.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python mojoxm_b200/build.py` (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i64p, i32p, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32), \
            ctypes.POINTER(ctypes.c_double)
        L.mxm_dg_create.argtypes = [ctypes.POINTER(_MeshDesc), ctypes.POINTER(_PhysDesc), ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_void_p)]
        L.mxm_dg_destroy.argtypes = [vp]
        L.mxm_dg_sizes.argtypes = [vp, i64p, i32p, i32p, i32p, i32p]
        L.mxm_dg_dof_count.argtypes = [vp, i64p]
        L.mxm_dg_state_bytes_per_step.argtypes = [vp, i64p]
        L.mxm_dg_state_ptr.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.mxm_dg_node_xyz_ptr.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
        L.mxm_dg_node_xyz.argtypes = [vp, dp]
        L.mxm_dg_node_xyz_f32.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
        L.mxm_dg_upload_state.argtypes = [vp, ctypes.c_int, vp, ctypes.c_size_t]
        L.mxm_dg_download_state.argtypes = [vp, ctypes.c_int, vp, ctypes.c_size_t]
        L.mxm_dg_download_component.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
        L.mxm_dg_download_component_f64.argtypes = [vp, ctypes.c_int, dp]
        L.mxm_dg_enable_limiter.argtypes = [vp, ctypes.c_int, ctypes.c_double]
        L.mxm_dg_step_ssprk3.argtypes = [vp, ctypes.c_double]
        L.mxm_dg_step_n.argtypes = [vp, ctypes.c_double, ctypes.c_int]
        L.mxm_dg_rk_stage.argtypes = [vp, ctypes.c_int, ctypes.c_double]
        L.mxm_dg_eval_rhs.argtypes = [vp, vp, vp]
        L.mxm_dg_limit.argtypes = [vp, ctypes.c_int]
        L.mxm_dg_advance_host.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_double]
        L.mxm_dg_advance_host_async.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_double]
        L.mxm_dg_max_wavespeed.argtypes = [vp, dp]
        L.mxm_dg_reduce_conserved.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        L.mxm_dg_reduce_conserved_noalloc.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        L.mxm_dg_synchronize.argtypes = [vp]
        L.mxm_dg_time_steps.argtypes = [vp, ctypes.c_double, ctypes.c_int, dp]
        L.mxm_dg_launches_per_step.argtypes = [vp, i32p]
        L.mxm_dg_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L.mxm_dg_operator.argtypes = [vp, dp, i64p]
        L.mxm_dg_reference_operators.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
        L.mxm_dg_set_device.argtypes = [ctypes.c_int]
        L.mxm_dg_host_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]
        L.mxm_dg_host_free.argtypes = [vp]
        L.mxm_dg_batch_create.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
        L.mxm_dg_batch_destroy.argtypes = [vp]
        L.mxm_dg_batch_add.argtypes = [vp, vp, ctypes.c_double, i32p]
        L.mxm_dg_batch_autotune.argtypes = [vp]
        L.mxm_dg_batch_tile_cells.argtypes = [vp, ctypes.c_int, i32p]
        L.mxm_dg_batch_step.argtypes = [vp, ctypes.c_int]
        L.mxm_dg_batch_time_steps.argtypes = [vp, ctypes.c_int, dp]
        L.mxm_dg_batch_synchronize.argtypes = [vp]
        L.mxm_dg_batch_dof_count.argtypes = [vp, i64p]
        L.mxm_dg_batch_launches_per_step.argtypes = [vp, i32p]
        L.mxm_dg_batch_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L.mxm_dg_fill_ic.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
        L.mxm_dg_selftest_wait_timeout.argtypes = [ctypes.c_double, i32p, dp]
        L.mxm_dg_server_create.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.mxm_dg_server_destroy.argtypes = [vp]
        L.mxm_dg_server_submit.argtypes = [vp, ctypes.POINTER(_MeshDesc), ctypes.POINTER(_PhysDesc), ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_int, vp, i64p]
        L.mxm_dg_server_poll.argtypes = [vp, ctypes.c_int64, dp]
        L.mxm_dg_server_wait.argtypes = [vp, ctypes.c_int64, ctypes.c_double, dp]
        L.mxm_dg_server_stats.argtypes = [vp, dp, ctypes.c_int]
        L.mxm_dg_server_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L.mxm_dg_slab_plan.argtypes = [ctypes.c_int] * 5 + [i32p]
        L.mxm_dg_slab_exchange_ops.argtypes = [ctypes.c_int] * 5 + [i32p, ctypes.POINTER(ctypes.c_int)]
        L.mxm_dg_create_slab.argtypes = [ctypes.POINTER(_MeshDesc), ctypes.POINTER(_PhysDesc), ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.mxm_dg_slab_info.argtypes = [vp, i64p]
        L.mxm_dg_slab_layout.argtypes = [vp, i64p]
        L.mxm_dg_slab_stage.argtypes = [vp, ctypes.c_int, ctypes.c_double]
        L.mxm_dg_nccl_unique_id.argtypes = [ctypes.c_char_p]
        L.mxm_dg_slab_connect_nccl.argtypes = [vp, ctypes.c_char_p]
        L.mxm_dg_group_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.mxm_dg_group_step_n.argtypes = [vp, ctypes.c_double, ctypes.c_int]
        L.mxm_dg_group_synchronize.argtypes = [vp]
        L.mxm_dg_group_time_steps.argtypes = [vp, ctypes.c_double, ctypes.c_int, dp]
        L.mxm_dg_group_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
        L.mxm_dg_group_destroy.argtypes = [vp]
        _lib = L
    return _lib


def set_device(device: int):
    _check(lib().mxm_dg_set_device(device))


class PinnedArray:
    """numpy view over page-locked host memory (mxm_dg_host_alloc)."""

    def __init__(self, shape, dtype):
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        p = ctypes.c_void_p()
        _check(lib().mxm_dg_host_alloc(n, ctypes.byref(p)))
        self.ptr = p
        buf = (ctypes.c_char * n).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self):
        if self.ptr:
            self.array = None
            lib().mxm_dg_host_free(self.ptr)
            self.ptr = None


def _err(h=None):
    buf = ctypes.create_string_buffer(1024)
    lib().mxm_dg_last_error(h, buf, 1024)
    return buf.value.decode(errors="replace")


def _check(rc, h=None):
    if rc != OK:
        raise DGError(rc, _err(h))


# ------------------------------------------------------------------ physics
@dataclass
class Advection:  # src/advection.mojo:187-205
    vx: float
    vy: float
    vz: float = 0.0
    inflow_q: float = 0.0
    kind: int = field(default=PHYS_ADVECTION, init=False)
    flux_type: int = field(default=0, init=False)
    entropy_fix: bool = field(default=False, init=False)

    def params(self):
        return [self.vx, self.vy, self.vz, self.inflow_q]


@dataclass
class Euler:  # src/euler.mojo:531-584
    gamma: float = 1.4
    min_density: float = 1e-6
    min_pressure: float = 1e-6
    flux_type: int = FLUX_HLLEC
    entropy_fix: bool = False
    gx: float = 0.0
    gy: float = 0.0
    gz: float = 0.0
    inflow_rho: float = 0.0
    inflow_rhou: float = 0.0
    inflow_rhov: float = 0.0
    inflow_rhow: float = 0.0
    inflow_E: float = 0.0
    kind: int = field(default=PHYS_EULER, init=False)

    def params(self):
        return [self.gamma, self.min_density, self.min_pressure, self.gx, self.gy, self.gz, self.inflow_rho,
                self.inflow_rhou, self.inflow_rhov, self.inflow_rhow, self.inflow_E]


@dataclass
class Maxwell:  # src/maxwell.mojo:48-104
    c: float = 1.0
    Jx: float = 0.0
    Jy: float = 0.0
    Jz: float = 0.0
    Mx: float = 0.0
    My: float = 0.0
    Mz: float = 0.0
    inflow_Ex: float = 0.0
    inflow_Ey: float = 0.0
    inflow_Ez: float = 0.0
    inflow_Bx: float = 0.0
    inflow_By: float = 0.0
    inflow_Bz: float = 0.0
    kind: int = field(default=PHYS_MAXWELL, init=False)
    flux_type: int = field(default=0, init=False)
    entropy_fix: bool = field(default=False, init=False)

    def params(self):
        return [self.c, self.Jx, self.Jy, self.Jz, self.Mx, self.My, self.Mz, self.inflow_Ex, self.inflow_Ey,
                self.inflow_Ez, self.inflow_Bx, self.inflow_By, self.inflow_Bz]


@dataclass
class ShallowWater:  # src/shallow_water.mojo:31-47
    g: float = 9.81
    h_min: float = 1e-6
    inflow_h: float = 0.0
    inflow_hu: float = 0.0
    inflow_hv: float = 0.0
    flux_type: int = FLUX_RUSANOV
    kind: int = field(default=PHYS_SHALLOW_WATER, init=False)
    entropy_fix: bool = field(default=False, init=False)

    def params(self):
        return [self.g, self.h_min, self.inflow_h, self.inflow_hu, self.inflow_hv]


@dataclass
class IdealMHD:  # src/mhd.mojo:199-254 (3D; q = [rho, rho u, rho v, rho w, E, Bx, By, Bz, psi])
    gamma: float = 5.0 / 3.0
    min_density: float = 1e-6
    min_pressure: float = 1e-6
    c_h: float = 0.0
    alpha_d: float = 0.0
    inflow_rho: float = 0.0
    inflow_rhou: float = 0.0
    inflow_rhov: float = 0.0
    inflow_rhow: float = 0.0
    inflow_E: float = 0.0
    inflow_Bx: float = 0.0
    inflow_By: float = 0.0
    inflow_Bz: float = 0.0
    inflow_psi: float = 0.0
    kind: int = field(default=PHYS_MHD, init=False)
    flux_type: int = field(default=0, init=False)
    entropy_fix: bool = field(default=False, init=False)

    def params(self):
        return [self.gamma, self.min_density, self.min_pressure, self.c_h, self.alpha_d, self.inflow_rho,
                self.inflow_rhou, self.inflow_rhov, self.inflow_rhow, self.inflow_E, self.inflow_Bx, self.inflow_By,
                self.inflow_Bz, self.inflow_psi]


@dataclass
class IdealMHDPlain(IdealMHD):
    """2D ideal MHD without divergence cleaning (src/local_mesh_2d_gpu_mhd.mojo):
    state (rho, mx, my, Bx, By, E); c_h, alpha_d and psi are unused.  An
    IdealMHD on a 2D mesh is the GLM stack (src/local_mesh_2d_gpu_mhd_glm.mojo)
    with state (rho, mx, my, Bx, By, E, psi)."""
    kind: int = field(default=PHYS_MHD_PLAIN, init=False)


@dataclass
class FiveMomentTwoFluid:  # src/two_fluid.mojo:139-206 (3D, 17 components)
    gamma_e: float = 5.0 / 3.0
    gamma_i: float = 5.0 / 3.0
    q_e: float = -1.0
    m_e: float = 1.0
    q_i: float = 1.0
    m_i: float = 25.0
    eps0: float = 1.0
    c_light: float = 10.0
    c_h: float = 0.0
    alpha_d: float = 0.0
    min_density: float = 1e-6
    min_pressure: float = 1e-8
    inflow: tuple = (0.0,) * 17
    kind: int = field(default=PHYS_TWO_FLUID, init=False)
    flux_type: int = field(default=0, init=False)
    entropy_fix: bool = field(default=False, init=False)

    def params(self):
        return [self.gamma_e, self.gamma_i, self.q_e, self.m_e, self.q_i, self.m_i, self.eps0, self.c_light,
                self.c_h, self.alpha_d, self.min_density, self.min_pressure] + list(self.inflow)


def physics_dict(ph):
    """Flat descriptor {kind, flux, entropy_fix, p} shared with the oracle."""
    return dict(kind=ph.kind, flux=ph.flux_type, entropy_fix=int(ph.entropy_fix), p=list(ph.params()))


@dataclass
class BoundaryConditions:  # src/boundary.mojo:326-343 ([-x, +x, -y, +y, -z, +z])
    bc_x_lo: int = BC_INTERIOR
    bc_x_hi: int = BC_INTERIOR
    bc_y_lo: int = BC_INTERIOR
    bc_y_hi: int = BC_INTERIOR
    bc_z_lo: int = BC_INTERIOR
    bc_z_hi: int = BC_INTERIOR

    @staticmethod
    def periodic():
        return BoundaryConditions()

    def all_periodic(self):
        return all(b == BC_INTERIOR for b in self.as_list())

    def as_list(self):
        return [self.bc_x_lo, self.bc_x_hi, self.bc_y_lo, self.bc_y_hi, self.bc_z_lo, self.bc_z_hi]


@dataclass
class Mesh:
    """Kuhn mesh: dim 3 -> nx*ny*nz cubes x 6 tets; dim 2 -> nx*ny cells x 2 triangles."""
    nx: int
    ny: int
    nz: int = 1
    lx: float = 1.0
    ly: float = 1.0
    lz: float = 1.0
    bcs: BoundaryConditions = field(default_factory=BoundaryConditions.periodic)
    dim: int = 3

    def desc(self):
        d = _MeshDesc()
        d.dim, d.nx, d.ny, d.nz = self.dim, self.nx, self.ny, self.nz
        d.lx, d.ly, d.lz = self.lx, self.ly, self.lz
        for k, b in enumerate(self.bcs.as_list()):
            d.bc[k] = b
        return d


class Solver:
    """Solver[PhysT, P] over the C ABI: device state q/q1/q2, SSPRK3, limiter."""

    def __init__(self, mesh: Mesh, physics, P: int = 2, precision: str = "f64", nparts: int = 1, part: int = 0):
        """`nparts` > 1: part `part` of a z-slab decomposition of `mesh` (3D), the
        reference's per-rank Solver over build_partition (src/partition.mojo:162)."""
        L = lib()
        pd = _PhysDesc()
        pd.kind, pd.flux_type, pd.entropy_fix = physics.kind, physics.flux_type, int(physics.entropy_fix)
        for k, v in enumerate(physics.params()):
            pd.p[k] = v
        md = mesh.desc()
        h = ctypes.c_void_p()
        if nparts == 1:
            _check(L.mxm_dg_create(ctypes.byref(md), ctypes.byref(pd), P, PREC[precision], ctypes.byref(h)))
        else:
            _check(L.mxm_dg_create_slab(ctypes.byref(md), ctypes.byref(pd), P, PREC[precision], nparts, part,
                                        ctypes.byref(h)))
        self.h = h
        self.mesh, self.physics, self.P, self.precision = mesh, physics, P, precision
        ne, np_, nfp, nc, rb = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _check(L.mxm_dg_sizes(h, ctypes.byref(ne), ctypes.byref(np_), ctypes.byref(nfp), ctypes.byref(nc),
                              ctypes.byref(rb)), h)
        self.num_elements, self.NP, self.NFP, self.NC = ne.value, np_.value, nfp.value, nc.value
        self.dtype = np.float64 if rb.value == 8 else np.float32
        self.shape = (self.num_elements, self.NP, self.NC)
        info = (ctypes.c_int64 * 8)()
        _check(L.mxm_dg_slab_info(h, info), h)
        self.nparts, self.part, cz0, cz1, glo, ghi, self.owned_e0, self.owned_ne = list(info)
        self.owned_layers, self.ghosts = (cz0, cz1), (glo, ghi)

    def close(self):
        if getattr(self, "h", None):
            lib().mxm_dg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        _check(rc, self.h)

    # -- state
    def state_ptr(self, which=0):
        p = ctypes.c_void_p()
        self._c(lib().mxm_dg_state_ptr(self.h, which, ctypes.byref(p)))
        return p.value

    @property
    def d_q(self):
        return self.state_ptr(0)

    def node_xyz(self):
        out = np.zeros((self.num_elements, self.NP, self.mesh.dim))
        self._c(lib().mxm_dg_node_xyz(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def node_xyz_f32(self):
        """Float32 node coordinates as the reference builds elem_node_xyz."""
        out = np.zeros((self.num_elements, self.NP, self.mesh.dim), np.float32)
        self._c(lib().mxm_dg_node_xyz_f32(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def node_xyz_ptr(self):
        p = ctypes.c_void_p()
        self._c(lib().mxm_dg_node_xyz_ptr(self.h, ctypes.byref(p)))
        return p.value

    def fill_ic(self, kind, params, which=0):
        """Device initial condition (mxm_dg_fill_ic) from node coordinates."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        self._c(lib().mxm_dg_fill_ic(self.h, which, kind, p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), p.size))

    def upload_state(self, q, which=0):
        a = np.ascontiguousarray(q, dtype=self.dtype).reshape(-1)
        assert a.size == self.num_elements * self.NP * self.NC, "state size mismatch"
        self._c(lib().mxm_dg_upload_state(self.h, which, a.ctypes.data, a.nbytes))

    def download_state(self, which=0):
        out = np.empty(self.shape, dtype=self.dtype)
        self._c(lib().mxm_dg_download_state(self.h, which, out.ctypes.data, out.nbytes))
        return out

    def download_owned_component(self, c):  # solver.mojo:711-729 (Float32 as the reference)
        out = np.empty(self.owned_ne * self.NP, dtype=np.float32)
        self._c(lib().mxm_dg_download_component(self.h, c, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    # -- stepping
    def enable_cell_limiter(self, enabled=True, venkat_eps=0.1):
        self._c(lib().mxm_dg_enable_limiter(self.h, int(enabled), venkat_eps))

    def step_ssprk3(self, dt):
        self._c(lib().mxm_dg_step_ssprk3(self.h, dt))

    def step_n(self, dt, nsteps):
        self._c(lib().mxm_dg_step_n(self.h, dt, nsteps))

    def rk_stage(self, stage, dt):
        self._c(lib().mxm_dg_rk_stage(self.h, stage, dt))

    def limit(self, which=0):
        self._c(lib().mxm_dg_limit(self.h, which))

    def rhs(self, q):
        """Semi-discrete RHS L(q) of a host array (uses q1 as scratch, q2 as output)."""
        self.upload_state(q, 1)
        self._c(lib().mxm_dg_eval_rhs(self.h, self.state_ptr(1), self.state_ptr(2)))
        return self.download_state(2)

    def advance_host(self, q_host, nsteps, dt, out=None):
        a = np.ascontiguousarray(q_host, dtype=self.dtype)
        out = np.empty_like(a) if out is None else out
        self._c(lib().mxm_dg_advance_host(self.h, a.ctypes.data, out.ctypes.data, nsteps, dt))
        return out

    def advance_host_async(self, q_host, nsteps, dt, out):
        """Enqueue upload + steps + download; `q_host` and `out` (pinned, e.g.
        PinnedArray) must stay alive until synchronize()."""
        assert q_host.flags["C_CONTIGUOUS"] and out.flags["C_CONTIGUOUS"] and out.nbytes == q_host.nbytes
        self._c(lib().mxm_dg_advance_host_async(self.h, q_host.ctypes.data, out.ctypes.data, nsteps, dt))

    def synchronize(self):
        self._c(lib().mxm_dg_synchronize(self.h))

    # -- z-slab decomposition
    def slab_layout(self):
        """{values per z layer, offsets of the bottom/top owned and lower/upper
        ghost layers in a state buffer (-1 = none)}."""
        out = (ctypes.c_int64 * 5)()
        self._c(lib().mxm_dg_slab_layout(self.h, out))
        return dict(zip(("layer", "owned_lo", "owned_hi", "ghost_lo", "ghost_hi"), list(out)))

    def slab_stage(self, stage, dt):
        """Stage kernel over the owned cells, without exchange or limiter."""
        self._c(lib().mxm_dg_slab_stage(self.h, stage, dt))

    def connect_nccl(self, unique_id: bytes):
        """Join the parts' NCCL communicator (collective over all parts)."""
        self._c(lib().mxm_dg_slab_connect_nccl(self.h, unique_id))

    # -- diagnostics
    def max_wavespeed(self):
        v = ctypes.c_double()
        self._c(lib().mxm_dg_max_wavespeed(self.h, ctypes.byref(v)))
        return v.value

    def integral(self, c, which=0, kind=0):
        v = ctypes.c_double()
        self._c(lib().mxm_dg_reduce_conserved(self.h, which, c, kind, ctypes.byref(v)))
        return v.value

    def dof_count(self):  # solver.mojo:757-763
        v = ctypes.c_int64()
        self._c(lib().mxm_dg_dof_count(self.h, ctypes.byref(v)))
        return v.value

    def state_bytes_per_step(self):  # solver.mojo:804-824
        v = ctypes.c_int64()
        self._c(lib().mxm_dg_state_bytes_per_step(self.h, ctypes.byref(v)))
        return v.value

    def launches_per_step(self):
        v = ctypes.c_int32()
        self._c(lib().mxm_dg_launches_per_step(self.h, ctypes.byref(v)))
        return v.value

    def time_steps(self, dt, nsteps):
        ms = ctypes.c_double()
        self._c(lib().mxm_dg_time_steps(self.h, dt, nsteps, ctypes.byref(ms)))
        return ms.value

    def bench_step_loop(self, dt, warmup_steps=5, measure_steps=50):
        """solver.mojo:765-802: warm up, then time `measure_steps` steps (CUDA events)."""
        self.step_n(dt, warmup_steps)
        self.synchronize()
        ms = self.time_steps(dt, measure_steps)
        dof = self.dof_count()
        return dict(steps=measure_steps, seconds=ms * 1e-3, dof_per_step=dof,
                    dof_stage_per_s=3 * dof * measure_steps / (ms * 1e-3),
                    state_gbs=self.state_bytes_per_step() * measure_steps / (ms * 1e-3) / 1e9)

    def operator(self):
        n = ctypes.c_int64(0)
        self._c(lib().mxm_dg_operator(self.h, None, ctypes.byref(n)))
        out = np.zeros(n.value)
        self._c(lib().mxm_dg_operator(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(n)))
        return out


def nccl_unique_id() -> bytes:
    """128-byte NCCL id for mxm_dg_slab_connect_nccl (made on one part, sent to all)."""
    buf = ctypes.create_string_buffer(128)
    _check(lib().mxm_dg_nccl_unique_id(buf))
    return buf.raw


class SlabGroup:
    """Parts 0..n-1 of one slab decomposition stepped in lock-step from this
    process (mxm_dg_group_*): ghost layers by cudaMemcpyPeerAsync."""

    def __init__(self, parts):
        self.parts = list(parts)
        arr = (ctypes.c_void_p * len(self.parts))(*[p.h.value for p in self.parts])
        g = ctypes.c_void_p()
        _check(lib().mxm_dg_group_create(arr, len(self.parts), ctypes.byref(g)))
        self.g = g

    def _c(self, rc):
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            lib().mxm_dg_group_last_error(self.g, buf, 512)
            raise DGError(rc, buf.value.decode())

    def step_n(self, dt, nsteps):
        self._c(lib().mxm_dg_group_step_n(self.g, dt, nsteps))

    def synchronize(self):
        self._c(lib().mxm_dg_group_synchronize(self.g))

    def time_steps(self, dt, nsteps):
        """Device time (ms) of `nsteps` group steps (CUDA events)."""
        v = ctypes.c_double()
        self._c(lib().mxm_dg_group_time_steps(self.g, dt, nsteps, ctypes.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "g", None):
            lib().mxm_dg_group_destroy(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DiagComponents:  # src/diagnostics.mojo:73-94
    """Named components for DiagnosticsWriter: linear (sum q), squared (sum q^2), max |q|."""

    def __init__(self):
        self.linear_, self.squared_, self.maxabs_ = [], [], []

    def linear(self, name, c):
        self.linear_.append((name, c))
        return self

    def squared(self, name, c):
        self.squared_.append((name, c))
        return self

    def maxabs(self, name, c):
        self.maxabs_.append((name, c))
        return self


class DiagnosticsWriter:  # src/diagnostics.mojo:96-229
    """CSV diagnostics of a Solver with the reference's columns and
    definitions (linear / squared rows: node sums times domain volume /
    (elements x nodes); max |q|), computed by FP64 device reductions
    (reduction kinds 3, 4, 2) instead of downloading each component."""

    def __init__(self, solver, components, csv_path=None):
        self.solver, self.comp, self.csv_path = solver, components, csv_path
        self.last_row = []
        if csv_path:
            cols = ["t"] + [n for n, _ in components.linear_ + components.squared_ + components.maxabs_]
            with open(csv_path, "w") as f:
                f.write(",".join(cols) + "\n")

    def record(self, t, which=0):
        s = self.solver
        self.last_row = ([s.integral(c, which, kind=3) for _, c in self.comp.linear_] +
                         [s.integral(c, which, kind=4) for _, c in self.comp.squared_] +
                         [s.integral(c, which, kind=2) for _, c in self.comp.maxabs_])
        if self.csv_path:
            with open(self.csv_path, "a") as f:
                f.write(",".join(repr(float(v)) for v in [t] + self.last_row) + "\n")
        return self.last_row


class Batch:
    """Many independent solves advanced together (mxm_dg_batch_*), the SSPRK3
    step captured as a CUDA graph: 2D solves in one persistent stage launch
    per physics group and stage (tile sizes autotuned per (group, P)); 3D
    tensor-core solves (precision "mixed" / "tf32") in one launch per
    (physics, order, operand kind) and stage; other 3D solves by their own
    launches in the same graph."""

    def __init__(self):
        h = ctypes.c_void_p()
        rc = lib().mxm_dg_batch_create(ctypes.byref(h))
        if rc != OK:
            raise DGError(rc, self._err(None))
        self.h = h
        self.members = []
        self.dts = []

    @staticmethod
    def _err(h):
        buf = ctypes.create_string_buffer(1024)
        lib().mxm_dg_batch_last_error(h, buf, 1024)
        return buf.value.decode(errors="replace")

    def _c(self, rc):
        if rc != OK:
            raise DGError(rc, self._err(self.h))

    def add(self, solver: Solver, dt: float) -> int:
        i = ctypes.c_int32()
        self._c(lib().mxm_dg_batch_add(self.h, solver.h, dt, ctypes.byref(i)))
        self.members.append(solver)
        self.dts.append(dt)
        return i.value

    def autotune(self):
        self._c(lib().mxm_dg_batch_autotune(self.h))

    def tile_cells(self, member):
        v = ctypes.c_int32()
        self._c(lib().mxm_dg_batch_tile_cells(self.h, member, ctypes.byref(v)))
        return v.value

    def step(self, nsteps=1):
        self._c(lib().mxm_dg_batch_step(self.h, nsteps))

    def time_steps(self, nsteps):
        ms = ctypes.c_double()
        self._c(lib().mxm_dg_batch_time_steps(self.h, nsteps, ctypes.byref(ms)))
        return ms.value

    def synchronize(self):
        self._c(lib().mxm_dg_batch_synchronize(self.h))

    def dof_count(self):
        v = ctypes.c_int64()
        self._c(lib().mxm_dg_batch_dof_count(self.h, ctypes.byref(v)))
        return v.value

    def launches_per_step(self):
        v = ctypes.c_int32()
        self._c(lib().mxm_dg_batch_launches_per_step(self.h, ctypes.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            lib().mxm_dg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _phys_desc(physics):
    pd = _PhysDesc()
    pd.kind, pd.flux_type, pd.entropy_fix = physics.kind, physics.flux_type, int(physics.entropy_fix)
    for k, v in enumerate(physics.params()):
        pd.p[k] = v
    return pd


def state_shape(mesh: Mesh, physics, P: int):
    """(Ne, NP, NC) of a solve on `mesh` with `physics` at order P."""
    dim = mesh.dim
    ne = mesh.nx * mesh.ny * (mesh.nz if dim == 3 else 1) * (6 if dim == 3 else 2)
    NP = (P + 1) * (P + 2) * (P + 3) // 6 if dim == 3 else (P + 1) * (P + 2) // 2
    NC = {PHYS_ADVECTION: 1, PHYS_EULER: 5 if dim == 3 else 4, PHYS_MAXWELL: 6, PHYS_SHALLOW_WATER: 3}[physics.kind]
    return ne, NP, NC


class Server:
    """Continuous-batching serving loop (mxm_dg_server_*): requests are
    admitted by HBM budget, run concurrently on their own streams, and their
    final states land in host arrays."""

    def __init__(self, hbm_budget_bytes=150e9, max_active=64, steps_per_chunk=10):
        h = ctypes.c_void_p()
        _check(lib().mxm_dg_server_create(hbm_budget_bytes, max_active, steps_per_chunk, ctypes.byref(h)))
        self.h = h
        self._out = {}

    def _errmsg(self):
        buf = ctypes.create_string_buffer(1024)
        lib().mxm_dg_server_last_error(self.h, buf, 1024)
        return buf.value.decode(errors="replace")

    def submit(self, mesh: Mesh, physics, P, precision, ic_kind, ic_params, dt, nsteps, limiter_eps=None,
               keep_result=True):
        """Queue one solve; its final state lands in a host array (result())
        unless keep_result is False (the server then copies nothing back)."""
        shape = state_shape(mesh, physics, P)
        out = np.empty(shape, dtype=np.float64 if precision == "f64" else np.float32) if keep_result else None
        p = np.ascontiguousarray(ic_params, dtype=np.float64)
        md, pd = mesh.desc(), _phys_desc(physics)
        rid = ctypes.c_int64()
        rc = lib().mxm_dg_server_submit(self.h, ctypes.byref(md), ctypes.byref(pd), P, PREC[precision], ic_kind,
                                        p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), p.size,
                                        0 if limiter_eps is None else 1,
                                        0.1 if limiter_eps is None else limiter_eps, dt, nsteps,
                                        None if out is None else out.ctypes.data, ctypes.byref(rid))
        if rc != OK:
            raise DGError(rc, self._errmsg())
        self._out[rid.value] = out
        return rid.value

    def poll(self, rid):
        lat = ctypes.c_double()
        rc = lib().mxm_dg_server_poll(self.h, rid, ctypes.byref(lat))
        if rc == ENOTREADY:
            return None
        if rc != OK:
            raise DGError(rc, self._errmsg())
        return lat.value

    def wait(self, rid, timeout_s=600.0):
        """Latency in ms once the request finished."""
        lat = ctypes.c_double()
        rc = lib().mxm_dg_server_wait(self.h, rid, timeout_s, ctypes.byref(lat))
        if rc != OK:
            raise DGError(rc, self._errmsg())
        return lat.value

    def result(self, rid):
        self.wait(rid)
        return self._out[rid]

    def stats(self):
        v = np.zeros(12)
        _check(lib().mxm_dg_server_stats(self.h, v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 12))
        keys = ["completed", "failed", "p50_ms", "p99_ms", "mean_ms", "solves_per_s", "dof_stage_per_s",
                "peak_bytes", "peak_concurrent", "queued", "running", "bytes_in_use"]
        return dict(zip(keys, v.tolist()))

    def close(self):
        if getattr(self, "h", None):
            lib().mxm_dg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def selftest_wait_timeout(limit_ms=50.0):
    """(gave_up, waited_ms) of a device wait on a barrier nothing completes."""
    g, w = ctypes.c_int32(), ctypes.c_double()
    _check(lib().mxm_dg_selftest_wait_timeout(limit_ms, ctypes.byref(g), ctypes.byref(w)))
    return g.value, w.value


def reference_operators(dim, P):
    """Host FP64 operators the library builds: D [dim,NP,NP], Lift [nf,NP,NFP] (reference face order), w [NP]."""
    NP = (P + 1) * (P + 2) * (P + 3) // 6 if dim == 3 else (P + 1) * (P + 2) // 2
    NFP = (P + 1) * (P + 2) // 2 if dim == 3 else P + 1
    nf = dim + 1
    D = np.zeros(dim * NP * NP)
    Lf = np.zeros(nf * NP * NFP)
    w = np.zeros(NP)
    dp = ctypes.POINTER(ctypes.c_double)
    _check(lib().mxm_dg_reference_operators(dim, P, D.ctypes.data_as(dp), Lf.ctypes.data_as(dp), w.ctypes.data_as(dp)))
    return D.reshape(dim, NP, NP), Lf.reshape(nf, NP, NFP), w
