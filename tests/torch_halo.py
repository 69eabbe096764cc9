"""Caller-driven halo exchange of a z-slab decomposition over torch.distributed
(a test-side driver: the library itself uses no PyTorch; its own transports
are NCCL point-to-point and the in-process group of slab.cu).

The reference steps one patch per MPI rank and refills the patch's ghost
ring once per RK stage (HaloExchange.exchange, src/halo_exchange.mojo:
313-395, called from src/solver.mojo:1038-1068).  The library does the same
by itself once a part is connected to NCCL (`Solver.connect_nccl`); this
module is the other route, for a process group the caller already has: the
ghost layers move as torch.distributed point-to-point messages (NCCL on
GPUs, gloo on CPUs) and the part's kernels run through `Solver.slab_stage`
and `Solver.limit`.

Schedule of one SSPRK3 stage s (buffers q, q1, q2 = 0, 1, 2):
    exchange(in_s); stage s over the owned cells; and with the limiter on,
    exchange(out_s); limiter of out_s (its cell means reach the ghosts).

Messages: a part sends its top owned layer to its upper neighbour ("up",
tag 0) and its bottom owned layer to its lower neighbour ("down", tag 1);
it receives the up message from below into its lower ghost layer and the
down message from above into its upper ghost layer.  Sends are issued
(up, down) and receives (from below, from above) on every part, so two
parts that neighbour each other on both sides (two periodic parts) still
match when the transport pairs messages by issue order.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from mojoxm_b200 import DGError, lib

STAGE_IN = (0, 1, 2)   # Shu-Osher stage s reads q, q1, q2 ...
STAGE_OUT = (1, 2, 0)  # ... and writes q1, q2, q
TAG_UP, TAG_DOWN = 0, 1


@dataclass(frozen=True)
class SlabPlan:
    """Part `part` of an nparts-slab split of nz global z layers (the library's
    own plan, mxm_dg_slab_plan; host-only, needs no GPU)."""
    cz0: int
    cz1: int
    ghost_lo: int
    ghost_hi: int
    bc_lo: int
    bc_hi: int
    nb_lo: int
    nb_hi: int

    @staticmethod
    def of(nz: int, bc_z_lo: int, bc_z_hi: int, nparts: int, part: int) -> "SlabPlan":
        out = (ctypes.c_int32 * 8)()
        rc = lib().mxm_dg_slab_plan(nz, bc_z_lo, bc_z_hi, nparts, part, out)
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            lib().mxm_dg_last_error(None, buf, 512)
            raise DGError(rc, buf.value.decode())
        return SlabPlan(*list(out))

    @property
    def local_layers(self) -> int:
        return self.cz1 - self.cz0 + self.ghost_lo + self.ghost_hi


def layer_offsets(plan: SlabPlan, layer_values: int) -> dict:
    """Offsets (in values) of the owned boundary and ghost layers in a part's
    state buffer, as mxm_dg_slab_layout reports them."""
    top = plan.local_layers - plan.ghost_hi - 1
    return dict(layer=layer_values, owned_lo=plan.ghost_lo * layer_values, owned_hi=top * layer_values,
                ghost_lo=0 if plan.ghost_lo else -1,
                ghost_hi=(plan.local_layers - 1) * layer_values if plan.ghost_hi else -1)


def exchange(buf, plan: SlabPlan, offs: dict, group=None):
    """Refill the ghost layers of the flat tensor `buf` from the neighbours."""
    import torch.distributed as dist
    L = offs["layer"]
    ops = []
    if plan.ghost_hi:
        ops.append(dist.P2POp(dist.isend, buf[offs["owned_hi"]:offs["owned_hi"] + L], plan.nb_hi, group, TAG_UP))
    if plan.ghost_lo:
        ops.append(dist.P2POp(dist.isend, buf[offs["owned_lo"]:offs["owned_lo"] + L], plan.nb_lo, group, TAG_DOWN))
    recv = []
    if plan.ghost_lo:
        t = buf[offs["ghost_lo"]:offs["ghost_lo"] + L]
        recv.append(t)
        ops.append(dist.P2POp(dist.irecv, t, plan.nb_lo, group, TAG_UP))
    if plan.ghost_hi:
        t = buf[offs["ghost_hi"]:offs["ghost_hi"] + L]
        recv.append(t)
        ops.append(dist.P2POp(dist.irecv, t, plan.nb_hi, group, TAG_DOWN))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class _DeviceBuffer:
    """A state buffer of a Solver seen by torch through __cuda_array_interface__."""

    def __init__(self, ptr: int, n: int, dtype):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": np.dtype(dtype).str, "data": (ptr, False),
                                         "version": 3, "strides": None}


class SolverBackend:
    """The product side of SlabDriver: a slab part (`Solver(..., nparts, part)`)
    whose ghost layers travel as CUDA tensors (NCCL process group)."""

    def __init__(self, solver):
        import torch
        self.s, self.torch = solver, torch
        self.limiter_on = False
        self.eps = 0.1
        lay = solver.slab_layout()
        self.offs = lay
        self.n = solver.num_elements * solver.NP * solver.NC

    def enable_cell_limiter(self, on=True, eps=0.1):
        self.limiter_on, self.eps = bool(on), eps
        self.s.enable_cell_limiter(on, eps)

    def begin_exchange(self, which):
        self.s.synchronize()  # the part's stream has written the layers
        t = self.torch.as_tensor(_DeviceBuffer(self.s.state_ptr(which), self.n, self.s.dtype), device="cuda")
        return t

    def end_exchange(self, which, t):
        self.torch.cuda.current_stream().synchronize()  # the ghosts have landed

    def stage(self, s, dt):
        self.s.slab_stage(s, dt)

    def limit(self, which):
        self.s.limit(which)


class SlabDriver:
    """SSPRK3 stepping of one slab part with caller-driven exchanges."""

    def __init__(self, backend, plan: SlabPlan, group=None):
        self.b, self.plan, self.group = backend, plan, group

    def _exchange(self, which):
        t = self.b.begin_exchange(which)
        exchange(t, self.plan, self.b.offs, self.group)
        self.b.end_exchange(which, t)

    def step(self, dt, nsteps=1):
        for _ in range(nsteps):
            for s in range(3):
                self._exchange(STAGE_IN[s])
                self.b.stage(s, dt)
                if self.b.limiter_on:
                    self._exchange(STAGE_OUT[s])
                    self.b.limit(STAGE_OUT[s])
