"""z-slab domain decomposition with a one-layer halo (the reference's np > 1
path: src/partition.mojo:106-228, src/halo_exchange.mojo:187-395).

CPU: the library's slab plan (host-only), and the caller-driven exchange
schedule of tests/torch_halo.py over torch.distributed gloo with 2 and 3 ranks,
each rank stepping its slab with the oracle; the gathered owned layers must
equal the undecomposed oracle solve bit for bit.
GPU: slab parts stepped as an in-process group against the plain solve (bit
identical in FP64, FP32 and MIXED, with and without the limiter), the owned
diagnostics, the layout report and the NCCL transport's set-up.
"""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import mojoxm_b200 as M
from tests import torch_halo as halo
from tests import dgcases

P_CPU = 2
NX = NY = 2
NZ = 8  # cell size 1/8: local slab lengths are exact in binary


def test_slab_plan_partitions():
    for nz in range(1, 10):
        for nparts in range(1, min(nz, 5) + 1):
            for bc in ((0, 0), (1, 1), (2, 3)):
                plans = [halo.SlabPlan.of(nz, bc[0], bc[1], nparts, r) for r in range(nparts)]
                cover = [z for p in plans for z in range(p.cz0, p.cz1)]
                assert cover == list(range(nz))
                for r, p in enumerate(plans):
                    assert p.cz1 > p.cz0
                    if nparts == 1:
                        assert (p.ghost_lo, p.ghost_hi, p.bc_lo, p.bc_hi) == (0, 0, bc[0], bc[1])
                        continue
                    periodic = bc[0] == 0
                    assert p.ghost_lo == int(r > 0 or periodic) and p.ghost_hi == int(r < nparts - 1 or periodic)
                    assert p.bc_lo == (0 if p.ghost_lo else bc[0]) and p.bc_hi == (0 if p.ghost_hi else bc[1])
                    if p.ghost_hi:  # my upper neighbour's lower neighbour is me
                        assert plans[p.nb_hi].nb_lo == r
                        assert plans[p.nb_hi].cz0 == p.cz1 % nz
                    if p.ghost_lo:
                        assert plans[p.nb_lo].nb_hi == r
    with pytest.raises(M.DGError):
        halo.SlabPlan.of(2, 0, 0, 3, 0)  # fewer layers than parts
    with pytest.raises(M.DGError):
        halo.SlabPlan.of(8, 0, 1, 2, 0)  # one z boundary periodic, the other bounded


def _exchange_ops(nz, bc_lo, bc_hi, nparts, part):
    out = (ctypes.c_int32 * 12)()
    n = ctypes.c_int()
    assert M.lib().mxm_dg_slab_exchange_ops(nz, bc_lo, bc_hi, nparts, part, out, ctypes.byref(n)) == M.OK
    return [tuple(out[3 * k:3 * k + 3]) for k in range(n.value)]


def test_nccl_exchange_schedule_delivers_every_ghost_layer():
    """The library's own NCCL exchange order (mxm_dg_slab_exchange_ops, the
    list nccl_exchange issues), replayed without any transport: sends from
    part a to part b pair with receives on b from a in issue order, as NCCL
    point-to-point does.  Every ghost layer must receive exactly the
    neighbour's owned layer that it stands for (same global z layer), no
    owned layer may be received into, and no message may be left unpaired."""
    for nz in range(1, 10):
        for nparts in range(1, min(nz, 5) + 1):
            for bc in ((0, 0), (1, 1)):
                plans = [halo.SlabPlan.of(nz, bc[0], bc[1], nparts, r) for r in range(nparts)]
                ops = [_exchange_ops(nz, bc[0], bc[1], nparts, r) for r in range(nparts)]

                def glob(r, layer):  # global z layer of part r's local layer
                    return (plans[r].cz0 - plans[r].ghost_lo + layer) % nz

                sends, recvs = {}, {}
                for r, lst in enumerate(ops):
                    assert len(lst) == 2 * (plans[r].ghost_lo + plans[r].ghost_hi)
                    # a group's sends are issued before its receives
                    kinds = [k for k, _, _ in lst]
                    assert kinds == sorted(kinds)
                    for kind, peer, layer in lst:
                        assert 0 <= layer < plans[r].local_layers
                        (recvs if kind else sends).setdefault((r, peer) if not kind else (peer, r), []).append(
                            (r, layer))
                assert sorted(sends) == sorted(recvs)
                got = {}
                for key in sends:
                    assert len(sends[key]) == len(recvs[key])
                    for (a, la), (b, lb) in zip(sends[key], recvs[key]):
                        owned_a = plans[a].ghost_lo <= la < plans[a].local_layers - plans[a].ghost_hi
                        ghost_b = (lb == 0 and plans[b].ghost_lo) or (lb == plans[b].local_layers - 1 and plans[b].ghost_hi)
                        assert owned_a and ghost_b
                        assert glob(a, la) == glob(b, lb)
                        assert (b, lb) not in got
                        got[(b, lb)] = a
                want = {(r, 0) for r in range(nparts) if plans[r].ghost_lo} | \
                    {(r, plans[r].local_layers - 1) for r in range(nparts) if plans[r].ghost_hi}
                assert set(got) == want


def test_layer_offsets():
    p = halo.SlabPlan.of(8, 0, 0, 4, 1)
    o = halo.layer_offsets(p, 10)
    assert p.local_layers == 4 and o == dict(layer=10, owned_lo=10, owned_hi=20, ghost_lo=0, ghost_hi=30)
    p = halo.SlabPlan.of(8, 1, 1, 2, 0)  # first part of a bounded split: no lower ghost
    o = halo.layer_offsets(p, 10)
    assert p.local_layers == 5 and o == dict(layer=10, owned_lo=0, owned_hi=30, ghost_lo=-1, ghost_hi=40)


# ---- caller-driven exchange over gloo, the oracle as each rank's kernels ----

def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleBackend:
    """A rank's slab stepped by the oracle (test stand-in for SolverBackend):
    it computes its ghost elements too, which the next exchange overwrites."""

    def __init__(self, o, offs):
        self.o, self.offs, self.limiter_on = o, offs, False

    def begin_exchange(self, which):
        return torch.from_numpy(np.ascontiguousarray(self.o.get(which).reshape(-1)))

    def end_exchange(self, which, t):
        self.o.set(t.numpy(), which)

    def stage(self, s, dt):
        self.o.stage(s, dt)

    def limit(self, which):
        self.o.limit(which)


def _case(name):
    if name == "periodic":
        return dgcases.euler(M.FLUX_RUSANOV), (0,) * 6, False
    return dgcases.euler(M.FLUX_HLLEC), (0, 0, 1, 1, 1, 1), True  # walls in y and z, limiter on


def _local_slice(q, plan, nz, per_layer):
    """The part's local layers (ghosts included) cut from a global state."""
    layers = [(z % nz) for z in range(plan.cz0 - plan.ghost_lo, plan.cz1 + plan.ghost_hi)]
    return np.concatenate([q[z * per_layer:(z + 1) * per_layer] for z in layers])


def _gloo_worker(rank, world, port, case, steps, outq):
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ph, bcs, lim = _case(case)
        pd = M.physics_dict(ph)
        g = oracle.Oracle3D(P_CPU, (NX, NY, NZ), 1.0, pd, bcs=bcs)
        q0 = dgcases.random_state(g.shape, ph, seed=7).reshape(-1)
        plan = halo.SlabPlan.of(NZ, bcs[4], bcs[5], world, rank)
        per_layer = NX * NY * 6 * g.NP * g.NC
        lb = list(bcs[:4]) + [plan.bc_lo, plan.bc_hi]
        loc = oracle.Oracle3D(P_CPU, (NX, NY, plan.local_layers), (1.0, 1.0, plan.local_layers / NZ), pd, bcs=lb)
        loc.set(_local_slice(q0, plan, NZ, per_layer))
        be = OracleBackend(loc, halo.layer_offsets(plan, per_layer))
        be.limiter_on = lim
        halo.SlabDriver(be, plan).step(2e-3, steps)
        own = loc.get(0).reshape(-1)[plan.ghost_lo * per_layer:(plan.ghost_lo + plan.cz1 - plan.cz0) * per_layer]
        parts = [None] * world
        dist.all_gather_object(parts, (plan.cz0, own))
        if rank == 0:
            if lim:
                g.enable_limiter(True, 0.1)
            g.set(q0)
            g.step(2e-3, steps)
            ref = g.get(0).reshape(-1)
            got = np.concatenate([o for _, o in sorted(parts, key=lambda t: t[0])])
            outq.put((float(np.abs(got - ref).max()), bool(np.array_equal(got, ref)), float(np.abs(ref).max())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,case", [(2, "periodic"), (3, "bounded_limited")])
def test_gloo_slab_exchange_matches_undecomposed(oracle_mod, world, case):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, case, 3, q)) for r in range(world)]
    for p in procs:
        p.start()
    diff, equal, scale = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert equal, f"max |diff| {diff} (state scale {scale})"


# ---- GPU: the library's own slab path --------------------------------------

def _plain_and_parts(ph, bcs, P, prec, nparts, n=(4, 4, 8), lim=False, seed=3):
    mesh = M.Mesh(*n, 1.0, 1.0, 1.0, bcs=M.BoundaryConditions(*bcs))
    plain = M.Solver(mesh, ph, P=P, precision=prec)
    parts = [M.Solver(mesh, ph, P=P, precision=prec, nparts=nparts, part=r) for r in range(nparts)]
    q0 = dgcases.random_state(plain.shape, ph, seed=seed).astype(plain.dtype).reshape(-1)
    plain.upload_state(q0)
    per_layer = n[0] * n[1] * 6 * plain.NP * plain.NC
    for s in parts:
        plan = halo.SlabPlan.of(n[2], bcs[4], bcs[5], nparts, s.part)
        s.upload_state(_local_slice(q0, plan, n[2], per_layer))
        if lim:
            s.enable_cell_limiter(True, 0.1)
    if lim:
        plain.enable_cell_limiter(True, 0.1)
    return plain, parts, per_layer


def _owned(s, which=0):
    return s.download_state(which).reshape(-1)[s.owned_e0 * s.NP * s.NC:(s.owned_e0 + s.owned_ne) * s.NP * s.NC]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32", "mixed"])
@pytest.mark.parametrize("nparts", [1, 2, 3, 4])
@pytest.mark.parametrize("case", ["periodic", "bounded_limited"])
def test_group_bit_identical_to_plain(prec, nparts, case):
    ph, bcs, lim = _case(case)
    plain, parts, _ = _plain_and_parts(ph, bcs, 3, prec, nparts, lim=lim)
    grp = M.SlabGroup(parts)
    grp.step_n(1e-3, 4)
    grp.synchronize()
    plain.step_n(1e-3, 4)
    ref = plain.download_state(0).reshape(-1)
    got = np.concatenate([_owned(s) for s in parts])
    assert np.array_equal(got, ref), float(np.abs(got.astype(np.float64) - ref).max())
    grp.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,prec,bcs", [
    ("maxwell", "mixed", (0, 0, 1, 1, 1, 1)),
    ("mhd", "f32", (0,) * 6),
    ("shallow_water", "f64", (1, 1, 0, 0, 1, 1)),
    ("advection", "mixed", (3, 2, 0, 0, 3, 2)),
    ("two_fluid", "f32", (0,) * 6),
])
def test_group_bit_identical_other_physics(name, prec, bcs):
    ph = dgcases.two_fluid() if name == "two_fluid" else dgcases.PHYSICS_3D[name]()
    plain, parts, _ = _plain_and_parts(ph, bcs, 2, prec, 3, n=(2, 2, 6), lim=True)
    grp = M.SlabGroup(parts)
    assert grp.time_steps(5e-4, 3) > 0.0  # the same three steps, timed on the device
    grp.synchronize()
    plain.step_n(5e-4, 3)
    got = np.concatenate([_owned(s) for s in parts])
    assert np.array_equal(got, plain.download_state(0).reshape(-1))
    grp.close()


@pytest.mark.gpu
def test_slab_owned_diagnostics_and_layout():
    ph, bcs, _ = _case("periodic")
    plain, parts, per_layer = _plain_and_parts(ph, bcs, 2, "f64", 3, n=(4, 2, 7))
    grp = M.SlabGroup(parts)
    grp.step_n(1e-3, 2)
    grp.synchronize()
    plain.step_n(1e-3, 2)
    for kind in (0, 1, 3, 4):
        tot = sum(s.integral(0, kind=kind) for s in parts)
        ref = plain.integral(0, kind=kind)
        assert abs(tot - ref) <= 1e-12 * abs(ref)
    assert max(s.integral(4, kind=2) for s in parts) == plain.integral(4, kind=2)
    comp = np.concatenate([s.download_owned_component(4) for s in parts])
    assert np.array_equal(comp, plain.download_owned_component(4))
    xyz = np.concatenate([s.node_xyz()[s.owned_e0:s.owned_e0 + s.owned_ne] for s in parts])
    assert np.array_equal(xyz, plain.node_xyz())
    for s in parts:
        plan = halo.SlabPlan.of(7, 0, 0, 3, s.part)
        assert s.slab_layout() == halo.layer_offsets(plan, per_layer)
        assert s.owned_layers == (plan.cz0, plan.cz1) and s.ghosts == (plan.ghost_lo, plan.ghost_hi)
        # interior cells (when a part owns more than two layers) + the two boundary layers
        assert s.launches_per_step() == 3 * (2 + int(plan.cz1 - plan.cz0 > 2))
    grp.close()


@pytest.mark.gpu
def test_slab_ic_uses_global_positions():
    ph = dgcases.euler(M.FLUX_RUSANOV)
    mesh = M.Mesh(4, 4, 8, 1.0, 1.0, 1.0)
    plain = M.Solver(mesh, ph, P=2, precision="f64")
    plain.fill_ic(M.IC_SINE_WAVE, [1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0])
    for r in range(2):
        s = M.Solver(mesh, ph, P=2, precision="f64", nparts=2, part=r)
        s.fill_ic(M.IC_SINE_WAVE, [1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0])
        n = s.NP * s.NC
        got = _owned(s)
        ref = plain.download_state(0).reshape(-1)[s.owned_layers[0] * 4 * 4 * 6 * n:s.owned_layers[1] * 4 * 4 * 6 * n]
        assert np.array_equal(got, ref)


@pytest.mark.gpu
def test_slab_part_without_transport_refuses_to_step():
    ph, bcs, _ = _case("periodic")
    mesh = M.Mesh(2, 2, 4, 1.0, 1.0, 1.0, bcs=M.BoundaryConditions(*bcs))
    s = M.Solver(mesh, ph, P=2, precision="f64", nparts=2, part=0)
    with pytest.raises(M.DGError, match="group"):
        s.step_ssprk3(1e-3)


@pytest.mark.gpu
def test_solver_backend_tensor_aliases_state():
    ph, bcs, _ = _case("periodic")
    mesh = M.Mesh(2, 2, 4, 1.0, 1.0, 1.0, bcs=M.BoundaryConditions(*bcs))
    s = M.Solver(mesh, ph, P=2, precision="f32", nparts=2, part=1)
    be = halo.SolverBackend(s)
    t = be.begin_exchange(1)
    assert t.is_cuda and t.dtype == torch.float32 and t.numel() == s.num_elements * s.NP * s.NC
    t.copy_(torch.arange(t.numel(), dtype=torch.float32, device="cuda"))
    be.end_exchange(1, t)
    assert np.array_equal(s.download_state(1).reshape(-1), np.arange(t.numel(), dtype=np.float32))


@pytest.mark.gpu
def test_nccl_transport_single_part():
    """NCCL loads and a one-part communicator forms on one GPU (more parts
    need one GPU each)."""
    ph, bcs, _ = _case("periodic")
    mesh = M.Mesh(2, 2, 4, 1.0, 1.0, 1.0, bcs=M.BoundaryConditions(*bcs))
    s = M.Solver(mesh, ph, P=2, precision="f64")
    ref = M.Solver(mesh, ph, P=2, precision="f64")
    q0 = dgcases.random_state(s.shape, ph, seed=5).reshape(-1)
    s.upload_state(q0)
    ref.upload_state(q0)
    uid = M.nccl_unique_id()
    assert len(uid) == 128
    s.connect_nccl(uid)
    s.step_n(1e-3, 2)
    ref.step_n(1e-3, 2)
    assert np.array_equal(s.download_state(0), ref.download_state(0))
    s.close()
