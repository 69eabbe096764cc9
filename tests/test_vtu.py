"""VTU / PVD frame output in the reference's on-disk layout (src/vtu.mojo,
src/vtu_2d.mojo, src/frame_writer.mojo): arrays read back from the appended
block, cell types per order, identity connectivity, collection file."""
import os

import numpy as np
import pytest

import mojoxm_b200 as M
from mojoxm_b200 import vtu
from tests import dgcases


@pytest.mark.parametrize("P,ctype", [(2, 24), (3, 71), (5, 71)])
def test_vtu_3d_roundtrip(oracle_mod, tmp_path, P, ctype):
    o = oracle_mod.Oracle3D(P, (2, 1, 1), 1.0, M.physics_dict(dgcases.euler(M.FLUX_RUSANOV)))
    xyz = o.node_xyz().reshape(-1, 3)
    rho = np.random.default_rng(P).uniform(size=len(xyz))
    p = np.random.default_rng(P + 1).uniform(size=len(xyz))
    path = str(tmp_path / "f.vtu")
    vtu.write_vtu(path, xyz, [("rho", rho), ("p", p)], o.NP, 3)
    r = vtu.read_vtu(path)
    assert r["npoints"] == len(xyz) and r["ncells"] == o.Ne
    assert np.array_equal(r["rho"], rho.astype(np.float32)) and np.array_equal(r["p"], p.astype(np.float32))
    assert np.array_equal(r["points"].reshape(-1, 3), xyz.astype(np.float32))
    assert np.array_equal(r["connectivity"], np.arange(len(xyz)))
    assert np.array_equal(r["offsets"], (np.arange(o.Ne) + 1) * o.NP)
    assert set(r["types"].tolist()) == {ctype}
    assert r["header"].startswith('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="0.1" '
                                  'byte_order="LittleEndian" header_type="UInt32">\n')
    assert '<PointData Scalars="rho">' in r["header"]
    assert open(path, "rb").read().endswith(b"\n</AppendedData>\n</VTKFile>\n")


@pytest.mark.parametrize("P,ctype", [(1, 5), (2, 22), (4, 69)])
def test_vtu_2d_points_have_zero_z(oracle_mod, tmp_path, P, ctype):
    o = oracle_mod.Oracle2D(P, 2, 1.0, M.physics_dict(dgcases.euler(M.FLUX_RUSANOV)))
    xy = o.node_xy().reshape(-1, 2)
    path = str(tmp_path / "f.vtu")
    vtu.write_vtu(path, xy, [("q", np.arange(len(xy)))], o.NP, 2)
    r = vtu.read_vtu(path)
    pts = r["points"].reshape(-1, 3)
    assert np.array_equal(pts[:, :2], xy.astype(np.float32)) and not pts[:, 2].any()
    assert set(r["types"].tolist()) == {ctype}


def test_pvd_and_names(tmp_path):
    assert vtu.vtu_frame_name("frame_", 7) == "frame_00007.vtu"
    assert vtu.vtu_frame_name("f", 123456, 3) == "f123456.vtu"
    path = str(tmp_path / "run.pvd")
    vtu.write_pvd(path, ["a.vtu", "b.vtu"], [0.0, 0.25])
    txt = open(path).read()
    assert txt.count("<DataSet ") == 2 and 'timestep="0.25" group="" part="0" file="b.vtu"' in txt
    with pytest.raises(ValueError):
        vtu.write_pvd(path, ["a.vtu"], [0.0, 1.0])
    with pytest.raises(ValueError):
        vtu.vtu_bytes(np.zeros((10, 3)), [("q", np.zeros(9))], 10, 3)


@pytest.mark.gpu
def test_frame_writer_solver_and_slab_part(tmp_path):
    ph = dgcases.euler(M.FLUX_RUSANOV)
    mesh = M.Mesh(4, 2, 4, 1.0, 1.0, 1.0)
    s = M.Solver(mesh, ph, P=3, precision="f32")
    s.fill_ic(M.IC_SINE_WAVE, [1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0])
    fw = vtu.FrameWriter(s, str(tmp_path / "plain"))
    fw.write_frame(0.0)
    s.step_n(1e-3, 2)
    fw.write_frame(2e-3)
    pvd = fw.finalize("out/run.pvd")
    assert os.path.basename(pvd) == "run.pvd" and fw.num_frames_written() == 2
    r = vtu.read_vtu(str(tmp_path / "plain" / "frame_00001.vtu"))
    assert np.array_equal(r["density"], s.download_owned_component(0))
    part = M.Solver(mesh, ph, P=3, precision="f32", nparts=2, part=1)
    fw2 = vtu.FrameWriter(part, str(tmp_path / "dec"))
    fw2.write_frame(0.0)
    fw2.finalize("run.pvd")
    r2 = vtu.read_vtu(str(tmp_path / "dec" / "rank_001" / "frame_00000.vtu"))
    assert r2["ncells"] == part.owned_ne
    g0 = part.owned_layers[0] * 4 * 2 * 6  # first owned element in the undecomposed numbering
    xyz = s.node_xyz_f32().reshape(-1, 3)[g0 * s.NP:(g0 + part.owned_ne) * s.NP]
    assert np.array_equal(r2["points"].reshape(-1, 3), xyz)
    assert np.abs(s.node_xyz_f32() - s.node_xyz()).max() < 1e-6
