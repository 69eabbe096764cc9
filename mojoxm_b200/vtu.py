"""VTU frame output of DG fields (ParaView), the reference's on-disk format.

Reference: VtuWriter / dump_vtu_3d_frame_multi (src/vtu.mojo:103-250,
:291-418), dump_vtu_2d_frame_multi and vtu_frame_name (src/vtu_2d.mojo:
188-330), write_pvd (src/vtu.mojo:251-289) and FrameWriter
(src/frame_writer.mojo:60-206).  The file layout is an interface and is kept
as the reference writes it: a VTK UnstructuredGrid, little-endian,
UInt32 headers, every array in one raw appended block, each array preceded by
its UInt32 byte count, in the order fields..., points (3 x Float32, z = 0 in
2D), connectivity (identity: every element owns its NP nodes, so DG jumps
stay visible), offsets ((e+1) NP) and cell types (tet: 24 at NP = 10, else 71;
triangle: 5 at P = 1, 22 at P = 2, else 69).

B200 side: the frame's field is one component of the device state, copied
to the host once (the owned elements, FP32 as the reference downloads it);
the Float32 node coordinates (the reference's elem_node_xyz) are fetched
once per writer and kept; serialisation is
vectorised numpy and the file write runs on a background thread, so the
solver keeps stepping while the previous frame goes to disk (the role of the
reference's AsyncWriter).
"""
from __future__ import annotations

import os
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

VTK_TRIANGLE, VTK_QUADRATIC_TRIANGLE, VTK_LAGRANGE_TRIANGLE = 5, 22, 69
VTK_QUADRATIC_TETRA, VTK_LAGRANGE_TETRAHEDRON = 24, 71


def cell_type(dim: int, nodes_per_elem: int) -> int:
    if dim == 3:
        return VTK_QUADRATIC_TETRA if nodes_per_elem == 10 else VTK_LAGRANGE_TETRAHEDRON
    return {3: VTK_TRIANGLE, 6: VTK_QUADRATIC_TRIANGLE}.get(nodes_per_elem, VTK_LAGRANGE_TRIANGLE)


def vtu_frame_name(prefix: str, i: int, width: int = 5) -> str:
    """`prefix` + zero-padded index + `.vtu` (src/vtu_2d.mojo:314-326)."""
    return f"{prefix}{i:0{width}d}.vtu"


def vtu_bytes(xyz, fields, nodes_per_elem: int, dim: int) -> bytes:
    """One frame as bytes.  `xyz`: (points, dim) node coordinates (element-
    major); `fields`: [(name, values per point)], the first is the default
    Scalars array."""
    if not fields:
        raise ValueError("at least one field required")
    xyz = np.asarray(xyz, dtype=np.float32).reshape(-1, dim)
    npts = xyz.shape[0]
    if npts % nodes_per_elem:
        raise ValueError("point count is not a multiple of nodes_per_elem")
    ne = npts // nodes_per_elem
    pts = np.zeros((npts, 3), np.float32)
    pts[:, :dim] = xyz
    arrays = []
    for name, v in fields:
        v = np.asarray(v, dtype=np.float32).reshape(-1)
        if v.size != npts:
            raise ValueError(f"field {name!r} has {v.size} values, expected {npts}")
        arrays.append(v)
    conn = np.arange(npts, dtype="<i4")
    offs = (np.arange(1, ne + 1, dtype=np.int64) * nodes_per_elem).astype("<i4")
    types = np.full(ne, cell_type(dim, nodes_per_elem), np.uint8)
    blobs = [a.astype("<f4", copy=False) for a in arrays] + [pts.astype("<f4", copy=False), conn, offs, types]
    at, offsets = 0, []
    for b in blobs:
        offsets.append(at)
        at += 4 + b.nbytes
    nf = len(fields)
    h = ['<?xml version="1.0"?>\n',
         '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian" header_type="UInt32">\n',
         "<UnstructuredGrid>\n",
         f'<Piece NumberOfPoints="{npts}" NumberOfCells="{ne}">\n',
         f'<PointData Scalars="{fields[0][0]}">\n']
    for i, (name, _) in enumerate(fields):
        h.append(f'<DataArray type="Float32" Name="{name}" format="appended" offset="{offsets[i]}"/>\n')
    h += ["</PointData>\n", "<Points>\n",
          f'<DataArray type="Float32" NumberOfComponents="3" format="appended" offset="{offsets[nf]}"/>\n',
          "</Points>\n", "<Cells>\n",
          f'<DataArray type="Int32" Name="connectivity" format="appended" offset="{offsets[nf + 1]}"/>\n',
          f'<DataArray type="Int32" Name="offsets" format="appended" offset="{offsets[nf + 2]}"/>\n',
          f'<DataArray type="UInt8" Name="types" format="appended" offset="{offsets[nf + 3]}"/>\n',
          "</Cells>\n", "</Piece>\n", "</UnstructuredGrid>\n", '<AppendedData encoding="raw">\n_']
    out = [("".join(h)).encode()]
    for b in blobs:
        out.append(np.uint32(b.nbytes).astype("<u4").tobytes())
        out.append(b.tobytes())
    out.append(b"\n</AppendedData>\n</VTKFile>\n")
    return b"".join(out)


def write_vtu(path: str, xyz, fields, nodes_per_elem: int, dim: int) -> None:
    with open(path, "wb") as f:
        f.write(vtu_bytes(xyz, fields, nodes_per_elem, dim))


def write_pvd(path: str, vtu_paths, times) -> None:
    """ParaView collection of frames (src/vtu.mojo:251-289); paths relative to
    the .pvd's directory."""
    if len(vtu_paths) != len(times):
        raise ValueError(f"vtu_paths/times length mismatch ({len(vtu_paths)} vs {len(times)})")
    s = ['<?xml version="1.0"?>\n', '<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">\n',
         "<Collection>\n"]
    for p, t in zip(vtu_paths, times):
        s.append(f'<DataSet timestep="{float(t)!r}" group="" part="0" file="{p}"/>\n')
    s += ["</Collection>\n", "</VTKFile>\n"]
    with open(path, "w") as f:
        f.write("".join(s))


def read_vtu(path: str) -> dict:
    """Parse a frame written by this module back into arrays (for checks)."""
    import re
    raw = open(path, "rb").read()
    mark = b'<AppendedData encoding="raw">\n_'
    cut = raw.index(mark) + len(mark)
    head, blob = raw[:cut].decode(), raw[cut:]
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: Name="(\w+)")?(?: NumberOfComponents="3")? format="appended" '
                         r'offset="(\d+)"/>', head):
        typ, name, off = m.group(1), m.group(2) or "points", int(m.group(3))
        n = int(np.frombuffer(blob[off:off + 4], "<u4")[0])
        dt = {"Float32": "<f4", "Int32": "<i4", "UInt8": "u1"}[typ]
        out[name] = np.frombuffer(blob[off + 4:off + 4 + n], dt)
    m = re.search(r'NumberOfPoints="(\d+)" NumberOfCells="(\d+)"', head)
    out["npoints"], out["ncells"] = int(m.group(1)), int(m.group(2))
    out["header"] = head
    return out


class FrameWriter:
    """Per-frame VTU output of a Solver (FrameWriter, src/frame_writer.mojo:
    60-206): owned elements only; a part of a slab decomposition writes under
    `output_dir/rank_NNN` as the reference's ranks do."""

    def __init__(self, solver, output_dir: str, component: int = 0, field_name: str = "density"):
        self.s, self.component, self.field_name = solver, component, field_name
        nparts = getattr(solver, "nparts", 1)
        self.output_dir = os.path.join(output_dir, f"rank_{solver.part:03d}") if nparts > 1 else output_dir
        os.makedirs(self.output_dir, exist_ok=True)
        dim = solver.mesh.dim
        e0, ne = getattr(solver, "owned_e0", 0), getattr(solver, "owned_ne", solver.num_elements)
        self.xyz = np.ascontiguousarray(solver.node_xyz_f32()[e0:e0 + ne])  # once per writer
        self.dim, self.NP = dim, solver.NP
        self.paths, self.times = [], []
        self._pool = ThreadPoolExecutor(max_workers=1)
        self._pending = []
        self._lock = threading.Lock()

    def _submit(self, fname, fields):
        path = os.path.join(self.output_dir, fname)
        fut = self._pool.submit(write_vtu, path, self.xyz, fields, self.NP, self.dim)
        with self._lock:
            self._pending.append(fut)

    def write_frame(self, t: float) -> str:
        """Download the component and write the frame in the background."""
        q = self.s.download_owned_component(self.component)  # FP32, owned elements
        fname = vtu_frame_name("frame_", len(self.paths))
        self._submit(fname, [(self.field_name, q)])
        self.paths.append(fname)
        self.times.append(t)
        return fname

    def write_frame_multi(self, t: float, field_names, field_data) -> str:
        """Several host-side fields (one value per owned node each)."""
        if len(field_names) != len(field_data):
            raise ValueError("field_names/field_data length mismatch")
        fname = vtu_frame_name("frame_", len(self.paths))
        self._submit(fname, list(zip(field_names, [np.asarray(d) for d in field_data])))
        self.paths.append(fname)
        self.times.append(t)
        return fname

    def num_frames_written(self) -> int:
        return len(self.paths)

    def finalize(self, pvd_path: str) -> str:
        """Wait for the pending writes, then write the collection file next to
        the frames (basename of `pvd_path`)."""
        with self._lock:
            pending, self._pending = self._pending, []
        for f in pending:
            f.result()
        dst = os.path.join(self.output_dir, os.path.basename(pvd_path))
        write_pvd(dst, self.paths, self.times)
        self._pool.shutdown(wait=True)
        return dst
