"""VTU export of cell fields with inverse-distance-weighted point data.

Mirrors prism::output (export.h / export.cpp): `to_vtu` writes every given
scalar, vector and tensor field as CellData and as PointData interpolated to
the mesh vertices (cellToPoint, computed on the device by the library);
`FieldRegistry` collects fields for repeated exports and `TimeWriter` writes
`<prefix>_<step:04d>.vtu` every `write_interval` steps with an optional
`<prefix>.pvd` collection. The file layout is the VTK XML UnstructuredGrid
format: points are every mesh vertex, cells list their vertices in UNV element
node order with VTK types 12 (hexahedron), 10 (tetrahedron) and 13 (wedge).
Two encodings, as the reference offers: ASCII, and raw appended data
compressed with zlib (the vtkZLibDataCompressor block layout, UInt64 headers).
"""
import enum
import html
import struct
import xml.etree.ElementTree as ET
import zlib

import numpy as np

from . import _abi as A
from .api import Scalar, Tensor, Vector

VTK_TYPE = {8: 12, 4: 10, 6: 13}  # vertex count -> VTK cell type (export.cpp:210-218)
BLOCK = 1 << 15  # uncompressed bytes per zlib block


class WriteMode(enum.Enum):
    """output::WriteMode (export.h)."""
    Ascii = "Ascii"
    RawBinaryCompressed = "RawBinaryCompressed"


def _flatten(field):
    """Cell data interleaved per cell: scalar n, vector (x, y, z) per cell,
    tensor row-major per cell (flattenScalar/Vector/Tensor, export.cpp:126-176)."""
    if isinstance(field, Scalar):
        return field.values(), 1
    if isinstance(field, Vector):
        return field.values().T.reshape(-1).copy(), 3
    if isinstance(field, Tensor):
        return field.values().T.reshape(-1).copy(), 9
    raise TypeError(f"cannot export {type(field).__name__}")


def _points(field, cell_data, ncomp):
    if isinstance(field, Scalar):
        return field.to_points()
    if isinstance(field, Vector):
        return field.to_points().reshape(-1)
    return field.mesh.cell_to_point(cell_data, ncomp)


class _Array:
    def __init__(self, name, vtk_type, ncomp, data):
        self.name, self.vtk_type, self.ncomp, self.data = name, vtk_type, ncomp, data


_NP = {"Float64": "<f8", "Int64": "<i8", "UInt8": "u1"}


def _ascii(a):
    if a.vtk_type == "Float64":
        return " ".join(repr(float(v)) for v in a.data)
    return " ".join(str(int(v)) for v in a.data)


def _compressed(a):
    raw = np.ascontiguousarray(a.data, dtype=_NP[a.vtk_type]).tobytes()
    blocks = [zlib.compress(raw[i:i + BLOCK]) for i in range(0, len(raw), BLOCK)]
    header = [len(blocks), BLOCK, len(raw) % BLOCK] + [len(b) for b in blocks]
    return struct.pack(f"<{len(header)}Q", *header) + b"".join(blocks)


def _write(file_name, mesh, cell_arrays, point_arrays, mode):
    xyz, off, ids = mesh.topology()
    counts = np.diff(off)
    bad = [int(c) for c in np.unique(counts) if int(c) not in VTK_TYPE]
    if bad:
        raise RuntimeError("Unsupported cell type for vtu export.")
    geometry = [
        ("Points", _Array(None, "Float64", 3, xyz.reshape(-1))),
        ("Cells", _Array("connectivity", "Int64", 1, ids)),
        ("Cells", _Array("offsets", "Int64", 1, off[1:])),
        ("Cells", _Array("types", "UInt8", 1, np.array([VTK_TYPE[int(c)] for c in counts], np.uint8))),
    ]
    sections = geometry + [("PointData", a) for a in point_arrays] + [("CellData", a) for a in cell_arrays]
    binary = mode == WriteMode.RawBinaryCompressed
    payload, pos = [], 0
    out = ['<?xml version="1.0"?>\n']
    attrs = 'type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64"'
    if binary:
        attrs += ' compressor="vtkZLibDataCompressor"'
    out.append(f"<VTKFile {attrs}>\n<UnstructuredGrid>\n")
    out.append(f'<Piece NumberOfPoints="{xyz.shape[0]}" NumberOfCells="{mesh.n_cells}">\n')
    current = None
    for sec, a in sections:
        if sec != current:
            if current is not None:
                out.append(f"</{current}>\n")
            out.append(f"<{sec}>\n")
            current = sec
        name = f' Name="{html.escape(a.name, quote=True)}"' if a.name is not None else ""
        comps = f' NumberOfComponents="{a.ncomp}"' if a.ncomp > 1 else ""
        if binary:
            blob = _compressed(a)
            out.append(f'<DataArray type="{a.vtk_type}"{name}{comps} format="appended" offset="{pos}"/>\n')
            payload.append(blob)
            pos += len(blob)
        else:
            out.append(f'<DataArray type="{a.vtk_type}"{name}{comps} format="ascii">\n{_ascii(a)}\n</DataArray>\n')
    out.append(f"</{current}>\n</Piece>\n</UnstructuredGrid>\n")
    with open(file_name, "wb") as f:
        f.write("".join(out).encode())
        if binary:
            f.write(b'<AppendedData encoding="raw">\n_')
            for blob in payload:
                f.write(blob)
            f.write(b"\n</AppendedData>\n")
        f.write(b"</VTKFile>\n")


def to_vtu(file_name, scalars=(), vectors=(), tensors=(), mode=WriteMode.Ascii):
    """output::toVtu (export.cpp:256-301): fields must share one mesh; with no
    field nothing is written."""
    fields = list(scalars) + list(vectors) + list(tensors)
    if not fields:
        return
    mesh = fields[0].mesh
    cell_arrays, point_arrays = [], []
    for f in fields:
        if f.mesh is not mesh:
            raise A.PrismError(A.INVALID_MESH,
                               f"Field '{f.name}' does not share the mesh of the other exported fields.")
        data, ncomp = _flatten(f)
        cell_arrays.append(_Array(f.name, "Float64", ncomp, data))
        point_arrays.append(_Array(f.name, "Float64", ncomp, _points(f, data, ncomp)))
    _write(file_name, mesh, cell_arrays, point_arrays, WriteMode(mode))


class FieldRegistry:
    """output::FieldRegistry (export.cpp:303-337)."""

    def __init__(self):
        self.scalars, self.vectors, self.tensors = [], [], []

    def add(self, f):
        if isinstance(f, Scalar):
            self.scalars.append(f)
        elif isinstance(f, Vector):
            self.vectors.append(f)
        elif isinstance(f, Tensor):
            self.tensors.append(f)
        else:
            raise TypeError(f"cannot export {type(f).__name__}")

    def export_all(self, file_name, mode=WriteMode.Ascii):
        to_vtu(file_name, self.scalars, self.vectors, self.tensors, mode)


class TimeWriter:
    """output::TimeWriter (export.cpp:339-411)."""

    def __init__(self, prefix, write_interval=1, mode=WriteMode.Ascii, write_pvd=True):
        if write_interval <= 0:
            raise ValueError(f"write_interval must be positive, got {write_interval}")
        self.prefix, self.interval, self.mode, self.write_pvd = prefix, int(write_interval), mode, write_pvd
        self.registry = FieldRegistry()
        self.step, self.time = 0, 0.0
        self.pvd_entries = []

    def add(self, f):
        self.registry.add(f)

    def advance(self, dt):
        self.step += 1
        self.time += dt

    def write(self):
        if self.step % self.interval != 0:
            return
        r = self.registry
        if not (r.scalars or r.vectors or r.tensors):
            return
        name = f"{self.prefix}_{self.step:04d}.vtu"
        r.export_all(name, self.mode)
        if self.write_pvd:
            self.pvd_entries.append((self.time, name))
            self.flush_pvd()

    def write_and_advance(self, dt):
        self.advance(dt)
        self.write()

    def flush_pvd(self):
        with open(f"{self.prefix}.pvd", "w") as f:
            f.write('<?xml version="1.0"?>\n<VTKFile type="Collection" version="0.1">\n  <Collection>\n')
            for t, name in self.pvd_entries:
                f.write(f'    <DataSet timestep="{t:.6g}" file="{name}"/>\n')
            f.write("  </Collection>\n</VTKFile>\n")


def read_vtu(file_name):
    """Reads a file written by `to_vtu` back: {"points", "connectivity", "offsets",
    "types", "cell_data": {name: array}, "point_data": {name: array}} with arrays
    shaped (n, ncomp) where ncomp > 1."""
    with open(file_name, "rb") as f:
        content = f.read()
    appended = b""
    k = content.find(b'<AppendedData encoding="raw">')
    if k >= 0:
        start = content.index(b"_", k) + 1
        end = content.rindex(b"</AppendedData>")
        appended = content[start:end]
        content = content[:k] + b"</VTKFile>"
    root = ET.fromstring(content)
    piece = root.find("UnstructuredGrid/Piece")

    def decode(el):
        dt = _NP[el.get("type")]
        if el.get("format") == "appended":
            off = int(el.get("offset"))
            nb = struct.unpack_from("<Q", appended, off)[0]
            hdr = struct.unpack_from(f"<{3 + nb}Q", appended, off)
            pos, raw = off + 8 * (3 + nb), b""
            for s in hdr[3:]:
                raw += zlib.decompress(appended[pos:pos + s])
                pos += s
            a = np.frombuffer(raw, dtype=dt)
        else:
            a = np.array((el.text or "").split(), dtype=dt)
        nc = int(el.get("NumberOfComponents", "1"))
        return a.reshape(-1, nc) if nc > 1 else a

    out = {"points": decode(piece.find("Points/DataArray")), "cell_data": {}, "point_data": {}}
    for el in piece.findall("Cells/DataArray"):
        out[el.get("Name")] = decode(el)
    for sec, key in (("CellData", "cell_data"), ("PointData", "point_data")):
        for el in piece.findall(f"{sec}/DataArray"):
            out[key][el.get("Name")] = decode(el)
    return out
