"""Headless VTK output: XML StructuredGrid (``.vts``) files and the ``.pvd`` collection.

The reference writes its results with pyvista (``export_VTK_pyvista``,
src/LBM/LBM2D/_io.py:621-635): a structured grid whose node coordinates are
``linspace(0, X, nx)`` x ``linspace(0, Y, ny)`` x ``linspace(0, Z, nz)``
(src/LBM/LBM2D/_core.py:38-43), point data flattened in Fortran order (x fastest),
and a ``name.pvd`` collection listing every file with its time
(src/LBM/visualization_tool/PVD.py:9-84).  pyvista is not available here, so this
module writes the same VTK XML format directly: one binary ``AppendedData`` block
(raw, little-endian, UInt64 size headers), readable by ParaView, VTK and pyvista.
``read_vts`` reads such a file back (for tests and post-processing without VTK).
"""
from __future__ import annotations

import os
import re
import xml.etree.ElementTree as ET
from typing import Dict, Optional, Sequence, Tuple
from xml.dom import minidom

import numpy as np

_VTK_TYPES = {np.dtype(np.float32): "Float32", np.dtype(np.float64): "Float64",
              np.dtype(np.int32): "Int32", np.dtype(np.uint8): "UInt8", np.dtype(np.int64): "Int64"}
_NP_TYPES = {v: k for k, v in _VTK_TYPES.items()}


def _point_array(a: np.ndarray, shape: Tuple[int, int, int]) -> np.ndarray:
    """(nx, ny, nz[, c]) array -> (N[, c]) in VTK point order (x fastest)."""
    a = np.asarray(a)
    n = shape[0] * shape[1] * shape[2]
    if a.ndim >= 3 and a.shape[:3] == tuple(shape):
        if a.ndim == 3:
            return a.ravel(order="F")
        return a.reshape(n, -1, order="F")
    if a.shape[0] == n:
        return a
    raise ValueError(f"array of shape {a.shape} does not match the grid {shape}")


def write_vts(path: str, fields: Dict[str, np.ndarray], shape: Sequence[int],
              coords: Optional[Sequence[np.ndarray]] = None) -> str:
    """Write a structured grid of ``shape = (nx, ny, nz)`` nodes with point ``fields``.

    Each field is (nx, ny, nz) for a scalar, (nx, ny, nz, c) for c components, or
    already flat in VTK point order.  ``coords`` = the node coordinates along x, y, z
    (default: the node indices).  Float and integer arrays keep their type (float16
    is written as float32; bool as UInt8)."""
    nx, ny, nz = (int(s) for s in shape)
    shp = (nx, ny, nz)
    if coords is None:
        coords = (np.arange(nx), np.arange(ny), np.arange(nz))
    cx, cy, cz = (np.asarray(c, dtype=np.float64) for c in coords)
    gx, gy, gz = np.meshgrid(cx, cy, cz, indexing="ij")
    pts = np.stack([gx.ravel(order="F"), gy.ravel(order="F"), gz.ravel(order="F")], axis=1).astype(np.float32)
    blocks = []
    extent = f"0 {nx - 1} 0 {ny - 1} 0 {nz - 1}"
    root = ET.Element("VTKFile", type="StructuredGrid", version="1.0", byte_order="LittleEndian",
                      header_type="UInt64")
    grid = ET.SubElement(root, "StructuredGrid", WholeExtent=extent)
    piece = ET.SubElement(grid, "Piece", Extent=extent)
    pd = ET.SubElement(piece, "PointData")
    offset = 0

    def add(parent, name: Optional[str], a: np.ndarray):
        nonlocal offset
        if a.dtype == np.bool_:
            a = a.astype(np.uint8)
        elif a.dtype == np.float16:
            a = a.astype(np.float32)
        elif a.dtype not in _VTK_TYPES:
            a = a.astype(np.float64 if a.dtype.kind == "f" else np.int64)
        a = np.ascontiguousarray(a.astype(a.dtype.newbyteorder("<"), copy=False))
        attrs = {"type": _VTK_TYPES[np.dtype(a.dtype.newbyteorder("="))], "format": "appended",
                 "offset": str(offset)}
        if name is not None:
            attrs["Name"] = name
        ncomp = 1 if a.ndim == 1 else a.shape[1]
        if ncomp > 1 or name is None:
            attrs["NumberOfComponents"] = str(ncomp)
        ET.SubElement(parent, "DataArray", **attrs)
        raw = a.tobytes()
        blocks.append(np.uint64(len(raw)).tobytes() + raw)
        offset += 8 + len(raw)

    for name, a in fields.items():
        add(pd, name, _point_array(a, shp))
    add(ET.SubElement(piece, "Points"), None, pts)
    head = ET.tostring(root, encoding="unicode")
    head = head[: -len("</VTKFile>")]
    with open(path, "wb") as f:
        f.write(b'<?xml version="1.0"?>\n')
        f.write(head.encode())
        f.write(b'\n  <AppendedData encoding="raw">\n   _')
        for b in blocks:
            f.write(b)
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")
    return path


def read_vts(path: str) -> Dict[str, np.ndarray]:
    """Point data and points of a ``.vts`` written by ``write_vts``: flat arrays in VTK
    point order (x fastest), ``(N, c)`` for vectors; the grid shape under ``"_shape"``."""
    with open(path, "rb") as f:
        data = f.read()
    start = data.index(b'<AppendedData encoding="raw">')
    under = data.index(b"_", start) + 1
    head = data[:start].decode() + "</VTKFile>"
    head = re.sub(r"<\?xml[^>]*\?>", "", head)
    root = ET.fromstring(head)
    piece = root.find("StructuredGrid/Piece")
    e = [int(v) for v in piece.get("Extent").split()]
    shape = (e[1] - e[0] + 1, e[3] - e[2] + 1, e[5] - e[4] + 1)
    out: Dict[str, np.ndarray] = {"_shape": np.array(shape)}

    def load(da) -> np.ndarray:
        off = under + int(da.get("offset"))
        nbytes = int(np.frombuffer(data[off:off + 8], dtype="<u8")[0])
        dt = np.dtype(_NP_TYPES[da.get("type")]).newbyteorder("<")
        a = np.frombuffer(data[off + 8:off + 8 + nbytes], dtype=dt)
        nc = int(da.get("NumberOfComponents", "1"))
        return a.reshape(-1, nc) if nc > 1 else a

    for da in piece.findall("PointData/DataArray"):
        out[da.get("Name")] = load(da)
    out["_points"] = load(piece.find("Points/DataArray"))
    return out


class PVDWriter:
    """``name.pvd`` collection of time steps (src/LBM/visualization_tool/PVD.py:9-84):
    ``add(time, file)`` records a data set, ``write()`` rewrites ``path/name.pvd``."""

    def __init__(self, path: str = "output", name: str = "default_name"):
        self.exportPath = path
        self.name = name
        self.entries: list = []

    def add(self, time: float, filename: str) -> None:
        self.entries.append((float(time), filename))

    addVTK = add

    def write(self) -> str:
        root = ET.Element("VTKFile", type="Collection", version="0.1", byte_order="LittleEndian")
        col = ET.SubElement(root, "Collection")
        for t, fn in self.entries:
            ET.SubElement(col, "DataSet", timestep=repr(t), group="", part="0", file=fn, name=self.name)
        text = minidom.parseString(ET.tostring(root, encoding="utf-8")).toprettyxml(indent="    ")
        os.makedirs(self.exportPath or ".", exist_ok=True)
        out = os.path.join(self.exportPath, self.name + ".pvd")
        with open(out, "w", encoding="utf8") as f:
            f.write(text)
        return out

    writePVD = write


def read_pvd(path: str) -> list:
    """(time, file) of every data set of a ``.pvd`` collection."""
    root = ET.parse(path).getroot()
    return [(float(d.get("timestep")), d.get("file")) for d in root.iter("DataSet")]
