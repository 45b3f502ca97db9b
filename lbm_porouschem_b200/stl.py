"""STL geometry: read a triangle mesh, place it, voxelise it on the GPU.

The reference's ``StlReader.voxel_stl`` (src/LBM/GEO/STL.py:118-268) reads the mesh
with pyvista, scales it, rotates it about z, then y, then x (degrees), translates it,
voxelises it and returns ``(voxel_array, surface_array)`` on the (nx, ny, nz) grid.
This module keeps that call and its transform order; the voxelisation is
``lbm_voxelise_stl`` (csrc/stl_kernels.cu): a cell is solid when its centre lies
inside the closed mesh.  Binary and ASCII STL files are read here (no pyvista).
"""
from __future__ import annotations

import ctypes
import logging
import os
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _native as N


def read_stl(path: str) -> np.ndarray:
    """Triangles of a binary or ASCII STL file as float32 [T, 3, 3] (vertex, xyz)."""
    with open(path, "rb") as f:
        data = f.read()
    if len(data) >= 84:
        n = int(np.frombuffer(data[80:84], dtype="<u4")[0])
        if len(data) == 84 + 50 * n:
            rec = np.frombuffer(data[84:], dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]), count=n)
            return rec["v"].reshape(n, 3, 3).astype(np.float32)
    text = data.decode("ascii", errors="replace")
    if not text.lstrip().lower().startswith("solid"):
        raise ValueError(f"{path}: neither a binary nor an ASCII STL file")
    verts = [line.split()[1:4] for line in text.splitlines() if line.strip().lower().startswith("vertex")]
    if len(verts) % 3:
        raise ValueError(f"{path}: vertex count is not a multiple of 3")
    return np.asarray(verts, dtype=np.float32).reshape(-1, 3, 3)


def write_stl(path: str, triangles: np.ndarray) -> str:
    """Binary STL of float [T, 3, 3] triangles (normals from the vertex order)."""
    t = np.asarray(triangles, dtype=np.float32).reshape(-1, 3, 3)
    nrm = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    ln = np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm = np.where(ln > 0, nrm / np.where(ln > 0, ln, 1), 0).astype(np.float32)
    rec = np.zeros(len(t), dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]))
    rec["n"], rec["v"] = nrm, t.reshape(-1, 9)
    with open(path, "wb") as f:
        f.write(b"lbm_b200 binary STL".ljust(80, b" "))
        f.write(np.uint32(len(t)).tobytes())
        f.write(rec.tobytes())
    return path


def _rot(axis: int, deg: float) -> np.ndarray:
    a = np.deg2rad(deg)
    c, s = np.cos(a), np.sin(a)
    i, j = [(1, 2), (2, 0), (0, 1)][axis]
    r = np.eye(3)
    r[i, i], r[i, j], r[j, i], r[j, j] = c, -s, s, c
    return r


def place(triangles: np.ndarray, scale=1.0, translate=(0, 0, 0), rotate=(0, 0, 0)) -> np.ndarray:
    """The reference's placement (src/LBM/GEO/STL.py:185-191): scale (scalar or per axis),
    rotate about z, then y, then x by ``rotate = [rx, ry, rz]`` degrees (about the origin),
    then translate."""
    v = np.asarray(triangles, dtype=np.float64).reshape(-1, 3)
    v = v * np.broadcast_to(np.asarray(1.0 if scale is None else scale, dtype=np.float64), (3,))
    rx, ry, rz = (0.0, 0.0, 0.0) if rotate is None else [float(a) for a in rotate]
    r = _rot(0, rx) @ _rot(1, ry) @ _rot(2, rz)
    v = v @ r.T + np.asarray((0, 0, 0) if translate is None else translate, dtype=np.float64)
    return v.reshape(-1, 3, 3).astype(np.float32)


def voxelise(triangles: np.ndarray, shape: Sequence[int], dx: float, dim: int,
             device: str = "cuda") -> Tuple[np.ndarray, np.ndarray]:
    """(solid bool, surface weight float32) of placed triangles on the (nx, ny, nz) grid of
    cell size ``dx`` (cell centres at (i + 1/2) dx; the 2D lattice is the plane z = 0)."""
    import torch
    nx, ny, nz = (int(s) for s in shape)
    lib = N.load()
    tri = torch.from_numpy(np.ascontiguousarray(triangles, dtype=np.float32).reshape(-1)).to(device)
    nbytes = ctypes.c_size_t()
    N.check(lib.lbm_stl_work_bytes(nx, ny, nz, dim, ctypes.byref(nbytes)))
    work = torch.empty(nbytes.value, dtype=torch.uint8, device=device)
    n = nx * ny * nz
    solid = torch.empty(n, dtype=torch.uint8, device=device)
    surf = torch.empty(n, dtype=torch.float32, device=device)
    s = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    N.check(lib.lbm_voxelise_stl(ctypes.c_void_p(tri.data_ptr()), len(triangles) if tri.numel() else 0,
                                 nx, ny, nz, dim, float(dx), ctypes.c_void_p(work.data_ptr()), nbytes.value,
                                 ctypes.c_void_p(solid.data_ptr()), ctypes.c_void_p(surf.data_ptr()), s))
    sol = solid.cpu().numpy().reshape((nx, ny, nz), order="F").astype(bool)
    return sol, surf.cpu().numpy().reshape((nx, ny, nz), order="F")


class StlReader:
    """The reference's reader (src/LBM/GEO/STL.py:118-146): domain size x, y, z and cell
    size dx, dimension 2 or 3."""

    def __init__(self, x, y, z, dx, dimension, logger: Optional[logging.Logger] = None):
        self.X, self.Y, self.Z, self.dx = x, y, z, dx
        self.nx, self.ny = int(x / dx), int(y / dx)
        self.nz = int(z / dx) if dimension == 3 else 1
        self.dimension = dimension
        self.logger = logger or logging.getLogger("lbm_b200.stl")

    def voxel_stl(self, stl_path, scale=1.0, translate=(0, 0, 0), rotate=(0, 0, 0)):
        """(voxel_array, surface_array), both float (nx, ny, nz): 1 inside the placed mesh,
        and the surface weight of solid cells."""
        self.logger.info(f"Stl {stl_path} loading...")
        tri = place(read_stl(os.fspath(stl_path)), scale, translate, rotate)
        solid, surf = voxelise(tri, (self.nx, self.ny, self.nz), self.dx, self.dimension)
        self.logger.info(f"Stl {stl_path} loaded.")
        return solid.astype(np.float64), surf.astype(np.float64)
