"""Seeded porous geometries (disk and sphere packings) for the lattice update.

The reference builds solids from STL voxelisation (src/LBM/GEO/STL.py:147-268);
the benchmark workloads instead use seeded random packings generated here, on
the host, so that the CUDA path and the oracle receive bit-identical masks.

Placement is random sequential addition with ``numpy.random.default_rng(seed)``:
non-overlapping while that can still reach the target porosity, then (for
porosities below the RSA jamming limit, about 0.45 for disks and 0.62 for
spheres) overlapping placement until the solid fraction reaches the target.
Particles keep ``margin`` cells away from non-periodic sides so that the
boundary planes and their inner neighbours stay fluid.
"""
from __future__ import annotations

import numpy as np


def _stamp(mask: np.ndarray, center, r: float, periodic) -> int:
    """Set cells whose centres lie within distance r of ``center`` (with wrap on periodic
    axes); return how many cells became solid."""
    dim = mask.ndim
    lo = [int(np.floor(center[a] - r)) for a in range(dim)]
    hi = [int(np.ceil(center[a] + r)) for a in range(dim)]
    axes = []
    for a in range(dim):
        idx = np.arange(lo[a], hi[a] + 1)
        d = idx - center[a]
        if periodic[a]:
            idx = idx % mask.shape[a]
        else:
            keep = (idx >= 0) & (idx < mask.shape[a])
            idx, d = idx[keep], d[keep]
        axes.append((idx, d))
    if dim == 2:
        (ix, dx), (iy, dy) = axes
        inside = dx[:, None] ** 2 + dy[None, :] ** 2 <= r * r
        sub = mask[np.ix_(ix, iy)]
        mask[np.ix_(ix, iy)] = sub | inside
        return int(np.count_nonzero(inside & ~sub))
    else:
        (ix, dx), (iy, dy), (iz, dz) = axes
        inside = dx[:, None, None] ** 2 + dy[None, :, None] ** 2 + dz[None, None, :] ** 2 <= r * r
        sub = mask[np.ix_(ix, iy, iz)]
        mask[np.ix_(ix, iy, iz)] = sub | inside
        return int(np.count_nonzero(inside & ~sub))


def _min_image(d: np.ndarray, n: int) -> np.ndarray:
    return d - n * np.round(d / n)


def packing(shape, rmin: float, rmax: float, porosity: float, seed: int, *,
            periodic=(True, True, True), margin: int = 0, allow_overlap: bool = True,
            max_attempts: int = 5000) -> np.ndarray:
    """Random disk (2D shape) or sphere (3D shape) packing.

    Returns a boolean array of ``shape`` (True = solid) whose fluid fraction is
    at most ``porosity`` (the first particle that crosses the target is kept).
    """
    shape = tuple(int(s) for s in shape)
    dim = len(shape)
    periodic = tuple(periodic[:dim])
    rng = np.random.default_rng(seed)
    mask = np.zeros(shape, dtype=bool)
    target_solid = 1.0 - porosity
    cap = 1024
    centers = np.zeros((cap, dim))
    radii = np.zeros(cap)
    count = 0
    total = mask.size
    solid = 0
    attempts = 0        # consecutive rejected non-overlapping placements
    stall = 0           # consecutive overlapping placements that added no cell
    overlap = False
    while solid / total < target_solid:
        if stall > 20000:
            raise ValueError(f"porosity {porosity} unreachable for shape {shape} with margin {margin}")
        r = rng.uniform(rmin, rmax)
        c = []
        for a in range(dim):
            if periodic[a]:
                c.append(rng.uniform(0, shape[a]))
            else:
                lo, hi = margin + r, shape[a] - 1 - margin - r
                if hi <= lo:
                    raise ValueError("domain too small for the particle radius and margin")
                c.append(rng.uniform(lo, hi))
        c = np.array(c)
        if not overlap and count:
            d = centers[:count] - c
            for a in range(dim):
                if periodic[a]:
                    d[:, a] = _min_image(d[:, a], shape[a])
            dist2 = (d * d).sum(1)
            if np.any(dist2 < (radii[:count] + r) ** 2):
                attempts += 1
                if attempts >= max_attempts:
                    if not allow_overlap:
                        raise ValueError("could not reach the porosity without overlap")
                    overlap = True
                continue
        attempts = 0
        if count == cap:
            cap *= 2
            centers = np.resize(centers, (cap, dim))
            radii = np.resize(radii, cap)
        centers[count] = c
        radii[count] = r
        count += 1
        added = _stamp(mask, c, r, periodic)
        stall = stall + 1 if added == 0 else 0
        solid += added
    return mask


# surface weight by the number of solid face neighbours (src/LBM/GEO/STL.py:216-259)
_SURFACE_2D = {4: 0.0, 3: 1.0, 2: 1.414, 1: 2.0, 0: 4.0}
_SURFACE_3D = {6: 0.0, 5: 1.0, 4: 1.414, 3: 2.0, 2: 3.0, 1: 4.0, 0: 6.0}


def surface_weights(solid: np.ndarray, dim: int) -> np.ndarray:
    """Surface weight of every solid cell of an (nx, ny, nz) indicator from its number of solid
    face neighbours (in-plane ones in 2D), cells beyond the grid counting as empty; 0 for
    empty cells.  The same table as the STL voxeliser's (stl_surface)."""
    m = np.asarray(solid) > 0
    pad = np.pad(m, 1)
    n = np.zeros(m.shape, dtype=np.int32)
    for ax in range(dim):
        for sh in (1, -1):
            n += np.roll(pad, sh, axis=ax)[1:-1, 1:-1, 1:-1]
    table = _SURFACE_2D if dim == 2 else _SURFACE_3D
    out = np.zeros(m.shape)
    for k, w in table.items():
        out[m & (n == k)] = w
    return out


def fortran_flat(a: np.ndarray) -> np.ndarray:
    """(nx,ny[,nz]) array -> flat device order c = x + nx*(y + ny*z)."""
    if a.ndim == 2:
        a = a[:, :, None]
    return np.ascontiguousarray(np.transpose(a, (2, 1, 0))).reshape(-1)


def from_flat(v: np.ndarray, shape) -> np.ndarray:
    """Inverse of :func:`fortran_flat` for an (nx,ny,nz) shape."""
    nx, ny, nz = shape
    return np.ascontiguousarray(v.reshape(nz, ny, nx).transpose(2, 1, 0))


def mask_bytes(solid: np.ndarray, reactive: np.ndarray | None = None) -> np.ndarray:
    """Device mask bytes (flat): bit0 solid, bit2 reactive."""
    m = fortran_flat(solid.astype(bool)).astype(np.uint8)
    if reactive is not None:
        m |= (fortran_flat(reactive.astype(bool)).astype(np.uint8) << 2)
    return m
