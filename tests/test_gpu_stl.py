"""GPU voxelisation of closed triangle meshes (lbm_voxelise_stl) against exact inside tests.

Convex solids are inside exactly where a point lies behind every face plane; a hollow box
(an outer box and an inward-facing inner box) and two disjoint boxes check the ray parity
on non-convex and multi-part meshes.  Placements are random, so no cell centre lies on a
face: the masks must agree cell for cell.  Surface weights are checked against the
reference's neighbour-count table on the padded grid (src/LBM/GEO/STL.py:217-255)."""
import numpy as np
import pytest

from lbm_porouschem_b200.stl import StlReader, place, voxelise, write_stl

pytestmark = pytest.mark.gpu


def _box_tris(lo, hi, inward=False):
    """12 outward-facing triangles of an axis-aligned box (inward-facing if asked)."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    c = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]])
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (2, 3, 7, 6), (1, 2, 6, 5), (0, 4, 7, 3)]
    tris = []
    for a, b, cc, d in quads:
        tris += [(a, b, cc), (a, cc, d)]
    t = c[np.array(tris)]
    return t[:, ::-1] if inward else t


def _icosphere(level):
    p = (1 + 5 ** 0.5) / 2
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
         (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    tris = [np.array([v[a], v[b], v[c]], dtype=np.float64) for a, b, c in f]
    tris = [t / np.linalg.norm(t, axis=1, keepdims=True) for t in tris]
    for _ in range(level):
        nxt = []
        for a, b, c in tris:
            ab, bc, ca = [(m / np.linalg.norm(m)) for m in ((a + b) / 2, (b + c) / 2, (c + a) / 2)]
            nxt += [np.array(q) for q in ((a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca))]
        tris = nxt
    t = np.stack(tris)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    flip = np.einsum("fk,fk->f", n, t.mean(1)) < 0          # orient every face outward
    t[flip] = t[flip][:, ::-1]
    return t


def _inside_convex(tris, pts):
    """Behind every face plane (outward normals from the vertex order)."""
    t = np.asarray(tris, dtype=np.float64)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    d = np.einsum("fk,fk->f", n, t[:, 0])
    return np.all(pts @ n.T <= d, axis=1)


def _centres(shape, dx, dim, pad=0):
    nx, ny, nz = shape
    ax = [(np.arange(-pad, n + pad) + 0.5) * dx for n in (nx, ny)]
    az = (np.arange(-pad, nz + pad) + 0.5) * dx if dim == 3 else np.zeros(1)
    g = np.meshgrid(*ax, az, indexing="ij")
    return np.stack([a.ravel() for a in g], 1), g[0].shape


def _surface_ref(solid_pad, dim):
    """src/LBM/GEO/STL.py:217-255 on a grid padded by one cell (cropped)."""
    s = solid_pad.astype(int)
    if dim == 3:
        c = s[2:, 1:-1, 1:-1] + s[:-2, 1:-1, 1:-1] + s[1:-1, 2:, 1:-1] + s[1:-1, :-2, 1:-1] \
            + s[1:-1, 1:-1, 2:] + s[1:-1, 1:-1, :-2]
        tab = np.array([6.0, 4.0, 3.0, 2.0, 1.414, 1.0, 0.0])
        inner = s[1:-1, 1:-1, 1:-1]
    else:
        c = s[2:, 1:-1] + s[:-2, 1:-1] + s[1:-1, 2:] + s[1:-1, :-2]
        tab = np.array([4.0, 2.0, 1.414, 1.0, 0.0])
        inner = s[1:-1, 1:-1]
    return np.where(inner > 0, tab[c], 0.0).astype(np.float32)


def _rotated_box(rng):
    t = _box_tris((-0.45, -0.3, -0.2), (0.45, 0.3, 0.2))
    return place(t, scale=[20.0, 20.0, 20.0], rotate=rng.uniform(0, 90, 3), translate=rng.uniform(15, 17, 3))


@pytest.mark.parametrize("kind", ["rotated_box", "icosphere"])
def test_convex_solids_cell_for_cell(kind):
    rng = np.random.default_rng(7 if kind == "icosphere" else 8)
    shape, dx = (33, 30, 31), 1.0
    if kind == "icosphere":
        tri = place(_icosphere(3), scale=11.3, translate=rng.uniform(14, 16, 3))
    else:
        tri = _rotated_box(rng)
    solid, surf = voxelise(tri, shape, dx, 3)
    pts, _ = _centres(shape, dx, 3)
    ref = _inside_convex(tri, pts).reshape(shape)
    assert ref.sum() > 1000
    assert np.array_equal(solid, ref)
    ptsp, shp = _centres(shape, dx, 3, pad=1)
    refp = _inside_convex(tri, ptsp).reshape(shp)
    assert np.array_equal(surf, _surface_ref(refp, 3))


def test_hollow_and_disjoint_boxes_by_parity():
    rng = np.random.default_rng(9)
    shape, dx = (40, 28, 26), 0.5
    o = rng.uniform(0.0, 0.4, 3)
    outer = _box_tris((2.1, 2.2, 2.3) + o, (15.7, 11.6, 10.9) + o)
    hole = _box_tris((5.2, 4.9, 4.1) + o, (9.8, 8.3, 7.7) + o, inward=True)
    other = _box_tris((16.6, 3.3, 1.2) + o, (18.9, 12.1, 11.6) + o)
    tri = np.concatenate([outer, hole, other]).astype(np.float32)
    solid, _ = voxelise(tri, shape, dx, 3)
    pts, _ = _centres(shape, dx, 3)
    t = tri.astype(np.float64)
    ref = (_inside_convex(t[:12], pts) & ~_inside_convex(t[12:24][:, ::-1], pts)) | _inside_convex(t[24:], pts)
    assert np.array_equal(solid, ref.reshape(shape))
    assert solid[int(7.5 / dx), int(6.5 / dx), int(6.0 / dx)] == 0          # inside the hole


def test_2d_cross_section_and_reader(tmp_path):
    """2D: the plane z = 0 through a prism; the reference-shaped StlReader with a unit
    box file placed by scale / rotate / translate."""
    rng = np.random.default_rng(10)
    tri = _rotated_box(rng)
    tri[..., 2] -= tri[..., 2].mean()            # straddle z = 0
    shape = (34, 31, 1)
    solid, surf = voxelise(tri, shape, 1.0, 2)
    pts, _ = _centres(shape, 1.0, 2)
    assert np.array_equal(solid, _inside_convex(tri, pts).reshape(shape))
    ptsp, shp = _centres(shape, 1.0, 2, pad=1)
    refp = _inside_convex(tri, ptsp).reshape(shp[:2])
    assert np.array_equal(surf[..., 0], _surface_ref(refp, 2))

    p = write_stl(str(tmp_path / "box.stl"), _box_tris((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5)))
    r = StlReader(30.0, 20.0, 16.0, 0.5, 3)
    vox, sw = r.voxel_stl(p, scale=[8.1, 5.3, 4.2], translate=[14.9, 10.2, 7.9], rotate=[0, 0, 30])
    assert vox.shape == (60, 40, 32) and sw.shape == vox.shape
    t = place(_box_tris((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5)), [8.1, 5.3, 4.2], [14.9, 10.2, 7.9], [0, 0, 30])
    pts, _ = _centres((60, 40, 32), 0.5, 3)
    assert np.array_equal(vox > 0, _inside_convex(t, pts).reshape(60, 40, 32))
    assert np.all(sw[vox == 0] == 0) and sw.max() > 0


def test_yaml_geometry_stl(tmp_path):
    from lbm_porouschem_b200.app import _centres as centres
    from lbm_porouschem_b200.app import voxelise as app_voxelise
    p = write_stl(str(tmp_path / "g.stl"), _icosphere(2))
    g = centres(40, 40, 40, 1.0, 3)
    a = app_voxelise({"type": "stl", "path": p, "scale": [12.2, 12.2, 12.2], "translate": [20.1, 19.7, 20.3]}, g, 1.0)
    sph = app_voxelise({"type": "sphere", "center": [20.1, 19.7, 20.3], "radius": 12.2}, g, 1.0)
    assert abs(a.sum() - sph.sum()) / sph.sum() < 0.05      # the level-2 icosphere is ~2.4 % smaller
    assert np.all(a <= sph)                                   # inscribed in the sphere
