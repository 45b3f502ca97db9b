"""STL reading and placement (CPU); the GPU voxeliser is in test_gpu_stl.py."""
import numpy as np

from lbm_porouschem_b200.stl import place, read_stl, write_stl


def _tetra():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float32)
    return np.stack([v[[0, 2, 1]], v[[0, 1, 3]], v[[0, 3, 2]], v[[1, 2, 3]]])


def test_binary_round_trip(tmp_path):
    t = _tetra() * 0.37 + 1.5
    p = write_stl(str(tmp_path / "t.stl"), t)
    assert np.array_equal(read_stl(p), t.astype(np.float32))


def test_ascii_stl(tmp_path):
    t = _tetra()
    lines = ["solid tetra"]
    for tri in t:
        lines += ["  facet normal 0 0 0", "    outer loop"]
        lines += [f"      vertex {a:.6e} {b:.6e} {c:.6e}" for a, b, c in tri]
        lines += ["    endloop", "  endfacet"]
    lines.append("endsolid tetra")
    p = tmp_path / "a.stl"
    p.write_text("\n".join(lines) + "\n")
    assert np.allclose(read_stl(str(p)), t)


def test_place_order_scale_rotate_translate():
    """The reference scales, rotates about z, then y, then x (degrees), then translates
    (src/LBM/GEO/STL.py:185-191)."""
    t = _tetra()
    got = place(t, scale=[2.0, 1.0, 0.5], translate=[1, 2, 3], rotate=[90, 0, 90])
    # (x, y, z) -> scale -> rz90: (-y, x, z) -> rx90: (x, -z, y) -> translate
    v = t.reshape(-1, 3).astype(np.float64) * [2.0, 1.0, 0.5]
    v = np.stack([-v[:, 1], v[:, 0], v[:, 2]], 1)
    v = np.stack([v[:, 0], -v[:, 2], v[:, 1]], 1) + [1, 2, 3]
    assert np.allclose(got.reshape(-1, 3), v, atol=1e-6)
