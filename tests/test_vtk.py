"""Headless VTK output (lbm_porouschem_b200.vtk) and the checkpoint configuration
round trip; no GPU needed."""
import json
import xml.etree.ElementTree as ET

import numpy as np

from lbm_porouschem_b200.config import FIXED_VALUE, LatticeConfig, SideBC
from lbm_porouschem_b200.vtk import PVDWriter, read_pvd, read_vts, write_vts


def test_vts_round_trip_point_order_and_types(tmp_path):
    rng = np.random.default_rng(0)
    shape = (5, 4, 3)
    rho = rng.random(shape)
    vel = rng.random(shape + (3,)).astype(np.float32)
    solid = rng.random(shape) < 0.3
    half = rng.random(shape).astype(np.float16)
    x, y, z = np.linspace(0, 1, 5), np.linspace(0, 0.6, 4), np.linspace(0, 0.4, 3)
    fn = write_vts(str(tmp_path / "a.vts"), {"rho": rho, "velocity": vel, "solid": solid, "h": half},
                   shape, coords=(x, y, z))
    d = read_vts(fn)
    assert tuple(d["_shape"]) == shape
    # VTK point order: x fastest (Fortran order of the (nx, ny, nz) arrays)
    assert d["rho"].dtype == np.float64 and np.array_equal(d["rho"], rho.ravel(order="F"))
    assert d["velocity"].shape == (60, 3) and np.array_equal(d["velocity"], vel.reshape(60, 3, order="F"))
    assert d["solid"].dtype == np.uint8 and np.array_equal(d["solid"], solid.ravel(order="F").astype(np.uint8))
    assert d["h"].dtype == np.float32 and np.array_equal(d["h"], half.ravel(order="F").astype(np.float32))
    pts = d["_points"]
    assert pts.shape == (60, 3)
    assert np.allclose(pts[:5, 0], x) and np.allclose(pts[::5, 1][:4], y) and np.allclose(pts[::20, 2], z)


def test_vts_header_is_vtk_xml(tmp_path):
    fn = write_vts(str(tmp_path / "b.vts"), {"rho": np.ones((3, 3, 1))}, (3, 3, 1))
    raw = open(fn, "rb").read()
    head = raw[:raw.index(b"<AppendedData")].decode() + "</VTKFile>"
    root = ET.fromstring(head.split("?>", 1)[1])
    assert root.tag == "VTKFile" and root.get("type") == "StructuredGrid"
    assert root.get("byte_order") == "LittleEndian" and root.get("header_type") == "UInt64"
    piece = root.find("StructuredGrid/Piece")
    assert piece.get("Extent") == "0 2 0 2 0 0"
    offs = [int(a.get("offset")) for a in root.iter("DataArray")]
    assert offs == sorted(offs) and offs[0] == 0
    assert raw.rstrip().endswith(b"</VTKFile>")


def test_pvd_series(tmp_path):
    w = PVDWriter(str(tmp_path), "case")
    for t in (0, 10, 20):
        w.add(t * 1e-4, f"case_{t}.vts")
    out = w.write()
    assert read_pvd(out) == [(0.0, "case_0.vts"), (1e-3, "case_10.vts"), (2e-3, "case_20.vts")]
    ds = ET.parse(out).getroot().find("Collection/DataSet")
    assert ds.get("name") == "case" and ds.get("part") == "0"


def test_config_dict_round_trip():
    cfg = LatticeConfig(dim=3, nx=8, ny=6, nz=4, collision="mrt", precision="fp16", thermal="conjugate",
                        pyro=True, force=(1e-5, 0.0, 0.0), mrt_rates={4: 1.2, 6: 1.1},
                        sides=[SideBC.inlet((0.01, 0.0, 0.0), FIXED_VALUE, 1.0), SideBC.outlet(1.0)]
                        + [SideBC() for _ in range(4)])
    back = LatticeConfig.from_dict(json.loads(json.dumps(cfg.to_dict())))
    assert back == cfg
    assert bytes(back.to_desc()) == bytes(cfg.to_desc())
