"""YAML case driver: geometry voxelisation and case building (CPU), a short run (GPU)."""
import logging

import numpy as np
import pytest
import yaml

from lbm_porouschem_b200.app import _centres, build_case, voxelise
from lbm_porouschem_b200.config import FIXED_VALUE, FLOW_RATE, ZERO_GRADIENT

CASE2D = """
basic:
  name: channel_pyro
  dimension: 2
  arch: gpu
  collision: mrt
module:
  temperature: true
  chemistry: true
spaceControl:
  geometry: [0.096, 0.032]
  DX: 1.0e-3
timeControl:
  startTime: 0
  endTime: 0.002
  DT: 1.0e-4
flowProperties:
  viscosity: {type: constant, value: 2.0e-5}
thermalPropertiesFluid:
  normalize: {Trange: [300, 800]}
  thermalDiff: {type: constant, value: 3.0e-5}
thermalPropertiesSolid:
  normalize: {Trange: [300, 800]}
  thermalDiff: {type: constant, value: 1.0e-5}
chemicalProperties:
  type: pyrolysis
  zone: [grain]
  A: 1.0e8
  Ea: 1.25e5
geometry:
  grain: {type: sphere, center: [0.03, 0.016, 0], radius: 0.006}
  post: {type: box, center: [0.06, 0.016, 0], size: [0.008, 0.01, 0.01]}
initialCondition:
  flow: {rho: 1, velocity: [0, 0, 0]}
  thermal: {T: 300}
  solid:
    s1: {zone: ALL, type: concrete}
boundaryCondition:
  left:
    flow: {type: inlet, velocity: [0.01, 0, 0]}
    thermalFluid: {type: fixedValue, value: 800}
  right:
    flow: {type: outlet, rho: 1}
    thermalFluid: {type: zeroGradient}
  down:
    flow: {type: wall}
  up:
    flow: {type: wall}
outputControl:
  log: {interval: 5.0e-4}
"""


def _log():
    lg = logging.getLogger("test_app")
    lg.setLevel(logging.WARNING)
    return lg


def test_voxelise_shapes_3d():
    dx = 1.0
    g = _centres(40, 40, 40, dx, 3)
    sph = voxelise({"type": "sphere", "center": [20, 20, 20], "radius": 10}, g, dx)
    assert abs(sph.sum() - 4 / 3 * np.pi * 1000) / (4 / 3 * np.pi * 1000) < 0.03
    cyl = voxelise({"type": "cylinder", "center": [20, 20, 20], "radius": 8, "height": 20, "axis": [1, 0, 0]}, g, dx)
    assert abs(cyl.sum() - np.pi * 64 * 20) / (np.pi * 64 * 20) < 0.05
    assert cyl[20, 20, 27] == 1 and cyl[20, 20, 29] == 0 and cyl[31, 20, 20] == 0
    cone = voxelise({"type": "cone", "center": [20, 20, 20], "radius": 10, "height": 20}, g, dx)
    assert abs(cone.sum() - np.pi * 100 * 20 / 3) / (np.pi * 100 * 20 / 3) < 0.08
    assert cone[20, 20, 11] == 1 and cone[28, 20, 11] == 1 and cone[28, 20, 28] == 0
    box = voxelise({"type": "box", "center": [20, 20, 20], "size": [10, 6, 4]}, g, dx)
    assert box.sum() == 10 * 6 * 4


def test_build_case_from_yaml():
    cfg = yaml.safe_load(CASE2D)
    lb = build_case(cfg, _log())
    assert (lb.nx, lb.ny, lb.nz) == (96, 32, 1)
    c = lb._config()
    assert c.collision == "mrt" and c.thermal == "conjugate" and c.pyro
    s = lb.solid.to_numpy()
    assert s.max() == 1.0 and abs(s.sum() - (np.pi * 36 + 8 * 10)) < 12
    # reactive cells: only the sphere zone
    assert lb._reactive.sum() == pytest.approx(np.pi * 36, abs=8)
    assert not lb._reactive[60, 16, 0] and s[60, 16, 0] == 1
    sd = c.sides
    assert sd[0].v_type == FIXED_VALUE and sd[0].v == (0.01, 0.0, 0.0) and sd[0].T == pytest.approx(1.0)
    assert sd[1].rho_type == FIXED_VALUE and sd[1].T_type == ZERO_GRADIENT
    assert sd[2].active and sd[3].active
    assert np.all(lb.TF.S.to_numpy() == 0.0)                         # 300 K normalised


def test_flowrate_inlet_from_yaml():
    """`inlet_flowrate` (src/LBM/app.py:358-364): the 2D left side becomes the steered
    flow-rate inlet with its target flux; rho is extrapolated."""
    cfg = yaml.safe_load(CASE2D)
    cfg["boundaryCondition"]["left"]["flow"] = {"type": "inlet_flowrate", "flowrate": 0.05}
    sd = build_case(cfg, _log())._config().sides
    assert sd[0].active and sd[0].v_type == FLOW_RATE and sd[0].v == (0.05, 0.0, 0.0)
    assert sd[0].rho_type == ZERO_GRADIENT and sd[0].T_type == FIXED_VALUE


def test_sutherland_viscosity_from_yaml():
    """flowProperties.viscosity {type: sutherland, As, Ts} (src/LBM/app.py:117-120)."""
    cfg = yaml.safe_load(CASE2D)
    cfg["flowProperties"]["viscosity"] = {"type": "sutherland", "As": 1.5e-6, "Ts": 110.4}
    c = build_case(cfg, _log())._config()
    assert c.viscosity == "sutherland" and c.suth_Ts == 110.4
    assert c.suth_A == pytest.approx(1.5e-6 * 1e-4 / 1e-6)


def test_unsupported_options_stop_the_run():
    cfg = yaml.safe_load(CASE2D)
    cfg["chemicalProperties"] = {"type": "cantera", "canteraFile": "mech.yaml"}
    with pytest.raises(NotImplementedError):
        build_case(cfg, _log())
    # porous zones with pyrolysis (the case's chemistry) are not on the CUDA path
    cfg = yaml.safe_load(CASE2D)
    cfg["module"]["porous_media"] = True
    cfg["initialCondition"]["solid"]["s1"] = {"zone": "ALL", "type": "poro", "porosity": 0.5}
    with pytest.raises(NotImplementedError):
        build_case(cfg, _log())._config()


def test_porous_zone_maps_to_the_lattice():
    """initialCondition.solid of type 'poro' (src/LBM/app.py:537-573): solid fraction
    1 - porosity and the drag model's coefficients over the zone."""
    cfg = yaml.safe_load(CASE2D)
    cfg["module"]["temperature"] = False
    cfg["module"]["chemistry"] = False
    cfg.pop("chemicalProperties")
    cfg["module"]["porous_media"] = True
    cfg["initialCondition"]["solid"]["s1"] = {"zone": "ALL", "type": "poro", "porosity": 0.6,
                                              "porousModel": "darcyForchheimer", "darcy": 2.0e6,
                                              "forchheimer": 300.0}
    lb = build_case(cfg, _log())
    c = lb._config()
    assert c.porous == "darcy_forchheimer" and c.thermal == "none"
    s = lb.solid._host
    zone = s > 0
    assert zone.any() and np.allclose(s[zone], 0.4)
    assert np.allclose(lb.coefDarcy._host[zone], 2.0e6 * lb.dx ** 2)
    assert np.allclose(lb.coefForchheimer._host[zone], 300.0 * lb.dx)
    assert np.all(lb.coefDarcy._host[~zone] == 0)


def test_porous_zone_with_heat_and_radiation():
    """A porous zone with the temperature field: two fields exchanging heat in it (exchange
    surface and coefficient, solid density) and, with module.radiation and radiationProperties
    mean_temp, its border radiating with the zone's emissivity (src/LBM/app.py:220-227, 537-566)."""
    from lbm_porouschem_b200.geometry import surface_weights
    cfg = yaml.safe_load(CASE2D)
    cfg["module"]["chemistry"] = False
    cfg.pop("chemicalProperties")
    cfg["module"]["porous_media"] = True
    cfg["module"]["radiation"] = True
    cfg["radiationProperties"] = {"type": "mean_temp", "Tambient": 310.0}
    geo = next(iter(cfg["geometry"]))
    cfg["initialCondition"]["solid"] = {"s1": {"zone": geo, "type": "poro", "porosity": 0.6, "rho": 3.0,
                                               "exchangeSurface": 2.0, "exchangeCoef": 5.0,
                                               "emisssivity": 0.8}}
    lb = build_case(cfg, _log())
    c = lb._config()
    assert c.porous == "ergun" and c.thermal == "two_field" and c.porous_heat
    assert c.radiation and c.T_ambient == 310.0 and c.dt_phys == lb.dt and c.dx_phys == lb.dx
    zone = lb.solid._host > 0
    assert zone.any() and np.allclose(lb.solid._host[zone], 0.4)
    assert np.allclose(lb.TS.exchangeSurface._host[zone], 2.0) and np.allclose(lb.TS.exchangeCoef._host[zone], 5.0)
    assert np.allclose(lb.rhos._host[zone], 3.0)
    border = surface_weights(zone * 1.0, 2)
    assert border.max() > 0 and np.array_equal(lb.TS.radiation_surface._host, border)
    assert np.allclose(lb.TS.emissivity._host, 0.8 * border)


def test_surface_weights_table():
    """Solid face neighbours -> weight (src/LBM/GEO/STL.py:216-259), cells beyond the grid empty."""
    from lbm_porouschem_b200.geometry import surface_weights
    m = np.zeros((5, 5, 1))
    m[1:4, 1:4] = 1
    w = surface_weights(m, 2)
    assert w[2, 2, 0] == 0.0 and w[1, 2, 0] == 1.0 and w[1, 1, 0] == 1.414 and w[0, 0, 0] == 0.0
    single = np.zeros((3, 3, 3))
    single[1, 1, 1] = 1
    assert surface_weights(single, 3)[1, 1, 1] == 6.0
    assert surface_weights(np.ones((1, 1, 1)), 3)[0, 0, 0] == 6.0


@pytest.mark.gpu
def test_cli_runs_case(tmp_path, monkeypatch):
    from lbm_porouschem_b200.cli import run
    cfg = yaml.safe_load(CASE2D)
    cfg["outputControl"]["vtk"] = {"interval": 1.0e-3, "path": str(tmp_path / "out")}
    p = tmp_path / "case.yaml"
    p.write_text(yaml.safe_dump(cfg))
    monkeypatch.chdir(tmp_path)
    assert run(["-c", str(p), "-v", "0"]) == 0
    from lbm_porouschem_b200.vtk import read_pvd, read_vts
    series = read_pvd(str(next((tmp_path / "out").glob("*.pvd"))))
    assert [f for _, f in series] == [f"{cfg['basic']['name']}_{t}.vts" for t in (0, 10, 20)]
    d = read_vts(str(tmp_path / "out" / series[-1][1]))
    assert np.isfinite(d["rho"]).all() and d["Tf"].max() > 300.0    # the hot inlet has warmed the fluid
    assert d["velocity"].shape == (d["rho"].size, 3)


@pytest.mark.gpu
def test_cli_runs_temperature_dependent_properties(tmp_path, monkeypatch):
    """thermalDiff derived with a polynomial conductivity and a NASA7 capacity (the form of
    the reference's examples/2D/pyrolysis/config.yaml), and the Prandtl model: the YAML run
    reaches the kernels' per-cell rates and the two give different temperatures."""
    from lbm_porouschem_b200.cli import run
    from lbm_porouschem_b200.vtk import read_pvd, read_vts
    out = {}
    for mode in ("derived", "prandtl"):
        cfg = yaml.safe_load(CASE2D)
        tf = cfg["thermalPropertiesFluid"]
        if mode == "derived":
            tf["thermalDiff"] = {"type": "derived"}
            tf["conductivity"] = {"type": "polynomial", "data": [0.01, 5e-5, 0, 0, 0]}
            tf["capacity"] = {"type": "NASA7", "Trange": [200, 1000, 3500],
                              "data": [[3.5, 1e-4, 0, 0, 0, 0, 0], [3.6, 5e-5, 0, 0, 0, 0, 0]]}
        else:
            tf["thermalDiff"] = {"type": "Prandtl", "Pr": 0.71}
        cfg["basic"]["name"] = mode
        cfg["outputControl"]["vtk"] = {"interval": 2.0e-3, "path": str(tmp_path / mode)}
        p = tmp_path / f"{mode}.yaml"
        p.write_text(yaml.safe_dump(cfg))
        monkeypatch.chdir(tmp_path)
        assert run(["-c", str(p), "-v", "0"]) == 0
        series = read_pvd(str(next((tmp_path / mode).glob("*.pvd"))))
        out[mode] = read_vts(str(tmp_path / mode / series[-1][1]))
        assert np.isfinite(out[mode]["Tf"]).all() and out[mode]["Tf"].max() > 300.0
    assert not np.allclose(out["derived"]["Tf"], out["prandtl"]["Tf"])


def test_derived_thermal_properties_from_yaml():
    """thermalDiff type derived with constant conductivity and capacity (src/LBM/app.py:132-175);
    a polynomial capacity becomes the fluid's per-cell property set, a mixture stops the run."""
    cfg = yaml.safe_load(CASE2D)
    cfg["thermalPropertiesFluid"]["thermalDiff"] = {"type": "derived"}
    cfg["thermalPropertiesFluid"]["conductivity"] = {"type": "constant", "value": 0.03}
    cfg["thermalPropertiesFluid"]["capacity"] = {"type": "constant", "value": 1000.0}
    lb = build_case(cfg, _log())
    assert lb.TF.derived and lb.TF.cond == 0.03 and lb.TF.cm == 1000.0
    cfg["thermalPropertiesFluid"]["capacity"] = {"type": "polynomial", "data": [1000, 0, 0, 0, 0]}
    lb = build_case(cfg, _log())
    assert lb.TF.cm is None and lb.TF.cm_poly == [1000, 0, 0, 0, 0]
    assert lb._config().tprop_fluid["cap_lo"] == [1000.0, 0.0, 0.0, 0.0, 0.0]
    cfg["thermalPropertiesFluid"]["capacity"] = {"type": "mixture"}
    with pytest.raises(NotImplementedError, match="capacity_mixture"):
        build_case(cfg, _log())
