"""YAML case driver with the reference's schema (src/LBM/app.py:16-680), on the CUDA path.

Sections read: ``basic`` (dimension, name; ``arch`` is ignored, the lattice always runs on the
GPU; ``collision`` / ``precision`` select BGK|MRT and fp32|fp16|fp64), ``spaceControl``
(geometry, DX), ``timeControl`` (DT, startTime, endTime), ``module``, ``flowProperties``
(constant viscosity, optional ``force``), ``thermalPropertiesFluid`` / ``thermalPropertiesSolid``
(normalize.Trange, thermalDiff constant|Prandtl|derived, constant or polynomial conductivity,
constant, polynomial or NASA7 capacity),
``chemicalProperties`` with ``type: pyrolysis``
(single-step pyrolysis of reactive solid zones), ``boundaryCondition`` (inlet / outlet / wall /
periodic flow sides, fixedValue / zeroGradient / periodic temperature), ``geometry`` (sphere,
cylinder, cone, box voxelised analytically at cell centres), ``initialCondition`` (flow, thermal,
concrete / substract / poro solids, a porous zone with its heat exchange and, with
``module.radiation`` and ``radiationProperties`` type mean_temp, its radiating border) and ``outputControl`` (log interval; ``vtk`` writes ``.vts`` files
and the ``.pvd`` series; ``snapshot`` writes checkpoints).  ``timeControl.restart`` names a
checkpoint to continue from instead of initialising (no reference counterpart).  Options outside
that set stop the run with NotImplementedError naming the option.
"""
from __future__ import annotations

import logging
import os
import time

import numpy as np

from .flag import BC, BC_FLOW, RADIATION_MODEL
from .geometry import surface_weights

_SIDES = ["left", "right", "down", "up", "forward", "back"]


# ----------------------------------------------------------------------------- geometry
def _centres(nx, ny, nz, dx, dim):
    """Cell-centre coordinates; the 2D lattice is the z = 0 plane."""
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    z = (np.arange(nz) + 0.5) * dx if dim == 3 else np.zeros(1)
    return np.meshgrid(x, y, z, indexing="ij")


def _axis_frame(axis):
    a = np.asarray(axis, dtype=np.float64)
    n = np.linalg.norm(a)
    if n == 0:
        raise ValueError("geometry axis must be non-zero")
    return a / n


def voxelise(shape: dict, grid, dx: float) -> np.ndarray:
    """Solid indicator (float 0/1) of one primitive of the reference's ``geometry`` section.

    The reference builds unit STL primitives (src/LBM/GEO/STL.py: sphere radius 0.5, cylinder
    radius 0.5 height 1, box edge 1, cone base radius 0.5 height 1, all centred at the origin),
    scales, rotates (z -> ``axis``) and translates them, then voxelises; here the same solids are
    tested analytically at cell centres."""
    X, Y, Z = grid
    kind = shape["type"]
    c = np.asarray(shape.get("center", [0.0, 0.0, 0.0]), dtype=np.float64)
    c = np.concatenate([c, np.zeros(3 - len(c))])
    d = np.stack([X - c[0], Y - c[1], Z - c[2]])
    if kind == "sphere":
        r = np.broadcast_to(np.asarray(shape.get("radius", 0.5), dtype=np.float64), (3,))
        inside = ((d / r[:, None, None, None]) ** 2).sum(0) <= 1.0
    elif kind in ("cylinder", "cone"):
        a = _axis_frame(shape.get("axis", [0.0, 0.0, 1.0]))
        h = float(shape.get("height", 1.0))
        r = float(shape.get("radius", 0.5))
        s = np.tensordot(a, d, axes=1)                        # coordinate along the axis
        rad2 = (d ** 2).sum(0) - s ** 2
        in_h = np.abs(s) <= 0.5 * h
        if kind == "cylinder":
            inside = in_h & (rad2 <= r * r)
        else:                                                 # base at -h/2, apex at +h/2
            rr = r * (0.5 - s / h)
            inside = in_h & (rad2 <= np.maximum(rr, 0.0) ** 2)
    elif kind == "box":
        size = np.broadcast_to(np.asarray(shape.get("size", [1.0, 1.0, 1.0]), dtype=np.float64), (3,))
        inside = np.ones(X.shape, dtype=bool)
        for k, ext in enumerate(size):
            if k == 2 and X.shape[2] == 1:
                continue                                      # 2D: the box spans the plane
            inside &= np.abs(d[k]) <= 0.5 * ext
    elif kind == "stl":
        # src/LBM/app.py:466-473: path, scale, translate, rotate; voxelised on the GPU
        from .stl import place, read_stl, voxelise as stl_voxelise
        tri = place(read_stl(shape["path"]), shape.get("scale", [1, 1, 1]), shape.get("translate"),
                    shape.get("rotate"))
        dim = 3 if X.shape[2] > 1 else 2                       # the 2D grid is one z = 0 plane
        inside, _ = stl_voxelise(tri, X.shape, dx, dim)
    else:
        raise ValueError(f"geometry type {kind!r} not valid")
    return inside.astype(np.float64)


def _zone_names(zone, geo: dict) -> list:
    if zone in ("ALL", "all"):
        return list(geo)
    if isinstance(zone, (list, tuple)):
        return list(zone)
    return [zone]


def _zone_mask(zone, geo: dict, shape) -> np.ndarray:
    s = np.zeros(shape)
    if zone in ("ALL", "all"):
        for m in geo.values():
            s += m
    elif isinstance(zone, (list, tuple)):
        for z in zone:
            s += geo[z]
    elif isinstance(zone, str):
        s += geo[zone]
    return (s > 0).astype(np.float64)


def _scalar(v, key="value"):
    return v.get(key) if isinstance(v, dict) else v


# ----------------------------------------------------------------------------- application
def build_case(config: dict, logger: logging.Logger):
    """Create and configure the solver from a parsed YAML mapping (no stepping)."""
    basic = config.get("basic") or {}
    dim = basic.get("dimension", 2)
    if dim == 2:
        from .solver import LBM2DSolver as lbm
    elif dim == 3:
        from .solver import LBM3DSolver as lbm
    else:
        raise ValueError("basic.dimension must be 2 or 3")
    name = basic.get("name") or "default_LBM"
    space = config["spaceControl"]
    geom = list(space["geometry"])
    dx = float(space["DX"])
    x, y = float(geom[0]), float(geom[1])
    z = float(geom[2]) if dim == 3 else 1.0
    dt = float(config["timeControl"]["DT"])
    module = config.get("module") or {}
    is_thermal = bool(module.get("temperature", False))
    is_poro = bool(module.get("porous_media", False))
    is_chem = bool(module.get("chemistry", False))
    is_rad = bool(module.get("radiation", False))

    lb = lbm(x, y, z, dx, dt, name, is_thermal, is_chem, is_poro, is_rad)
    lb.set_collision(str(basic.get("collision", "bgk")))
    lb.set_precision(str(basic.get("precision", "fp32")))

    flow = config.get("flowProperties") or {}
    visc = flow.get("viscosity")
    if visc is not None:
        vtype = visc.get("type", "constant") if isinstance(visc, dict) else "constant"
        if vtype == "sutherland":
            lb.set_viscosity_sutherland(float(visc["As"]), float(visc["Ts"]))    # src/LBM/app.py:117-120
        elif vtype != "constant":
            raise NotImplementedError(f"flowProperties.viscosity.type {vtype!r} is not on the CUDA path")
        else:
            lb.set_viscosity(float(_scalar(visc)))
    if flow.get("force") is not None:
        lb.set_body_force([float(v) for v in flow["force"]])

    for key, side in (("thermalPropertiesFluid", "fluid"), ("thermalPropertiesSolid", "solid")):
        tp = config.get(key)
        if not (is_thermal and tp):
            continue
        setter = lambda name: getattr(lb, f"set_{side}_{name}")     # noqa: E731
        norm = tp.get("normalize")
        if norm:
            setter("Trange")(norm.get("Trange", [0, 1]))
        td = tp.get("thermalDiff")
        if td:
            ttype = td.get("type", "constant")
            if ttype == "constant":
                setter("thermal_diff")(float(td["value"]))
            elif ttype == "Prandtl" and side == "fluid":
                lb.set_fluid_Prandtl(float(td["Pr"]))
            elif ttype == "derived":
                setter("thermal_diff_derived")()
            else:
                raise NotImplementedError(f"{key}.thermalDiff.type {ttype!r} is not on the CUDA path")
        # src/LBM/app.py:143-175: constant, polynomial and NASA7 values; mixture raises in the setters
        for prop in ("conductivity", "capacity"):
            pd = tp.get(prop)
            if not pd:
                continue
            ptype = pd.get("type", "constant")
            if ptype == "constant":
                setter(prop)(float(pd["value"]))
            elif ptype == "polynomial":
                setter(prop + "_poly")(pd.get("data"))
            elif ptype == "NASA7" and prop == "capacity":
                setter("capacity_NASA7")(pd.get("Trange"), pd.get("data"))
            elif ptype == "mixture":
                setter(prop + "_mixture")()
            else:
                raise ValueError(f"{key}.{prop}.type {ptype!r} not valid")

    # src/LBM/app.py:220-227: surface radiation to a uniform ambient temperature
    rad = config.get("radiationProperties")
    if is_rad and rad is not None:
        if rad.get("type") == "mean_temp":
            lb.set_radiation(RADIATION_MODEL.SURFACE_UNIFORM, float(rad.get("Tambient", 300)))
        else:
            raise ValueError(f"radiationProperties.type {rad.get('type')!r} not valid")

    chem = config.get("chemicalProperties")
    pyro_zone = None
    if is_chem and chem:
        ctype = chem.get("type")
        if ctype != "pyrolysis":
            raise NotImplementedError(f"chemicalProperties.type {ctype!r} is not on the CUDA path "
                                      "(single-step 'pyrolysis' only)")
        pyro_zone = chem.get("zone", "ALL")
        lb.set_pyrolysis(A=float(chem.get("A", 1e8)), Ea=float(chem.get("Ea", 1.25e5)), b=float(chem.get("b", 0.0)),
                         dH=float(chem.get("dH", 4e5)), capacity=float(chem.get("capacity", 1000.0)),
                         rho_solid=float(chem.get("rho_solid", 1.0)), char_yield=float(chem.get("char_yield", 0.25)),
                         alpha_flip=float(chem.get("alpha_flip", 0.01)))

    nb = 6 if dim == 3 else 4
    bcs = config.get("boundaryCondition") or {}
    for i in range(nb):
        bc = bcs.get(_SIDES[i]) or {}
        bf = bc.get("flow") or {}
        t = bf.get("type", "periodic")
        if t == "inlet":
            lb.set_BC(i, BC_FLOW.inlet)
            lb.set_v_BC_value(i, [float(v) for v in bf["velocity"]])
            if bf.get("rho"):
                lb.set_rho_BC_value(i, float(bf["rho"]))
        elif t == "outlet":
            lb.set_BC(i, BC_FLOW.outlet)
            lb.set_rho_BC_value(i, float(bf["rho"]))
        elif t == "wall":
            lb.set_BC(i, BC_FLOW.wall)
        elif t == "symmetric":
            lb.set_BC(i, BC_FLOW.symmetric)
        elif t == "inlet_flowrate":
            # src/LBM/app.py:358-364
            lb.set_BC(i, BC_FLOW.inlet_flow)
            lb.set_flow_BC_value(i, float(bf["flowrate"]))
            if bf.get("rho", 1):
                lb.set_rho_BC_value(i, float(bf.get("rho", 1)))
        elif t not in ("periodic", None):
            raise ValueError(f"boundaryCondition.{_SIDES[i]}.flow.type {t!r} not valid")
        if is_thermal:
            for key, set_bc, set_val in (("thermalFluid", lb.set_TF_BC, lb.set_TF_BC_value),
                                         ("thermalSolid", lb.set_TS_BC, lb.set_TS_BC_value)):
                bt = bc.get(key)
                if not bt or not bt.get("type") or bt.get("type") == "none":
                    continue
                bt_type = bt["type"]
                if bt_type == "fixedValue":
                    set_bc(i, BC.fixedValue)
                    set_val(i, float(bt.get("value", 0.0)))
                elif bt_type == "zeroGradient":
                    set_bc(i, BC.zeroGradient)
                elif bt_type == "periodic":
                    set_bc(i, BC.periodic)
                else:
                    raise ValueError(f"boundaryCondition.{_SIDES[i]}.{key}.type {bt_type!r} not valid")

    grid = _centres(lb.nx, lb.ny, lb.nz, dx, dim)
    geo = {}
    for gname, g in (config.get("geometry") or {}).items():
        geo[gname] = voxelise(g, grid, dx)
        logger.info(f"geometry {gname}: {int(geo[gname].sum())} cells")

    ic = config.get("initialCondition") or {}
    fic = ic.get("flow")
    if fic:
        vel = list(fic.get("velocity", [0, 0, 0])) + [0.0] * 3
        lb.init_field(lb.rho, float(fic.get("rho", 1.0)))
        lb.init_field3(lb.v, float(vel[0]), float(vel[1]), float(vel[2]))
    if is_thermal and ic.get("thermal"):
        tic = ic["thermal"]
        T = tic.get("TF", tic.get("T", 0.0))
        lb.init_field(lb.TF.S, lb.TF.get_normalized_value(float(T)))
        lb.init_field(lb.TS.S, lb.TS.get_normalized_value(float(tic.get("TS", tic.get("T", 0.0)))))
    for sdef in (ic.get("solid") or {}).values():
        stype = sdef.get("type")
        zone = sdef.get("zone", "ALL")
        s = _zone_mask(zone, geo, lb._shape)
        if stype == "concrete":
            lb.add_solid(s)
            lb.add_rho_solid(float(sdef.get("rho", 1.0)) * s)
        elif stype == "substract":
            lb.add_solid(-s)
        elif stype == "poro" and is_poro:
            # src/LBM/app.py:537-573: solid fraction 1 - porosity over the zone, its density,
            # heat exchange surface and coefficient, radiating border and emissivity (the
            # reference reads the key "emisssivity"), the drag model's coefficients over it
            # ("ergun" keeps the default SPHERICAL model)
            zs = (s > 0) * 1.0
            lb.add_solid((1.0 - float(sdef["porosity"])) * zs)
            lb.add_rho_solid(float(sdef.get("rho", 1.0)) * zs)
            lb.set_heat_exchange_surface(float(sdef.get("exchangeSurface", 1.0)) * zs)
            lb.set_heat_exchange_coef(float(sdef.get("exchangeCoef", 1.0)) * zs)
            if is_rad:
                border = sum((surface_weights(geo[z], dim) for z in _zone_names(zone, geo)), np.zeros(lb._shape))
                emis = float(sdef.get("emisssivity", sdef.get("emissivity", 1.0)))
                lb.init_field(lb.TS.radiation_surface, border)
                lb.init_field(lb.TS.emissivity, border * emis)
            model = sdef.get("porousModel")
            if model == "darcy":
                lb.set_poro_Darcy(zs, float(sdef["darcy"]))
            elif model == "darcyForchheimer":
                lb.set_poro_Darcy_Forchheimer(zs, float(sdef["darcy"]), float(sdef["forchheimer"]))
            elif model not in (None, "ergun"):
                raise ValueError(f"initialCondition.solid porousModel {model!r} not valid")
        elif stype == "poro":
            # the reference skips a porous zone when module.porous_media is off (app.py:537)
            logger.warning("initialCondition.solid of type 'poro' ignored: module.porous_media is off")
        else:
            raise ValueError(f"initialCondition.solid type {stype!r} not valid")
    lb.solid.from_numpy(np.clip(lb.solid._host, 0.0, 1.0))
    if pyro_zone is not None:
        lb._reactive = _zone_mask(pyro_zone, geo, lb._shape) > 0 if geo else None
    return lb


def application(config: dict, logger: logging.Logger, max_steps: int | None = None):
    """Run a case: configure, initialise, then step to ``timeControl.endTime`` logging every
    ``outputControl.log.interval`` (src/LBM/app.py:600-680)."""
    start = time.time()
    lb = build_case(config, logger)
    tc = config["timeControl"]
    lb.tLattice = int(float(tc.get("startTime", 0)) / lb.dt)
    end_lattice = float(tc.get("endTime", 0)) / lb.dt
    oc = config.get("outputControl") or {}
    print_every = max(1, int(round(float((oc.get("log") or {}).get("interval", lb.dt)) / lb.dt)))
    vtk = oc.get("vtk") or {}
    export_every = int(round(float(vtk.get("interval", 100)) / lb.dt)) if vtk else 0
    export_path = vtk.get("path") or "output"
    if vtk:
        if vtk.get("clear"):
            import shutil
            shutil.rmtree(export_path, ignore_errors=True)
        os.makedirs(export_path, exist_ok=True)
        lb.set_vtk_path(export_path)
    # src/LBM/app.py:639-643, 670-671 (the reference's export_snapshot is empty)
    snap = oc.get("snapshot") or {}
    snapshot_every = int(round(float(snap.get("interval", 100)) / lb.dt)) if snap else 0
    if snap.get("path"):
        lb.snapshotPath = snap["path"]

    restart = tc.get("restart")
    if restart:
        logger.info(f"Continuing from {restart}")
        lb.load_snapshot(restart)
    else:
        logger.info("Simulation initializing...")
        lb.init_simulation()
    logger.info(lb.description())
    cells = lb.nx * lb.ny * lb.nz
    pre = time.time()
    steps = 0
    while lb.tLattice <= end_lattice and (max_steps is None or steps < max_steps):
        if lb.tLattice % print_every == 0:
            dtw = time.time() - pre
            pre = time.time()
            mlups = cells * print_every / dtw / 1e6 if dtw > 0 and steps else 0.0
            logger.info(f"Execution time:{dtw:.2f} s , Collapsed time:{time.time() - start:.2f} s, MLUPS = {mlups:.2f}")
            logger.info(lb.log_info())
        if export_every and lb.tLattice % export_every == 0:
            lb.export_VTK_pyvista()
        if snapshot_every and lb.tLattice % snapshot_every == 0:
            lb.export_snapshot(config)
        lb.step()
        steps += 1
    logger.info("LBM finished.")
    return lb
