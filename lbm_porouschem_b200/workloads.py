"""Seeded workloads of the lattice update (synthetic geometry, no datasets).

Each builder returns a ``Workload``: the lattice descriptor, the solid mask,
the reactive mask and the initial fields.  Sizes can be overridden so the same
physics runs at test sizes.

- ``flow2d``: D2Q9 BGK isothermal, all sides periodic, body force g_x = 1e-6,
  tau = 0.8, non-overlapping disks r ~ U[4, 8] until porosity <= 0.65 (256 x 128).
- ``pyro2d``: D2Q9 + D2Q5 conjugate heat + pyrolysis, pressure inlet rho = 1.0005
  at x = 0 (T = 1), outlet rho = 1 at x = nx-1, walls at y = 0, ny-1, flow tau 0.7,
  thermal tau 0.6 fluid / 0.9 solid, disks r ~ U[10, 20] at porosity 0.45 (512 x 256).
- ``pyro3d``: D3Q19 (MRT) + D3Q7 + pyrolysis, rho 1.001 -> 1.0 along x, periodic
  in y and z, spheres r ~ U[6, 12] at porosity 0.40 (256^3).
- ``sweep2d``: a parameter sweep of ``pyro2d``-type lattices, one seed each: size drawn
  from {128x64, 256x128, 512x256, 1024x512}, porosity ~ U[0.35, 0.65] (overlapping
  disks r ~ U[0.04, 0.08] ny), flow tau ~ U[0.6, 1.2], inlet T ~ U[0.5, 1.0] (96 lattices).
Pyrolysis: k = A exp(-E/(R T_K)), T_K = 300 + 500 T, A = 1e8 1/s, E = 1.25e5 J/mol,
dt = 1e-4 s per step, dH = 4e5 J/kg (endothermic), c_s = 1000 J/(kg K), char yield
0.25, rho_s = 1 (lattice), a cell turns fluid below reactive fraction 0.01.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .config import FIXED_VALUE, ZERO_GRADIENT, LatticeConfig, SideBC
from .geometry import packing


@dataclass
class Workload:
    name: str
    cfg: LatticeConfig
    solid: np.ndarray
    reactive: np.ndarray | None
    init: dict = field(default_factory=dict)

    @property
    def porosity(self) -> float:
        return 1.0 - float(self.solid.mean())


def flow2d(nx: int = 256, ny: int = 128, seed: int = 0, precision: str = "fp32",
           collision: str = "bgk") -> Workload:
    tau = 0.8
    cfg = LatticeConfig(dim=2, nx=nx, ny=ny, nz=1, collision=collision, precision=precision,
                        nu=(tau - 0.5) / 3.0, force=(1e-6, 0.0, 0.0))
    rmin, rmax = (4.0, 8.0) if min(nx, ny) >= 64 else (2.0, 4.0)
    solid = packing((nx, ny), rmin, rmax, 0.65, seed, periodic=(True, True), allow_overlap=False)
    return Workload(f"flow2d_{nx}x{ny}", cfg, solid, None, {"rho": 1.0, "u": (0.0, 0.0, 0.0)})


def _pyro_cfg(dim, nx, ny, nz, precision, collision, rho_in, walls: bool) -> LatticeConfig:
    tau = 0.7
    sides = [SideBC() for _ in range(6)]
    sides[0] = SideBC.pressure(rho_in, T_type=FIXED_VALUE, T=1.0)
    sides[1] = SideBC.outlet(1.0, T_type=ZERO_GRADIENT)
    if walls:
        sides[2] = SideBC.wall(T_type=ZERO_GRADIENT)
        sides[3] = SideBC.wall(T_type=ZERO_GRADIENT)
    # T0: FP16 storage shift of the temperature populations, mid-range of T in [0, 1]
    return LatticeConfig(dim=dim, nx=nx, ny=ny, nz=nz, collision=collision, precision=precision,
                         nu=(tau - 0.5) / 3.0, thermal="conjugate", tauT_fluid=0.6, tauT_solid=0.9,
                         pyro=True, sides=sides, T0=0.5)


def pyro2d(nx: int = 512, ny: int = 256, seed: int = 0, precision: str = "fp32",
           collision: str = "bgk", margin: int = 2) -> Workload:
    cfg = _pyro_cfg(2, nx, ny, 1, precision, collision, 1.0005, walls=True)
    rmin, rmax = (10.0, 20.0) if min(nx, ny) >= 128 else (2.0, 4.0)
    solid = packing((nx, ny), rmin, rmax, 0.45, seed, periodic=(False, False), margin=margin)
    return Workload(f"pyro2d_{nx}x{ny}", cfg, solid, solid.copy(),
                    {"rho": 1.0, "u": (0.0, 0.0, 0.0), "T": 0.0})


def pyro3d(n: int = 256, seed: int = 0, precision: str = "fp32", collision: str = "mrt",
           margin: int = 2, ny: int | None = None, nz: int | None = None) -> Workload:
    nx, ny, nz = n, ny or n, nz or n
    cfg = _pyro_cfg(3, nx, ny, nz, precision, collision, 1.001, walls=False)
    rmin, rmax = (6.0, 12.0) if min(nx, ny, nz) >= 64 else (1.5, 3.0)
    solid = packing((nx, ny, nz), rmin, rmax, 0.40, seed, periodic=(False, True, True), margin=margin,
                    max_attempts=2000)
    return Workload(f"pyro3d_{nx}x{ny}x{nz}", cfg, solid, solid.copy(),
                    {"rho": 1.0, "u": (0.0, 0.0, 0.0), "T": 0.0})


def bytes_per_lattice_update(cfg: LatticeConfig) -> int:
    """Bytes one lattice update moves by the dense A/B pull count: read and write every
    flow and temperature population, read the mask byte, read and write the per-cell
    reaction state (B = 2 Q s + 2 QT s + 1 + 2 s_state [pyrolysis]).  D3Q19 + D3Q7 +
    pyrolysis: 217 B in FP32, 113 B with FP16 storage, 433 B in FP64; D2Q9 alone: 73 B.
    This is the per-update figure the roofline fraction is quoted on."""
    s = {"fp32": 4, "fp16": 2, "fp64": 8}[cfg.precision]
    b = 2 * cfg.Q * s + 1
    if cfg.thermal != "none":
        b += 2 * cfg.QT * s
    if cfg.pyro:
        b += 2 * (8 if cfg.precision == "fp64" else 4)
    return b


def algorithmic_bytes_per_step(cfg: LatticeConfig, solid: np.ndarray) -> int:
    """Minimum DRAM bytes one step must move in this design, where solid cells carry no
    flow populations (a lower bound below the dense per-update count).

    Fluid cells read and write Q flow populations; every cell reads and writes QT
    temperature populations (conjugate mode); every cell reads its mask byte;
    reacting solid cells read and write their reactive fraction and write one
    gas-release value, which fluid neighbours read once.  Solid cells carry no
    flow populations."""
    s = {"fp32": 4, "fp16": 2, "fp64": 8}[cfg.precision]
    n = cfg.ncells
    nsolid = int(np.count_nonzero(solid))
    nfluid = n - nsolid
    b = nfluid * 2 * cfg.Q * s + n * 1
    if cfg.thermal != "none":
        b += n * 2 * cfg.QT * s
    if cfg.pyro:
        cb = 8 if cfg.precision == "fp64" else 4
        b += nsolid * 4 * cb   # alpha read + write, release write, release read by neighbours
    return b


SWEEP_SIZES = ((128, 64), (256, 128), (512, 256), (1024, 512))


def sweep2d(n: int = 96, seed0: int = 0, precision: str = "fp32", collision: str = "bgk",
            sizes=SWEEP_SIZES) -> list[Workload]:
    """Lattices of a parameter sweep (uneven sizes), each with cell lists so that they
    can be stepped as one batch."""
    out = []
    for i in range(n):
        rng = np.random.default_rng(10_000 + seed0 + i)
        nx, ny = sizes[int(rng.integers(len(sizes)))]
        phi = float(rng.uniform(0.35, 0.65))
        tau = float(rng.uniform(0.6, 1.2))
        t_in = float(rng.uniform(0.5, 1.0))
        cfg = _pyro_cfg(2, nx, ny, 1, precision, collision, 1.0005, walls=True)
        cfg.nu = (tau - 0.5) / 3.0
        cfg.sides[0].T = t_in
        cfg.bulk_form = "list"
        solid = packing((nx, ny), 0.04 * ny, 0.08 * ny, phi, seed0 + i, periodic=(False, False), margin=2)
        out.append(Workload(f"sweep2d_{i:03d}_{nx}x{ny}", cfg, solid, solid.copy(),
                            {"rho": 1.0, "u": (0.0, 0.0, 0.0), "T": 0.0}))
    return out
