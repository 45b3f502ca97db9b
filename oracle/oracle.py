"""ctypes wrapper of the C oracle (``lbm_oracle.c``), the CPU checker of the CUDA path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``.  Never part of the product path.

PARITY PINNED: ``tests/test_oracle_vs_reference.py`` checks the FP64 build against
golden outputs of the reference's own solver modules (``tests/golden/ref_*.npz``, made by
``tests/golden/make_reference_fixtures.py``); behaviour the reference lacks is pinned by
analytic known answers (``tests/test_oracle_physics.py``).

``build_oracle()`` compiles ``lbm_oracle.c`` twice (FP32 and FP64) with
``gcc -O3 -fopenmp`` into ``oracle/_build/``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "lbm_oracle.c"
BUILD = HERE / "_build"


class orc_side(C.Structure):
    _fields_ = [("active", C.c_int), ("v_type", C.c_int), ("rho_type", C.c_int), ("T_type", C.c_int),
                ("v", C.c_double * 3), ("rho", C.c_double), ("T", C.c_double)]


class orc_cfg(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("collision", C.c_int), ("eos", C.c_int), ("nu", C.c_double), ("force", C.c_double * 3),
        ("half_force_velocity", C.c_int), ("thermal", C.c_int), ("tauT_fluid", C.c_double),
        ("tauT_solid", C.c_double), ("pyro", C.c_int), ("pyro_A", C.c_double), ("pyro_b", C.c_double),
        ("pyro_Ea", C.c_double), ("pyro_Tmin", C.c_double), ("T_ref", C.c_double), ("T_scale", C.c_double),
        ("dt_phys", C.c_double), ("heat_norm", C.c_double), ("gas_coef", C.c_double),
        ("alpha_flip", C.c_double), ("mrt_s", C.c_double * 19), ("side", orc_side * 6),
        ("visc_model", C.c_int), ("suth_A", C.c_double), ("suth_Ts", C.c_double),
        ("ref_quirk_frozen_solid_T", C.c_int), ("poro_model", C.c_int),
        ("Ts_ref", C.c_double), ("Ts_scale", C.c_double), ("cap_fluid", C.c_double), ("cap_solid", C.c_double),
        ("dx_phys", C.c_double), ("radiation", C.c_int), ("T_ambient", C.c_double),
        ("ref_quirk_nebb", C.c_int),
        ("tprop", C.c_int), ("tp_cond", (C.c_double * 5) * 2), ("tp_cap_lo", (C.c_double * 5) * 2),
        ("tp_cap_hi", (C.c_double * 5) * 2), ("tp_cap_Tmid", C.c_double * 2), ("tp_cap_mul", C.c_double * 2),
        ("tp_rhos", C.c_double), ("tp_dt", C.c_double), ("tp_dx2", C.c_double), ("tp_prandtl", C.c_double),
    ]


def lib_path(real: str) -> Path:
    return BUILD / f"liblbm_oracle_{real}.so"


def build_oracle(force: bool = False) -> None:
    """Compile the FP32 and FP64 oracle libraries (gcc, OpenMP)."""
    BUILD.mkdir(exist_ok=True)
    for real, ctype in (("f32", "float"), ("f64", "double")):
        out = lib_path(real)
        if not force and out.exists() and out.stat().st_mtime >= SRC.stat().st_mtime:
            continue
        cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", f"-DREAL={ctype}", "-o", str(out), str(SRC), "-lm"]
        subprocess.run(cmd, check=True)


_LIBS: dict = {}


def _load(real: str) -> C.CDLL:
    if real in _LIBS:
        return _LIBS[real]
    p = lib_path(real)
    if not p.exists():
        build_oracle()
    lib = C.CDLL(str(p))
    lib.orc_create.argtypes = [C.POINTER(orc_cfg)]
    lib.orc_create.restype = C.c_void_p
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_init.argtypes = [C.c_void_p] + [C.c_void_p] * 5
    lib.orc_set_porous.argtypes = [C.c_void_p] * 4
    lib.orc_set_porous_heat.argtypes = [C.c_void_p] * 6
    lib.orc_init_solid_T.argtypes = [C.c_void_p] * 2
    lib.orc_get_solid_T.argtypes = [C.c_void_p] * 3
    lib.orc_array.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    lib.orc_array.restype = C.c_void_p
    lib.orc_step.argtypes = [C.c_void_p, C.c_int]
    lib.orc_get.argtypes = [C.c_void_p] + [C.c_void_p] * 5
    lib.orc_get_dist.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.orc_diag.argtypes = [C.c_void_p, C.c_void_p]
    lib.orc_M.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.orc_M.restype = C.c_double
    lib.orc_num_threads.restype = C.c_int
    lib.orc_set_threads.argtypes = [C.c_int]
    _LIBS[real] = lib
    return lib


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class Oracle:
    """CPU restatement of the reference step for one ``LatticeConfig``.

    ``real`` is "f32" or "f64" (the arithmetic precision of the restatement).
    Arrays in and out use the reference's (nx, ny, nz) layout."""

    def __init__(self, cfg, real: str = "f64", threads: int | None = None,
                 ref_quirk_frozen_solid_T: bool = False, ref_quirk_nebb: bool = False):
        """``ref_quirk_frozen_solid_T`` (two-field temperature only) reproduces the reference's
        pure-solid cells, whose temperature ``macro`` never refreshes
        (src/LBM/LBM2D/_evolution.py:119); the default diffuses heat through the solid."""
        self.cfg = cfg
        self.lib = _load(real)
        if threads:
            self.lib.orc_set_threads(int(threads))
        c = orc_cfg()
        c.dim, c.nx, c.ny, c.nz = cfg.dim, cfg.nx, cfg.ny, (1 if cfg.dim == 2 else cfg.nz)
        c.collision = 0 if cfg.collision == "bgk" else 1
        c.eos = 0 if cfg.eos == "ideal_gas" else 1
        c.nu = cfg.nu
        for i in range(3):
            c.force[i] = float(cfg.force[i])
        c.half_force_velocity = int(cfg.half_force_velocity)
        c.thermal = {"none": 0, "conjugate": 1, "two_field": 2}[cfg.thermal]
        c.tauT_fluid, c.tauT_solid = cfg.tauT_fluid, cfg.tauT_solid
        c.pyro = int(cfg.pyro)
        c.pyro_A, c.pyro_b, c.pyro_Ea, c.pyro_Tmin = cfg.pyro_A, cfg.pyro_b, cfg.pyro_Ea, cfg.pyro_Tmin
        c.T_ref, c.T_scale, c.dt_phys = cfg.T_ref, cfg.T_scale, cfg.dt_phys
        c.heat_norm, c.gas_coef, c.alpha_flip = cfg.heat_norm, cfg.gas_coef, cfg.alpha_flip
        c.visc_model = 1 if cfg.viscosity == "sutherland" else 0
        c.suth_A, c.suth_Ts = cfg.suth_A, cfg.suth_Ts
        c.ref_quirk_frozen_solid_T = int(ref_quirk_frozen_solid_T)
        c.ref_quirk_nebb = int(ref_quirk_nebb)
        c.poro_model = {"none": 0, "ergun": 1, "darcy": 2, "darcy_forchheimer": 3}[getattr(cfg, "porous", "none")]
        c.Ts_ref = cfg.T_ref if cfg.Ts_ref is None else cfg.Ts_ref
        c.Ts_scale = cfg.T_scale if cfg.Ts_scale is None else cfg.Ts_scale
        c.cap_fluid, c.cap_solid, c.dx_phys = cfg.cap_fluid, cfg.cap_solid, cfg.dx_phys
        c.radiation, c.T_ambient = int(cfg.radiation), cfg.T_ambient
        for ph, tp in enumerate((getattr(cfg, "tprop_fluid", None), getattr(cfg, "tprop_solid", None))):
            if tp is None:
                continue
            c.tprop |= 1 << ph
            for i in range(5):
                c.tp_cond[ph][i] = float(tp["cond"][i])
                c.tp_cap_lo[ph][i] = float(tp["cap_lo"][i])
                c.tp_cap_hi[ph][i] = float(tp["cap_hi"][i])
            c.tp_cap_Tmid[ph], c.tp_cap_mul[ph] = float(tp["cap_Tmid"]), float(tp["cap_mul"])
        c.tp_rhos = getattr(cfg, "tp_rhos", 1.0)
        c.tp_dt, c.tp_dx2 = getattr(cfg, "tp_dt", 1.0), getattr(cfg, "tp_dx2", 1.0)
        if getattr(cfg, "tp_prandtl", 0.0) > 0:
            c.tprop |= 4
            c.tp_prandtl = cfg.tp_prandtl
        for r, v in enumerate(cfg.mrt_s()):
            c.mrt_s[r] = v
        for i, s in enumerate(cfg.sides):
            c.side[i].active = s.code()
            c.side[i].v_type, c.side[i].rho_type, c.side[i].T_type = int(s.v_type), int(s.rho_type), int(s.T_type)
            for k in range(3):
                c.side[i].v[k] = float(s.v[k])
            c.side[i].rho, c.side[i].T = float(s.rho), float(s.T)
        self._c = c
        self._h = self.lib.orc_create(C.byref(c))
        self.n = cfg.ncells

    def _flat(self, v, ncomp=1) -> np.ndarray:
        from lbm_porouschem_b200.geometry import fortran_flat
        n = self.n
        if np.isscalar(v):
            return np.full(ncomp * n, float(v), dtype=np.float64)
        a = np.asarray(v, dtype=np.float64)
        if ncomp == 1:
            return fortran_flat(a.reshape(self.cfg.shape)).astype(np.float64)
        return np.concatenate([fortran_flat(a[i].reshape(self.cfg.shape)) for i in range(ncomp)]).astype(np.float64)

    def set_porous(self, fraction, darcy=None, forchheimer=None) -> None:
        """Porous cells before ``init``: solid fraction per cell (0 fluid, 1 solid, between
        porous) and the Darcy / Forchheimer coefficients, (nx, ny, nz) arrays."""
        self._porous = tuple(self._flat(a) if a is not None else None for a in (fraction, darcy, forchheimer))
        self.lib.orc_set_porous(self._h, *(_ptr(a) for a in self._porous))

    def set_porous_heat(self, h=None, a=None, rho_solid=None, emissivity=None, radiation_surface=None) -> None:
        """Two fields with porous cells, before ``init``: the exchange coefficient and surface,
        the solid density and the radiation inputs per cell, (nx, ny, nz) arrays or None."""
        self._heat = tuple(self._flat(x) if x is not None else None
                           for x in (h, a, rho_solid, emissivity, radiation_surface))
        self.lib.orc_set_porous_heat(self._h, *(_ptr(x) for x in self._heat))

    def init(self, solid, reactive=None, rho=1.0, u=(0.0, 0.0, 0.0), T=0.0, alpha=None,
             round_inputs_to_f32: bool = True, Ts=None) -> None:
        """Same inputs as ``Lattice.set_geometry`` + ``Lattice.init``.  Inputs are rounded to
        float32 first (the CUDA path takes float32 initial fields).  ``Ts``: the solid
        temperature of porous and pure-solid cells when it differs from ``T`` (two fields)."""
        from lbm_porouschem_b200.geometry import mask_bytes
        m = mask_bytes(np.asarray(solid), reactive)
        r = self._flat(rho)
        if isinstance(u, (tuple, list)) and all(np.isscalar(x) for x in u):
            uu = np.concatenate([np.full(self.n, float(x)) for x in u])
        else:
            uu = self._flat(u, 3)
        t = self._flat(T)
        a = self._flat(alpha) if alpha is not None else np.where(m & 4, 1.0, 0.0).astype(np.float64)
        if round_inputs_to_f32:
            r, uu, t, a = (x.astype(np.float32).astype(np.float64) for x in (r, uu, t, a))
        self._keep = (m, r, uu, t, a)
        self.lib.orc_init(self._h, _ptr(r), _ptr(uu), _ptr(t), _ptr(m), _ptr(a))
        if Ts is not None:
            ts = self._flat(Ts)
            if round_inputs_to_f32:
                ts = ts.astype(np.float32).astype(np.float64)
            self.lib.orc_init_solid_T(self._h, _ptr(ts))

    def step(self, n: int = 1) -> None:
        self.lib.orc_step(self._h, int(n))

    def fields(self) -> dict:
        from lbm_porouschem_b200.geometry import from_flat
        n = self.n
        rho = np.empty(n)
        u = np.empty(3 * n)
        T = np.empty(n)
        m = np.empty(n, dtype=np.uint8)
        a = np.empty(n)
        self.lib.orc_get(self._h, _ptr(rho), _ptr(u), _ptr(T), _ptr(m), _ptr(a))
        sh = self.cfg.shape
        out = {"rho": from_flat(rho, sh), "u": np.stack([from_flat(u[i * n:(i + 1) * n], sh) for i in range(3)]),
               "solid": from_flat((m & 1).astype(bool), sh), "alpha": from_flat(a, sh)}
        if self.cfg.thermal != "none":
            out["T"] = from_flat(T, sh)
        if self.cfg.thermal == "two_field" and self.cfg.porous != "none":
            ts = np.empty(n)
            self.lib.orc_get_solid_T(self._h, _ptr(ts), None)
            out["Ts"] = from_flat(ts, sh)
        return out

    def dist(self) -> tuple:
        """Post-stream distributions, planar [Q, N] and [QT, N] (device cell order)."""
        f = np.empty(self.cfg.Q * self.n)
        g = np.empty(self.cfg.QT * self.n)
        self.lib.orc_get_dist(self._h, _ptr(f), _ptr(g))
        return f.reshape(self.cfg.Q, self.n), g.reshape(self.cfg.QT, self.n)

    STATE_IDS = {"f": 0, "g": 1, "rho": 2, "u": 3, "T": 4, "dS": 5, "alpha": 6, "rel": 7, "mask": 8,
                 "gs": 9, "Ts": 10, "dSs": 11}

    def state_arrays(self) -> dict:
        """Zero-copy views of the per-cell state the next step reads, each shaped
        (nz, nx*ny, components) in the device cell order (cells of a z plane contiguous)."""
        real = np.float64 if self.lib is _LIBS.get("f64") else np.float32
        P = self.cfg.nx * self.cfg.ny
        nz = self.n // P
        out = {}
        for name, i in self.STATE_IDS.items():
            m = C.c_int()
            ptr = self.lib.orc_array(self._h, i, C.byref(m))
            if not ptr or m.value == 0:
                continue
            dt = np.uint8 if name == "mask" else real
            buf = (C.c_ubyte * (self.n * m.value * np.dtype(dt).itemsize)).from_address(ptr)
            out[name] = np.frombuffer(buf, dtype=dt).reshape(nz, P, m.value)
        return out

    def dist_solid(self) -> np.ndarray:
        """TS populations of porous cells, planar [QT, N] (zero elsewhere)."""
        gs = np.empty(self.cfg.QT * self.n)
        self.lib.orc_get_solid_T(self._h, None, _ptr(gs))
        return gs.reshape(self.cfg.QT, self.n)

    def diag(self) -> dict:
        out = np.empty(8)
        self.lib.orc_diag(self._h, _ptr(out))
        keys = ("mass", "energy", "solid_alpha", "umax", "Tmin", "Tmax", "nonfinite", "nfluid")
        return dict(zip(keys, out.tolist()))

    def mrt_matrix(self) -> np.ndarray:
        Q = self.cfg.Q
        return np.array([[self.lib.orc_M(self._h, r, k) for k in range(Q)] for r in range(Q)])

    def threads(self) -> int:
        return int(self.lib.orc_num_threads())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
