"""Parity of the CUDA lattice update (called through the C ABI) with the C oracle.

Tolerances (relative L2 over the compared cells):
  - FP64 storage vs the FP64 oracle: 1e-10 for rho, u, T; the solid mask and
    the flip steps are identical.  This is the strict algorithmic check.
  - FP32 storage vs the FP32 oracle: 1e-5 for rho and T.  Velocity is a small
    difference of O(1) populations, so two FP32 implementations that round
    differently (the kernel fuses multiply-adds) cannot agree on it to 1e-5;
    instead the kernel's FP32 velocity error against the FP64 oracle must stay
    within 2x the FP32 oracle's own error against the FP64 oracle (plus 1e-9).
    Flip steps agree within +-1.
  - FP16 deviation storage vs the FP64 oracle: 1e-2 relative L2 for u on a
    developed flow, 1e-3 for rho, 1e-2 for T (FP16 keeps 11 significant bits
    of each deviation; rounding is systematic once the flow is steady).
"""
import numpy as np
import pytest

from lbm_porouschem_b200 import workloads
from lbm_porouschem_b200.config import LatticeConfig

pytestmark = pytest.mark.gpu


def _rel(a, b, mask=None):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[..., mask], b[..., mask]
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def _run_pair(oracle_mod, w, n, real, prec=None):
    from lbm_porouschem_b200.lattice import Lattice
    cfg = w.cfg if prec is None else w.cfg.replace(precision=prec)
    lat = Lattice(cfg)
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    o = oracle_mod.Oracle(cfg, real=real)
    o.init(w.solid, w.reactive, **w.init)
    lat.step(n)
    o.step(n)
    return lat, o


def _compare(lat, o, tol_rho, tol_T, tol_u, u_scale_rel=False):
    g, r = lat.fields(), o.fields()
    assert np.array_equal(g["solid"], r["solid"])
    fl = ~r["solid"]
    e_rho = _rel(g["rho"], r["rho"], fl)
    if u_scale_rel:
        scale = np.abs(r["u"][:, fl]).max()
        e_u = np.sqrt(np.mean((g["u"][:, fl] - r["u"][:, fl]) ** 2)) / scale
    else:
        e_u = _rel(g["u"], r["u"], fl)
    assert e_rho < tol_rho, e_rho
    assert e_u < tol_u, e_u
    if "T" in r:
        e_T = _rel(g["T"], r["T"])
        assert e_T < tol_T, e_T
    return g, r


@pytest.mark.parametrize("coll", ["bgk", "mrt"])
def test_flow2d_fp64(oracle_mod, coll):
    w = workloads.flow2d(64, 48, seed=1, collision=coll)
    w.cfg.force = (1e-5, 0.0, 0.0)
    lat, o = _run_pair(oracle_mod, w, 300, "f64", "fp64")
    _compare(lat, o, 1e-10, 1e-10, 1e-10)


def _fp32_check(oracle_mod, w, n, tol=1e-5):
    """rho/T against the FP32 oracle; u against the FP64 oracle, bounded by the
    FP32 oracle's own rounding error."""
    lat, o32 = _run_pair(oracle_mod, w, n, "f32")
    g, r32 = lat.fields(), o32.fields()
    o64 = oracle_mod.Oracle(w.cfg, real="f64")
    o64.init(w.solid, w.reactive, **w.init)
    o64.step(n)
    r64 = o64.fields()
    assert np.array_equal(g["solid"], r32["solid"])
    fl = ~r64["solid"]
    assert _rel(g["rho"], r32["rho"], fl) < tol
    if "T" in r32:
        assert _rel(g["T"], r32["T"]) < tol
    e_kernel = np.linalg.norm(g["u"][:, fl] - r64["u"][:, fl])
    e_oracle = np.linalg.norm(r32["u"][:, fl] - r64["u"][:, fl])
    assert e_kernel <= 2.0 * e_oracle + 1e-9 * np.sqrt(fl.sum()), (e_kernel, e_oracle)
    return g, r64


@pytest.mark.parametrize("coll", ["bgk", "mrt"])
def test_flow2d_fp32(oracle_mod, coll):
    w = workloads.flow2d(64, 48, seed=1, collision=coll)
    w.cfg.force = (1e-5, 0.0, 0.0)
    _fp32_check(oracle_mod, w, 300)


def _fast_pyro(w, A=4.5e10):
    # hot start, faster rate, small heat sink and gas release so that every
    # reactive cell converts within a short test (k dt ~ 0.03 per step at T = 1)
    w.cfg.pyro_A = A
    w.cfg.heat_norm = 0.02
    w.cfg.gas_coef = 0.05
    w.init["T"] = 1.0
    return w


@pytest.mark.parametrize("coll", ["bgk", "mrt"])
def test_pyro2d_fp64_with_flips(oracle_mod, coll):
    w = _fast_pyro(workloads.pyro2d(48, 32, seed=2, collision=coll))
    lat, o = _run_pair(oracle_mod, w, 400, "f64", "fp64")
    g, r = _compare(lat, o, 1e-10, 1e-10, 1e-10)
    assert (w.solid & ~r["solid"][..., 0]).any(), "the test case should convert some cells"
    react = w.reactive[..., None]
    assert np.max(np.abs(g["alpha"] - r["alpha"])[react]) < 1e-10


def test_pyro2d_fp32(oracle_mod):
    w = _fast_pyro(workloads.pyro2d(48, 32, seed=2))
    _fp32_check(oracle_mod, w, 300)


@pytest.mark.parametrize("coll", ["bgk", "mrt"])
def test_pyro3d_fp64(oracle_mod, coll):
    w = _fast_pyro(workloads.pyro3d(20, seed=3, collision=coll, ny=16, nz=12), A=1.2e11)
    lat, o = _run_pair(oracle_mod, w, 120, "f64", "fp64")
    g, r = _compare(lat, o, 1e-10, 1e-10, 1e-10)


def test_pyro3d_fp32(oracle_mod):
    w = _fast_pyro(workloads.pyro3d(20, seed=3, ny=16, nz=12), A=1.2e11)
    _fp32_check(oracle_mod, w, 120)


def test_flow2d_fp16_vs_fp64_oracle(oracle_mod):
    w = workloads.flow2d(48, 32, seed=3)
    w.cfg.force = (2e-5, 0.0, 0.0)
    w.cfg.half_force_velocity = True
    lat, o = _run_pair(oracle_mod, w, 3000, "f64", "fp16")
    _compare(lat, o, 1e-3, 1e-3, 1e-2)


def test_pyro3d_fp16_runs_close_to_fp64(oracle_mod):
    w = _fast_pyro(workloads.pyro3d(20, seed=3, ny=16, nz=12), A=1.2e11)
    w.cfg.T0 = 1.0   # FP16 stores g - wt*T0: the shift sits at the working temperature
    lat, o = _run_pair(oracle_mod, w, 120, "f64", "fp16")
    g, r = lat.fields(), o.fields()
    assert np.array_equal(g["solid"], r["solid"])
    # a transient in which every reactive cell converts within ~20 steps: FP16
    # rounding of the deviations shows up at the 1e-3 level of rho
    assert _rel(g["rho"], r["rho"], ~r["solid"]) < 1e-2
    assert _rel(g["T"], r["T"]) < 1e-2


def test_diagnostics_match_oracle(oracle_mod):
    w = _fast_pyro(workloads.pyro2d(48, 32, seed=4))
    lat, o = _run_pair(oracle_mod, w, 150, "f64", "fp64")
    d, r = lat.diagnostics(), o.diag()
    for k in ("mass", "energy", "solid_alpha", "umax", "Tmin", "Tmax", "nfluid"):
        assert abs(d[k] - r[k]) <= 1e-9 * max(1.0, abs(r[k])), (k, d[k], r[k])
    assert d["nonfinite"] == 0


def test_fused_diag_equals_peek(oracle_mod):
    w = _fast_pyro(workloads.pyro2d(48, 32, seed=5))
    from lbm_porouschem_b200.lattice import Lattice
    lat = Lattice(w.cfg.replace(precision="fp64"))
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    lat.step(60, diag=True)
    fused = lat.read_diag()
    peek = lat.diagnostics()
    for k in ("mass", "energy", "solid_alpha", "umax", "nfluid"):
        assert fused[k] == pytest.approx(peek[k], rel=1e-12, abs=1e-14), k


def test_flip_steps_within_one(oracle_mod):
    w = _fast_pyro(workloads.pyro2d(40, 24, seed=6))
    from lbm_porouschem_b200.lattice import Lattice
    lat = Lattice(w.cfg)
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    o = oracle_mod.Oracle(w.cfg, real="f32")
    o.init(w.solid, w.reactive, **w.init)
    fg = np.full(w.solid.shape, -1)
    fo = np.full(w.solid.shape, -1)
    for n in range(1, 301):
        lat.step(1)
        o.step(1)
        sg = lat.fields()["solid"][..., 0]
        so = o.fields()["solid"][..., 0]
        fg[(fg < 0) & w.solid & ~sg] = n
        fo[(fo < 0) & w.solid & ~so] = n
    conv = fo > 0
    assert conv.sum() > 10
    assert np.all(np.abs(fg[conv] - fo[conv]) <= 1)
    assert np.array_equal(fg > 0, conv)


@pytest.mark.parametrize("dim", [2, 3])
def test_two_field_thermal_fp64(oracle_mod, dim):
    """The reference's two temperature fields (adiabatic fluid-solid interface) with a
    pressure-driven flow through a packing: FP64 kernels vs the FP64 oracle."""
    from lbm_porouschem_b200.config import FIXED_VALUE, ZERO_GRADIENT, SideBC
    from lbm_porouschem_b200.geometry import packing
    shape = (40, 24) if dim == 2 else (24, 16, 12)
    solid = packing(shape, 2.0, 4.0, 0.6, 4, periodic=(False, True, True), margin=2)
    sides = [SideBC() for _ in range(6)]
    sides[0] = SideBC.pressure(1.002, T_type=FIXED_VALUE, T=1.0)
    sides[1] = SideBC.outlet(1.0, T_type=ZERO_GRADIENT)
    cfg = LatticeConfig(dim=dim, nx=shape[0], ny=shape[1], nz=(1 if dim == 2 else shape[2]), nu=0.1,
                        thermal="two_field", tauT_fluid=0.6, tauT_solid=0.9, precision="fp64", sides=sides)

    class W:
        pass

    w = W()
    w.cfg, w.solid, w.reactive = cfg, solid, None
    w.init = {"rho": 1.0, "u": (0.0, 0.0, 0.0), "T": np.where(solid, 0.5, 0.0)}
    lat, o = _run_pair(oracle_mod, w, 300, "f64")
    g, r = _compare(lat, o, 1e-10, 1e-10, 1e-10)
    # the solid keeps its temperature: no heat crosses the interface
    assert np.allclose(g["T"].reshape(shape)[solid], 0.5, atol=1e-12)


@pytest.mark.parametrize("model", ["nee", "es"])
@pytest.mark.parametrize("dim", [2, 3])
def test_nee_every_side_mixed_types_fp64(oracle_mod, dim, model):
    """Every side active, with v, rho and T each fixed, extrapolated or kept (PERIODIC
    type: the side cell's own post-stream value) on some side; corner cells take two or
    three passes.  NEE and the equilibrium scheme (ES).  FP64 kernels vs the FP64
    oracle, conjugate heat with pyrolysis."""
    from lbm_porouschem_b200.config import FIXED_VALUE, PERIODIC, ZERO_GRADIENT, SideBC
    rng = np.random.default_rng(31 + dim)
    shape = (36, 28) if dim == 2 else (20, 17, 14)
    solid = rng.random(shape) < 0.2
    keep = np.zeros(shape, dtype=bool)
    keep[tuple(slice(2, n - 2) for n in shape)] = True
    solid &= keep
    sides = [SideBC.inlet((0.02, 0.005, 0.0), FIXED_VALUE, 1.0),
             SideBC.outlet(1.0),
             SideBC.wall(FIXED_VALUE, 0.5),
             SideBC(True, PERIODIC, FIXED_VALUE, ZERO_GRADIENT, rho=1.001)]
    sides += ([SideBC.wall(ZERO_GRADIENT), SideBC(True, ZERO_GRADIENT, PERIODIC, FIXED_VALUE, T=0.2)]
              if dim == 3 else [SideBC(), SideBC()])
    for sd in sides:
        sd.model = model
    cfg = LatticeConfig(dim=dim, nx=shape[0], ny=shape[1], nz=(1 if dim == 2 else shape[2]), collision="mrt",
                        nu=0.05, thermal="conjugate", pyro=True, pyro_A=1.2e11, heat_norm=0.02, gas_coef=0.05,
                        precision="fp64", sides=sides)

    class W:
        pass

    w = W()
    w.cfg, w.solid, w.reactive = cfg, solid, solid
    w.init = {"rho": 1.0, "u": (0.0, 0.0, 0.0), "T": 0.8}
    lat, o = _run_pair(oracle_mod, w, 120, "f64")
    _compare(lat, o, 1e-10, 1e-10, 1e-10)
