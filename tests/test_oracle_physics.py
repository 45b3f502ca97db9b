"""Pins of the C oracle against analytic known answers and lattice invariants.

The reference's own tests pin no lattice numbers (tests/test_lbm2d.py:8-27 only
constructs the solver) and the reference cannot run here, so the oracle is
pinned by physics instead:
  - equilibrium is a fixed point; mass is conserved with periodic sides;
  - body-force Poiseuille flow between bounce-back walls matches the parabola,
    with the reference's forcing (u without F/2: effective force (1-1/(2tau))F)
    and with the standard Guo velocity (u with F/2: full force F);
  - MRT with every rate equal to 1/tau reproduces BGK; the MRT bases are orthogonal;
  - a solid cell held at fixed temperature follows the explicit-Euler Arrhenius
    decay, turns fluid on the predicted step, and its gas and heat balances close.
"""
import math

import numpy as np
import pytest

from lbm_porouschem_b200.config import LatticeConfig, SideBC, FIXED_VALUE, ZERO_GRADIENT
from lbm_porouschem_b200.geometry import packing


def _run(oracle_mod, cfg, solid, n, real="f64", **init):
    o = oracle_mod.Oracle(cfg, real=real)
    o.init(solid, init.pop("reactive", None), **init)
    o.step(n)
    return o


@pytest.mark.parametrize("dim", [2, 3])
def test_equilibrium_fixed_point(oracle_mod, dim):
    cfg = LatticeConfig(dim=dim, nx=6, ny=5, nz=4 if dim == 3 else 1, nu=0.1)
    solid = np.zeros(cfg.shape[:dim], dtype=bool)
    o = _run(oracle_mod, cfg, solid, 7, rho=1.02, u=(0.01, -0.02, 0.005 if dim == 3 else 0.0))
    f = o.fields()
    assert np.allclose(f["rho"], 1.02, atol=1e-13)
    assert np.allclose(f["u"][0], 0.01, atol=1e-13)


@pytest.mark.parametrize("dim,coll", [(2, "bgk"), (2, "mrt"), (3, "bgk"), (3, "mrt")])
def test_mass_conservation_periodic(oracle_mod, dim, coll):
    shape = (24, 20) if dim == 2 else (12, 10, 8)
    cfg = LatticeConfig(dim=dim, nx=shape[0], ny=shape[1], nz=shape[2] if dim == 3 else 1,
                        collision=coll, nu=0.05)
    solid = packing(shape, 1.5, 3.0, 0.7, seed=3)
    rng = np.random.default_rng(0)
    full = cfg.shape
    rho = 1.0 + 0.01 * rng.standard_normal(full)
    o = oracle_mod.Oracle(cfg, real="f64")
    o.init(solid, rho=rho, u=(0.0, 0.0, 0.0))
    m0 = o.diag()["mass"]
    o.step(200)
    m1 = o.diag()["mass"]
    assert abs(m1 - m0) / m0 < 1e-12


@pytest.mark.parametrize("half", [False, True])
def test_poiseuille_body_force(oracle_mod, half):
    # BGK halfway bounce-back puts the wall exactly halfway at tau = 1/2 + sqrt(3/16)
    nx, ny, tau, g = 4, 22, 0.5 + math.sqrt(3.0 / 16.0), 1e-6
    nu = (tau - 0.5) / 3.0
    cfg = LatticeConfig(dim=2, nx=nx, ny=ny, nu=nu, force=(g, 0.0, 0.0), half_force_velocity=half)
    solid = np.zeros((nx, ny), dtype=bool)
    solid[:, 0] = solid[:, -1] = True
    o = _run(oracle_mod, cfg, solid, 12000)
    ux = o.fields()["u"][0][0, 1:-1, 0]
    y = np.arange(1, ny - 1) - 0.5          # halfway walls at y = 0.5 and ny - 1.5
    H = ny - 2
    geff = g if half else g * (1.0 - 1.0 / (2.0 * tau))
    ua = geff / (2 * nu) * y * (H - y)
    if not half:
        ua -= geff / 2.0   # the reference's u = sum(e f)/rho omits half of the applied momentum
    assert np.max(np.abs(ux - ua)) / ua.max() < 1e-6


def test_mrt_bases_orthogonal(oracle_mod):
    for dim in (2, 3):
        cfg = LatticeConfig(dim=dim, nx=4, ny=4, nz=4 if dim == 3 else 1)
        o = oracle_mod.Oracle(cfg)
        M = o.mrt_matrix()
        G = M @ M.T
        assert np.allclose(G - np.diag(np.diag(G)), 0.0)
        assert np.all(np.diag(G) > 0)


@pytest.mark.parametrize("dim", [2, 3])
def test_mrt_with_bgk_rates_equals_bgk(oracle_mod, dim):
    shape = (10, 8) if dim == 2 else (8, 6, 6)
    tau = 0.9
    base = LatticeConfig(dim=dim, nx=shape[0], ny=shape[1], nz=shape[2] if dim == 3 else 1,
                         nu=(tau - 0.5) / 3.0, eos="incompressible", force=(1e-5, 0, 0))
    mrt = base.replace(collision="mrt", mrt_rates={r: 1.0 / tau for r in range(base.Q)})
    solid = packing(shape, 1.2, 2.0, 0.8, seed=1)
    a = _run(oracle_mod, base, solid, 50).fields()
    b = _run(oracle_mod, mrt, solid, 50).fields()
    assert np.max(np.abs(a["u"] - b["u"])) < 1e-13
    assert np.max(np.abs(a["rho"] - b["rho"])) < 1e-13


def _single_cell_pyro(T=0.9, heat_norm=0.0, A=1e8, alpha_flip=0.01, gas_coef=0.75):
    cfg = LatticeConfig(dim=2, nx=9, ny=9, nu=0.1, thermal="conjugate", tauT_fluid=0.7,
                        tauT_solid=0.9, pyro=True, pyro_A=A, heat_norm=heat_norm, alpha_flip=alpha_flip,
                        gas_coef=gas_coef)
    solid = np.zeros((9, 9), dtype=bool)
    solid[4, 4] = True
    return cfg, solid


def test_arrhenius_decay_and_flip_step(oracle_mod):
    # no gas release and no heat sink: the cell stays at its initial temperature
    T, A = 0.9, 3e9
    cfg, solid = _single_cell_pyro(T=T, A=A, gas_coef=0.0)
    TK = 300.0 + 500.0 * float(np.float32(T)) + 1e-6      # src/LBM/LBM2D/_chemical.py:209
    k = A * math.exp(-1.25e5 / TK / 8.314441)
    r = 1.0 - k * 1e-4
    n_flip = next(n for n in range(1, 10 ** 6) if r ** n < 0.01)
    o = oracle_mod.Oracle(cfg, real="f64")
    o.init(solid, solid, rho=1.0, T=T)
    o.step(10)
    a10 = o.fields()["alpha"][4, 4, 0]
    assert abs(a10 - r ** 10) < 1e-12
    o.step(n_flip - 11)
    assert o.fields()["solid"][4, 4]
    o.step(1)                                  # the step on which alpha crosses 0.01
    assert not o.fields()["solid"][4, 4]


def test_pyrolysis_gas_and_heat_balance(oracle_mod):
    T, hn = 0.9, 0.8
    cfg, solid = _single_cell_pyro(T=T, heat_norm=hn, A=3e9)
    o = oracle_mod.Oracle(cfg, real="f64")
    o.init(solid, solid, rho=1.0, T=T)
    d0 = o.diag()
    alphas = [1.0]
    for _ in range(40):
        o.step(1)
        alphas.append(o.fields()["alpha"][4, 4])
    d = o.diag()
    # gas released at step n enters the fluid on step n+1; heat likewise
    consumed_prev = alphas[0] - alphas[-2]
    assert abs((d["mass"] - d0["mass"]) - cfg.gas_coef * consumed_prev) < 1e-10
    assert abs((d["energy"] - d0["energy"]) + hn * consumed_prev) < 1e-10


def test_nee_pressure_channel(oracle_mod):
    nx, ny = 24, 12
    sides = [SideBC() for _ in range(6)]
    sides[0] = SideBC.pressure(1.001, T_type=FIXED_VALUE, T=1.0)
    sides[1] = SideBC.outlet(1.0, T_type=ZERO_GRADIENT)
    sides[2] = SideBC.wall(T_type=ZERO_GRADIENT)
    sides[3] = SideBC.wall(T_type=ZERO_GRADIENT)
    cfg = LatticeConfig(dim=2, nx=nx, ny=ny, nu=0.1, thermal="conjugate", sides=sides)
    solid = np.zeros((nx, ny), dtype=bool)
    o = _run(oracle_mod, cfg, solid, 3000, T=0.0)
    f = o.fields()
    ux = f["u"][0]
    assert np.all(ux[2:-2, 2:-2] > 0)
    # steady: the flux through every cross-section agrees
    flux = (f["rho"] * ux)[2:-2, :].sum(axis=1)
    assert np.std(flux) / np.mean(flux) < 1e-2
    assert np.allclose(f["T"][0, :], 1.0)
    assert abs(f["rho"][0, ny // 2] - 1.001) < 1e-12


@pytest.mark.parametrize("dim", [2, 3])
def test_two_field_interface_is_adiabatic(oracle_mod, dim):
    """Two-field temperature (the reference's TF / TS with a binary mask): no heat crosses
    the fluid-solid interface, so with periodic sides the fluid and the solid each keep
    their own total temperature, while the conjugate field exchanges it."""
    shape = (16, 12) if dim == 2 else (12, 10, 8)
    solid = np.zeros(shape, dtype=bool)
    solid[4:9, 3:8] = True
    T0 = np.where(solid, 1.0, 0.0)
    tot = {}
    for mode in ("two_field", "conjugate"):
        cfg = LatticeConfig(dim=dim, nx=shape[0], ny=shape[1], nz=(1 if dim == 2 else shape[2]), nu=0.1,
                            thermal=mode, tauT_fluid=0.7, tauT_solid=0.9)
        o = _run(oracle_mod, cfg, solid, 200, T=T0)
        T = o.fields()["T"].reshape(shape)
        tot[mode] = (T[solid].sum(), T[~solid].sum())
    assert abs(tot["two_field"][0] - solid.sum()) < 1e-9
    assert abs(tot["two_field"][1]) < 1e-9
    assert tot["conjugate"][1] > 0.1 * solid.sum()


def _flowrate_channel(dim, F, coll="bgk"):
    sides = [SideBC() for _ in range(6)]
    sides[0] = SideBC.inlet_flowrate(F)
    sides[1] = SideBC.outlet(1.0)
    sides[2], sides[3] = SideBC.wall(), SideBC.wall()
    return LatticeConfig(dim=dim, nx=24, ny=10, nz=4 if dim == 3 else 1, collision=coll, nu=0.1, sides=sides)


@pytest.mark.parametrize("dim", [2, 3])
def test_flowrate_inlet_follows_the_reference_controller(oracle_mod, dim):
    """The flow-rate inlet law of src/LBM/LBM2D/_boundary.py:324-333, restated here in
    numpy from the fields of the previous step: flow0 = sum rho*u_x at x = 0,
    coef = F/flow0, u(0,j) = (0.01*coef + 1 - 0.01) * u(1,j) on every side cell that no
    other side overrides; the columns x = 0, 1 start at v0 = F/ny/nz
    (_initialize.py:67-74)."""
    F = 0.12
    cfg = _flowrate_channel(dim, F)
    o = oracle_mod.Oracle(cfg, real="f64")
    o.init(np.zeros(cfg.shape[:dim], dtype=bool), rho=1.0, u=(0.0, 0.0, 0.0))
    f = o.fields()
    v0 = F / cfg.ny / cfg.nz
    assert np.all(f["u"][0][:2] == v0) and np.all(f["u"][1][:2] == 0)
    inner = slice(1, cfg.ny - 1)                       # y = 0, ny-1 belong to the walls
    for _ in range(40):
        rho0, ux0 = f["rho"][0].reshape(-1), f["u"][0][0].reshape(-1)
        flow0 = 0.0
        for a, b in zip(rho0, ux0):                   # the oracle's summation order (j = y + ny*z)
            flow0 += a * b
        gain = 0.01 * (F / flow0) + 1 - 0.01
        want = gain * f["u"][:, 1]
        o.step(1)
        f = o.fields()
        assert np.allclose(f["u"][:, 0][:, inner], want[:, inner], rtol=1e-13, atol=1e-17)
        assert np.all(f["u"][:, 0][:, [0, -1]] == 0)   # wall corners


def test_flowrate_inlet_steady_state(oracle_mod):
    """After the flow develops the controller holds a steady inlet flux: the law's fixed
    point u(0,j) = g u(1,j), with one gain g = 0.01 F/flux + 0.99 over the side.  The
    law is proportional, so the steady flux is F only where u(0) = u(1); on this short
    walled channel it settles near 0.42 F."""
    F = 0.12
    cfg = _flowrate_channel(2, F)
    o = oracle_mod.Oracle(cfg, real="f64")
    o.init(np.zeros(cfg.shape[:2], dtype=bool), rho=1.0, u=(0.0, 0.0, 0.0))
    o.step(3000)
    a = o.fields()
    o.step(200)
    b = o.fields()
    flux = [float((f["rho"][0, :, 0] * f["u"][0, 0, :, 0]).sum()) for f in (a, b)]
    assert abs(flux[1] - flux[0]) < 1e-9 * F
    g = 0.01 * F / flux[1] + 0.99
    assert np.allclose(b["u"][0, 0, 1:-1, 0], g * b["u"][0, 1, 1:-1, 0], rtol=1e-10)
    assert 0 < flux[1] < F


@pytest.mark.parametrize("dim", [2, 3])
def test_es_side_cells_hold_equilibrium(oracle_mod, dim):
    """BC_MODEL.ES (src/LBM/LBM2D/_boundary.py:269-315): after a step every side cell's
    populations are feq of its own (rho, u), with u the fixed inlet velocity and rho the
    fixed outlet density; the reference's feq9/feq19 (_evolution.py:213-225)."""
    sides = [SideBC.inlet((0.03, 0.0, 0.0)), SideBC.outlet(1.01), SideBC.wall(), SideBC.wall(),
             SideBC(), SideBC()]
    for sd in sides:
        sd.model = "es"
    cfg = LatticeConfig(dim=dim, nx=16, ny=10, nz=4 if dim == 3 else 1, nu=0.1, sides=sides)
    o = oracle_mod.Oracle(cfg, real="f64")
    o.init(np.zeros(cfg.shape[:dim], dtype=bool), rho=1.0, u=(0.0, 0.0, 0.0))
    o.step(25)
    fl = o.fields()
    f, _ = o.dist()
    Q = f.shape[0]
    f = np.stack([fk.reshape(cfg.shape, order="F") for fk in f])
    e, w = np.array(_E[dim], dtype=float), _W[dim]
    for x in (0, cfg.nx - 1):
        rho = fl["rho"][x]
        u = fl["u"][:, x]
        eu = np.tensordot(e, u, axes=(1, 0))
        uu = (u * u).sum(0)
        feq = w.reshape((Q,) + (1,) * rho.ndim) * rho * (1 + 3 * eu + 4.5 * eu ** 2 - 1.5 * uu)
        assert np.allclose(f[:, x][:, 1:-1], feq[:, 1:-1], rtol=0, atol=1e-15)
    assert np.allclose(fl["u"][0][0][1:-1], 0.03) and np.allclose(fl["rho"][-1][1:-1], 1.01)


_E = {2: [(0, 0, 0), (1, 0, 0), (0, 1, 0), (-1, 0, 0), (0, -1, 0), (1, 1, 0), (-1, 1, 0), (-1, -1, 0), (1, -1, 0)],
      3: [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0), (-1, 1, 0),
          (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 1), (0, -1, 1),
          (0, 1, -1), (0, -1, -1)]}
_W = {2: np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4), 3: np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)}


@pytest.mark.parametrize("coll", ["bgk", "mrt"])
def test_sutherland_at_uniform_temperature_equals_constant_viscosity(oracle_mod, coll):
    """Sutherland viscosity (src/LBM/LBM2D/_evolution.py:232-234) at a uniform temperature
    is the constant viscosity suth_A TK^1.5/(TK + Ts).  The flow moves the temperature by
    ~1e-5 (compressibility, solid interfaces), so the runs agree to 1e-4 of the velocity
    scale; a wrong law or unit mapping differs at order one."""
    shape = (20, 14)
    solid = packing(shape, 1.5, 2.5, 0.8, seed=4)
    base = LatticeConfig(dim=2, nx=20, ny=14, collision=coll, nu=0.1, thermal="conjugate",
                         force=(2e-5, 0.0, 0.0), T_ref=300.0, T_scale=500.0)
    TK = 300.0 + 500.0 * 0.6
    A, Ts = 0.004, 170.0
    suth = base.replace(viscosity="sutherland", suth_A=A, suth_Ts=Ts)
    const = base.replace(nu=A * TK ** 1.5 / (TK + Ts))
    out = []
    for cfg in (suth, const):
        o = oracle_mod.Oracle(cfg, real="f64")
        o.init(solid, rho=1.0, u=(0.0, 0.0, 0.0), T=0.6)
        o.step(150)
        out.append(o.fields())
    fl = ~out[0]["solid"]
    umax = np.abs(out[0]["u"][:, fl]).max()
    assert umax > 1e-5
    assert np.abs(out[0]["T"] - 0.6).max() < 1e-4
    assert np.abs(out[0]["u"] - out[1]["u"]).max() < 1e-4 * umax
    assert np.abs(out[0]["rho"] - out[1]["rho"]).max() < 1e-8
