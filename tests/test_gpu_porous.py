"""Porous cells (0 < solid fraction < 1) in the CUDA kernels, through the C ABI.

The reference's porous model (src/LBM/LBM2D/_evolution.py:131-151, 213-225, 250-298; 3D
twins in LBM3D/_evolution.py): the eps-equilibrium, the Ergun / Darcy / Darcy-Forchheimer
drag through the Guo term and macro's velocity correction.  tests/test_gpu_reference.py
checks the kernels against the reference's own outputs on small lattices; here:
  - FP64 kernels against the FP64 oracle on larger lattices, BGK and MRT, every model,
    with impermeable solids next to the porous zones: 1e-10 relative L2 on rho and u;
  - FP32 kernels: rho within 1e-5 of the FP32 oracle, the velocity error against FP64
    within 2x the FP32 oracle's own;
  - the cell-list and dense (3D) forms against the FP64 oracle too, and the three forms
    against one another in FP32 / FP16 to the last bits of the storage precision.
"""
import numpy as np
import pytest

from lbm_porouschem_b200.config import LatticeConfig, SideBC

pytestmark = pytest.mark.gpu


def _zone(shape, centres, r):
    g = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    m = np.zeros(shape, dtype=bool)
    for c in centres:
        m |= sum((gi - ci) ** 2 for gi, ci in zip(g, c)) <= r * r
    return m


def _case(dim, model, collision="bgk", precision="fp64", channel=True):
    if dim == 2:
        shape, full = (96, 48), (96, 48, 1)
        porous = _zone(shape, [(30.3, 20.2), (62.7, 29.1)], 9.5)
        solid = _zone(shape, [(47.1, 12.4), (78.3, 35.2)], 5.2) & ~porous
    else:
        shape = full = (64, 24, 16)
        porous = _zone(shape, [(20.4, 11.2, 7.6), (44.1, 12.8, 8.3)], 5.4)
        solid = _zone(shape, [(32.2, 6.5, 6.1)], 3.3) & ~porous
    porous, solid = porous.reshape(full), solid.reshape(full)
    sides = [SideBC() for _ in range(6)]
    if channel:
        sides[0] = SideBC.inlet((0.02, 0.0, 0.0))
        sides[1] = SideBC.outlet(1.0)
    force = (0.0, 0.0, 0.0) if channel else (2e-5, 0.0, 0.0)
    cfg = LatticeConfig(dim=dim, nx=full[0], ny=full[1], nz=full[2], collision=collision, precision=precision,
                        nu=0.08, porous=model, sides=sides, force=force)
    eps = 0.55
    frac = (1.0 - eps) * porous
    darcy = 0.04 * porous if model != "ergun" else None
    forch = 0.3 * porous if model == "darcy_forchheimer" else None
    return cfg, solid, frac, darcy, forch


def _gpu(cfg, solid, frac, darcy, forch, steps, form=None):
    from lbm_porouschem_b200.lattice import Lattice
    lat = Lattice(cfg if form is None else cfg.replace(bulk_form=form))
    lat.set_geometry(solid)
    lat.set_porous(frac, darcy, forch)
    lat.init(rho=1.0, u=(0.0, 0.0, 0.0))
    lat.step(steps)
    out = lat.fields()
    lat.close()
    return out


def _oracle(oracle_mod, cfg, solid, frac, darcy, forch, steps, real):
    o = oracle_mod.Oracle(cfg, real=real)
    z = lambda a: np.zeros(frac.shape) if a is None else a
    o.set_porous(frac + solid, z(darcy), z(forch))
    o.init(solid, None, rho=1.0, u=(0.0, 0.0, 0.0))
    o.step(steps)
    return o.fields()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("model", ["ergun", "darcy", "darcy_forchheimer"])
@pytest.mark.parametrize("collision", ["bgk", "mrt"])
@pytest.mark.parametrize("dim", [2, 3])
def test_porous_fp64_vs_oracle(oracle_mod, dim, model, collision):
    cfg, solid, frac, darcy, forch = _case(dim, model, collision)
    n = 300 if dim == 2 else 120
    g = _gpu(cfg, solid, frac, darcy, forch, n)
    r = _oracle(oracle_mod, cfg, solid, frac, darcy, forch, n, "f64")
    fl = ~solid
    assert np.array_equal(g["solid"], r["solid"])
    assert _rel(g["rho"][fl], r["rho"][fl]) < 1e-10
    assert _rel(g["u"][:, fl], r["u"][:, fl]) < 1e-10


@pytest.mark.parametrize("model", ["ergun", "darcy_forchheimer"])
def test_porous_fp32(oracle_mod, model):
    cfg, solid, frac, darcy, forch = _case(2, model, "bgk", "fp32", channel=False)
    n = 300
    g = _gpu(cfg, solid, frac, darcy, forch, n)
    r32 = _oracle(oracle_mod, cfg, solid, frac, darcy, forch, n, "f32")
    r64 = _oracle(oracle_mod, cfg, solid, frac, darcy, forch, n, "f64")
    fl = ~solid
    assert _rel(g["rho"][fl], r32["rho"][fl]) < 1e-5
    e_k = np.linalg.norm(g["u"][:, fl] - r64["u"][:, fl])
    e_o = np.linalg.norm(r32["u"][:, fl] - r64["u"][:, fl])
    assert e_k <= 2.0 * e_o + 1e-9 * np.sqrt(fl.sum()), (e_k, e_o)


@pytest.mark.parametrize("form", ["list", "dense"])
def test_porous_forms_fp64_vs_oracle(oracle_mod, form):
    """The cell-list and dense (TMA-staged) forms on porous cells, against the oracle."""
    cfg, solid, frac, darcy, forch = _case(3, "darcy_forchheimer", "mrt", "fp64")
    g = _gpu(cfg, solid, frac, darcy, forch, 120, form)
    r = _oracle(oracle_mod, cfg, solid, frac, darcy, forch, 120, "f64")
    fl = ~solid
    assert _rel(g["rho"][fl], r["rho"][fl]) < 1e-10
    assert _rel(g["u"][:, fl], r["u"][:, fl]) < 1e-10


@pytest.mark.parametrize("precision,tol", [("fp32", 1e-6), ("fp16", 1e-4)])
def test_porous_forms_agree(precision, tol):
    """The three forms run the same arithmetic; with porous cells the compiler may contract
    a product into a fused multiply-add in one kernel and not in another, so they agree to
    the last bits of the storage precision rather than bit for bit."""
    cfg, solid, frac, darcy, forch = _case(3, "darcy_forchheimer", "mrt", precision)
    a = _gpu(cfg, solid, frac, darcy, forch, 60, "tile")
    for form in ("list", "dense"):
        b = _gpu(cfg, solid, frac, darcy, forch, 60, form)
        assert np.array_equal(a["solid"], b["solid"])
        fl = ~solid
        assert _rel(b["rho"][fl].astype(np.float64), a["rho"][fl].astype(np.float64)) < tol, form
        assert _rel(b["u"][:, fl].astype(np.float64), a["u"][:, fl].astype(np.float64)) < 100 * tol, form


def test_porous_side_layers_rejected():
    from lbm_porouschem_b200._native import LBMNativeError
    cfg, solid, frac, darcy, forch = _case(2, "darcy")
    frac = frac.copy()
    frac[1, 20, 0] = 0.3      # next to the inlet
    from lbm_porouschem_b200.lattice import Lattice
    lat = Lattice(cfg)
    lat.set_geometry(solid)
    lat.set_porous(frac, darcy, forch)
    with pytest.raises(LBMNativeError):
        lat.init(rho=1.0, u=(0.0, 0.0, 0.0))
    lat.close()


def test_solver_surface_runs_porous_cells(oracle_mod):
    """The reference's setters on the solver class (isPoro=True, add_solid with a fraction,
    set_poro_Darcy; src/LBM/LBM2D/_io.py:123-164) drive the same porous run as the oracle."""
    from lbm_porouschem_b200.flag import BC_FLOW
    from lbm_porouschem_b200.solver import LBM2DSolver
    nx, ny = 64, 32
    lb = LBM2DSolver(nx, ny, 1, 1, 1, "poro", False, False, True, False)
    lb.precision = "fp64"
    lb.set_viscosity(0.1)
    lb.set_BC(0, BC_FLOW.inlet)
    lb.set_v_BC_value(0, [0.02, 0.0, 0.0])
    lb.set_BC(1, BC_FLOW.outlet)
    lb.set_rho_BC_value(1, 1.0)
    zone = _zone((nx, ny), [(24.2, 15.3)], 7.1).reshape(nx, ny, 1) * 1.0
    lb.add_solid(0.4 * zone)
    lb.set_poro_Darcy(zone, 0.05)
    lb.init_simulation()
    for _ in range(200):
        lb.step()
    cfg = lb._cfg
    assert cfg.porous == "darcy"
    o = oracle_mod.Oracle(cfg, real="f64")
    o.set_porous(0.4 * zone, 0.05 * zone, None)
    o.init(np.zeros(zone.shape, dtype=bool), None, rho=1.0, u=(0.0, 0.0, 0.0))
    o.step(200)
    r = o.fields()
    g = lb._lat.fields()
    assert _rel(g["rho"], r["rho"]) < 1e-10
    assert _rel(g["u"], r["u"]) < 1e-10
