"""Porous cells with two temperature fields in the CUDA kernels, through the C ABI.

In the reference's two-field model a porous cell (0 < solid < 1) carries both the fluid
temperature TF and the solid temperature TS; they exchange heat there,
dH = h a (T_f,phys - T_s,phys) dt, and the porous surface radiates to the ambient
(src/LBM/LBM2D/_evolution.py:30-100, 186-202; src/LBM/LBM2D/_thermal.py:213-220; 3D twins in
LBM3D/).  tests/test_gpu_reference.py checks the kernels against the reference's own
outputs on small lattices; here, against the oracle:
  - FP64 tile and cell-list forms on larger lattices where the porous zones touch
    impermeable solids (TS crosses between porous and pure-solid cells), radiation on,
    2D and 3D, BGK and MRT: 1e-10 relative L2 on rho, u, T and the porous cells' TS (the
    oracle without the reference's frozen pure-solid temperature, as the kernels do);
  - FP32: rho, T and TS within 1e-5 of the FP32 oracle;
  - a checkpoint resumed mid-run equals the uninterrupted run bit for bit;
  - combinations the kernels do not run are refused.
"""
import numpy as np
import pytest

from lbm_porouschem_b200.config import FIXED_VALUE, ZERO_GRADIENT, LatticeConfig, SideBC

pytestmark = pytest.mark.gpu


def _zone(shape, centres, r):
    g = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    m = np.zeros(shape, dtype=bool)
    for c in centres:
        m |= sum((gi - ci) ** 2 for gi, ci in zip(g, c)) <= r * r
    return m


def _border(zone):
    b = np.zeros(zone.shape, dtype=bool)
    for ax in range(zone.ndim):
        if zone.shape[ax] > 1:
            for sh in (1, -1):
                b |= zone & ~np.roll(zone, sh, axis=ax)
    return b.astype(np.float64)


def _case(dim, collision="bgk", precision="fp64", model="darcy", radiation=True):
    if dim == 2:
        shape = full = (80, 40, 1)
        porous = _zone(shape[:2], [(26.3, 18.2), (52.7, 22.1)], 8.5).reshape(full)
        solid = _zone(shape[:2], [(38.1, 12.4), (60.3, 31.2)], 4.8).reshape(full) & ~porous
    else:
        shape = full = (48, 20, 16)
        porous = _zone(shape, [(18.4, 9.2, 7.6), (31.1, 10.8, 8.3)], 4.6)
        solid = _zone(shape, [(24.2, 5.5, 6.1)], 3.1) & ~porous
    rng = np.random.default_rng(5)
    sides = [SideBC() for _ in range(6)]
    sides[0] = SideBC.inlet((0.02, 0.0, 0.0), FIXED_VALUE, 1.0)
    sides[1] = SideBC.outlet(1.0, ZERO_GRADIENT, 0.0)
    tau = (lambda D: 3 * D + 0.5) if dim == 2 else (lambda D: 4 * D + 0.5)
    cfg = LatticeConfig(dim=dim, nx=full[0], ny=full[1], nz=full[2], collision=collision, precision=precision,
                        nu=0.08, porous=model, sides=sides, thermal="two_field", tauT_fluid=tau(0.04),
                        tauT_solid=tau(0.09), T_ref=300.0, T_scale=500.0, Ts_ref=260.0, Ts_scale=580.0,
                        cap_fluid=1100.0, cap_solid=750.0, dt_phys=1.0, dx_phys=1.0, radiation=radiation,
                        T_ambient=320.0)
    zf = porous.astype(np.float64)
    inputs = dict(
        solid=solid, frac=0.45 * zf, darcy=0.05 * zf if model != "ergun" else None,
        forch=0.2 * zf if model == "darcy_forchheimer" else None,
        h=2.5 * zf, a=(1.0 + rng.uniform(0, 0.5, full)) * zf, rhos=(1.5 + rng.uniform(0, 1, full)) * zf + (1 - zf),
        emis=0.7 * _border(porous), rsurf=_border(porous),
        T=np.where(solid, 0.5, 0.1 + 0.05 * rng.uniform(0, 1, full)).astype(np.float32).astype(np.float64),
        Ts=(0.55 + 0.1 * rng.uniform(0, 1, full)).astype(np.float32).astype(np.float64))
    return cfg, inputs


def _gpu(cfg, x, steps, form="tile", lat_out=False):
    from lbm_porouschem_b200.lattice import Lattice
    lat = Lattice(cfg.replace(bulk_form=form))
    lat.set_geometry(x["solid"])
    lat.set_porous(x["frac"], x["darcy"], x["forch"], h=x["h"], a=x["a"], rho_solid=x["rhos"],
                   emissivity=x["emis"], radiation_surface=x["rsurf"])
    lat.init(rho=1.0, u=(0.0, 0.0, 0.0), T=x["T"], Ts=x["Ts"])
    if lat_out:
        return lat
    lat.step(steps)
    out = lat.fields()
    lat.close()
    return out


def _oracle(oracle_mod, cfg, x, steps, real):
    o = oracle_mod.Oracle(cfg, real=real)
    o.set_porous(x["frac"] + x["solid"], x["darcy"], x["forch"])
    o.set_porous_heat(x["h"], x["a"], x["rhos"], x["emis"], x["rsurf"])
    o.init(x["solid"], None, rho=1.0, u=(0.0, 0.0, 0.0), T=x["T"], Ts=x["Ts"])
    o.step(steps)
    return o.fields()


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("form", ["tile", "list"])
@pytest.mark.parametrize("collision", ["bgk", "mrt"])
@pytest.mark.parametrize("dim,model", [(2, "darcy"), (2, "ergun"), (3, "darcy_forchheimer"), (3, "ergun")])
def test_fp64_matches_oracle(oracle_mod, dim, model, collision, form):
    cfg, x = _case(dim, collision, model=model)
    steps = 150 if dim == 2 else 60
    g = _gpu(cfg, x, steps, form)
    r = _oracle(oracle_mod, cfg, x, steps, "f64")
    fl = ~x["solid"]
    pc = x["frac"] > 0
    assert np.array_equal(g["solid"], r["solid"])
    assert _rel(g["rho"][fl], r["rho"][fl]) < 1e-10
    assert _rel(g["u"][:, fl], r["u"][:, fl]) < 1e-10
    assert _rel(g["T"], r["T"]) < 1e-10
    assert _rel(g["Ts"][pc], r["Ts"][pc]) < 1e-10
    # the exchange moved heat: TS of the porous cells left its start
    assert _rel(g["Ts"][pc], x["Ts"][pc]) > 1e-3


@pytest.mark.parametrize("dim", [2, 3])
def test_fp32_matches_oracle(oracle_mod, dim):
    cfg, x = _case(dim, precision="fp32")
    steps = 150 if dim == 2 else 60
    g = _gpu(cfg, x, steps, "list")
    r = _oracle(oracle_mod, cfg, x, steps, "f32")
    fl = ~x["solid"]
    pc = x["frac"] > 0
    assert _rel(g["rho"][fl], r["rho"][fl]) < 1e-5
    assert _rel(g["T"], r["T"]) < 1e-5
    assert _rel(g["Ts"][pc], r["Ts"][pc]) < 1e-5


def test_checkpoint_resume_bit_exact(tmp_path):
    from lbm_porouschem_b200.lattice import Lattice
    cfg, x = _case(2, "mrt", precision="fp32")
    a = _gpu(cfg, x, 0, "list", lat_out=True)
    a.step(37)
    path = a.save_checkpoint(tmp_path / "ph.npz")
    a.step(40)
    fa = a.fields()
    a.close()
    b = Lattice.load_checkpoint(path)
    b.step(40)
    fb = b.fields()
    b.close()
    for k in ("rho", "u", "T", "Ts"):
        assert np.array_equal(fa[k], fb[k]), k


def test_refused_combinations():
    from lbm_porouschem_b200 import _native as N
    from lbm_porouschem_b200.lattice import Lattice
    cfg, _ = _case(2)
    with pytest.raises(N.LBMNativeError, match="constant viscosity"):
        Lattice(cfg.replace(thermal="conjugate", radiation=False))
    with pytest.raises(N.LBMNativeError, match="radiation"):
        Lattice(cfg.replace(porous="none"))
    with pytest.raises(N.LBMNativeError, match="cap_fluid"):
        Lattice(cfg.replace(cap_solid=0.0))
    with pytest.raises(N.LBMNativeError, match="dense"):
        Lattice(cfg.replace(dim=3, nx=32, ny=8, nz=8, bulk_form="dense"))
