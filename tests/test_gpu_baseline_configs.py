"""The CUDA path on the benchmark configurations at their own parameters, against the oracle.

  - Config 1: D2Q9 BGK 256 x 128, tau 0.8, g_x = 1e-6, periodic, porosity 0.65, the full
    20,000 steps.  FP64 kernel vs FP64 oracle: 1e-10 relative L2 on rho, 1e-9 on u (the
    kernels contract multiply-adds the oracle rounds twice; over 20,000 steps that moves a
    velocity of ~1e-4 by 1.5e-10 of its norm).  FP32
    kernel: rho and velocity errors against FP64 within 2x the FP32 oracle's own (FP32 mass
    drifts by ~1.7e-4 over 20,000 steps in both, through rounding that differs in the last
    bits; the measured figures are printed); Darcy permeability k = nu <u_x> / g_x within 2x
    the FP32 oracle's own error against FP64 (both ~1.5e-2: FP32 populations of ~0.1 resolve
    the ~1e-4 velocity of this flow to about 1 %).
  - Config 2: D2Q9 + D2Q5 + pyrolysis 512 x 256 with its Arrhenius parameters (A = 1e8 1/s,
    E = 1.25e5 J/mol, heat 0.8, gas 0.75, dt 1e-4 s), 5,000 steps: FP64 1e-10 and the same
    mask; FP32 rho / T within 1e-5.  At that rate a cell needs ~7e4 steps to convert, so
    the conversion steps are compared on a 96 x 48 packing started hot (T = 1), ~95,000 steps
    to the first conversion: every cell's conversion step within +-1 of the oracle's in FP64,
    and within 1e-4 of the step count in FP32 (rounding that differs in the last bits moves
    the slow Arrhenius clock: measured 4 to 6 steps of ~97,000).
  - Config 3: D3Q19-MRT + D3Q7 + pyrolysis at 64^3 (the 256^3 case's parameters), 400
    steps: FP64 1e-10; FP32 rho / T 1e-5; FP16 deviation storage u within 1e-2 (measured
    2.4e-3), rho within 1e-3 and T within 1e-2 of FP64.
"""
import numpy as np
import pytest

from lbm_porouschem_b200 import workloads

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def _gpu(w, n, precision=None, chunk=None):
    from lbm_porouschem_b200.lattice import Lattice
    cfg = w.cfg if precision is None else w.cfg.replace(precision=precision)
    lat = Lattice(cfg)
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    lat.step(n)
    out = lat.fields()
    lat.close()
    return out


def _oracle(oracle_mod, w, n, real):
    o = oracle_mod.Oracle(w.cfg, real=real)
    o.init(w.solid, w.reactive, **w.init)
    o.step(n)
    return o.fields()


def test_config1_20000_steps(oracle_mod, capsys):
    n = 20000
    w64 = workloads.flow2d(256, 128, seed=0, precision="fp64")
    g64 = _gpu(w64, n)
    r64 = _oracle(oracle_mod, w64, n, "f64")
    fl = ~r64["solid"]
    assert np.array_equal(g64["solid"], r64["solid"])
    assert _rel(g64["rho"][fl], r64["rho"][fl]) < 1e-10
    assert _rel(g64["u"][:, fl], r64["u"][:, fl]) < 1e-9
    w32 = workloads.flow2d(256, 128, seed=0, precision="fp32")
    g32 = _gpu(w32, n)
    r32 = _oracle(oracle_mod, w32, n, "f32")
    e_rho = _rel(g32["rho"][fl], r64["rho"][fl])
    e_rho32 = _rel(r32["rho"][fl], r64["rho"][fl])
    e_kernel = _rel(g32["u"][:, fl], r64["u"][:, fl])
    e_f32 = _rel(r32["u"][:, fl], r64["u"][:, fl])
    e_vs32 = _rel(g32["u"][:, fl], r32["u"][:, fl])
    nu, gx = w32.cfg.nu, w32.cfg.force[0]
    k = lambda f: nu * float(np.mean(f["u"][0])) / gx    # superficial velocity over all cells
    with capsys.disabled():
        print(f"\nconfig 1, 20000 steps FP32: rho relL2 vs FP64 {e_rho:.3e} (FP32 oracle {e_rho32:.3e}); "
              f"u relL2 vs FP64 {e_kernel:.3e} (FP32 oracle {e_f32:.3e}), "
              f"vs FP32 oracle {e_vs32:.3e}; permeability {k(g32):.6e} (FP32 oracle {k(r32):.6e}) "
              f"vs FP64 {k(r64):.6e}")
    assert e_rho <= 2.0 * e_rho32 + 1e-7
    assert e_kernel <= 2.0 * e_f32 + 1e-9
    assert abs(k(g32) - k(r64)) <= 2.0 * abs(k(r32) - k(r64)) + 1e-6 * abs(k(r64))


def test_config2_parameters_5000_steps(oracle_mod):
    n = 5000
    w = workloads.pyro2d(512, 256, seed=0, precision="fp64")
    assert w.cfg.pyro_A == 1e8 and w.cfg.heat_norm == 0.8 and w.cfg.gas_coef == 0.75
    g = _gpu(w, n)
    r = _oracle(oracle_mod, w, n, "f64")
    fl = ~r["solid"]
    assert np.array_equal(g["solid"], r["solid"])
    assert _rel(g["rho"][fl], r["rho"][fl]) < 1e-10
    assert _rel(g["u"][:, fl], r["u"][:, fl]) < 1e-10
    assert _rel(g["T"], r["T"]) < 1e-10
    w32 = workloads.pyro2d(512, 256, seed=0, precision="fp32")
    g32 = _gpu(w32, n)
    r32 = _oracle(oracle_mod, w32, n, "f32")
    assert _rel(g32["rho"][fl], r32["rho"][fl]) < 1e-5
    assert _rel(g32["T"], r32["T"]) < 1e-5


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_config2_conversion_steps_at_the_real_rate(oracle_mod, precision, capsys):
    """Flip steps at config 2's own Arrhenius rate: the oracle is stepped to just before its
    first conversion, then both step one at a time and every cell's step is recorded."""
    from lbm_porouschem_b200.lattice import Lattice
    w = workloads.pyro2d(96, 48, seed=3, precision=precision)
    real = "f64" if precision == "fp64" else "f32"
    w.init["T"] = 1.0
    solid0 = w.solid.reshape(w.cfg.shape)
    o = oracle_mod.Oracle(w.cfg, real=real)
    o.init(w.solid, w.reactive, **w.init)
    lat = Lattice(w.cfg)
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    t, chunk = 0, 2000
    while True:                      # coarse search for the first conversion
        o.step(chunk)
        if (solid0 & ~o.fields()["solid"]).any():
            break
        t += chunk
        lat.step(chunk)
        assert t < 400000, "no conversion"
    o = oracle_mod.Oracle(w.cfg, real=real)
    o.init(w.solid, w.reactive, **w.init)
    o.step(t)
    first_g = np.full(solid0.shape, -1)
    first_o = np.full(solid0.shape, -1)
    end = t + chunk + 3000
    for s in range(t + 1, end):
        lat.step(1)
        o.step(1)
        for first, f in ((first_g, lat.fields()["solid"]), (first_o, o.fields()["solid"])):
            new = solid0 & ~f & (first < 0)
            first[new] = s
    conv = first_o > 0
    assert conv.sum() >= 1, conv.sum()
    tol = 1 if precision == "fp64" else max(1, int(1e-4 * first_o[conv].max()))
    conv_g = first_g > 0
    both = conv & conv_g
    d = np.abs(first_g[both] - first_o[both])
    with capsys.disabled():
        print(f"\nconfig 2 conversion, {precision}: {conv.sum()} cells from step {first_o[conv].min()}, "
              f"max |step difference| {d.max()}")
    assert d.max() <= tol
    edge = end - tol                 # a cell converting this close to the window's end may fall outside it
    assert np.all(conv_g[conv & (first_o < edge)]) and np.all(conv[conv_g & (first_g < edge)])
    lat.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16"])
def test_config3_parameters_64cubed(oracle_mod, precision):
    n = 400
    w = workloads.pyro3d(64, seed=0, precision=precision)
    g = _gpu(w, n)
    r64 = _oracle(oracle_mod, w, n, "f64")
    fl = ~r64["solid"]
    if precision == "fp64":
        assert np.array_equal(g["solid"], r64["solid"])
        assert _rel(g["rho"][fl], r64["rho"][fl]) < 1e-10
        assert _rel(g["u"][:, fl], r64["u"][:, fl]) < 1e-10
        assert _rel(g["T"], r64["T"]) < 1e-10
    elif precision == "fp32":
        r32 = _oracle(oracle_mod, w, n, "f32")
        assert _rel(g["rho"][fl], r32["rho"][fl]) < 1e-5
        assert _rel(g["T"], r32["T"]) < 1e-5
    else:
        e_u = _rel(g["u"][:, fl], r64["u"][:, fl])
        print(f"config 3 at 64^3, 400 steps, FP16 storage: u relL2 vs FP64 {e_u:.3e}")   # 2.4e-3
        assert _rel(g["rho"][fl], r64["rho"][fl]) < 1e-3
        assert _rel(g["T"], r64["T"]) < 1e-2
        assert e_u < 1e-2
