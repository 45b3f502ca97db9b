"""Reference-shaped solver surface: setter -> lattice configuration mapping (CPU) and
stepping through the CUDA path (GPU)."""
import numpy as np
import pytest

from lbm_porouschem_b200 import LatticeConfig, SideBC
from lbm_porouschem_b200.config import FIXED_VALUE, FLOW_RATE, PERIODIC, ZERO_GRADIENT
from lbm_porouschem_b200.flag import BC, BC_FLOW, BC_MODEL
from lbm_porouschem_b200.solver import LBM2DSolver, LBM3DSolver


def _channel2d():
    s = LBM2DSolver(X=0.064, Y=0.032, Z=0.0, dx=1e-3, dt=1e-4, name="channel", isThermal=True)
    s.set_viscosity(2e-5)
    s.set_fluid_Trange([300.0, 800.0])
    s.set_solid_Trange([300.0, 800.0])
    s.set_fluid_thermal_diff(3e-5)
    s.set_solid_thermal_diff(1e-5)
    s.set_BC(0, BC_FLOW.inlet)
    s.set_BC(1, BC_FLOW.outlet)
    s.set_BC(2, BC_FLOW.wall)
    s.set_BC(3, BC_FLOW.wall)
    s.set_v_BC_value(0, [0.01, 0.0])
    s.set_rho_BC_value(1, 1.0)
    s.set_TF_BC(0, BC.fixedValue)
    s.set_TF_BC_value(0, 800.0)
    s.set_TF_BC(1, BC.zeroGradient)
    return s


def test_grid_from_physical_size():
    s = LBM3DSolver(X=0.02, Y=0.01, Z=0.005, dx=1e-3)
    assert (s.nx, s.ny, s.nz) == (20, 10, 5)
    s2 = LBM2DSolver(X=64, Y=32, Z=0)
    assert (s2.nx, s2.ny, s2.nz) == (64, 32, 1)


def test_setters_map_to_lattice_config():
    s = _channel2d()
    cfg = s._config()
    assert isinstance(cfg, LatticeConfig)
    assert (cfg.dim, cfg.nx, cfg.ny, cfg.nz) == (2, 64, 32, 1)
    assert cfg.nu == pytest.approx(2e-5 * 1e-4 / 1e-6)             # visco dt / dx^2
    assert cfg.tau() == pytest.approx(3 * cfg.nu + 0.5)
    assert cfg.thermal == "two_field"                                  # the reference's TF / TS
    # D2Q5: tau = 3 D + 1/2 with D = diff dt / dx^2 (src/LBM/LBM2D/_scalarField.py tau)
    assert cfg.tauT_fluid == pytest.approx(3 * 3e-5 * 1e-4 / 1e-6 + 0.5)
    assert cfg.tauT_solid == pytest.approx(3 * 1e-5 * 1e-4 / 1e-6 + 0.5)
    assert (cfg.T_ref, cfg.T_scale) == (300.0, 500.0)
    sd = cfg.sides
    assert sd[0].active and sd[0].v_type == FIXED_VALUE and sd[0].rho_type == ZERO_GRADIENT
    assert sd[0].v == (0.01, 0.0, 0.0)
    assert sd[0].T_type == FIXED_VALUE and sd[0].T == pytest.approx(1.0)   # (800 - 300) / 500
    assert sd[1].active and sd[1].v_type == ZERO_GRADIENT and sd[1].rho_type == FIXED_VALUE
    assert sd[1].T_type == ZERO_GRADIENT
    assert sd[2].active and sd[2].v == (0.0, 0.0, 0.0) and sd[2].v_type == FIXED_VALUE
    assert not sd[4].active and not sd[5].active                       # 2D: no z sides


def test_3d_thermal_tau_and_periodic_sides():
    s = LBM3DSolver(X=16, Y=8, Z=8, dx=1, dt=1, isThermal=True)
    s.set_viscosity(0.1)
    s.set_fluid_thermal_diff(0.05)
    s.set_solid_thermal_diff(0.1)
    s.set_BC(0, BC_FLOW.inlet)
    s.set_v_BC_value(0, [0.02, 0.0, 0.0])
    cfg = s._config()
    assert cfg.tauT_fluid == pytest.approx(4 * 0.05 + 0.5)              # D3Q7: 4 D + 1/2
    assert cfg.tauT_solid == pytest.approx(4 * 0.1 + 0.5)
    assert [x.active for x in cfg.sides] == [True, False, False, False, False, False]
    s.ref_quirk_nee_on_periodic = True                                 # reference applies NEE on all sides
    assert all(x.active for x in s._config().sides)
    s.boundary_condition_model = BC_MODEL.NONE
    assert not any(x.active for x in s._config().sides)


def test_prandtl_and_pyrolysis_mapping():
    s = LBM3DSolver(X=0.008, Y=0.008, Z=0.008, dx=1e-3, dt=1e-4, isThermal=True)
    s.set_viscosity(2e-5)
    s.set_fluid_Prandtl(0.7)
    assert s._config().tauT_fluid == pytest.approx(4 * (2e-5 * 1e-4 / 1e-6) / 0.7 + 0.5)
    s.set_fluid_Trange([300.0, 800.0])
    s.set_pyrolysis(A=1e8, Ea=1.25e5, dH=4e5, capacity=1000.0, char_yield=0.25, alpha_flip=0.02)
    cfg = s._config()
    assert cfg.pyro and cfg.pyro_A == 1e8 and cfg.pyro_Ea == 1.25e5 and cfg.dt_phys == 1e-4
    assert cfg.heat_norm == pytest.approx(4e5 / (1000.0 * 500.0))
    assert cfg.gas_coef == pytest.approx(0.75) and cfg.alpha_flip == 0.02
    with pytest.raises(ValueError):
        LBM2DSolver(X=8, Y=8, Z=0).set_pyrolysis()                    # needs the temperature field


def test_unsupported_features_raise():
    s = LBM2DSolver(X=8, Y=8, Z=0)
    with pytest.raises(NotImplementedError):
        s.load_cantera("gri30.yaml")
    s.boundary_condition_model = BC_MODEL.NEBB
    s.set_BC(0, BC_FLOW.outlet)
    sd = s._config().sides                              # NEBB in 2D without temperature
    assert sd[0].model == "nebb" and sd[0].code() == 3 and sd[2].code() == 0
    s3 = LBM3DSolver(X=8, Y=8, Z=8)
    s3.boundary_condition_model = BC_MODEL.NEBB        # the 3D solver has no NEBB
    s3.set_BC(0, BC_FLOW.outlet)
    with pytest.raises(NotImplementedError):
        s3._config()
    st = LBM2DSolver(X=8, Y=8, Z=0, isThermal=True)
    st.boundary_condition_model = BC_MODEL.NEBB        # its scalar boundary reads last step's fields
    st.set_BC(0, BC_FLOW.outlet)
    with pytest.raises(NotImplementedError):
        st._config()
    s.boundary_condition_model = BC_MODEL.ES            # the equilibrium scheme is on the path
    sd = s._config().sides
    assert sd[0].active and sd[0].model == "es" and sd[0].code() == 2 and sd[2].code() == 0


def test_flowrate_inlet_mapping():
    """BC_FLOW.inlet_flow: side 0 steered each step in 2D (LBM_BC_FLOWRATE, target in
    v[0]), the uniform v0 = F/ny/nz in 3D, zero velocity on any other side (the
    reference sets an inlet profile for side 0 only)."""
    s = LBM2DSolver(X=16, Y=8, Z=0)
    s.set_BC(0, BC_FLOW.inlet_flow)
    s.set_flow_BC_value(0, 0.4)
    s.set_BC(1, BC_FLOW.outlet)
    s.set_rho_BC_value(1, 1.0)
    sd = s._config().sides
    assert sd[0].active and sd[0].v_type == FLOW_RATE and sd[0].rho_type == ZERO_GRADIENT
    assert sd[0].v == (0.4, 0.0, 0.0)
    s3 = LBM3DSolver(X=8, Y=4, Z=5)
    for i in (0, 1):
        s3.set_BC(i, BC_FLOW.inlet_flow)
        s3.set_flow_BC_value(i, 0.4)
    sd = s3._config().sides
    assert sd[0].v_type == FIXED_VALUE and sd[0].v == pytest.approx((0.4 / 4 / 5, 0.0, 0.0))
    assert sd[1].v_type == FIXED_VALUE and sd[1].v == (0.0, 0.0, 0.0)


def test_sutherland_viscosity_mapping():
    """set_viscosity_sutherland (src/LBM/LBM2D/_io.py:144-147): with the temperature field
    the lattice takes As dt/dx^2 and Ts; without it the reference evaluates the law at
    273.15 K (GetTF, _evolution.py:304-307), a constant viscosity."""
    s = _channel2d()
    s.set_viscosity_sutherland(1.6e-6, 170.0)
    c = s._config()
    assert c.viscosity == "sutherland" and c.suth_Ts == 170.0
    assert c.suth_A == pytest.approx(1.6e-6 * 1e-4 / 1e-6)
    d = c.to_desc()
    assert d.viscosity == 1 and d.suth_A == pytest.approx(1.6e-4)
    s2 = LBM2DSolver(X=8, Y=8, Z=0, dx=1e-3, dt=1e-4)
    s2.set_viscosity_sutherland(1.6e-6, 170.0)
    c2 = s2._config()
    assert c2.viscosity == "constant"
    assert c2.nu == pytest.approx(1.6e-6 * 273.15 ** 1.5 / (273.15 + 170.0) * 1e-4 / 1e-6)


def test_init_field_forms(tmp_path):
    s = LBM2DSolver(X=6, Y=4, Z=0)
    s.init_field(s.rho, 1.02)
    assert np.all(s.rho.to_numpy() == 1.02)
    a = np.arange(24, dtype=np.float64).reshape(6, 4, 1)
    p = tmp_path / "rho.txt"
    np.savetxt(p, a.flatten(order="F"))
    s.init_field(s.rho, str(p))
    assert np.array_equal(s.rho.to_numpy(), a)
    s.init_field3(s.v, 0.01, a, 0.0)
    v = s.v.to_numpy()
    assert v.shape == (6, 4, 1, 3) and np.all(v[..., 0] == 0.01) and np.array_equal(v[..., 1], a)
    s.add_solid(np.ones((6, 4, 1)) * (a > 20))
    assert s.solid.to_numpy().sum() == 3
    assert "6 x 4 x 1" in s.description()
    assert "t(LU)=0" in s.log_info()


@pytest.mark.gpu
def test_solver_steps_like_lattice():
    """The solver is a thin front: stepping it equals stepping a Lattice configured directly."""
    from lbm_porouschem_b200 import Lattice
    s = _channel2d()
    rng = np.random.default_rng(3)
    solid = np.zeros((64, 32, 1))
    solid[20:28, 10:18] = 1.0
    s.add_solid(solid)
    T0 = 300.0 + 100.0 * rng.random((64, 32, 1))
    s.init_field(s.TF.S, (T0 - 300.0) / 500.0)
    s.init_field(s.TS.S, (T0 - 300.0) / 500.0)   # the driver sets both (src/LBM/app.py:503-509)
    s.init_field(s.rho, 1.0)
    s.init_simulation()
    for _ in range(50):
        s.step()
    got = {"rho": s.rho.to_numpy(), "v": s.v.to_numpy(), "T": s.TF.S.to_numpy()}

    cfg = LatticeConfig(dim=2, nx=64, ny=32, nz=1, nu=2e-5 * 1e-4 / 1e-6, thermal="two_field",
                        tauT_fluid=3 * 3e-5 * 1e-4 / 1e-6 + 0.5, tauT_solid=3 * 1e-5 * 1e-4 / 1e-6 + 0.5,
                        T_ref=300.0, T_scale=500.0,
                        sides=[SideBC.inlet((0.01, 0.0, 0.0), FIXED_VALUE, 1.0),
                               SideBC.outlet(1.0, ZERO_GRADIENT, 0.0),
                               SideBC.wall(PERIODIC), SideBC.wall(PERIODIC), SideBC(), SideBC()])
    lat = Lattice(cfg)
    lat.set_geometry(solid >= 1)
    lat.init(rho=1.0, u=(0.0, 0.0, 0.0), T=(T0 - 300.0) / 500.0)
    lat.step(50)
    ref = lat.fields()
    fl = ~ref["solid"]
    np.testing.assert_array_equal(got["rho"][fl], ref["rho"][fl])
    np.testing.assert_array_equal(got["v"][fl], np.moveaxis(ref["u"], 0, -1)[fl])
    np.testing.assert_array_equal(got["T"], ref["T"])
    assert s.tLattice == 50 and s.t == pytest.approx(50 * 1e-4)
    assert "Max velocity magnitude" in s.log_info()
    s.close()
    lat.close()


def test_reference_surface_is_complete():
    """Every method and attribute the reference's driver touches exists (src/LBM/app.py:
    101-677); those outside the CUDA path raise NotImplementedError naming themselves."""
    s = LBM3DSolver(X=8, Y=8, Z=8, dx=1, isThermal=True)
    for n in ("set_fluid_conductivity_mixture", "set_solid_capacity_mixture",
              "set_specie_diff", "set_specie_BC", "set_species_BC", "init_specie", "set_radiation"):
        with pytest.raises(NotImplementedError, match=n if n != "set_radiation" else "radiation"):
            getattr(s, n)(*([None] * (2 if n == "set_radiation" else 1)))
    assert s.specieName == [] and s.TS.radiation_surface is not None and s.TS.emissivity is not None


def test_derived_thermal_diffusivity():
    """D = cond / (rho cm) with constant conductivity and capacity (src/LBM/LBM2D/_thermal.py:62-107):
    fluid at rho0 = 1, solid at its (uniform) density."""
    s = LBM2DSolver(X=0.016, Y=0.008, Z=0, dx=1e-3, dt=1e-4, isThermal=True)
    s.set_viscosity(2e-5)
    solid = np.zeros((16, 8, 1))
    solid[6:10, 2:6] = 1.0
    s.add_solid(solid)
    s.add_rho_solid(solid * 500.0)
    s.set_fluid_thermal_diff_derived()
    s.set_fluid_conductivity(0.03)
    s.set_fluid_capacity(1000.0)
    s.set_solid_thermal_diff_derived()
    s.set_solid_conductivity(0.5)
    s.set_solid_capacity(1500.0)
    cfg = s._config()
    lu = 1e-4 / 1e-6
    assert cfg.tauT_fluid == pytest.approx(3 * (0.03 / 1000.0) * lu + 0.5)
    assert cfg.tauT_solid == pytest.approx(3 * (0.5 / (500.0 * 1500.0)) * lu + 0.5)
    s.add_rho_solid(solid * np.linspace(0, 1, 16)[:, None, None])     # no longer uniform
    with pytest.raises(NotImplementedError, match="solid density"):
        s._config()


def test_temperature_dependent_properties_map_to_tprop():
    """Polynomial conductivity and NASA7 / polynomial capacity under the derived model
    (src/LBM/LBM2D/_io.py:182-251) become the descriptor's per-cell property sets, in the
    reference's nested coefficient form; a later constant setter replaces the model."""
    from lbm_porouschem_b200.config import GAS_CONSTANT
    s = LBM2DSolver(X=0.016, Y=0.008, Z=0, dx=1e-3, dt=1e-4, isThermal=True)
    s.set_viscosity(2e-5)
    solid = np.zeros((16, 8, 1))
    solid[6:10, 2:6] = 1.0
    s.add_solid(solid)
    s.add_rho_solid(solid * 500.0)
    s.set_fluid_Trange([300.0, 800.0])
    s.set_fluid_thermal_diff_derived()
    s.set_fluid_conductivity_poly([0.02, 1e-4, 0, 0, 0])
    s.set_fluid_capacity_NASA7([200.0, 1000.0, 3500.0], [[3.5, 1e-4, 0, 0, 0, 0, 0], [3.0, 2e-4, 0, 0, 0, 0, 0]])
    s.set_solid_thermal_diff_derived()
    s.set_solid_conductivity_poly([0.5, 1e-3, 0, 2e-9, 7.0])
    s.set_solid_capacity_poly([1500.0, 0.1, 0, 0, 0])
    cfg = s._config()
    f, so = cfg.tprop_fluid, cfg.tprop_solid
    assert f["cond"] == [0.02, 1e-4, 0.0, 0.0, 0.0] and f["cap_Tmid"] == 1000.0 and f["cap_mul"] == GAS_CONSTANT
    assert f["cap_lo"][0] == 3.5 and f["cap_hi"][0] == 3.0
    assert so["cond"] == [0.5, 1e-3, 0.0, 2e-9, 0.0]      # the solid's conductivity uses four coefficients
    assert so["cap_lo"] == so["cap_hi"] == [1500.0, 0.1, 0.0, 0.0, 0.0] and so["cap_mul"] == 1.0
    assert cfg.tp_rhos == 500.0 and cfg.tp_dt == 1e-4 and cfg.tp_dx2 == pytest.approx(1e-6)
    d = cfg.to_desc()
    assert d.tprop == 3 and d.tp_cap_mul[0] == GAS_CONSTANT and d.tp_cond[1][3] == 2e-9
    s.set_fluid_capacity(1000.0)
    assert s._config().tprop_fluid["cap_lo"] == [1000.0, 0.0, 0.0, 0.0, 0.0]
    s.set_fluid_thermal_diff(3e-5)           # back to the constant model: no per-cell fluid rate
    assert s._config().tprop_fluid is None


def test_temperature_dependent_properties_refused_with_porous_cells():
    s = LBM2DSolver(X=0.016, Y=0.008, Z=0, dx=1e-3, dt=1e-4, isThermal=True, isPoro=True)
    s.set_viscosity(2e-5)
    frac = np.zeros((16, 8, 1))
    frac[6:10, 2:6] = 0.5
    s.add_solid(frac)
    s.set_fluid_thermal_diff_derived()
    s.set_fluid_conductivity_poly([0.02, 1e-4, 0, 0, 0])
    s.set_fluid_capacity(1000.0)
    with pytest.raises(NotImplementedError, match="porous"):
        s._config()
