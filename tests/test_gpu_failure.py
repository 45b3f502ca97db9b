"""Failure detection without a GPU fault: the non-finite detector of the diagnostics.

A NaN enters through the host-side input of lbm_init_equilibrium (the initial density of
one fluid cell); the next step's diagnostics count it and lbm_read_diag returns
LBM_ERR_NONFINITE, while the device stays usable.  (The bounded-wait timeout of the dense
bulk form is tested in test_gpu_dense.py.)
"""
import ctypes

import numpy as np
import pytest

from lbm_porouschem_b200 import _native as N
from lbm_porouschem_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["tile", "list"])
def test_nan_in_initial_fields_is_reported(form):
    from lbm_porouschem_b200.lattice import Lattice
    w = workloads.pyro3d(64, seed=3, ny=16, nz=12)
    lat = Lattice(w.cfg.replace(bulk_form=form))
    lat.set_geometry(w.solid, w.reactive)
    rho = np.ones(w.cfg.shape)
    fluid = np.argwhere(~w.solid)
    rho[tuple(fluid[len(fluid) // 2])] = np.nan
    lat.init(rho=rho, u=(0.0, 0.0, 0.0), T=0.0)
    lat.step(2, diag=True)
    d = N.lbm_diag()
    rc = lat.lib.lbm_read_diag(lat._h, ctypes.byref(d), lat._s())
    assert rc == N.LBM_ERR_NONFINITE
    assert d.nonfinite >= 1
    assert lat.read_diag()["nonfinite"] >= 1       # the Python layer reports it too
    lat.close()
    # a fresh lattice on the same device runs clean
    ok = Lattice(w.cfg.replace(bulk_form=form))
    ok.set_geometry(w.solid, w.reactive)
    ok.init(rho=1.0, u=(0.0, 0.0, 0.0), T=0.0)
    ok.step(2, diag=True)
    assert ok.read_diag()["nonfinite"] == 0
    ok.close()


def test_async_diag_equals_sync_and_reports_nonfinite():
    """lbm_read_diag_async: the values equal lbm_read_diag's for the same step, two reads may be
    in flight while later steps run, and a NaN shows as nonfinite > 0."""
    from lbm_porouschem_b200.lattice import Lattice
    w = workloads.pyro3d(64, seed=3, ny=16, nz=12)
    lat = Lattice(w.cfg.replace(bulk_form="list"))
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    lat.step(3, diag=True)
    a = lat.read_diag_async()
    lat.step(1, diag=True)
    b = lat.read_diag_async()
    ra, rb = a.result(), b.result()
    assert rb == lat.read_diag() and ra["step"] == 3 and rb["step"] == 4
    assert ra["mass"] != rb["mass"]
    lat.close()
    rho = np.ones(w.cfg.shape)
    rho[tuple(np.argwhere(~w.solid)[0])] = np.nan
    bad = Lattice(w.cfg.replace(bulk_form="list"))
    bad.set_geometry(w.solid, w.reactive)
    bad.init(rho=rho, u=(0.0, 0.0, 0.0), T=0.0)
    bad.step(2, diag=True)
    assert bad.read_diag_async().result()["nonfinite"] >= 1
    bad.close()
