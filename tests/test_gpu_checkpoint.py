"""Checkpoint / resume (Lattice.save_checkpoint, Lattice.load_checkpoint -> lbm_resume,
the solver's export_snapshot / load_snapshot and the YAML driver's timeControl.restart).

A run that is saved and continued in a new lattice must give the same fields, bit for bit,
as the run that went on: the saved state is exactly what the next step reads.  The resumed
lattice lists its cells afresh (cells that turned fluid are no longer at the end of the
fluid list), so FP64 diagnostic sums may differ in the last bits: 1e-12."""
import numpy as np
import pytest
import yaml

from lbm_porouschem_b200 import workloads

pytestmark = pytest.mark.gpu


def _fast_pyro(w):
    w.cfg.pyro_A = 1.2e11
    w.cfg.heat_norm = 0.02
    w.cfg.gas_coef = 0.05
    w.init["T"] = 1.0
    return w


def _same(a, b):
    for k in ("rho", "u", "T", "alpha", "solid"):
        if k in a:
            assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("precision", ["fp32", "fp16", "fp64"])
@pytest.mark.parametrize("bulk", ["list", "tile"])
def test_resume_continues_bit_for_bit(precision, bulk, tmp_path, monkeypatch):
    from lbm_porouschem_b200.lattice import Lattice
    monkeypatch.setenv("LBM_BULK", bulk)
    w = _fast_pyro(workloads.pyro3d(40, seed=21, ny=24, nz=20, precision=precision, collision="mrt"))
    lat = Lattice(w.cfg)
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    lat.step(45, residual=True)                # odd: the checkpoint reads the second half
    path = lat.save_checkpoint(tmp_path / "ck.npz")
    lat.step(40, residual=True)
    ref, dref = lat.fields(), lat.diagnostics()
    lat.close()

    back = Lattice.load_checkpoint(path)
    assert back.nsteps == 45 and back.bulk_kernel == bulk
    back.step(40, residual=True)
    got, dgot = back.fields(), back.diagnostics()
    assert back.nsteps == 85
    back.close()
    assert (w.solid & ~got["solid"]).any()   # cells turned fluid, some of them after the checkpoint
    _same(got, ref)
    for k in ("mass", "energy", "solid_alpha", "nfluid", "res_num", "res_den"):
        assert dgot[k] == pytest.approx(dref[k], rel=1e-12), k
    assert dgot["umax"] == dref["umax"]


def test_checkpoint_refuses_a_foreign_file(tmp_path):
    from lbm_porouschem_b200.lattice import Lattice
    p = tmp_path / "x.npz"
    np.savez(p, meta=np.frombuffer(b'{"format": "other"}', dtype=np.uint8))
    with pytest.raises(ValueError, match="not an lbm_b200 checkpoint"):
        Lattice.load_checkpoint(p)


def test_yaml_restart_reproduces_the_run(tmp_path, monkeypatch):
    """The YAML driver with snapshots every 10 steps; a second run restarts from the step-10
    snapshot and writes the same step-20 VTK file as the uninterrupted run."""
    from lbm_porouschem_b200.cli import run
    from lbm_porouschem_b200.vtk import read_vts
    from tests.test_app import CASE2D
    monkeypatch.chdir(tmp_path)
    cfg = yaml.safe_load(CASE2D)
    cfg["outputControl"]["vtk"] = {"interval": 1.0e-3, "path": str(tmp_path / "a")}
    cfg["outputControl"]["snapshot"] = {"interval": 1.0e-3, "path": str(tmp_path / "snap" / "s")}
    (tmp_path / "a.yaml").write_text(yaml.safe_dump(cfg))
    assert run(["-c", str(tmp_path / "a.yaml"), "-v", "0"]) == 0
    assert (tmp_path / "snap" / "s_10.npz").exists()
    cfg["outputControl"]["vtk"]["path"] = str(tmp_path / "b")
    cfg["outputControl"].pop("snapshot")
    cfg["timeControl"]["restart"] = str(tmp_path / "snap" / "s_10.npz")
    (tmp_path / "b.yaml").write_text(yaml.safe_dump(cfg))
    assert run(["-c", str(tmp_path / "b.yaml"), "-v", "0"]) == 0
    name = cfg["basic"]["name"]
    a = read_vts(str(tmp_path / "a" / f"{name}_20.vts"))
    b = read_vts(str(tmp_path / "b" / f"{name}_20.vts"))
    for k in ("rho", "velocity", "solid", "Tf"):
        assert np.array_equal(a[k], b[k]), k
    assert not (tmp_path / "b" / f"{name}_0.vts").exists()   # the restart began at step 10
