"""The C-ABI library loads on a CPU-only host, exports every symbol the header
declares, agrees with the header on struct layouts, and validates descriptors
(no GPU work is issued by any of these calls)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from lbm_porouschem_b200 import _native as N
from lbm_porouschem_b200.config import LatticeConfig, SideBC, thermal_props

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "lbm_b200.h"
HEADERS = sorted((ROOT / "include").glob("*.h"))


@pytest.fixture(scope="module")
def lib():
    from lbm_porouschem_b200 import _build
    _build.build()
    return N.load()


def _declared():
    txt = "\n".join(h.read_text() for h in HEADERS)
    return sorted(set(re.findall(r"LBM_API\s+[\w\s\*]+?\b(lbm_\w+)\s*\(", txt)))


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 12
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (lbm_\w+)", out))
    for n in names:
        assert n in exported, n
        assert hasattr(lib, n)
    assert set(N.EXPORTED) <= set(names)


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "lbm_b200.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(lbm_desc), sizeof(lbm_side_desc),'
                   ' sizeof(lbm_diag), offsetof(lbm_desc, side), offsetof(lbm_desc, mrt_s)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", "-o", str(exe), str(src)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    assert got == [ctypes.sizeof(N.lbm_desc), ctypes.sizeof(N.lbm_side_desc), ctypes.sizeof(N.lbm_diag),
                   N.lbm_desc.side.offset, N.lbm_desc.mrt_s.offset]


def test_required_bytes(lib):
    cfg = LatticeConfig(dim=3, nx=32, ny=16, nz=8, thermal="conjugate", pyro=True)
    d = cfg.to_desc()
    nb = ctypes.c_size_t()
    n = 32 * 16 * 8
    N.check(lib.lbm_required_bytes(ctypes.byref(d), N.LBM_FIELD_F, ctypes.byref(nb)))
    assert nb.value == 2 * 19 * n * 4
    N.check(lib.lbm_required_bytes(ctypes.byref(d), N.LBM_FIELD_G, ctypes.byref(nb)))
    assert nb.value == 2 * 7 * n * 4
    N.check(lib.lbm_required_bytes(ctypes.byref(d), N.LBM_FIELD_MASK, ctypes.byref(nb)))
    assert nb.value == n
    d16 = cfg.replace(precision="fp16").to_desc()
    N.check(lib.lbm_required_bytes(ctypes.byref(d16), N.LBM_FIELD_F, ctypes.byref(nb)))
    assert nb.value == 2 * 19 * n * 2


_TP = thermal_props(cond=0.5, cap=10.0)


@pytest.mark.parametrize("bad", [
    dict(dim=4), dict(nx=2), dict(nz=5), dict(thermal="none", pyro=True), dict(nu=0.0),
    dict(tauT_fluid=0.4, thermal="conjugate"),
    dict(tprop_fluid=_TP), dict(tprop_solid=_TP, thermal="conjugate", tp_rhos=0.0),
    dict(tprop_fluid=_TP, thermal="two_field", porous="darcy"), dict(tprop_fluid=_TP, thermal="conjugate", tp_dt=0.0),
    dict(tprop_fluid={**_TP, "cap_mul": 0.0}, thermal="conjugate"), dict(tp_prandtl=0.7),
])
def test_descriptor_validation(lib, bad):
    kw = dict(dim=2, nx=16, ny=8, nz=1)
    kw.update(bad)
    cfg = LatticeConfig(**kw)
    d = cfg.to_desc()
    d.nz = kw["nz"] if "nz" in bad else d.nz
    h = ctypes.c_void_p()
    rc = lib.lbm_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == N.LBM_ERR_ARG
    assert lib.lbm_last_error().decode()


def test_struct_size_guard(lib):
    d = LatticeConfig(dim=2, nx=16, ny=8).to_desc()
    d.struct_size = 12
    h = ctypes.c_void_p()
    assert lib.lbm_create(ctypes.byref(d), ctypes.byref(h)) == N.LBM_ERR_ARG
    assert b"struct_size" in lib.lbm_last_error()


def test_bind_checks_size_and_alignment(lib):
    cfg = LatticeConfig(dim=2, nx=16, ny=8)
    d = cfg.to_desc()
    h = ctypes.c_void_p()
    N.check(lib.lbm_create(ctypes.byref(d), ctypes.byref(h)))
    try:
        assert lib.lbm_bind(h, N.LBM_FIELD_MASK, ctypes.c_void_p(4096), 10) == N.LBM_ERR_ARG
        assert lib.lbm_bind(h, N.LBM_FIELD_MASK, ctypes.c_void_p(4097), 1 << 20) == N.LBM_ERR_ARG
        assert lib.lbm_bind(h, 99, ctypes.c_void_p(4096), 1 << 20) == N.LBM_ERR_ARG
        # stepping without bound buffers fails before any launch
        assert lib.lbm_step(h, 1, 0, None) == N.LBM_ERR_UNBOUND
        assert lib.lbm_step_count(h) == 0
    finally:
        lib.lbm_destroy(h)


def test_set_sides_rejects_type_change(lib):
    sides = [SideBC.pressure(1.001), SideBC.outlet(1.0)] + [SideBC() for _ in range(4)]
    cfg = LatticeConfig(dim=2, nx=16, ny=8, sides=sides)
    d = cfg.to_desc()
    h = ctypes.c_void_p()
    N.check(lib.lbm_create(ctypes.byref(d), ctypes.byref(h)))
    try:
        # scratch unbound -> refused before any copy
        arr = (N.lbm_side_desc * 6)()
        assert lib.lbm_set_sides(h, arr, None) == N.LBM_ERR_UNBOUND
    finally:
        lib.lbm_destroy(h)
