"""FP16 deviation storage against FP64, both on the GPU.

FP16 storage keeps f_k - w_k rho0 and g_k - wt_k T0 in half precision with FP32
arithmetic.  This module runs the same seeded cases in FP16 and FP64 and states the
error of the FP16 form in the four quantities that decide a porous-media result:
velocity, temperature, permeability and the position of the conversion front.  The
FP64 kernels are the reference (they match the FP64 CPU oracle to 1e-10).

- ``front_case``: a pyrolysis channel (pyro2d: pressure-driven flow through a disk
  packing, hot inlet T = 1, cold start T = 0, every disk reactive; A = 1e12 /s and a weak
  heat sink, so that disks convert where the heat from the inlet brings them above
  T ~ 0.65 and the conversion front follows that isotherm into the packing).  After
  ``steps`` steps: relative L2 errors
  of u (fluid cells) and T (all cells), the largest reactive-fraction difference, the
  number of cells whose solid state differs, and the front position (the first x from
  the inlet where the column mean of the conversion 1 - alpha over reactive cells
  falls below 1/2, interpolated) in cells.
- ``permeability_case``: body-force flow through a periodic disk packing (flow2d):
  Darcy permeability k = nu <u_x> / g_x over every cell (superficial velocity) after
  ``steps`` steps, relative difference.

- ``config3_case``: the 3D packing at 256^3 with its own parameters (D3Q19 MRT + D3Q7
  conjugate heat + pyrolysis, A = 1e8 /s, heat 0.8, pressure inlet/outlet on x, periodic
  y/z) for 20,000 steps from identical inputs in FP32, FP16 deviation storage and FP64:
  relative L2 errors of rho, u (fluid cells) and T (all cells) against FP64, cells whose
  solid state differs, and each run's lattice updates per second.

``python -m lbm_porouschem_b200.accuracy`` prints the first two as one JSON object;
``--config3 [--n N] [--steps S]`` prints the third.
"""
from __future__ import annotations

import json

import numpy as np

from . import workloads


def _rel(a, b) -> float:
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


def front_position(alpha: np.ndarray, reactive: np.ndarray) -> float:
    """First x (cells) from the inlet where the column mean of 1 - alpha over reactive
    cells drops below 1/2, linearly interpolated; nx if it never does."""
    a = alpha.reshape(reactive.shape[0], -1)
    r = reactive.reshape(reactive.shape[0], -1)
    cnt = r.sum(1)
    conv = np.where(cnt > 0, ((1.0 - a) * r).sum(1) / np.maximum(cnt, 1), np.nan)
    xs = np.flatnonzero(~np.isnan(conv))
    prev_x, prev_c = None, None
    for x in xs:
        c = conv[x]
        if c < 0.5:
            if prev_x is None:
                return float(x)
            return float(prev_x + (prev_c - 0.5) / (prev_c - c) * (x - prev_x))
        prev_x, prev_c = x, c
    return float(reactive.shape[0])


def _run(w, precision: str, steps: int, **cfg_kw):
    from .lattice import Lattice
    cfg = w.cfg.replace(precision=precision, **cfg_kw)
    lat = Lattice(cfg)
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    lat.step(steps)
    out = lat.fields()
    lat.close()
    return out


def front_case(nx: int = 256, ny: int = 64, seed: int = 5, steps: int = 4000, pyro_A: float = 1e12) -> dict:
    w = workloads.pyro2d(nx, ny, seed=seed)
    kw = dict(pyro_A=pyro_A, heat_norm=0.02, gas_coef=0.05, T0=0.5)
    a = _run(w, "fp16", steps, **kw)
    b = _run(w, "fp64", steps, **kw)
    fl = ~a["solid"] & ~b["solid"]
    react = w.reactive.reshape(a["alpha"].shape)
    xa, xb = front_position(a["alpha"], react), front_position(b["alpha"], react)
    return {"case": f"pyro2d {nx}x{ny} seed {seed}, A {pyro_A:g}/s, {steps} steps",
            "u_rel_l2": _rel(a["u"][:, fl], b["u"][:, fl]),
            "u_max_fp64": float(np.sqrt((b["u"][:, fl] ** 2).sum(0)).max()),
            "T_rel_l2": _rel(a["T"], b["T"]),
            "alpha_max_abs": float(np.abs(a["alpha"] - b["alpha"])[react].max()),
            "solid_cells_differing": int((a["solid"] != b["solid"]).sum()),
            "cells_converted_fp64": int((react & ~b["solid"]).sum()),
            "front_x_fp16": xa, "front_x_fp64": xb, "front_dx_cells": abs(xa - xb)}


def permeability_case(nx: int = 128, ny: int = 64, seed: int = 2, steps: int = 8000, g: float = 1e-5) -> dict:
    w = workloads.flow2d(nx, ny, seed=seed)
    kw = dict(force=(g, 0.0, 0.0), half_force_velocity=True)
    nu = w.cfg.nu
    ks = {}
    us = {}
    for prec in ("fp16", "fp64"):
        f = _run(w, prec, steps, **kw)
        us[prec] = f
        ks[prec] = nu * float(np.mean(np.where(f["solid"], 0.0, f["u"][0]))) / g
    fl = ~us["fp64"]["solid"]
    return {"case": f"flow2d {nx}x{ny} seed {seed}, g {g:g}, {steps} steps",
            "k_fp16": ks["fp16"], "k_fp64": ks["fp64"],
            "k_rel_diff": abs(ks["fp16"] - ks["fp64"]) / abs(ks["fp64"]),
            "u_rel_l2": _rel(us["fp16"]["u"][:, fl], us["fp64"]["u"][:, fl])}


def config3_case(n: int = 256, steps: int = 20000, seed: int = 0, T0: float | None = None,
                 precisions: tuple = ("fp32", "fp16")) -> dict:
    """``T0``: the FP16 temperature shift (None: the workload's)."""
    import time

    import torch

    from .lattice import Lattice
    w = workloads.pyro3d(n, seed=seed)
    if T0 is not None:
        w.cfg.T0 = T0
    out, rates = {}, {}
    for prec in ("fp64",) + tuple(precisions):
        # "fp16-nearest": FP16 storage with the temperature populations rounded to nearest
        kw = dict(precision="fp16", fp16_rounding="nearest") if prec == "fp16-nearest" else dict(precision=prec)
        lat = Lattice(w.cfg.replace(**kw))
        lat.set_geometry(w.solid, w.reactive)
        lat.init(**w.init)
        lat.step(10)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lat.step(steps - 10)
        torch.cuda.synchronize()
        rates[prec] = w.cfg.ncells * (steps - 10) / (time.perf_counter() - t0) / 1e6
        out[prec] = lat.fields()
        lat.close()
    ref = out["fp64"]
    res = {"case": f"pyro3d {n}^3 seed {seed}, {steps} steps, identical inputs, FP16 shifts rho0 "
                   f"{w.cfg.rho0:g} T0 {w.cfg.T0:g}",
           "mlups": rates, "cells_converted_fp64": int((w.solid.reshape(ref["solid"].shape) & ~ref["solid"]).sum())}
    for prec in precisions:
        f = out[prec]
        fl = ~ref["solid"] & ~f["solid"]
        res[prec] = {"rho_rel_l2": _rel(f["rho"][fl], ref["rho"][fl]),
                     "u_rel_l2": _rel(f["u"][:, fl], ref["u"][:, fl]),
                     "T_rel_l2": _rel(f["T"], ref["T"]),
                     "alpha_max_abs": float(np.abs(f["alpha"] - ref["alpha"]).max()),
                     "solid_cells_differing": int((f["solid"] != ref["solid"]).sum())}
    res["u_max_fp64"] = float(np.sqrt((ref["u"][:, ~ref["solid"]] ** 2).sum(0)).max())
    return res


def main() -> None:
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--config3", action="store_true")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--T0", type=float, default=None, help="FP16 temperature shift (default: the workload's)")
    ap.add_argument("--precisions", default="fp32,fp16")
    a = ap.parse_args()
    if a.config3:
        print(json.dumps(config3_case(a.n, a.steps, T0=a.T0, precisions=tuple(a.precisions.split(",")))))
    else:
        print(json.dumps({"front": front_case(), "permeability": permeability_case()}))


if __name__ == "__main__":
    main()
