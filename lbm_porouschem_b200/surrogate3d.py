"""Learned warm start, 3D variant: the 2D pipeline of ``surrogate`` on sphere packings,
with the U-Net in its 3D form (3 x 3 x 3 convolutions, 2 x 2 x 2 pooling, 16 base
channels) on the 3D kernels of ``include/lbm_nn.h``.

Case family (FP64 lattices, so that the residual tolerance 1e-6 is reachable): D3Q19
BGK + D3Q7 conjugate heat on S^3, incompressible EOS, body force g along y, walls at
x = 0 (T = 1) and x = S-1 (T = 0), periodic in y and z; seeded spheres (radius
U[2.5, 6] S/32) until the porosity reaches U[0.35, 0.70]; the two cell layers next to
each wall stay fluid.  Network inputs and outputs as in 2D, with u_z added: solid
mask, signed distance (/ 16), x / S, log10(g) + 6, porosity, log10 of a Kozeny-Carman
estimate; (rho - 1)/g, u in units of the case's velocity scale g*s, T, log10(s).
As in 2D, the network only chooses the initial state; the lattice relaxes to the
same residual tolerance as a cold start.
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .config import FIXED_VALUE, LatticeConfig, SideBC
from .surrogate import CIN, COUT, RHO_SCALE, UNet, relax, residual, start_residual, train


@dataclass
class Case3D:
    S: int
    solid: np.ndarray           # (S, S, S) bool
    g: float
    porosity: float
    seed: int
    target: dict = field(default_factory=dict)   # converged rho, u (3, S, S, S), T
    converged: bool = False

    def config(self, precision: str = "fp64", bulk_form: str = "auto") -> LatticeConfig:
        sides = [SideBC() for _ in range(6)]
        sides[0] = SideBC.wall(T_type=FIXED_VALUE, T=1.0)
        sides[1] = SideBC.wall(T_type=FIXED_VALUE, T=0.0)
        return LatticeConfig(dim=3, nx=self.S, ny=self.S, nz=self.S, collision="bgk", precision=precision,
                             eos="incompressible", nu=0.1, force=(0.0, self.g, 0.0), half_force_velocity=True,
                             thermal="conjugate", tauT_fluid=0.6, tauT_solid=0.9, sides=sides, T0=0.5,
                             bulk_form=bulk_form)


def make_case(S: int, seed: int) -> Case3D:
    rng = np.random.default_rng(seed)
    phi = float(rng.uniform(0.35, 0.70))
    g = float(10 ** rng.uniform(-7.0, -5.0))
    solid = np.zeros((S, S, S), dtype=bool)
    X, Y, Z = np.meshgrid(np.arange(S), np.arange(S), np.arange(S), indexing="ij")
    scale = S / 32.0
    while 1.0 - solid.mean() > phi:
        cx, cy, cz = rng.uniform(0, S, 3)
        r = rng.uniform(2.5, 6.0) * scale
        dy = (Y - cy + S / 2) % S - S / 2          # periodic in y and z
        dz = (Z - cz + S / 2) % S - S / 2
        solid |= (X - cx) ** 2 + dy ** 2 + dz ** 2 <= r * r
        solid[:2] = False
        solid[-2:] = False
    return Case3D(S, solid, g, 1.0 - float(solid.mean()), seed)


def kozeny_carman(case: Case3D) -> float:
    """phi^3 / (5 a^2), a = solid-fluid interface area per unit volume of the mask."""
    s = case.solid
    faces = (np.count_nonzero(s[1:] != s[:-1]) + np.count_nonzero(s != np.roll(s, 1, axis=1))
             + np.count_nonzero(s != np.roll(s, 1, axis=2)))
    a = max(faces / s.size, 1e-6)
    return case.porosity ** 3 / (5.0 * a * a)


def inputs(cases: list[Case3D]) -> np.ndarray:
    """Network inputs, NDHWC float32 (B, S, S, S, 8)."""
    from scipy.ndimage import distance_transform_edt
    S = cases[0].S
    out = np.zeros((len(cases), S, S, S, CIN), dtype=np.float32)
    for i, c in enumerate(cases):
        sdf = distance_transform_edt(~c.solid) - distance_transform_edt(c.solid)
        out[i, ..., 0] = c.solid
        out[i, ..., 1] = np.clip(sdf / 16.0, -2, 2)
        out[i, ..., 2] = (np.arange(S) / S)[:, None, None]
        out[i, ..., 3] = math.log10(c.g) + 6.0
        out[i, ..., 4] = c.porosity
        out[i, ..., 5] = math.log10(kozeny_carman(c))
    return out


def velocity_scale(case: Case3D) -> float:
    fl = ~case.solid
    u = case.target["u"]
    return max(float(np.sqrt(np.mean((u[:, fl] ** 2).sum(0)))) / case.g, 1e-12)


def targets(cases: list[Case3D]) -> tuple[np.ndarray, np.ndarray]:
    """Scaled converged fields (B, S, S, S, 8) and loss weights (u and rho only where fluid)."""
    S = cases[0].S
    t = np.zeros((len(cases), S, S, S, COUT), dtype=np.float32)
    w = np.zeros_like(t)
    for i, c in enumerate(cases):
        f, fl = c.target, ~c.solid
        sc = velocity_scale(c)
        t[i, ..., 0] = np.where(fl, (f["rho"] - 1.0) / c.g * RHO_SCALE, 0.0)
        for a in range(3):
            t[i, ..., 1 + a] = np.where(fl, f["u"][a] / (c.g * sc), 0.0)
        t[i, ..., 4] = f["T"]
        t[i, ..., 5] = math.log10(sc)
        w[i, ..., 0:4] = fl[..., None]
        w[i, ..., 4] = 1.0
        w[i, ..., 5] = 10.0
    return t, w


def fields_from_prediction(pred: np.ndarray, case: Case3D) -> dict:
    """Initial fields from one prediction (S, S, S, 8): density 1, velocity and
    temperature from the network."""
    fl = ~case.solid
    sc = 10.0 ** float(np.mean(pred[..., 5]))
    u = np.stack([np.where(fl, pred[..., 1 + a] * case.g * sc, 0.0) for a in range(3)])
    return {"rho": np.ones(pred.shape[:3]), "u": u, "T": np.clip(pred[..., 4], 0.0, 1.0)}


def solve_cases(cases: list[Case3D], tol: float = 1e-6, check: int = 200, max_steps: int = 100_000,
                precision: str = "fp64") -> dict:
    """Solve every case to steady state as one batch of lattices; fills case.target."""
    from .lattice import Lattice, LatticeBatch
    lats = []
    for c in cases:
        lat = Lattice(c.config(precision, bulk_form="list"))
        lat.set_geometry(c.solid)
        lat.init(rho=1.0, u=(0.0, 0.0, 0.0), T=0.0)
        lats.append(lat)
    batch = LatticeBatch(lats)
    for lat in lats:
        lat.stream = batch.stream
        start_residual(lat)
    done = np.zeros(len(cases), dtype=bool)
    steps = 0
    t0 = time.perf_counter()
    while steps < max_steps and not done.all():
        batch.step(check)
        steps += check
        for i, lat in enumerate(lats):
            if not done[i] and residual(lat) <= tol:
                done[i] = True
    wall = time.perf_counter() - t0
    for c, lat, ok in zip(cases, lats, done):
        f = lat.fields()
        c.target = {"rho": f["rho"], "u": f["u"], "T": f["T"]}
        c.converged = bool(ok)
        lat.stream = None
    batch.close()
    for lat in lats:
        lat.close()
    return {"steps": steps, "converged": int(done.sum()), "wall_s": wall, "cells": sum(c.S ** 3 for c in cases)}


def permeability(case: Case3D, fields: dict, nu: float = 0.1) -> float:
    """Darcy permeability k = nu <u_y> / g over every cell (superficial velocity)."""
    return nu * float(np.mean(fields["u"][1])) / case.g


def evaluate(net: UNet, cases: list[Case3D], tol: float = 1e-6, check: int = 100, max_steps: int = 200_000) -> dict:
    """Steps to the residual tolerance from rest (cold) and from the prediction (warm),
    one lattice at a time, and the converged permeability of both runs."""
    from .lattice import Lattice
    pred = net.predict(inputs(cases), batch=4)
    rows = []
    for c, p in zip(cases, pred):
        out = {}
        for mode in ("cold", "warm"):
            lat = Lattice(c.config("fp64"))
            lat.set_geometry(c.solid)
            if mode == "cold":
                lat.init(rho=1.0, u=(0.0, 0.0, 0.0), T=0.0)
            else:
                f0 = fields_from_prediction(p, c)
                lat.init(rho=f0["rho"], u=f0["u"], T=f0["T"])
            t0 = time.perf_counter()
            n = relax(lat, tol, check, max_steps)
            torch.cuda.synchronize()
            out[mode] = (n, time.perf_counter() - t0, permeability(c, lat.fields()))
            lat.close()
        rows.append({"seed": c.seed, "porosity": round(c.porosity, 3), "cold_steps": out["cold"][0],
                     "warm_steps": out["warm"][0], "cold_s": out["cold"][1], "warm_s": out["warm"][1],
                     "k_cold": out["cold"][2], "k_warm": out["warm"][2],
                     "k_rel_diff": abs(out["warm"][2] - out["cold"][2]) / max(abs(out["cold"][2]), 1e-30)})
    cold = sum(r["cold_steps"] for r in rows)
    warm = sum(r["warm_steps"] for r in rows)
    return {"cases": rows, "mean": {"warm_over_cold_steps": warm / max(cold, 1),
                                    "k_rel_diff_mean": float(np.mean([r["k_rel_diff"] for r in rows])),
                                    "k_rel_diff_max": float(np.max([r["k_rel_diff"] for r in rows]))}}


def experiment(S: int = 32, n_train: int = 64, n_test: int = 8, epochs: int = 80, batch: int = 8,
               lr: float = 2e-3, log=None) -> dict:
    """Solve n_train + n_test seeded cases, train the 3D network (16 base channels) on the
    training cases and compare warm and cold starts on the held-out ones."""
    train_cases = [make_case(S, 100 + i) for i in range(n_train)]
    test_cases = [make_case(S, 20_000 + i) for i in range(n_test)]
    t0 = time.perf_counter()
    solved = solve_cases(train_cases, tol=1e-6, check=100, max_steps=100_000)
    used = [c for c in train_cases if c.converged]
    net = UNet(dim=3, base=16, seed=0)
    x = inputs(used)
    t, w = targets(used)
    hist = train(net, x, t, w, epochs=epochs, batch=batch, lr=lr, log=log)
    res = evaluate(net, test_cases, tol=1e-6, check=100, max_steps=100_000)
    return {"S": S, "train_cases": len(used), "train_solve": solved, "train_s": hist["train_s"],
            "loss_first": hist["loss"][0], "loss_last": hist["loss"][-1], "params": net.nparams,
            "wall_s": time.perf_counter() - t0, **res}


def main() -> None:
    ap = argparse.ArgumentParser(description="3D learned warm start: warm vs cold time to steady state")
    ap.add_argument("--size", type=int, default=32)
    ap.add_argument("--train", type=int, default=64)
    ap.add_argument("--test", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=80)
    a = ap.parse_args()
    print(json.dumps(experiment(a.size, a.train, a.test, a.epochs), default=float))


if __name__ == "__main__":
    main()
