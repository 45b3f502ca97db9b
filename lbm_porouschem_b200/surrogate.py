"""Learned warm start: a small 2D U-Net that predicts the steady rho, u, T of a
porous geometry, so that the lattice starts near its steady state.

The network (4 levels, 32 base channels, 3x3 convolutions, bf16 weights and
activations, FP32 accumulation) runs entirely on the kernels of ``include/lbm_nn.h``
(implicit-GEMM convolutions on the tensor cores, written for this project); the
forward and backward passes are written out layer by layer below, with torch
tensors used only as device memory.  The surrogate only chooses the initial state:
the lattice then relaxes to the same residual tolerance as a cold start (relative
change of the velocity and of the temperature over the check interval), so the
converged answer is the plain solver's.  The reference has no learned part
(its only torch code is an import test, tests/test_pytorch.py).

Case family (steady channel flow through a porous layer, FP64 lattices so that the
residual tolerance 1e-6 is reachable): D2Q9 BGK + D2Q5 conjugate heat, walls at x = 0 (T = 1) and x = S-1 (T = 0), periodic in y, flow
driven by a body force g along y, seeded disks and ellipses at a random porosity.
Network input channels: solid mask, signed distance to the solid (/ 16), x / S,
log10(g) + 6, porosity, log10 of a Kozeny-Carman permeability estimate; outputs: (rho - 1)/g, u_x and u_y in units of the case's own
velocity scale g*s, T, and log10(s) (a field whose mean gives s), so that every case
is learned to the same relative accuracy whatever its permeability.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from .config import FIXED_VALUE, LatticeConfig, SideBC

CIN, COUT = 8, 8           # padded input / output channel counts (6 / 5 used)
RHO_SCALE = 1e-1           # (rho - 1) / g predicted in units of 1e1


# ----------------------------------------------------------------------------- cases
@dataclass
class Case:
    """One steady porous-channel problem."""
    S: int
    solid: np.ndarray           # (S, S) bool
    g: float                    # body force along y (lattice units)
    porosity: float
    seed: int
    target: dict = field(default_factory=dict)   # converged rho, u (2, S, S), T
    converged: bool = False

    def config(self, precision: str = "fp64", bulk_form: str = "auto") -> LatticeConfig:
        sides = [SideBC() for _ in range(6)]
        sides[0] = SideBC.wall(T_type=FIXED_VALUE, T=1.0)
        sides[1] = SideBC.wall(T_type=FIXED_VALUE, T=0.0)
        # incompressible EOS: the wall extrapolation does not pin the total mass, and with
        # the ideal-gas EOS a slow mass drift would drift the viscosity with it; u with F/2
        # (the Darcy velocity), which nearly blocked cases would otherwise report negative
        return LatticeConfig(dim=2, nx=self.S, ny=self.S, nz=1, collision="bgk", precision=precision,
                             eos="incompressible", nu=0.1, force=(0.0, self.g, 0.0), half_force_velocity=True,
                             thermal="conjugate", tauT_fluid=0.6, tauT_solid=0.9, sides=sides, T0=0.5,
                             bulk_form=bulk_form)


def make_case(S: int, seed: int) -> Case:
    """Seeded disks and ellipses until the fluid fraction drops to a porosity drawn from
    U[0.35, 0.70]; the two cell layers next to the walls stay fluid."""
    rng = np.random.default_rng(seed)
    phi = float(rng.uniform(0.35, 0.70))
    g = float(10 ** rng.uniform(-7.0, -5.0))
    solid = np.zeros((S, S), dtype=bool)
    X, Y = np.meshgrid(np.arange(S), np.arange(S), indexing="ij")
    scale = S / 128.0
    while 1.0 - solid.mean() > phi:
        cx, cy = rng.uniform(0, S), rng.uniform(0, S)
        if rng.random() < 0.5:
            a = b = rng.uniform(4, 10) * scale
            th = 0.0
        else:
            a, b = rng.uniform(4, 12) * scale, rng.uniform(2, 6) * scale
            th = rng.uniform(0, np.pi)
        dx = X - cx
        dy = (Y - cy + S / 2) % S - S / 2          # periodic in y
        u = dx * np.cos(th) + dy * np.sin(th)
        v = -dx * np.sin(th) + dy * np.cos(th)
        solid |= (u / a) ** 2 + (v / b) ** 2 <= 1.0
        solid[:2] = False
        solid[-2:] = False
    return Case(S, solid, g, 1.0 - float(solid.mean()), seed)


def kozeny_carman(case: Case) -> float:
    """Permeability estimate phi^3 / (5 a^2) from the porosity phi and the solid-fluid
    interface length per unit area a, measured on the mask (lattice units)."""
    s = case.solid
    faces = np.count_nonzero(s[1:, :] != s[:-1, :]) + np.count_nonzero(s != np.roll(s, 1, axis=1))
    a = max(faces / s.size, 1e-6)
    return case.porosity ** 3 / (5.0 * a * a)


def inputs(cases: list[Case]) -> np.ndarray:
    """Network inputs, NHWC float32 (B, S, S, 8)."""
    from scipy.ndimage import distance_transform_edt
    out = np.zeros((len(cases), cases[0].S, cases[0].S, CIN), dtype=np.float32)
    for i, c in enumerate(cases):
        S = c.S
        sdf = distance_transform_edt(~c.solid) - distance_transform_edt(c.solid)
        out[i, ..., 0] = c.solid
        out[i, ..., 1] = np.clip(sdf / 16.0, -2, 2)
        out[i, ..., 2] = (np.arange(S)[:, None] / S).repeat(S, 1)
        out[i, ..., 3] = math.log10(c.g) + 6.0
        out[i, ..., 4] = c.porosity
        out[i, ..., 5] = math.log10(kozeny_carman(c))
    return out


def velocity_scale(case: Case) -> float:
    """RMS fluid velocity of the converged case divided by g."""
    fl = ~case.solid
    u = case.target["u"]
    return max(float(np.sqrt(np.mean(u[0][fl] ** 2 + u[1][fl] ** 2))) / case.g, 1e-12)


def targets(cases: list[Case]) -> tuple[np.ndarray, np.ndarray]:
    """Scaled converged fields (B, S, S, 8) and the loss weights (u and rho only where
    fluid)."""
    B, S = len(cases), cases[0].S
    t = np.zeros((B, S, S, COUT), dtype=np.float32)
    w = np.zeros_like(t)
    for i, c in enumerate(cases):
        f = c.target
        fl = ~c.solid
        sc = velocity_scale(c)
        t[i, ..., 0] = np.where(fl, (f["rho"] - 1.0) / c.g * RHO_SCALE, 0.0)
        t[i, ..., 1] = np.where(fl, f["u"][0] / (c.g * sc), 0.0)
        t[i, ..., 2] = np.where(fl, f["u"][1] / (c.g * sc), 0.0)
        t[i, ..., 3] = f["T"]
        t[i, ..., 4] = math.log10(sc)
        w[i, ..., 0:3] = fl[..., None]
        w[i, ..., 3] = 1.0
        w[i, ..., 4] = 10.0        # one number per case that sets the whole flow's magnitude
    return t, w


def fields_from_prediction(pred: np.ndarray, case: Case) -> dict:
    """Initial fields of the lattice from one prediction (S, S, 8).  The density stays
    1 (the cold start's mass); velocity and temperature come from the network."""
    fl = ~case.solid
    sc = 10.0 ** float(np.mean(pred[..., 4]))
    rho = np.ones_like(pred[..., 0])
    ux = np.where(fl, pred[..., 1] * case.g * sc, 0.0)
    uy = np.where(fl, pred[..., 2] * case.g * sc, 0.0)
    T = np.clip(pred[..., 3], 0.0, 1.0)
    u = np.stack([ux, uy, np.zeros_like(ux)])[..., None]
    return {"rho": rho[..., None], "u": u, "T": T[..., None]}


def project_solenoidal(ux: np.ndarray, uy: np.ndarray, solid: np.ndarray) -> tuple:
    """The divergence-free part of a predicted velocity (S, S): u - grad(phi) with
    lap(phi) = div(u) (forward-difference divergence, its adjoint as the gradient, so the
    discrete divergence of the result is zero), periodic in y, no normal flow at the x walls;
    then zero in the solid.  A guess with divergence starts pressure waves the relaxation has
    to wait out; this removes the part of the guess that makes them."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    S = ux.shape[0]
    n = S * S
    idx = np.arange(n).reshape(S, S)
    # forward differences: x (no flux through the walls: the last row's difference is 0), y periodic
    rows, cols, vals = [], [], []
    for i in range(S - 1):
        rows += list(idx[i]); cols += list(idx[i + 1]); vals += [1.0] * S
        rows += list(idx[i]); cols += list(idx[i]); vals += [-1.0] * S
    Dx = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    Dy = (sp.csr_matrix((np.ones(n), (idx.ravel(), np.roll(idx, -1, axis=1).ravel())), shape=(n, n))
          - sp.identity(n, format="csr"))
    # gradient G = (Dx, Dy), divergence D = -G^T, so D G = -(Dx^T Dx + Dy^T Dy)
    div = -(Dx.T @ ux.ravel()) - (Dy.T @ uy.ravel())
    L = -(Dx.T @ Dx + Dy.T @ Dy) - 1e-9 * sp.identity(n)
    phi = spl.spsolve(L.tocsc(), div)
    vx = ux.ravel() - Dx @ phi
    vy = uy.ravel() - Dy @ phi
    vx = np.where(solid.ravel(), 0.0, vx).reshape(S, S)
    vy = np.where(solid.ravel(), 0.0, vy).reshape(S, S)
    return vx, vy


# ----------------------------------------------------------------------------- steady solves
def _t_plane(lat) -> torch.Tensor:
    from .lattice import _COMPUTE_DTYPE
    return lat._view(N.LBM_FIELD_T, _COMPUTE_DTYPE[lat.cfg.precision])


def start_residual(lat) -> None:
    """Reference states of the residuals: the initial velocity (held by the library) and
    the initial temperature."""
    lat._T_prev = _t_plane(lat).clone()


def residual(lat) -> float:
    """max(r_u, r_T): relative L2 change of the fluid velocity and of the temperature
    since the last call (the steady state of the coupled problem needs both)."""
    lat.compute(diag=False, macro=True, residual=True)
    d = lat.read_diag()
    r_u = math.sqrt(d["res_num"] / d["res_den"]) if d["res_den"] > 0 else float("inf")
    T = _t_plane(lat)
    prev = getattr(lat, "_T_prev", None)
    r_T = float((T - prev).norm() / T.norm()) if prev is not None and float(T.norm()) > 0 else float("inf")
    lat._T_prev = T.clone()
    return max(r_u, r_T)


def relax(lat, tol: float = 1e-6, check: int = 100, max_steps: int = 200_000) -> int:
    """Step until the velocity and temperature residuals over `check` steps are <= tol
    (the first check compares with the initial state); returns the steps."""
    start_residual(lat)
    steps = 0
    while steps < max_steps:
        lat.step(check)
        steps += check
        if residual(lat) <= tol:
            break
    return steps


def solve_cases(cases: list[Case], tol: float = 1e-6, check: int = 200, max_steps: int = 100_000,
                precision: str = "fp64") -> dict:
    """Solve every case to steady state as one batch of lattices; fills case.target.
    FP64 by default: with velocities of 1e-6..1e-3 the FP32 round-off of the
    populations puts a floor near 1e-5 under the relative velocity residual."""
    from .lattice import Lattice, LatticeBatch
    lats = []
    for c in cases:
        lat = Lattice(c.config(precision, bulk_form="list"))
        lat.set_geometry(c.solid[..., None])
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
        c.target = {"rho": f["rho"][..., 0], "u": f["u"][:2, ..., 0], "T": f["T"][..., 0]}
        c.converged = bool(ok)
        lat.stream = None
    batch.close()
    for lat in lats:
        lat.close()
    return {"steps": steps, "converged": int(done.sum()), "wall_s": wall,
            "cells": sum(c.S * c.S for c in cases)}


# ----------------------------------------------------------------------------- the network
@dataclass
class Conv:
    cin: int
    cout: int
    k: int
    relu: bool = True


def layers(base: int = 32) -> dict:
    """name -> layer, in the order of the forward pass; channels base, 2, 4, 8 x base."""
    c0, c1, c2, c3 = base, 2 * base, 4 * base, 8 * base
    return {
        "e0a": Conv(CIN, c0, 3), "e0b": Conv(c0, c0, 3),
        "e1a": Conv(c0, c1, 3), "e1b": Conv(c1, c1, 3),
        "e2a": Conv(c1, c2, 3), "e2b": Conv(c2, c2, 3),
        "b3a": Conv(c2, c3, 3), "b3b": Conv(c3, c3, 3),
        "r3": Conv(c3, c2, 1), "d2a": Conv(c3, c2, 3), "d2b": Conv(c2, c2, 3),
        "r2": Conv(c2, c1, 1), "d1a": Conv(c2, c1, 3), "d1b": Conv(c1, c1, 3),
        "r1": Conv(c1, c0, 1), "d0a": Conv(c1, c0, 3), "d0b": Conv(c0, c0, 3),
        "out": Conv(c0, COUT, 1, relu=False),
    }


LAYERS = layers(32)        # the 2D network


class UNet:
    """U-Net on the lbm_nn kernels.  Forward and backward keep every activation of
    a batch of B images of S x S (3D: S x S x S; S a multiple of 8).  dim 2 with 32
    base channels is the 2D network; dim 3 with 16 the 3D variant (3 x 3 x 3
    convolutions, 2 x 2 x 2 pooling)."""

    def __init__(self, device="cuda", seed: int = 0, dim: int = 2, base: int = 32):
        if dim not in (2, 3) or base % 8:
            raise ValueError("dim must be 2 or 3 and base a multiple of 8")
        self.lib = N.load()
        self.dev = torch.device(device)
        self.dim, self.base = dim, base
        self.layers = layers(base)
        gen = torch.Generator().manual_seed(seed)
        self.w, self.b, self.wb = {}, {}, {}
        for name, L in self.layers.items():
            taps = L.k ** dim
            fan_in = L.cin * taps
            std = math.sqrt(2.0 / fan_in) if L.relu else math.sqrt(1.0 / fan_in)
            w = torch.randn(L.cout, taps, L.cin, generator=gen) * std
            if name == "e0a":
                w[:, :, 6:] = 0.0                       # padded input channels
            self.w[name] = w.to(self.dev).contiguous()
            self.b[name] = torch.zeros(L.cout, device=self.dev)
            self.wb[name] = self.w[name].to(torch.bfloat16).contiguous()
        self.adam = {k: (torch.zeros_like(v), torch.zeros_like(v)) for k, v in list(self.w.items())}
        self.adam.update({"b_" + k: (torch.zeros_like(v), torch.zeros_like(v)) for k, v in self.b.items()})
        self.step_count = 0
        self._shape = None
        self.norm = (np.zeros(COUT, np.float32), np.ones(COUT, np.float32))  # per-channel target mean / std

    @property
    def nparams(self) -> int:
        return sum(v.numel() for v in self.w.values()) + sum(v.numel() for v in self.b.values())

    # -------------------------------------------------------------- buffers
    def _buffers(self, B: int, S: int):
        if self._shape == (B, S):
            return
        d, bf, dim = self.dev, torch.bfloat16, self.dim
        e = lambda s, c: torch.empty(B, *(s,) * dim, c, dtype=bf, device=d)  # noqa: E731
        z = lambda s, c: torch.zeros(B, *(s,) * dim, c, dtype=bf, device=d)  # noqa: E731
        s0, s1, s2, s3 = S, S // 2, S // 4, S // 8
        c0, c1, c2, c3 = self.base, 2 * self.base, 4 * self.base, 8 * self.base
        self.a = {
            "x": z(s0, CIN),
            "e0a": e(s0, c0), "cat0": e(s0, c1), "p1": e(s1, c0),
            "e1a": e(s1, c1), "cat1": e(s1, c2), "p2": e(s2, c1),
            "e2a": e(s2, c2), "cat2": e(s2, c3), "p3": e(s3, c2),
            "b3a": e(s3, c3), "b3b": e(s3, c3), "r3": e(s3, c2),
            "d2a": e(s2, c2), "d2b": e(s2, c2), "r2": e(s2, c1),
            "d1a": e(s1, c1), "d1b": e(s1, c1), "r1": e(s1, c0),
            "d0a": e(s0, c0), "d0b": e(s0, c0),
        }
        self.y = torch.empty(B, *(S,) * dim, COUT, dtype=torch.float32, device=d)
        # gradients, same layouts
        self.g = {k: torch.empty_like(v) for k, v in self.a.items() if k != "x"}
        self.gy = torch.empty(B, *(S,) * dim, COUT, dtype=bf, device=d)
        self.dw = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.db = {k: torch.zeros_like(v) for k, v in self.b.items()}
        L = self.layers
        self.wt = {k: torch.empty(L[k].cin, L[k].k ** dim, L[k].cout, dtype=bf, device=d) for k in self.w}
        self.partial = torch.empty(1024, dtype=torch.float32, device=d)
        self._shape = (B, S)

    def _s(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    @staticmethod
    def _p(t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else None

    # the input / output views of every layer: (buffer, channel stride, offset)
    def _views(self):
        a = self.a
        c0, c1, c2, c3 = self.base, 2 * self.base, 4 * self.base, 8 * self.base
        return {
            "e0a": ((a["x"], CIN, 0), (a["e0a"], c0, 0)), "e0b": ((a["e0a"], c0, 0), (a["cat0"], c1, c0)),
            "e1a": ((a["p1"], c0, 0), (a["e1a"], c1, 0)), "e1b": ((a["e1a"], c1, 0), (a["cat1"], c2, c1)),
            "e2a": ((a["p2"], c1, 0), (a["e2a"], c2, 0)), "e2b": ((a["e2a"], c2, 0), (a["cat2"], c3, c2)),
            "b3a": ((a["p3"], c2, 0), (a["b3a"], c3, 0)), "b3b": ((a["b3a"], c3, 0), (a["b3b"], c3, 0)),
            "r3": ((a["b3b"], c3, 0), (a["r3"], c2, 0)),
            "d2a": ((a["cat2"], c3, 0), (a["d2a"], c2, 0)), "d2b": ((a["d2a"], c2, 0), (a["d2b"], c2, 0)),
            "r2": ((a["d2b"], c2, 0), (a["r2"], c1, 0)),
            "d1a": ((a["cat1"], c2, 0), (a["d1a"], c1, 0)), "d1b": ((a["d1a"], c1, 0), (a["d1b"], c1, 0)),
            "r1": ((a["d1b"], c1, 0), (a["r1"], c0, 0)),
            "d0a": ((a["cat0"], c1, 0), (a["d0a"], c0, 0)), "d0b": ((a["d0a"], c0, 0), (a["d0b"], c0, 0)),
            "out": ((a["d0b"], c0, 0), (self.y, COUT, 0)),
        }

    # the library calls, 2D or 3D (spatial sizes of the input: s x s [x s])
    def _sp(self, s):
        return (s,) * self.dim

    def _conv_call(self, ib, ics, ico, w, bias, ob_bf, ob_f32, ocs, oco, B, s, cin, cout, k, relu):
        f = self.lib.lbm_nn_conv if self.dim == 2 else self.lib.lbm_nn_conv3d
        N.check(f(self._p(ib), ics, ico, self._p(w), self._p(bias), None, self._p(ob_bf), self._p(ob_f32), ocs, oco,
                  B, *self._sp(s), cin, cout, k, int(relu), 0, self._s()))

    def _pool(self, src, cs, co, dst, B, s, c):
        f = self.lib.lbm_nn_avgpool2 if self.dim == 2 else self.lib.lbm_nn_avgpool2_3d
        N.check(f(self._p(src), cs, co, self._p(dst), B, *self._sp(s), c, self._s()))

    def _pool_bwd(self, gout, gin, cs, co, B, s, c):
        f = self.lib.lbm_nn_avgpool2_bwd if self.dim == 2 else self.lib.lbm_nn_avgpool2_3d_bwd
        N.check(f(self._p(gout), self._p(gin), cs, co, B, *self._sp(s), c, 1, self._s()))

    def _up(self, src, dst, cs, co, B, s, c):
        f = self.lib.lbm_nn_upsample2 if self.dim == 2 else self.lib.lbm_nn_upsample2_3d
        N.check(f(self._p(src), self._p(dst), cs, co, B, *self._sp(s), c, self._s()))

    def _up_bwd(self, gout, cs, co, gin, B, s, c):
        f = self.lib.lbm_nn_upsample2_bwd if self.dim == 2 else self.lib.lbm_nn_upsample2_3d_bwd
        N.check(f(self._p(gout), cs, co, self._p(gin), B, *self._sp(s), c, self._s()))

    def _gview(self, name):
        """Gradient buffer of a layer's output, same (stride, offset) as the output."""
        _, (buf, cs, co) = self._views()[name]
        if name == "out":
            return self.gy, cs, co
        key = [k for k, v in self.a.items() if v is buf][0]
        return self.g[key], cs, co

    def _res(self, name, B, S):
        level = {"e0": 0, "e1": 1, "e2": 2, "b3": 3, "r3": 3, "d2": 2, "r2": 2, "d1": 1, "r1": 1, "d0": 0, "ou": 0}
        return S >> level[name[:2]]

    # -------------------------------------------------------------- forward
    def _conv(self, name, B, S):
        L = self.layers[name]
        (ib, ics, ico), (ob, ocs, oco) = self._views()[name]
        s = self._res(name, B, S)
        is_f32 = ob.dtype == torch.float32
        self._conv_call(ib, ics, ico, self.wb[name], self.b[name], None if is_f32 else ob, ob if is_f32 else None,
                        ocs, oco, B, s, L.cin, L.cout, L.k, L.relu)

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x: (B, S, S[, S], 8) float32 on the device; returns the FP32 output of the same
        shape."""
        B, S = x.shape[0], x.shape[1]
        if S % 8 or x.dim() != self.dim + 2:
            raise ValueError(f"x must be (B, S{', S' * (self.dim - 1)}, 8) with S a multiple of 8")
        self._buffers(B, S)
        a = self.a
        c0, c1, c2, c3 = self.base, 2 * self.base, 4 * self.base, 8 * self.base
        N.check(self.lib.lbm_nn_to_bf16(self._p(x.contiguous()), self._p(a["x"]), x.numel(), self._s()))
        self._conv("e0a", B, S); self._conv("e0b", B, S)
        self._pool(a["cat0"], c1, c0, a["p1"], B, S, c0)
        self._conv("e1a", B, S); self._conv("e1b", B, S)
        self._pool(a["cat1"], c2, c1, a["p2"], B, S // 2, c1)
        self._conv("e2a", B, S); self._conv("e2b", B, S)
        self._pool(a["cat2"], c3, c2, a["p3"], B, S // 4, c2)
        self._conv("b3a", B, S); self._conv("b3b", B, S); self._conv("r3", B, S)
        self._up(a["r3"], a["cat2"], c3, 0, B, S // 8, c2)
        self._conv("d2a", B, S); self._conv("d2b", B, S); self._conv("r2", B, S)
        self._up(a["r2"], a["cat1"], c2, 0, B, S // 4, c1)
        self._conv("d1a", B, S); self._conv("d1b", B, S); self._conv("r1", B, S)
        self._up(a["r1"], a["cat0"], c1, 0, B, S // 2, c0)
        self._conv("d0a", B, S); self._conv("d0b", B, S); self._conv("out", B, S)
        return self.y

    # -------------------------------------------------------------- backward
    def _conv_bwd(self, name, B, S, need_dx=True):
        """Gradients of one layer from the gradient of its output (already in its view)."""
        L = self.layers[name]
        lib, s = self.lib, self._s()
        (ib, ics, ico), (ob, ocs, oco) = self._views()[name]
        gb, gcs, gco = self._gview(name)
        r = self._res(name, B, S)
        P = B * r ** self.dim
        if L.relu:
            N.check(lib.lbm_nn_relu_bwd(self._p(gb), gcs, gco, self._p(ob), ocs, oco, P, L.cout, s))
        wg = lib.lbm_nn_conv_wgrad if self.dim == 2 else lib.lbm_nn_conv3d_wgrad
        N.check(wg(self._p(ib), ics, ico, self._p(gb), gcs, gco, self._p(self.dw[name]),
                   B, *self._sp(r), L.cin, L.cout, L.k, s))
        N.check(lib.lbm_nn_bias_grad(self._p(gb), gcs, gco, P, L.cout, self._p(self.db[name]), s))
        if not need_dx:
            return
        N.check(lib.lbm_nn_flip_weights(self._p(self.wb[name]), self._p(self.wt[name]), L.cout, L.k ** self.dim,
                                        L.cin, s))
        key = [k for k, v in self.a.items() if v is ib][0]
        self._conv_call(gb, gcs, gco, self.wt[name], None, self.g[key], None, ics, ico, B, r, L.cout, L.cin, L.k,
                        False)

    def backward(self, B: int, S: int) -> None:
        """Back-propagate self.gy (gradient of the loss w.r.t. the output)."""
        g = self.g
        c0, c1, c2, c3 = self.base, 2 * self.base, 4 * self.base, 8 * self.base
        for k in self.dw:
            self.dw[k].zero_()
            self.db[k].zero_()
        for name in ("out", "d0b", "d0a"):
            self._conv_bwd(name, B, S)
        self._up_bwd(g["cat0"], c1, 0, g["r1"], B, S // 2, c0)
        for name in ("r1", "d1b", "d1a"):
            self._conv_bwd(name, B, S)
        self._up_bwd(g["cat1"], c2, 0, g["r2"], B, S // 4, c1)
        for name in ("r2", "d2b", "d2a"):
            self._conv_bwd(name, B, S)
        self._up_bwd(g["cat2"], c3, 0, g["r3"], B, S // 8, c2)
        for name in ("r3", "b3b", "b3a"):
            self._conv_bwd(name, B, S)
        self._pool_bwd(g["p3"], g["cat2"], c3, c2, B, S // 4, c2)
        for name in ("e2b", "e2a"):
            self._conv_bwd(name, B, S)
        self._pool_bwd(g["p2"], g["cat1"], c2, c1, B, S // 2, c1)
        for name in ("e1b", "e1a"):
            self._conv_bwd(name, B, S)
        self._pool_bwd(g["p1"], g["cat0"], c1, c0, B, S, c0)
        self._conv_bwd("e0b", B, S)
        self._conv_bwd("e0a", B, S, need_dx=False)

    def loss_grad(self, target: torch.Tensor, weight: torch.Tensor) -> float:
        """Weighted MSE of self.y against target; writes self.gy; returns the loss."""
        n = target.numel()
        wsum = float(weight.sum().item())
        nb = 512
        N.check(self.lib.lbm_nn_mse(self._p(self.y), self._p(target), self._p(weight), n, 1.0 / wsum,
                                    self._p(self.gy), self._p(self.partial), nb, self._s()))
        return float(self.partial[:nb].sum().item()) / wsum

    def adam_step(self, lr: float = 1e-3, wd: float = 0.0) -> None:
        self.step_count += 1
        s = self._s()
        for k in self.w:
            m, v = self.adam[k]
            N.check(self.lib.lbm_nn_adam(self._p(self.w[k]), self._p(self.dw[k]), self._p(m), self._p(v),
                                         self._p(self.wb[k]), self.w[k].numel(), lr, 0.9, 0.999, 1e-8,
                                         self.step_count, wd, s))
            m, v = self.adam["b_" + k]
            N.check(self.lib.lbm_nn_adam(self._p(self.b[k]), self._p(self.db[k]), self._p(m), self._p(v), None,
                                         self.b[k].numel(), lr, 0.9, 0.999, 1e-8, self.step_count, 0.0, s))
        # the padded input channels stay unused
        self.w["e0a"][:, :, 6:] = 0.0
        self.wb["e0a"][:, :, 6:] = 0.0

    def predict(self, x: np.ndarray, batch: int = 16) -> np.ndarray:
        """Outputs in target units (the normalisation of the training targets undone)."""
        out = []
        mu, sd = self.norm
        for i in range(0, len(x), batch):
            xb = torch.from_numpy(x[i:i + batch]).to(self.dev)
            out.append(self.forward(xb).cpu().numpy() * sd + mu)
        return np.concatenate(out)


def train(net: UNet, x: np.ndarray, t: np.ndarray, w: np.ndarray, epochs: int = 30, batch: int = 16,
          lr: float = 2e-3, seed: int = 0, log=None, augment: bool = True) -> dict:
    """Adam on the weighted MSE of per-channel normalised targets; cosine learning-rate
    decay; random periodic shifts along y (axis 2; 2D or 3D cases) as augmentation.
    Returns the loss history."""
    rng = np.random.default_rng(seed)
    dev = net.dev
    # per-channel normalisation of the targets (weighted mean and std)
    ax = tuple(range(t.ndim - 1))                 # every axis but the channel
    wsum = np.maximum(w.sum(axis=ax), 1e-30)
    mu = (w * t).sum(axis=ax) / wsum
    sd = np.sqrt((w * (t - mu) ** 2).sum(axis=ax) / wsum)
    sd = np.where(sd > 0, sd, 1.0).astype(np.float32)
    net.norm = (mu.astype(np.float32), sd)
    t = ((t - mu) / sd * (w > 0)).astype(np.float32)
    X = torch.from_numpy(x).to(dev)
    T = torch.from_numpy(t).to(dev)
    Wt = torch.from_numpy(w).to(dev)
    n = len(x)
    steps = epochs * max(1, n // batch)
    hist = []
    k = 0
    t0 = time.perf_counter()
    for ep in range(epochs):
        perm = rng.permutation(n)
        tot = 0.0
        for i in range(0, n - batch + 1, batch):
            idx = torch.from_numpy(perm[i:i + batch]).to(dev)
            shift = int(rng.integers(x.shape[2])) if augment else 0   # periodic in y: an exact symmetry
            xb = torch.roll(X[idx], shift, dims=2).contiguous()
            tb = torch.roll(T[idx], shift, dims=2).contiguous()
            wb = torch.roll(Wt[idx], shift, dims=2).contiguous()
            net.forward(xb)
            loss = net.loss_grad(tb, wb)
            net.backward(xb.shape[0], xb.shape[1])
            cur = lr * 0.5 * (1 + math.cos(math.pi * k / steps))
            net.adam_step(cur)
            tot += loss
            k += 1
        hist.append(tot / max(1, n // batch))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.5f}")
    torch.cuda.synchronize()
    return {"loss": hist, "train_s": time.perf_counter() - t0, "steps": k}


def prediction_errors(net: UNet, cases: list[Case]) -> dict:
    """Mean relative L2 errors of the predicted u (fluid cells) and T against the cases'
    converged targets, and the mean relative error of the predicted velocity scale."""
    pred = net.predict(inputs(cases))
    eu, eT, es = [], [], []
    for c, p in zip(cases, pred):
        f0 = fields_from_prediction(p, c)
        fl = ~c.solid
        u0 = np.stack([f0["u"][0, ..., 0], f0["u"][1, ..., 0]])[:, fl]
        ref = c.target["u"][:, fl]
        eu.append(np.linalg.norm(u0 - ref) / max(np.linalg.norm(ref), 1e-30))
        eT.append(np.linalg.norm(f0["T"][..., 0] - c.target["T"]) / max(np.linalg.norm(c.target["T"]), 1e-30))
        es.append(abs(10.0 ** float(np.mean(p[..., 4])) / velocity_scale(c) - 1.0))
    return {"u": float(np.mean(eu)), "T": float(np.mean(eT)), "scale": float(np.mean(es))}


def permeability(case: Case, fields: dict, nu: float = 0.1) -> float:
    """Darcy permeability k = nu <u_y> / g over every cell (superficial velocity)."""
    return nu * float(np.mean(fields["u"][1])) / case.g


def warm_fields(pred: np.ndarray, case: Case, mode: str) -> dict:
    """Initial fields of a warm start: "warm" the prediction as it is, "warm_T" the predicted
    temperature with the fluid at rest, "warm_proj" the prediction with its velocity made
    divergence-free (project_solenoidal)."""
    f0 = fields_from_prediction(pred, case)
    if mode == "warm_T":
        f0["u"] = np.zeros_like(f0["u"])
    elif mode == "warm_proj":
        vx, vy = project_solenoidal(f0["u"][0, ..., 0], f0["u"][1, ..., 0], case.solid)
        f0["u"] = np.stack([vx, vy, np.zeros_like(vx)])[..., None]
    return f0


def evaluate(net: UNet, cases: list[Case], tol: float = 1e-6, check: int = 100, max_steps: int = 200_000,
             modes: tuple = ("warm",)) -> dict:
    """Time to the residual tolerance from rest (cold) and from the network's prediction
    (warm modes, warm_fields) for each case, one lattice at a time; the pre-relaxation error
    of the prediction and the converged permeability of the runs.  The warm time includes
    the inference and any projection."""
    from .lattice import Lattice
    modes = ("warm",) + tuple(m for m in modes if m != "warm")
    x = inputs(cases)
    t_pred = time.perf_counter()
    pred = net.predict(x)
    torch.cuda.synchronize()
    infer_s = (time.perf_counter() - t_pred) / len(cases)
    rows = []
    for c, p in zip(cases, pred):
        out = {}
        for mode in ("cold",) + tuple(modes):
            lat = Lattice(c.config())
            lat.set_geometry(c.solid[..., None])
            t_prep = time.perf_counter()
            if mode == "cold":
                lat.init(rho=1.0, u=(0.0, 0.0, 0.0), T=0.0)
            else:
                f0 = warm_fields(p, c, mode)
                lat.init(rho=f0["rho"], u=f0["u"], T=f0["T"])
            prep_s = time.perf_counter() - t_prep if mode == "warm_proj" else 0.0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            steps = relax(lat, tol, check, max_steps)
            torch.cuda.synchronize()
            out.setdefault("converged", True)
            out["converged"] &= steps < max_steps
            wall = time.perf_counter() - t0
            f = lat.fields()
            fl = {"rho": f["rho"][..., 0], "u": f["u"][:2, ..., 0], "T": f["T"][..., 0]}
            out[mode] = {"steps": steps, "wall_s": wall + (infer_s + prep_s if mode != "cold" else 0.0),
                         "k": permeability(c, fl), "fields": fl}
            lat.close()
        ref = out["cold"]["fields"]
        f0 = fields_from_prediction(p, c)
        fluid = ~c.solid
        du = np.stack([f0["u"][0, ..., 0], f0["u"][1, ..., 0]])[:, fluid] - ref["u"][:, fluid]
        err_u = float(np.linalg.norm(du) / max(np.linalg.norm(ref["u"][:, fluid]), 1e-30))
        err_T = float(np.linalg.norm(f0["T"][..., 0] - ref["T"]) / max(np.linalg.norm(ref["T"]), 1e-30))
        rows.append({"seed": c.seed, "porosity": c.porosity, "g": c.g, "converged": bool(out["converged"]),
                     "cold_steps": out["cold"]["steps"], "warm_steps": out["warm"]["steps"],
                     "cold_s": out["cold"]["wall_s"], "warm_s": out["warm"]["wall_s"],
                     "k_cold": out["cold"]["k"], "k_warm": out["warm"]["k"],
                     "k_rel_diff": abs(out["warm"]["k"] - out["cold"]["k"]) / abs(out["cold"]["k"]),
                     "pre_err_u": err_u, "pre_err_T": err_T,
                     **{f"{m}_steps": out[m]["steps"] for m in modes if m != "warm"},
                     **{f"{m}_s": out[m]["wall_s"] for m in modes if m != "warm"}})
    ok = [r for r in rows if r["converged"]] or rows
    agg = {k: float(np.mean([r[k] for r in ok])) for k in ok[0] if k not in ("seed", "converged")}
    agg["time_ratio"] = float(np.sum([r["warm_s"] for r in ok]) / np.sum([r["cold_s"] for r in ok]))
    agg["steps_ratio"] = float(np.sum([r["warm_steps"] for r in ok]) / np.sum([r["cold_steps"] for r in ok]))
    agg["k_rel_diff_max"] = float(max(r["k_rel_diff"] for r in ok))
    for m in modes:
        if m != "warm":
            agg[f"{m}_time_ratio"] = float(np.sum([r[f"{m}_s"] for r in ok]) / np.sum([r["cold_s"] for r in ok]))
            agg[f"{m}_steps_ratio"] = float(np.sum([r[f"{m}_steps"] for r in ok]) /
                                            np.sum([r["cold_steps"] for r in ok]))
    agg["infer_s_per_case"] = infer_s
    agg["cases_converged"] = len([r for r in rows if r["converged"]])
    agg["cases"] = len(rows)
    return {"cases": rows, "mean": agg}


def experiment(S: int = 128, n_train: int = 1024, n_test: int = 32, epochs: int = 60, batch: int = 16,
               lr: float = 2e-3, tol: float = 1e-6, seed0: int = 0, log=print, modes: tuple = ("warm",)) -> dict:
    """The warm-start experiment: solve n_train seeded cases to steady state (one batch of
    lattices), train the U-Net on them, then compare warm and cold starts on n_test
    held-out cases.  Training and data-generation times are reported separately."""
    t0 = time.perf_counter()
    train_cases = [make_case(S, seed0 + i) for i in range(n_train)]
    test_cases = [make_case(S, seed0 + 1_000_000 + i) for i in range(n_test)]
    gen = solve_cases(train_cases, tol=tol, check=200, max_steps=200_000)
    log(f"solved {gen['converged']}/{n_train} training cases in {gen['wall_s']:.1f} s ({gen['steps']} steps)")
    used = [c for c in train_cases if c.converged]
    x = inputs(used)
    t, w = targets(used)
    net = UNet(seed=seed0)
    hist = train(net, x, t, w, epochs=epochs, batch=batch, lr=lr, log=log)
    log(f"trained {net.nparams} parameters in {hist['train_s']:.1f} s, loss {hist['loss'][0]:.4f} -> {hist['loss'][-1]:.5f}")
    fit = prediction_errors(net, used[:32])
    log(f"prediction error on training cases: u {fit['u']:.3f}, T {fit['T']:.3f}, velocity scale {fit['scale']:.3f}")
    res = evaluate(net, test_cases, tol=tol, check=100, max_steps=400_000, modes=modes)
    m = res["mean"]
    log(f"warm/cold: steps {m['steps_ratio']:.3f}, time {m['time_ratio']:.3f}; pre-relaxation error u "
        f"{m['pre_err_u']:.3f}, T {m['pre_err_T']:.3f}; permeability difference max {m['k_rel_diff_max']:.2e}")
    return {"S": S, "n_train": n_train, "n_train_converged": len(used), "n_test": n_test, "tol": tol,
            "train_fit": fit,
            "data_gen": gen, "train": {"s": hist["train_s"], "steps": hist["steps"], "loss": hist["loss"],
                                       "params": net.nparams, "epochs": epochs, "batch": batch},
            "eval": res, "total_s": time.perf_counter() - t0}


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="learned warm start: data, training, warm vs cold evaluation")
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--train", type=int, default=1024)
    ap.add_argument("--test", type=int, default=32)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--out", default="")
    ap.add_argument("--modes", default="warm", help="warm starts to time: warm, warm_T, warm_proj (comma list)")
    a = ap.parse_args()
    r = experiment(a.size, a.train, a.test, a.epochs, modes=tuple(a.modes.split(",")))
    txt = json.dumps(r, default=float)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt)
    print(json.dumps(r["eval"]["mean"], default=float))
