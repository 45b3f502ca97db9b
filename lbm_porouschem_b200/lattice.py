"""Device-resident lattice driven through the C ABI.

``Lattice`` owns the device buffers (torch tensors used purely as memory),
binds them to a native handle and exposes init / step / diagnostics / field
read-back.  It is the layer the reference-shaped solver classes in
``solver.py`` sit on.  There is no CPU path: constructing a ``Lattice``
without CUDA or without the built library raises.
"""
from __future__ import annotations

import ctypes
import json
import os
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native as N
from .config import LatticeConfig, fill_sides
from .geometry import fortran_flat, from_flat, mask_bytes

_STORE_DTYPE = {"fp32": torch.float32, "fp16": torch.float16, "fp64": torch.float64}
_COMPUTE_DTYPE = {"fp32": torch.float32, "fp16": torch.float32, "fp64": torch.float64}


def _stream_handle(stream: Optional[torch.cuda.Stream]) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


class Lattice:
    """One lattice instance on one GPU."""

    def __init__(self, cfg: LatticeConfig, device: str | torch.device = "cuda",
                 stream: Optional[torch.cuda.Stream] = None):
        if not torch.cuda.is_available():
            raise RuntimeError("the CUDA lattice update needs a GPU (no CPU fallback)")
        self.lib = N.load()
        self.cfg = cfg
        self.device = torch.device(device)
        self.stream = stream
        self._desc = cfg.to_desc()
        h = ctypes.c_void_p()
        N.check(self.lib.lbm_create(ctypes.byref(self._desc), ctypes.byref(h)))
        self._h = h
        self.buf: dict[int, torch.Tensor] = {}
        with torch.cuda.device(self.device):
            for fid in range(N.LBM_NUM_FIELDS):
                nbytes = ctypes.c_size_t()
                N.check(self.lib.lbm_required_bytes(ctypes.byref(self._desc), fid, ctypes.byref(nbytes)))
                if nbytes.value == 0:
                    continue
                t = torch.zeros(nbytes.value, dtype=torch.uint8, device=self.device)
                N.check(self.lib.lbm_bind(self._h, fid, ctypes.c_void_p(t.data_ptr()), nbytes.value))
                self.buf[fid] = t
        self._init_fields: Optional[dict] = None
        # pinned host staging for per-step boundary values (asynchronous H2D copy)
        nb = ctypes.sizeof(N.lbm_side_desc) * 6
        self._sides_pinned = torch.empty(nb, dtype=torch.uint8, pin_memory=True)
        self._host_sides = (N.lbm_side_desc * 6).from_address(self._sides_pinned.data_ptr())
        self._sides_evt: Optional[torch.cuda.Event] = None

    # ----------------------------------------------------------- views
    def _view(self, fid: int, dtype: torch.dtype) -> torch.Tensor:
        return self.buf[fid].view(dtype)

    @property
    def f(self) -> torch.Tensor:
        """Flow populations [2, Q, N] in storage precision (A/B buffers)."""
        return self._view(N.LBM_FIELD_F, _STORE_DTYPE[self.cfg.precision]).view(2, self.cfg.Q, -1)

    @property
    def mask(self) -> torch.Tensor:
        return self.buf[N.LBM_FIELD_MASK]

    @property
    def bulk_kernel(self) -> str:
        """Form of the bulk update this lattice runs, fixed when the lattice is created:
        "list" (cell lists; the default from 65536 cells, or LBM_BULK=list), "tile" (smaller
        lattices, or LBM_BULK=tile) or "dense" (TMA-staged tiles, 3D: bulk_form="dense" or
        LBM_BULK=dense)."""
        return {1: "tile", 2: "list", 3: "dense"}[int(self.lib.lbm_bulk_form(self._h))]

    def set_wait_limit(self, tries: int) -> None:
        """Bound of the dense form's staged-load waits (tries of about a microsecond; 0 gives
        up at once, which is how the timeout path is tested)."""
        N.check(self.lib.lbm_set_wait_limit(self._h, int(tries)))

    @property
    def nsteps(self) -> int:
        return int(self.lib.lbm_step_count(self._h))

    def _s(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(_stream_handle(self.stream))

    # ------------------------------------------------------- set-up
    def set_geometry(self, solid: np.ndarray, reactive: Optional[np.ndarray] = None) -> None:
        """Solid mask in the reference's (nx, ny[, nz]) numpy layout (True = solid)."""
        m = mask_bytes(np.asarray(solid), None if reactive is None else np.asarray(reactive))
        if m.size != self.cfg.ncells:
            raise ValueError("mask shape does not match the lattice")
        with self._on_stream():
            self.mask.copy_(torch.from_numpy(m).to(self.device))

    def set_porous(self, fraction, darcy=None, forchheimer=None, h=None, a=None, rho_solid=1.0,
                   emissivity=None, radiation_surface=None) -> None:
        """Porous cells (``LatticeConfig.porous`` not "none"), before ``init``: the solid
        fraction per cell (0 fluid, between 0 and 1 porous with porosity 1 - fraction; the
        impermeable solid is the mask of ``set_geometry``) and, for the "darcy" and
        "darcy_forchheimer" models, the Darcy / Forchheimer coefficients per cell, all in the
        reference's (nx, ny[, nz]) layout or scalars (set_poro_Darcy /
        set_poro_Darcy_Forchheimer, src/LBM/LBM2D/_io.py:152-172).

        With two temperature fields (``thermal="two_field"``) the porous cells also take the
        heat exchange coefficient ``h`` and surface ``a`` (set_heat_exchange_coef / _surface),
        the solid density ``rho_solid`` (add_rho_solid) and, with ``radiation``, the
        ``emissivity`` and ``radiation_surface`` per cell (src/LBM/app.py:537-566)."""
        if self.cfg.porous == "none":
            raise ValueError("the lattice has no porous model (LatticeConfig.porous)")
        cd = _COMPUTE_DTYPE[self.cfg.precision]

        def arr(v):
            return np.full(self.cfg.shape, float(v)) if np.isscalar(v) else np.asarray(v, np.float64).reshape(self.cfg.shape)

        with self._on_stream():
            for fid, v in ((N.LBM_FIELD_PORO, fraction), (N.LBM_FIELD_DARCY, darcy),
                           (N.LBM_FIELD_FORCH, forchheimer)):
                if fid not in self.buf:
                    continue
                x = 0.0 if v is None else v
                if np.isscalar(x):
                    self._view(fid, cd).fill_(float(x))
                else:
                    flat = fortran_flat(np.asarray(x, dtype=np.float64).reshape(self.cfg.shape))
                    self._view(fid, cd).copy_(torch.from_numpy(flat).to(self.device, cd))
            if N.LBM_FIELD_XHEAT in self.buf:
                ha = arr(0.0 if h is None else h) * arr(0.0 if a is None else a)
                er = arr(0.0 if emissivity is None else emissivity) * arr(0.0 if radiation_surface is None
                                                                           else radiation_surface)
                planes = np.concatenate([fortran_flat(x) for x in (ha, arr(rho_solid), er)])
                self._view(N.LBM_FIELD_XHEAT, cd).copy_(torch.from_numpy(planes).to(self.device, cd))

    def _on_stream(self):
        """Issue torch work on the lattice's stream so it orders with the kernels."""
        return torch.cuda.stream(self.stream) if self.stream is not None else torch.cuda.stream(
            torch.cuda.current_stream())

    def _plane(self, v, ncomp: int = 1) -> torch.Tensor:
        n = self.cfg.ncells
        if np.isscalar(v):
            return torch.full((ncomp * n,), float(v), dtype=torch.float32, device=self.device)
        a = np.asarray(v, dtype=np.float64)
        if ncomp == 1:
            flat = fortran_flat(a.reshape(self.cfg.shape))
        else:
            flat = np.concatenate([fortran_flat(a[i].reshape(self.cfg.shape)) for i in range(ncomp)])
        return torch.from_numpy(flat.astype(np.float32)).to(self.device)

    def init(self, rho=1.0, u=(0.0, 0.0, 0.0), T=0.0, alpha=None, Ts=None) -> None:
        """Equilibrium initialisation (reference init_kernel) from scalars or (nx,ny,nz) arrays.

        ``u`` is a 3-tuple of scalars or an array shaped (3, nx, ny, nz).  ``Ts``: with two
        temperature fields, the solid temperature (TS.S) where it differs from ``T`` (TF.S):
        pure-solid cells and the TS of porous cells start from it."""
        with self._on_stream():
            self._init(rho, u, T, alpha, Ts)

    def _init(self, rho, u, T, alpha, Ts=None) -> None:
        cfg = self.cfg
        r = self._plane(rho)
        if isinstance(u, (tuple, list)) and all(np.isscalar(x) for x in u):
            uu = torch.cat([torch.full((cfg.ncells,), float(x), dtype=torch.float32, device=self.device)
                            for x in u])
        else:
            uu = self._plane(u, 3)
        tt = self._plane(T) if cfg.thermal != "none" else None
        tin = tt
        if cfg.thermal == "two_field" and (Ts is not None or cfg.porous_heat):
            ts = self._plane(T if Ts is None else Ts)
            tt = torch.where((self.mask & 1).bool(), ts, tt)
            tin = torch.cat([tt, ts]) if cfg.porous_heat else tt
        aa = self._plane(alpha) if (cfg.pyro and alpha is not None) else None
        self._init_fields = {"rho": r, "u": uu, "T": tt}
        N.check(self.lib.lbm_init_equilibrium(
            self._h, ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(uu.data_ptr()),
            ctypes.c_void_p(tin.data_ptr()) if tin is not None else None,
            ctypes.c_void_p(aa.data_ptr()) if aa is not None else None, self._s()))
        # macro planes start at the initial state (solid cells keep these values)
        if N.LBM_FIELD_RHO in self.buf:
            cd = _COMPUTE_DTYPE[cfg.precision]
            self._view(N.LBM_FIELD_RHO, cd).copy_(r.to(cd))
            self._view(N.LBM_FIELD_U, cd).copy_(uu.to(cd))
            if tt is not None:
                self._view(N.LBM_FIELD_T, cd).copy_(tin.to(cd))
        if N.LBM_FIELD_UPREV in self.buf:
            # residual reference: the initial velocity (the first residual measures
            # the change since the start)
            self._view(N.LBM_FIELD_UPREV, torch.float32).copy_(uu)

    def set_sides(self, sides) -> None:
        """Change boundary values (not types) between steps; a pinned host->device copy."""
        if self._sides_evt is not None:
            self._sides_evt.synchronize()      # the previous copy has read the staging buffer
        fill_sides(self._host_sides, sides)
        N.check(self.lib.lbm_set_sides(self._h, self._host_sides, self._s()))
        self._sides_evt = torch.cuda.Event()
        self._sides_evt.record(self.stream if self.stream is not None else torch.cuda.current_stream())
        self.cfg.sides = list(sides)

    # ------------------------------------------------------- stepping
    def step(self, n: int = 1, diag: bool = False, macro: bool = False, residual: bool = False) -> None:
        flags = (N.LBM_STEP_DIAG if diag else 0) | (N.LBM_STEP_MACRO if macro else 0) | \
                (N.LBM_STEP_RESIDUAL if residual else 0)
        N.check(self.lib.lbm_step(self._h, int(n), flags, self._s()))

    def capture(self, n: int) -> None:
        """Record n ordinary steps (n even) as a CUDA graph on the lattice's stream (one
        is required).  Capturing runs no kernel but moves the step counter by n; the first
        replay() brings the state level with it, every later replay advances both."""
        if self.stream is None:
            raise RuntimeError("capture needs the lattice to own a stream (Lattice(cfg, stream=...))")
        if n <= 0 or n % 2:
            raise ValueError("a captured sequence must have an even number of steps")
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            N.check(self.lib.lbm_step(self._h, int(n), 0, self._s()))
        self.graph, self._graph_steps, self._counted = g, n, True

    def replay(self) -> None:
        """Run the captured steps once more (capture() first)."""
        if getattr(self, "graph", None) is None:
            raise RuntimeError("capture() first")
        with torch.cuda.stream(self.stream):
            self.graph.replay()
        if self._counted:
            self._counted = False
        else:
            N.check(self.lib.lbm_advance(self._h, self._graph_steps))

    def compute(self, diag: bool = True, macro: bool = False, residual: bool = False) -> None:
        """Recompute outputs for the current state without advancing it."""
        flags = (N.LBM_STEP_DIAG if diag else 0) | (N.LBM_STEP_MACRO if macro else 0) | \
                (N.LBM_STEP_RESIDUAL if residual else 0)
        N.check(self.lib.lbm_compute_macro(self._h, flags, self._s()))

    def read_diag(self) -> dict:
        d = N.lbm_diag()
        rc = self.lib.lbm_read_diag(self._h, ctypes.byref(d), self._s())
        out = {k: getattr(d, k) for k, _ in N.lbm_diag._fields_}
        if rc == N.LBM_ERR_NONFINITE:
            out["nonfinite"] = max(out["nonfinite"], 1.0)
            return out
        N.check(rc)
        return out

    def read_diag_async(self) -> "PendingDiag":
        """The last LBM_STEP_DIAG step's diagnostics, copied to page-locked host memory
        without waiting (lbm_read_diag_async): ``result()`` waits for that copy only, so a
        driver loop can launch the next step first.  Two reads may be outstanding at a time
        (the staging buffers alternate)."""
        if getattr(self, "_diag_pinned", None) is None:
            nb = ctypes.sizeof(N.lbm_diag) + 8
            self._diag_pinned = [torch.zeros(nb, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
            self._diag_slot = 0
        buf = self._diag_pinned[self._diag_slot]
        self._diag_slot ^= 1
        base = buf.data_ptr()
        err = base + ctypes.sizeof(N.lbm_diag)
        N.check(self.lib.lbm_read_diag_async(self._h, ctypes.c_void_p(base), ctypes.c_void_p(err), self._s()))
        ev = torch.cuda.Event()
        ev.record(self.stream if self.stream is not None else torch.cuda.current_stream())
        return PendingDiag(buf, ev)

    def diagnostics(self) -> dict:
        """Diagnostics of the current state (recomputed if needed)."""
        if self.nsteps == 0:
            raise RuntimeError("no step taken yet")
        self.compute(diag=True)
        return self.read_diag()

    def fields(self) -> dict:
        """rho, u (3,nx,ny,nz) and T of the current state as numpy arrays (reference layout)."""
        cfg = self.cfg
        cd = _COMPUTE_DTYPE[cfg.precision]
        if self.nsteps > 0:
            self.compute(diag=True, macro=True)
        torch.cuda.current_stream().synchronize() if self.stream is None else self.stream.synchronize()
        rho = from_flat(self._view(N.LBM_FIELD_RHO, cd).cpu().numpy(), cfg.shape)
        uf = self._view(N.LBM_FIELD_U, cd).cpu().numpy()
        n = cfg.ncells
        u = np.stack([from_flat(uf[i * n:(i + 1) * n], cfg.shape) for i in range(3)])
        out = {"rho": rho, "u": u}
        if cfg.thermal != "none":
            out["T"] = from_flat(self._view(N.LBM_FIELD_T, cd)[:n].cpu().numpy(), cfg.shape)
        if cfg.pyro:
            out["alpha"] = from_flat(self._view(N.LBM_FIELD_ALPHA, cd).cpu().numpy(), cfg.shape)
        par = self.nsteps & 1
        m = self.mask.cpu().numpy()
        out["solid"] = from_flat(((m >> par) & 1).astype(bool), cfg.shape)
        if cfg.porous_heat:
            # TS: of porous cells the second plane of the macro temperature, of pure-solid
            # cells their one field, 0 in pure-fluid cells
            poro = self._view(N.LBM_FIELD_PORO, cd).cpu().numpy()
            ts = np.where(poro > 0, self._view(N.LBM_FIELD_T, cd)[n:].cpu().numpy(), 0.0)
            out["Ts"] = np.where(out["solid"], out["T"], from_flat(ts, cfg.shape))
        return out

    # ------------------------------------------------------- checkpoint / resume
    def _state_arrays(self) -> dict:
        """Device state the next step reads, as host arrays (storage precision)."""
        cfg, n = self.cfg, self.cfg.ncells
        half = self.nsteps & 1
        sd, cd = _STORE_DTYPE[cfg.precision], _COMPUTE_DTYPE[cfg.precision]
        (self.stream or torch.cuda.current_stream()).synchronize()
        out = {"f": self._view(N.LBM_FIELD_F, sd).view(2, cfg.Q, n)[half].cpu().numpy(),
               "mask": self.mask.cpu().numpy()}
        if N.LBM_FIELD_G in self.buf:
            out["g"] = self._view(N.LBM_FIELD_G, sd).view(2, cfg.QT, n)[half].cpu().numpy()
        if N.LBM_FIELD_ALPHA in self.buf:
            out["alpha"] = self._view(N.LBM_FIELD_ALPHA, cd).cpu().numpy()
        if N.LBM_FIELD_REL in self.buf:
            out["rel"] = self._view(N.LBM_FIELD_REL, cd).view(2, n)[half].cpu().numpy()
        for fid, name in ((N.LBM_FIELD_RHO, "rho"), (N.LBM_FIELD_U, "u"), (N.LBM_FIELD_T, "T")):
            if fid in self.buf:
                out[name] = self._view(fid, cd).cpu().numpy()
        if N.LBM_FIELD_UPREV in self.buf:
            out["uprev"] = self._view(N.LBM_FIELD_UPREV, torch.float32).cpu().numpy()
        if N.LBM_FIELD_INLET in self.buf:
            out["inlet"] = self._view(N.LBM_FIELD_INLET, cd).cpu().numpy()
        for fid, name in ((N.LBM_FIELD_PORO, "poro"), (N.LBM_FIELD_DARCY, "darcy"), (N.LBM_FIELD_FORCH, "forch"),
                          (N.LBM_FIELD_XHEAT, "xheat")):
            if fid in self.buf:
                out[name] = self._view(fid, cd).cpu().numpy()
        if N.LBM_FIELD_GS in self.buf:
            out["gs"] = self._view(N.LBM_FIELD_GS, sd).view(2, cfg.QT, n)[half].cpu().numpy()
        return out

    def save_checkpoint(self, path) -> str:
        """Write the state to ``path`` (numpy .npz, uncompressed): the halves of the flow and
        temperature populations and the gas-release plane that the next step reads, the
        mask, reactive fraction, residual reference, macro planes and flow-rate inlet
        state, in their device precision, with the step count and the configuration.  ``Lattice.load_checkpoint``
        continues from it with the same fields, bit for bit.  (The reference has no
        restart; its export_snapshot is a reserved no-op, src/LBM/LBM2D/_io.py:589-598.)"""
        if not self.nsteps and self._init_fields is None:
            raise RuntimeError("nothing to save: the lattice is not initialised")
        meta = {"format": "lbm_b200 checkpoint", "version": 1, "step": self.nsteps,
                "config": self.cfg.to_dict()}
        arrays = self._state_arrays()
        path = os.fspath(path)
        with open(path, "wb") as fh:
            np.savez(fh, meta=np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8), **arrays)
        return path

    @classmethod
    def load_checkpoint(cls, path, device: str | torch.device = "cuda",
                        stream: Optional[torch.cuda.Stream] = None) -> "Lattice":
        """A new lattice holding the state saved by ``save_checkpoint`` (lbm_resume)."""
        with np.load(os.fspath(path)) as z:
            meta = json.loads(bytes(z["meta"]).decode())
            if meta.get("format") != "lbm_b200 checkpoint" or meta.get("version") != 1:
                raise ValueError(f"{path}: not an lbm_b200 checkpoint (version 1)")
            lat = cls(LatticeConfig.from_dict(meta["config"]), device=device, stream=stream)
            lat._restore({k: z[k] for k in z.files if k != "meta"}, int(meta["step"]))
        return lat

    def _restore(self, arrays: dict, step: int) -> None:
        cfg, n = self.cfg, self.cfg.ncells
        half = step & 1
        sd, cd = _STORE_DTYPE[cfg.precision], _COMPUTE_DTYPE[cfg.precision]

        def put(dst: torch.Tensor, name: str):
            a = arrays.get(name)
            if a is None or a.size != dst.numel():
                raise ValueError(f"checkpoint field {name!r} is missing or has the wrong size")
            dst.copy_(torch.from_numpy(np.ascontiguousarray(a).reshape(dst.shape)).to(self.device))

        with self._on_stream():
            put(self._view(N.LBM_FIELD_F, sd).view(2, cfg.Q, n)[half], "f")
            put(self.mask, "mask")
            if N.LBM_FIELD_G in self.buf:
                put(self._view(N.LBM_FIELD_G, sd).view(2, cfg.QT, n)[half], "g")
            if N.LBM_FIELD_ALPHA in self.buf:
                put(self._view(N.LBM_FIELD_ALPHA, cd), "alpha")
            if N.LBM_FIELD_REL in self.buf:
                put(self._view(N.LBM_FIELD_REL, cd).view(2, n)[half], "rel")
            for fid, name in ((N.LBM_FIELD_RHO, "rho"), (N.LBM_FIELD_U, "u"), (N.LBM_FIELD_T, "T")):
                if fid in self.buf:
                    put(self._view(fid, cd), name)
            if N.LBM_FIELD_UPREV in self.buf:
                put(self._view(N.LBM_FIELD_UPREV, torch.float32), "uprev")
            if N.LBM_FIELD_INLET in self.buf:
                put(self._view(N.LBM_FIELD_INLET, cd), "inlet")
            for fid, name in ((N.LBM_FIELD_PORO, "poro"), (N.LBM_FIELD_DARCY, "darcy"),
                              (N.LBM_FIELD_FORCH, "forch"), (N.LBM_FIELD_XHEAT, "xheat")):
                if fid in self.buf:
                    put(self._view(fid, cd), name)
            if N.LBM_FIELD_GS in self.buf:
                put(self._view(N.LBM_FIELD_GS, sd).view(2, cfg.QT, n)[half], "gs")
            N.check(self.lib.lbm_resume(self._h, int(step), self._s()))
        self._init_fields = {}

    def close(self) -> None:
        if getattr(self, "buf", None):
            (self.stream or torch.cuda.current_stream()).synchronize()
        self.graph = None
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.lbm_destroy(self._h)
            self._h = ctypes.c_void_p()
        self.buf.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PendingDiag:
    """Diagnostics on their way to the host (``Lattice.read_diag_async``)."""

    def __init__(self, buf: torch.Tensor, event: torch.cuda.Event):
        self._buf, self._event = buf, event

    def result(self) -> dict:
        """Wait for the copy and return the values as ``Lattice.read_diag`` does (an error
        flag raised by the step kernels raises ``LBMNativeError``)."""
        self._event.synchronize()
        base = self._buf.data_ptr()
        d = N.lbm_diag.from_address(base)
        err = ctypes.c_int32.from_address(base + ctypes.sizeof(N.lbm_diag)).value
        if err & 1:
            raise N.LBMNativeError(N.LBM_ERR_TIMEOUT, "a bounded wait in the step kernel timed out; the state is invalid")
        if err & 2:
            raise N.LBMNativeError(N.LBM_ERR_CUDA, "the fluid cell list overflowed; the state is invalid")
        return {k: getattr(d, k) for k, _ in N.lbm_diag._fields_}


class LatticeBatch:
    """Many initialised lattices stepped together (one persistent launch per kernel).

    The lattices must share dim, precision, collision, thermal and pyrolysis
    settings and use cell lists (``LatticeConfig(bulk_form="list")``); sizes,
    geometries and parameters are free.  ``capture(n)`` records ``n`` steps (even)
    as a CUDA graph that ``replay()`` runs again without host work per step."""

    def __init__(self, lattices: Sequence[Lattice], stream: Optional[torch.cuda.Stream] = None):
        if not lattices:
            raise ValueError("a batch needs at least one lattice")
        self.lattices = list(lattices)
        self.lib = self.lattices[0].lib
        self.device = self.lattices[0].device
        self.stream = stream if stream is not None else torch.cuda.Stream(device=self.device)
        for lat in self.lattices:
            (lat.stream or torch.cuda.current_stream(lat.device)).synchronize()
        n = len(self.lattices)
        self._hs = (ctypes.c_void_p * n)(*[lat._h.value for lat in self.lattices])
        nbytes = ctypes.c_size_t()
        s = ctypes.c_void_p(int(self.stream.cuda_stream))
        N.check(self.lib.lbm_batch_required_bytes(self._hs, n, s, ctypes.byref(nbytes)))
        self.buf = torch.empty(max(int(nbytes.value), 256), dtype=torch.uint8, device=self.device)
        b = ctypes.c_void_p()
        N.check(self.lib.lbm_batch_create(self._hs, n, ctypes.c_void_p(self.buf.data_ptr()), self.buf.numel(), s,
                                          ctypes.byref(b)))
        self._b = b
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self._graph_steps = 0
        self._counted = False

    @property
    def ncells(self) -> int:
        return sum(lat.cfg.ncells for lat in self.lattices)

    def step(self, n: int = 1) -> None:
        N.check(self.lib.lbm_batch_step(self._b, int(n), ctypes.c_void_p(int(self.stream.cuda_stream))))

    def tune(self, steps: int = 4, candidates=None) -> dict:
        """Pick the persistent grid (blocks per SM) of the bulk kernel by timing ``steps``
        real batch steps per candidate (they advance the lattices); keeps the fastest.
        Returns {blocks_per_sm: ms per step}.  Call before capture()."""
        fp64 = self.lattices[0].cfg.precision == "fp64"
        cands = candidates or ((1, 2) if fp64 else (2, 3, 4))
        times = {}
        for bps in cands:
            N.check(self.lib.lbm_batch_set_blocks(self._b, int(bps)))
            self.step(2)                       # settle
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            self.step(steps)
            e1.record(self.stream)
            e1.synchronize()
            times[bps] = e0.elapsed_time(e1) / steps
        self.blocks_per_sm = min(times, key=times.get)
        N.check(self.lib.lbm_batch_set_blocks(self._b, int(self.blocks_per_sm)))
        return times

    def capture(self, n: int) -> None:
        """Record n batch steps (n even) as a CUDA graph.  Capturing runs no kernel but
        moves the step counters by n; the first replay() brings the state level with
        them, every later replay advances both."""
        if n <= 0 or n % 2:
            raise ValueError("a captured sequence must have an even number of steps")
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            N.check(self.lib.lbm_batch_step(self._b, int(n), ctypes.c_void_p(int(self.stream.cuda_stream))))
        self.graph, self._graph_steps, self._counted = g, n, True

    def replay(self) -> None:
        if self.graph is None:
            raise RuntimeError("capture() first")
        with torch.cuda.stream(self.stream):
            self.graph.replay()
        if self._counted:
            self._counted = False
        else:
            N.check(self.lib.lbm_batch_advance(self._b, self._graph_steps))

    def synchronize(self) -> None:
        self.stream.synchronize()

    def close(self) -> None:
        if getattr(self, "_b", None) is not None and self._b.value:
            self.stream.synchronize()
            self.graph = None
            self.lib.lbm_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
