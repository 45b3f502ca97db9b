"""Slab decomposition of one 3D lattice along z over several GPUs (one process per GPU).

The lattice is cut into z-slabs, one per rank.  Each rank's lattice holds its slab plus
``halo`` ghost planes on either side and is periodic in z on its own.  After every step each
rank copies the whole per-cell state that the next step reads -- the read halves of the
flow, temperature and porous-TS populations, the mask byte, the reactive fraction and the
gas-release plane -- of its ``halo`` outermost interior planes into the ghost planes of its
neighbours.  With ``halo = 2`` the interior planes then evolve exactly as in the undivided
lattice: a cell pulls from the read state of its neighbours (first ghost plane), and a cell
that turns fluid starts from the mean post-stream state of its fluid neighbours, whose own
pulls reach the second ghost plane.  The ghost planes are stepped with the rest (the next
exchange overwrites what they compute), so the kernels run unchanged; the price is
``2 * halo`` planes of extra work per rank and ``halo`` planes of state per neighbour and
step.  The ranks run the tile form of the bulk update, which reads the mask every step (the
cell lists would carry the neighbour bits of ghost cells between exchanges).

Transport: ``torch.distributed`` point-to-point (NCCL between GPUs over NVLink, gloo between
CPU processes) in ``DistExchange``, or copies between slabs that live in one process
(``exchange_local``; ``SlabSet`` runs every slab of a lattice on one device).  The reference
has no multi-device path (one Taichi runtime per process, src/LBM/app.py:41-58).

Limits: 3D lattices whose z sides are periodic (inactive), no flow-rate inlet, at least
``halo`` planes per rank.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .config import LatticeConfig


@dataclass
class SlabPlan:
    """Split of ``nz`` planes over ``nranks`` ranks; rank r owns global planes
    ``starts[r] .. starts[r] + counts[r] - 1`` and holds ``halo`` ghost planes on each side."""
    nz: int
    nranks: int
    halo: int = 2
    counts: list = field(init=False)
    starts: list = field(init=False)

    def __post_init__(self):
        base, extra = divmod(self.nz, self.nranks)
        self.counts = [base + (1 if r < extra else 0) for r in range(self.nranks)]
        self.starts = [sum(self.counts[:r]) for r in range(self.nranks)]
        if min(self.counts) < self.halo:
            raise ValueError(f"{self.nz} planes over {self.nranks} ranks leave fewer than halo = {self.halo} "
                             "planes on a rank")

    def local_nz(self, r: int) -> int:
        return self.counts[r] + 2 * self.halo

    def planes(self, r: int) -> np.ndarray:
        """Global z of each local plane of rank r (ghosts wrap around the periodic z)."""
        return (self.starts[r] - self.halo + np.arange(self.local_nz(r))) % self.nz

    def interior(self, r: int) -> slice:
        return slice(self.halo, self.halo + self.counts[r])

    def below(self, r: int) -> int:
        return (r - 1) % self.nranks

    def above(self, r: int) -> int:
        return (r + 1) % self.nranks


def local_config(cfg: LatticeConfig, plan: SlabPlan, r: int) -> LatticeConfig:
    """The lattice of rank r: its slab and ghost planes, tile form."""
    if cfg.dim != 3:
        raise ValueError("the slab decomposition splits 3D lattices along z")
    if cfg.sides[4].active or cfg.sides[5].active:
        raise ValueError("the slab decomposition needs periodic (inactive) z sides")
    if any(s.active and s.v_type == 3 for s in cfg.sides):
        raise ValueError("the flow-rate inlet sums over a whole side: not in a slab decomposition")
    if plan.nz != cfg.nz:
        raise ValueError("plan and configuration disagree on nz")
    return cfg.replace(nz=plan.local_nz(r), bulk_form="tile")


def local_slice(a, plan: SlabPlan, r: int, shape):
    """Rank r's planes (ghosts included) of a global (nx, ny, nz) array, or a scalar as is;
    leading component axes (e.g. (3, nx, ny, nz)) are kept."""
    if a is None or np.isscalar(a) or (isinstance(a, (tuple, list)) and all(np.isscalar(x) for x in a)):
        return a
    a = np.asarray(a)
    if a.shape[-3:] != tuple(shape):
        a = a.reshape((-1,) + tuple(shape) if a.size > np.prod(shape) else tuple(shape))
    return np.take(a, plan.planes(r), axis=-1)


# ------------------------------------------------------------------------ the exchange
def _sl(v, ax: int, start: int, n: int):
    idx = [slice(None)] * v.ndim
    idx[ax] = slice(start, start + n)
    return tuple(idx)


def exchange_local(views_by_rank: list, axes: list, plan: SlabPlan) -> None:
    """Ghost planes of every slab from its neighbours' interior planes, all slabs in this
    process.  views_by_rank[r]: the state arrays of rank r (torch tensors or numpy arrays),
    axes[i]: the plane axis of array i.  Sends are interior planes and receives ghost planes,
    so the copies never overlap (one rank included: its ghosts take its own edge planes)."""
    H = plan.halo
    for r, views in enumerate(views_by_rank):
        lo, hi = plan.below(r), plan.above(r)
        for i, v in enumerate(views):
            ax = axes[i]
            c_lo, c_r = plan.counts[lo], plan.counts[r]
            # lower ghosts <- top interior planes of the rank below
            v[_sl(v, ax, 0, H)] = views_by_rank[lo][i][_sl(v, ax, c_lo, H)]
            # upper ghosts <- bottom interior planes of the rank above
            v[_sl(v, ax, H + c_r, H)] = views_by_rank[hi][i][_sl(v, ax, H, H)]


class DistExchange:
    """The same exchange between processes with torch.distributed point-to-point: each rank
    packs its two edge bands (bytes of every state array) into one buffer per direction, sends
    them to the ranks below and above and unpacks what it receives into its ghost planes."""

    def __init__(self, plan: SlabPlan, rank: int, group=None):
        self.plan, self.rank, self.group = plan, rank, group

    def __call__(self, views: list, axes: list) -> None:
        import torch
        import torch.distributed as dist
        p, r, H = self.plan, self.rank, self.plan.halo
        if p.nranks == 1:
            exchange_local([views], axes, p)
            return
        tv = [torch.from_numpy(v) if isinstance(v, np.ndarray) else v for v in views]

        def pack(start):
            return torch.cat([t[_sl(t, ax, start, H)].contiguous().reshape(-1).view(torch.uint8)
                              for t, ax in zip(tv, axes)])

        down, up = pack(H), pack(p.counts[r])
        from_above, from_below = torch.empty_like(down), torch.empty_like(up)
        lo, hi = p.below(r), p.above(r)
        ops = [dist.P2POp(dist.isend, down, lo, self.group, tag=1),
               dist.P2POp(dist.isend, up, hi, self.group, tag=2),
               dist.P2POp(dist.irecv, from_above, hi, self.group, tag=1),
               dist.P2POp(dist.irecv, from_below, lo, self.group, tag=2)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()

        def unpack(buf, start):
            off = 0
            for t, ax in zip(tv, axes):
                dst = t[_sl(t, ax, start, H)]
                n = dst.numel() * dst.element_size()
                dst.copy_(buf[off:off + n].view(t.dtype).view(dst.shape))
                off += n

        unpack(from_below, 0)
        unpack(from_above, H + p.counts[r])


# ------------------------------------------------------------------------ lattices
def lattice_views(lat) -> tuple:
    """The per-cell state of a ``Lattice`` that the next step reads, as views with the z
    planes on axis 1: ([components, nz, nx*ny] tensors, plane axes)."""
    from . import _native as N
    from .lattice import _COMPUTE_DTYPE, _STORE_DTYPE
    cfg = lat.cfg
    P, nz, half = cfg.nx * cfg.ny, cfg.nz, lat.nsteps & 1
    sd, cd = _STORE_DTYPE[cfg.precision], _COMPUTE_DTYPE[cfg.precision]
    v = [lat._view(N.LBM_FIELD_F, sd).view(2, cfg.Q, nz, P)[half]]
    if N.LBM_FIELD_G in lat.buf:
        v.append(lat._view(N.LBM_FIELD_G, sd).view(2, cfg.QT, nz, P)[half])
    if N.LBM_FIELD_GS in lat.buf:
        v.append(lat._view(N.LBM_FIELD_GS, sd).view(2, cfg.QT, nz, P)[half])
    if N.LBM_FIELD_ALPHA in lat.buf:
        v.append(lat._view(N.LBM_FIELD_ALPHA, cd).view(1, nz, P))
    if N.LBM_FIELD_REL in lat.buf:
        v.append(lat._view(N.LBM_FIELD_REL, cd).view(2, 1, nz, P)[half])
    v.append(lat.mask.view(1, nz, P))   # bytes last: the packed buffer keeps the others aligned
    return v, [1] * len(v)


class _SlabBase:
    """Global-array front of the per-rank lattices: inputs are sliced per rank (ghosts
    included), outputs keep the interior planes."""
    cfg: LatticeConfig
    plan: SlabPlan

    def _local(self, a, r):
        return local_slice(a, self.plan, r, self.cfg.shape)


class SlabSet(_SlabBase):
    """Every slab of one lattice in this process, on one device; the exchange is a set of
    device copies.  Steps equal the undivided lattice's bit for bit (tile form)."""

    def __init__(self, cfg: LatticeConfig, nslabs: int, halo: int = 2, device="cuda"):
        from .lattice import Lattice
        self.cfg, self.plan = cfg, SlabPlan(cfg.nz, nslabs, halo)
        self.lats = [Lattice(local_config(cfg, self.plan, r), device=device) for r in range(nslabs)]

    def set_geometry(self, solid, reactive=None):
        for r, lat in enumerate(self.lats):
            lat.set_geometry(self._local(np.asarray(solid).reshape(self.cfg.shape), r),
                             None if reactive is None else self._local(np.asarray(reactive).reshape(self.cfg.shape), r))

    def set_porous(self, fraction, darcy=None, forchheimer=None, **heat):
        for r, lat in enumerate(self.lats):
            lat.set_porous(self._local(fraction, r), self._local(darcy, r), self._local(forchheimer, r),
                           **{k: self._local(v, r) for k, v in heat.items()})

    def init(self, rho=1.0, u=(0.0, 0.0, 0.0), T=0.0, alpha=None, Ts=None):
        for r, lat in enumerate(self.lats):
            lat.init(rho=self._local(rho, r), u=self._local(u, r), T=self._local(T, r),
                     alpha=self._local(alpha, r), Ts=self._local(Ts, r))

    @property
    def nsteps(self) -> int:
        return self.lats[0].nsteps

    def step(self, n: int = 1) -> None:
        for _ in range(n):
            for lat in self.lats:
                lat.step(1)
            views = [lattice_views(lat) for lat in self.lats]
            exchange_local([v for v, _ in views], views[0][1], self.plan)

    def fields(self) -> dict:
        parts = [lat.fields() for lat in self.lats]
        out = {}
        for k in parts[0]:
            out[k] = np.concatenate([p[k][..., self.plan.interior(r)] for r, p in enumerate(parts)], axis=-1)
        return out

    def close(self) -> None:
        for lat in self.lats:
            lat.close()


class SlabLattice(_SlabBase):
    """This rank's slab of a lattice split over the ranks of a torch.distributed group (one
    process per GPU)."""

    def __init__(self, cfg: LatticeConfig, halo: int = 2, group=None, device="cuda"):
        import torch.distributed as dist
        from .lattice import Lattice
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.cfg, self.plan = cfg, SlabPlan(cfg.nz, world, halo)
        self.lat = Lattice(local_config(cfg, self.plan, self.rank), device=device)
        self.exchange = DistExchange(self.plan, self.rank, group)

    def set_geometry(self, solid, reactive=None):
        r = self.rank
        self.lat.set_geometry(self._local(np.asarray(solid).reshape(self.cfg.shape), r),
                              None if reactive is None else self._local(np.asarray(reactive).reshape(self.cfg.shape), r))

    def set_porous(self, fraction, darcy=None, forchheimer=None, **heat):
        r = self.rank
        self.lat.set_porous(self._local(fraction, r), self._local(darcy, r), self._local(forchheimer, r),
                            **{k: self._local(v, r) for k, v in heat.items()})

    def init(self, rho=1.0, u=(0.0, 0.0, 0.0), T=0.0, alpha=None, Ts=None):
        r = self.rank
        self.lat.init(rho=self._local(rho, r), u=self._local(u, r), T=self._local(T, r),
                      alpha=self._local(alpha, r), Ts=self._local(Ts, r))

    @property
    def nsteps(self) -> int:
        return self.lat.nsteps

    def step(self, n: int = 1) -> None:
        for _ in range(n):
            self.lat.step(1)
            self.exchange(*lattice_views(self.lat))

    def local_fields(self) -> dict:
        """This rank's interior planes."""
        f = self.lat.fields()
        return {k: v[..., self.plan.interior(self.rank)] for k, v in f.items()}

    def fields(self) -> dict:
        """The whole lattice on every rank (all-gather of the interior planes)."""
        import torch.distributed as dist
        mine = self.local_fields()
        if self.plan.nranks == 1:
            return mine
        parts = [None] * self.plan.nranks
        dist.all_gather_object(parts, mine, group=self.group)
        return {k: np.concatenate([p[k] for p in parts], axis=-1) for k in mine}

    def close(self) -> None:
        self.lat.close()
