"""B200-native (sm_100a) lattice update of LBM_porousChem.

The hot path (fused collide-stream with bounce-back, conjugate temperature,
Arrhenius pyrolysis with solid->fluid flip, FP64 diagnostics) runs as
hand-written CUDA kernels in ``liblbm_b200.so`` behind the C ABI of
``include/lbm_b200.h``.  Python keeps the reference's solver-class surface
(``LBM2DSolver`` / ``LBM3DSolver``) and drives the kernels through ctypes.
"""
from .config import LatticeConfig, SideBC  # noqa: F401

__all__ = ["LatticeConfig", "SideBC", "Lattice", "LBM2DSolver", "LBM3DSolver"]


def __getattr__(name):
    if name == "Lattice":
        from .lattice import Lattice
        return Lattice
    if name in ("LBM2DSolver", "LBM3DSolver"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
