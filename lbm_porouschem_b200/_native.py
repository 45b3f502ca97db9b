"""ctypes binding of ``liblbm_b200.so`` (the C ABI in ``include/lbm_b200.h``).

The structures below mirror the header field for field; ``lbm_desc.struct_size``
is checked by the library so that a drift between the two fails loudly.  There
is no fallback: if the library cannot be loaded, every solver call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "liblbm_b200.so"

# status codes
LBM_OK = 0
LBM_ERR_ARG = 1
LBM_ERR_UNBOUND = 2
LBM_ERR_CUDA = 3
LBM_ERR_NONFINITE = 4
LBM_ERR_SIZE = 5
LBM_ERR_TIMEOUT = 6

LBM_COLL_BGK, LBM_COLL_MRT = 0, 1
LBM_PREC_FP32, LBM_PREC_FP16, LBM_PREC_FP64 = 0, 1, 2
LBM_FP16_STOCHASTIC, LBM_FP16_NEAREST = 0, 1
LBM_EOS_IDEAL_GAS, LBM_EOS_INCOMPRESSIBLE = 0, 1
LBM_THERMAL_NONE, LBM_THERMAL_CONJUGATE, LBM_THERMAL_TWOFIELD = 0, 1, 2
LBM_BC_PERIODIC, LBM_BC_ZEROGRADIENT, LBM_BC_FIXEDVALUE, LBM_BC_FLOWRATE = 0, 1, 2, 3
LBM_VISC_CONSTANT, LBM_VISC_SUTHERLAND = 0, 1
LBM_MASK_SOLID = 3
LBM_MASK_REACTIVE = 4

(LBM_FIELD_F, LBM_FIELD_G, LBM_FIELD_MASK, LBM_FIELD_ALPHA, LBM_FIELD_REL, LBM_FIELD_RHO,
 LBM_FIELD_U, LBM_FIELD_T, LBM_FIELD_UPREV, LBM_FIELD_SCRATCH, LBM_FIELD_INLET,
 LBM_FIELD_PORO, LBM_FIELD_DARCY, LBM_FIELD_FORCH, LBM_FIELD_GS, LBM_FIELD_XHEAT) = range(16)
LBM_NUM_FIELDS = 16
LBM_PORO_NONE, LBM_PORO_ERGUN, LBM_PORO_DARCY, LBM_PORO_DARCY_FORCHHEIMER = 0, 1, 2, 3

LBM_STEP_DIAG = 1
LBM_STEP_MACRO = 2
LBM_STEP_RESIDUAL = 4

EXPORTED = (
    "lbm_abi_version", "lbm_last_error", "lbm_required_bytes", "lbm_create", "lbm_destroy",
    "lbm_bind", "lbm_set_sides", "lbm_init_equilibrium", "lbm_resume", "lbm_step", "lbm_compute_macro",
    "lbm_read_diag", "lbm_read_diag_async",
    "lbm_step_count", "lbm_bulk_form", "lbm_set_wait_limit", "lbm_advance", "lbm_diag_noalloc", "lbm_stl_work_bytes", "lbm_voxelise_stl",
    "lbm_batch_required_bytes", "lbm_batch_create", "lbm_batch_step", "lbm_batch_advance", "lbm_batch_destroy",
    "lbm_batch_set_blocks",
    "lbm_nn_conv", "lbm_nn_conv_wgrad", "lbm_nn_bias_grad", "lbm_nn_flip_weights", "lbm_nn_avgpool2",
    "lbm_nn_avgpool2_bwd", "lbm_nn_upsample2", "lbm_nn_upsample2_bwd", "lbm_nn_mse", "lbm_nn_adam",
    "lbm_nn_relu_bwd", "lbm_nn_to_bf16",
    "lbm_nn_conv3d", "lbm_nn_conv3d_wgrad", "lbm_nn_avgpool2_3d", "lbm_nn_avgpool2_3d_bwd", "lbm_nn_upsample2_3d",
    "lbm_nn_upsample2_3d_bwd",
)
LBM_NOALLOC_MAX_ROWS = 32768


class lbm_side_desc(C.Structure):
    _fields_ = [
        ("active", C.c_int32), ("v_type", C.c_int32), ("rho_type", C.c_int32), ("T_type", C.c_int32),
        ("v", C.c_double * 3), ("rho", C.c_double), ("T", C.c_double),
    ]


class lbm_desc(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32), ("dim", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32),
        ("nz", C.c_int32), ("collision", C.c_int32), ("precision", C.c_int32), ("eos", C.c_int32),
        ("thermal", C.c_int32), ("pyro", C.c_int32), ("half_force_velocity", C.c_int32),
        ("bulk_form", C.c_int32),
        ("nu", C.c_double), ("force", C.c_double * 3), ("tauT_fluid", C.c_double),
        ("tauT_solid", C.c_double), ("pyro_A", C.c_double), ("pyro_b", C.c_double),
        ("pyro_Ea", C.c_double), ("pyro_Tmin", C.c_double), ("T_ref", C.c_double),
        ("T_scale", C.c_double), ("dt_phys", C.c_double), ("heat_norm", C.c_double),
        ("gas_coef", C.c_double), ("alpha_flip", C.c_double), ("mrt_s", C.c_double * 19),
        ("rho0", C.c_double), ("T0", C.c_double), ("side", lbm_side_desc * 6),
        ("viscosity", C.c_int32), ("porous", C.c_int32), ("suth_A", C.c_double), ("suth_Ts", C.c_double),
        ("Ts_ref", C.c_double), ("Ts_scale", C.c_double), ("cap_fluid", C.c_double), ("cap_solid", C.c_double),
        ("dx_phys", C.c_double), ("T_ambient", C.c_double), ("radiation", C.c_int32), ("fp16_rounding", C.c_int32),
        ("tprop", C.c_int32), ("tp_cond", (C.c_double * 5) * 2), ("tp_cap_lo", (C.c_double * 5) * 2),
        ("tp_cap_hi", (C.c_double * 5) * 2), ("tp_cap_Tmid", C.c_double * 2), ("tp_cap_mul", C.c_double * 2),
        ("tp_rhos", C.c_double), ("tp_dt", C.c_double), ("tp_dx2", C.c_double), ("tp_prandtl", C.c_double),
    ]


class lbm_diag(C.Structure):
    _fields_ = [
        ("mass", C.c_double), ("energy", C.c_double), ("solid_alpha", C.c_double),
        ("umax", C.c_double), ("Tmin", C.c_double), ("Tmax", C.c_double),
        ("nonfinite", C.c_double), ("nfluid", C.c_double), ("res_num", C.c_double),
        ("res_den", C.c_double), ("step", C.c_int64),
    ]


class LBMNativeError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"lbm status {code}: {msg}")
        self.code = code


_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the shared library (once).  Raises if it is missing: no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path or os.environ.get("LBM_LIBRARY") or LIB_PATH)
    if not p.exists():
        raise RuntimeError(
            f"{p} not found: build it with `python -m lbm_porouschem_b200._build` "
            "(the CUDA path has no CPU fallback)")
    lib = C.CDLL(str(p))
    vp, i32, i64, sz = C.c_void_p, C.c_int32, C.c_int64, C.c_size_t
    lib.lbm_abi_version.restype = i32
    lib.lbm_last_error.restype = C.c_char_p
    lib.lbm_required_bytes.argtypes = [C.POINTER(lbm_desc), i32, C.POINTER(sz)]
    lib.lbm_required_bytes.restype = i32
    lib.lbm_create.argtypes = [C.POINTER(lbm_desc), C.POINTER(vp)]
    lib.lbm_create.restype = i32
    lib.lbm_destroy.argtypes = [vp]
    lib.lbm_destroy.restype = i32
    lib.lbm_bind.argtypes = [vp, i32, vp, sz]
    lib.lbm_bind.restype = i32
    lib.lbm_set_sides.argtypes = [vp, C.POINTER(lbm_side_desc), vp]
    lib.lbm_set_sides.restype = i32
    lib.lbm_init_equilibrium.argtypes = [vp, vp, vp, vp, vp, vp]
    lib.lbm_init_equilibrium.restype = i32
    lib.lbm_resume.argtypes = [vp, i64, vp]
    lib.lbm_resume.restype = i32
    lib.lbm_advance.argtypes = [vp, i32]
    lib.lbm_advance.restype = i32
    lib.lbm_stl_work_bytes.argtypes = [i32, i32, i32, i32, C.POINTER(sz)]
    lib.lbm_stl_work_bytes.restype = i32
    lib.lbm_voxelise_stl.argtypes = [vp, i64, i32, i32, i32, i32, C.c_double, vp, sz, vp, vp, vp]
    lib.lbm_voxelise_stl.restype = i32
    lib.lbm_step.argtypes = [vp, i32, i32, vp]
    lib.lbm_step.restype = i32
    lib.lbm_compute_macro.argtypes = [vp, i32, vp]
    lib.lbm_compute_macro.restype = i32
    lib.lbm_read_diag.argtypes = [vp, C.POINTER(lbm_diag), vp]
    lib.lbm_read_diag.restype = i32
    lib.lbm_read_diag_async.argtypes = [vp, vp, vp, vp]
    lib.lbm_read_diag_async.restype = i32
    lib.lbm_step_count.argtypes = [vp]
    lib.lbm_step_count.restype = i64
    lib.lbm_bulk_form.argtypes = [vp]
    lib.lbm_bulk_form.restype = i32
    lib.lbm_set_wait_limit.argtypes = [vp, C.c_uint32]
    lib.lbm_set_wait_limit.restype = i32
    lib.lbm_diag_noalloc.argtypes = [vp, C.POINTER(lbm_diag), vp]
    lib.lbm_diag_noalloc.restype = i32
    lib.lbm_batch_required_bytes.argtypes = [C.POINTER(vp), i32, vp, C.POINTER(sz)]
    lib.lbm_batch_required_bytes.restype = i32
    lib.lbm_batch_create.argtypes = [C.POINTER(vp), i32, vp, sz, vp, C.POINTER(vp)]
    lib.lbm_batch_create.restype = i32
    lib.lbm_batch_step.argtypes = [vp, i32, vp]
    lib.lbm_batch_step.restype = i32
    lib.lbm_batch_advance.argtypes = [vp, i32]
    lib.lbm_batch_advance.restype = i32
    lib.lbm_batch_set_blocks.argtypes = [vp, i32]
    lib.lbm_batch_set_blocks.restype = i32
    f32 = C.c_float
    nn = {
        "lbm_nn_conv": [vp, i32, i32, vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, i32, i32, i32, i32, i32, vp],
        "lbm_nn_conv_wgrad": [vp, i32, i32, vp, i32, i32, vp, i32, i32, i32, i32, i32, i32, vp],
        "lbm_nn_bias_grad": [vp, i32, i32, i32, i32, vp, vp],
        "lbm_nn_flip_weights": [vp, vp, i32, i32, i32, vp],
        "lbm_nn_avgpool2": [vp, i32, i32, vp, i32, i32, i32, i32, vp],
        "lbm_nn_avgpool2_bwd": [vp, vp, i32, i32, i32, i32, i32, i32, i32, vp],
        "lbm_nn_upsample2": [vp, vp, i32, i32, i32, i32, i32, i32, vp],
        "lbm_nn_upsample2_bwd": [vp, i32, i32, vp, i32, i32, i32, i32, vp],
        "lbm_nn_mse": [vp, vp, vp, sz, f32, vp, vp, i32, vp],
        "lbm_nn_adam": [vp, vp, vp, vp, vp, sz, f32, f32, f32, f32, i32, f32, vp],
        "lbm_nn_relu_bwd": [vp, i32, i32, vp, i32, i32, i32, i32, vp],
        "lbm_nn_to_bf16": [vp, vp, sz, vp],
        "lbm_nn_conv3d": [vp, i32, i32, vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, i32, i32, i32, i32, i32, i32, vp],
        "lbm_nn_conv3d_wgrad": [vp, i32, i32, vp, i32, i32, vp, i32, i32, i32, i32, i32, i32, i32, vp],
        "lbm_nn_avgpool2_3d": [vp, i32, i32, vp, i32, i32, i32, i32, i32, vp],
        "lbm_nn_avgpool2_3d_bwd": [vp, vp, i32, i32, i32, i32, i32, i32, i32, i32, vp],
        "lbm_nn_upsample2_3d": [vp, vp, i32, i32, i32, i32, i32, i32, i32, vp],
        "lbm_nn_upsample2_3d_bwd": [vp, i32, i32, vp, i32, i32, i32, i32, i32, vp],
    }
    for name, args in nn.items():
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = i32
    lib.lbm_batch_destroy.argtypes = [vp]
    lib.lbm_batch_destroy.restype = i32
    if lib.lbm_abi_version() != 1:
        raise RuntimeError("liblbm_b200.so ABI version mismatch")
    _lib = lib
    return lib


def check(code: int) -> None:
    if code != LBM_OK:
        msg = _lib.lbm_last_error().decode() if _lib is not None else "library not loaded"
        raise LBMNativeError(code, msg)
