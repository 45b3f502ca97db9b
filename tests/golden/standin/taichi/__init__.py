"""Sequential NumPy stand-in for the subset of Taichi 1.7 that LBM_porousChem's solver files use.

TEST INFRASTRUCTURE ONLY.  ``tests/golden/make_reference_fixtures.py`` puts this directory
first on ``sys.path`` so that the reference's own, unmodified solver modules
(``src/LBM/LBM2D/*.py``, ``src/LBM/LBM3D/*.py``) import and run on the CPU without Taichi,
which is not installable here.  Nothing in the package imports it.

What it emulates, and why running it sequentially gives the reference's answer:

* ``@ti.kernel`` / ``@ti.func`` / ``@ti.data_oriented`` are identity decorators: a Taichi
  func is inlined into its kernel, and each outermost ``for`` of a kernel becomes one
  parallel task, the tasks running one after the other.  Here each outermost loop runs its
  iterations one after the other instead.  That is the same answer whenever no iteration
  reads a location another iteration of the same loop writes, which holds for the loops
  this stand-in is used on: the push step writes each ``F[ip][k]`` / ``F[i][LR[k]]`` slot
  from exactly one cell and reads only its own cell's state, ``macro`` touches only its own
  cell, and each boundary pass reads the inner layer that the pass does not write.
* ``ti.static(x)`` is ``x`` (compile-time branches and unrolled ranges are plain Python).
* Fields are NumPy arrays; ``float`` (the default real type) is float64, so the fixtures are
  the reference's arithmetic in double precision.  Scalar reads are NumPy scalars, so a
  division by zero yields inf / nan as in the compiled kernels rather than an exception.  Every operation is plain IEEE arithmetic
  in source order; Taichi's fast-math contractions would differ only in the last bits.
* ``ti.Vector`` is a small value type.  Reading an element of a vector field returns a
  snapshot that also writes through on item assignment, so both ``u = self.v[i]`` (a value)
  and ``self.f[i][k] = x`` (a store) mean what they mean in Taichi.

Not emulated (raises): atomics, ``ti.template`` kernels and anything outside this list.
"""
from __future__ import annotations

import builtins as _builtins
import itertools
import math as _m

import numpy as np

from . import math  # noqa: F401  (ti.math.*)

np.seterr(all="ignore")

# ---------------------------------------------------------------- types and runtime
i8, i16, i32, i64 = "i8", "i16", "i32", "i64"
u8, u16, u32, u64 = "u8", "u16", "u32", "u64"
f16, f32, f64 = "f16", "f32", "f64"
cpu, gpu, cuda, vulkan, metal, opengl, x64, arm64 = ("cpu", "gpu", "cuda", "vulkan", "metal",
                                                      "opengl", "x64", "arm64")

_NP = {"i8": np.int8, "i16": np.int16, "i32": np.int32, "i64": np.int64, "u8": np.uint8,
       "u16": np.uint16, "u32": np.uint32, "u64": np.uint64, "f16": np.float64,
       "f32": np.float64, "f64": np.float64, float: np.float64, int: np.int32}


def _np_dtype(dtype):
    if dtype in _NP:
        return _NP[dtype]
    raise NotImplementedError(f"stand-in: dtype {dtype!r}")


def init(*args, **kwargs) -> None:
    pass


def reset() -> None:
    pass


def data_oriented(cls):
    return cls


def kernel(fn):
    return fn


def func(fn):
    return fn


def static(x, *rest):
    return x if not rest else (x,) + rest


class MatrixField:  # used only as an annotation by the reference
    pass


# ---------------------------------------------------------------- small vectors
class Vector:
    """Value-semantics small vector (``ti.Vector``)."""
    __slots__ = ("v",)
    __array_ufunc__ = None   # NumPy scalars defer to the reflected operators below

    def __init__(self, v, dt=None):
        self.v = list(v)

    @staticmethod
    def field(n, dtype=float, shape=(), **kw):
        return VectorField(n, dtype, shape)

    # element access
    def __getitem__(self, k):
        return self.v[k]

    def __setitem__(self, k, x):
        self.v[k] = x

    def __len__(self):
        return len(self.v)

    def __iter__(self):
        return iter(list(self.v))

    def __repr__(self):
        return f"Vector({self.v})"

    # arithmetic (element-wise, or with a scalar)
    def _bin(self, o, op):
        if isinstance(o, Vector):
            return Vector([op(a, b) for a, b in zip(self.v, o.v)])
        return Vector([op(a, o) for a in self.v])

    def _rbin(self, o, op):
        return Vector([op(o, a) for a in self.v])

    def __add__(self, o):
        return self._bin(o, lambda a, b: a + b)

    def __radd__(self, o):
        return self._rbin(o, lambda a, b: a + b)

    def __sub__(self, o):
        return self._bin(o, lambda a, b: a - b)

    def __rsub__(self, o):
        return self._rbin(o, lambda a, b: a - b)

    def __mul__(self, o):
        return self._bin(o, lambda a, b: a * b)

    def __rmul__(self, o):
        return self._rbin(o, lambda a, b: a * b)

    def __truediv__(self, o):
        return self._bin(o, lambda a, b: a / b)

    def __rtruediv__(self, o):
        return self._rbin(o, lambda a, b: a / b)

    def __pow__(self, o):
        return self._bin(o, lambda a, b: a ** b)

    def __neg__(self):
        return Vector([-a for a in self.v])

    # in-place forms return new values (Python then stores them through __setitem__)
    __iadd__ = __add__
    __isub__ = __sub__
    __imul__ = __mul__
    __itruediv__ = __truediv__

    def dot(self, o):
        s = self.v[0] * o.v[0]
        for a, b in zip(self.v[1:], o.v[1:]):
            s = s + a * b
        return s

    def norm(self):
        return _m.sqrt(self.dot(self))

    def norm_sqr(self):
        return self.dot(self)

    def sum(self):
        s = self.v[0]
        for a in self.v[1:]:
            s = s + a
        return s


class _ElemRef(Vector):
    """Element of a vector field: a value snapshot whose item stores write through."""
    __slots__ = ("_arr", "_idx")

    def __init__(self, arr, idx):
        Vector.__init__(self, arr[idx].tolist())
        self._arr = arr
        self._idx = idx

    def __setitem__(self, k, x):
        self.v[k] = x
        self._arr[self._idx + (k,)] = x


# ---------------------------------------------------------------- fields
def _norm_shape(shape):
    if shape is None:
        return ()
    if isinstance(shape, int):
        return (shape,)
    return tuple(int(s) for s in shape)


def _norm_idx(idx):
    if idx is None:
        return ()
    if isinstance(idx, Vector):
        return tuple(int(a) for a in idx.v)
    if isinstance(idx, tuple):
        out = []
        for a in idx:
            if isinstance(a, Vector):
                out.extend(int(b) for b in a.v)
            else:
                out.append(int(a))
        return tuple(out)
    return (int(idx),)


class ScalarField:
    def __init__(self, dtype, shape):
        self.dtype = dtype
        self.shape = _norm_shape(shape)
        self.a = np.zeros(self.shape, dtype=_np_dtype(dtype))

    def __getitem__(self, idx):
        # a NumPy scalar, so that arithmetic follows IEEE rules as compiled Taichi code does
        # (a division by zero gives inf / nan instead of raising)
        return self.a[_norm_idx(idx)]

    def __setitem__(self, idx, val):
        self.a[_norm_idx(idx)] = val

    def from_numpy(self, arr):
        arr = np.asarray(arr)
        if arr.shape != self.a.shape:
            raise ValueError(f"stand-in from_numpy: shape {arr.shape} != {self.a.shape}")
        self.a[...] = arr

    def to_numpy(self):
        return self.a.copy()

    def fill(self, v):
        self.a[...] = v


class VectorField:
    def __init__(self, n, dtype, shape):
        self.n = int(n)
        self.dtype = dtype
        self.shape = _norm_shape(shape)
        self.a = np.zeros(self.shape + (self.n,), dtype=_np_dtype(dtype))

    def __getitem__(self, idx):
        return _ElemRef(self.a, _norm_idx(idx))

    def __setitem__(self, idx, val):
        if isinstance(val, (int, float)):
            self.a[_norm_idx(idx)] = val
        else:
            self.a[_norm_idx(idx)] = list(val)

    def from_numpy(self, arr):
        arr = np.asarray(arr)
        if arr.shape != self.a.shape:
            raise ValueError(f"stand-in from_numpy: shape {arr.shape} != {self.a.shape}")
        self.a[...] = arr

    def to_numpy(self):
        return self.a.copy()

    def fill(self, v):
        self.a[...] = v


def field(dtype, shape=(), **kw):
    return ScalarField(dtype, shape)


# ---------------------------------------------------------------- loops
def grouped(f):
    for idx in np.ndindex(*f.shape):
        yield Vector(list(idx))


def ndrange(*dims):
    ranges = [range(d[0], d[1]) if isinstance(d, (tuple, list)) else range(int(d)) for d in dims]
    if len(ranges) == 1:
        yield from ranges[0]
        return
    yield from itertools.product(*ranges)


# ---------------------------------------------------------------- math
def sqrt(x):
    return _m.sqrt(x)


def pow(x, n):  # noqa: A001 (Taichi's name)
    return x ** n


def exp(x):
    return _m.exp(x)


def log(x):
    return _m.log(x)


def abs(x):  # noqa: A001
    return x.__abs__()


def max(*a):  # noqa: A001
    return _builtins.max(*a)


def min(*a):  # noqa: A001
    return _builtins.min(*a)


def atomic_max(*a):
    raise NotImplementedError("stand-in: atomics are not emulated")


def atomic_min(*a):
    raise NotImplementedError("stand-in: atomics are not emulated")


def atomic_add(*a):
    raise NotImplementedError("stand-in: atomics are not emulated")
