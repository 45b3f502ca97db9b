"""``ti.math`` subset for the sequential Taichi stand-in (test infrastructure only)."""
import math as _m


def length(v):
    return _m.sqrt(v.dot(v))


def dot(a, b):
    return a.dot(b)


def exp(x):
    return _m.exp(x)


def sqrt(x):
    return _m.sqrt(x)


def log(x):
    return _m.log(x)
