"""NumPy-like namespace for model functions.

Model functions written for the reference call ``jnp.log``, ``jnp.where``,
``jnp.exp``, ``jnp.array([...])`` and friends.  Import this module as ``jnp``
in model code.  Every function here works on two kinds of input:

- traced values (:mod:`pylcm_b200.ir` expressions): the call builds IR nodes,
  which is how the solver lowers the model to CUDA C;
- ordinary numbers / NumPy arrays: the call is forwarded to NumPy, which is how
  host-side helpers and the CPU oracle evaluate the same functions.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from pylcm_b200 import ir

inf = np.inf
nan = np.nan
pi = np.pi
e = np.e
float64 = np.float64
float32 = np.float32
int32 = np.int32
int64 = np.int64
bool_ = np.bool_


def _any_traced(*xs: Any) -> bool:
    return any(ir.is_traced(x) for x in xs)


def _unary(name: str, npfn):
    def f(x):
        if _any_traced(x):
            return ir.un(name, x)
        return npfn(x)

    f.__name__ = name
    return f


log = _unary("log", np.log)
log1p = _unary("log1p", np.log1p)
log2 = _unary("log2", np.log2)
log10 = _unary("log10", np.log10)
exp = _unary("exp", np.exp)
expm1 = _unary("expm1", np.expm1)
exp2 = _unary("exp2", np.exp2)
sqrt = _unary("sqrt", np.sqrt)
cbrt = _unary("cbrt", np.cbrt)
sin = _unary("sin", np.sin)
cos = _unary("cos", np.cos)
tan = _unary("tan", np.tan)
tanh = _unary("tanh", np.tanh)
sinh = _unary("sinh", np.sinh)
cosh = _unary("cosh", np.cosh)
arctan = _unary("arctan", np.arctan)
floor = _unary("floor", np.floor)
ceil = _unary("ceil", np.ceil)
round = _unary("round", np.round)  # noqa: A001
trunc = _unary("trunc", np.trunc)
isfinite = _unary("isfinite", np.isfinite)
isnan = _unary("isnan", np.isnan)
isinf = _unary("isinf", np.isinf)
signbit = _unary("signbit", np.signbit)
abs = _unary("abs", np.abs)  # noqa: A001
absolute = abs
negative = _unary("neg", np.negative)


def square(x):
    return x * x


def power(x, y):
    if _any_traced(x, y):
        return ir._bin("pow", x, y)
    return np.power(x, y)


float_power = power


def maximum(x, y):
    if _any_traced(x, y):
        return ir._bin("max", x, y)
    return np.maximum(x, y)


def minimum(x, y):
    if _any_traced(x, y):
        return ir._bin("min", x, y)
    return np.minimum(x, y)


def clip(x, a_min=None, a_max=None):
    out = x
    if a_min is not None:
        out = maximum(out, a_min)
    if a_max is not None:
        out = minimum(out, a_max)
    return out


def where(cond, x, y):
    if _any_traced(cond, x, y):
        return ir.where(cond, x, y)
    return np.where(cond, x, y)


def logical_and(x, y):
    if _any_traced(x, y):
        return ir.logical("and", x, y)
    return np.logical_and(x, y)


def logical_or(x, y):
    if _any_traced(x, y):
        return ir.logical("or", x, y)
    return np.logical_or(x, y)


def logical_not(x):
    if _any_traced(x):
        return ~x
    return np.logical_not(x)


def array(obj, dtype=None):
    if isinstance(obj, (list, tuple)) and _any_traced(*obj):
        vec = ir.VecExpr(list(obj))
        if dtype is not None:
            vec = ir.VecExpr([ir.const(x).astype(dtype) for x in vec.items])
        return vec
    if ir.is_traced(obj):
        return obj
    return np.array(obj, dtype=dtype)


asarray = array


def sum(x, axis=None):  # noqa: A001
    if isinstance(x, ir.VecExpr):
        return x.sum()
    return np.sum(x, axis=axis)


def full(shape, fill_value, dtype=None):
    return np.full(shape, fill_value, dtype=dtype)


def zeros(shape, dtype=None):
    return np.zeros(shape, dtype=dtype)


def ones(shape, dtype=None):
    return np.ones(shape, dtype=dtype)


def linspace(start, stop, num, **kw):
    return np.linspace(start, stop, num, **kw)


def erf(x):
    if _any_traced(x):
        return ir.un("erf", x)
    from scipy.special import erf as _erf

    return _erf(x)
