"""Expression IR for model functions.

User functions (utility, constraints, laws of motion, regime transitions) are
written against a NumPy-like namespace (``pylcm_b200.jnp``).  When they are
called with :class:`Expr` arguments they build a small, hash-consed expression
DAG instead of computing numbers.  The DAG is what the CUDA code generator
emits, and it is also what the dependency analysis (state-only / action-only /
mixed) runs on.

The reference composes the same functions by argument name with ``dags``
(``src/_lcm/regime_building/Q_and_F.py:1321-1351``) and evaluates them under
JAX tracing; this module is the B200 build's replacement for that tracing step.

Node kinds (``Expr.op``):

``const``   literal (``args = (value,)``)
``var``     a named scalar input: ``args = (kind, name)`` with kind one of
            ``state``, ``action``, ``period``, ``age``
``param``   a scalar runtime parameter: ``args = (flat_name,)``
``pidx``    an element of an array parameter: ``args = (flat_name, idx...)``
``pgrid``   a process node value: ``args = (state_name, idx)``
``bin``     ``args = (opname, a, b)`` with opname in + - * / // % pow min max
``un``      ``args = (fname, a)`` elementwise math function
``cmp``     ``args = (opname, a, b)`` with opname in < <= > >= == !=
``where``   ``args = (cond, a, b)``
``and`` / ``or`` / ``not`` boolean connectives
``cast``    ``args = (dtype, a)``
"""

from __future__ import annotations

import math
import numbers
from typing import Any

import numpy as np

from pylcm_b200.exceptions import TracingError

# dtype tags: 'f' floating, 'i' integer, 'b' boolean
_FLOAT, _INT, _BOOL = "f", "i", "b"


def _promote(a: str, b: str) -> str:
    if _FLOAT in (a, b):
        return _FLOAT
    if _INT in (a, b):
        return _INT
    return _BOOL


_INTERN: dict[tuple, "Expr"] = {}


class Expr:
    """One node of the expression DAG (hash-consed: equal nodes are identical)."""

    __slots__ = ("op", "args", "dtype", "__weakref__", "_deps")

    def __new__(cls, op: str, args: tuple, dtype: str) -> "Expr":
        key = (op, tuple(_key_of(a) for a in args), dtype)
        hit = _INTERN.get(key)
        if hit is not None:
            return hit
        self = object.__new__(cls)
        self.op = op
        self.args = args
        self.dtype = dtype
        self._deps = None
        _INTERN[key] = self
        return self

    # ------------------------------------------------------------------ misc
    def __repr__(self) -> str:
        return f"Expr({self.op}, {self.args!r}, {self.dtype})"

    def __hash__(self) -> int:
        return id(self)

    def __eq__(self, other: Any) -> "Expr":  # type: ignore[override]
        return _cmp("==", self, other)

    def __ne__(self, other: Any) -> "Expr":  # type: ignore[override]
        return _cmp("!=", self, other)

    def __bool__(self) -> bool:
        raise TracingError(
            "A model function used a traced value in Python control flow "
            "(`if`, `and`, `or`, `bool(...)`). Use `jnp.where` / `&` / `|` instead."
        )

    def __index__(self) -> int:
        raise TracingError("A traced value cannot be used as a Python index.")

    def __float__(self) -> float:
        raise TracingError("A traced value cannot be converted to a Python float.")

    # ---------------------------------------------------------- arithmetic
    def __add__(self, o):
        return _bin("+", self, o)

    def __radd__(self, o):
        return _bin("+", o, self)

    def __sub__(self, o):
        return _bin("-", self, o)

    def __rsub__(self, o):
        return _bin("-", o, self)

    def __mul__(self, o):
        return _bin("*", self, o)

    def __rmul__(self, o):
        return _bin("*", o, self)

    def __truediv__(self, o):
        return _bin("/", self, o)

    def __rtruediv__(self, o):
        return _bin("/", o, self)

    def __floordiv__(self, o):
        return _bin("//", self, o)

    def __rfloordiv__(self, o):
        return _bin("//", o, self)

    def __mod__(self, o):
        return _bin("%", self, o)

    def __rmod__(self, o):
        return _bin("%", o, self)

    def __pow__(self, o):
        return _bin("pow", self, o)

    def __rpow__(self, o):
        return _bin("pow", o, self)

    def __neg__(self):
        return un("neg", self)

    def __pos__(self):
        return self

    def __abs__(self):
        return un("abs", self)

    def __lt__(self, o):
        return _cmp("<", self, o)

    def __le__(self, o):
        return _cmp("<=", self, o)

    def __gt__(self, o):
        return _cmp(">", self, o)

    def __ge__(self, o):
        return _cmp(">=", self, o)

    def __and__(self, o):
        return logical("and", self, o)

    def __rand__(self, o):
        return logical("and", o, self)

    def __or__(self, o):
        return logical("or", self, o)

    def __ror__(self, o):
        return logical("or", o, self)

    def __invert__(self):
        if self.dtype == _BOOL:
            return Expr("not", (self,), _BOOL)
        raise TracingError("bitwise not on a non-boolean traced value")

    def astype(self, dtype: Any) -> "Expr":
        tag = dtype_tag(dtype)
        if tag == self.dtype:
            return self
        return Expr("cast", (tag, self), tag)

    # -------------------------------------------------------- dependencies
    def deps(self) -> frozenset:
        """Set of (kind, name) inputs this node depends on."""
        if self._deps is None:
            if self.op == "var":
                self._deps = frozenset({(self.args[0], self.args[1])})
            elif self.op in ("param", "const"):
                self._deps = frozenset()
            else:
                out: set = set()
                for a in self.args:
                    if isinstance(a, Expr):
                        out |= a.deps()
                self._deps = frozenset(out)
        return self._deps


def _key_of(a: Any) -> Any:
    if isinstance(a, Expr):
        return ("E", id(a))
    if isinstance(a, float):
        # distinguish -0.0 / nan
        return ("F", a.hex() if not math.isnan(a) else "nan")
    return a


def dtype_tag(dtype: Any) -> str:
    if isinstance(dtype, str) and dtype in (_FLOAT, _INT, _BOOL):
        return dtype
    kind = np.dtype(dtype).kind
    if kind == "f":
        return _FLOAT
    if kind in "iu":
        return _INT
    if kind == "b":
        return _BOOL
    raise TracingError(f"unsupported dtype {dtype!r}")


def const(value: Any) -> Expr:
    if isinstance(value, Expr):
        return value
    if isinstance(value, (bool, np.bool_)):
        return Expr("const", (bool(value),), _BOOL)
    if isinstance(value, (numbers.Integral, np.integer)):
        return Expr("const", (int(value),), _INT)
    if isinstance(value, (numbers.Real, np.floating)):
        return Expr("const", (float(value),), _FLOAT)
    if isinstance(value, np.ndarray) and value.ndim == 0:
        return const(value.item())
    raise TracingError(f"cannot use {type(value).__name__} as a traced scalar")


def var(kind: str, name: str, dtype: str) -> Expr:
    return Expr("var", (kind, name), dtype)


def param(flat_name: str, dtype: str = _FLOAT) -> Expr:
    return Expr("param", (flat_name,), dtype)


def is_const(e: Any) -> bool:
    return isinstance(e, Expr) and e.op == "const"


def _fold_bin(op: str, x: Any, y: Any) -> Any:
    if op == "+":
        return x + y
    if op == "-":
        return x - y
    if op == "*":
        return x * y
    if op == "/":
        return x / y
    if op == "//":
        return x // y
    if op == "%":
        return x % y
    if op == "pow":
        return x**y
    if op == "min":
        return min(x, y)
    if op == "max":
        return max(x, y)
    raise AssertionError(op)


def _bin(op: str, a: Any, b: Any) -> Any:
    if isinstance(a, VecExpr) or isinstance(b, VecExpr):
        return VecExpr.broadcast2(lambda x, y: _bin(op, x, y), a, b)
    a = const(a)
    b = const(b)
    if a.op == "const" and b.op == "const":
        try:
            return const(_fold_bin(op, a.args[0], b.args[0]))
        except ZeroDivisionError:
            pass
    if op == "/":
        dt = _FLOAT
    elif op == "pow":
        dt = _FLOAT if _FLOAT in (a.dtype, b.dtype) else _INT
    else:
        dt = _promote(a.dtype, b.dtype)
        if dt == _BOOL:
            dt = _INT
    return Expr("bin", (op, a, b), dt)


def _cmp(op: str, a: Any, b: Any) -> Any:
    if isinstance(a, VecExpr) or isinstance(b, VecExpr):
        return VecExpr.broadcast2(lambda x, y: _cmp(op, x, y), a, b)
    a = const(a)
    b = const(b)
    return Expr("cmp", (op, a, b), _BOOL)


def un(fname: str, a: Any) -> Any:
    if isinstance(a, VecExpr):
        return VecExpr([un(fname, x) for x in a.items])
    a = const(a)
    if fname in ("neg", "abs"):
        dt = a.dtype if a.dtype != _BOOL else _INT
    elif fname in ("floor", "ceil", "round", "trunc"):
        dt = _FLOAT
    elif fname in ("isfinite", "isnan", "isinf", "signbit"):
        dt = _BOOL
    else:
        dt = _FLOAT
    if a.op == "const" and fname == "neg":
        return const(-a.args[0])
    return Expr("un", (fname, a), dt)


def logical(op: str, a: Any, b: Any) -> Any:
    if isinstance(a, VecExpr) or isinstance(b, VecExpr):
        return VecExpr.broadcast2(lambda x, y: logical(op, x, y), a, b)
    a = const(a)
    b = const(b)
    if a.dtype != _BOOL or b.dtype != _BOOL:
        # bitwise ops on integers are not part of the supported subset
        raise TracingError(f"'{op}' needs boolean operands, got {a.dtype}/{b.dtype}")
    return Expr(op, (a, b), _BOOL)


def where(c: Any, a: Any, b: Any) -> Any:
    if any(isinstance(x, VecExpr) for x in (c, a, b)):
        return VecExpr.broadcast3(where, c, a, b)
    c = const(c)
    a = const(a)
    b = const(b)
    if c.dtype != _BOOL:
        c = _cmp("!=", c, 0)
    if c.op == "const":
        return a if c.args[0] else b
    dt = _promote(a.dtype, b.dtype)
    return Expr("where", (c, a, b), dt)


class VecExpr:
    """A short vector of scalar expressions (e.g. ``jnp.array([p, 1 - p])``)."""

    __slots__ = ("items",)

    def __init__(self, items: list) -> None:
        self.items = [const(x) if not isinstance(x, VecExpr) else x for x in items]
        for x in self.items:
            if isinstance(x, VecExpr):
                raise TracingError("nested vectors are not supported")

    def __len__(self) -> int:
        return len(self.items)

    def __getitem__(self, idx: Any) -> Any:
        if isinstance(idx, (int, np.integer)):
            return self.items[int(idx)]
        if isinstance(idx, Expr) and idx.op == "const":
            return self.items[int(idx.args[0])]
        if isinstance(idx, Expr):
            # select by traced index: chain of wheres
            out = self.items[-1]
            for k in range(len(self.items) - 2, -1, -1):
                out = where(_cmp("==", idx, k), self.items[k], out)
            return out
        raise TracingError(f"unsupported vector index {idx!r}")

    @staticmethod
    def _as_vec(x: Any, n: int) -> list:
        if isinstance(x, VecExpr):
            if len(x) != n:
                raise TracingError("vector length mismatch")
            return x.items
        return [x] * n

    @staticmethod
    def broadcast2(fn, a, b) -> "VecExpr":
        n = len(a) if isinstance(a, VecExpr) else len(b)
        return VecExpr([fn(x, y) for x, y in zip(VecExpr._as_vec(a, n), VecExpr._as_vec(b, n))])

    @staticmethod
    def broadcast3(fn, a, b, c) -> "VecExpr":
        n = next(len(x) for x in (a, b, c) if isinstance(x, VecExpr))
        return VecExpr(
            [
                fn(x, y, z)
                for x, y, z in zip(
                    VecExpr._as_vec(a, n), VecExpr._as_vec(b, n), VecExpr._as_vec(c, n)
                )
            ]
        )

    def __add__(self, o):
        return _bin("+", self, o)

    def __radd__(self, o):
        return _bin("+", o, self)

    def __sub__(self, o):
        return _bin("-", self, o)

    def __rsub__(self, o):
        return _bin("-", o, self)

    def __mul__(self, o):
        return _bin("*", self, o)

    def __rmul__(self, o):
        return _bin("*", o, self)

    def __truediv__(self, o):
        return _bin("/", self, o)

    def __rtruediv__(self, o):
        return _bin("/", o, self)

    def __neg__(self):
        return un("neg", self)

    def sum(self) -> Expr:
        out = self.items[0]
        for x in self.items[1:]:
            out = _bin("+", out, x)
        return out


class ParamArray:
    """An array-valued runtime parameter seen by a traced function.

    Indexing it with traced integer scalars yields ``pidx`` nodes; indexing with
    fewer indices than dimensions yields a :class:`VecExpr` over the last axis.
    """

    __slots__ = ("flat_name", "shape")

    def __init__(self, flat_name: str, shape: tuple[int, ...]) -> None:
        self.flat_name = flat_name
        self.shape = tuple(int(s) for s in shape)

    @property
    def ndim(self) -> int:
        return len(self.shape)

    def __len__(self) -> int:
        return self.shape[0]

    def __getitem__(self, idx: Any) -> Any:
        if not isinstance(idx, tuple):
            idx = (idx,)
        idx = tuple(const(i) for i in idx)
        for i in idx:
            if i.dtype == _FLOAT:
                raise TracingError(f"array parameter {self.flat_name!r} indexed by a float")
        if len(idx) > self.ndim:
            raise TracingError(f"too many indices for array parameter {self.flat_name!r}")
        if len(idx) == self.ndim:
            return Expr("pidx", (self.flat_name, *idx), _FLOAT)
        if len(idx) == self.ndim - 1:
            return VecExpr(
                [Expr("pidx", (self.flat_name, *idx, const(k)), _FLOAT) for k in range(self.shape[-1])]
            )
        raise TracingError(
            f"array parameter {self.flat_name!r} must be indexed down to at most one axis"
        )


def is_traced(x: Any) -> bool:
    return isinstance(x, (Expr, VecExpr, ParamArray))


def topo_order(roots: list) -> list[Expr]:
    """Post-order (dependencies first) list of the unique nodes under `roots`."""
    seen: set[int] = set()
    order: list[Expr] = []
    stack: list[tuple[Expr, bool]] = []
    for r in roots:
        if isinstance(r, Expr):
            stack.append((r, False))
        while stack:
            node, done = stack.pop()
            if done:
                order.append(node)
                continue
            if id(node) in seen:
                continue
            seen.add(id(node))
            stack.append((node, True))
            for a in reversed(node.args):
                if isinstance(a, Expr) and id(a) not in seen:
                    stack.append((a, False))
    return order


def evaluate(expr: Any, env: dict, params: dict, pgrid: dict | None = None) -> Any:
    """Evaluate an IR expression with NumPy (host-side helper).

    `env` maps (kind, name) -> array; `params` maps flat_name -> array/scalar;
    `pgrid` maps state_name -> node values.  Used for host-side lottery tables
    and in tests; the device path never calls it.
    """
    if isinstance(expr, VecExpr):
        return [evaluate(x, env, params, pgrid) for x in expr.items]
    cache: dict[int, Any] = {}
    for node in topo_order([expr]):
        cache[id(node)] = _eval_node(node, cache, env, params, pgrid)
    return cache[id(expr)]


def _eval_node(node: Expr, cache, env, params, pgrid):
    op = node.op
    A = [cache[id(a)] if isinstance(a, Expr) else a for a in node.args]
    if op == "const":
        return A[0]
    if op == "var":
        return env[(A[0], A[1])]
    if op == "param":
        return params[A[0]]
    if op == "pidx":
        arr = np.asarray(params[A[0]])
        idx = tuple(np.asarray(i).astype(np.int64) for i in A[1:])
        return arr[idx]
    if op == "pgrid":
        return np.asarray(pgrid[A[0]])[np.asarray(A[1]).astype(np.int64)]
    if op == "bin":
        o, x, y = A
        with np.errstate(all="ignore"):
            if o == "pow":
                if not isinstance(node.args[2], Expr) or node.args[2].op != "const":
                    return np.power(np.asarray(x, dtype=float), y)
                return np.power(np.asarray(x, dtype=float) if node.dtype == _FLOAT else x, y)
            if o == "/":
                return np.true_divide(x, y)
            if o == "min":
                return np.minimum(x, y)
            if o == "max":
                return np.maximum(x, y)
            return _fold_bin(o, x, y)
    if op == "un":
        f, x = A
        with np.errstate(all="ignore"):
            return _NP_UNARY[f](x)
    if op == "cmp":
        o, x, y = A
        return {
            "<": np.less,
            "<=": np.less_equal,
            ">": np.greater,
            ">=": np.greater_equal,
            "==": np.equal,
            "!=": np.not_equal,
        }[o](x, y)
    if op == "where":
        return np.where(A[0], A[1], A[2])
    if op == "and":
        return np.logical_and(A[0], A[1])
    if op == "or":
        return np.logical_or(A[0], A[1])
    if op == "not":
        return np.logical_not(A[0])
    if op == "cast":
        t, x = A
        return np.asarray(x).astype({"f": np.float64, "i": np.int64, "b": np.bool_}[t])
    raise AssertionError(op)


_NP_UNARY = {
    "neg": np.negative,
    "abs": np.abs,
    "log": np.log,
    "log1p": np.log1p,
    "log2": np.log2,
    "log10": np.log10,
    "exp": np.exp,
    "expm1": np.expm1,
    "exp2": np.exp2,
    "sqrt": np.sqrt,
    "cbrt": np.cbrt,
    "sin": np.sin,
    "cos": np.cos,
    "tan": np.tan,
    "tanh": np.tanh,
    "sinh": np.sinh,
    "cosh": np.cosh,
    "arctan": np.arctan,
    "floor": np.floor,
    "ceil": np.ceil,
    "round": np.round,
    "trunc": np.trunc,
    "isfinite": np.isfinite,
    "isnan": np.isnan,
    "isinf": np.isinf,
    "signbit": np.signbit,
    "erf": None,  # filled lazily below
}


def _erf(x):
    from scipy.special import erf

    return erf(x)


_NP_UNARY["erf"] = _erf


def diff(expr: Any, wrt: Expr) -> Expr:
    """Symbolic derivative of a scalar expression with respect to a variable.

    Used where the reference differentiates with ``jax.grad``: the marginal
    utility u'(c) of the EGM carry rows and the savings derivative dR'/dA of
    the law of motion.  Non-differentiable pieces (comparisons, floor, integer
    arithmetic) have derivative zero; ``where`` differentiates its branches.
    """
    memo: dict[int, Expr] = {}
    zero, one = const(0.0), const(1.0)

    def d(e: Expr) -> Expr:
        if id(e) in memo:
            return memo[id(e)]
        r = _d(e)
        memo[id(e)] = r
        return r

    def _d(e: Expr) -> Expr:
        if e is wrt:
            return one
        if e.dtype != _FLOAT or e.op in ("const", "param", "pidx", "var", "pgrid"):
            return zero
        if not any(x is wrt or (isinstance(x, Expr) and wrt in _leaves(x)) for x in e.args if isinstance(x, Expr)):
            return zero
        if e.op == "bin":
            o, a, b = e.args
            da, db = d(a), d(b)
            za, zb = _is_zero(da), _is_zero(db)  # a symbolic zero derivative drops its term
            if o == "+":
                return db if za else (da if zb else da + db)
            if o == "-":
                return -db if za else (da if zb else da - db)
            if o == "*":
                if za:
                    return a * db
                if zb:
                    return da * b
                return da * b + a * db
            if o == "/":
                if zb:
                    return da / b
                return (da * b - a * db) / (b * b)
            if o == "pow":
                # a**b: b * a**(b-1) * da + log(a) * a**b * db
                out = zero
                if not (isinstance(db, Expr) and db.op == "const" and db.args[0] == 0.0):
                    out = out + un("log", a) * e * db
                if not (isinstance(da, Expr) and da.op == "const" and da.args[0] == 0.0):
                    out = out + b * _bin("pow", a, b - 1.0) * da
                return out
            if o == "min":
                return where(_cmp("<=", a, b), da, db)
            if o == "max":
                return where(_cmp(">=", a, b), da, db)
            return zero
        if e.op == "un":
            f, a = e.args
            da = d(a)
            table = {
                "neg": lambda: -da,
                "log": lambda: da / a,
                "log1p": lambda: da / (1.0 + a),
                "exp": lambda: e * da,
                "expm1": lambda: un("exp", a) * da,
                "sqrt": lambda: da / (2.0 * e),
                "abs": lambda: where(_cmp(">=", a, 0.0), da, -da),
                "sin": lambda: un("cos", a) * da,
                "cos": lambda: -un("sin", a) * da,
                "tanh": lambda: (1.0 - e * e) * da,
            }
            if f in table:
                return table[f]()
            return zero
        if e.op == "where":
            c, a, b = e.args
            return where(c, d(a), d(b))
        if e.op == "cast":
            return d(e.args[1]) if e.args[0] == _FLOAT else zero
        return zero

    return const(d(const(expr)))


def _is_zero(x: Any) -> bool:
    return isinstance(x, Expr) and x.op == "const" and x.args[0] == 0.0


def _leaves(e: Expr) -> set:
    out = getattr(e, "_leaf_cache", None)
    if out is None:
        out = {id(n) for n in topo_order([e])}
    return _IdSet(out)


class _IdSet:
    __slots__ = ("ids",)

    def __init__(self, ids: set) -> None:
        self.ids = ids

    def __contains__(self, x: Any) -> bool:
        return id(x) in self.ids


def substitute(expr: Any, wrt: Expr, value: float) -> Expr:
    """`expr` with the variable `wrt` replaced by the constant `value` (nodes
    rebuilt bottom-up; nodes without `wrt` below them are kept)."""
    e0 = const(expr)
    rep = const(value)
    new: dict[int, Any] = {}
    for n in topo_order([e0]):
        if n is wrt:
            new[id(n)] = rep
            continue
        args = tuple(new.get(id(a), a) if isinstance(a, Expr) else a for a in n.args)
        if all(x is y for x, y in zip(args, n.args)):
            new[id(n)] = n
        else:
            new[id(n)] = Expr(n.op, args, n.dtype)
    return new[id(e0)]
