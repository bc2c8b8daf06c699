"""Lower a traced regime to CUDA C for sm_100a.

Two kernels are generated per (regime, set of next-period targets):

``lcm_bellman_<tag>`` -- kernel (a), the fused Q_and_F + max/argmax step.
    One CTA owns a tile of ``BLOCK / LANES`` states; ``LANES`` consecutive
    threads share a state and stride over its actions.  Actions are processed
    in chunks whose action-only sub-expressions (typically the utility) are
    evaluated once per chunk into shared memory; state-only sub-expressions are
    evaluated once per thread; only the mixed part runs in the inner loop.
    Infeasible actions are rejected before the continuation is touched.  The
    running (max, first argmax) is combined across lanes with warp shuffles.

``lcm_expect_<tag>_<target>`` -- kernel (b), the shock expectation
    EV[k, col] = sum_j W[k, j] V'[j, col] / sum_j W[k, j]
    where j runs over the target's stochastic node axes (Markov laws and
    processes), k over the discrete inputs the weights depend on, and col over
    the remaining (deterministic discrete x continuous) axes.  The weight
    table is built in shared memory per tile; each thread owns one column and
    keeps all k accumulators in registers, so V' is read once.

Precision modes: ``fp64`` runs both kernels in double precision.  ``fp32``
runs the inner search of (a) in single precision on a float copy of EV and then
re-evaluates Q at the chosen action in double precision from the double EV, so
the published V is a double-precision Bellman value at the single-precision
argmax.

Reference semantics restated here: ``Q_and_F.py:138-168, 466-681, 1145-1209``,
``max_Q_over_a.py:160``, ``argmax.py:6-69``, ``ndimage.py:29-109``,
``coordinates.py:30-167``.
"""

from __future__ import annotations

import dataclasses
import hashlib
import math
from pathlib import Path

import numpy as np

from pylcm_b200 import ir
from pylcm_b200.exceptions import TracingError
from pylcm_b200.spec import RegimeSpec, TracedRegime, proc_P_name

KERNEL_DIR = Path(__file__).resolve().parent / "csrc" / "kernels"


def device_header() -> str:
    return (KERNEL_DIR / "lcm_device.cuh").read_text()


# ---------------------------------------------------------------------------
# expression emission
# ---------------------------------------------------------------------------
_CMP = {"<": "<", "<=": "<=", ">": ">", ">=": ">=", "==": "==", "!=": "!="}
_UNARY_C = {
    "log": "log",
    "log1p": "log1p",
    "log2": "log2",
    "log10": "log10",
    "exp": "exp",
    "expm1": "expm1",
    "exp2": "exp2",
    "sqrt": "sqrt",
    "cbrt": "cbrt",
    "sin": "sin",
    "cos": "cos",
    "tan": "tan",
    "tanh": "tanh",
    "sinh": "sinh",
    "cosh": "cosh",
    "arctan": "atan",
    "floor": "floor",
    "ceil": "ceil",
    "round": "rint",
    "trunc": "trunc",
    "erf": "erf",
}


def _c_float(v: float, ftype: str) -> str:
    if math.isnan(v):
        return f"lcm_lim<{ftype}>::nan()"
    if math.isinf(v):
        return f"({'-' if v < 0 else ''}lcm_lim<{ftype}>::inf())"
    r = repr(float(v))
    if "e" not in r and "." not in r and "inf" not in r:
        r += ".0"
    return f"(({ftype}){r})"


class Emitter:
    """Emits C statements for IR nodes, memoising node -> C expression."""

    def __init__(self, ftype: str, param_off: dict, provided: dict, prefix: str) -> None:
        self.ftype = ftype
        self.param_off = param_off  # flat name -> (offset, shape)
        self.vals: dict[int, str] = dict(provided)  # id(node) -> C expression
        self.lines: list[str] = []
        self.prefix = prefix
        self.n = 0

    def ctype(self, dt: str) -> str:
        return {"f": self.ftype, "i": "int", "b": "bool"}[dt]

    def emit(self, node: ir.Expr) -> str:
        if id(node) in self.vals:
            return self.vals[id(node)]
        # post-order walk that stops at nodes already bound (provided / emitted)
        stack: list[tuple[ir.Expr, bool]] = [(node, False)]
        while stack:
            n, done = stack.pop()
            if id(n) in self.vals:
                continue
            if done:
                self.vals[id(n)] = self._emit_one(n)
                continue
            stack.append((n, True))
            for a in reversed(n.args):
                if isinstance(a, ir.Expr) and id(a) not in self.vals:
                    stack.append((a, False))
        return self.vals[id(node)]

    def _tmp(self, dt: str, expr: str) -> str:
        name = f"{self.prefix}{self.n}"
        self.n += 1
        self.lines.append(f"{self.ctype(dt)} {name} = {expr};")
        return name

    def _arg(self, a: ir.Expr, want: str | None = None) -> str:
        s = self.vals[id(a)]
        if want == "f" and a.dtype != "f":
            return f"(({self.ftype}){s})"
        return s

    def _emit_one(self, n: ir.Expr) -> str:
        op = n.op
        ft = self.ftype
        if op == "const":
            v = n.args[0]
            if n.dtype == "b":
                return "true" if v else "false"
            if n.dtype == "i":
                return f"({int(v)})"
            return _c_float(v, ft)
        if op == "var":
            raise TracingError(f"internal: unbound variable {n.args}")
        if op == "param":
            off, shape = self.param_off[n.args[0]]
            return self._tmp("f", f"(({ft})PV[{off}])")
        if op == "pidx":
            name = n.args[0]
            off, shape = self.param_off[name]
            idx = [self._arg(a) for a in n.args[1:]]
            if len(idx) != len(shape):
                raise TracingError(f"array parameter {name} needs {len(shape)} indices")
            # JAX clamps out-of-range gathers; clamp likewise (and stay in bounds)
            lin = "0"
            for k, (i, s) in enumerate(zip(idx, shape)):
                ci = f"min(max((int)({i}), 0), {s - 1})"
                lin = ci if k == 0 else f"({lin}) * {s} + {ci}"
            return self._tmp("f", f"(({ft})PV[{off} + {lin}])")
        if op == "bin":
            o, a, b = n.args
            if n.dtype == "f":
                xa, xb = self._arg(a, "f"), self._arg(b, "f")
            else:
                xa, xb = self._arg(a), self._arg(b)
            if o in "+-*":
                return self._tmp(n.dtype, f"{xa} {o} {xb}")
            if o == "/":
                return self._tmp("f", f"{xa} / {xb}")
            if o == "//":
                if n.dtype == "f":
                    return self._tmp("f", f"floor({xa} / {xb})")
                return self._tmp("i", f"lcm_floordiv({xa}, {xb})")
            if o == "%":
                if n.dtype == "f":
                    return self._tmp("f", f"({xa} - floor({xa} / {xb}) * {xb})")
                return self._tmp("i", f"lcm_floormod({xa}, {xb})")
            if o == "pow":
                if b.op == "const" and b.dtype in ("i", "f") and float(b.args[0]) == 2.0:
                    return self._tmp(n.dtype, f"{xa} * {xa}")
                if n.dtype == "i":
                    return self._tmp("i", f"(int)rint(pow((double){xa}, (double){xb}))")
                return self._tmp("f", f"pow({xa}, {xb})")
            if o == "min":
                if n.dtype == "f":
                    return self._tmp("f", f"lcm_min({xa}, {xb})")
                return self._tmp(n.dtype, f"min({xa}, {xb})")
            if o == "max":
                if n.dtype == "f":
                    return self._tmp("f", f"lcm_max({xa}, {xb})")
                return self._tmp(n.dtype, f"max({xa}, {xb})")
            raise TracingError(f"unsupported binary op {o}")
        if op == "un":
            f, a = n.args
            x = self._arg(a, "f" if n.dtype == "f" else None)
            if f == "neg":
                return self._tmp(n.dtype, f"-{x}")
            if f == "abs":
                return self._tmp(n.dtype, f"fabs({x})" if n.dtype == "f" else f"abs({x})")
            if f == "isfinite":
                return self._tmp("b", f"lcm_isfinite(({ft}){x})")
            if f == "isnan":
                return self._tmp("b", f"lcm_isnan(({ft}){x})")
            if f == "isinf":
                return self._tmp("b", f"(!lcm_isfinite(({ft}){x}) && !lcm_isnan(({ft}){x}))")
            if f == "signbit":
                return self._tmp("b", f"signbit(({ft}){x})")
            if f in _UNARY_C:
                return self._tmp("f", f"{_UNARY_C[f]}(({ft}){x})")
            raise TracingError(f"unsupported function {f}")
        if op == "cmp":
            o, a, b = n.args
            if "f" in (a.dtype, b.dtype):
                xa, xb = self._arg(a, "f"), self._arg(b, "f")
            else:
                xa, xb = self._arg(a), self._arg(b)
            return self._tmp("b", f"{xa} {_CMP[o]} {xb}")
        if op == "where":
            c, a, b = n.args
            want = "f" if n.dtype == "f" else None
            return self._tmp(n.dtype, f"{self._arg(c)} ? {self._arg(a, want)} : {self._arg(b, want)}")
        if op == "and":
            return self._tmp("b", f"{self._arg(n.args[0])} && {self._arg(n.args[1])}")
        if op == "or":
            return self._tmp("b", f"{self._arg(n.args[0])} || {self._arg(n.args[1])}")
        if op == "not":
            return self._tmp("b", f"!{self._arg(n.args[0])}")
        if op == "cast":
            t, a = n.args
            x = self._arg(a)
            if t == "f":
                return self._tmp("f", f"(({ft}){x})")
            if t == "i":
                if a.dtype == "f":
                    return self._tmp("i", f"(int)trunc({x})")
                return self._tmp("i", f"(int)({x})")
            return self._tmp("b", f"(({x}) != 0)")
        raise TracingError(f"unsupported IR op {op}")


_EXTRA_DEVICE = r"""
__device__ __forceinline__ int lcm_floordiv(int a, int b) { int q = a / b; return (q * b != a && ((a < 0) != (b < 0))) ? q - 1 : q; }
__device__ __forceinline__ int lcm_floormod(int a, int b) { int m = a % b; return (m != 0 && ((m < 0) != (b < 0))) ? m + b : m; }
// NaN-propagating min/max (jnp.minimum / jnp.maximum semantics)
__device__ __forceinline__ double lcm_min(double a, double b) { return (a != a || b != b) ? a + b : (a < b ? a : b); }
__device__ __forceinline__ double lcm_max(double a, double b) { return (a != a || b != b) ? a + b : (a > b ? a : b); }
__device__ __forceinline__ float lcm_min(float a, float b) { return (a != a || b != b) ? a + b : (a < b ? a : b); }
__device__ __forceinline__ float lcm_max(float a, float b) { return (a != a || b != b) ? a + b : (a > b ? a : b); }
template <typename E> struct lcm_evsel;
template <> struct lcm_evsel<double> { static __device__ __forceinline__ const double* get(const i64* it, int w64, int w32) { return reinterpret_cast<const double*>(it[w64]); } };
template <> struct lcm_evsel<float> { static __device__ __forceinline__ const float* get(const i64* it, int w64, int w32) { return reinterpret_cast<const float*>(it[w32]); } };
"""


def _phase(node: ir.Expr) -> str:
    d = node.deps()
    has_s = any(k == "state" for k, _ in d)
    has_a = any(k == "action" for k, _ in d)
    if has_s and has_a:
        return "SA"
    if has_s:
        return "S"
    if has_a:
        return "A"
    return "P"


def _boundary(roots: list[ir.Expr]) -> list[ir.Expr]:
    """Non-SA nodes whose values the SA phase consumes (roots included)."""
    out: dict[int, ir.Expr] = {}
    seen: set[int] = set()
    stack = [r for r in roots if isinstance(r, ir.Expr)]
    while stack:
        n = stack.pop()
        if id(n) in seen:
            continue
        seen.add(id(n))
        if n.op == "const":
            continue
        if _phase(n) != "SA":
            out[id(n)] = n
            continue
        for a in n.args:
            if isinstance(a, ir.Expr):
                stack.append(a)
    return list(out.values())


@dataclasses.dataclass
class TargetPlan:
    spec: RegimeSpec
    scalar: bool
    prob: ir.Expr
    stoch_pos: list[int]  # positions (in target state order) of stochastic axes
    det_pos: list[int]
    cont_pos: list[int]
    key_vars: list[tuple[str, str, int]]  # (kind, name, size) in key order
    laws: dict
    w_ev64: int = -1
    w_ev32: int = -1
    w_sizes: int = -1
    w_coord: int = -1
    w_scalar: int = -1

    @property
    def K(self) -> int:
        return int(np.prod([s for _, _, s in self.key_vars])) if self.key_vars else 1

    @property
    def J(self) -> int:
        return int(np.prod([self.spec.states[p].size for p in self.stoch_pos])) if self.stoch_pos else 1

    @property
    def needs_contraction(self) -> bool:
        return bool(self.stoch_pos)


def _target_plan(tr: TracedRegime, tgt: RegimeSpec) -> TargetPlan:
    spec = tr.spec
    prob = tr.regime_probs[tgt.rid]
    if not tgt.states:
        return TargetPlan(tgt, True, prob, [], [], [], [], {})
    laws = tr.next_states[tgt.name]
    stoch, det, cont = [], [], []
    key_deps: set = set()
    for pos, ax in enumerate(tgt.states):
        law = laws[ax.name]
        if law.kind in ("markov", "process"):
            stoch.append(pos)
            if law.kind == "process":
                key_deps.add(("state", law.source_process))
            else:
                for it in law.expr.items:
                    key_deps |= set(it.deps())
        elif law.kind == "det":
            det.append(pos)
        else:
            cont.append(pos)
    key_vars = []
    for ax in spec.states:
        if ("state", ax.name) in key_deps:
            if ax.kind == "continuous":
                raise TracingError(
                    f"{spec.name}->{tgt.name}: transition weights that depend on the continuous "
                    f"state {ax.name!r} are not supported"
                )
            key_vars.append(("state", ax.name, ax.size))
    for ax in spec.actions:
        if ("action", ax.name) in key_deps:
            if ax.kind == "continuous":
                raise TracingError(
                    f"{spec.name}->{tgt.name}: transition weights that depend on the continuous "
                    f"action {ax.name!r} are not supported"
                )
            key_vars.append(("action", ax.name, ax.size))
    return TargetPlan(tgt, False, prob, stoch, det, cont, key_vars, laws)


@dataclasses.dataclass(frozen=True)
class LaunchConfig:
    block: int = 256
    lanes: int = 1
    chunk: int = 512

    @property
    def states_per_tile(self) -> int:
        return self.block // self.lanes


class RegimeKernels:
    """Generated source + item-record layout for one regime / target set."""

    def __init__(
        self,
        tr: TracedRegime,
        targets: list[RegimeSpec],
        precision: str,
        cfg: LaunchConfig,
    ) -> None:
        if precision not in ("fp64", "fp32"):
            raise ValueError(precision)
        self.tr = tr
        self.spec = tr.spec
        self.precision = precision
        self.cfg = cfg
        self.param_off, self.param_len = tr.param_layout()
        order = sorted(targets, key=lambda s: (bool(s.states), s.rid))
        self.targets = [_target_plan(tr, t) for t in order] if not self.spec.terminal else []
        self._layout()
        tag_src = repr(
            (self.spec.name, [t.spec.name for t in self.targets], precision, dataclasses.astuple(cfg))
        )
        self.tag = self.spec.name.replace("-", "_") + "_" + hashlib.sha1(tag_src.encode()).hexdigest()[:8]

    # -------------------------------------------------------------- layout
    def _layout(self) -> None:
        spec = self.spec
        w = 0

        def take(n: int = 1) -> int:
            nonlocal w
            k = w
            w += n
            return k

        self.W_P = take()
        self.W_V = take()
        self.W_POL = take()
        self.W_PERIOD = take()
        self.W_AGE = take()
        self.W_NSTATES = take()
        self.W_NACT = take()
        self.W_SSIZE = take(len(spec.states))
        self.W_SGRID = take(len(spec.states))
        self.W_ASIZE = take(len(spec.actions))
        self.W_AGRID = take(len(spec.actions))
        self.W_TASTE = take()
        for t in self.targets:
            if t.scalar:
                t.w_scalar = take()
            else:
                t.w_ev64 = take()
                t.w_ev32 = take()
                t.w_sizes = take(len(t.spec.states))
                t.w_coord = take(3 * len(t.cont_pos))
        self.n_words = max(w, 1)

    # -------------------------------------------------------------- source
    def source(self) -> str:
        parts = [device_header(), _EXTRA_DEVICE, self._bellman_source()]
        for t in self.targets:
            if not t.scalar and (t.needs_contraction or self.precision == "fp32"):
                parts.append(self._expect_source(t))
        return "\n".join(parts)

    def e_words_for(self, t: TargetPlan) -> int:
        return 8 + len(t.spec.states)

    def bellman_name(self) -> str:
        return f"lcm_bellman_{self.tag}"

    def expect_name(self, t: TargetPlan) -> str:
        return f"lcm_expect_{self.tag}_{t.spec.name}"

    # ..................................................................
    def _roots(self):
        """Root IR nodes the per-(state, action) code needs."""
        tr = self.tr
        roots = [tr.F, tr.U]
        if tr.beta is not None:
            roots.append(tr.beta)
        for t in self.targets:
            roots.append(t.prob)
            if t.scalar:
                continue
            for pos in t.det_pos:
                roots.append(t.laws[t.spec.states[pos].name].expr)
            for pos in t.cont_pos:
                roots.append(t.laws[t.spec.states[pos].name].expr)
        return [ir.const(r) for r in roots]

    def _bellman_source(self) -> str:
        spec = self.spec
        cfg = self.cfg
        fp32 = self.precision == "fp32"
        ST = "float" if fp32 else "double"  # search type
        roots = self._roots()
        boundary = _boundary(roots)
        bP = [n for n in boundary if _phase(n) == "P"]
        bS = [n for n in boundary if _phase(n) == "S"]
        bA = [n for n in boundary if _phase(n) == "A"]
        key_actions = sorted(
            {name for t in self.targets for (k, name, _) in t.key_vars if k == "action"}
        )
        taste = spec.taste_shocks
        ND = spec.n_discrete_actions
        # A-table fields: boundary A nodes + discrete action indices used by keys
        a_fields: list[tuple[str, object]] = [("node", n) for n in bA]
        a_fields += [("aidx", name) for name in key_actions]
        if taste:
            a_fields.append(("ad", None))
        NAF = max(len(a_fields), 1)
        L: list[str] = []
        ap = L.append
        ap(f"// ---- regime {spec.name}: Bellman step (kernel a), precision {self.precision}")
        ap(f"#define NAF_{self.tag} {NAF}")

        # ---------------- helpers: decode an action index into per-axis values
        def decode_action(lines: list[str], a_expr: str, pref: str) -> dict:
            """Emit decode of flat action index -> {name: (idx_var, val_expr)}."""
            out = {}
            rem = f"{pref}rem"
            lines.append(f"int {rem} = {a_expr};")
            for k in range(len(spec.actions) - 1, -1, -1):
                ax = spec.actions[k]
                sz = f"lcm_wi(it, {self.W_ASIZE + k})"
                iv = f"{pref}i_{ax.name}"
                lines.append(f"int {iv} = {rem} % {sz}; {rem} /= {sz};")
                if ax.kind == "continuous":
                    vv = f"{pref}v_{ax.name}"
                    lines.append(f"double {vv} = lcm_wp<const double>(it, {self.W_AGRID + k})[{iv}];")
                    out[ax.name] = (iv, vv)
                else:
                    out[ax.name] = (iv, iv)
            return out

        def action_provided(dec: dict, pvals: dict) -> dict:
            prov = dict(pvals)
            for ax in spec.actions:
                node = ir.var("action", ax.name, "f" if ax.kind == "continuous" else "i")
                prov[id(node)] = dec[ax.name][1]
            return prov

        def p_provided() -> dict:
            return {
                id(ir.var("period", "period", "i")): "period",
                id(ir.var("age", "age", "f")): "age",
            }

        # ---------------- P phase (double), per tile
        eP = Emitter("double", self.param_off, p_provided(), "p")
        pvals = {}
        for n in bP:
            pvals[id(n)] = eP.emit(n)
        # P-values of nodes used inside S and A subgraphs are emitted lazily by
        # those emitters (they see P nodes as ordinary nodes) -- cheap & hoisted.

        # ---------------- S phase (double), per thread
        s_prov = p_provided()
        s_prov.update(pvals)
        s_decl: list[str] = []
        for k, ax in enumerate(spec.states):
            if ax.kind == "continuous":
                s_prov[id(ir.var("state", ax.name, "f"))] = f"sv_{ax.name}"
            else:
                s_prov[id(ir.var("state", ax.name, "i"))] = f"si_{ax.name}"
        eS = Emitter("double", self.param_off, s_prov, "s")
        svals = {}
        for n in bS:
            svals[id(n)] = eS.emit(n)

        # ---------------- A phase (double) -> table fields
        def emit_A(lines: list[str], a_expr: str, pref: str):
            dec = decode_action(lines, a_expr, pref)
            eA = Emitter("double", self.param_off, action_provided(dec, p_provided() | pvals), pref + "a")
            fields = []
            for kind, obj in a_fields:
                if kind == "node":
                    fields.append((eA.emit(obj), obj.dtype))
                elif kind == "aidx":
                    fields.append((dec[obj][0], "i"))
                else:  # ad: discrete-action combo index
                    nc = "1"
                    expr = "0"
                    for k in range(len(spec.actions)):
                        ax = spec.actions[k]
                        if ax.kind == "continuous":
                            continue
                        expr = f"({expr}) * lcm_wi(it, {self.W_ASIZE + k}) + {dec[ax.name][0]}"
                    fields.append((expr, "i"))
            lines.extend(eA.lines)
            return fields

        # ---------------- SA phase (templated)
        def sa_body(T: str, E: str) -> list[str]:
            prov = {}
            prov.update(p_provided())
            for pi, n in enumerate(bP):
                prov[id(n)] = f"(({T})PVd[{pi}])" if n.dtype == "f" else f"(({_ctype(n.dtype)})PVd[{pi}])"
            for i, n in enumerate(bS):
                prov[id(n)] = _cast(f"SV[{i}]", n.dtype, T)
            for i, (kind, obj) in enumerate(a_fields):
                if kind == "node":
                    prov[id(obj)] = _cast(f"AF({i})", obj.dtype, T)
            for ax in spec.states:
                if ax.kind == "continuous":
                    pass
                else:
                    prov[id(ir.var("state", ax.name, "i"))] = f"si_{ax.name}"
            e = Emitter(T, self.param_off, prov, "q")
            out: list[str] = []
            fexpr = e.emit(self.tr.F)
            out += e.lines
            out.append(f"if (!({fexpr})) return false;")
            e.lines = []
            uexpr = e.emit(self.tr.U)
            out += e.lines
            e.lines = []
            if spec.terminal:
                out.append(f"Q = ({T})({uexpr});")
                return out
            bexpr = e.emit(self.tr.beta)
            out += e.lines
            e.lines = []
            # every target's probability and next-state expressions are bound at
            # function scope first (shared sub-expressions stay in scope)
            pnames, dnames, xnames = {}, {}, {}
            for ti, t in enumerate(self.targets):
                pnames[ti] = e.emit(t.prob)
                if t.scalar:
                    continue
                for pos in t.det_pos:
                    dnames[(ti, pos)] = e.emit(t.laws[t.spec.states[pos].name].expr)
                for pos in t.cont_pos:
                    xnames[(ti, pos)] = e.emit(t.laws[t.spec.states[pos].name].expr)
            out += e.lines
            e.lines = []
            out.append(f"{T} ce = ({T})0; {T} mass = ({T})0; bool neg = false;")
            for ti, t in enumerate(self.targets):
                out.append(f"{{ {T} p = ({T})({pnames[ti]}); mass += p; neg = neg || (p < ({T})0);")
                out.append("  if (p != 0) {")
                if t.scalar:
                    out.append(f"    {T} ev = ({T})(*lcm_wp<const double>(it, {t.w_scalar}));")
                else:
                    # row offset: key, deterministic discrete, then continuous block
                    inner: list[str] = []
                    key = "0"
                    for kind, name, size in t.key_vars:
                        if kind == "state":
                            iv = f"si_{name}"
                        else:
                            fi = [i for i, (k2, o) in enumerate(a_fields) if k2 == "aidx" and o == name][0]
                            iv = f"(int)AF({fi})"
                        key = f"({key}) * {size} + {iv}"
                    off = key
                    for pos in t.det_pos:
                        sz = f"lcm_wi(it, {t.w_sizes + pos})"
                        off = f"({off}) * {sz} + min(max((int)({dnames[(ti, pos)]}), 0), {sz} - 1)"
                    cblk = "1"
                    for pos in t.cont_pos:
                        cblk = f"{cblk} * lcm_wi(it, {t.w_sizes + pos})"
                    for ci, pos in enumerate(t.cont_pos):
                        ax = t.spec.states[pos]
                        xexpr = xnames[(ti, pos)]
                        w0 = t.w_coord + 3 * ci
                        kind = ax.grid.kind
                        if kind == "lin":
                            c = f"lcm_coord_lin<{T}>(({T})({xexpr}), ({T})lcm_wd(it, {w0}), ({T})lcm_wd(it, {w0 + 1}))"
                        elif kind == "log":
                            c = f"lcm_coord_log<{T}>(({T})({xexpr}), ({T})lcm_wd(it, {w0}), ({T})lcm_wd(it, {w0 + 1}))"
                        else:
                            c = f"lcm_coord_irreg<{T}>(({T})({xexpr}), lcm_wp<const double>(it, {w0 + 2}), lcm_wi(it, {t.w_sizes + pos}))"
                        inner.append(f"{T} c{ci} = {c};")
                    inner.append(
                        f"const {E}* row = lcm_evsel<{E}>::get(it, {t.w_ev64}, {t.w_ev32}) + (i64)({off}) * ({cblk});"
                    )
                    if len(t.cont_pos) == 0:
                        inner.append(f"{T} ev = ({T})row[0];")
                    elif len(t.cont_pos) == 1:
                        n0 = f"lcm_wi(it, {t.w_sizes + t.cont_pos[0]})"
                        inner.append(f"{T} ev = lcm_interp1<{T}, {E}>(row, {n0}, c0);")
                    elif len(t.cont_pos) == 2:
                        n0 = f"lcm_wi(it, {t.w_sizes + t.cont_pos[0]})"
                        n1 = f"lcm_wi(it, {t.w_sizes + t.cont_pos[1]})"
                        inner.append(f"{T} ev = lcm_interp2<{T}, {E}>(row, {n0}, {n1}, c0, c1);")
                    else:
                        raise TracingError("more than two continuous states per target are not supported")
                    out += ["    " + s for s in inner]
                out.append(f"    ce = ce + lcm_zs(p, ev);")
                out.append("  }")
                out.append("}")
            out.append(
                f"bool valid = (fabs(mass - ({T})1) <= ({T})1e-3) && !neg;"
            )
            out.append(f"ce = valid ? ce / mass : lcm_lim<{T}>::nan();")
            out.append(f"Q = ({T})({uexpr}) + ({T})({bexpr}) * ce;")
            return out

        # shared-memory action table element type
        TT = ST
        n_bP = max(len(bP), 1)
        n_bS = max(len(bS), 1)
        # --- SA device function
        ap(
            f"template <typename T, typename E, typename AFN>\n"
            f"__device__ __forceinline__ bool lcm_sa_{self.tag}(const i64* __restrict__ it, const double* __restrict__ PV, "
            f"const double* PVd, const double* SV, const AFN& AF, {''.join(f'int si_{a.name}, ' for a in spec.states if a.kind != 'continuous')}int period, double age, T& Q) {{"
        )
        for s in sa_body("T", "E"):
            ap("  " + s)
        ap("  return true;\n}")

        # --- accessors for action fields
        ap(
            f"template <typename T> struct AFTab_{self.tag} {{ const {TT}* tab; int j; int chunk;\n"
            f"  __device__ __forceinline__ T operator()(int f) const {{ return (T)tab[f * chunk + j]; }} }};"
        )
        ap(
            f"struct AFLoc_{self.tag} {{ double v[NAF_{self.tag}];\n"
            f"  __device__ __forceinline__ double operator()(int f) const {{ return v[f]; }} }};"
        )

        # --- the kernel
        B, LANES, CH = cfg.block, cfg.lanes, cfg.chunk
        SPT = cfg.states_per_tile
        si_args = "".join(f"si_{a.name}, " for a in spec.states if a.kind != "continuous")
        ap(
            f'extern "C" __global__ void __launch_bounds__({B}) {self.bellman_name()}('
            "const i64* __restrict__ items, const int* __restrict__ tile_prefix, int n_items, int n_tiles) {"
        )
        ap(f"  extern __shared__ __align__(16) unsigned char lcm_smem[];")
        ap(f"  {TT}* tab = reinterpret_cast<{TT}*>(lcm_smem);")
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* it = items + (i64)item * {self.n_words};")
        ap(f"    const double* __restrict__ PV = lcm_wp<const double>(it, {self.W_P});")
        ap(f"    const int period = lcm_wi(it, {self.W_PERIOD});")
        ap(f"    const double age = lcm_wd(it, {self.W_AGE});")
        ap(f"    const int n_states = lcm_wi(it, {self.W_NSTATES});")
        ap(f"    const int n_actions = lcm_wi(it, {self.W_NACT});")
        ap(f"    const int s = (tile - tile_prefix[item]) * {SPT} + (int)threadIdx.x / {LANES};")
        ap(f"    const int lane = (int)threadIdx.x % {LANES};")
        ap("    const bool active = s < n_states;")
        # decode state
        ap("    int srem = active ? s : 0;")
        for k in range(len(spec.states) - 1, -1, -1):
            ax = spec.states[k]
            ap(f"    const int si_{ax.name} = srem % lcm_wi(it, {self.W_SSIZE + k}); srem /= lcm_wi(it, {self.W_SSIZE + k});")
        for k, ax in enumerate(spec.states):
            if ax.kind == "continuous":
                ap(f"    const double sv_{ax.name} = lcm_wp<const double>(it, {self.W_SGRID + k})[si_{ax.name}];")
        # P phase
        for s_ in eP.lines:
            ap("    " + s_)
        ap(f"    double PVd[{n_bP}];")
        for i, n in enumerate(bP):
            ap(f"    PVd[{i}] = (double)({pvals[id(n)]});")
        if not bP:
            ap("    PVd[0] = 0.0;")
        # S phase
        for s_ in eS.lines:
            ap("    " + s_)
        ap(f"    double SV[{n_bS}];")
        for i, n in enumerate(bS):
            ap(f"    SV[{i}] = (double)({svals[id(n)]});")
        if not bS:
            ap("    SV[0] = 0.0;")
        BEST = "LcmBest2" if (fp32 and not taste) else "LcmBest"
        if taste:
            ap(f"    LcmBest<{ST}> bd[{ND}];")
            ap(f"    #pragma unroll\n    for (int d = 0; d < {ND}; ++d) bd[d].init();")
        else:
            ap(f"    {BEST}<{ST}> best; best.init();")
        ap(f"    for (int a0 = 0; a0 < n_actions; a0 += {CH}) {{")
        ap(f"      const int cn = min({CH}, n_actions - a0);")
        ap("      __syncthreads();")
        ap(f"      for (int j = threadIdx.x; j < cn; j += {B}) {{")
        fill: list[str] = []
        flds = emit_A(fill, "a0 + j", "t")
        for s_ in fill:
            ap("        " + s_)
        for i, (expr, dt) in enumerate(flds):
            ap(f"        tab[{i} * {CH} + j] = ({TT})({expr});")
        ap("      }")
        ap("      __syncthreads();")
        ap("      if (active) {")
        ap(f"        for (int j = lane; j < cn; j += {LANES}) {{")
        ap(f"          AFTab_{self.tag}<{ST}> af{{tab, j, {CH}}};")
        ap(f"          {ST} q;")
        ap(
            f"          if (lcm_sa_{self.tag}<{ST}, {ST}>(it, PV, PVd, SV, af, {si_args}period, age, q)) "
            + (f"bd[(int)af({len(a_fields) - 1})].push(q, a0 + j);" if taste else "best.push(q, a0 + j);")
        )
        ap("        }")
        ap("      }")
        ap("    }")
        # reduction
        if taste:
            ap(f"    #pragma unroll\n    for (int d = 0; d < {ND}; ++d) lcm_group_reduce<{LANES}, {ST}>(bd[d]);")
        elif fp32:
            ap(f"    lcm_group_reduce2<{LANES}, {ST}>(best);")
        else:
            ap(f"    lcm_group_reduce<{LANES}, {ST}>(best);")
        ap("    if (active && lane == 0) {")
        ap(f"      double* Vout = lcm_wp<double>(it, {self.W_V});")
        ap(f"      int* Pout = lcm_wp<int>(it, {self.W_POL});")

        # final evaluation at an action index (double), used by fp32 mode
        def final_eval(a_var: str, out_var: str) -> list[str]:
            lines: list[str] = [f"AFLoc_{self.tag} afl;"]
            fl = emit_A(lines, a_var, "f")
            for i, (expr, dt) in enumerate(fl):
                lines.append(f"afl.v[{i}] = (double)({expr});")
            lines.append(f"double {out_var};")
            lines.append(
                f"if (!lcm_sa_{self.tag}<double, double>(it, PV, PVd, SV, afl, {si_args}period, age, {out_var})) {out_var} = -lcm_lim<double>::inf();"
            )
            return lines

        if taste:
            ap(f"      double vals[{ND}]; int bdi = -1; double bv = -lcm_lim<double>::inf(); int anynan = 0;")
            ap(f"      for (int d = 0; d < {ND}; ++d) {{")
            ap("        anynan |= bd[d].nan;")
            ap("        if (bd[d].idx < 0) { vals[d] = -lcm_lim<double>::inf(); continue; }")
            if fp32:
                ap("        { const int aa = bd[d].idx;")
                for s_ in final_eval("aa", "qd"):
                    ap("          " + s_)
                ap("          vals[d] = qd; }")
            else:
                ap("        vals[d] = bd[d].v;")
            ap("        if (bdi < 0 || vals[d] > bv) { bv = vals[d]; bdi = d; }")
            ap("      }")
            ap(f"      const double scale = lcm_wd(it, {self.W_TASTE});")
            ap(f"      double v = lcm_logsum<double, {ND}>(vals, scale);")
            ap("      if (anynan) v = lcm_lim<double>::nan();")
            ap("      Vout[s] = v; Pout[s] = (bdi < 0 || anynan) ? 0 : bd[bdi].idx;")
        else:
            ap("      double v; int pol;")
            ap("      if (best.nan) { v = lcm_lim<double>::nan(); pol = 0; }")
            ap("      else if (best.idx < 0) { v = -lcm_lim<double>::inf(); pol = 0; }")
            if fp32:
                # re-rank the two single-precision candidates in double precision
                ap("      else { const int aa = best.idx;")
                for s_ in final_eval("aa", "qd"):
                    ap("        " + s_)
                ap("        v = qd; pol = aa;")
                ap("        if (best.idx2 >= 0) { const int ab = best.idx2;")
                for s_ in final_eval("ab", "qd2"):
                    ap("          " + s_.replace("afl", "afl2"))
                ap("          if (qd2 > v || (qd2 == v && ab < pol)) { v = qd2; pol = ab; } }")
                ap("      }")
            else:
                ap("      else { v = (double)best.v; pol = best.idx; }")
            ap("      Vout[s] = v; Pout[s] = pol;")
        ap("    }")
        ap("  }")
        ap("}")
        self.smem_bytes = NAF * CH * (4 if fp32 else 8)
        return "\n".join(L)

    # ------------------------------------------------------------------ (b)
    def _expect_source(self, t: TargetPlan) -> str:
        """Kernel (b): contraction of V' over the target's stochastic axes."""
        spec = self.spec
        tg = t.spec
        K, J = t.K, t.J
        stoch = t.stoch_pos
        B = 256
        KC = min(K, 32)
        # weight expressions per stochastic axis
        L: list[str] = []
        ap = L.append
        name = self.expect_name(t)
        # item layout for (b)
        # 0 Vt (double*), 1 EV64 out, 2 EV32 out (0 if none), 3 PV (params of source)
        # 4 period, 5 age, 6 cblk, 7 n_cols, 8.. sizes of target axes
        self.EW = {"V": 0, "EV64": 1, "EV32": 2, "P": 3, "PERIOD": 4, "AGE": 5, "CBLK": 6, "NCOLS": 7, "SIZES": 8}
        self.e_words = 8 + len(tg.states)
        ap(f"// ---- expectation {spec.name} -> {tg.name}: K={K} J={J}")
        ap(
            f'extern "C" __global__ void __launch_bounds__({B}) {name}('
            "const i64* __restrict__ items, const int* __restrict__ tile_prefix, int n_items, int n_tiles) {"
        )
        ap(f"  __shared__ double W[{K * J}];")
        ap(f"  __shared__ double Winv[{K}];")
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* it = items + (i64)item * {self.e_words};")
        ap("    const double* __restrict__ Vt = lcm_wp<const double>(it, 0);")
        ap("    double* EV64 = lcm_wp<double>(it, 1);")
        ap("    float* EV32 = lcm_wp<float>(it, 2);")
        ap("    const double* __restrict__ PV = lcm_wp<const double>(it, 3);")
        ap("    const int period = lcm_wi(it, 4);")
        ap("    const double age = lcm_wd(it, 5);")
        ap("    const int cblk = lcm_wi(it, 6);")
        ap("    const int n_cols = lcm_wi(it, 7);")
        ap("    (void)period; (void)age;")
        ap("    __syncthreads();")
        # weight table fill
        ap(f"    for (int e = threadIdx.x; e < {K * J}; e += {B}) {{")
        ap(f"      const int k = e / {J}; const int j = e % {J};")
        # decode k into key vars
        ap("      int kr = k;")
        for kind, kname, size in reversed(t.key_vars):
            ap(f"      const int key_{kind}_{kname} = kr % {size}; kr /= {size};")
        ap("      int jr = j;")
        for pos in reversed(stoch):
            ax = tg.states[pos]
            ap(f"      const int jn_{ax.name} = jr % {ax.size}; jr /= {ax.size};")
        prov = {
            id(ir.var("period", "period", "i")): "period",
            id(ir.var("age", "age", "f")): "age",
        }
        for kind, kname, size in t.key_vars:
            prov[id(ir.var(kind, kname, "i"))] = f"key_{kind}_{kname}"
        e = Emitter("double", self.param_off, prov, "w")
        factors = []
        for pos in stoch:
            ax = tg.states[pos]
            law = t.laws[ax.name]
            if law.kind == "process":
                off, shape = self.param_off[proc_P_name(law.source_process)]
                n = shape[0]
                factors.append(f"PV[{off} + key_state_{law.source_process} * {n} + jn_{ax.name}]")
            else:
                # select item j of the Markov vector
                exprs = [e.emit(x) for x in law.expr.items]
                sel = exprs[-1]
                for q in range(len(exprs) - 2, -1, -1):
                    sel = f"(jn_{ax.name} == {q} ? (double)({exprs[q]}) : {sel})"
                factors.append(f"(double)({sel})")
        for s_ in e.lines:
            ap("      " + s_)
        prod = factors[0] if factors else "1.0"
        for f_ in factors[1:]:
            prod = f"({prod}) * ({f_})"
        ap(f"      W[e] = {prod};")
        ap("    }")
        ap("    __syncthreads();")
        ap(f"    for (int k = threadIdx.x; k < {K}; k += {B}) {{")
        ap(f"      double sw = 0.0; for (int j = 0; j < {J}; ++j) sw += W[k * {J} + j];")
        ap("      Winv[k] = sw > 0.0 ? sw : 1.0;")
        ap("    }")
        ap("    __syncthreads();")
        ap(f"    const int col = (tile - tile_prefix[item]) * {B} + (int)threadIdx.x;")
        ap("    if (col < n_cols) {")
        # decode col -> det indices + cflat ; compute base offset per j
        ap("      const int cflat = col % cblk; int dr = col / cblk;")
        det_names = []
        for pos in reversed(t.det_pos):
            ax = tg.states[pos]
            ap(f"      const int di_{ax.name} = dr % {ax.size}; dr /= {ax.size};")
        # strides over target discrete axes in order
        disc_pos = [p for p, ax in enumerate(tg.states) if ax.kind != "continuous"]
        ap(f"      for (int k0 = 0; k0 < {K}; k0 += {KC}) {{")
        ap(f"        double acc[{KC}];")
        ap(f"        #pragma unroll\n        for (int kk = 0; kk < {KC}; ++kk) acc[kk] = 0.0;")
        ap(f"        for (int j = 0; j < {J}; ++j) {{")
        ap("          int jr = j;")
        for pos in reversed(stoch):
            ax = tg.states[pos]
            ap(f"          const int jn_{ax.name} = jr % {ax.size}; jr /= {ax.size};")
        off = "0"
        for pos in disc_pos:
            ax = tg.states[pos]
            iv = f"jn_{ax.name}" if pos in stoch else f"di_{ax.name}"
            off = f"({off}) * {ax.size} + {iv}"
        ap(f"          const double v = Vt[(i64)({off}) * cblk + cflat];")
        ap(f"          #pragma unroll\n          for (int kk = 0; kk < {KC}; ++kk) {{")
        ap(f"            const int k = k0 + kk; if (k < {K}) acc[kk] += lcm_zs(W[k * {J} + j], v);")
        ap("          }")
        ap("        }")
        ap(f"        #pragma unroll\n        for (int kk = 0; kk < {KC}; ++kk) {{")
        ap(f"          const int k = k0 + kk; if (k < {K}) {{")
        ap("            const double r = acc[kk] / Winv[k];")
        ap("            EV64[(i64)k * n_cols + col] = r;")
        ap("            if (EV32) EV32[(i64)k * n_cols + col] = (float)r;")
        ap("          }")
        ap("        }")
        ap("      }")
        ap("    }")
        ap("  }")
        ap("}")
        return "\n".join(L)


def _ctype(dt: str) -> str:
    return {"f": "double", "i": "int", "b": "bool"}[dt]


def _cast(expr: str, dt: str, T: str) -> str:
    if dt == "f":
        return f"(({T}){expr})"
    if dt == "i":
        return f"((int){expr})"
    return f"(({expr}) != 0)"
