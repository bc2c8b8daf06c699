"""CUDA C for the DC-EGM step of one regime (kernel c), double precision.

Three generated kernels per regime and next-period target set, around the
library FUES scan (``lcmx_fues_scan``):

``lcm_egmc_<tag>``  one thread per (row, savings node A_j), a row being one
    (discrete state x discrete action) combination: the continuation -- for
    every target, every combination of the target's discrete states, every
    target discrete choice, a Hermite read of the target's carry row at
    R'(A_j) -- then the Euler inversion c = (u')^{-1}(max(beta E[mu'], eps)),
    R = A + c, v = u(c) + beta E[V'].  The thread of A_0 also writes the
    constrained candidates.  Restates ``egm/step_core.py:156-514`` and
    ``egm/continuation.py:959-1534``.
``lcm_egmu_<tag>``  one thread per refined point: the carry marginal-utility
    row u'(c), and the overflow / no-live-candidate / infeasible rules.
``lcm_egmp_<tag>``  one thread per (discrete-state combination, state-grid
    point): the Hermite read of each discrete choice's refined row at the
    grid's resources, floored by (and below the first refined point replaced
    by) the closed-form constrained value, then the max (or logsum) over the
    discrete choices (``step_core.py:517-616``).
"""

from __future__ import annotations

import hashlib

from pylcm_b200 import ir
from pylcm_b200.codegen import _EXTRA_DEVICE, Emitter, device_header
from pylcm_b200.egm import A_VAR, MU, EgmRegime
from pylcm_b200.exceptions import TracingError
from pylcm_b200.spec import proc_P_name


class EgmKernels:
    def __init__(self, er: EgmRegime) -> None:
        self.er = er
        self.spec = er.spec
        self.param_off, self.param_len = er.tracer_layout()
        self._layout()
        src = self._source()
        self.src = src
        self.key = "lcm_egm_" + hashlib.sha1(src.encode()).hexdigest()[:24]

    # item record words
    def _layout(self) -> None:
        w = 0

        def take(n=1):
            nonlocal w
            k = w
            w += n
            return k

        self.W_P = take()
        self.W_PERIOD = take()
        self.W_AGE = take()
        self.W_NSAV = take()
        self.W_SAV = take()
        self.W_NGRID = take()
        self.W_GRID = take()
        self.W_CG, self.W_CC, self.W_CV, self.W_CS = take(), take(), take(), take()
        # candidate marginal utility u'(c) (the value rows' supgradient, read
        # by the RFC envelope; 0 for dead candidates)
        self.W_CM = take() if self.er.envelope == "rfc" else -1
        self.W_EV0 = take()
        self.W_RG, self.W_RC, self.W_RV, self.W_MU, self.W_NK = take(), take(), take(), take(), take()
        self.W_V = take()
        self.W_POL = take()
        self.W_NPAD = take()
        self.W_TASTE = take()
        self.W_T = []
        for t in self.er.targets:
            if t.unreachable:
                self.W_T.append({})
            elif t.next_R is None:
                self.W_T.append({"scalar": take()})
            elif t.is_value:
                self.W_T.append({"tv": take(), "tm": take(), "tg": take(), "tn": take()})
            else:
                self.W_T.append({"rg": take(), "rv": take(), "mu": take(), "nk": take(), "npad": take(), "taste": take()})
        self.n_words = w

    def names(self) -> tuple[str, str, str]:
        tag = self.spec.name
        h = hashlib.sha1(repr([t.spec.name for t in self.er.targets]).encode()).hexdigest()[:6]
        return (f"lcm_egmc_{tag}_{h}", f"lcm_egmu_{tag}_{h}", f"lcm_egmp_{tag}_{h}")

    def _row_decode(self, lines: list[str], row_expr: str) -> dict:
        """Emit decode of a row index into discrete codes; returns provided map."""
        er = self.er
        lines.append(f"int rrem = {row_expr};")
        prov = {}
        for a in reversed(er.disc_states + er.disc_actions):
            kind = "state" if a in er.disc_states else "action"
            lines.append(f"const int dc_{a.name} = rrem % {a.size}; rrem /= {a.size};")
            prov[id(ir.var(kind, a.name, "i"))] = f"dc_{a.name}"
        return prov

    @staticmethod
    def _row_exprs(t) -> list:
        """Expressions that decide which carry rows a continuation read
        touches and with what weight: the regime probability and the laws of
        the target's discrete states."""
        out = [t.prob]
        for ax in [a for a in t.spec.states if a.kind != "continuous"]:
            law = t.disc_laws[ax.name]
            if law.kind == "markov":
                out += list(law.expr.items)
            elif law.kind == "det":
                out.append(law.expr)
        return [x for x in out if isinstance(ir.const(x), ir.Expr)]

    def _weights(self, body: list, ti: int, t, names: dict) -> list:
        """Emit the weight vector of every discrete state of target `t`
        (process row, Markov row or one-hot deterministic law)."""
        wl_names = []
        for ax in [a for a in t.spec.states if a.kind != "continuous"]:
            law = t.disc_laws[ax.name]
            arr = f"w_{ti}_{ax.name}"
            wl_names.append((ax, arr))
            body.append(f"    double {arr}[{ax.size}];")
            if law.kind == "process":
                off, shape = self.param_off[proc_P_name(law.source_process)]
                body.append(
                    f"    for (int q = 0; q < {ax.size}; ++q) {arr}[q] = PV[{off} + dc_{law.source_process} * {shape[1]} + q];"
                )
            elif law.kind == "markov":
                for q, v in enumerate(names[("m", ax.name)]):
                    body.append(f"    {arr}[{q}] = (double)({v});")
            else:
                de = names[("d", ax.name)]
                body.append(f"    {{ const int kk = min(max((int)({de}), 0), {ax.size - 1});")
                body.append(f"      for (int q = 0; q < {ax.size}; ++q) {arr}[q] = (q == kk) ? 1.0 : 0.0; }}")
        return wl_names

    def _value_read(self, body: list, ti: int, t, names: dict, w: dict) -> None:
        """Continuation read of a target that carries its value array (a
        terminal or grid-search regime) on its own state grid, the Euler
        state's marginal value beside it (``egm/terminal.py:76-330``).  All
        rows share the grid, so the expectation over the target's discrete
        states folds into the rows before one read, as the reference folds a
        value-only child's node axes (``egm/continuation.py:551-674``: the
        weighted sums w * row over the nodes, a zero weight contributing
        nothing; an integer-indexed deterministic state is the one-hot case);
        the value read is the limited cubic Hermite with the marginal row as
        node slopes, the marginal read linear, pinned to zero where the value
        read is -inf, times dR'/dA (``continuation.py:1460-1520``)."""
        tg = t.spec
        body.append(f"    const double Rn = (double)({names['R']}); const double dR = (double)({names['dR']});")
        wl_names = self._weights(body, ti, t, names)
        body.append(f"    const double* TV = lcm_wp<const double>(it, {w['tv']});")
        body.append(f"    const double* TM = lcm_wp<const double>(it, {w['tm']});")
        body.append(f"    const double* TG = lcm_wp<const double>(it, {w['tg']});")
        body.append(f"    const int tn = lcm_wi(it, {w['tn']});")
        body.append("    const int ix = tn > 1 ? lcm_row_bracket(TG, tn, Rn) : 0;")
        body.append("    const int b0 = tn > 1 ? (ix < 0 ? 0 : (ix > tn - 2 ? tn - 2 : ix)) : 0;")
        body.append("    const int b1 = tn > 1 ? b0 + 1 : 0;")
        body.append("    double f0 = 0.0, f1 = 0.0, g0 = 0.0, g1 = 0.0;")
        J = 1
        for ax, _ in wl_names:
            J *= ax.size
        body.append(f"    for (int jc = 0; jc < {J}; ++jc) {{")
        body.append("      int jr = jc; double wt = 1.0;")
        for ax, arr in reversed(wl_names):
            body.append(f"      const int jn_{ax.name} = jr % {ax.size}; jr /= {ax.size}; wt *= {arr}[jn_{ax.name}];")
        body.append("      (void)jr;")
        body.append("      if (wt == 0.0) continue;")
        # flat index into the target's value array (states in declaration
        # order, the Euler axis tn long)
        i0 = i1 = "(i64)0"
        for ax in tg.states:
            if ax.name == t.value_euler:
                i0, i1 = f"({i0}) * tn + b0", f"({i1}) * tn + b1"
            else:
                i0, i1 = f"({i0}) * {ax.size} + jn_{ax.name}", f"({i1}) * {ax.size} + jn_{ax.name}"
        body.append(f"      const i64 i0 = {i0}, i1 = {i1};")
        body.append("      f0 += wt * TV[i0]; f1 += wt * TV[i1]; g0 += wt * TM[i0]; g1 += wt * TM[i1];")
        body.append("    }")
        body.append("    double vr, mr;")
        body.append("    if (tn <= 1) { vr = f0; mr = g0; }")
        body.append("    else if (ix >= tn - 1) { vr = f1; mr = g1; }")
        body.append("    else lcm_bracket_read(TG[b0], TG[b1], f0, f1, g0, g1, true, ix, Rn, vr, mr);")
        body.append("    EV += p * vr; EMU += p * (vr == -LCM_INF ? 0.0 : mr * dR);")

    def _source(self) -> str:
        er = self.er
        cname, uname, pname = self.names()
        nd = er.n_disc_actions
        nrow = er.n_rows
        L: list[str] = [device_header(), _EXTRA_DEVICE]
        ap = L.append
        base_prov = {id(ir.var("period", "period", "i")): "period", id(ir.var("age", "age", "f")): "age"}

        # ------------------------------------------------------------ (c1)
        # latency-bound (dependent binary-search loads): at least 3 CTAs per
        # SM (<= 85 registers) -- measured 26 % faster than the compiler's
        # 88-register, 2-CTA choice on the 2000-node DC-EGM model
        ap(f'extern "C" __global__ void __launch_bounds__(256, 3) {cname}(const i64* __restrict__ items, '
           "const int* __restrict__ tile_prefix, int n_items, int n_tiles) {")
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* __restrict__ it = items + (i64)item * {self.n_words};")
        ap(f"    const double* __restrict__ PV = lcm_wp<const double>(it, {self.W_P});")
        ap(f"    const int period = lcm_wi(it, {self.W_PERIOD}); const double age = lcm_wd(it, {self.W_AGE});")
        ap("    (void)period; (void)age;")
        ap(f"    const int n_sav = lcm_wi(it, {self.W_NSAV});")
        ap(f"    const int nc = {er.n_constrained};")
        ap("    const int n_cand = nc + n_sav;")
        ap("    const int e_t = (tile - tile_prefix[item]) * 256 + (int)threadIdx.x;")
        # lanes past the end repeat the last element (their results are not
        # written) so that every warp stays converged for the shared reads
        ap(f"    const bool live = e_t < {nrow} * n_sav;")
        ap(f"    const int e = live ? e_t : {nrow} * n_sav - 1;")
        ap("    const int row = e / n_sav, j = e % n_sav;")
        # one candidate row for the whole warp: its carry-row reads share
        # their bracket search (lcm_row_bracket_warp)
        # (the shuffle runs on every lane: a shuffle inside the short-circuit
        # of `live && ...` would leave the warp's non-live lanes out of it)
        ap("    const int row_l0 = __shfl_sync(0xffffffffu, row, 0);")
        ap("    const bool warp_row = __all_sync(0xffffffffu, live && row == row_l0);")
        body: list[str] = []
        prov = dict(base_prov)
        prov.update(self._row_decode(body, "row"))
        body.append(f"const double A = lcm_wp<const double>(it, {self.W_SAV})[j];")
        prov[id(A_VAR)] = "A"
        em = Emitter("double", self.param_off, prov, "c")
        beta = em.emit(er.beta)
        body += em.lines
        em.lines = []
        # bind every target expression at function scope (shared sub-expressions
        # must stay in scope for later targets)
        tnames = {}
        for ti, t in enumerate(er.targets):
            d = {"p": em.emit(t.prob)}
            if t.next_R is not None and not t.unreachable:
                d["R"] = em.emit(t.next_R)
                d["dR"] = em.emit(t.dR_dA)
                for ax in [a for a in t.spec.states if a.kind != "continuous"]:
                    law = t.disc_laws[ax.name]
                    if law.kind == "markov":
                        d[("m", ax.name)] = [em.emit(x) for x in law.expr.items]
                    elif law.kind == "det":
                        d[("d", ax.name)] = em.emit(law.expr)
            tnames[ti] = d
        body += em.lines
        em.lines = []
        body.append("double EV = 0.0, EMU = 0.0, mass = 0.0; bool neg = false;")
        for ti, t in enumerate(er.targets):
            w = self.W_T[ti]
            pe = tnames[ti]["p"]
            body.append(f"{{ const double p = (double)({pe}); mass += p; neg = neg || p < 0.0;")
            body.append("  if (p != 0.0) {")
            if t.unreachable:
                body.append("    EV = LCM_NAN;  // probability toward a target this regime cannot reach")
            elif t.next_R is None:
                body.append(f"    EV += lcm_zs(p, *lcm_wp<const double>(it, {w['scalar']}));")
            elif t.is_value:
                self._value_read(body, ti, t, tnames[ti], w)
            else:
                tg = t.spec
                Re = tnames[ti]["R"]
                dRe = tnames[ti]["dR"]
                body.append(f"    const double Rn = (double)({Re}); const double dR = (double)({dRe});")
                dstates = [a for a in tg.states if a.kind != "continuous"]
                wl_names = self._weights(body, ti, t, tnames[ti])
                nd_t = 1
                for a in tg.actions:
                    if a.kind != "continuous":
                        nd_t *= a.size
                J = 1
                for ax in dstates:
                    J *= ax.size
                body.append(f"    const double* RG = lcm_wp<const double>(it, {w['rg']});")
                body.append(f"    const double* RV = lcm_wp<const double>(it, {w['rv']});")
                body.append(f"    const double* RM = lcm_wp<const double>(it, {w['mu']});")
                body.append(f"    const int* NK = lcm_wp<const int>(it, {w['nk']});")
                body.append(f"    const int npad = lcm_wi(it, {w['npad']}); const double lam = lcm_wd(it, {w['taste']});")
                body.append("    double nv = 0.0, nm = 0.0, den = 0.0;")
                body.append(f"    for (int jc = 0; jc < {J}; ++jc) {{")
                body.append("      int jr = jc; double wt = 1.0;")
                for ax, arr in reversed(wl_names):
                    body.append(f"      const int jn_{ax.name} = jr % {ax.size}; jr /= {ax.size}; wt *= {arr}[jn_{ax.name}];")
                body.append("      den += wt;")
                body.append("      if (wt == 0.0) continue;")
                body.append(f"      double vals[{nd_t}], mus[{nd_t}];")
                # the shared search needs the row's control flow to be the
                # same on every lane: the regime probability and the node
                # weights must not depend on the savings node
                uniform = not any(n is A_VAR for n in ir.topo_order([ir.const(x) for x in self._row_exprs(t)]))
                flag = "warp_row" if uniform else "false"
                single = [f"      for (int d = 0; d < {nd_t}; ++d) {{",
                          f"        const i64 crow = (i64)jc * {nd_t} + d;",
                          "        const int Lk = min(NK[crow], npad);",
                          "        lcm_row_read(RG + crow * npad, RV + crow * npad, RM + crow * npad, "
                          f"NK[crow] > npad ? 0 : Lk, Rn, vals[d], mus[d], {{flag}});",
                          "      }"]
                if uniform and nd_t >= 2:
                    # a warp reading one candidate row reads the choices'
                    # child rows in pairs, their searches interleaved
                    body.append("      if (warp_row) {")
                    for d0 in range(0, nd_t - 1, 2):
                        body.append("        {")
                        body.append("          const double* xs[2]; const double* fs[2]; const double* ds[2]; int Ls[2];")
                        for k in range(2):
                            body.append(f"          {{ const i64 crow = (i64)jc * {nd_t} + {d0 + k}; const int Lk = min(NK[crow], npad);")
                            body.append(f"            xs[{k}] = RG + crow * npad; fs[{k}] = RV + crow * npad; ds[{k}] = RM + crow * npad;")
                            body.append(f"            Ls[{k}] = NK[crow] > npad ? 0 : Lk; }}")
                        body.append("          double pv[2], pm[2];")
                        body.append("          lcm_row_read_warpk<2>(xs, fs, ds, Ls, Rn, pv, pm);")
                        body.append(f"          vals[{d0}] = pv[0]; mus[{d0}] = pm[0]; vals[{d0 + 1}] = pv[1]; mus[{d0 + 1}] = pm[1];")
                        body.append("        }")
                    if nd_t % 2:
                        body.append(f"        {{ const i64 crow = (i64)jc * {nd_t} + {nd_t - 1}; const int Lk = min(NK[crow], npad);")
                        body.append("          lcm_row_read(RG + crow * npad, RV + crow * npad, RM + crow * npad, "
                                    f"NK[crow] > npad ? 0 : Lk, Rn, vals[{nd_t - 1}], mus[{nd_t - 1}], true); }}")
                    body.append("      } else {")
                    body += ["  " + x.replace("{flag}", "false") for x in single]
                    body.append("      }")
                else:
                    body += [x.replace("{flag}", flag) for x in single]
                if tg.taste_shocks:
                    body.append("      double vmax = -LCM_INF;")
                    body.append(f"      for (int d = 0; d < {nd_t}; ++d) vmax = vals[d] > vmax ? vals[d] : vmax;")
                    body.append("      const double fin = (vmax == -LCM_INF) ? 0.0 : vmax;")
                    body.append("      double ssum = 0.0, ex[%d];" % nd_t)
                    body.append(f"      for (int d = 0; d < {nd_t}; ++d) {{ ex[d] = exp((vals[d] - fin) / lam); ssum += ex[d]; }}")
                    body.append("      const double Vs = fin + lam * log(ssum);")
                    body.append("      double MUs = 0.0;")
                    body.append(f"      for (int d = 0; d < {nd_t}; ++d) {{ const double pr = ex[d] / (ssum > 0.0 ? ssum : 1.0); if (pr > 0.0) MUs += pr * mus[d]; }}")
                else:
                    body.append("      int arg = 0; double Vs = vals[0];")
                    body.append(f"      for (int d = 1; d < {nd_t}; ++d) if (vals[d] > Vs) {{ Vs = vals[d]; arg = d; }}")
                    body.append("      double MUs = mus[0];")
                    body.append(f"      for (int d = 1; d < {nd_t}; ++d) if (d == arg) MUs = mus[d];")
                body.append("      nv += wt * ((wt == 0.0 && !lcm_isfinite(Vs)) ? 0.0 : Vs);")
                body.append("      nm += wt * MUs * dR;")
                body.append("    }")
                body.append("    const double dd = den > 0.0 ? den : 1.0;")
                body.append("    EV += p * (nv / dd); EMU += p * (nm / dd);")
            body.append("  }")
            body.append("}")
        body.append("if (!(fabs(mass - 1.0) <= 1e-3) || neg) EV = LCM_NAN;")
        body.append("else if (mass != 1.0) { EV /= mass; EMU /= mass; }")
        body.append(f"const double disc = ({beta}) * EMU;")
        body.append("const double tgt = disc < 0.0 ? LCM_NAN : (disc > 2.220446049250313e-16 ? disc : 2.220446049250313e-16);")
        prov_mu = dict(em.vals)
        prov_mu[id(MU)] = "tgt"
        em2 = Emitter("double", self.param_off, prov_mu, "m")
        ce = em2.emit(er.invmu)
        body += em2.lines
        body.append(f"const double cj = (double)({ce});")
        body.append("const double mj = A + cj;")
        cvar = ir.var("action", er.C, "f")

        def utility_at(cexpr: str, pref: str) -> tuple[list, str]:
            p2 = dict(em.vals)
            p2[id(cvar)] = cexpr
            e3 = Emitter("double", self.param_off, p2, pref)
            ue = e3.emit(er.U)
            return e3.lines, ue

        def marginal_at(cexpr: str, pref: str) -> tuple[list, str]:
            p2 = dict(em.vals)
            p2[id(cvar)] = cexpr
            e3 = Emitter("double", self.param_off, p2, pref)
            de = e3.emit(er.dU)
            return e3.lines, de

        rfc = er.envelope == "rfc"
        ul, ue = utility_at("cj", "u")
        body += ul
        body.append(f"const double vj = (double)({ue}) + ({beta}) * EV;")
        body.append(f"double* CG = lcm_wp<double>(it, {self.W_CG}) + (i64)row * n_cand;")
        body.append(f"double* CC = lcm_wp<double>(it, {self.W_CC}) + (i64)row * n_cand;")
        body.append(f"double* CV = lcm_wp<double>(it, {self.W_CV}) + (i64)row * n_cand;")
        body.append(f"double* CS = lcm_wp<double>(it, {self.W_CS}) + (i64)row * n_cand;")
        body.append("if (live) { const bool dead = vj == -LCM_INF;")
        body.append("  CG[nc + j] = dead ? LCM_NAN : mj; CC[nc + j] = dead ? LCM_NAN : cj;")
        body.append("  CV[nc + j] = dead ? LCM_NAN : vj; CS[nc + j] = dead ? LCM_NAN : A;")
        if rfc:
            ml, me = marginal_at("cj", "w")
            body += ["  " + x for x in ml]
            body.append(f"  lcm_wp<double>(it, {self.W_CM})[(i64)row * n_cand + nc + j] = dead ? 0.0 : (double)({me});")
        body.append("}")
        body.append("if (live && j == 0) {")
        body.append(f"  lcm_wp<double>(it, {self.W_EV0})[row] = EV;")
        body.append(f"  const int ng = lcm_wi(it, {self.W_NGRID});")
        body.append(f"  const double Rmax = lcm_wp<const double>(it, {self.W_GRID})[ng - 1];")
        body.append("  const double span = (mj < Rmax ? mj : Rmax) - A;")
        body.append("  const bool empty = !(span > 0.0 && lcm_isfinite(span));")
        body.append(f"  double ck = (empty ? 1.0 : span) * {1e-4!r};")
        body.append("  for (int k = 0; k < nc; ++k) {")
        ul2, ue2 = utility_at("ck", "k")
        body += ["    " + s for s in ul2]
        body.append(f"    const double vk = (double)({ue2}) + ({beta}) * EV;")
        body.append("    const bool dead = empty || vk == -LCM_INF;")
        body.append("    CG[k] = dead ? LCM_NAN : A + ck; CC[k] = dead ? LCM_NAN : ck;")
        body.append("    CV[k] = dead ? LCM_NAN : vk; CS[k] = dead ? LCM_NAN : A;")
        if rfc:
            ml2, me2 = marginal_at("ck", "z")
            body += ["    " + x for x in ml2]
            body.append(f"    lcm_wp<double>(it, {self.W_CM})[(i64)row * n_cand + k] = dead ? 0.0 : (double)({me2});")
        body.append(f"    ck *= {er.ratio!r};")
        body.append("  }")
        body.append("}")
        for s in body:
            ap("    " + s)
        ap("  }")
        ap("}")

        # ------------------------------------------------------------ (c3a) carry mu rows
        ap(f'extern "C" __global__ void __launch_bounds__(256) {uname}(const i64* __restrict__ items, '
           "const int* __restrict__ tile_prefix, int n_items, int n_tiles) {")
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* __restrict__ it = items + (i64)item * {self.n_words};")
        ap(f"    const double* __restrict__ PV = lcm_wp<const double>(it, {self.W_P});")
        ap(f"    const int period = lcm_wi(it, {self.W_PERIOD}); const double age = lcm_wd(it, {self.W_AGE});")
        ap("    (void)period; (void)age;")
        ap(f"    const int npad = lcm_wi(it, {self.W_NPAD});")
        ap("    const int e = (tile - tile_prefix[item]) * 256 + (int)threadIdx.x;")
        ap(f"    if (e >= {nrow} * npad) continue;")
        ap("    const int row = e / npad, k = e % npad;")
        body = []
        prov = dict(base_prov)
        prov.update(self._row_decode(body, "row"))
        body.append(f"double* RC = lcm_wp<double>(it, {self.W_RC}) + (i64)row * npad;")
        body.append(f"double* RV = lcm_wp<double>(it, {self.W_RV}) + (i64)row * npad;")
        body.append(f"double* RM = lcm_wp<double>(it, {self.W_MU}) + (i64)row * npad;")
        body.append(f"const int nk = lcm_wp<const int>(it, {self.W_NK})[row];")
        body.append("const double c = RC[k];")
        body.append("const double cc = (c != c) ? 1.0 : c;")
        prov[id(cvar)] = "cc"
        e4 = Emitter("double", self.param_off, prov, "g")
        de = e4.emit(er.dU)
        fe = e4.emit(er.feasible)
        body += e4.lines
        body.append(f"double mu = (double)({de});")
        body.append("if (c != c) mu = LCM_NAN;")
        body.append("if (RV[k] == -LCM_INF) mu = 0.0;")
        body.append("if (nk > npad) { RV[k] = LCM_NAN; mu = LCM_NAN; }")
        body.append(f"if (nk == 0 || !({fe})) {{ RV[k] = -LCM_INF; mu = 0.0; }}")
        body.append("RM[k] = mu;")
        for s in body:
            ap("    " + s)
        ap("  }")
        ap("}")

        # ------------------------------------------------------------ (c3b) publication
        ns = nrow // nd
        ap(f'extern "C" __global__ void __launch_bounds__(256) {pname}(const i64* __restrict__ items, '
           "const int* __restrict__ tile_prefix, int n_items, int n_tiles) {")
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* __restrict__ it = items + (i64)item * {self.n_words};")
        ap(f"    const double* __restrict__ PV = lcm_wp<const double>(it, {self.W_P});")
        ap(f"    const int period = lcm_wi(it, {self.W_PERIOD}); const double age = lcm_wd(it, {self.W_AGE});")
        ap("    (void)period; (void)age;")
        ap(f"    const int ng = lcm_wi(it, {self.W_NGRID}); const int npad = lcm_wi(it, {self.W_NPAD});")
        ap("    const int e = (tile - tile_prefix[item]) * 256 + (int)threadIdx.x;")
        ap(f"    if (e >= {ns} * ng) continue;")
        ap("    const int srow = e / ng, gi = e % ng;")
        ap(f"    const double R = lcm_wp<const double>(it, {self.W_GRID})[gi];")
        ap(f"    const double A0 = lcm_wp<const double>(it, {self.W_SAV})[0];")
        ap(f"    double best = -LCM_INF; int barg = 0; double vd[{nd}];")
        ap(f"    for (int d = 0; d < {nd}; ++d) {{")
        body = []
        prov = dict(base_prov)
        prov.update(self._row_decode(body, f"srow * {nd} + d"))
        body.append(f"const int row = srow * {nd} + d;")
        body.append(f"const double* RG = lcm_wp<const double>(it, {self.W_RG}) + (i64)row * npad;")
        body.append(f"const double* RV = lcm_wp<const double>(it, {self.W_RV}) + (i64)row * npad;")
        body.append(f"const double* RM = lcm_wp<const double>(it, {self.W_MU}) + (i64)row * npad;")
        body.append(f"const int nk = lcm_wp<const int>(it, {self.W_NK})[row];")
        body.append(f"const double EV0 = lcm_wp<const double>(it, {self.W_EV0})[row];")
        body.append("double val, sl;")
        body.append("lcm_row_read(RG, RV, RM, nk > npad ? 0 : min(nk, npad), R, val, sl);")
        body.append("const double cf = R - A0;")
        body.append("const double cfs = cf > 2.2250738585072014e-308 ? cf : 2.2250738585072014e-308;")
        prov[id(cvar)] = "cfs"
        e5 = Emitter("double", self.param_off, prov, "h")
        ue5 = e5.emit(er.U)
        be5 = e5.emit(er.beta)
        fe5 = e5.emit(er.feasible)
        body += e5.lines
        body.append(f"const double vcons = cf > 0.0 ? (double)({ue5}) + ({be5}) * EV0 : -LCM_INF;")
        body.append("double V = (cf > 0.0 && R <= RG[0]) ? vcons : (val > vcons ? val : vcons);")
        body.append("if (val != val && !(cf > 0.0 && R <= RG[0])) V = LCM_NAN;")
        body.append("if (nk > npad) V = LCM_NAN;")
        body.append(f"if (nk == 0 || !({fe5})) V = -LCM_INF;")
        body.append("vd[d] = V;")
        body.append("if (d == 0 || V > best) { best = V; barg = d; }")
        for s in body:
            ap("      " + s)
        ap("    }")
        if er.taste_scale is not None:
            ap(f"    const double lam = lcm_wd(it, {self.W_TASTE});")
            ap(f"    best = lcm_logsum<double, {nd}>(vd, lam);")
        ap(f"    lcm_wp<double>(it, {self.W_V})[(i64)srow * ng + gi] = best;")
        ap(f"    lcm_wp<int>(it, {self.W_POL})[(i64)srow * ng + gi] = barg;")
        ap("  }")
        ap("}")
        return "\n".join(L)


class ValueCarryKernel:
    """The marginal-value rows of a target that carries its value array into
    a DC-EGM parent (``egm/terminal.py:76-330``), one thread per state of the
    target, written in the value array's layout:

    - terminal target: the derivative of its utility with respect to the
      Euler state at the grid node (the reference's ``jax.grad``; here
      :func:`pylcm_b200.ir.diff`), zero where the value is -inf;
    - grid-search target: the value array's slope along the Euler grid --
      NumPy's second-order non-uniform stencil where both neighbours are
      feasible, the one-sided difference toward the one feasible neighbour,
      zero without one or at an infeasible state (``terminal.py:272-314``).
    """

    def __init__(self, spec, euler: str, U=None, param_off=None) -> None:
        self.spec = spec
        self.euler = euler
        self.terminal = U is not None
        self.param_off = param_off or {}
        self.U = U
        self.W_P, self.W_PERIOD, self.W_AGE, self.W_V, self.W_M, self.W_G, self.W_NG = range(7)
        self.n_words = 7
        self.src = self._source()
        self.key = "lcm_vmu_" + hashlib.sha1(self.src.encode()).hexdigest()[:24]

    def name(self) -> str:
        return f"lcm_vmu_{self.spec.name}"

    def _source(self) -> str:
        spec = self.spec
        L: list[str] = [device_header(), _EXTRA_DEVICE]
        ap = L.append
        ap(f'extern "C" __global__ void __launch_bounds__(256) {self.name()}(const i64* __restrict__ items, '
           "const int* __restrict__ tile_prefix, int n_items, int n_tiles) {")
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* __restrict__ it = items + (i64)item * {self.n_words};")
        ap(f"    const double* __restrict__ PV = lcm_wp<const double>(it, {self.W_P});")
        ap(f"    const int period = lcm_wi(it, {self.W_PERIOD}); const double age = lcm_wd(it, {self.W_AGE});")
        ap("    (void)period; (void)age; (void)PV;")
        ap(f"    const double* __restrict__ V = lcm_wp<const double>(it, {self.W_V});")
        ap(f"    double* __restrict__ M = lcm_wp<double>(it, {self.W_M});")
        ap(f"    const double* __restrict__ G = lcm_wp<const double>(it, {self.W_G});")
        ap(f"    const int ng = lcm_wi(it, {self.W_NG});")
        ap("    const i64 e = (i64)(tile - tile_prefix[item]) * 256 + (int)threadIdx.x;")
        n_other = 1
        for a in spec.states:
            if a.name != self.euler:
                n_other *= a.size
        ap(f"    if (e >= (i64){n_other} * ng) continue;")
        # decode the flat state index (declaration order, last fastest)
        ap("    i64 rem = e; i64 se = 1; (void)se;")
        after = True
        for a in reversed(spec.states):
            size = "ng" if a.name == self.euler else str(a.size)
            ap(f"    const int c_{a.name} = (int)(rem % {size}); rem /= {size};")
            if a.name == self.euler:
                after = False
            elif after:
                ap(f"    se *= {a.size};")
        ap(f"    const int gi = c_{self.euler};")
        ap("    const double v = V[e];")
        if self.terminal:
            prov = {id(ir.var("period", "period", "i")): "period", id(ir.var("age", "age", "f")): "age"}
            for a in spec.states:
                if a.name == self.euler:
                    ap(f"    const double sv_{a.name} = G[gi];")
                    prov[id(ir.var("state", a.name, "f"))] = f"sv_{a.name}"
                elif a.kind == "continuous":
                    raise TracingError("passive continuous states are not carried")
                else:
                    prov[id(ir.var("state", a.name, "i"))] = f"c_{a.name}"
            em = Emitter("double", self.param_off, prov, "u")
            de = em.emit(ir.diff(self.U, ir.var("state", self.euler, "f")))
            for ln in em.lines:
                ap("    " + ln)
            ap(f"    M[e] = (v == -LCM_INF) ? 0.0 : (double)({de});")
        else:
            ap("    const bool fe = lcm_isfinite(v);")
            ap("    const bool hl = gi > 0 && lcm_isfinite(V[e - se]);")
            ap("    const bool hr = gi < ng - 1 && lcm_isfinite(V[e + se]);")
            ap("    double m = 0.0;")
            ap("    if (fe && hl && hr) {")
            ap("      const double hs = G[gi] - G[gi - 1], hd = G[gi + 1] - G[gi];")
            ap("      const double a = -hd / (hs * (hd + hs)), b = (hd - hs) / (hs * hd), c = hs / (hd * (hd + hs));")
            ap("      m = a * V[e - se] + b * v + c * V[e + se];")
            ap("    } else if (fe && hr) {")
            ap("      m = (V[e + se] - v) / (G[gi + 1] - G[gi]);")
            ap("    } else if (fe && hl) {")
            ap("      m = (v - V[e - se]) / (G[gi] - G[gi - 1]);")
            ap("    }")
            ap("    M[e] = m;")
        ap("  }")
        ap("}")
        return "\n".join(L)
