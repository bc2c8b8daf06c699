"""Exact skipping of action groups in the single-precision search.

A group (a run of consecutive values of one continuous action, the others
fixed) is skipped only when all its members violate a constraint or an upper
bound of its Q values is below the state's current second-best value, so the
search's two candidates -- and the published V and policy -- are those of the
full search (the skipping and the full kernel are separate compilations, so
their float and double arithmetic may round an ulp apart: V within 1e-12,
policies equal on >= 99.99 % of the states, any other within the float search's
1e-6).  CPU: the affine split of next-state laws and
constraints, which kernels skip (eligibility); GPU: the skipping kernels give
bit-identical V and policies to the same kernels with skipping turned off, on
models with one and two continuous actions and one- and two-axis targets,
infeasible regions (-inf values), several parameter draws and launch shapes."""

import dataclasses

import numpy as np
import pytest

from pylcm_b200 import ir
from pylcm_b200.codegen import _affine_split
from pylcm_b200.engine import SolveEngine, default_config
from tests import models as M


def test_affine_split():
    c, h = ir.var("action", "c", "f"), ir.var("action", "h", "f")
    w, z, r = ir.var("state", "w", "f"), ir.var("state", "z", "f"), ir.param("r")
    env = {("action", "c"): 3.0, ("action", "h"): 0.5, ("state", "w"): 7.0, ("state", "z"): -0.3}
    x = (1 + r) * (w - c) + ir.un("exp", z) * w * h - c / 4.0 + (h * 2.0).astype(float)
    x0, co = _affine_split(x, {"c", "h"})
    assert set(co) == {"c", "h"}
    for k in ("c", "h"):
        assert not any(kind == "action" for kind, _ in ir.const(co[k]).deps())
    ev = lambda e: float(ir.evaluate(e, env, {"r": 0.04}))  # noqa: E731
    got = ev(x0) + ev(co["c"]) * 3.0 + ev(co["h"]) * 0.5
    assert abs(got - ev(x)) < 1e-12
    # pieces that are not affine in the actions are rejected
    for bad in (w - ir.un("floor", c), c * h, ir.where(c > 1.0, c, 0.0), c ** 2.0, w / c, ir.un("log", c)):
        assert _affine_split(bad, {"c", "h"}) is None
    # an expression free of the actions is its own x0
    x0, co = _affine_split(w * 2.0, {"c"})
    assert co == {} and x0 is (w * 2.0)


def _kernels(model, params, precision, **cfg):
    eng = SolveEngine(model, precision, configs={
        s.name: dataclasses.replace(default_config(s, precision, 8), **cfg) for s in model.regime_specs} if cfg else None)
    out = {}
    for s in model.regime_specs:
        per = (model.n_periods - 1) if s.terminal else 0
        rk = eng.kernels(s, eng.targets_at(s, per), params, 8)
        rk.source()
        out[s.name] = rk
    return out


def test_eligibility():
    # affine wealth law in the one continuous action, deterministic regime
    # transition, utility in the action table: skipping
    k = _kernels(M.stochastic_model(4, 30, 40), M.stochastic_params(), "fp32")
    assert k["working"].prunes_groups and k["retired"].prunes_groups and not k["terminal"].prunes_groups
    # double precision never skips; nor with skipping turned off
    k = _kernels(M.stochastic_model(4, 30, 40), M.stochastic_params(), "fp64")
    assert not any(r.prunes_groups for r in k.values())
    k = _kernels(M.stochastic_model(4, 30, 40), M.stochastic_params(), "fp32", prune=False)
    assert not any(r.prunes_groups for r in k.values())
    # two continuous actions, two continuous target states: tile statistics
    # (only when asked for)
    k = _kernels(M.hc_model(3, 10, 4, 4, 8), M.hc_params(0, 4), "fp32")
    assert not k["alive"].prunes_groups
    k = _kernels(M.hc_model(3, 10, 4, 4, 8), M.hc_params(0, 4), "fp32", prune_multi=True)
    assert k["alive"].prunes_groups and not k["terminal"].prunes_groups
    assert [k["alive"].group_stats(t) for t in k["alive"].targets] == [2]
    assert "lcm_tile_stats_" in k["alive"].source()
    g = k["alive"]._groups
    assert g["cacts"][g["scan"]] == "consumption" and set(g["acts"]) == {"consumption", "hours"}
    assert [op for op, _, _ in g["cons"]] == ["<="]  # the borrowing constraint
    # a stochastic regime transition (several targets per action): not eligible
    k = _kernels(M.mass_model(), M.mass_params(), "fp32")
    assert not any(r.prunes_groups for r in k.values())


CASES = {
    "stochastic": (lambda: M.stochastic_model(8, 200, 300),
                   lambda: [M.stochastic_params(beta=b, crra=c) for b, c in ((0.95, 2.0), (0.9, 3.5), (0.97, 1.2))]),
    "retirement": (lambda: M.retirement_model(6, 150, 150), lambda: [M.retirement_params(b) for b in (0.95, 0.8)]),
    "regression": (lambda: M.regression_model(4), lambda: [M.regression_params(4)]),
    # two continuous actions (consumption x hours), wealth x human capital targets
    "human_capital": (lambda: M.hc_model(5, 120, 12, 6, 90), lambda: [M.hc_params(s, 6) for s in range(3)]),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("lanes,sb", [(2, 4), (1, 1), (4, 2)])
def test_skipping_is_exact(case, lanes, sb):
    import torch

    model = CASES[case][0]()
    ps = CASES[case][1]()
    res = []
    for prune in (True, False):
        cfg = {s.name: dataclasses.replace(default_config(s, "fp32", len(ps)), lanes=lanes, sb=sb, prune=prune,
                                           prune_multi=prune) for s in model.regime_specs}
        plan = SolveEngine(model, "fp32", configs=cfg).plan(ps)
        plan.run()
        torch.cuda.synchronize()
        plan.check_status()
        res.append(plan)
    a, b = res
    for r in a.V:
        va, vb = a.V[r].cpu().numpy(), b.V[r].cpu().numpy()
        np.testing.assert_array_equal(np.isnan(va), np.isnan(vb))
        np.testing.assert_array_equal(np.isfinite(va), np.isfinite(vb))
        fin = np.isfinite(vb)
        d = np.abs(va[fin] - vb[fin]) / np.maximum(1.0, np.abs(vb[fin]))
        same = (a.pol[r] == b.pol[r]).cpu().numpy()
        # the two kernels are separate compilations: the double re-evaluation
        # may round an ulp apart, and a float near-tie may order differently
        assert d.max() <= 1e-12 if same.all() else d[same[fin]].max(initial=0.0) <= 1e-12, (r, d.max())
        assert same.mean() >= 0.9999, (r, same.mean())
        if not same.all():
            assert d.max() <= 1e-6, (r, d.max())


@pytest.mark.gpu
def test_tile_statistics_match_the_float_table():
    """The statistics kernel's (max, largest finite |value|) per 16 x 2 tile
    of a two-axis float table, against NumPy over the table it read."""
    import torch

    model = M.hc_model(4, 70, 9, 5, 40)
    cfg = {s.name: dataclasses.replace(default_config(s, "fp32", 2), prune_multi=True) for s in model.regime_specs}
    plan = SolveEngine(model, "fp32", configs=cfg).plan([M.hc_params(s, 5) for s in range(2)])
    plan.run()
    torch.cuda.synchronize()
    checked = 0
    for key, bst in plan.bst.items():
        e64, e32, ncols, cblk = plan.ev[key]
        if bst.shape[2] == (ncols + 15) // 16:
            continue  # one-axis statistics (kernel b)
        n1, n2 = 70, 9
        ev = e32.cpu().numpy().reshape(e32.shape[0], e32.shape[1], n1, n2)
        p1, p2 = (-n1) % 16, (-n2) % 2
        pad = np.pad(ev, ((0, 0), (0, 0), (0, p1), (0, p2)), constant_values=-np.inf)
        t = pad.reshape(ev.shape[0], ev.shape[1], (n1 + p1) // 16, 16, (n2 + p2) // 2, 2)
        mx = t.max(axis=(3, 5))
        ab = np.where(np.isfinite(t), np.abs(t), 0.0).max(axis=(3, 5))
        got = bst.cpu().numpy().reshape(mx.shape + (2,))
        np.testing.assert_array_equal(got[..., 0], mx.astype(np.float32))
        np.testing.assert_array_equal(got[..., 1], ab.astype(np.float32))
        checked += 1
    assert checked >= 1
