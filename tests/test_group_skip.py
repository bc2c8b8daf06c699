"""Exact skipping of action groups in the single-precision search.

A group of consecutive continuous actions is skipped only when an upper bound
of its Q values is below the state's current second-best value, so the
search's two candidates -- and the published V and policy -- are exactly
those of the full search.  CPU: which kernels skip (eligibility); GPU: the
skipping kernels give bit-identical V and policies to the same kernels with
skipping turned off, on models with infeasible regions (-inf values), several
parameter draws and launch shapes."""

import dataclasses

import numpy as np
import pytest

from pylcm_b200.engine import SolveEngine, default_config
from tests import models as M


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
    # two continuous target states: not eligible
    k = _kernels(M.hc_model(3, 10, 4, 4, 8), M.hc_params(0, 4), "fp32")
    assert not any(r.prunes_groups for r in k.values())
    # a stochastic regime transition (several targets per action): not eligible
    k = _kernels(M.mass_model(), M.mass_params(), "fp32")
    assert not any(r.prunes_groups for r in k.values())


CASES = {
    "stochastic": (lambda: M.stochastic_model(8, 200, 300),
                   lambda: [M.stochastic_params(beta=b, crra=c) for b, c in ((0.95, 2.0), (0.9, 3.5), (0.97, 1.2))]),
    "retirement": (lambda: M.retirement_model(6, 150, 150), lambda: [M.retirement_params(b) for b in (0.95, 0.8)]),
    "regression": (lambda: M.regression_model(4), lambda: [M.regression_params(4)]),
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
        cfg = {s.name: dataclasses.replace(default_config(s, "fp32", len(ps)), lanes=lanes, sb=sb, prune=prune)
               for s in model.regime_specs}
        plan = SolveEngine(model, "fp32", configs=cfg).plan(ps)
        plan.run()
        torch.cuda.synchronize()
        plan.check_status()
        res.append(plan)
    a, b = res
    for r in a.V:
        assert torch.equal(torch.nan_to_num(a.V[r], nan=7.0), torch.nan_to_num(b.V[r], nan=7.0)), r
        assert torch.equal(a.pol[r], b.pol[r]), r
