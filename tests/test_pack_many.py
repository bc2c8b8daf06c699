"""Column-wise packing of many parameter sets equals the per-set packing,
row for row, and rejects what the per-set packing rejects."""

import copy

import numpy as np
import pytest

from pylcm_b200.egm import is_egm, trace_egm_regime
from pylcm_b200.exceptions import InvalidParamsError
from pylcm_b200.spec import ParamResolver, trace_regime
from tests import models as M


def _resolvers(model, plist):
    names = tuple(s.name for s in model.regime_specs)
    return [ParamResolver(p, model.fixed_params, names) for p in plist]


def _traces(model, params):
    specs = model.regime_specs
    res = _resolvers(model, [params])[0]
    out = []
    for s in specs:
        targets = () if s.terminal else tuple(x.name for x in specs)
        if is_egm(s) and not s.terminal:
            er = trace_egm_regime(s, specs, res, targets)
            out.append((er.pack_many, er.pack_for))
        else:
            tr = trace_regime(s, specs, res, targets)
            out.append((tr.pack_many, lambda r, tr=tr: tr.pack_params(tr.values_for(r))))
    return out


@pytest.mark.parametrize("case", ["stochastic", "processes", "dcegm", "hc"])
def test_pack_many_equals_per_set_packing(case):
    rng = np.random.default_rng(3)
    if case == "stochastic":
        model = M.stochastic_model(4, 30, 30)
        plist = [M.stochastic_params(beta=float(rng.uniform(0.9, 0.97)), crra=float(rng.uniform(1.5, 2.5)))
                 for _ in range(7)]
    elif case == "processes":
        model = M.processes_model(3, "tauchen")
        plist = [copy.deepcopy(M.processes_params("tauchen")) for _ in range(3)]
        plist[1]["alive"]["income"]["rho"] = 0.5  # a second process table
    elif case == "dcegm":
        model = M.dcegm_model(n_periods=4, n_savings=50, n_wealth=40, taste=True)
        plist = [M.dcegm_params(k, taste_scale=0.05) for k in range(5)]
    else:
        model = M.hc_model(n_periods=4, n_wealth=8, n_hc=6, n_shock=5, n_consumption=20)
        plist = [M.hc_params(seed=k, n_shock=5) for k in range(3)]
    res = _resolvers(model, plist)
    memo: dict = {}
    for many, one in _traces(model, plist[0]):
        got = many(res, memo)
        want = np.stack([one(r) for r in res])
        np.testing.assert_array_equal(got, want)
        if case == "processes" and got.shape[1] > 20:
            assert not np.array_equal(got[0], got[1])  # the two process tables differ


def test_pack_many_rejects_missing_and_misshaped_parameters():
    model = M.stochastic_model(4, 30, 30)
    good = M.stochastic_params()
    bad = {k: v for k, v in good.items() if k != "discount_factor"}
    traces = _traces(model, good)
    with pytest.raises(InvalidParamsError):
        for many, _ in traces:
            many(_resolvers(model, [good, bad]))
    wrong = dict(good)
    wrong["discount_factor"] = [0.9, 0.95]
    with pytest.raises(InvalidParamsError):
        for many, _ in traces:
            many(_resolvers(model, [good, wrong]))
