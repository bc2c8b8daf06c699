"""Heterogeneous batches (one launch per kernel over models of one family with
different grid sizes and horizons) and the continuous-batching server."""

import dataclasses
import gc

import numpy as np
import pytest

from pylcm_b200 import examples as E
from pylcm_b200.engine import BatchPlan, LaunchConfig, SolveEngine
from pylcm_b200.serving import Server, footprint_bytes

pytestmark = pytest.mark.gpu


def _engine(model, precision):
    cfg = {s.name: LaunchConfig() for s in model.regime_specs}
    return SolveEngine(model, precision, configs=cfg)


def _assert_same_solution(bp_res, one_res):
    V1, P1 = bp_res
    V2, P2 = one_res
    assert V1.keys() == V2.keys()
    for p in V1:
        for r in V1[p]:
            np.testing.assert_array_equal(V1[p][r].cpu().numpy(), V2[p][r].cpu().numpy())
            np.testing.assert_array_equal(P1[p][r].cpu().numpy(), P2[p][r].cpu().numpy())


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_plan_of_uneven_models_matches_single_solves(precision):
    import torch

    shapes = [(6, 40, 30), (9, 70, 45), (4, 25, 60)]
    models = [E.stochastic_model(T, n, c) for T, n, c in shapes]
    params = [E.stochastic_params(beta=0.93 + 0.01 * k, crra=1.5 + k, interest_rate=0.02 + 0.01 * k) for k in range(3)]
    engs = [_engine(m, precision) for m in models]
    bp = BatchPlan(list(zip(engs, params)))
    bp.run()
    torch.cuda.synchronize()
    # one launch per (step, kernel): fewer launches than the instances' sum
    assert bp.gpu_launches < sum(len(p.launches) for p in bp.plans)
    for k in range(3):
        one = engs[k].plan([params[k]])
        one.run()
        torch.cuda.synchronize()
        _assert_same_solution(bp.result(k), one.result(0))


def test_batch_plan_of_dcegm_models_matches_single_solves():
    import torch

    shapes = [(5, 120), (7, 90)]
    models = [E.dcegm_model(n_periods=T, n_savings=n, n_wealth=n, taste=True) for T, n in shapes]
    params = [E.dcegm_params(seed=k, taste_scale=0.05, crra=1.5 + k) for k in range(2)]
    engs = [_engine(m, "fp64") for m in models]
    bp = BatchPlan(list(zip(engs, params)))
    bp.run()
    torch.cuda.synchronize()
    for k in range(2):
        one = engs[k].plan([params[k]])
        one.run()
        torch.cuda.synchronize()
        _assert_same_solution(bp.result(k), one.result(0))


def test_simulation_over_a_batch_plan_matches_single_runs():
    import torch

    from pylcm_b200.simulate import SimPlan

    reqs = E.serving_requests(6, seed=4, n_agents=300, sizes=(40, 70), horizons=(4, 6), n_consumption=50)
    fam = [r for r in reqs if r.family == "stochastic_retirement"][:3]
    assert len(fam) >= 2
    engs = [_engine(r.model, "fp64") for r in fam]
    bp = BatchPlan([(e, r.params) for e, r in zip(engs, fam)])
    bp.run()
    sim = SimPlan(bp, instances=[(k, r.initial_conditions, r.seed) for k, r in enumerate(fam)])
    sim.run()
    torch.cuda.synchronize()
    for k, r in enumerate(fam):
        got = sim.result(k=k)
        plan = engs[k].plan([r.params])
        plan.run()
        one = SimPlan(plan, r.initial_conditions, r.seed)
        one.run()
        exp = one.result()
        for p in exp.periods:
            np.testing.assert_array_equal(got.periods[p]["regime_id"], exp.periods[p]["regime_id"])
            np.testing.assert_array_equal(got.periods[p]["value"], exp.periods[p]["value"])
            for n in ("wealth", "income"):
                np.testing.assert_array_equal(got.periods[p]["states"][n], exp.periods[p]["states"][n])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_served_request_is_the_same_alone_and_in_the_mix(precision):
    """Exact equality (tolerance 0): a request's moments and value functions
    do not depend on the batch or on the jobs it overlaps with."""
    reqs = E.serving_requests(14, seed=3, n_agents=500, sizes=(40, 80), horizons=(4, 7), n_consumption=60,
                              return_V_every=1)
    mix_server = Server(precision=precision, max_batch=8, n_streams=3)
    mix = mix_server.run(reqs, realtime=False)
    assert max(mix_server.batch_sizes) > 1  # batches actually formed
    for pick in (0, 5, 9):
        alone = Server(precision=precision, max_batch=1, n_streams=1).run([dataclasses.replace(reqs[pick])],
                                                                            realtime=False)[0]
        a, m = alone, mix[pick]
        assert a.rid == m.rid == pick
        for name in a.moments:
            np.testing.assert_array_equal(a.moments[name], m.moments[name])
        for p in a.V:
            for r in a.V[p]:
                np.testing.assert_array_equal(a.V[p][r], m.V[p][r])


def test_fast_serving_matches_fp64_values():
    """Single-precision search, double-precision values: V within 1e-6
    (relative) of the FP64 form on served requests."""
    reqs = E.serving_requests(8, seed=6, n_agents=200, sizes=(60, 120), horizons=(5, 8), n_consumption=80,
                              return_V_every=1)
    fast = Server(precision="fp32", max_batch=8).run([dataclasses.replace(r) for r in reqs], realtime=False)
    plain = Server(precision="fp64", max_batch=1, n_streams=1).run([dataclasses.replace(r) for r in reqs],
                                                                   realtime=False)
    worst = 0.0
    for f, p in zip(fast, plain):
        for per in p.V:
            for r in p.V[per]:
                a, b = f.V[per][r], p.V[per][r]
                fin = np.isfinite(b)
                np.testing.assert_array_equal(np.isfinite(a), fin)
                err = np.abs(a[fin] - b[fin]) / np.maximum(1.0, np.abs(b[fin]))
                worst = max(worst, float(err.max(initial=0.0)))
    assert worst <= 1e-6


def test_admission_holds_the_hbm_budget():
    reqs = E.serving_requests(8, seed=7, n_agents=400, sizes=(40, 80), horizons=(4, 7), n_consumption=60)
    srv = Server(precision="fp32", max_batch=8, n_streams=4, hbm_budget_bytes=1)
    fps = [srv.footprint(r) for r in reqs]
    budget = int(max(fps) * 1.5)
    srv = Server(precision="fp32", max_batch=8, n_streams=4, hbm_budget_bytes=budget)
    res = srv.run(reqs, realtime=False)
    assert len(res) == len(reqs)
    assert srv.peak_in_use <= budget
    with pytest.raises(MemoryError):
        Server(precision="fp32", hbm_budget_bytes=max(fps) // 2).run(reqs[:1], realtime=False)


def test_footprint_estimate_covers_the_allocations():
    import torch

    from pylcm_b200.simulate import SimPlan

    for r in E.serving_requests(4, seed=8, n_agents=2000, sizes=(200,), horizons=(10,), n_consumption=100):
        eng = _engine(r.model, "fp32")
        gc.collect()  # plans of the previous iteration hold reference cycles
        torch.cuda.synchronize()
        before = torch.cuda.memory_allocated()
        bp = BatchPlan([(eng, r.params)])
        sim = SimPlan(bp, instances=[(0, r.initial_conditions, r.seed)])
        torch.cuda.synchronize()
        used = torch.cuda.memory_allocated() - before
        est = footprint_bytes(eng, 2000)
        assert 0.5 * used <= est <= 3.0 * used, (r.family, est, used)
        del bp, sim


def test_pools_are_reused_and_evicted_without_changing_results():
    """A second pass over the same requests reuses the pooled slots (no new
    pools) and gives the same numbers; a budget that holds only a few pools
    forces evictions and still gives the same numbers."""
    reqs = E.serving_requests(10, seed=9, n_agents=300, sizes=(40, 80), horizons=(4, 7), n_consumption=60,
                              return_V_every=1)
    srv = Server(precision="fp32", max_batch=4, n_streams=2)
    first = srv.run([dataclasses.replace(r) for r in reqs], realtime=False)
    built = srv.pools_built
    second = srv.run([dataclasses.replace(r) for r in reqs], realtime=False)
    assert srv.pools_built == built
    fps = [srv.footprint(r) for r in reqs]
    tight = Server(precision="fp32", max_batch=4, n_streams=2, hbm_budget_bytes=int(3 * max(fps)), pool_slots=1)
    third = tight.run([dataclasses.replace(r) for r in reqs], realtime=False)
    assert tight.pools_evicted > 0
    assert tight.peak_in_use <= tight.budget
    for a, b, c in zip(first, second, third):
        for name in a.moments:
            np.testing.assert_array_equal(a.moments[name], b.moments[name])
            np.testing.assert_array_equal(a.moments[name], c.moments[name])
        for p in a.V:
            for r in a.V[p]:
                np.testing.assert_array_equal(a.V[p][r], c.V[p][r])
