"""GPU simulation (kernel d) vs the reference's stored simulation and the oracle."""

import numpy as np
import pytest

from oracle.simulate import simulate as oracle_simulate
from tests import models as M
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_regression_simulation_matches_reference_golden():
    """Deterministic model: the reference's stored simulation (float32 columns,
    compared at atol 1e-5 like the reference's own test)."""
    g = np.load(GOLDEN / "regression_simulation.npz", allow_pickle=True)
    model = M.regression_model(4)
    params = M.regression_params(4)
    res = model.simulate(
        params=params,
        initial_conditions={
            "wealth": np.array([5.0, 20, 40, 70]),
            "age": np.array([18.0, 18.0, 18.0, 18.0]),
            "regime_id": np.array([0, 0, 0, 0]),
        },
        period_to_regime_to_V_arr=None,
    )
    df = res.to_dataframe(terminal_rows="all").sort_values(["subject_id", "period"]).reset_index(drop=True)
    assert len(df) == len(g["subject_id"])
    np.testing.assert_array_equal(df["subject_id"].to_numpy(), g["subject_id"])
    np.testing.assert_array_equal(df["period"].to_numpy(), g["period"])
    np.testing.assert_array_equal(df["regime_name"].astype(str).to_numpy(), g["regime"])
    for col in ("value", "wealth", "consumption", "age"):
        np.testing.assert_allclose(df[col].to_numpy(), g[col], atol=1e-5, rtol=0, equal_nan=True)
    got_ls = df["labor_supply"].astype(object).where(df["labor_supply"].notna(), "nan").astype(str).to_numpy()
    np.testing.assert_array_equal(got_ls, g["labor_supply"].astype(str))


@pytest.mark.parametrize("kind", ["tauchen", "rouwenhorst", "normal", "uniform"])
def test_stochastic_simulation_matches_oracle_draw_for_draw(kind):
    model = M.processes_model(4, kind)
    params = M.processes_params(kind)
    n = 64
    rng = np.random.default_rng(0)
    ic = {
        "wealth": rng.uniform(1, 5, n),
        "income": np.zeros(n),
        "health": rng.integers(0, 2, n).astype(float),
        "age": np.zeros(n),
        "regime_id": np.zeros(n, dtype=int),
    }
    res = model.simulate(params=params, initial_conditions=ic, seed=1234)
    ora = oracle_simulate(model, params, ic, seed=1234)
    for p in ora:
        np.testing.assert_array_equal(res.periods[p]["regime_id"], ora[p]["regime_id"])
        for name in ("wealth", "income", "health"):
            np.testing.assert_allclose(res.periods[p]["states"][name], ora[p]["states"][name], rtol=1e-10, atol=1e-12, equal_nan=True)
        np.testing.assert_allclose(res.periods[p]["value"], ora[p]["value"], rtol=1e-10, atol=1e-12, equal_nan=True)
        np.testing.assert_allclose(res.periods[p]["actions"]["consumption"], ora[p]["actions"]["consumption"], equal_nan=True)


def test_stochastic_model_simulation_matches_oracle():
    model = M.stochastic_model(6, 40, 50)
    params = M.stochastic_params()
    n = 100
    rng = np.random.default_rng(3)
    ic = {
        "wealth": rng.uniform(1, 50, n),
        "income": rng.normal(0, 0.1, n),
        "age": np.zeros(n),
        "regime_id": np.zeros(n, dtype=int),
    }
    res = model.simulate(params=params, initial_conditions=ic, seed=7)
    ora = oracle_simulate(model, params, ic, seed=7)
    for p in ora:
        np.testing.assert_array_equal(res.periods[p]["regime_id"], ora[p]["regime_id"])
        for name in ("wealth", "income"):
            np.testing.assert_allclose(res.periods[p]["states"][name], ora[p]["states"][name], rtol=1e-9, atol=1e-9, equal_nan=True)


def test_simulated_draws_have_the_process_moments():
    """AR(1) draws: the simulated income process has the innovation's
    conditional mean and variance (distributional check, seeded)."""
    model = M.stochastic_model(4, 30, 40)
    params = M.stochastic_params()
    n = 20000
    ic = {"wealth": np.full(n, 20.0), "income": np.zeros(n), "age": np.zeros(n), "regime_id": np.zeros(n, dtype=int)}
    res = model.simulate(params=params, initial_conditions=ic, seed=99)
    y1 = res.periods[1]["states"]["income"]
    # y' = 0 + 0.9 * 0 + 0.1 * eps
    assert abs(np.mean(y1)) < 4 * 0.1 / np.sqrt(n)
    assert abs(np.std(y1) - 0.1) < 0.005


@pytest.mark.parametrize("rng", ["philox", "jax"])
def test_batched_simulation_equals_single_instance_runs(rng):
    """One kernel (d) launch per (period, regime) over several solve instances,
    each with its own seed and subjects, gives each instance's single run."""
    from pylcm_b200.simulate import SimPlan

    model = M.stochastic_model(5, 40, 50)
    plist = [M.stochastic_params(), {**M.stochastic_params(), "discount_factor": 0.9}, M.stochastic_params()]
    eng = model.engine("fp64")
    plan = eng.plan(plist)
    plan.run()
    gen = np.random.default_rng(8)
    ics, seeds = [], [3, 4, 3]
    for k in range(3):
        n = 40 + 17 * k
        ics.append({
            "wealth": gen.uniform(1, 50, n),
            "income": gen.normal(0, 0.1, n),
            "age": np.zeros(n),
            "regime_id": np.zeros(n, dtype=int),
        })
    sim = SimPlan(plan, instances=[(k, ics[k], seeds[k]) for k in range(3)], rng=rng, params=plist)
    sim.run()
    for k in range(3):
        got = sim.result(model, k)
        one = model.simulate(params=plist[k], initial_conditions=ics[k], seed=seeds[k], rng=rng)
        for p in one.periods:
            np.testing.assert_array_equal(got.periods[p]["regime_id"], one.periods[p]["regime_id"])
            np.testing.assert_array_equal(got.periods[p]["value"], one.periods[p]["value"])
            for name in ("wealth", "income"):
                np.testing.assert_array_equal(got.periods[p]["states"][name], one.periods[p]["states"][name])


@pytest.mark.parametrize("kind", ["irreg", "log", "piece_lin", "piece_log"])
def test_simulation_on_every_grid_kind_matches_oracle(kind):
    """Subjects read the next-period values on irregular, log-spaced and
    piecewise grids (above the top node too: extrapolation by the last
    segment's spacing), draw for draw against the oracle."""
    model = M.grid_kinds_model(kind)
    params = M.grid_kinds_params()
    n = 64
    rng = np.random.default_rng(9)
    ic = {"wealth": rng.uniform(1.0, 70.0, n), "health": rng.integers(0, 2, n).astype(float), "age": np.zeros(n),
          "regime_id": np.zeros(n, dtype=int)}
    res = model.simulate(params=params, initial_conditions=ic, seed=6)
    ora = oracle_simulate(model, params, ic, seed=6)
    for p in ora:
        np.testing.assert_array_equal(res.periods[p]["regime_id"], ora[p]["regime_id"])
        for name in ("wealth", "health"):
            np.testing.assert_allclose(res.periods[p]["states"][name], ora[p]["states"][name], rtol=1e-9, atol=1e-9,
                                       equal_nan=True)
        np.testing.assert_allclose(res.periods[p]["value"], ora[p]["value"], rtol=1e-9, atol=1e-9, equal_nan=True)
        np.testing.assert_allclose(res.periods[p]["actions"]["consumption"], ora[p]["actions"]["consumption"],
                                   equal_nan=True)
