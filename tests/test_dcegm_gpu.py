"""DC-EGM on the GPU (kernels c1/FUES/c3) vs the DC-EGM oracle and the
Iskhakov et al. (2017) closed form.

Bar: V within 1e-10 relative (|a-b| / max(1,|b|)) of the oracle -- FUES
crossings and the Hermite reads round differently under fused multiply-add;
within 1e-3 absolute of the closed form (nodes above the two lowest)."""

import numpy as np
import pytest

from oracle.dcegm import solve as oracle_solve
from tests import models as M
from tests.conftest import rel_err
from tests.golden import analytical_models as AM

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["five_periods", "low_delta"])
def test_dcegm_gpu_matches_oracle_and_closed_form(case):
    model, params = AM.dcegm_model_and_params(case)
    V = model.solve(params=params, log_level="off")
    Vo, _ = oracle_solve(model, params)
    for p in Vo:
        for r in Vo[p]:
            assert rel_err(V[p][r], Vo[p][r]) < 1e-10, (p, r)
    periods = sorted(V)
    for kind, reg in (("worker", "working_life"), ("retired", "retirement")):
        num = np.stack([V[p][reg] for p in periods[:-1]])
        ana = np.load(f"tests/golden/analytical_{case}__values_{kind}.npy")
        assert np.abs(num - ana)[:, 2:].max() < 1e-3


@pytest.mark.parametrize("taste", [None, 0.05])
def test_dcegm_income_shock_model_matches_oracle(taste):
    model = M.dcegm_model(n_periods=5, n_savings=200, n_wealth=100, taste=taste is not None)
    params = M.dcegm_params(0, taste_scale=taste)
    V = model.solve(params=params, log_level="off")
    Vo, _ = oracle_solve(model, params)
    for p in Vo:
        for r in Vo[p]:
            assert rel_err(V[p][r], Vo[p][r]) < 1e-10, (taste, p, r)


@pytest.mark.parametrize("window", [3, 25])
def test_dcegm_bounded_look_ahead_matches_oracle(window):
    """FUESEnvelope(n_points_to_scan=k) on the GPU and in the oracle."""
    model = M.dcegm_model(n_periods=5, n_savings=200, n_wealth=100, n_points_to_scan=window)
    params = M.dcegm_params(4)
    V = model.solve(params=params, log_level="off")
    Vo, _ = oracle_solve(model, params)
    for p in Vo:
        for r in Vo[p]:
            assert rel_err(V[p][r], Vo[p][r]) < 1e-10, (window, p, r)


def test_dcegm_batch_equals_single():
    model = M.dcegm_model(n_periods=4, n_savings=120, n_wealth=60)
    ps = [M.dcegm_params(s) for s in range(3)]
    eng = model.engine("fp64")
    batch = eng.solve_batch(ps)
    for p, (Vb, _) in zip(ps, batch):
        V1, _ = eng.solve(p)
        for per in V1:
            for r in V1[per]:
                assert np.array_equal(V1[per][r].cpu().numpy(), Vb[per][r].cpu().numpy())


@pytest.mark.parametrize("taste", [None, 0.05])
def test_dcegm_simulation_matches_oracle(taste):
    """Simulation of DC-EGM regimes: grid argmax of Q over the consumption grid
    with the intrinsic budget mask, against the DC-EGM value functions, draw
    for draw against the oracle."""
    from oracle.simulate import simulate as oracle_simulate

    model = M.dcegm_model(n_periods=5, n_savings=200, n_wealth=100, taste=taste is not None)
    params = M.dcegm_params(seed=2, taste_scale=taste)
    n = 96
    rng = np.random.default_rng(5)
    rid = {s.name: s.rid for s in model.regime_specs}
    ic = {
        "wealth": rng.uniform(1, 50, n),
        "shock": rng.integers(0, 16, n).astype(float),
        "age": np.zeros(n),
        "regime_id": np.where(rng.uniform(size=n) < 0.8, rid["working"], rid["retired"]),
    }
    res = model.simulate(params=params, initial_conditions=ic, seed=11)
    ora = oracle_simulate(model, params, ic, seed=11)
    for p in ora:
        np.testing.assert_array_equal(res.periods[p]["regime_id"], ora[p]["regime_id"])
        for name in ("wealth", "shock"):
            np.testing.assert_allclose(res.periods[p]["states"][name], ora[p]["states"][name], rtol=1e-9, atol=1e-9, equal_nan=True)
        np.testing.assert_allclose(res.periods[p]["value"], ora[p]["value"], rtol=1e-9, atol=1e-9, equal_nan=True)
        for name in ("consumption", "labor_supply"):
            np.testing.assert_allclose(res.periods[p]["actions"][name], ora[p]["actions"][name], equal_nan=True)


@pytest.mark.parametrize("taste", [None, 0.1])
def test_dcegm_reads_grid_search_and_terminal_value_arrays(taste):
    """DC-EGM regime whose targets are a grid-search regime and a terminal
    regime over wealth x Markov health: both carried as value arrays (the
    grid-search one with its finite-difference wealth slope, the terminal
    one with its utility gradient), the health law folded into the rows;
    -inf values at zero wealth."""
    model = M.value_children_model(taste=taste is not None)
    for params in (M.value_children_params(taste), M.value_children_params(taste, p_stay_good=0.7)):
        V = model.solve(params=params, log_level="off")
        Vo, _ = oracle_solve(model, params)
        for p in Vo:
            for r in Vo[p]:
                assert rel_err(V[p][r], Vo[p][r]) < 1e-10, (p, r)


@pytest.mark.parametrize("taste", [None, 0.1])
def test_simulation_through_value_array_targets_matches_oracle(taste):
    """Subjects of the DC-EGM / grid-search / terminal model, draw for draw
    against the oracle: regime draws, Markov health draws and (with taste
    shocks) Gumbel draws into the grid-search and terminal regimes."""
    from oracle.simulate import simulate as oracle_simulate

    model = M.value_children_model(taste=taste is not None)
    params = M.value_children_params(taste)
    n = 64
    rng = np.random.default_rng(5)
    rid = {s.name: s.rid for s in model.regime_specs}
    ic = {
        "wealth": rng.uniform(0.5, 30, n),
        "health": rng.integers(0, 2, n).astype(float),
        "age": np.zeros(n),
        "regime_id": np.where(rng.uniform(size=n) < 0.7, rid["working"], rid["retired"]),
    }
    res = model.simulate(params=params, initial_conditions=ic, seed=3)
    ora = oracle_simulate(model, params, ic, seed=3)
    for p in ora:
        np.testing.assert_array_equal(res.periods[p]["regime_id"], ora[p]["regime_id"])
        for name in ("wealth", "health"):
            np.testing.assert_allclose(res.periods[p]["states"][name], ora[p]["states"][name], rtol=1e-9, atol=1e-9,
                                       equal_nan=True)
        np.testing.assert_allclose(res.periods[p]["value"], ora[p]["value"], rtol=1e-9, atol=1e-9, equal_nan=True)
        for name in ("consumption", "work_choice"):
            np.testing.assert_allclose(res.periods[p]["actions"][name], ora[p]["actions"][name], equal_nan=True)


@pytest.mark.parametrize("taste", [None, 0.1])
def test_dcegm_with_an_income_process_matches_oracle(taste):
    """DC-EGM rows over an AR(1) income process (Tauchen transition rows as
    the weights of its own carry and of a grid-search target's value array),
    solve and simulation against the oracle."""
    from oracle.simulate import simulate as oracle_simulate

    model = M.egm_process_model(taste=taste is not None)
    for params in (M.egm_process_params(taste), M.egm_process_params(taste, rho=0.5)):
        V = model.solve(params=params, log_level="off")
        Vo, _ = oracle_solve(model, params)
        for p in Vo:
            for r in Vo[p]:
                assert rel_err(V[p][r], Vo[p][r]) < 1e-10, (p, r)
    n = 64
    rng = np.random.default_rng(8)
    rid = {s.name: s.rid for s in model.regime_specs}
    ic = {"wealth": rng.uniform(0.5, 30, n), "income": rng.normal(0.0, 0.3, n), "age": np.zeros(n),
          "regime_id": np.where(rng.uniform(size=n) < 0.7, rid["working"], rid["retired"])}
    res = model.simulate(params=params, initial_conditions=ic, seed=4)
    ora = oracle_simulate(model, params, ic, seed=4)
    for p in ora:
        np.testing.assert_array_equal(res.periods[p]["regime_id"], ora[p]["regime_id"])
        for name in ("wealth", "income"):
            np.testing.assert_allclose(res.periods[p]["states"][name], ora[p]["states"][name], rtol=1e-9, atol=1e-9,
                                       equal_nan=True)
        np.testing.assert_allclose(res.periods[p]["value"], ora[p]["value"], rtol=1e-9, atol=1e-9, equal_nan=True)


@pytest.mark.parametrize("envelope", ["ltm", "rfc", "mss"])
@pytest.mark.parametrize("case", ["five_periods", "low_delta"])
def test_dcegm_other_envelopes_match_oracle_and_closed_form(envelope, case):
    """DCEGM(envelope=LTMEnvelope() / RFCEnvelope() / MSSEnvelope()) on the
    GPU against the oracle with the same envelope (1e-10), and within 1e-3 of
    the closed form (LTM and RFC insert no segment crossing, so a kink is
    recovered to within the grid spacing)."""
    from pylcm_b200 import LTMEnvelope, MSSEnvelope, RFCEnvelope

    env = {"ltm": LTMEnvelope(), "rfc": RFCEnvelope(), "mss": MSSEnvelope()}[envelope]
    model, params = AM.dcegm_model_and_params(case, env)
    V = model.solve(params=params, log_level="off")
    Vo, _ = oracle_solve(model, params)
    for p in Vo:
        for r in Vo[p]:
            assert rel_err(V[p][r], Vo[p][r]) < 1e-10, (envelope, p, r)
    periods = sorted(V)
    for kind, reg in (("worker", "working_life"), ("retired", "retirement")):
        num = np.stack([V[p][reg] for p in periods[:-1]])
        ana = np.load(f"tests/golden/analytical_{case}__values_{kind}.npy")
        assert np.abs(num - ana)[:, 2:].max() < 1e-3


@pytest.mark.parametrize("taste", [None, 0.05])
def test_dcegm_rfc_income_shock_model_matches_oracle(taste):
    from pylcm_b200 import RFCEnvelope

    model = M.dcegm_model(n_periods=5, n_savings=200, n_wealth=100, taste=taste is not None,
                          envelope=RFCEnvelope(search_radius=6, jump_thresh=1.5))
    params = M.dcegm_params(2, taste_scale=taste)
    V = model.solve(params=params, log_level="off")
    Vo, _ = oracle_solve(model, params)
    for p in Vo:
        for r in Vo[p]:
            assert rel_err(V[p][r], Vo[p][r]) < 1e-10, (taste, p, r)
