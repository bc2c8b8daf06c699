"""Transition checks before solve (the reference's ``validate_transitions``,
``src/_lcm/transition_checks.py:51-647``) and the continuation's mass check
(``src/_lcm/regime_building/Q_and_F.py:1401-1432``) in the oracle.

The GPU side of the mass check is in ``tests/test_mass_check_gpu.py``."""

import warnings

import numpy as np
import pytest

from oracle.grid_search import solve as oracle_solve
from pylcm_b200 import InvalidRegimeTransitionProbabilitiesError, InvalidStateTransitionProbabilitiesError
from pylcm_b200.validation import validate_transitions
from tests import models as M

BAD = {
    "mass_above_tolerance": M.mass_params(mass=1.01),
    "negative_probability": M.mass_params(p_survive=-0.1),
}


@pytest.mark.parametrize("case", sorted(BAD))
def test_debug_raises_on_a_malformed_regime_transition(case):
    model = M.mass_model()
    with pytest.raises(InvalidRegimeTransitionProbabilitiesError):
        validate_transitions(model, BAD[case], "debug")
    # solve validates first: it raises before any device work
    with pytest.raises(InvalidRegimeTransitionProbabilitiesError):
        model.solve(params=BAD[case], log_level="debug")


@pytest.mark.parametrize("level", ["warning", "progress"])
def test_warning_levels_warn_and_continue(level):
    with pytest.warns(UserWarning, match="do not sum to 1.0|outside"):
        validate_transitions(M.mass_model(), BAD["mass_above_tolerance"], level)


def test_off_skips_the_checks():
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        validate_transitions(M.mass_model(), BAD["mass_above_tolerance"], "off")


def test_a_mass_off_by_more_than_sixteen_epsilons_is_reported():
    # the check is tight by design (1e-12 is far above 16 float64 epsilons)
    with pytest.raises(InvalidRegimeTransitionProbabilitiesError, match="do not sum"):
        validate_transitions(M.mass_model(), M.mass_params(mass=1.0 + 1e-12), "debug")
    validate_transitions(M.mass_model(), M.mass_params(mass=1.0), "debug")


def test_positive_probability_toward_an_inactive_regime_is_reported():
    # the dead regime is terminal and active in every period; a retirement
    # model whose terminal regime is active only at the last age is reached
    # early by a transition that ignores the period
    from pylcm_b200 import AgeGrid, LinSpacedGrid, Model, Regime
    from pylcm_b200.examples import RetirementRegimeId

    w = LinSpacedGrid(start=1, stop=10, n_points=5)
    c = LinSpacedGrid(start=1, stop=10, n_points=5)
    regimes = {
        "working": Regime(actions={"consumption": c}, states={"wealth": w},
                          state_transitions={"wealth": lambda wealth, consumption: wealth - consumption},
                          transition=lambda: RetirementRegimeId.terminal, functions={"utility": lambda consumption: consumption},
                          active=lambda age: age < 2),
        "retired": Regime(actions={"consumption": c}, states={"wealth": w},
                          state_transitions={"wealth": lambda wealth, consumption: wealth - consumption},
                          transition=lambda: RetirementRegimeId.retired, functions={"utility": lambda consumption: consumption},
                          active=lambda age: age < 2),
        "terminal": Regime(transition=None, states={"wealth": w}, functions={"utility": lambda wealth: wealth},
                           active=lambda age: age == 2),
    }
    model = Model(regimes=regimes, ages=AgeGrid(start=0, stop=2, step="Y"), regime_id_class=RetirementRegimeId)
    with pytest.raises(InvalidRegimeTransitionProbabilitiesError, match="inactive"):
        validate_transitions(model, {"discount_factor": 0.9}, "debug")


def test_markov_state_rows_are_checked():
    model = M.value_children_model()
    params = M.value_children_params(p_stay_good=1.2)
    with pytest.raises(InvalidStateTransitionProbabilitiesError, match="outside"):
        validate_transitions(model, params, "debug")


def test_oracle_mass_check_poisons_only_the_malformed_states():
    """mass within 1e-3 of one: divided out (finite); off by more, or a
    negative weight: NaN at exactly the states whose transition is malformed
    (wealth above the threshold), as the reference."""
    model = M.mass_model()
    wealth = np.linspace(1, 50, 30)
    above = wealth > 25.0
    ok, _ = oracle_solve(model, M.mass_params(mass=1.0005))
    ref, _ = oracle_solve(model, M.mass_params(mass=1.0))
    for p in range(model.n_periods - 1):
        v = ok[p]["alive"]
        assert np.isfinite(v).all()
        assert np.allclose(v[~above], ref[p]["alive"][~above], rtol=0, atol=1e-2)
    # mass 1.01 above the threshold: the last decision period (everyone goes
    # to the dead regime) is NaN exactly there; earlier periods too
    Vb, _ = oracle_solve(model, BAD["mass_above_tolerance"])
    last = model.n_periods - 2
    np.testing.assert_array_equal(np.isnan(Vb[last]["alive"]), above)
    assert np.isnan(Vb[0]["alive"][above]).all()
    # a negative survival weight (periods before the last decision period):
    # NaN at every state, although the weights sum to one
    Vn, _ = oracle_solve(model, BAD["negative_probability"])
    assert np.isfinite(Vn[last]["alive"]).all()
    assert np.isnan(Vn[0]["alive"]).all()
