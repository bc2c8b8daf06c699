"""EV1 taste shocks under grid search: the reference's known-answer checks
(`tests/test_taste_shocks.py` of the reference) restated -- the toy model's
solved value against a NumPy logsum recomputation on the same grids, the
smoothed value dominating the hard max, and the rejected declarations."""

import numpy as np
import pytest

from pylcm_b200.exceptions import InvalidParamsError, ModelInitializationError, RegimeInitializationError
from tests import models as M


def _numpy_alive_V(scale: float, discount_factor: float) -> np.ndarray:
    """Qc(w, d) = max over feasible c of log c - kappa d + beta interp(V_done)(w - c + wage d),
    V = scale * logsumexp_d(Qc / scale) (max-shifted)."""
    wealth = np.linspace(1.0, 10.0, 6)
    terminal_wealth = np.linspace(0.0, 12.0, 25)
    consumption = np.linspace(0.5, 5.0, 8)
    v_done = np.log(terminal_wealth + 1.0)
    qc = np.empty((wealth.size, 2))
    for d in (0, 1):
        nw = wealth[:, None] - consumption[None, :] + M.TOY_WAGE * d
        q = np.log(consumption)[None, :] - M.TOY_KAPPA * d + discount_factor * np.interp(nw, terminal_wealth, v_done)
        qc[:, d] = np.max(np.where(consumption[None, :] <= wealth[:, None], q, -np.inf), axis=1)
    m = qc.max(axis=1, keepdims=True)
    return m[:, 0] + scale * np.log(np.sum(np.exp((qc - m) / scale), axis=1))


@pytest.mark.gpu
def test_solved_value_matches_the_numpy_logsum_value():
    model = M.taste_toy_model()
    V = model.solve(params=M.taste_toy_params(scale=0.2, discount_factor=0.95))
    got = np.asarray(V[0]["alive"].cpu() if hasattr(V[0]["alive"], "cpu") else V[0]["alive"])
    np.testing.assert_allclose(got, _numpy_alive_V(0.2, 0.95), rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_smoothed_value_weakly_exceeds_the_hard_max_value():
    model = M.taste_toy_model()
    a = model.solve(params=M.taste_toy_params(scale=0.5))[0]["alive"]
    b = model.solve(params=M.taste_toy_params(scale=1e-8))[0]["alive"]
    a = np.asarray(a.cpu() if hasattr(a, "cpu") else a)
    b = np.asarray(b.cpu() if hasattr(b, "cpu") else b)
    assert np.all(a >= b - 1e-12)


@pytest.mark.parametrize("scale", [0.0, -0.1])
def test_nonpositive_taste_shock_scale_is_rejected(scale):
    from pylcm_b200.engine import SolveEngine

    model = M.taste_toy_model()
    eng = SolveEngine(model, "fp64")
    spec = next(s for s in eng.specs if s.name == "alive")
    with pytest.raises(InvalidParamsError, match="scale"):
        eng.kernels(spec, eng.targets_at(spec, 0), M.taste_toy_params(scale=scale))


def test_taste_shocks_without_a_discrete_action_are_rejected():
    from pylcm_b200 import ExtremeValueTasteShocks, LinSpacedGrid, Regime

    with pytest.raises(ModelInitializationError, match="discrete action"):
        Regime(
            transition=lambda age: 0,
            states={"wealth": LinSpacedGrid(start=1.0, stop=10.0, n_points=6)},
            actions={"consumption": LinSpacedGrid(start=0.5, stop=5.0, n_points=8)},
            functions={"utility": lambda consumption: consumption},
            taste_shocks=ExtremeValueTasteShocks(),
        )
    assert issubclass(RegimeInitializationError, ModelInitializationError)


def test_oracle_matches_the_numpy_logsum_value():
    from oracle.grid_search import solve as oracle_solve

    V, _ = oracle_solve(M.taste_toy_model(), M.taste_toy_params(scale=0.2, discount_factor=0.95))
    np.testing.assert_allclose(V[0]["alive"], _numpy_alive_V(0.2, 0.95), rtol=1e-12, atol=1e-12)
