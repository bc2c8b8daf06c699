"""Model definitions used by the tests and the benchmark.

`regression_model` and `processes_model` restate, in this package's API, the
models behind the reference's stored solutions (reference test models
``tests/test_models/deterministic/regression.py`` and
``tests/test_models/processes.py``); the golden vectors in ``tests/golden``
come from those solutions.  The `config*` builders are the seeded synthetic
workloads of the benchmark (retirement model, stochastic income, 2-state
human-capital model).
"""

from __future__ import annotations

import numpy as np

from pylcm_b200 import (
    AgeGrid,
    DiscreteGrid,
    LinSpacedGrid,
    LogNormalIIDProcess,
    MarkovTransition,
    Model,
    NormalIIDProcess,
    Regime,
    RouwenhorstAR1Process,
    TauchenAR1Process,
    UniformIIDProcess,
    categorical,
)
from pylcm_b200 import jnp


# --------------------------------------------------------------------------
# regression model: work/retire + consumption, deterministic (4 periods)
# --------------------------------------------------------------------------
@categorical(ordered=True)
class LaborSupply:
    work: int
    retire: int


@categorical(ordered=False)
class RegressionRegimeId:
    working_life: int
    dead: int


def _utility_working(consumption, is_working, disutility_of_work):
    return jnp.log(consumption) - jnp.where(is_working, disutility_of_work, 0.0)


def _labor_income(is_working, wage):
    return jnp.where(is_working, wage, 0.0)


def _is_working(labor_supply):
    return labor_supply == LaborSupply.work


def _next_wealth(wealth, consumption, labor_income, interest_rate):
    return (1 + interest_rate) * (wealth - consumption) + labor_income


def _borrowing_constraint(consumption, wealth):
    return consumption <= wealth


def _age_wage(age):
    return 1 + 0.1 * age


def _regression_next_regime(age, final_age_alive):
    return jnp.where(age >= final_age_alive, RegressionRegimeId.dead, RegressionRegimeId.working_life)


def regression_model(n_periods: int = 4, n_wealth: int = 100, n_consumption: int = 500):
    start_age = 18
    final_age_alive = start_age + n_periods - 2
    working = Regime(
        actions={
            "labor_supply": DiscreteGrid(LaborSupply),
            "consumption": LinSpacedGrid(start=1, stop=400, n_points=n_consumption),
        },
        states={"wealth": LinSpacedGrid(start=1, stop=400, n_points=n_wealth)},
        state_transitions={"wealth": _next_wealth},
        constraints={"borrowing_constraint": _borrowing_constraint},
        transition=_regression_next_regime,
        functions={
            "utility": _utility_working,
            "labor_income": _labor_income,
            "is_working": _is_working,
            "wage": _age_wage,
        },
        active=lambda age: age <= final_age_alive,
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(
        regimes={"working_life": working, "dead": dead},
        ages=AgeGrid(start=start_age, stop=final_age_alive + 1, step="Y"),
        regime_id_class=RegressionRegimeId,
    )


def regression_params(n_periods=4, discount_factor=0.95, disutility_of_work=1.0, interest_rate=0.05):
    final_age_alive = 18 + n_periods - 2
    return {
        "discount_factor": discount_factor,
        "working_life": {
            "utility": {"disutility_of_work": disutility_of_work},
            "next_wealth": {"interest_rate": interest_rate},
            "next_regime": {"final_age_alive": final_age_alive},
        },
    }


# --------------------------------------------------------------------------
# processes model: Markov health x income process x wealth
# --------------------------------------------------------------------------
@categorical(ordered=True)
class Health:
    bad: int
    good: int


@categorical(ordered=False)
class AliveDeadId:
    alive: int
    dead: int


def _next_health(health, probs_array):
    return probs_array[health]


def _proc_next_wealth(consumption, wealth):
    return wealth - consumption


def _proc_next_regime(age, final_age_alive):
    return jnp.where(age >= final_age_alive, AliveDeadId.dead, AliveDeadId.alive)


def _proc_wealth_constraint(wealth, income, consumption):
    return wealth - consumption + jnp.exp(income) >= 0


def _proc_utility(wealth, income, health, consumption):
    return jnp.log(consumption) * (1.0 - (1.0 - health) * 0.3)


_PROCESS_CLASSES = {
    "uniform": (UniformIIDProcess, {}),
    "normal": (NormalIIDProcess, {"gauss_hermite": True}),
    "lognormal": (LogNormalIIDProcess, {"gauss_hermite": True}),
    "tauchen": (TauchenAR1Process, {"gauss_hermite": True}),
    "rouwenhorst": (RouwenhorstAR1Process, {}),
}

PROCESS_PARAMS = {
    "uniform": {"start": 0.0, "stop": 1.0},
    "normal": {"mu": 0.0, "sigma": 1.0},
    "lognormal": {"mu": 0.0, "sigma": 1.0},
    "tauchen": {"rho": 0.975, "sigma": 1.0, "mu": 0.0},
    "rouwenhorst": {"rho": 0.975, "sigma": 1.0, "mu": 0.0},
}


def processes_model(n_periods: int, kind: str):
    final_age_alive = n_periods - 2
    cls, kw = _PROCESS_CLASSES[kind]
    alive = Regime(
        active=lambda age, n=final_age_alive: age <= n,
        states={
            "wealth": LinSpacedGrid(start=1, stop=5, n_points=5),
            "income": cls(n_points=5, **kw),
            "health": DiscreteGrid(Health),
        },
        state_transitions={
            "wealth": _proc_next_wealth,
            "health": MarkovTransition(_next_health),
        },
        actions={"consumption": LinSpacedGrid(start=0.1, stop=2, n_points=4)},
        transition=_proc_next_regime,
        constraints={"wealth_constraint": _proc_wealth_constraint},
        functions={"utility": _proc_utility},
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(
        regimes={"alive": alive, "dead": dead},
        regime_id_class=AliveDeadId,
        ages=AgeGrid(start=0, stop=n_periods - 1, step="Y"),
        fixed_params={"final_age_alive": final_age_alive},
    )


def processes_params(kind: str):
    return {
        "alive": {
            "discount_factor": 1.0,
            "next_health": {"probs_array": np.full((2, 2), 0.5)},
            "income": PROCESS_PARAMS[kind],
        },
        "dead": {},
    }


# --------------------------------------------------------------------------
# benchmark workloads (defined in the package's example models)
# --------------------------------------------------------------------------
from pylcm_b200.examples import (  # noqa: E402
    EgmRegimeId,
    GHShock16,
    HCRegimeId,
    RetirementRegimeId,
    dcegm_model,
    dcegm_params,
    hc_model,
    hc_params,
    retirement_model,
    retirement_params,
    stochastic_model,
    stochastic_params,
)


# --------------------------------------------------------------------------
# taste-shock toy model: one decision period (log consumption, binary work
# choice, EV1 taste shocks on it) and a terminal bequest regime; restates the
# reference's `tests/test_models/taste_shocks_toy.py` in this package's API
# --------------------------------------------------------------------------
TOY_KAPPA = 0.3
TOY_WAGE = 2.0


@categorical(ordered=False)
class ToyRegimeId:
    alive: int
    done: int


@categorical(ordered=True)
class WorkChoice:
    off: int
    on: int


def _toy_utility_alive(consumption, work, kappa):
    return jnp.log(consumption) - kappa * work


def _toy_utility_done(wealth):
    return jnp.log(wealth + 1.0)


def _toy_next_wealth(wealth, consumption, work, wage):
    return wealth - consumption + wage * work


def _toy_budget(consumption, wealth):
    return consumption <= wealth


def _toy_next_regime(age):
    return ToyRegimeId.done


def taste_toy_model(taste=True):
    from pylcm_b200 import ExtremeValueTasteShocks

    alive = Regime(
        transition=_toy_next_regime,
        states={"wealth": LinSpacedGrid(start=1.0, stop=10.0, n_points=6)},
        state_transitions={"wealth": _toy_next_wealth},
        actions={"work": DiscreteGrid(WorkChoice), "consumption": LinSpacedGrid(start=0.5, stop=5.0, n_points=8)},
        constraints={"budget_constraint": _toy_budget},
        functions={"utility": _toy_utility_alive},
        taste_shocks=ExtremeValueTasteShocks() if taste else None,
        active=lambda age: age < 41,
    )
    done = Regime(
        transition=None,
        states={"wealth": LinSpacedGrid(start=0.0, stop=12.0, n_points=25)},
        functions={"utility": _toy_utility_done},
    )
    return Model(regimes={"alive": alive, "done": done}, ages=AgeGrid(start=40, stop=41, step="Y"),
                 regime_id_class=ToyRegimeId)


def taste_toy_params(scale, discount_factor=0.95):
    return {
        "discount_factor": discount_factor,
        "alive": {"utility": {"kappa": TOY_KAPPA}, "next_wealth": {"wage": TOY_WAGE}, "taste_shocks": {"scale": scale}},
    }


# --------------------------------------------------------------------------
# pen-and-paper toy model with discrete actions only (deterministic): restates
# the reference's `tests/test_solution_on_toy_model_deterministic.py` model
# --------------------------------------------------------------------------
@categorical(ordered=False)
class ToyConsumption:
    low: int
    high: int


@categorical(ordered=False)
class ToyLabor:
    do_not_work: int
    work: int


@categorical(ordered=False)
class ToyDetRegimeId:
    alive: int
    dead: int


def _det_utility(consumption, labor_supply, wealth, health):
    return jnp.log(1.0 + health * consumption) - 0.5 * labor_supply


def _det_next_wealth(wealth, consumption, labor_supply):
    return wealth - consumption + labor_supply


def _det_next_regime(age, final_age_alive):
    return jnp.where(age >= final_age_alive, ToyDetRegimeId.dead, ToyDetRegimeId.alive)


def _det_borrowing(consumption, wealth):
    return consumption <= wealth


def toy_deterministic_model(n_wealth=100, n_periods=3):
    alive = Regime(
        actions={"consumption": DiscreteGrid(ToyConsumption), "labor_supply": DiscreteGrid(ToyLabor)},
        states={"wealth": LinSpacedGrid(start=0, stop=2, n_points=n_wealth)},
        state_transitions={"wealth": _det_next_wealth},
        functions={"utility": _det_utility},
        constraints={"borrowing_constraint": _det_borrowing},
        transition=_det_next_regime,
        active=lambda age, last=n_periods - 1: age < last,
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0},
                  active=lambda age, last=n_periods - 1: age >= last)
    return Model(regimes={"alive": alive, "dead": dead}, ages=AgeGrid(start=0, stop=n_periods - 1, step="Y"),
                 regime_id_class=ToyDetRegimeId)


def toy_deterministic_params(discount_factor, n_periods=3):
    return {"discount_factor": discount_factor,
            "alive": {"utility": {"health": 1}, "next_regime": {"final_age_alive": n_periods - 2}}}


def toy_deterministic_analytic(wealth, discount_factor):
    """Pen-and-paper value functions of the first and second period: in the
    last decision period consume one unit when wealth allows and do not work;
    in the first, compare working for next period's unit (beta log 2 - 1/2)
    with not working."""
    v1 = np.log(1.0 + np.minimum(1.0, np.floor(wealth)))
    gain = max(0.0, discount_factor * np.log(2.0) - 0.5)
    v0 = np.array([gain, gain + np.log(2.0), (1.0 + discount_factor) * np.log(2.0)])[np.floor(wealth).astype(int)]
    return v0, v1


@categorical(ordered=False)
class ToyHealth:
    bad: int
    good: int


def _sto_next_health(health, probs_array):
    return probs_array[health]


def _sto_utility(consumption, labor_supply, wealth, health):
    return jnp.log(1.0 + health * consumption) - 0.5 * labor_supply


def toy_stochastic_model(n_wealth=100, n_periods=3):
    """The pen-and-paper toy model with a Markov health state (reference
    `tests/test_solution_on_toy_model_stochastic.py`)."""
    alive = Regime(
        actions={"consumption": DiscreteGrid(ToyConsumption), "labor_supply": DiscreteGrid(ToyLabor)},
        states={"wealth": LinSpacedGrid(start=0, stop=2, n_points=n_wealth), "health": DiscreteGrid(ToyHealth)},
        state_transitions={"wealth": _det_next_wealth, "health": MarkovTransition(_sto_next_health)},
        functions={"utility": _sto_utility},
        constraints={"borrowing_constraint": _det_borrowing},
        transition=_det_next_regime,
        active=lambda age, last=n_periods - 1: age < last,
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0},
                  active=lambda age, last=n_periods - 1: age >= last)
    return Model(regimes={"alive": alive, "dead": dead}, ages=AgeGrid(start=0, stop=n_periods - 1, step="Y"),
                 regime_id_class=ToyDetRegimeId)


def toy_stochastic_params(discount_factor, probs_array, n_periods=3):
    return {"discount_factor": discount_factor,
            "alive": {"next_health": {"probs_array": np.asarray(probs_array, dtype=np.float64)},
                      "next_regime": {"final_age_alive": n_periods - 2}}}


def toy_stochastic_analytic(wealth, health, discount_factor, P):
    """Pen-and-paper values and policies of the stochastic toy model at
    (wealth, health) points: in bad health consumption is worthless today,
    so the only value is next period's unit in good health; in good health
    the deterministic solution applies with the discount factor scaled by
    the probability of staying healthy."""
    P = np.asarray(P, dtype=np.float64)
    wealth = np.asarray(wealth, dtype=np.float64)
    health = np.asarray(health).astype(int)
    beta_g = discount_factor * P[1, 1]
    gain_b = discount_factor * P[0, 1] * np.log(2.0)
    v0_bad = np.where(wealth < 1, max(0.0, gain_b - 0.5), gain_b)
    l0_bad = np.where(wealth < 1, int(np.argmax((0.0, gain_b - 0.5))), 0)
    v0_good, _ = toy_deterministic_analytic(wealth, beta_g)
    gain_g = beta_g * np.log(2.0) - 0.5
    idx = np.floor(wealth).astype(int)
    c0_good = np.array([0, 1, 1])[idx]
    l0_good = np.array([int(np.argmax((0.0, gain_g))), int(np.argmax((0.0, gain_g))), 0])[idx]
    v0 = np.where(health == 1, v0_good, v0_bad)
    c0 = np.where(health == 1, c0_good, 0)
    l0 = np.where(health == 1, l0_good, l0_bad)
    return v0, c0, l0


def toy_stochastic_v1(wealth, health):
    return np.log(1.0 + np.minimum(1.0, np.floor(np.asarray(wealth, dtype=np.float64)))) * np.asarray(health)


# --------------------------------------------------------------------------
# brute-force twin of the IJRS retirement model with EV1 taste shocks, whose
# solution the independent `dcegm` package provides (reference cross-check
# fixture `tests/data/dcegm_reference/ijrs_taste_shocks_reference.csv`,
# model documented with the reference's `tests/test_models/dcegm_paper_twin.py`)
# --------------------------------------------------------------------------
IJRS_MIN_AGE = 20
IJRS_N_PERIODS = 10
IJRS_LAST_ALIVE_AGE = IJRS_MIN_AGE + IJRS_N_PERIODS - 2


@categorical(ordered=False)
class IjrsRegimeId:
    working_life: int
    retirement: int
    done_from_working: int
    done_retired: int


@categorical(ordered=True)
class IjrsWork:
    work: int
    retire: int


def ijrs_wealth_points():
    """Geometric below 0.5, 0.05-steps to 5, 0.25-steps to 50: the fixture's
    wealth points (1, 2, 5, 10, 20, 35) are grid nodes."""
    low = tuple(0.001 * (0.5 / 0.001) ** (i / 120) for i in range(120))
    mid = tuple(0.5 + 0.05 * i for i in range(90))
    top = tuple(5.0 + 0.25 * i for i in range(181))
    return low + mid + top


def _ijrs_crra(c, rho):
    return (c ** (1.0 - rho) - 1.0) / (1.0 - rho)


def _ijrs_is_working(work_choice):
    return work_choice == IjrsWork.work


def _ijrs_u_work(consumption, is_working, rho, delta):
    return _ijrs_crra(consumption, rho) - jnp.where(is_working, delta, 0.0)


def _ijrs_u_ret(consumption, rho):
    return _ijrs_crra(consumption, rho)


def _ijrs_u_done_working(wealth, rho, delta, taste_scale):
    # consume everything; the final period's work/retire taste shock smooths
    # the (income-less) choice
    return _ijrs_crra(wealth, rho) + taste_scale * jnp.log(1.0 + jnp.exp(-delta / taste_scale))


def _ijrs_u_done_retired(wealth, rho):
    return _ijrs_crra(wealth, rho)


def _ijrs_labor_income(is_working, age, constant, exp_coeff, exp_squared):
    # earned this period, paid next period at next period's age
    a = age + 1.0
    return jnp.where(is_working, jnp.exp(constant + exp_coeff * a + exp_squared * a ** 2), 0.0)


def _ijrs_next_wealth(wealth, consumption, labor_income, interest_rate, floor):
    return jnp.maximum((1.0 + interest_rate) * (wealth - consumption) + labor_income, floor)


def _ijrs_borrowing(consumption, wealth):
    return consumption <= wealth


def _ijrs_nr_working(work_choice, age):
    last = age >= IJRS_LAST_ALIVE_AGE
    retire = work_choice == IjrsWork.retire
    return jnp.where(last, jnp.where(retire, IjrsRegimeId.done_retired, IjrsRegimeId.done_from_working),
                     jnp.where(retire, IjrsRegimeId.retirement, IjrsRegimeId.working_life))


def _ijrs_nr_retired(age):
    return jnp.where(age >= IJRS_LAST_ALIVE_AGE, IjrsRegimeId.done_retired, IjrsRegimeId.retirement)


def ijrs_brute_model():
    from pylcm_b200 import ExtremeValueTasteShocks, IrregSpacedGrid, LogSpacedGrid

    wealth = IrregSpacedGrid(points=ijrs_wealth_points())
    cons = LogSpacedGrid(start=0.001, stop=50.0, n_points=400)
    alive = lambda age: age <= IJRS_LAST_ALIVE_AGE  # noqa: E731
    working = Regime(
        transition=_ijrs_nr_working, states={"wealth": wealth},
        actions={"work_choice": DiscreteGrid(IjrsWork), "consumption": cons},
        taste_shocks=ExtremeValueTasteShocks(), active=alive,
        state_transitions={"wealth": _ijrs_next_wealth}, constraints={"borrowing_constraint": _ijrs_borrowing},
        functions={"utility": _ijrs_u_work, "is_working": _ijrs_is_working, "labor_income": _ijrs_labor_income},
    )
    retired = Regime(
        transition=_ijrs_nr_retired, states={"wealth": wealth}, actions={"consumption": cons}, active=alive,
        state_transitions={"wealth": _ijrs_next_wealth}, constraints={"borrowing_constraint": _ijrs_borrowing},
        functions={"utility": _ijrs_u_ret},
    )
    done_w = Regime(transition=None, states={"wealth": wealth}, functions={"utility": _ijrs_u_done_working})
    done_r = Regime(transition=None, states={"wealth": wealth}, functions={"utility": _ijrs_u_done_retired})
    return Model(regimes={"working_life": working, "retirement": retired, "done_from_working": done_w,
                          "done_retired": done_r},
                 ages=AgeGrid(start=IJRS_MIN_AGE, stop=IJRS_MIN_AGE + IJRS_N_PERIODS - 1, step="Y"),
                 regime_id_class=IjrsRegimeId)


def ijrs_params(taste_scale=0.2):
    return {
        "discount_factor": 0.95, "interest_rate": 0.05, "rho": 1.95, "delta": 0.35, "constant": 0.75,
        "exp_coeff": 0.04, "exp_squared": -0.0002, "floor": 0.001,
        "done_from_working": {"utility": {"taste_scale": taste_scale}},
        "working_life": {"taste_shocks": {"scale": taste_scale}},
        "retirement": {"next_wealth": {"labor_income": 0.0}},
    }


def _ijrs_savings(wealth, consumption):
    return wealth - consumption


def _ijrs_next_wealth_from_savings(savings, labor_income, interest_rate, floor):
    return jnp.maximum((1.0 + interest_rate) * savings + labor_income, floor)


def _ijrs_inverse_mu(marginal_continuation, rho):
    return marginal_continuation ** (-1.0 / rho)


def ijrs_dcegm_model(savings_points=None):
    """The DC-EGM twin: the same model with both living regimes solved by
    DC-EGM on the fixture run's savings grid (uniform, 500 points on
    [0, 50]) unless `savings_points` is given; the terminal regimes carry
    their utility and its wealth gradient."""
    from pylcm_b200 import (
        ConsumptionSavingsRegime, ExtremeValueTasteShocks, IrregSpacedGrid, LinSpacedGrid, LiquidMargin,
        LogSpacedGrid,
    )
    from pylcm_b200.solvers import DCEGM

    sav = LinSpacedGrid(start=0.0, stop=50.0, n_points=500) if savings_points is None else \
        IrregSpacedGrid(points=tuple(savings_points))
    solver = DCEGM(savings_grid=sav)
    margin = LiquidMargin(state="wealth", action="consumption", resources="wealth", post_decision_state="savings")
    wealth = IrregSpacedGrid(points=ijrs_wealth_points())
    cons = LogSpacedGrid(start=0.001, stop=50.0, n_points=400)
    alive = lambda age: age <= IJRS_LAST_ALIVE_AGE  # noqa: E731
    working = ConsumptionSavingsRegime(
        transition=_ijrs_nr_working, states={"wealth": wealth},
        actions={"work_choice": DiscreteGrid(IjrsWork), "consumption": cons},
        taste_shocks=ExtremeValueTasteShocks(), active=alive,
        state_transitions={"wealth": _ijrs_next_wealth_from_savings},
        functions={"utility": _ijrs_u_work, "is_working": _ijrs_is_working, "labor_income": _ijrs_labor_income,
                   "savings": _ijrs_savings, "inverse_marginal_utility": _ijrs_inverse_mu},
        solver=solver, liquid=margin,
    )
    retired = ConsumptionSavingsRegime(
        transition=_ijrs_nr_retired, states={"wealth": wealth}, actions={"consumption": cons}, active=alive,
        state_transitions={"wealth": _ijrs_next_wealth_from_savings},
        functions={"utility": _ijrs_u_ret, "savings": _ijrs_savings, "inverse_marginal_utility": _ijrs_inverse_mu},
        solver=solver, liquid=margin,
    )
    done_w = Regime(transition=None, states={"wealth": wealth}, functions={"utility": _ijrs_u_done_working})
    done_r = Regime(transition=None, states={"wealth": wealth}, functions={"utility": _ijrs_u_done_retired})
    return Model(regimes={"working_life": working, "retirement": retired, "done_from_working": done_w,
                          "done_retired": done_r},
                 ages=AgeGrid(start=IJRS_MIN_AGE, stop=IJRS_MIN_AGE + IJRS_N_PERIODS - 1, step="Y"),
                 regime_id_class=IjrsRegimeId)


# --------------------------------------------------------------------------
# DC-EGM into value arrays: a DC-EGM regime with a Markov health state whose
# targets are a grid-search regime (wealth x health) and a terminal regime
# (bequest over wealth x health); both are read as carried value arrays, the
# Markov health law folded into their rows.  The grids start at zero wealth,
# where nothing is affordable (-inf values at the first node).
# --------------------------------------------------------------------------
@categorical(ordered=False)
class VcRegimeId:
    working: int
    retired: int
    done: int


VC_N_PERIODS = 6


def _vc_crra(c, rho):
    return (c ** (1.0 - rho) - 1.0) / (1.0 - rho)


def _vc_u_work(consumption, work_choice, health, rho, disutility):
    return _vc_crra(consumption, rho) - jnp.where(work_choice == IjrsWork.work, disutility, 0.0) \
        - 0.2 * (health == Health.bad)


def _vc_u_ret(consumption, health, rho):
    return _vc_crra(consumption, rho) - 0.2 * (health == Health.bad)


def _vc_u_done(wealth, health, rho, weight):
    return weight * (1.0 + 0.5 * (health == Health.good)) * _vc_crra(wealth + 1.0, rho)


def _vc_savings(wealth, consumption):
    return wealth - consumption


def _vc_next_wealth_work(savings, work_choice, health, interest_rate, wage):
    earn = jnp.where(work_choice == IjrsWork.work, wage * (0.6 + 0.4 * (health == Health.good)), 0.0)
    return (1.0 + interest_rate) * savings + earn


def _vc_next_wealth_ret(wealth, consumption, interest_rate):
    return (1.0 + interest_rate) * (wealth - consumption)


def _vc_next_health(health, p_stay_good, p_recover):
    good = health == Health.good
    p_good = jnp.where(good, p_stay_good, p_recover)
    return jnp.array([1.0 - p_good, p_good])


def _vc_inverse_mu(marginal_continuation, rho):
    return marginal_continuation ** (-1.0 / rho)


def _vc_budget(consumption, wealth):
    return consumption <= wealth


def _vc_nr_working(work_choice, age):
    return jnp.where(age >= VC_N_PERIODS - 2, VcRegimeId.done,
                     jnp.where(work_choice == IjrsWork.retire, VcRegimeId.retired, VcRegimeId.working))


def _vc_nr_retired(age):
    return jnp.where(age >= VC_N_PERIODS - 2, VcRegimeId.done, VcRegimeId.retired)


def value_children_model(taste=False, n_wealth=60, n_savings=80):
    from pylcm_b200 import ConsumptionSavingsRegime, ExtremeValueTasteShocks, LiquidMargin
    from pylcm_b200.solvers import DCEGM

    wealth = LinSpacedGrid(start=0.0, stop=40.0, n_points=n_wealth)
    cons = LinSpacedGrid(start=0.05, stop=40.0, n_points=120)
    health = DiscreteGrid(Health)
    alive = lambda age: age <= VC_N_PERIODS - 2  # noqa: E731
    working = ConsumptionSavingsRegime(
        transition=_vc_nr_working, states={"health": health, "wealth": wealth},
        actions={"work_choice": DiscreteGrid(IjrsWork), "consumption": cons},
        taste_shocks=ExtremeValueTasteShocks() if taste else None, active=alive,
        state_transitions={"wealth": _vc_next_wealth_work, "health": MarkovTransition(_vc_next_health)},
        functions={"utility": _vc_u_work, "savings": _vc_savings, "inverse_marginal_utility": _vc_inverse_mu},
        solver=DCEGM(savings_grid=LinSpacedGrid(start=0.0, stop=40.0, n_points=n_savings)),
        liquid=LiquidMargin(state="wealth", action="consumption", resources="wealth", post_decision_state="savings"),
    )
    retired = Regime(
        transition=_vc_nr_retired, states={"wealth": wealth, "health": health}, actions={"consumption": cons},
        active=alive, state_transitions={"wealth": _vc_next_wealth_ret, "health": MarkovTransition(_vc_next_health)},
        constraints={"budget": _vc_budget}, functions={"utility": _vc_u_ret},
    )
    done = Regime(transition=None, states={"wealth": wealth, "health": health}, functions={"utility": _vc_u_done})
    return Model(regimes={"working": working, "retired": retired, "done": done},
                 ages=AgeGrid(start=0, stop=VC_N_PERIODS - 1, step="Y"), regime_id_class=VcRegimeId)


def value_children_params(taste_scale=None, p_stay_good=0.9):
    p = {"discount_factor": 0.95, "rho": 2.0, "disutility": 0.3, "interest_rate": 0.04, "wage": 3.0,
         "p_stay_good": p_stay_good, "p_recover": 0.4, "weight": 2.0}
    if taste_scale is not None:
        p["working"] = {"taste_shocks": {"scale": taste_scale}}
    return p


# --------------------------------------------------------------------------
# DC-EGM with an AR(1) income process (Tauchen): the DC-EGM regime's rows
# include the process state; its targets are itself and a grid-search
# regime over (wealth, income), the process law's transition-matrix row
# folded into the carried value array.
# --------------------------------------------------------------------------
@categorical(ordered=False)
class EpRegimeId:
    working: int
    retired: int
    dead: int


EP_N_PERIODS = 6


def _ep_u_work(consumption, work_choice, rho, disutility):
    return _vc_crra(consumption, rho) - jnp.where(work_choice == IjrsWork.work, disutility, 0.0)


def _ep_u_ret(consumption, rho):
    return _vc_crra(consumption, rho)


def _ep_next_wealth_work(savings, work_choice, income, interest_rate, wage):
    return (1.0 + interest_rate) * savings + jnp.where(work_choice == IjrsWork.work, wage * jnp.exp(income), 0.0)


def _ep_next_wealth_ret(wealth, consumption, interest_rate, pension):
    return (1.0 + interest_rate) * (wealth - consumption) + pension


def _ep_nr_working(work_choice, age):
    return jnp.where(age >= EP_N_PERIODS - 2, EpRegimeId.dead,
                     jnp.where(work_choice == IjrsWork.retire, EpRegimeId.retired, EpRegimeId.working))


def _ep_nr_retired(age):
    return jnp.where(age >= EP_N_PERIODS - 2, EpRegimeId.dead, EpRegimeId.retired)


def egm_process_model(taste=False, n_wealth=50, n_savings=60):
    from pylcm_b200 import ConsumptionSavingsRegime, ExtremeValueTasteShocks, LiquidMargin
    from pylcm_b200.solvers import DCEGM

    wealth = LinSpacedGrid(start=0.0, stop=40.0, n_points=n_wealth)
    cons = LinSpacedGrid(start=0.05, stop=40.0, n_points=100)
    income = TauchenAR1Process(n_points=5, gauss_hermite=False, n_std=2.0)
    alive = lambda age: age <= EP_N_PERIODS - 2  # noqa: E731
    working = ConsumptionSavingsRegime(
        transition=_ep_nr_working, states={"wealth": wealth, "income": income},
        actions={"work_choice": DiscreteGrid(IjrsWork), "consumption": cons},
        taste_shocks=ExtremeValueTasteShocks() if taste else None, active=alive,
        state_transitions={"wealth": _ep_next_wealth_work},
        functions={"utility": _ep_u_work, "savings": _vc_savings, "inverse_marginal_utility": _vc_inverse_mu},
        solver=DCEGM(savings_grid=LinSpacedGrid(start=0.0, stop=40.0, n_points=n_savings)),
        liquid=LiquidMargin(state="wealth", action="consumption", resources="wealth", post_decision_state="savings"),
    )
    retired = Regime(
        transition=_ep_nr_retired, states={"wealth": wealth, "income": income}, actions={"consumption": cons},
        active=alive, state_transitions={"wealth": _ep_next_wealth_ret},
        constraints={"budget": _vc_budget}, functions={"utility": _ep_u_ret},
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(regimes={"working": working, "retired": retired, "dead": dead},
                 ages=AgeGrid(start=0, stop=EP_N_PERIODS - 1, step="Y"), regime_id_class=EpRegimeId)


def egm_process_params(taste_scale=None, rho=0.9):
    p = {"discount_factor": 0.95, "rho": 2.0, "disutility": 0.4, "interest_rate": 0.04, "wage": 2.0,
         "pension": 0.5, "income": {"rho": rho, "sigma": 0.2, "mu": 0.0}}
    if taste_scale is not None:
        p["working"] = {"taste_shocks": {"scale": taste_scale}}
    return p


# --------------------------------------------------------------------------
# normal-mixture processes: an AR(1) income with mixture innovations, or an
# IID mixture income, as the process state of a grid-search regime
# --------------------------------------------------------------------------
MIX_N_PERIODS = 5


def _mix_u(consumption, rho):
    return (consumption ** (1.0 - rho) - 1.0) / (1.0 - rho)


def _mix_next_wealth(wealth, consumption, income, interest_rate):
    return (1.0 + interest_rate) * (wealth - consumption) + jnp.exp(income)


def _mix_budget(consumption, wealth):
    return consumption <= wealth


def _mix_nr(age):
    return jnp.where(age >= MIX_N_PERIODS - 2, AliveDeadId.dead, AliveDeadId.alive)


def _mix_next_wealth_two(wealth, consumption, income, shock, interest_rate):
    return (1.0 + interest_rate) * (wealth - consumption) + jnp.exp(income) + 0.1 * shock


def mixture_model(kind="ar1", n_wealth=40, n_cons=60):
    """kind "ar1" / "iid": one mixture income process; "two": the AR(1)
    mixture income and an IID normal shock (two process states)."""
    from pylcm_b200 import NormalMixtureIIDProcess, TauchenNormalMixtureAR1Process

    proc = NormalMixtureIIDProcess(n_points=4) if kind == "iid" else TauchenNormalMixtureAR1Process(n_points=5)
    states = {"wealth": LinSpacedGrid(start=0.5, stop=20.0, n_points=n_wealth), "income": proc}
    if kind == "two":
        states["shock"] = NormalIIDProcess(n_points=3, gauss_hermite=False)
    alive = Regime(
        active=lambda age: age <= MIX_N_PERIODS - 2,
        states=states,
        state_transitions={"wealth": _mix_next_wealth_two if kind == "two" else _mix_next_wealth},
        actions={"consumption": LinSpacedGrid(start=0.1, stop=20.0, n_points=n_cons)},
        transition=_mix_nr, constraints={"budget": _mix_budget}, functions={"utility": _mix_u},
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(regimes={"alive": alive, "dead": dead}, regime_id_class=AliveDeadId,
                 ages=AgeGrid(start=0, stop=MIX_N_PERIODS - 1, step="Y"))


def mixture_params(kind="ar1", p1=0.8):
    if kind == "iid":
        inc = {"n_std": 2.0, "p1": p1, "mu1": -0.3, "sigma1": 0.1, "mu2": 0.3, "sigma2": 0.2}
    else:
        inc = {"rho": 0.8, "mu": 0.0, "n_std": 2.5, "p1": p1, "mu1": 0.05, "sigma1": 0.1, "mu2": -0.2, "sigma2": 0.3}
    out = {"discount_factor": 0.95, "rho": 2.0, "interest_rate": 0.03, "income": inc}
    if kind == "two":
        out["shock"] = {"mu": 0.0, "sigma": 1.0, "n_std": 2.0}
    return out


# --------------------------------------------------------------------------
# wealth grids of every continuous kind (irregular, log-spaced, piecewise
# linear, piecewise log) with an affine next-wealth law that leaves the grid
# at the top (extrapolation) and a Markov health state
# --------------------------------------------------------------------------
GK_N_PERIODS = 5


def _gk_u(consumption, health):
    return jnp.log(consumption) - 0.1 * (health == Health.bad)


def _gk_next_wealth(wealth, consumption, health, interest_rate, income):
    return (1.0 + interest_rate) * (wealth - consumption) + income * jnp.where(health == Health.good, 1.0, 0.5)


def _gk_next_health(health):
    p_good = jnp.where(health == Health.good, 0.9, 0.4)
    return jnp.array([1.0 - p_good, p_good])


def _gk_budget(consumption, wealth):
    return consumption <= wealth


def _gk_nr(age):
    return jnp.where(age >= GK_N_PERIODS - 2, AliveDeadId.dead, AliveDeadId.alive)


def grid_kinds_model(kind):
    from pylcm_b200 import (
        IrregSpacedGrid, LogSpacedGrid, PiecewiseGridSegment, PiecewiseLinSpacedGrid, PiecewiseLogSpacedGrid,
    )

    cons = LinSpacedGrid(start=0.5, stop=60.0, n_points=80)
    if kind == "irreg":
        wealth = IrregSpacedGrid(points=tuple(1.0 + 59.0 * (i / 39) ** 2 for i in range(40)))
    elif kind == "log":
        wealth = LogSpacedGrid(start=1.0, stop=60.0, n_points=40)
    elif kind == "piece_lin":
        wealth = PiecewiseLinSpacedGrid(segments=(PiecewiseGridSegment("[1, 10)", 20),
                                                  PiecewiseGridSegment("[10, 60]", 20)))
        cons = PiecewiseLinSpacedGrid(segments=(PiecewiseGridSegment("[0.5, 5]", 40),
                                                PiecewiseGridSegment("(5, 60]", 40)))
    else:
        wealth = PiecewiseLogSpacedGrid(segments=(PiecewiseGridSegment("[1, 10]", 15),
                                                  PiecewiseGridSegment("(10, 60]", 25)))
    alive = Regime(
        active=lambda age: age <= GK_N_PERIODS - 2,
        states={"health": DiscreteGrid(Health), "wealth": wealth},
        state_transitions={"wealth": _gk_next_wealth, "health": MarkovTransition(_gk_next_health)},
        actions={"consumption": cons},
        transition=_gk_nr, constraints={"budget": _gk_budget}, functions={"utility": _gk_u},
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(regimes={"alive": alive, "dead": dead}, regime_id_class=AliveDeadId,
                 ages=AgeGrid(start=0, stop=GK_N_PERIODS - 1, step="Y"))


def grid_kinds_params():
    return {"discount_factor": 0.95, "interest_rate": 0.04, "income": 8.0}


# --------------------------------------------------------------------------
# mortality model (restating the reference's lcm_examples/mortality.py):
# working life, retirement and death, 10-year periods from age 40,
# survival probabilities indexed by period in Markov regime transitions
# --------------------------------------------------------------------------
@categorical(ordered=False)
class MortalityRegimeId:
    working_life: int
    retirement: int
    dead: int


MORTALITY_LAST_AGE = 70


def _mo_u_work(consumption, is_working, disutility_of_work):
    return jnp.log(consumption) - jnp.where(is_working, disutility_of_work, 0.0)


def _mo_u_ret(consumption):
    return jnp.log(consumption)


def _mo_income(is_working, wage):
    return jnp.where(is_working, wage, 0.0)


def _mo_is_working(labor_supply):
    return labor_supply == LaborSupply.work


def _mo_next_wealth(wealth, consumption, labor_income, interest_rate):
    return (1 + interest_rate) * (wealth - consumption) + labor_income


def _mo_nr_working(labor_supply, period, survival_probs):
    sp = survival_probs[period]
    retire = labor_supply == LaborSupply.retire
    return jnp.array([jnp.where(retire, 0.0, sp), jnp.where(retire, sp, 0.0), 1 - sp])


def _mo_nr_retired(period, survival_probs):
    sp = survival_probs[period]
    return jnp.array([0.0, sp, 1 - sp])


def _mo_budget(consumption, wealth):
    return consumption <= wealth


def mortality_model():
    wealth = LinSpacedGrid(start=1, stop=400, n_points=100)
    cons = LinSpacedGrid(start=1, stop=400, n_points=500)
    alive = lambda age: age < MORTALITY_LAST_AGE  # noqa: E731
    working = Regime(
        actions={"labor_supply": DiscreteGrid(LaborSupply), "consumption": cons},
        states={"wealth": wealth}, state_transitions={"wealth": _mo_next_wealth},
        constraints={"borrowing_constraint": _mo_budget}, transition=MarkovTransition(_mo_nr_working),
        functions={"utility": _mo_u_work, "labor_income": _mo_income, "is_working": _mo_is_working}, active=alive,
    )
    retired = Regime(
        transition=MarkovTransition(_mo_nr_retired), actions={"consumption": cons}, states={"wealth": wealth},
        state_transitions={"wealth": _mo_next_wealth}, constraints={"borrowing_constraint": _mo_budget},
        functions={"utility": _mo_u_ret}, active=alive,
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(regimes={"working_life": working, "retirement": retired, "dead": dead},
                 ages=AgeGrid(start=40, stop=MORTALITY_LAST_AGE, step="10Y"), regime_id_class=MortalityRegimeId)


def mortality_params():
    """The reference's defaults for 4 periods: survival 0.98, 0.82, then 0."""
    return {
        "discount_factor": 0.95, "interest_rate": 0.05, "survival_probs": np.array([0.98, 0.82, 0.0]),
        "working_life": {"utility": {"disutility_of_work": 0.5}, "labor_income": {"wage": 10.0}},
        "retirement": {"next_wealth": {"labor_income": 0.0}},
    }


# --------------------------------------------------------------------------
# regime-transition mass: survival probabilities scaled by a `mass` factor,
# for the continuation's mass check (the reference's
# ``Q_and_F.py:1401-1432``: CE / mass where |mass - 1| <= 1e-3 and no weight
# is negative, NaN otherwise) and the transition validation
# --------------------------------------------------------------------------
@categorical(ordered=False)
class MassRegimeId:
    alive: int
    dead: int


def _mass_u(consumption):
    return jnp.log(consumption)


def _mass_next_wealth(wealth, consumption, interest_rate):
    return (1 + interest_rate) * (wealth - consumption) + 5.0


def _mass_budget(consumption, wealth):
    return consumption <= wealth


def _mass_nr(wealth, period, p_survive, mass, threshold, last_alive_period):
    # nobody survives into the last period (the alive regime is inactive
    # there); the distortion applies only above `threshold` wealth, so part
    # of the state grid keeps a proper distribution
    p = jnp.where(period < last_alive_period, p_survive, 0.0)
    m = jnp.where(wealth > threshold, mass, 1.0)
    return jnp.array([p * m, (1.0 - p) * m])


def mass_model(n_periods: int = 4, n_wealth: int = 30, n_cons: int = 40):
    wealth = LinSpacedGrid(start=1, stop=50, n_points=n_wealth)
    cons = LinSpacedGrid(start=1, stop=50, n_points=n_cons)
    last = n_periods - 1
    alive = Regime(
        actions={"consumption": cons}, states={"wealth": wealth},
        state_transitions={"wealth": _mass_next_wealth}, constraints={"borrowing_constraint": _mass_budget},
        transition=MarkovTransition(_mass_nr), functions={"utility": _mass_u},
        active=lambda age, last=last: age < last,
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(regimes={"alive": alive, "dead": dead}, ages=AgeGrid(start=0, stop=last, step="Y"),
                 regime_id_class=MassRegimeId, fixed_params={"last_alive_period": last - 1})


def mass_params(mass=1.0, p_survive=0.9, threshold=25.0):
    return {"discount_factor": 0.95, "interest_rate": 0.03, "p_survive": p_survive, "mass": mass,
            "threshold": threshold}
