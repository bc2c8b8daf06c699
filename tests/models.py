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
# benchmark workloads
# --------------------------------------------------------------------------
@categorical(ordered=False)
class RetirementRegimeId:
    working: int
    retired: int
    terminal: int


def _ret_utility_working(consumption, labor_supply):
    return jnp.log(consumption) - 0.5 * (labor_supply == LaborSupply.work)


def _ret_utility_retired(consumption):
    return jnp.log(consumption)


def _ret_next_wealth_working(wealth, consumption, labor_supply):
    return 1.05 * (wealth - consumption) + 20.0 * (labor_supply == LaborSupply.work)


def _ret_next_wealth_retired(wealth, consumption):
    return 1.05 * (wealth - consumption)


def _ret_next_regime_working(labor_supply, period, last_decision_period):
    return jnp.where(
        period >= last_decision_period,
        RetirementRegimeId.terminal,
        jnp.where(labor_supply == LaborSupply.work, RetirementRegimeId.working, RetirementRegimeId.retired),
    )


def _ret_next_regime_retired(period, last_decision_period):
    return jnp.where(period >= last_decision_period, RetirementRegimeId.terminal, RetirementRegimeId.retired)


def retirement_model(n_periods: int = 5, n_wealth: int = 100, n_consumption: int = 100):
    """Deterministic retirement model: wealth linspace(1,400,n), work/retire
    (absorbing), u = log c - 0.5 work, w' = 1.05 (w - c) + 20 work, c <= w,
    terminal V_T = max_{c<=w} log c."""
    wealth = LinSpacedGrid(start=1, stop=400, n_points=n_wealth)
    cons = LinSpacedGrid(start=1, stop=400, n_points=n_consumption)
    last = n_periods - 1
    working = Regime(
        actions={"labor_supply": DiscreteGrid(LaborSupply), "consumption": cons},
        states={"wealth": wealth},
        state_transitions={"wealth": _ret_next_wealth_working},
        constraints={"borrowing_constraint": _borrowing_constraint},
        transition=_ret_next_regime_working,
        functions={"utility": _ret_utility_working},
        active=lambda age, last=last: age < last,
    )
    retired = Regime(
        actions={"consumption": cons},
        states={"wealth": wealth},
        state_transitions={"wealth": _ret_next_wealth_retired},
        constraints={"borrowing_constraint": _borrowing_constraint},
        transition=_ret_next_regime_retired,
        functions={"utility": _ret_utility_retired},
        active=lambda age, last=last: age < last,
    )
    terminal = Regime(
        transition=None,
        actions={"consumption": cons},
        states={"wealth": wealth},
        constraints={"borrowing_constraint": _borrowing_constraint},
        functions={"utility": _ret_utility_retired},
        active=lambda age, last=last: age == last,
    )
    return Model(
        regimes={"working": working, "retired": retired, "terminal": terminal},
        ages=AgeGrid(start=0, stop=last, step="Y"),
        regime_id_class=RetirementRegimeId,
        fixed_params={"last_decision_period": n_periods - 2},
    )


def retirement_params(beta: float = 0.95):
    return {"discount_factor": beta}


# stochastic income version (CRRA, Tauchen log income multiplying the wage)
def _crra(consumption, crra):
    return consumption ** (1.0 - crra) / (1.0 - crra)


def _sto_utility_working(consumption, labor_supply, crra):
    return _crra(consumption, crra) - 0.5 * (labor_supply == LaborSupply.work)


def _sto_utility_retired(consumption, crra):
    return _crra(consumption, crra)


def _sto_next_wealth_working(wealth, consumption, labor_supply, income, interest_rate, wage):
    return (1 + interest_rate) * (wealth - consumption) + wage * jnp.exp(income) * (
        labor_supply == LaborSupply.work
    )


def _sto_next_wealth_retired(wealth, consumption, interest_rate):
    return (1 + interest_rate) * (wealth - consumption)


def stochastic_model(n_periods: int = 40, n_wealth: int = 500, n_consumption: int = 500, n_income: int = 7):
    """Stochastic retirement model: 7-node Tauchen AR(1) log income
    (rho=0.9, sigma=0.1, +-3 sd) multiplying the wage, CRRA utility."""
    wealth = LinSpacedGrid(start=1, stop=400, n_points=n_wealth)
    cons = LinSpacedGrid(start=1, stop=400, n_points=n_consumption)
    income = TauchenAR1Process(n_points=n_income, gauss_hermite=False, rho=0.9, sigma=0.1, mu=0.0, n_std=3)
    last = n_periods - 1
    working = Regime(
        actions={"labor_supply": DiscreteGrid(LaborSupply), "consumption": cons},
        states={"wealth": wealth, "income": income},
        state_transitions={"wealth": _sto_next_wealth_working},
        constraints={"borrowing_constraint": _borrowing_constraint},
        transition=_ret_next_regime_working,
        functions={"utility": _sto_utility_working},
        active=lambda age, last=last: age < last,
    )
    retired = Regime(
        actions={"consumption": cons},
        states={"wealth": wealth, "income": income},
        state_transitions={"wealth": _sto_next_wealth_retired},
        constraints={"borrowing_constraint": _borrowing_constraint},
        transition=_ret_next_regime_retired,
        functions={"utility": _sto_utility_retired},
        active=lambda age, last=last: age < last,
    )
    terminal = Regime(
        transition=None,
        actions={"consumption": cons},
        states={"wealth": wealth, "income": income},
        constraints={"borrowing_constraint": _borrowing_constraint},
        functions={"utility": _sto_utility_retired},
        active=lambda age, last=last: age == last,
    )
    return Model(
        regimes={"working": working, "retired": retired, "terminal": terminal},
        ages=AgeGrid(start=0, stop=last, step="Y"),
        regime_id_class=RetirementRegimeId,
        fixed_params={"last_decision_period": n_periods - 2},
    )


def stochastic_params(beta=0.96, crra=2.0, interest_rate=0.04, wage=20.0):
    return {"discount_factor": beta, "crra": crra, "interest_rate": interest_rate, "wage": wage}


# 2-continuous-state human-capital model with a 32-state Markov shock
@categorical(ordered=False)
class HCRegimeId:
    alive: int
    terminal: int


def _hc_utility(consumption, hours, crra):
    return consumption ** (1.0 - crra) / (1.0 - crra) - 0.5 * hours


def _hc_next_wealth(wealth, consumption, hours, human_capital, shock, interest_rate, shock_levels):
    return (1 + interest_rate) * (wealth - consumption) + jnp.exp(shock_levels[shock]) * human_capital * hours


def _hc_next_hc(human_capital, hours):
    return 0.95 * human_capital + 0.1 * hours


def _hc_next_shock(shock, shock_transition):
    return shock_transition[shock]


def _hc_next_regime(period, last_decision_period):
    return jnp.where(period >= last_decision_period, HCRegimeId.terminal, HCRegimeId.alive)


def _make_shock_class(n):
    ns = {"__annotations__": {f"s{i}": int for i in range(n)}}
    return categorical(ordered=False)(type(f"Shock{n}", (), ns))


def hc_model(n_periods=60, n_wealth=1000, n_hc=50, n_shock=32, n_consumption=300):
    """Wealth linspace(0,1000), human capital linspace(1,5), Markov shock,
    consumption linspace(1,1000,300), hours {0,0.5,1}, h' = 0.95h + 0.1 hours,
    income exp(z) h hours, u = c^(1-rho)/(1-rho) - 0.5 hours."""
    Shock = _make_shock_class(n_shock)
    wealth = LinSpacedGrid(start=0, stop=1000, n_points=n_wealth)
    hc = LinSpacedGrid(start=1, stop=5, n_points=n_hc)
    cons = LinSpacedGrid(start=1, stop=1000, n_points=n_consumption)
    hours = LinSpacedGrid(start=0, stop=1, n_points=3)
    last = n_periods - 1
    alive = Regime(
        actions={"consumption": cons, "hours": hours},
        states={"shock": DiscreteGrid(Shock), "wealth": wealth, "human_capital": hc},
        state_transitions={
            "wealth": _hc_next_wealth,
            "human_capital": _hc_next_hc,
            "shock": MarkovTransition(_hc_next_shock),
        },
        constraints={"borrowing_constraint": _borrowing_constraint},
        transition=_hc_next_regime,
        functions={"utility": _hc_utility},
        active=lambda age, last=last: age < last,
    )
    terminal = Regime(
        transition=None,
        actions={"consumption": cons},
        states={"shock": DiscreteGrid(Shock), "wealth": wealth, "human_capital": hc},
        constraints={"borrowing_constraint": _borrowing_constraint},
        functions={"utility": lambda consumption, crra: consumption ** (1.0 - crra) / (1.0 - crra)},
        active=lambda age, last=last: age == last,
    )
    return Model(
        regimes={"alive": alive, "terminal": terminal},
        ages=AgeGrid(start=0, stop=last, step="Y"),
        regime_id_class=HCRegimeId,
        fixed_params={"last_decision_period": n_periods - 2},
    )


def hc_params(seed=0, n_shock=32, beta=None, crra=None, interest_rate=None):
    rng = np.random.default_rng(seed)
    P = rng.dirichlet(np.ones(n_shock), size=n_shock)
    levels = np.linspace(-0.5, 0.5, n_shock)
    return {
        "discount_factor": float(rng.uniform(0.90, 0.99)) if beta is None else beta,
        "crra": float(rng.uniform(1.0, 5.0)) if crra is None else crra,
        "interest_rate": float(rng.uniform(0.01, 0.06)) if interest_rate is None else interest_rate,
        "shock_transition": P,
        "shock_levels": levels,
    }


# --------------------------------------------------------------------------
# DC-EGM retirement model with income shocks (CRRA, 16-node Gauss-Hermite
# lognormal income weights carried by a discrete iid shock state, optional EV1
# taste shocks on the work/retire choice)
@categorical(ordered=False)
class EgmRegimeId:
    working: int
    retired: int
    dead: int


def _make_shock16():
    ns = {"__annotations__": {f"n{i}": int for i in range(16)}}
    return categorical(ordered=False)(type("GHShock16", (), ns))


GHShock16 = _make_shock16()


def _egm_savings(wealth, consumption):
    return wealth - consumption


def _egm_u_work(consumption, labor_supply, crra, disutility_of_work):
    return consumption ** (1.0 - crra) / (1.0 - crra) - disutility_of_work * (labor_supply == LaborSupply.work)


def _egm_u_ret(consumption, crra):
    return consumption ** (1.0 - crra) / (1.0 - crra)


def _egm_inv_mu(marginal_continuation, crra):
    return marginal_continuation ** (-1.0 / crra)


def _egm_next_wealth_work(savings, labor_supply, shock, interest_rate, wage, shock_values):
    return (1 + interest_rate) * savings + wage * shock_values[shock] * (labor_supply == LaborSupply.work)


def _egm_next_wealth_ret(savings, interest_rate):
    return (1 + interest_rate) * savings


def _egm_next_shock(shock, shock_weights):
    return shock_weights[shock]


def _egm_nr_work(labor_supply, period, last_decision_period):
    return jnp.where(
        period >= last_decision_period,
        EgmRegimeId.dead,
        jnp.where(labor_supply == LaborSupply.work, EgmRegimeId.working, EgmRegimeId.retired),
    )


def _egm_nr_ret(period, last_decision_period):
    return jnp.where(period >= last_decision_period, EgmRegimeId.dead, EgmRegimeId.retired)


def dcegm_model(n_periods=40, n_savings=2000, n_wealth=2000, taste=False, n_constrained=20):
    """Savings grid 500 (i/(n-1))^3, wealth grid linspace(0, 500, n_wealth)."""
    from pylcm_b200 import DCEGM, ConsumptionSavingsRegime, ExtremeValueTasteShocks, FUESEnvelope, IrregSpacedGrid, LiquidMargin

    sav = IrregSpacedGrid(points=tuple(500.0 * (i / (n_savings - 1)) ** 3 for i in range(n_savings)))
    solver = DCEGM(savings_grid=sav, n_constrained_points=n_constrained, envelope=FUESEnvelope())
    margin = LiquidMargin(state="wealth", action="consumption", resources="wealth", post_decision_state="savings")
    wealth = LinSpacedGrid(start=0, stop=500, n_points=n_wealth)
    cons = LinSpacedGrid(start=0.1, stop=500, n_points=200)
    last = n_periods - 1
    working = ConsumptionSavingsRegime(
        actions={"labor_supply": DiscreteGrid(LaborSupply), "consumption": cons},
        states={"shock": DiscreteGrid(GHShock16), "wealth": wealth},
        state_transitions={"wealth": _egm_next_wealth_work, "shock": MarkovTransition(_egm_next_shock)},
        transition=_egm_nr_work,
        functions={"utility": _egm_u_work, "savings": _egm_savings, "inverse_marginal_utility": _egm_inv_mu},
        solver=solver,
        liquid=margin,
        taste_shocks=ExtremeValueTasteShocks() if taste else None,
        active=lambda age, last=last: age < last,
    )
    retired = ConsumptionSavingsRegime(
        actions={"consumption": cons},
        states={"wealth": wealth},
        state_transitions={"wealth": _egm_next_wealth_ret},
        transition=_egm_nr_ret,
        functions={"utility": _egm_u_ret, "savings": _egm_savings, "inverse_marginal_utility": _egm_inv_mu},
        solver=solver,
        liquid=margin,
        active=lambda age, last=last: age < last,
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(
        regimes={"working": working, "retired": retired, "dead": dead},
        ages=AgeGrid(start=0, stop=last, step="Y"),
        regime_id_class=EgmRegimeId,
        fixed_params={"last_decision_period": n_periods - 2},
    )


def dcegm_params(seed=0, taste_scale=None, beta=0.97, crra=2.0, interest_rate=0.04, wage=20.0, sigma=0.1):
    rng = np.random.default_rng(seed)
    x, w = np.polynomial.hermite.hermgauss(16)
    values = np.exp(np.sqrt(2.0) * sigma * x)
    weights = w / np.sqrt(np.pi)
    p = {
        "discount_factor": beta,
        "crra": crra,
        "interest_rate": interest_rate,
        "wage": wage,
        "disutility_of_work": float(rng.uniform(0.2, 1.0)),
        "shock_values": values,
        "shock_weights": np.tile(weights, (16, 1)),
    }
    if taste_scale is not None:
        p["working"] = {"taste_shocks": {"scale": taste_scale}}
    return p
