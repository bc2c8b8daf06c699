"""Example models: the benchmark workloads.

Seeded synthetic workloads with the shapes of the benchmark configurations:

- ``retirement_model`` -- deterministic consumption-savings model with an
  absorbing work/retire choice (wealth and consumption on linspace(1, 400, n),
  u = log c - 0.5 work, w' = 1.05 (w - c) + 20 work);
- ``stochastic_model`` -- its stochastic version: 7-node Tauchen AR(1) log
  income multiplying the wage, CRRA utility;
- ``dcegm_model`` -- Iskhakov-style retirement model solved by DC-EGM with
  the FUES envelope, 16-node Gauss-Hermite lognormal income weights carried
  by a discrete iid shock state (the reference rejects an even Gauss-Hermite
  node count, ``src/_lcm/processes/base.py:150``), optional EV1 taste shocks;
- ``hc_model`` -- two continuous states (wealth, human capital) and a
  32-state Markov shock with Dirichlet(1) rows.

The structure follows the reference's example models
(``src/lcm_examples/iskhakov_et_al_2017.py:136-344``); the grid sizes and the
parameter draws are those of the benchmark.
"""

from __future__ import annotations

import numpy as np

from pylcm_b200 import jnp
from pylcm_b200.ages import AgeGrid
from pylcm_b200.grids import DiscreteGrid, IrregSpacedGrid, LinSpacedGrid, categorical
from pylcm_b200.model import Model
from pylcm_b200.processes import TauchenAR1Process
from pylcm_b200.regime import (
    ConsumptionSavingsRegime,
    ExtremeValueTasteShocks,
    LiquidMargin,
    MarkovTransition,
    Regime,
)
from pylcm_b200.solvers import DCEGM, FUESEnvelope


@categorical(ordered=True)
class LaborSupply:
    work: int
    retire: int


def _borrowing_constraint(consumption, wealth):
    return consumption <= wealth


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


def dcegm_model(n_periods=40, n_savings=2000, n_wealth=2000, taste=False, n_constrained=20, n_points_to_scan=None,
                envelope=None):
    """Savings grid 500 (i/(n-1))^3, wealth grid linspace(0, 500, n_wealth);
    FUES with an exhaustive look-ahead unless `n_points_to_scan` is given, or
    the given `envelope` configuration."""
    sav = IrregSpacedGrid(points=tuple(500.0 * (i / (n_savings - 1)) ** 3 for i in range(n_savings)))
    solver = DCEGM(savings_grid=sav, n_constrained_points=n_constrained,
                   envelope=envelope if envelope is not None else FUESEnvelope(n_points_to_scan=n_points_to_scan))
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


# --------------------------------------------------------------------------
# serving workload: a stream of solve+simulate requests
# --------------------------------------------------------------------------
def tauchen_stationary(model) -> tuple[np.ndarray, np.ndarray]:
    """(nodes, stationary distribution) of the income process of a
    `stochastic_model` (left unit eigenvector of its transition matrix)."""
    spec = next(s for s in model.regime_specs if any(a.kind == "process" for a in s.states))
    ax = next(a for a in spec.states if a.kind == "process")
    g = ax.grid
    kw = {"rho": g.rho, "sigma": g.sigma, "mu": g.mu, "n_std": g.n_std}
    nodes = g.compute_gridpoints(**kw)
    P = g.compute_transition_probs(**kw)
    w, v = np.linalg.eig(P.T)
    pi = np.real(v[:, np.argmin(np.abs(w - 1.0))])
    pi = np.abs(pi) / np.abs(pi).sum()
    return nodes, pi


def serving_requests(n_requests: int = 4096, seed: int = 0, rate: float | None = None, n_agents: int = 10_000,
                     sizes=(100, 250, 500, 1000, 2000), horizons=(10, 40, 60), n_consumption: int = 500,
                     return_V_every: int = 0) -> list:
    """Seeded request stream of the serving benchmark.

    Each request draws the stochastic retirement model (grid search) or the
    DC-EGM retirement model (taste-shock scale absent or 0.05) with
    probability 1/2, a wealth-grid size from `sizes` (also the DC-EGM
    savings-grid size; the grid-search consumption grid keeps
    `n_consumption` points, the DC-EGM one 200), a horizon from `horizons`,
    and parameters beta ~ U[0.90, 0.99], crra ~ U[1, 5], r ~ U[0.01, 0.06]
    (DC-EGM: disutility of work ~ U[0.2, 1.0]); it simulates `n_agents`
    subjects with initial wealth ~ U[1, 50] and the income state drawn from
    its stationary distribution (Tauchen: the transition matrix's; the iid
    Gauss-Hermite shock: its weights), all starting in the working regime.
    Arrivals are Poisson with `rate` requests/s (all at 0 when None).
    """
    from pylcm_b200.serving import Request

    rng = np.random.default_rng(seed)
    arrivals = np.random.default_rng([seed, 1])  # arrival times do not change the requests
    models: dict = {}
    out = []
    t = 0.0
    gh_w = np.polynomial.hermite.hermgauss(16)[1] / np.sqrt(np.pi)
    for i in range(n_requests):
        kind = "gs" if rng.uniform() < 0.5 else "egm"
        n = int(rng.choice(sizes))
        T = int(rng.choice(horizons))
        beta = float(rng.uniform(0.90, 0.99))
        crra = float(rng.uniform(1.0, 5.0))
        r = float(rng.uniform(0.01, 0.06))
        if kind == "gs":
            family = "stochastic_retirement"
            key = (family, n, T)
            if key not in models:
                models[key] = stochastic_model(T, n, n_consumption)
            model = models[key]
            params = stochastic_params(beta=beta, crra=crra, interest_rate=r)
            nodes, pi = tauchen_stationary(model)
            ic = {
                "wealth": rng.uniform(1.0, 50.0, n_agents),
                "income": nodes[rng.choice(len(nodes), size=n_agents, p=pi)],
            }
        else:
            taste = None if rng.uniform() < 0.5 else 0.05
            family = ("dcegm_retirement", taste is not None)
            key = (family, n, T)
            if key not in models:
                models[key] = dcegm_model(n_periods=T, n_savings=n, n_wealth=n, taste=taste is not None)
            model = models[key]
            params = dcegm_params(seed=int(rng.integers(1 << 31)), taste_scale=taste, beta=beta, crra=crra,
                                  interest_rate=r)
            ic = {
                "wealth": rng.uniform(1.0, 50.0, n_agents),
                "shock": rng.choice(16, size=n_agents, p=gh_w).astype(np.float64),
            }
        rid = {s.name: s.rid for s in model.regime_specs}["working"]
        ic["regime_id"] = np.full(n_agents, rid, dtype=np.int64)
        if rate:
            t += float(arrivals.exponential(1.0 / rate))
        out.append(Request(family=family, key=key, model=model, params=params, initial_conditions=ic,
                           seed=int(rng.integers(1 << 62)), arrival=t, rid=i,
                           return_V=bool(return_V_every) and i % return_V_every == 0))
    return out
