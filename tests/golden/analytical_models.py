"""The retirement model behind the reference's analytical-solution fixtures
(Iskhakov, Joergensen, Rust & Schjerning 2017): log utility, work disutility,
absorbing retirement, deterministic death; wealth and consumption on
linspace(1, 400, 100/500).  Parametrisations from the reference's
``tests/test_analytical_solution.py``."""

from pylcm_b200 import AgeGrid, DiscreteGrid, LinSpacedGrid, Model, Regime, categorical
from pylcm_b200 import jnp


@categorical(ordered=True)
class Labor:
    work: int
    retire: int


@categorical(ordered=False)
class Rid:
    working_life: int
    retirement: int
    dead: int


def _u_work(consumption, is_working, disutility_of_work):
    return jnp.log(consumption) - jnp.where(is_working, disutility_of_work, 0.0)


def _u_ret(consumption):
    return jnp.log(consumption)


def _income(is_working, wage):
    return jnp.where(is_working, wage, 0.0)


def _is_working(labor_supply):
    return labor_supply == Labor.work


def _next_wealth(wealth, consumption, labor_income, interest_rate):
    return (1 + interest_rate) * (wealth - consumption) + labor_income


def _bc(consumption, wealth):
    return consumption <= wealth


def _nr_work(labor_supply, age, final_age_alive):
    return jnp.where(
        age >= final_age_alive,
        Rid.dead,
        jnp.where(labor_supply == Labor.retire, Rid.retirement, Rid.working_life),
    )


def _nr_ret(age, final_age_alive):
    return jnp.where(age >= final_age_alive, Rid.dead, Rid.retirement)


def get_model(n_periods: int) -> Model:
    wealth = LinSpacedGrid(start=1, stop=400, n_points=100)
    cons = LinSpacedGrid(start=1, stop=400, n_points=500)
    ages = AgeGrid(start=40, stop=40 + (n_periods - 1) * 10, step="10Y")
    last = ages.exact_values[-1]
    work = Regime(
        actions={"labor_supply": DiscreteGrid(Labor), "consumption": cons},
        states={"wealth": wealth},
        state_transitions={"wealth": _next_wealth},
        constraints={"borrowing_constraint": _bc},
        transition=_nr_work,
        functions={"utility": _u_work, "labor_income": _income, "is_working": _is_working},
        active=lambda age, la=last: age < la,
    )
    ret = Regime(
        actions={"consumption": cons},
        states={"wealth": wealth},
        state_transitions={"wealth": _next_wealth},
        constraints={"borrowing_constraint": _bc},
        transition=_nr_ret,
        functions={"utility": _u_ret},
        active=lambda age, la=last: age < la,
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(regimes={"working_life": work, "retirement": ret, "dead": dead}, ages=ages, regime_id_class=Rid)


def get_params(n_periods, discount_factor, disutility_of_work, interest_rate, wage):
    return {
        "discount_factor": discount_factor,
        "interest_rate": interest_rate,
        "final_age_alive": 40 + (n_periods - 2) * 10,
        "working_life": {"utility": {"disutility_of_work": disutility_of_work}, "labor_income": {"wage": wage}},
        "retirement": {"next_wealth": {"labor_income": 0.0}},
    }


CASES = {
    "five_periods": dict(n_periods=6, discount_factor=0.98, disutility_of_work=1.0, interest_rate=0.0, wage=20.0),
    "low_delta": dict(n_periods=4, discount_factor=0.98, disutility_of_work=0.1, interest_rate=0.0, wage=20.0),
}


def model_and_params(case: str):
    kw = CASES[case]
    return get_model(kw["n_periods"]), get_params(**kw)


# ---------------------------------------------------------------------------
# the same model solved by DC-EGM with the FUES envelope
def _savings(wealth, consumption):
    return wealth - consumption


def _next_wealth_from_savings(savings, labor_income, interest_rate):
    return (1 + interest_rate) * savings + labor_income


def _inv_mu_log(marginal_continuation):
    return 1.0 / marginal_continuation


def get_dcegm_model(n_periods: int, n_savings: int = 200, n_constrained: int = 64, envelope=None) -> Model:
    from pylcm_b200 import DCEGM, ConsumptionSavingsRegime, FUESEnvelope, IrregSpacedGrid, LiquidMargin

    wealth = LinSpacedGrid(start=1, stop=400, n_points=100)
    cons = LinSpacedGrid(start=1, stop=400, n_points=500)
    ages = AgeGrid(start=40, stop=40 + (n_periods - 1) * 10, step="10Y")
    last = ages.exact_values[-1]
    sav = IrregSpacedGrid(points=tuple(400.0 * (i / (n_savings - 1)) ** 3 for i in range(n_savings)))
    solver = DCEGM(savings_grid=sav, n_constrained_points=n_constrained,
                   envelope=envelope if envelope is not None else FUESEnvelope())
    margin = LiquidMargin(state="wealth", action="consumption", resources="wealth", post_decision_state="savings")
    work = ConsumptionSavingsRegime(
        actions={"labor_supply": DiscreteGrid(Labor), "consumption": cons},
        states={"wealth": wealth},
        state_transitions={"wealth": _next_wealth_from_savings},
        transition=_nr_work,
        functions={
            "utility": _u_work,
            "labor_income": _income,
            "is_working": _is_working,
            "savings": _savings,
            "inverse_marginal_utility": _inv_mu_log,
        },
        solver=solver,
        liquid=margin,
        active=lambda age, la=last: age < la,
    )
    ret = ConsumptionSavingsRegime(
        actions={"consumption": cons},
        states={"wealth": wealth},
        state_transitions={"wealth": _next_wealth_from_savings},
        transition=_nr_ret,
        functions={"utility": _u_ret, "savings": _savings, "inverse_marginal_utility": _inv_mu_log},
        solver=solver,
        liquid=margin,
        active=lambda age, la=last: age < la,
    )
    dead = Regime(transition=None, functions={"utility": lambda: 0.0})
    return Model(regimes={"working_life": work, "retirement": ret, "dead": dead}, ages=ages, regime_id_class=Rid)


def dcegm_model_and_params(case: str, envelope=None):
    kw = CASES[case]
    return get_dcegm_model(kw["n_periods"], envelope=envelope), get_params(**kw)
