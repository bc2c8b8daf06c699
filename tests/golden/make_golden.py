"""Extract the reference's stored float64 solutions into small .npz fixtures.

Run once with the environment variable REFERENCE set to a checkout of the
reference project; the outputs are committed, so tests never read the
reference.

The reference's .pkl files hold cloudpickled JAX arrays; they unpickle without
JAX through a stub of ``jax._src.array._reconstruct_array`` that rebuilds the
NumPy payload.
"""

from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

def _reference() -> Path:
    ref = os.environ.get("REFERENCE")
    if not ref:
        raise SystemExit("set REFERENCE to the directory of a checkout of the reference project")
    return Path(ref)

OUT = Path(__file__).resolve().parent


def _install_jax_stub() -> None:
    jax = types.ModuleType("jax")
    src = types.ModuleType("jax._src")
    arr = types.ModuleType("jax._src.array")

    def _reconstruct_array(fun, args, arr_state, aval_state):  # noqa: ARG001
        a = fun(*args)
        if arr_state:
            a.__setstate__(arr_state)
        return a

    arr._reconstruct_array = _reconstruct_array
    sys.modules.setdefault("jax", jax)
    sys.modules.setdefault("jax._src", src)
    sys.modules.setdefault("jax._src.array", arr)


def _flatten(sol) -> dict[str, np.ndarray]:
    out = {}
    for period, regimes in sol.items():
        for regime, arr in regimes.items():
            out[f"{int(period)}/{regime}"] = np.asarray(arr, dtype=np.float64)
    return out


def main() -> None:
    _install_jax_stub()
    import pandas as pd

    data = _reference() / "tests" / "data"
    np.savez(OUT / "regression_solution.npz", **_flatten(pd.read_pickle(data / "regression_tests" / "solution.pkl")))
    for kind in ("uniform", "normal", "lognormal", "tauchen", "rouwenhorst"):
        sol = pd.read_pickle(data / "processes" / f"solution_{kind}.pkl")
        np.savez(OUT / f"processes_solution_{kind}.npz", **_flatten(sol))
    sim = pd.read_pickle(data / "regression_tests" / "simulation.pkl")
    np.savez(
        OUT / "regression_simulation.npz",
        subject_id=sim["subject_id"].to_numpy(np.int64),
        period=sim["period"].to_numpy(np.int64),
        regime=sim["regime_name"].astype(str).to_numpy(),
        value=sim["value"].to_numpy(np.float64),
        wealth=sim["wealth"].to_numpy(np.float64),
        consumption=sim["consumption"].to_numpy(np.float64),
        labor_supply=sim["labor_supply"].astype(str).to_numpy(),
        age=sim["age"].to_numpy(np.float64),
    )
    for kind in ("five_periods", "low_delta"):
        for what in ("values_worker", "values_retired", "consumption", "work_decision"):
            src = data / "analytical_solution" / f"iskhakov_2017_{kind}__{what}.csv"
            if src.exists():
                arr = np.genfromtxt(src, delimiter=",")
                np.save(OUT / f"analytical_{kind}__{what}.npy", arr)
    # the mortality example's stored float64 simulation (4 subjects from wealth
    # 100 at age 40; its survival path is one draw of the reference's stream)
    mort = pd.read_pickle(data / "regression_tests" / "f64" / "mortality_simulation.pkl")
    np.savez(
        OUT / "mortality_simulation.npz",
        subject_id=mort["subject_id"].to_numpy(np.int64),
        period=mort["period"].to_numpy(np.int64),
        regime=mort["regime_name"].astype(str).to_numpy().astype("U"),
        value=mort["value"].to_numpy(np.float64),
        wealth=mort["wealth"].to_numpy(np.float64),
        consumption=mort["consumption"].to_numpy(np.float64),
        labor_supply=mort["labor_supply"].astype(str).to_numpy().astype("U"),
        age=mort["age"].to_numpy(np.float64),
    )
    processes_simulations(data)
    # the independent `dcegm` package's solution of the IJRS retirement model
    # with taste shocks (the reference's cross-check fixture)
    df = pd.read_csv(data / "dcegm_reference" / "ijrs_taste_shocks_reference.csv")
    np.savez(OUT / "ijrs_taste_shocks_reference.npz", **{c: df[c].to_numpy(np.float64) for c in df.columns})


def processes_simulations(data: Path) -> None:
    """The stored stochastic simulations of the process models (2 subjects, 4
    periods, seed 42): drawn from JAX's default stream, so they pin a
    restatement of that stream (Markov health draws, process draws)."""
    import pandas as pd

    for kind in ("uniform", "normal", "lognormal", "tauchen", "rouwenhorst"):
        sim = pd.read_pickle(data / "processes" / f"simulation_{kind}.pkl")
        np.savez(
            OUT / f"processes_simulation_{kind}.npz",
            subject_id=sim["subject_id"].to_numpy(np.int64),
            period=sim["period"].to_numpy(np.int64),
            regime=sim["regime_name"].astype(str).to_numpy().astype("U"),
            value=sim["value"].to_numpy(np.float64),
            health=sim["health"].astype(str).to_numpy().astype("U"),
            income=sim["income"].to_numpy(np.float64),
            wealth=sim["wealth"].to_numpy(np.float64),
            consumption=sim["consumption"].to_numpy(np.float64),
            age=sim["age"].to_numpy(np.float64),
        )


if __name__ == "__main__":
    main()
