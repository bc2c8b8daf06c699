"""The reference's random stream (JAX's Threefry-2x32 with its key threading)
against the reference's stored stochastic simulations.

- Threefry-2x32-20 known-answer vectors (Random123's test vectors, which
  JAX's own tests use);
- the oracle with ``rng="jax"`` reproduces the stored simulations of the
  process models (``tests/test_processes.py``: 2 subjects, seed 42; Markov
  health draws and process draws) and of the mortality example
  (``tests/test_regression_test.py``: 4 subjects, seed 12345; survival drawn
  in Markov regime transitions) at the reference's atol of 1e-5;
- on the GPU, ``Model.simulate`` (whose default stream this is) reproduces the
  same stored simulations.
"""

import numpy as np
import pytest

from pylcm_b200 import jaxrng
from tests import models as M
from tests.conftest import GOLDEN

KINDS = ["uniform", "normal", "lognormal", "tauchen", "rouwenhorst"]


def test_threefry_known_answers():
    cases = [((0, 0), (0, 0), (0x6B200159, 0x99BA4EFE)),
             ((0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF, 0xFFFFFFFF), (0x1CB996FC, 0xBB002BE7)),
             ((0x13198A2E, 0x03707344), (0x243F6A88, 0x85A308D3), (0xC4923A9C, 0x483DF7A0))]
    for (k0, k1), (x0, x1), want in cases:
        got = jaxrng.threefry2x32(k0, k1, x0, x1)
        assert (int(got[0]), int(got[1])) == want


def test_split_and_draw_conventions():
    k = jaxrng.key(42)
    assert k.tolist() == [0, 42]
    ks = jaxrng.split(k, 4)
    assert ks.shape == (4, 2)
    # key i of a split is the hash of the counters (0, i)
    for i in range(4):
        h = jaxrng.threefry2x32(0, 42, 0, i)
        assert ks[i].tolist() == [int(h[0]), int(h[1])]
    u = jaxrng.uniform(ks)
    assert np.all((u >= 0) & (u < 1))
    # a vector draw's element 0 is the scalar draw of the same key
    assert jaxrng.uniform_shaped(ks, 3)[:, 0].tolist() == u.tolist()


def _proc_ic():
    return {"health": np.array([0, 0]), "income": np.array([0.0, 0.0]), "wealth": np.array([1.0, 1.0]),
            "age": np.zeros(2), "regime_id": np.array([0, 0])}


def _check_processes(periods, kind):
    g = np.load(GOLDEN / f"processes_simulation_{kind}.npz")
    names = {s.rid: s.name for s in M.processes_model(4, kind).regime_specs}
    health = {"bad": 0.0, "good": 1.0}
    for row in range(len(g["period"])):
        p, i = int(g["period"][row]), int(g["subject_id"][row])
        d = periods[p]
        assert names[int(np.asarray(d["regime_id"])[i])] == g["regime"][row], (kind, row)
        np.testing.assert_allclose(np.asarray(d["value"])[i], g["value"][row], atol=1e-5)
        if g["regime"][row] == "dead":
            continue
        np.testing.assert_allclose(np.asarray(d["states"]["income"])[i], g["income"][row], atol=1e-5, err_msg=kind)
        np.testing.assert_allclose(np.asarray(d["states"]["wealth"])[i], g["wealth"][row], atol=1e-5, err_msg=kind)
        assert np.asarray(d["states"]["health"])[i] == health[g["health"][row]], (kind, row)
        np.testing.assert_allclose(np.asarray(d["actions"]["consumption"])[i], g["consumption"][row], atol=1e-5)


@pytest.mark.parametrize("kind", KINDS)
def test_oracle_reproduces_the_reference_process_simulations(kind):
    from oracle.simulate import simulate

    out = simulate(M.processes_model(4, kind), M.processes_params(kind), _proc_ic(), seed=42, rng="jax")
    _check_processes(out, kind)


def _mort_ic():
    n = 4
    return {"wealth": np.full(n, 100.0), "age": np.full(n, 40.0), "regime_id": np.zeros(n, dtype=int)}


def _check_mortality(periods):
    g = np.load(GOLDEN / "mortality_simulation.npz")
    names = {s.rid: s.name for s in M.mortality_model().regime_specs}
    for row in range(len(g["period"])):
        p, i = int(g["period"][row]), int(g["subject_id"][row])
        d = periods[p]
        assert names[int(np.asarray(d["regime_id"])[i])] == g["regime"][row], row
        np.testing.assert_allclose(np.asarray(d["value"])[i], g["value"][row], atol=1e-5)
        if g["regime"][row] == "dead":
            continue
        np.testing.assert_allclose(np.asarray(d["states"]["wealth"])[i], g["wealth"][row], atol=1e-5)
        np.testing.assert_allclose(np.asarray(d["actions"]["consumption"])[i], g["consumption"][row], atol=1e-5)


def test_oracle_reproduces_the_reference_mortality_simulation_exactly():
    from oracle.simulate import simulate

    _check_mortality(simulate(M.mortality_model(), M.mortality_params(), _mort_ic(), seed=12345, rng="jax"))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_gpu_reproduces_the_reference_process_simulations(kind):
    res = M.processes_model(4, kind).simulate(params=M.processes_params(kind), initial_conditions=_proc_ic(),
                                              seed=42, log_level="off")
    _check_processes(res.periods, kind)


@pytest.mark.gpu
def test_gpu_reproduces_the_reference_mortality_simulation_exactly():
    res = M.mortality_model().simulate(params=M.mortality_params(), initial_conditions=_mort_ic(), seed=12345,
                                       log_level="off")
    _check_mortality(res.periods)
