"""The LTM, RFC and MSS upper-envelope oracles against the reference's own
known-answer cases (``tests/solution/test_ltm.py``, ``tests/solution/test_rfc.py``
and ``tests/solution/test_backend_oracle_parity.py``: crossing linear segments,
concave pass-through, a loop-back segment, a strictly dominated branch, value
dips, dead candidates, overflow)."""

import numpy as np

from oracle.envelopes import refine_ltm, refine_mss, refine_rfc


def _kept(a):
    a = np.asarray(a)
    return a[~np.isnan(a)]


def _crossing():
    """Segment A: v = 1 + 0.4 R, c = 0.3 R; segment B: v = 0.1 + 0.8 R,
    c = 0.55 R; they cross at R = 2.25.  Each arrives as its own run."""
    ra = np.array([0.6, 1.2, 1.8, 2.4])
    rb = np.array([0.8, 1.6, 2.6, 3.4])
    g = np.concatenate([ra, rb])
    v = np.concatenate([1.0 + 0.4 * ra, 0.1 + 0.8 * rb])
    p = np.concatenate([0.30 * ra, 0.55 * rb])
    mu = np.concatenate([np.full(4, 0.4), np.full(4, 0.8)])
    return g, p, v, mu


def _check_tail(row):
    raw = np.asarray(row)
    nan = np.isnan(raw)
    first = int(nan.argmax()) if nan.any() else raw.size
    assert not nan[:first].any() and nan[first:].all()
    assert np.all(np.diff(raw[:first]) >= -1e-12)


# ---------------------------------------------------------------- LTM
def test_ltm_concave_row_passes_through():
    g = np.linspace(1.0, 10.0, 10)
    rg, rp, rv, n = refine_ltm(g, 0.3 * g, np.log(g), 14)
    assert n == 10
    np.testing.assert_allclose(_kept(rg), g, atol=1e-12)
    np.testing.assert_allclose(_kept(rv), np.log(g), atol=1e-12)
    np.testing.assert_allclose(_kept(rp), 0.3 * g, atol=1e-12)


def test_ltm_value_at_each_node_is_the_segment_maximum():
    g, p, v, _ = _crossing()
    rg, rp, rv, n = refine_ltm(g, p, v, 12)
    kg, kv = _kept(rg), _kept(rv)
    np.testing.assert_allclose(kv, np.maximum(1.0 + 0.4 * kg, 0.1 + 0.8 * kg), atol=1e-12)
    kp = _kept(rp)
    np.testing.assert_allclose(kp[np.argmin(np.abs(kg - 1.2))], 0.30 * 1.2, atol=1e-12)
    np.testing.assert_allclose(kp[np.argmin(np.abs(kg - 2.6))], 0.55 * 2.6, atol=1e-12)
    _check_tail(rg)


def test_ltm_loop_back_segment_lifts_a_lower_node():
    rg, _, rv, _ = refine_ltm([1.0, 3.0, 2.0, 4.0], [0.5, 1.5, 1.0, 2.0], [1.0, 2.0, 5.0, 7.0], 8)
    kg, kv = _kept(rg), _kept(rv)
    np.testing.assert_allclose(kv[np.argmin(np.abs(kg - 2.0))], 5.0, atol=1e-12)


def test_ltm_overflow_and_dead_candidates():
    g, p, v, _ = _crossing()
    assert refine_ltm(g, p, v, 4)[3] > 4
    # a NaN value kills the candidate and both segments touching it; an
    # isolated live candidate (no live segment) is dropped too
    rg, _, _, n = refine_ltm([1.0, 2.0, 3.0, 4.0, 5.0], [1, 1, 1, 1, 1], [1.0, np.nan, 2.0, np.nan, 3.0], 6)
    assert n == 0 and np.isnan(rg).all()


# ---------------------------------------------------------------- RFC
def test_rfc_concave_row_passes_through():
    g = np.linspace(1.0, 10.0, 10)
    rg, rp, rv, n = refine_rfc(g, 0.3 * g, np.log(g), 1.0 / g, 14)
    assert n == 10
    np.testing.assert_allclose(_kept(rg), g, atol=1e-12)
    np.testing.assert_allclose(_kept(rp), 0.3 * g, atol=1e-12)
    np.testing.assert_allclose(_kept(rv), np.log(g), atol=1e-12)
    assert refine_rfc(g, 0.3 * g, np.log(g), 1.0 / g, 4)[3] > 4


def test_rfc_steep_continuous_policy_is_not_a_switch():
    g = np.linspace(1.0, 5.0, 9)
    assert refine_rfc(g, 5.0 - 0.9 * g, np.log(g), 1.0 / g, 12)[3] == 9


def test_rfc_crossing_segments_keep_the_upper_subset():
    g, p, v, mu = _crossing()
    rg, _, _, n = refine_rfc(g, p, v, mu, 12, jump_thresh=0.6)
    np.testing.assert_allclose(np.sort(_kept(rg)), [0.6, 1.2, 1.8, 2.6, 3.4], atol=1e-12)
    assert not np.any(np.isclose(_kept(rg), 2.25, atol=1e-6))
    _check_tail(rg)


def test_rfc_value_dip_and_dead_candidates_are_dropped():
    rg, _, _, _ = refine_rfc([1.0, 2.0, 3.0], [0.5, 1.8, 1.5], [1.0, 0.9, 2.0], [0.5, 0.5, 0.5], 6,
                             jump_thresh=0.5)
    assert not np.any(np.isclose(_kept(rg), 2.0))
    rg, _, rv, n = refine_rfc([1.0, 2.0, 3.0, 4.0], [0.5, 1.0, 1.5, 2.0], [1.0, np.nan, 2.0, 2.5],
                              [0.5, 0.0, 0.5, 0.5], 8)
    assert n == 3 and not np.any(np.isclose(_kept(rg), 2.0)) and not np.isnan(_kept(rv)).any()


def test_rfc_sorts_any_input_order():
    g, p, v, mu = _crossing()
    perm = np.random.default_rng(0).permutation(g.size)
    a = refine_rfc(g, p, v, mu, 12, jump_thresh=0.6)
    b = refine_rfc(g[perm], p[perm], v[perm], mu[perm], 12, jump_thresh=0.6)
    for x, y in zip(a[:3], b[:3]):
        np.testing.assert_array_equal(x, y)


def test_envelope_configurations():
    import pytest

    from pylcm_b200 import DCEGM, IrregSpacedGrid, LTMEnvelope, MSSEnvelope, RFCEnvelope

    sav = IrregSpacedGrid(points=(0.0, 1.0, 2.0))
    assert DCEGM(savings_grid=sav, envelope=LTMEnvelope()).envelope == LTMEnvelope()
    assert DCEGM(savings_grid=sav, envelope=RFCEnvelope(search_radius=3)).envelope.search_radius == 3
    assert DCEGM(savings_grid=sav, envelope=MSSEnvelope()).envelope == MSSEnvelope()
    with pytest.raises(NotImplementedError, match="str is not implemented"):
        DCEGM(savings_grid=sav, envelope="fues")
    from pylcm_b200 import ExactEnvelope

    with pytest.raises(NotImplementedError, match="ExactEnvelope is not implemented"):
        DCEGM(savings_grid=sav, envelope=ExactEnvelope())
    with pytest.raises(ValueError):
        ExactEnvelope(max_runs=1)
    with pytest.raises(ValueError):
        RFCEnvelope(jump_thresh=0.0)
    with pytest.raises(ValueError):
        RFCEnvelope(search_radius=0)


def test_oracle_dcegm_with_each_envelope_tracks_the_closed_form():
    """The oracle's DC-EGM solve with LTM, RFC and MSS stays within 1e-3 of
    the Iskhakov et al. (2017) closed form (LTM and RFC insert no crossing:
    kinks within the grid spacing)."""
    from oracle.dcegm import solve
    from pylcm_b200 import LTMEnvelope, MSSEnvelope, RFCEnvelope
    from tests.golden import analytical_models as AM

    for env in (LTMEnvelope(), RFCEnvelope(), MSSEnvelope()):
        model, params = AM.dcegm_model_and_params("five_periods", env)
        V, _ = solve(model, params)
        periods = sorted(V)
        for kind, reg in (("worker", "working_life"), ("retired", "retirement")):
            num = np.stack([V[p][reg] for p in periods[:-1]])
            ana = np.load(f"tests/golden/analytical_five_periods__values_{kind}.npy")
            assert np.abs(num - ana)[:, 2:].max() < 1e-3, (type(env).__name__, kind)


# ---------------------------------------------------------------- MSS
def test_mss_inserts_the_crossing_twice():
    g, p, v, _ = _crossing()
    rg, rp, rv, n = refine_mss(g, p, v, 16)
    kg, kp, kv = _kept(rg), _kept(rp), _kept(rv)
    assert n == 10
    at = np.flatnonzero(np.isclose(kg, 2.25, atol=1e-12))
    assert at.size == 2
    np.testing.assert_allclose(kv[at], 1.9, atol=1e-12)
    np.testing.assert_allclose(kp[at], [0.30 * 2.25, 0.55 * 2.25], atol=1e-12)  # left, then right policy
    nodes = np.delete(kg, at)
    np.testing.assert_allclose(np.delete(kv, at), np.maximum(1.0 + 0.4 * nodes, 0.1 + 0.8 * nodes), atol=1e-12)
    _check_tail(rg)
    assert refine_mss(g, p, v, 5)[3] == 10  # overflow: the count says so


def test_every_envelope_deletes_a_strictly_dominated_branch():
    """Branch 0: V = R, c = 0.3 R; branch 1: V = R - 1, c = 10, below it
    everywhere; the envelope is branch 0."""
    x = [0.0, 1.0, 2.0, 3.0]
    g = np.array(x + x)
    v = np.array(x + [t - 1.0 for t in x])
    p = np.array([0.3 * t for t in x] + [10.0] * 4)
    q = np.linspace(0.0, 3.0, 13)
    for name, (rg, rp, rv, _) in {
        "ltm": refine_ltm(g, p, v, 32), "mss": refine_mss(g, p, v, 32),
        "rfc": refine_rfc(g, p, v, np.ones_like(g), 32, search_radius=32),
    }.items():
        keep = ~np.isnan(rg)
        np.testing.assert_allclose(np.interp(q, rg[keep], rv[keep]), q, atol=1e-9, err_msg=name)
        np.testing.assert_allclose(np.interp(q, rg[keep], rp[keep]), 0.3 * q, atol=1e-9, err_msg=name)


def test_every_envelope_is_the_identity_on_one_concave_branch():
    g = np.array([0.0, 1.0, 2.0, 3.0, 4.0])
    v = np.array([0.0, 1.0, 1.7, 2.2, 2.5])
    p = np.array([0.0, 0.6, 1.0, 1.3, 1.5])
    mu = np.array([1.0, 0.85, 0.6, 0.45, 0.3])
    q = np.linspace(0.0, 4.0, 17)
    for rg, _, rv, n in (refine_ltm(g, p, v, 16), refine_mss(g, p, v, 16), refine_rfc(g, p, v, mu, 16)):
        keep = ~np.isnan(rg)
        assert n == 5
        np.testing.assert_allclose(np.interp(q, rg[keep], rv[keep]), np.interp(q, g, v), atol=1e-12)


def test_egm_and_negm_configurations_are_refused_clearly():
    """EGM and NEGM load as configurations (so models naming them import) and
    a regime declaring either is refused with NotImplementedError; an unknown
    solver object is refused too."""
    import pytest

    from pylcm_b200 import EGM, NEGM, DCEGM, IrregSpacedGrid, LinSpacedGrid, Regime
    from pylcm_b200.exceptions import RegimeInitializationError

    sav = IrregSpacedGrid(points=(0.0, 1.0, 2.0))
    egm = EGM(savings_grid=sav)
    negm = NEGM(inner=DCEGM(savings_grid=sav), outer_grid=LinSpacedGrid(start=0, stop=1, n_points=3))
    with pytest.raises(ValueError):
        NEGM(inner=DCEGM(savings_grid=sav), outer_grid=sav, outer_batch_size=-1)
    base = dict(actions={"c": LinSpacedGrid(start=1, stop=2, n_points=3)},
                states={"w": LinSpacedGrid(start=1, stop=2, n_points=3)},
                functions={"utility": lambda c: c}, transition=lambda: 0)
    for solver in (egm, negm):
        with pytest.raises(NotImplementedError, match=type(solver).__name__):
            Regime(solver=solver, **base)
    with pytest.raises(RegimeInitializationError, match="unknown solver"):
        Regime(solver=object(), **base)
