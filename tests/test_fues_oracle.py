"""FUES (oracle restatement) on analytic cases: crossing linear segments, a
concave row that passes through, a node-aligned crossing, tied savings."""

import numpy as np

from oracle.fues import refine


def _crossing():
    # segment A: v = 1 + 0.4 R, c = 0.3 R ; segment B: v = 0.1 + 0.8 R, c = 0.55 R
    ra = np.array([0.6, 1.2, 1.8, 2.4])
    rb = np.array([0.8, 1.6, 2.6, 3.4])
    g = np.concatenate([ra, rb])
    v = np.concatenate([1.0 + 0.4 * ra, 0.1 + 0.8 * rb])
    c = np.concatenate([0.30 * ra, 0.55 * rb])
    return g, c, v


def _interp(gr, vr, q):
    m = ~np.isnan(gr)
    return np.interp(q, gr[m], vr[m])


def test_crossing_segments_give_the_analytic_envelope():
    g, c, v = _crossing()
    rg, rc, rv, n = refine(g, c, v, g - c, 12)
    q = np.linspace(0.7, 3.3, 53)
    np.testing.assert_allclose(_interp(rg, rv, q), np.maximum(1.0 + 0.4 * q, 0.1 + 0.8 * q), atol=1e-9)
    kink = np.isclose(rg, 2.25, atol=1e-9)
    assert kink.sum() == 2
    np.testing.assert_allclose(np.sort(rc[kink]), np.sort([0.3 * 2.25, 0.55 * 2.25]), atol=1e-9)
    for dominated in (0.8, 1.6, 2.4):
        assert not np.any(np.isclose(rg[~np.isnan(rg)], dominated, atol=1e-8))


def test_concave_row_passes_through():
    g = np.linspace(1.0, 10.0, 10)
    rg, rc, rv, n = refine(g, 0.3 * g, np.log(g), 0.7 * g, 14)
    assert n == 10
    np.testing.assert_allclose(rg[:10], g)
    np.testing.assert_allclose(rv[:10], np.log(g))


def test_tied_savings_keep_every_node():
    g = np.array([0.5, 1.0, 1.5, 2.0, 2.5, 3.0, 3.5, 4.0])
    c = g - 0.01
    s = np.full_like(g, 0.01)
    _, _, _, n = refine(g, c, np.log(g), s, 12)
    assert n == 8


def test_node_aligned_crossing_keeps_both_branches():
    g = np.array([9.0, 10.0, 12.0, 10.0, 11.0])
    c = np.array([8.5, 9.0, 9.0, 4.0, 4.5])
    v = np.array([4.6, 5.0, -100.0, 5.0, 5.8])
    rg, rc, rv, n = refine(g, c, v, g - c, 10)
    m = ~np.isnan(rg)
    assert not np.any(rg[m] == 12.0)  # dominated point dropped
    at = rg[m] == 10.0
    assert at.sum() == 2  # both branch policies at the node
    np.testing.assert_allclose(np.sort(rc[m][at]), [4.0, 9.0])


def _interlopers(n_between: int):
    """One concave segment A (savings slope 0.5) with runs of `n_between`
    points of a lower segment B (savings slope 0.05, a policy jump) between
    consecutive A points."""
    ra = np.arange(1.0, 11.0)
    g, c, v = [], [], []
    for k, r in enumerate(ra):
        g.append(r)
        c.append(0.5 * r)
        v.append(np.log(0.5 * r) + 2.0)
        if k + 1 < len(ra):
            for q in range(n_between):
                rb = r + (q + 1) / (n_between + 1)
                g.append(rb)
                c.append(0.95 * rb)
                v.append(np.log(0.95 * rb) + 1.0 + 0.2 * np.sin(7 * rb))
    g, c, v = map(np.asarray, (g, c, v))
    return g, c, v, g - c


def test_a_window_shorter_than_the_interloper_runs_changes_the_envelope():
    """The reference's caveat (fues.py:114-128): a bounded look-ahead that
    cannot reach past a run of off-segment candidates treats a segment point
    as without continuation; an exhaustive scan (None, or a window covering
    the row) reaches it."""
    g, c, v, s = _interlopers(4)
    n_out = 4 * len(g)
    full = refine(g, c, v, s, n_out)
    wide = refine(g, c, v, s, n_out, n_points_to_scan=len(g))
    narrow = refine(g, c, v, s, n_out, n_points_to_scan=2)
    for a, b in zip(full[:3], wide[:3]):
        np.testing.assert_array_equal(a, b)
    assert full[3] == wide[3]
    assert not all(np.array_equal(a, b, equal_nan=True) for a, b in zip(full[:3], narrow[:3]))
