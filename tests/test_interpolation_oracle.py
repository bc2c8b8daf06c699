"""Known answers for the value-function reads the oracle restates
(``ndimage.py:29-109``, ``coordinates.py``), as the reference's own
interpolation tests check them: interior points against SciPy's order-1
``map_coordinates``; outside the grid, linear extrapolation from the first or
last bracket (the lower index clamped to [0, n-2]); a zero-weight corner
ignoring an infinite value; coordinates of linear, logarithmic and irregular
grids against their definitions."""

import numpy as np
from scipy import ndimage

from oracle.grid_search import grid_coordinate, interp_rows
from pylcm_b200 import IrregSpacedGrid, LinSpacedGrid, LogSpacedGrid


def test_interior_points_match_scipy_order_one():
    rng = np.random.default_rng(0)
    for shape in ((7,), (5, 6), (4, 3, 5)):
        a = rng.normal(size=shape)
        pts = [rng.uniform(0, n - 1, size=200) for n in shape]
        got = interp_rows(a, pts)
        want = ndimage.map_coordinates(a, pts, order=1)
        np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13)


def test_outside_points_extrapolate_linearly():
    a = np.array([1.0, 3.0, 4.0, 8.0])
    c = np.array([-1.5, -0.25, 3.0, 3.5, 5.0])
    want = np.array([1.0 - 1.5 * 2.0, 1.0 - 0.25 * 2.0, 8.0, 8.0 + 0.5 * 4.0, 8.0 + 2.0 * 4.0])
    np.testing.assert_allclose(interp_rows(a, [c]), want, rtol=1e-15)


def test_zero_weight_corner_ignores_infinite_value():
    a = np.array([-np.inf, 2.0, 5.0])
    got = interp_rows(a, [np.array([1.0, 1.5, 0.5])])
    np.testing.assert_array_equal(got, [2.0, 3.5, -np.inf])


def test_grid_coordinates():
    lin = LinSpacedGrid(start=1.0, stop=5.0, n_points=9)
    v = np.array([1.0, 1.25, 4.9, 6.0, 0.0])
    np.testing.assert_allclose(grid_coordinate(lin, v), (v - 1.0) / 0.5, rtol=1e-15)
    log = LogSpacedGrid(start=1.0, stop=100.0, n_points=3)
    pts = log.to_numpy()
    v = np.array([1.0, 5.5, 10.0, 55.0, 100.0])
    lo = np.array([0, 0, 1, 1, 1])
    want = lo + (v - pts[lo]) / (pts[lo + 1] - pts[lo])
    np.testing.assert_allclose(grid_coordinate(log, v), want, rtol=1e-12)
    irr = IrregSpacedGrid(points=(0.0, 1.0, 3.0, 7.0))
    v = np.array([0.5, 1.0, 2.0, 7.0, 9.0, -1.0])
    np.testing.assert_allclose(grid_coordinate(irr, v), [0.5, 1.0, 1.5, 3.0, 3.5, -1.0], rtol=1e-15)
    np.testing.assert_allclose(np.interp(v[:4], irr.to_numpy(), np.arange(4.0)), grid_coordinate(irr, v[:4]))


def test_piecewise_grid_coordinates():
    """Inside a segment the coordinate is the segment's own (linear or
    logarithmic) coordinate plus the segment's offset; beyond the last node
    the last segment's spacing continues (``piecewise.py:107-118, 178-188``)."""
    from pylcm_b200 import PiecewiseGridSegment as S
    from pylcm_b200 import PiecewiseLinSpacedGrid, PiecewiseLogSpacedGrid

    g = PiecewiseLinSpacedGrid(segments=(S("[1, 4)", 4), S("[4, 10]", 4)))
    pts = g.to_numpy()
    assert len(g) == 8 and pts[3] < 4.0 == pts[4]
    v = np.array([1.0, 2.5, 4.0, 5.0, 10.0, 12.0, 0.0])
    np.testing.assert_allclose(grid_coordinate(g, v), [0.0, 1.5, 4.0, 4.5, 7.0, 8.0, -1.0], rtol=1e-14, atol=1e-14)
    h = PiecewiseLogSpacedGrid(segments=(S("[0.1, 10)", 3), S("[10, 1000]", 3)))
    v = np.array([1.0, 10.0, 100.0, 1000.0])
    np.testing.assert_allclose(grid_coordinate(h, v), [1.0, 3.0, 4.0, 5.0], rtol=1e-12, atol=1e-12)
    # inside segments: the irregular-grid coordinate on the same points
    from pylcm_b200 import IrregSpacedGrid

    irr = IrregSpacedGrid(points=tuple(h.to_numpy()))
    v = np.array([0.2, 0.5, 3.0, 20.0, 500.0])
    np.testing.assert_allclose(grid_coordinate(h, v), grid_coordinate(irr, v), rtol=1e-12)


def test_piecewise_grid_rejects_gaps_and_overlaps():
    import pytest

    from pylcm_b200 import PiecewiseGridSegment as S
    from pylcm_b200 import PiecewiseLinSpacedGrid, PiecewiseLogSpacedGrid
    from pylcm_b200.exceptions import GridInitializationError

    for segs in ((S("[1, 4)", 4), S("[5, 10]", 4)), (S("[1, 4]", 4), S("[4, 10]", 4)), (S("[1, 4)", 1),),
                 (S("1, 4", 3),)):
        with pytest.raises(GridInitializationError):
            PiecewiseLinSpacedGrid(segments=segs)
    with pytest.raises(GridInitializationError):
        PiecewiseLogSpacedGrid(segments=(S("[0, 4]", 3),))


def test_piecewise_device_table_reproduces_the_coordinate():
    """The table the kernels read for a piecewise grid ([breakpoints | starts |
    scales | offsets]), evaluated the way the device does, gives the oracle's
    coordinate."""
    from pylcm_b200 import PiecewiseGridSegment as S
    from pylcm_b200 import PiecewiseLinSpacedGrid, PiecewiseLogSpacedGrid

    rng = np.random.default_rng(4)
    for grid in (PiecewiseLinSpacedGrid(segments=(S("[1, 4)", 7), S("[4, 10]", 5), S("(10, 30]", 9))),
                 PiecewiseLogSpacedGrid(segments=(S("[0.1, 10]", 6), S("(10, 1000]", 8)))):
        tab = grid.coordinate_table()
        k = len(grid.segments)
        v = rng.uniform(0.05, 1200.0 if grid.log else 35.0, 500)
        seg = (v[:, None] >= tab[: k - 1][None, :]).sum(axis=1)
        st, sc, off = tab[k - 1: 2 * k - 1], tab[2 * k - 1: 3 * k - 1], tab[3 * k - 1:]
        if grid.log:
            c = (np.log(v) - st[seg]) / sc[seg]
            lo = np.floor(c)
            lower, upper = np.exp(st[seg] + sc[seg] * lo), np.exp(st[seg] + sc[seg] * (lo + 1))
            local = lo + (v - lower) / (upper - lower)
        else:
            local = (v - st[seg]) * sc[seg]
        np.testing.assert_allclose(off[seg] + local, grid_coordinate(grid, v), rtol=1e-12, atol=1e-12)
