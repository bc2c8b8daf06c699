"""Oracle: the FUES upper envelope, one row at a time (test infrastructure only).

Restates the Fast Upper-Envelope Scan (Dobrescu & Shanker 2022) as the
reference implements it in ``src/_lcm/egm/upper_envelope/fues.py``:

- sort by (grid ascending, value descending, policy descending), NaN last
  (``fues.py:230-235``);
- reduce coincident-abscissa groups to their maximisers, collapsing
  maximisers that share an exogenous savings source (``fues.py:341-424``);
- a sequential scan keeping the last two envelope points k, j
  (``_inspect_candidate``, ``fues.py:640-968``): a candidate i is dropped when
  it is below j on the same segment, when savings decrease and the secant is
  below the previous gradient, or when it lies below the continuation of j's
  segment; segment crossings insert their intersection twice (left / right
  policy), strictly between j and i (``kink_5``), before j (``kink_6``), or
  snapped onto a node;
- the segment test is a jump of |dA/dR| of the implied savings A = R - c above
  ``jump_thresh`` (``_has_policy_jump``, ``fues.py:1082-1131``), the
  same-segment look-ahead is exhaustive by default and bounded to
  ``n_points_to_scan`` positions when given (``fues.py:114-128, 1016-1079``).

Outputs are NaN-padded rows of length `n_refined` plus the kept count
(> n_refined signals overflow).
"""

from __future__ import annotations

import math

import numpy as np

EPS = np.finfo(np.float64).eps


def _slope(xa, ya, xb, yb):
    dx = xb - xa
    return 0.0 if dx == 0.0 else (yb - ya) / dx


def _jump(ga, pa, gb, pb, thr, sa=None, sb=None):
    ia, ib = ga - pa, gb - pb
    if ga == gb:
        return (sa != sb) if (sa is not None and sb is not None) else (ia != ib)
    return abs(_slope(ga, ia, gb, ib)) > thr


def _intersect(xa, ya, sa, xb, yb, sb):
    den = sa - sb
    if den == 0.0:
        return math.nan, ya
    x = (yb - ya + sa * xa - sb * xb) / den
    return x, ya + sa * (x - xa)


def _find_same_segment(g, p, v, anchor_g, anchor_p, idx, direction, thr, window=None):
    """First candidate on the anchor's segment among positions idx + direction,
    ..., idx + direction * window (``_find_same_segment_point``,
    ``fues.py:1016-1079``; window None: every position, ``:114-128``)."""
    n = len(g)
    k = idx + direction
    while 0 <= k < n and (window is None or abs(k - idx) <= window):
        if not (math.isnan(g[k]) or math.isnan(v[k])) and not _jump(anchor_g, anchor_p, g[k], p[k], thr):
            return True, g[k], p[k], v[k]
        k += direction
    return False, math.nan, math.nan, math.nan


def sort_and_reduce(grid, policy, value, savings):
    grid = np.asarray(grid, float)
    policy = np.asarray(policy, float)
    value = np.asarray(value, float)
    savings = np.asarray(savings, float)
    gk = np.where(np.isnan(grid), np.inf, grid)
    vk = np.where(np.isnan(value), -np.inf, value)
    pk = np.where(np.isnan(policy), -np.inf, policy)
    order = np.lexsort((-pk, -vk, gk))
    g, p, v, s = grid[order].copy(), policy[order].copy(), value[order].copy(), savings[order].copy()
    n = len(g)
    fin = ~np.isnan(g)
    i = 0
    while i < n:
        if not fin[i]:
            i += 1
            continue
        j = i
        while j + 1 < n and fin[j + 1] and g[j + 1] == g[i]:
            j += 1
        grp = range(i, j + 1)
        vmax = max((v[k] if not math.isnan(v[k]) else -math.inf) for k in grp)
        seen = []
        for k in grp:
            keep = (v[k] == vmax)
            if keep and any(s[k] == s2 for s2 in seen):
                keep = False
            if keep:
                seen.append(s[k])
            else:
                g[k] = p[k] = v[k] = s[k] = math.nan
        i = j + 1
    return g, p, v, s


def refine(grid, policy, value, savings, n_refined: int, jump_thresh: float = 2.0, n_points_to_scan=None):
    """Refined (grid, policy, value) NaN-padded to n_refined, and n_kept.
    `n_points_to_scan` bounds the same-segment look-ahead (None: exhaustive)."""
    w = n_points_to_scan
    g, p, v, s = sort_and_reduce(grid, policy, value, savings)
    n = len(g)
    thr = jump_thresh
    out_g, out_p, out_v = [], [], []
    gk, pk, vk = g[0], p[0], v[0]
    gj, pj, vj, sj = g[0], p[0], v[0], s[0]
    near = 16.0 * EPS
    for idx in range(1, n):
        gi, pi, vi, si = g[idx], p[idx], v[idx], s[idx]
        valid = not (math.isnan(gi) or math.isnan(vi))
        switches = _jump(gj, pj, gi, pi, thr, sj, si) if valid else False
        node_crossing = valid and switches and gi == gj and vi == vj
        secant = _slope(gj, vj, gi, vi)
        grad_before = _slope(gk, vk, gj, vj)
        jf, jg, jp, jv = _find_same_segment(g, p, v, gj, pj, idx, 1, thr, w)
        if switches and jf:
            below_j = (vi < jv) if gi == jg else (secant < _slope(gi, vi, jg, jv))
        else:
            below_j = False
        sav_dec = si < sj
        dropped = (not valid) or ((vi < vj) and not switches) or (sav_dec and secant < grad_before) or below_j
        dropped = dropped and not node_crossing
        if dropped:
            continue
        ff, fg, fp, fv = _find_same_segment(g, p, v, gi, pi, idx, 1, thr, w)
        bf, bg, bp, bv = _find_same_segment(g, p, v, gi, pi, idx, -1, thr, w)
        found = ff or bf
        pg, pp, pv = (fg, fp, fv) if ff else (bg, bp, bv)
        i_slope = _slope(gi, vi, pg, pv)
        i_pslope = _slope(gi, pi, pg, pp)
        j_dom = switches and found and (secant > i_slope) and not node_crossing
        pslope_kj = _slope(gk, pk, gj, pj)
        k6g, k6v = _intersect(gj, vj, grad_before, gi, vi, i_slope)
        k6pl = pj + pslope_kj * (k6g - gj)
        k6pr = pi + i_pslope * (k6g - gi)
        kink6 = j_dom and (k6g > gk) and (k6g < gj) and (k6g < gi)
        j_slope = _slope(gj, vj, jg, jv) if jf else grad_before
        j_pslope = _slope(gj, pj, jg, jp) if jf else pslope_kj
        k5g, k5v = _intersect(gj, vj, j_slope, gi, vi, i_slope)
        k5pl = pj + j_pslope * (k5g - gj)
        k5pr = pi + i_pslope * (k5g - gi)
        crossing = (not j_dom) and (not node_crossing) and switches and found
        tol = near * max(abs(gj), abs(gi), 1.0)
        on_j = crossing and abs(k5g - gj) <= tol
        on_i = crossing and not on_j and abs(k5g - gi) <= tol
        kink5 = crossing and not on_j and not on_i and (k5g > gj) and (k5g < gi)
        plain = not j_dom and not kink5 and not on_j and not on_i
        # emissions (ascending grid)
        if kink6:
            out_g += [k6g, k6g]
            out_p += [k6pl, k6pr]
            out_v += [k6v, k6v]
        elif plain or kink5 or on_j or on_i:
            out_g.append(gj)
            out_p.append(pj)
            out_v.append(vj)
            if kink5:
                out_g += [k5g, k5g]
                out_p += [k5pl, k5pr]
                out_v += [k5v, k5v]
            elif on_j:
                out_g.append(gj)
                out_p.append(k5pr)
                out_v.append(k5v)
            elif on_i:
                out_g.append(gi)
                out_p.append(k5pl)
                out_v.append(k5v)
        # carry update
        keeps_k = j_dom and not kink6
        if not keeps_k:
            if kink5:
                gk, pk, vk = k5g, k5pr, k5v
            elif kink6:
                gk, pk, vk = k6g, k6pr, k6v
            else:
                gk = gj
                pk = k5pr if on_j else pj
                vk = k5v if on_j else vj
        gj, pj, vj, sj = gi, pi, vi, si
    if not (math.isnan(gj) or math.isnan(vj)):
        out_g.append(gj)
        out_p.append(pj)
        out_v.append(vj)
    n_kept = len(out_g)
    rg = np.full(n_refined, np.nan)
    rp = np.full(n_refined, np.nan)
    rv = np.full(n_refined, np.nan)
    m = min(n_kept, n_refined)
    rg[:m], rp[:m], rv[:m] = out_g[:m], out_p[:m], out_v[:m]
    return rg, rp, rv, n_kept
