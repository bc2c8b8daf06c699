"""Oracle: the LTM, RFC and MSS upper envelopes, one row at a time (test
infrastructure only; MSS is documented at `refine_mss`).

LTM, the local-upper-bound brute method, as the reference implements it in
``src/_lcm/egm/upper_envelope/ltm.py``:

- a candidate is dead when its grid point or value is NaN (``ltm.py:86``);
- the query abscissae are the candidate grid points sorted ascending, ties in
  input order, dead ones last (``ltm.py:90-93``);
- the segments join consecutive candidates in input order; a segment with a
  dead end is skipped (``ltm.py:156-168``);
- a segment brackets a query q when min(g_k, g_k+1) <= q <= max(g_k, g_k+1);
  the value and policy are interpolated linearly along it, with weight 0 on a
  zero-width segment (``ltm.py:170-181``);
- the envelope at q is the largest bracketing value, its policy that of the
  first segment reaching it (a NaN interpolant wins, as a NaN-propagating
  maximum has it); a query that no segment brackets, or whose value is -inf,
  is dropped (``ltm.py:183-190, 100-105``);
- the survivors are published in query order, NaN-padded to `n_refined`, with
  their count (> n_refined: overflow, a truncated prefix) (``ltm.py:107-121``).

RFC, the rooftop cut of Dobrescu and Shanker (2024), as in
``src/_lcm/egm/upper_envelope/rfc.py``:

- the candidates are sorted ascending by grid point, ties in input order, NaN
  last (``rfc.py:84-88``);
- a dead candidate (NaN grid point or value) enters the test with value -inf,
  grid point +inf and slope 0 (``rfc.py:94-97``);
- candidate l is deleted when some j within `search_radius` sorted positions
  has l strictly below j's tangent line, v_l - v_j < mu_j (R_l - R_j) - 16 eps
  max(|v_l - v_j|, |mu_j (R_l - R_j)|), across a policy jump |dc/dR| >
  `jump_thresh` (zero-width pairs carry no jump) (``rfc.py:124-220``);
- the survivors (live, not deleted) are published in sorted order as LTM's
  (``rfc.py:107-121``).
"""

from __future__ import annotations

import numpy as np

EPS = np.finfo(np.float64).eps


def refine_ltm(grid, policy, value, n_refined: int):
    """(grid, policy, value) rows of length n_refined (NaN-padded) and the
    kept count, of one candidate row."""
    g = np.asarray(grid, dtype=np.float64)
    p = np.asarray(policy, dtype=np.float64)
    v = np.asarray(value, dtype=np.float64)
    n = g.size
    dead = np.isnan(g) | np.isnan(v)
    key = np.where(dead, np.inf, g)
    order = np.argsort(key, kind="stable")
    live_seg = ~dead[:-1] & ~dead[1:] if n > 1 else np.zeros(0, dtype=bool)
    gl, gr, vl, vr, pl, pr = g[:-1], g[1:], v[:-1], v[1:], p[:-1], p[1:]
    lo, hi = np.minimum(gl, gr), np.maximum(gl, gr)
    w = gr - gl
    out_g, out_p, out_v = [], [], []
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        for i in order:
            if dead[i]:
                continue
            q = g[i]
            br = live_seg & (q >= lo) & (q <= hi)
            if not br.any():
                continue
            rel = np.where(w == 0.0, 0.0, (q - gl) / np.where(w == 0.0, 1.0, w))
            vi = np.where(br, vl + rel * (vr - vl), -np.inf)
            pi = pl + rel * (pr - pl)
            nan = np.isnan(vi)
            k = int(np.argmax(nan)) if nan.any() else int(np.argmax(vi))  # the first maximum
            if vi[k] == -np.inf:
                continue
            out_g.append(q)
            out_p.append(pi[k])
            out_v.append(vi[k])
    return _publish(out_g, out_p, out_v, n_refined)


def refine_rfc(grid, policy, value, marginal_utility, n_refined: int, search_radius: int = 10,
               jump_thresh: float = 2.0):
    """(grid, policy, value) rows of length n_refined (NaN-padded) and the
    kept count, of one candidate row."""
    g0 = np.asarray(grid, dtype=np.float64)
    order = np.argsort(g0, kind="stable")  # NaN last, after +inf
    g = g0[order]
    p = np.asarray(policy, dtype=np.float64)[order]
    v = np.asarray(value, dtype=np.float64)[order]
    mu = np.asarray(marginal_utility, dtype=np.float64)[order]
    n = g.size
    dead = np.isnan(g) | np.isnan(v)
    vt = np.where(dead, -np.inf, v)
    gt = np.where(dead, np.inf, g)
    mt = np.where(dead, 0.0, mu)
    keep = []
    with np.errstate(invalid="ignore", over="ignore"):
        for l_ in range(n):
            if dead[l_]:
                continue
            deleted = False
            for o in range(-search_radius, search_radius + 1):
                j = l_ + o
                if o == 0 or j < 0 or j >= n:
                    continue
                dg = gt[l_] - gt[j]
                gap = vt[l_] - vt[j]
                tan = mt[j] * dg
                floor = 16.0 * EPS * max(abs(gap), abs(tan))
                below = gap < tan - floor
                slope = 0.0 if dg == 0.0 else (p[l_] - p[j]) / dg
                if below and abs(slope) > jump_thresh:
                    deleted = True
                    break
            if not deleted:
                keep.append(l_)
    return _publish([g[i] for i in keep], [p[i] for i in keep], [v[i] for i in keep], n_refined)


def _mss_links(g, v, dead):
    """Per link k (candidates k, k+1 in input order): live flag and branch id
    (HARK's monotone split: a link across a grid decrease, or a value decrease
    past 16 eps max(|v_k|, |v_k+1|), starts a new branch and is not live)
    (``mss.py:153-171, 549-570``)."""
    gl, gr, vl, vr = g[:-1], g[1:], v[:-1], v[1:]
    with np.errstate(invalid="ignore"):
        floor = 16.0 * EPS * np.maximum(np.abs(vl), np.abs(vr))
        dec = (gr < gl) | (vr < vl - floor)
    seg = np.cumsum(dec.astype(np.int64))
    live = ~dead[:-1] & ~dead[1:] & ~dec
    return live, seg


def _mss_eval(q, g, p, v, live, seg):
    """(envelope value, policy, winning link, winning branch) at abscissa q:
    the largest finite interpolant over the live links bracketing q; the
    winner is the first link within 16 eps max(1, |max|) of it; no bracketing
    link: (-inf, NaN, 0, -1) (``mss.py:478-547``)."""
    gl, gr, vl, vr, pl, pr = g[:-1], g[1:], v[:-1], v[1:], p[:-1], p[1:]
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        br = live & (q >= np.minimum(gl, gr)) & (q <= np.maximum(gl, gr))
        w = gr - gl
        rel = np.where(w == 0.0, 0.0, (q - gl) / np.where(w == 0.0, 1.0, w))
        vi = vl + rel * (vr - vl)
        pi = pl + rel * (pr - pl)
        masked = np.where(br & np.isfinite(vi), vi, -np.inf)
        env = masked.max() if masked.size else -np.inf
        floor = 16.0 * EPS * max(1.0, abs(env))
        tie = br & (masked >= env - floor)
    if not br.any():
        return env, np.nan, 0, -1
    k = int(np.argmax(tie))
    return env, pi[k], k, int(seg[k])


def _line_slope(xa, ya, xb, yb):
    dx = xb - xa
    return 0.0 if dx == 0.0 else (yb - ya) / dx


def refine_mss(grid, policy, value, n_refined: int):
    """MSS (HARK's EGM upper envelope) as the reference implements it in
    ``src/_lcm/egm/upper_envelope/mss.py:72-310``: the LTM evaluation at the
    sorted live abscissae over the live monotone links (finite interpolants
    only), plus, where the winning branch changes between two consecutive
    live queries, the crossing of the two winning links' value lines --
    inserted twice (left, right policy) when it falls strictly between them
    and the envelope there matches it (finite, within 1e-7 + 1e-5 |value|)."""
    g = np.asarray(grid, dtype=np.float64)
    p = np.asarray(policy, dtype=np.float64)
    v = np.asarray(value, dtype=np.float64)
    n = g.size
    dead = np.isnan(g) | np.isnan(v)
    order = np.argsort(np.where(dead, np.inf, g), kind="stable")
    if n > 1:
        live, seg = _mss_links(g, v, dead)
    else:
        live, seg = np.zeros(0, dtype=bool), np.zeros(0, dtype=np.int64)
    atol = max(1e-7, 8.0 * EPS)
    rows = []
    prev_link, prev_seg, prev_grid = 0, -1, -np.inf
    for i in order:
        q = np.nan if dead[i] else g[i]
        env, pol, link, sg = _mss_eval(q, g, p, v, live, seg) if not dead[i] else (-np.inf, np.nan, 0, -1)
        node_live = (not dead[i]) and env != -np.inf
        if node_live and prev_seg >= 0 and sg != prev_seg:
            a, b = prev_link, link
            sa = _line_slope(g[a], v[a], g[a + 1], v[a + 1])
            sb = _line_slope(g[b], v[b], g[b + 1], v[b + 1])
            den = sa - sb
            with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
                if den == 0.0:
                    x, y = np.nan, v[a]
                else:
                    x = (v[b] - v[a] + sa * g[a] - sb * g[b]) / den
                    y = v[a] + sa * (x - g[a])
                psa = _line_slope(g[a], p[a], g[a + 1], p[a + 1])
                psb = _line_slope(g[b], p[b], g[b + 1], p[b + 1])
                pa = p[a] + psa * (x - g[a])
                pb = p[b] + psb * (x - g[b])
            if x > prev_grid and x < q:
                ce = _mss_eval(x, g, p, v, live, seg)[0]
                if np.isfinite(ce) and np.isfinite(y) and abs(ce - y) <= atol + 1e-5 * abs(y):
                    rows += [(x, pa, y), (x, pb, y)]
        if node_live:
            rows.append((q, pol, env))
            prev_link, prev_seg, prev_grid = link, sg, q
    return _publish([r[0] for r in rows], [r[1] for r in rows], [r[2] for r in rows], n_refined)


def _publish(gs, ps, vs, n_refined):
    out = np.full((3, n_refined), np.nan)
    m = min(len(gs), n_refined)
    out[0, :m], out[1, :m], out[2, :m] = gs[:m], ps[:m], vs[:m]
    return out[0], out[1], out[2], len(gs)
