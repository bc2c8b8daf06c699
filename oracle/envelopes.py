"""Oracle: the LTM and RFC upper envelopes, one row at a time (test
infrastructure only).

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


def _publish(gs, ps, vs, n_refined):
    out = np.full((3, n_refined), np.nan)
    m = min(len(gs), n_refined)
    out[0, :m], out[1, :m], out[2, :m] = gs[:m], ps[:m], vs[:m]
    return out[0], out[1], out[2], len(gs)
