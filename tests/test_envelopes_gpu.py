"""The LTM, RFC and MSS envelope kernels (liblcmx.so, through the C ABI) against
the oracle restatements, row by row: bit-identical rows and counts (the
kernels round every step as the oracle does), on the reference's known-answer
cases and on EGM-like candidate rows -- two runs (the constrained and the
Euler branch) that fold back over each other, some dead (NaN) candidates,
lengths 2 .. 4096 -- in the contiguous and the item form."""

import numpy as np
import pytest

from oracle.envelopes import refine_ltm, refine_mss, refine_rfc
from tests.test_envelopes_oracle import _crossing

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _outs(n_rows, n_out):
    import torch

    go = torch.empty((n_rows, n_out), dtype=torch.float64, device="cuda")
    return go, torch.empty_like(go), torch.empty_like(go), torch.empty(n_rows, dtype=torch.int32, device="cuda")


def _host(go, po, vo, nk):
    import torch

    torch.cuda.synchronize()
    return go.cpu().numpy(), po.cpu().numpy(), vo.cpu().numpy(), nk.cpu().numpy()


def _gpu(kind, G, P, V, M, n_out, radius=10, thr=2.0):
    import torch

    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    n_rows, n_in = G.shape
    g, p, v = _dev(G), _dev(P), _dev(V)
    go, po, vo, nk = _outs(n_rows, n_out)
    stream = torch.cuda.current_stream().cuda_stream
    if kind in ("ltm", "mss"):
        fn = ctx.ltm_scan if kind == "ltm" else ctx.mss_scan
        fn(g.data_ptr(), p.data_ptr(), v.data_ptr(), n_rows, n_in, go.data_ptr(), po.data_ptr(),
           vo.data_ptr(), n_out, nk.data_ptr(), stream)
    else:
        m = _dev(M)
        ctx.rfc_scan(g.data_ptr(), p.data_ptr(), v.data_ptr(), m.data_ptr(), n_rows, n_in, radius, thr,
                     go.data_ptr(), po.data_ptr(), vo.data_ptr(), n_out, nk.data_ptr(), stream)
    return _host(go, po, vo, nk)


def _oracle(kind, g, p, v, m, n_out, radius=10, thr=2.0):
    if kind == "ltm":
        return refine_ltm(g, p, v, n_out)
    if kind == "mss":
        return refine_mss(g, p, v, n_out)
    return refine_rfc(g, p, v, m, n_out, search_radius=radius, jump_thresh=thr)


def _rows(n_rows, n, seed):
    """EGM-like rows: a constrained run (c = R, value log c) then an Euler run
    whose endogenous grid folds back (a discrete-choice kink) onto a branch
    that crosses the first, dead entries."""
    rng = np.random.default_rng(seed)
    G, P, V, M = [], [], [], []
    for _ in range(n_rows):
        nc = max(1, n // 5)
        ne = n - nc
        rc = np.sort(rng.uniform(0.05, 1.0, nc))
        a = np.sort(rng.uniform(0.0, 10.0, ne))
        fold = ne // 2
        c = np.where(np.arange(ne) < fold, 0.6 + 0.35 * a, 0.2 + 0.55 * a)
        re_ = a + c - np.where(np.arange(ne) < fold, 0.0, rng.uniform(1.0, 3.0))
        # the folded branch starts below the first and ends above it: the
        # winning branch switches inside the overlap (a crossing)
        ve = np.log(c) + 0.3 * np.sqrt(a + 1.0) + np.where(np.arange(ne) < fold, 0.0, 0.08 * a - 0.4)
        g = np.concatenate([rc, re_])
        pol = np.concatenate([rc, c])
        val = np.concatenate([np.log(rc) - 0.1, ve])
        mu = 1.0 / pol
        dead = rng.random(n) < 0.03
        g = np.where(dead, np.nan, g)
        val = np.where(dead, np.nan, val)
        pol = np.where(dead, np.nan, pol)
        mu = np.where(dead, 0.0, mu)
        G.append(g); P.append(pol); V.append(val); M.append(mu)
    return np.array(G), np.array(P), np.array(V), np.array(M)


def _crossing_rows(n_rows, n, seed):
    """Two overlapping branches on [0, 10], one run each, whose values cross
    (at a random point) between grid points: the MSS crossing insertion."""
    rng = np.random.default_rng(seed)
    G, P, V, M = [], [], [], []
    for _ in range(n_rows):
        na = n // 2
        xa = np.sort(rng.uniform(0.0, 10.0, na))
        xb = np.sort(rng.uniform(0.0, 10.0, n - na))
        s = rng.uniform(0.05, 0.25)
        va = np.log1p(xa) + 0.1 * xa
        vb = np.log1p(xb) + (0.1 + s) * xb - s * rng.uniform(2.0, 8.0)
        g = np.concatenate([xa, xb])
        G.append(g)
        P.append(np.concatenate([0.3 * xa, 0.5 * xb + 0.2]))
        V.append(np.concatenate([va, vb]))
        M.append(np.concatenate([1.0 / (1.0 + xa) + 0.1, 1.0 / (1.0 + xb) + 0.1 + s]))
    return np.array(G), np.array(P), np.array(V), np.array(M)


def _same(got, want):
    for a, b in zip(got[:3], want[:3]):
        np.testing.assert_array_equal(a, b)
    assert got[3] == want[3]


@pytest.mark.parametrize("kind", ["ltm", "rfc", "mss"])
def test_known_answer_cases(kind):
    g, p, v, mu = _crossing()
    thr = 0.6 if kind == "rfc" else 2.0
    got = _gpu(kind, g[None], p[None], v[None], mu[None], 12, thr=thr)
    _same([x[0] for x in got], _oracle(kind, g, p, v, mu, 12, thr=thr))
    got = _gpu(kind, g[None], p[None], v[None], mu[None], 4, thr=thr)  # overflow: a truncated prefix
    _same([x[0] for x in got], _oracle(kind, g, p, v, mu, 4, thr=thr))
    lg = np.array([[1.0, 3.0, 2.0, 4.0]])
    got = _gpu(kind, lg, lg * 0.5, np.array([[1.0, 2.0, 5.0, 7.0]]), np.full((1, 4), 0.5), 8)
    _same([x[0] for x in got], _oracle(kind, lg[0], lg[0] * 0.5, [1.0, 2.0, 5.0, 7.0], [0.5] * 4, 8))


@pytest.mark.parametrize("kind", ["ltm", "rfc", "mss"])
@pytest.mark.parametrize("n", [2, 37, 300, 2020, 4096])
def test_rows_match_the_oracle(kind, n):
    G, P, V, M = _rows(5 if n < 4096 else 2, n, seed=n)
    n_out = 2 * n + 3
    got = _gpu(kind, G, P, V, M, n_out)
    for r in range(G.shape[0]):
        _same([x[r] for x in got], _oracle(kind, G[r], P[r], V[r], M[r], n_out))


@pytest.mark.parametrize("kind", ["ltm", "rfc", "mss"])
def test_crossing_branches_match_the_oracle(kind):
    G, P, V, M = _crossing_rows(6, 900, seed=5)
    got = _gpu(kind, G, P, V, M, 1900)
    for r in range(G.shape[0]):
        want = _oracle(kind, G[r], P[r], V[r], M[r], 1900)
        _same([x[r] for x in got], want)
        if kind == "mss":
            assert want[3] > _oracle("ltm", G[r], P[r], V[r], M[r], 1900)[3]  # crossings were inserted


def test_rfc_radius_and_threshold():
    G, P, V, M = _rows(4, 500, seed=3)
    for radius, thr in ((1, 2.0), (3, 0.5), (40, 5.0)):
        got = _gpu("rfc", G, P, V, M, 600, radius=radius, thr=thr)
        for r in range(4):
            _same([x[r] for x in got], _oracle("rfc", G[r], P[r], V[r], M[r], 600, radius=radius, thr=thr))


@pytest.mark.parametrize("kind", ["ltm", "rfc", "mss"])
def test_item_form_equals_the_contiguous_form(kind):
    """Two candidate blocks of different row lengths in one launch."""
    import torch

    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    blocks = [_rows(3, 150, seed=11), _rows(5, 700, seed=12)]
    keep, recs, prefix = [], [], [0]
    for G, P, V, M in blocks:
        n_rows, n_in = G.shape
        n_out = 2 * n_in + 5
        ins = [_dev(x) for x in (G, P, V, M)]
        outs = _outs(n_rows, n_out)
        keep.append((ins, outs, n_out))
        thr = np.float64(2.0).view(np.int64)
        recs.append([ins[0].data_ptr(), ins[1].data_ptr(), ins[2].data_ptr(),
                     ins[3].data_ptr() if kind == "rfc" else 0,
                     outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), outs[3].data_ptr(),
                     n_rows, n_in, n_out, int(thr), 10])
        prefix.append(prefix[-1] + n_rows)
    items = torch.as_tensor(np.array(recs, dtype=np.int64), device="cuda")
    pre = torch.as_tensor(np.array(prefix, dtype=np.int32), device="cuda")
    ctx.envelope_step({"ltm": 1, "rfc": 2, "mss": 3}[kind], items.data_ptr(), pre.data_ptr(), len(blocks),
                      prefix[-1], 700, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for (G, P, V, M), (_, outs, n_out) in zip(blocks, keep):
        got = _host(*outs)
        for r in range(G.shape[0]):
            _same([x[r] for x in got], _oracle(kind, G[r], P[r], V[r], M[r], n_out))


def test_rejects_bad_sizes():
    import torch

    from pylcm_b200.runtime import KernelError, get_context

    ctx = get_context(0)
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    nk = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(KernelError):
        ctx.ltm_scan(x.data_ptr(), x.data_ptr(), x.data_ptr(), 1, 5000, x.data_ptr(), x.data_ptr(), x.data_ptr(),
                     4, nk.data_ptr(), 0)
    with pytest.raises(KernelError):
        ctx.rfc_scan(x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(), 1, 4, 0, 2.0, x.data_ptr(),
                     x.data_ptr(), x.data_ptr(), 4, nk.data_ptr(), 0)
