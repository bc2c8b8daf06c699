"""FUES kernel (liblcmx.so) vs the oracle restatement, row by row."""

import numpy as np
import pytest

from oracle.fues import refine
from tests.test_fues_oracle import _crossing

pytestmark = pytest.mark.gpu


def _gpu_fues(rows_g, rows_c, rows_v, rows_s, n_out, thr=2.0, window=0):
    import torch

    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    n_rows, n_in = rows_g.shape
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    g, c, v, s = d(rows_g), d(rows_c), d(rows_v), d(rows_s)
    go = torch.empty((n_rows, n_out), dtype=torch.float64, device="cuda")
    co = torch.empty_like(go)
    vo = torch.empty_like(go)
    nk = torch.empty(n_rows, dtype=torch.int32, device="cuda")
    wb = ctx.fues_workspace_bytes(n_rows, n_in)
    ws = torch.empty(wb, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    ctx.fues_scan(g.data_ptr(), c.data_ptr(), v.data_ptr(), s.data_ptr(), n_rows, n_in, thr,
                  go.data_ptr(), co.data_ptr(), vo.data_ptr(), n_out, nk.data_ptr(), ws.data_ptr(), wb, stream,
                  n_points_to_scan=window)
    torch.cuda.synchronize()
    return go.cpu().numpy(), co.cpu().numpy(), vo.cpu().numpy(), nk.cpu().numpy()


def _same(a, b):
    """Same NaN pattern; values within 1e-12 (inserted crossings may differ by
    an ulp: fused multiply-add on the GPU)."""
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12, equal_nan=True)


def _rows_nonconcave(n_rows, n, seed):
    """Two interleaved concave branches with a jump in savings (a discrete-choice
    kink), shuffled, with a few NaN (absent) candidates."""
    rng = np.random.default_rng(seed)
    G, C, V, S = [], [], [], []
    for _ in range(n_rows):
        a = np.sort(rng.uniform(0, 10, n))
        half = n // 2
        c = np.where(np.arange(n) < half, 0.5 + 0.3 * a, 1.5 + 0.6 * a)
        shift = np.where(np.arange(n) < half, 0.0, rng.uniform(0.5, 2.0))
        g = a + c
        v = np.log(c) + 0.2 * np.sqrt(a + 1) + shift - 0.15 * np.arange(n) / n
        perm = rng.permutation(n)
        g, c, v, s = g[perm], c[perm], v[perm], a[perm]
        drop = rng.random(n) < 0.02
        g = np.where(drop, np.nan, g)
        v = np.where(drop, np.nan, v)
        G.append(g); C.append(c); V.append(v); S.append(s)
    return np.array(G), np.array(C), np.array(V), np.array(S)


def test_fues_kernel_matches_oracle_on_analytic_crossing():
    g, c, v = _crossing()
    go, co, vo, nk = _gpu_fues(g[None], c[None], v[None], (g - c)[None], 12)
    rg, rc, rv, n = refine(g, c, v, g - c, 12)
    assert nk[0] == n
    _same(go[0], rg)
    _same(co[0], rc)
    _same(vo[0], rv)


@pytest.mark.parametrize("n", [17, 300, 2020])
def test_fues_kernel_matches_oracle_on_nonconcave_rows(n):
    G, C, V, S = _rows_nonconcave(6, n, seed=n)
    n_out = 2 * n + 2
    go, co, vo, nk = _gpu_fues(G, C, V, S, n_out)
    for r in range(G.shape[0]):
        rg, rc, rv, k = refine(G[r], C[r], V[r], S[r], n_out)
        assert nk[r] == k
        _same(go[r], rg)
        _same(co[r], rc)
        _same(vo[r], rv)


def test_fues_kernel_reports_overflow():
    G, C, V, S = _rows_nonconcave(2, 64, seed=3)
    go, co, vo, nk = _gpu_fues(G, C, V, S, 4)
    assert np.all(nk > 4)
    assert np.all(np.isfinite(go[:, :4]))


def test_shared_memory_and_global_kernels_give_identical_rows():
    """Rows of 3000 candidates take the shared-memory kernel; the same rows
    padded with absent (NaN) candidates to 5000 take the global-workspace
    kernel.  NaN candidates sort last and are dropped, so the rows must be
    bit-identical."""
    G, C, V, S = _rows_nonconcave(5, 3000, seed=11)
    pad = lambda a: np.concatenate([a, np.full((a.shape[0], 2000), np.nan)], axis=1)  # noqa: E731
    a = _gpu_fues(G, C, V, S, 6100)
    b = _gpu_fues(pad(G), pad(C), pad(V), pad(S), 6100)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_item_form_matches_the_contiguous_form():
    """lcmx_fues_step over several candidate blocks (different row counts,
    row lengths and thresholds) gives each block's lcmx_fues_scan rows."""
    import torch

    from pylcm_b200.engine import _f2w
    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    blocks = [(4, 2020, 2.0, 1), (1, 300, 1.5, 2), (7, 777, 2.5, 3)]
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    keep, words, tiles = [], [], []
    for n_rows, n_in, thr, seed in blocks:
        G, C, V, S = _rows_nonconcave(n_rows, n_in, seed=seed)
        n_out = 2 * n_in + 2
        ins = [d(G), d(C), d(V), d(S)]
        outs = [torch.full((n_rows, n_out), 7.0, dtype=torch.float64, device="cuda") for _ in range(3)]
        nk = torch.zeros(n_rows, dtype=torch.int32, device="cuda")
        w = [t.data_ptr() for t in ins] + [t.data_ptr() for t in outs] + [nk.data_ptr(), n_rows, n_in, n_out, _f2w(thr),
                                                                            0]
        words.append(np.array(w, dtype=np.int64))
        tiles.append(n_rows)
        keep.append((G, C, V, S, n_out, thr, ins, outs, nk))
    items = torch.as_tensor(np.concatenate(words), dtype=torch.int64, device="cuda")
    prefix = torch.as_tensor(np.concatenate([[0], np.cumsum(tiles)]).astype(np.int32), device="cuda")
    ctx.fues_step(items.data_ptr(), prefix.data_ptr(), len(blocks), int(sum(tiles)), max(b[1] for b in blocks),
                  torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for G, C, V, S, n_out, thr, ins, outs, nk in keep:
        go, co, vo, k = _gpu_fues(G, C, V, S, n_out, thr)
        np.testing.assert_array_equal(outs[0].cpu().numpy(), go)
        np.testing.assert_array_equal(outs[1].cpu().numpy(), co)
        np.testing.assert_array_equal(outs[2].cpu().numpy(), vo)
        np.testing.assert_array_equal(nk.cpu().numpy(), k)


@pytest.mark.parametrize("n", [300, 5000])
@pytest.mark.parametrize("window", [2, 7, 40])
def test_bounded_look_ahead_matches_the_oracle(n, window):
    """FUESEnvelope(n_points_to_scan=k): the same-segment look-ahead inspects
    k positions on either side (fues.py:1016-1079), on the shared-memory
    (300) and the global-workspace (5000 candidates) kernels."""
    G, C, V, S = _rows_nonconcave(4, n, seed=n + window)
    n_out = 2 * n + 2
    go, co, vo, nk = _gpu_fues(G, C, V, S, n_out, window=window)
    for r in range(G.shape[0]):
        rg, rc, rv, k = refine(G[r], C[r], V[r], S[r], n_out, n_points_to_scan=window)
        assert nk[r] == k
        _same(go[r], rg)
        _same(co[r], rc)
        _same(vo[r], rv)


def test_item_form_honours_the_window_word():
    import torch

    from pylcm_b200.engine import _f2w
    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    n_rows, n_in, window = 3, 500, 3
    G, C, V, S = _rows_nonconcave(n_rows, n_in, seed=21)
    n_out = 2 * n_in + 2
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    ins = [d(G), d(C), d(V), d(S)]
    outs = [torch.full((n_rows, n_out), 7.0, dtype=torch.float64, device="cuda") for _ in range(3)]
    nk = torch.zeros(n_rows, dtype=torch.int32, device="cuda")
    w = [t.data_ptr() for t in ins] + [t.data_ptr() for t in outs] + [nk.data_ptr(), n_rows, n_in, n_out, _f2w(2.0),
                                                                        window]
    items = torch.as_tensor(np.array(w, dtype=np.int64), device="cuda")
    prefix = torch.as_tensor(np.array([0, n_rows], dtype=np.int32), device="cuda")
    ctx.fues_step(items.data_ptr(), prefix.data_ptr(), 1, n_rows, n_in, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    go, co, vo, k = _gpu_fues(G, C, V, S, n_out, window=window)
    np.testing.assert_array_equal(outs[0].cpu().numpy(), go)
    np.testing.assert_array_equal(outs[2].cpu().numpy(), vo)
    np.testing.assert_array_equal(nk.cpu().numpy(), k)
