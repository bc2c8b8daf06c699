"""lcmx_fues_scan_static: the FUES entry point that allocates nothing.

Callers that cannot call cudaMalloc on this path -- code running inside
another runtime's execution, such as an XLA FFI custom-call handler, where an
allocation would synchronise the device and bypass that runtime's allocator --
use this entry point; its scratch is a fixed 8 MiB device array inside the
library.  Only rows longer than 4096 candidates use that array (shorter rows
are sorted in shared memory), so the scratch cases here run rows of 5000 and
of 8192 candidates (32 rows of 8192 fill the 8 MiB exactly).

The test calls the entry point through the C ABI (ctypes, device pointers
from torch) and checks its output against the workspace-taking lcmx_fues_scan
on the same rows and against the FUES oracle, within the tolerance of the
other FUES tests, on calls made back to back (the array keeps the previous
call's contents).  It is collected last so that a run stopping at the first
failure has run every other test already; it does not depend on them and also
passes alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest

from oracle.fues import refine

pytestmark = pytest.mark.gpu


def _rows(n_rows, n, seed):
    """Two interleaved concave branches with a jump in savings (a discrete-choice
    kink), shuffled, with a few absent (NaN) candidates."""
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
        drop = rng.random(n) < 0.01
        g = np.where(drop, np.nan, g)
        v = np.where(drop, np.nan, v)
        G.append(g); C.append(c); V.append(v); S.append(s)
    return [np.ascontiguousarray(x) for x in (np.array(G), np.array(C), np.array(V), np.array(S))]


def _same(a, b):
    """Same NaN pattern; values within 1e-12 (as the other FUES tests)."""
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12, equal_nan=True)


def _run(ctx, kind, dev_rows, n_rows, n, n_out, stream):
    import torch

    lib = ctx.lib
    g, c, v, s = dev_rows
    go, co, vo = (torch.full((n_rows, n_out), -7.0, dtype=torch.float64, device="cuda") for _ in range(3))
    nk = torch.full((n_rows,), -1, dtype=torch.int32, device="cuda")
    if kind == "workspace":
        wb = lib.lcmx_fues_workspace_bytes(n_rows, n)
        ws = torch.empty(wb, dtype=torch.uint8, device="cuda")
        rc = lib.lcmx_fues_scan(ctx.h, g.data_ptr(), c.data_ptr(), v.data_ptr(), s.data_ptr(), n_rows, n, 2.0, 0,
                                go.data_ptr(), co.data_ptr(), vo.data_ptr(), n_out, nk.data_ptr(),
                                ws.data_ptr(), wb, stream)
    else:
        rc = lib.lcmx_fues_scan_static(ctx.h, g.data_ptr(), c.data_ptr(), v.data_ptr(), s.data_ptr(), n_rows, n,
                                       2.0, go.data_ptr(), co.data_ptr(), vo.data_ptr(), n_out, nk.data_ptr(),
                                       stream)
    assert rc == 0, lib.lcmx_last_error(ctx.h)
    torch.cuda.synchronize()
    return go.cpu().numpy(), co.cpu().numpy(), vo.cpu().numpy(), nk.cpu().numpy()


# (rows, candidates per row): the first two use the static array (rows longer
# than 4096 candidates; 32 x 8192 x 4 doubles is exactly the 8 MiB limit), the
# last runs in shared memory.
CALLS = [(16, 5000), (32, 8192), (12, 2020)]


def test_static_entry_point_matches_the_workspace_entry_point_and_the_oracle():
    import torch

    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    lib = ctx.lib
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.lcmx_fues_workspace_bytes(32, 8192) == 8 << 20
    for call, (n_rows, n) in enumerate(CALLS):
        G, C, V, S = _rows(n_rows, n, seed=11 + call)
        dev_rows = [torch.as_tensor(a, dtype=torch.float64, device="cuda") for a in (G, C, V, S)]
        n_out = 2 * n + 2
        ref = _run(ctx, "workspace", dev_rows, n_rows, n, n_out, stream)
        # back to back on the static array: the second call starts from the
        # first one's leftovers and must give the same rows
        for _ in range(2):
            out = _run(ctx, "static", dev_rows, n_rows, n, n_out, stream)
            np.testing.assert_array_equal(out[3], ref[3])
            for a, b in zip(out[:3], ref[:3]):
                _same(a, b)
        for r in (0, n_rows - 1):
            rg, rc, rv, k = refine(G[r], C[r], V[r], S[r], n_out)
            assert out[3][r] == k
            _same(out[0][r], rg)
            _same(out[1][r], rc)
            _same(out[2][r], rv)


def test_static_entry_point_restores_the_callers_device():
    import torch

    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    lib = ctx.lib
    n_rows, n = 2, 4500
    G, C, V, S = _rows(n_rows, n, seed=5)
    dev_rows = [torch.as_tensor(a, dtype=torch.float64, device="cuda") for a in (G, C, V, S)]
    before = torch.cuda.current_device()
    _run(ctx, "static", dev_rows, n_rows, n, 2 * n + 2, torch.cuda.current_stream().cuda_stream)
    assert torch.cuda.current_device() == before


def test_static_entry_point_rejects_calls_beyond_its_scratch():
    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    lib = ctx.lib
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    for n_rows, n in ((1000, 2020), (33, 8192)):
        rc = lib.lcmx_fues_scan_static(ctx.h, dummy, dummy, dummy, dummy, n_rows, n, 2.0, dummy, dummy, dummy,
                                       2 * n, dummy, None)
        assert rc == 1
        assert b"8 MiB" in lib.lcmx_last_error(ctx.h)
