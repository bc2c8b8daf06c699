"""lcmx_fues_scan_static: the FUES entry point that allocates nothing.

Callers that cannot call cudaMalloc on this path -- code running inside
another runtime's execution, such as an XLA FFI custom-call handler -- use this
entry point; its scratch is a fixed 8 MiB device array inside the library.
The test calls it through the C ABI (ctypes, device pointers from torch) and
checks its output against the workspace-taking lcmx_fues_scan on the same rows,
within the tolerance of the other FUES tests, on two calls in a row (the
array keeps the previous call's contents).  It is collected last so that a
run stopping at the first failure has run every other test already; it does
not depend on them and also passes alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(n_rows, n, seed):
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
        G.append(g[perm]); C.append(c[perm]); V.append(v[perm]); S.append(a[perm])
    return [np.ascontiguousarray(x) for x in (np.array(G), np.array(C), np.array(V), np.array(S))]


def _same(a, b):
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12, equal_nan=True)


def test_static_entry_point_matches_the_workspace_entry_point_twice():
    import torch

    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    lib = ctx.lib
    stream = torch.cuda.current_stream().cuda_stream
    for call, (n_rows, n) in enumerate([(12, 2020), (40, 300)]):
        G, C, V, S = _rows(n_rows, n, seed=11 + call)
        d = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
        g, c, v, s = d(G), d(C), d(V), d(S)
        n_out = 2 * n + 2
        outs = []
        for _ in range(2):  # the reference entry point and the static one
            outs.append([torch.empty((n_rows, n_out), dtype=torch.float64, device="cuda") for _ in range(3)]
                        + [torch.empty(n_rows, dtype=torch.int32, device="cuda")])
        wb = lib.lcmx_fues_workspace_bytes(n_rows, n)
        ws = torch.empty(wb, dtype=torch.uint8, device="cuda")
        go, co, vo, nk = outs[0]
        rc = lib.lcmx_fues_scan(ctx.h, g.data_ptr(), c.data_ptr(), v.data_ptr(), s.data_ptr(), n_rows, n, 2.0,
                                go.data_ptr(), co.data_ptr(), vo.data_ptr(), n_out, nk.data_ptr(),
                                ws.data_ptr(), wb, stream)
        assert rc == 0, lib.lcmx_last_error(ctx.h)
        go2, co2, vo2, nk2 = outs[1]
        rc = lib.lcmx_fues_scan_static(ctx.h, g.data_ptr(), c.data_ptr(), v.data_ptr(), s.data_ptr(), n_rows, n,
                                       2.0, go2.data_ptr(), co2.data_ptr(), vo2.data_ptr(), n_out, nk2.data_ptr(),
                                       stream)
        assert rc == 0, lib.lcmx_last_error(ctx.h)
        torch.cuda.synchronize()
        assert torch.equal(nk.cpu(), nk2.cpu())
        for a, b in ((go, go2), (co, co2), (vo, vo2)):
            _same(b.cpu().numpy(), a.cpu().numpy())


def test_static_entry_point_rejects_calls_beyond_its_scratch():
    from pylcm_b200.runtime import get_context

    ctx = get_context(0)
    lib = ctx.lib
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.lcmx_fues_scan_static(ctx.h, dummy, dummy, dummy, dummy, 1000, 2020, 2.0, dummy, dummy, dummy,
                                   4040, dummy, None)
    assert rc == 1
    assert b"8 MiB" in lib.lcmx_last_error(ctx.h)
