"""Host-side arithmetic of the batch API's per-period result copies: each
(regime, period) copy is n instance rows of n_states entries, strided by the
slot count; emulated here with host memory moves on CPU tensors."""

import ctypes
import types

import numpy as np
import torch

from pylcm_b200.batch import BatchSolver


class _MemmoveCtx:
    """Stands in for the runtime context: performs the strided copy with
    host memory moves (both tensors live in host memory here)."""

    def __init__(self) -> None:
        self.calls = []

    def copy_rows_d2h(self, dst, dst_pitch, src, src_pitch, row_bytes, rows, stream):
        self.calls.append((dst_pitch, src_pitch, row_bytes, rows))
        for r in range(rows):
            ctypes.memmove(dst + r * dst_pitch, src + r * src_pitch, row_bytes)


def _solver(n=3, slots=5, ns=7):
    bs = object.__new__(BatchSolver)
    V = torch.arange(n * slots * ns, dtype=torch.float64).reshape(n, slots, ns)
    P = torch.arange(n * slots * ns, dtype=torch.int32).reshape(n, slots, ns) * 3
    bs.plan = types.SimpleNamespace(V={"alive": V}, pol={"alive": P})
    bs._host_V = {"alive": torch.zeros_like(V)}
    bs._host_pol = {"alive": torch.zeros_like(P)}
    return bs, V, P


def test_one_slot_copy_moves_exactly_that_period_of_every_instance():
    bs, V, P = _solver()
    ctx = _MemmoveCtx()
    spec = types.SimpleNamespace(name="alive")
    nbytes = bs._copy_slot(ctx, spec, 2, True, 0)
    assert nbytes == 3 * 7 * 8 + 3 * 7 * 4
    hv, hp = bs._host_V["alive"], bs._host_pol["alive"]
    assert torch.equal(hv[:, 2], V[:, 2]) and torch.equal(hp[:, 2], P[:, 2])
    others = [k for k in range(5) if k != 2]
    assert not hv[:, others].any() and not hp[:, others].any()
    assert ctx.calls[0] == (5 * 7 * 8, 5 * 7 * 8, 7 * 8, 3)


def test_all_slots_reassemble_the_arrays():
    bs, V, P = _solver()
    ctx = _MemmoveCtx()
    spec = types.SimpleNamespace(name="alive")
    for k in (4, 0, 3, 1, 2):
        bs._copy_slot(ctx, spec, k, False, 0)
    assert torch.equal(bs._host_V["alive"], V)
    assert not bs._host_pol["alive"].any()  # policies only when asked for
    assert np.all([c[3] == 3 for c in ctx.calls])
