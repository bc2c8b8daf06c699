"""ctypes binding of liblcmx.so (the C ABI in include/lcmx.h).

The library is built in-tree (``pylcm_b200/_lib/liblcmx.so``).  There is no
fallback: if the library or a GPU is missing, solving raises.
"""

from __future__ import annotations

import ctypes
import threading
from collections.abc import Callable
from pathlib import Path

from pylcm_b200.exceptions import KernelError

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "liblcmx.so"

EXPORTED = (
    "lcmx_ctx_create",
    "lcmx_ctx_destroy",
    "lcmx_last_error",
    "lcmx_device_info",
    "lcmx_module_compile",
    "lcmx_module_destroy",
    "lcmx_occupancy",
    "lcmx_bellman_step",
    "lcmx_expectation",
    "lcmx_simulate",
    "lcmx_egm_step",
    "lcmx_count_nonfinite",
    "lcmx_fues_workspace_bytes",
    "lcmx_fues_scan",
    "lcmx_fues_scan_static",
    "lcmx_fues_step",
    "lcmx_copy_rows_d2h",
    "lcmx_module_status",
    "lcmx_ltm_scan",
    "lcmx_rfc_scan",
    "lcmx_mss_scan",
    "lcmx_envelope_step",
    "lcmx_launch_list",
)


class LaunchArgs(ctypes.Structure):
    _fields_ = [
        ("items", ctypes.c_void_p),
        ("tile_prefix", ctypes.c_void_p),
        ("n_items", ctypes.c_int),
        ("n_tiles", ctypes.c_int),
        ("grid", ctypes.c_int),
        ("block", ctypes.c_int),
        ("smem_bytes", ctypes.c_int),
    ]


class LaunchRec(ctypes.Structure):
    """One entry of lcmx_launch_list (include/lcmx.h)."""

    _fields_ = [
        ("module", ctypes.c_void_p),
        ("kernel", ctypes.c_char_p),
        ("args", LaunchArgs),
        ("seed", ctypes.c_ulonglong),
        ("with_seed", ctypes.c_int),
    ]


_lib = None
_lib_lock = threading.Lock()


def load_library() -> ctypes.CDLL:
    """Load liblcmx.so (building it first if the sources are newer)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            from pylcm_b200 import build as _build

            try:
                _build.build()
            except Exception as e:  # noqa: BLE001
                raise KernelError(-1, f"liblcmx.so is missing and could not be built: {e}") from e
        lib = ctypes.CDLL(str(LIB_PATH))
        vp, ip, cp = ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p
        sig = {
            "lcmx_ctx_create": ([ip, ctypes.POINTER(vp)], ip),
            "lcmx_ctx_destroy": ([vp], ip),
            "lcmx_last_error": ([vp], cp),
            "lcmx_device_info": ([vp, ctypes.POINTER(ip), ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)], ip),
            "lcmx_module_compile": ([vp, cp, cp, cp, ctypes.POINTER(vp)], ip),
            "lcmx_module_destroy": ([vp], ip),
            "lcmx_occupancy": ([vp, cp, ip, ip, ctypes.POINTER(ip)], ip),
            "lcmx_bellman_step": ([vp, cp, ctypes.POINTER(LaunchArgs), vp], ip),
            "lcmx_expectation": ([vp, cp, ctypes.POINTER(LaunchArgs), vp], ip),
            "lcmx_simulate": ([vp, cp, ctypes.POINTER(LaunchArgs), ctypes.c_ulonglong, vp], ip),
            "lcmx_egm_step": ([vp, cp, ctypes.POINTER(LaunchArgs), vp], ip),
            "lcmx_count_nonfinite": ([vp, vp, ctypes.c_longlong, vp, vp], ip),
            "lcmx_copy_rows_d2h": ([vp, vp, ctypes.c_size_t, vp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, vp],
                                   ip),
            "lcmx_fues_workspace_bytes": ([ip, ip], ctypes.c_size_t),
            "lcmx_fues_scan": (
                [vp, vp, vp, vp, vp, ip, ip, ctypes.c_double, ip, vp, vp, vp, ip, vp, vp, ctypes.c_size_t, vp],
                ip,
            ),
            "lcmx_fues_scan_static": ([vp, vp, vp, vp, vp, ip, ip, ctypes.c_double, vp, vp, vp, ip, vp, vp], ip),
            "lcmx_fues_step": ([vp, vp, vp, ip, ip, ip, vp], ip),
            "lcmx_module_status": ([vp, cp, ctypes.POINTER(ip), ip], ip),
            "lcmx_ltm_scan": ([vp, vp, vp, vp, ip, ip, vp, vp, vp, ip, vp, vp], ip),
            "lcmx_rfc_scan": ([vp, vp, vp, vp, vp, ip, ip, ip, ctypes.c_double, vp, vp, vp, ip, vp, vp], ip),
            "lcmx_mss_scan": ([vp, vp, vp, vp, ip, ip, vp, vp, vp, ip, vp, vp], ip),
            "lcmx_envelope_step": ([vp, ip, vp, vp, ip, ip, ip, vp], ip),
            "lcmx_launch_list": ([ctypes.POINTER(LaunchRec), ip, vp], ip),
        }
        for name, (args, res) in sig.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
        _lib = lib
        return lib


class Context:
    """A liblcmx context on one CUDA device."""

    def __init__(self, device: int = 0) -> None:
        self.lib = load_library()
        self.device = device
        h = ctypes.c_void_p()
        rc = self.lib.lcmx_ctx_create(device, ctypes.byref(h))
        if rc != 0:
            raise KernelError(rc, self.lib.lcmx_last_error(None).decode())
        self.h = h
        self._mods: dict[str, Module] = {}
        self._lock = threading.Lock()

    def check(self, rc: int) -> None:
        if rc != 0:
            raise KernelError(rc, self.lib.lcmx_last_error(self.h).decode())

    def device_info(self) -> tuple[int, int, int]:
        sm = ctypes.c_int()
        free = ctypes.c_size_t()
        total = ctypes.c_size_t()
        self.check(self.lib.lcmx_device_info(self.h, ctypes.byref(sm), ctypes.byref(free), ctypes.byref(total)))
        return sm.value, free.value, total.value

    def compile(self, src: str, key: str, options: str = "") -> "Module":
        with self._lock:
            m = self._mods.get(key)
            if m is not None:
                return m
            h = ctypes.c_void_p()
            self.check(self.lib.lcmx_module_compile(self.h, src.encode(), key.encode(), options.encode(), ctypes.byref(h)))
            m = Module(self, h, key)
            self._mods[key] = m
            return m

    def count_nonfinite(self, ptr: int, n: int, counts_ptr: int, stream: int) -> None:
        self.check(self.lib.lcmx_count_nonfinite(self.h, ptr, n, counts_ptr, stream))

    def copy_rows_d2h(self, dst: int, dst_pitch: int, src: int, src_pitch: int, row_bytes: int, rows: int,
                      stream: int) -> None:
        """Strided device->host copy (host `dst` page-locked for overlap)."""
        self.check(self.lib.lcmx_copy_rows_d2h(self.h, dst, dst_pitch, src, src_pitch, row_bytes, rows, stream))

    def fues_step(self, items: int, prefix: int, n_items: int, n_rows: int, max_n_in: int, stream: int) -> None:
        """FUES of the rows of several candidate blocks (device item records)."""
        self.check(self.lib.lcmx_fues_step(self.h, items, prefix, n_items, n_rows, max_n_in, stream))

    def fues_workspace_bytes(self, n_rows: int, n_in: int) -> int:
        return int(self.lib.lcmx_fues_workspace_bytes(n_rows, n_in))

    def fues_scan(self, grid, policy, value, savings, n_rows, n_in, jump_thresh, grid_out, policy_out,
                  value_out, n_out, n_kept, workspace, workspace_bytes, stream, n_points_to_scan: int = 0) -> None:
        """FUES envelope of candidate rows (all arguments are device pointers;
        `n_points_to_scan` <= 0: exhaustive look-ahead)."""
        self.check(
            self.lib.lcmx_fues_scan(self.h, grid, policy, value, savings, n_rows, n_in, float(jump_thresh),
                                    int(n_points_to_scan), grid_out, policy_out, value_out, n_out, n_kept,
                                    workspace, workspace_bytes, stream)
        )


    def ltm_scan(self, grid, policy, value, n_rows, n_in, grid_out, policy_out, value_out, n_out, n_kept,
                 stream) -> None:
        """LTM envelope of contiguous candidate rows (device pointers)."""
        self.check(self.lib.lcmx_ltm_scan(self.h, grid, policy, value, n_rows, n_in, grid_out, policy_out,
                                          value_out, n_out, n_kept, stream))

    def rfc_scan(self, grid, policy, value, marginal_utility, n_rows, n_in, search_radius, jump_thresh, grid_out,
                 policy_out, value_out, n_out, n_kept, stream) -> None:
        """RFC envelope of contiguous candidate rows (device pointers)."""
        self.check(self.lib.lcmx_rfc_scan(self.h, grid, policy, value, marginal_utility, n_rows, n_in,
                                          int(search_radius), float(jump_thresh), grid_out, policy_out, value_out,
                                          n_out, n_kept, stream))

    def mss_scan(self, grid, policy, value, n_rows, n_in, grid_out, policy_out, value_out, n_out, n_kept,
                 stream) -> None:
        """MSS envelope of contiguous candidate rows (device pointers)."""
        self.check(self.lib.lcmx_mss_scan(self.h, grid, policy, value, n_rows, n_in, grid_out, policy_out,
                                          value_out, n_out, n_kept, stream))

    def envelope_step(self, kind: int, items, prefix, n_items, n_rows, max_n_in, stream) -> None:
        """Item form of the LTM (kind 1) / RFC (kind 2) / MSS (kind 3) envelopes."""
        self.check(self.lib.lcmx_envelope_step(self.h, kind, items, prefix, n_items, n_rows, max_n_in, stream))


class Module:
    def __init__(self, ctx: Context, h: ctypes.c_void_p, key: str) -> None:
        self.ctx = ctx
        self.h = h
        self.key = key

    def prepared(self, kind: str, kernel: str, items_ptr, prefix_ptr, n_items, n_tiles, block, smem, grid=0,
                 seed=None) -> "PreparedLaunch":
        """One item launch of a generated kernel, callable with a stream;
        consecutive ones run as a single lcmx_launch_list call through
        `bundle`."""
        if kind not in _ITEM_KINDS:
            raise KeyError(kind)
        return PreparedLaunch(self.ctx, (self.h.value, kernel.encode(), items_ptr, prefix_ptr, n_items, n_tiles, grid,
                                         block, smem, seed))

    def status(self, reset: bool = True) -> int:
        """The module's device status word (0: every bounded wait of its
        kernels completed).  Synchronous."""
        v = ctypes.c_int()
        self.ctx.check(self.ctx.lib.lcmx_module_status(self.h, b"lcm_status", ctypes.byref(v), int(reset)))
        return v.value

    def occupancy(self, kernel: str, block: int, smem: int) -> int:
        n = ctypes.c_int()
        self.ctx.check(self.ctx.lib.lcmx_occupancy(self.h, kernel.encode(), block, smem, ctypes.byref(n)))
        return n.value

    def _args(self, items_ptr, prefix_ptr, n_items, n_tiles, block, smem, grid) -> LaunchArgs:
        return LaunchArgs(items_ptr, prefix_ptr, n_items, n_tiles, grid, block, smem)

    def bellman_step(self, kernel, items_ptr, prefix_ptr, n_items, n_tiles, block, smem, stream, grid=0) -> None:
        a = self._args(items_ptr, prefix_ptr, n_items, n_tiles, block, smem, grid)
        self.ctx.check(self.ctx.lib.lcmx_bellman_step(self.h, kernel.encode(), ctypes.byref(a), stream))

    def expectation(self, kernel, items_ptr, prefix_ptr, n_items, n_tiles, block, smem, stream, grid=0) -> None:
        a = self._args(items_ptr, prefix_ptr, n_items, n_tiles, block, smem, grid)
        self.ctx.check(self.ctx.lib.lcmx_expectation(self.h, kernel.encode(), ctypes.byref(a), stream))

    def simulate(self, kernel, items_ptr, prefix_ptr, n_items, n_tiles, block, smem, seed, stream, grid=0) -> None:
        a = self._args(items_ptr, prefix_ptr, n_items, n_tiles, block, smem, grid)
        self.ctx.check(self.ctx.lib.lcmx_simulate(self.h, kernel.encode(), ctypes.byref(a), seed, stream))

    def egm_step(self, kernel, items_ptr, prefix_ptr, n_items, n_tiles, block, smem, stream, grid=0) -> None:
        a = self._args(items_ptr, prefix_ptr, n_items, n_tiles, block, smem, grid)
        self.ctx.check(self.ctx.lib.lcmx_egm_step(self.h, kernel.encode(), ctypes.byref(a), stream))


_contexts: dict[int, Context] = {}
_ctx_lock = threading.Lock()


def get_context(device: int = 0) -> Context:
    import torch

    if not torch.cuda.is_available():
        raise KernelError(-1, "no CUDA device is available; pylcm_b200 solves on the GPU only")
    with _ctx_lock:
        c = _contexts.get(device)
        if c is None:
            c = Context(device)
            _contexts[device] = c
        return c


_ITEM_KINDS = frozenset(("bellman", "atab", "expect", "expect_tc", "stats", "egm", "sim"))


class PreparedLaunch:
    """One lcmx_launch_list entry: (module handle, kernel name, items,
    tile prefix, n_items, n_tiles, grid, block, shared bytes, seed or None)."""

    __slots__ = ("ctx", "rec", "_call")

    def __init__(self, ctx, rec) -> None:
        self.ctx = ctx
        self.rec = rec
        self._call = None

    def __call__(self, stream) -> None:
        if self._call is None:
            self._call = launch_list(self.ctx, [self.rec])
        self._call(stream)


def launch_list(ctx, recs) -> Callable:
    """A callable issuing the item launches `recs` (PreparedLaunch.rec
    tuples) in order on a stream with one lcmx_launch_list call."""
    n = len(recs)
    arr = (LaunchRec * n)()
    for i, (h, name, ib, pb, ni, nt, grid, block, smem, seed) in enumerate(recs):
        r = arr[i]
        r.module = h
        r.kernel = name
        a = r.args
        a.items, a.tile_prefix, a.n_items, a.n_tiles, a.grid, a.block, a.smem_bytes = ib, pb, ni, nt, grid, block, smem
        if seed is not None:
            r.seed = seed
            r.with_seed = 1
    names = [x[1] for x in recs]
    fn = ctx.lib.lcmx_launch_list

    def launch(stream):
        rc = fn(arr, n, stream)
        if rc:
            ctx.check(rc)

    launch.keepalive = (arr, names)
    return launch


def bundle(ops) -> list:
    """Callables of `ops` (per-launch callables) with every run of
    consecutive PreparedLaunch entries merged into one lcmx_launch_list call."""
    out: list = []
    pend: list = []
    ctx = None
    for op in ops:
        if isinstance(op, PreparedLaunch):
            pend.append(op.rec)
            ctx = op.ctx
            continue
        if pend:
            out.append(launch_list(ctx, pend))
            pend = []
        out.append(op)
    if pend:
        out.append(launch_list(ctx, pend))
    return out
