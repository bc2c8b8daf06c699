"""The C-ABI library builds, loads and exports every declared entry point.

No compute call is made here (no GPU needed)."""

import ctypes
import re
from pathlib import Path

from pylcm_b200 import build as B

HEADER = Path(__file__).resolve().parent.parent / "include" / "lcmx.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(lcmx_[a-z0-9_]+)\s*\(", text))


def test_library_exports_every_declared_symbol():
    lib_path = B.build()
    lib = ctypes.CDLL(str(lib_path))
    syms = declared_symbols()
    assert "lcmx_bellman_step" in syms and len(syms) >= 10
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_runtime_binding_matches_header():
    from pylcm_b200 import runtime

    assert declared_symbols() == set(runtime.EXPORTED)


def test_last_error_without_context_is_a_string():
    from pylcm_b200 import runtime

    lib = runtime.load_library()
    assert isinstance(lib.lcmx_last_error(None), bytes)


def test_compile_rejects_null_arguments_without_gpu():
    """Argument validation happens before any CUDA call."""
    from pylcm_b200 import runtime

    lib = runtime.load_library()
    out = ctypes.c_void_p()
    rc = lib.lcmx_module_compile(None, b"", b"k", None, ctypes.byref(out))
    assert rc == 1  # LCMX_ERR_ARGS


def test_launch_record_layout_matches_the_header(tmp_path):
    """lcmx_launch_rec / lcmx_launch_args as the C compiler lays them out and
    as the ctypes mirrors in runtime.py do."""
    import shutil
    import subprocess

    import pytest

    from pylcm_b200.runtime import LaunchArgs, LaunchRec

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "lcmx.h"\n'
        "int main(void) { printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(lcmx_launch_rec),"
        " offsetof(lcmx_launch_rec, kernel), offsetof(lcmx_launch_rec, args), offsetof(lcmx_launch_rec, seed),"
        " offsetof(lcmx_launch_rec, with_seed), sizeof(lcmx_launch_args)); return 0; }\n"
    )
    exe = tmp_path / "layout"
    subprocess.run([cc, f"-I{HEADER.parent}", str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [ctypes.sizeof(LaunchRec), LaunchRec.kernel.offset, LaunchRec.args.offset, LaunchRec.seed.offset,
            LaunchRec.with_seed.offset, ctypes.sizeof(LaunchArgs)]
    assert got == want


def test_launch_list_rejects_bad_arguments_without_gpu():
    """Argument validation of lcmx_launch_list happens before any CUDA call."""
    from pylcm_b200 import runtime

    lib = runtime.load_library()
    assert lib.lcmx_launch_list(None, 0, None) == 0  # nothing to launch
    assert lib.lcmx_launch_list(None, 2, None) == 1  # LCMX_ERR_ARGS
    recs = (runtime.LaunchRec * 1)()  # a record without module or kernel
    assert lib.lcmx_launch_list(recs, 1, None) == 1


def test_bundle_merges_runs_of_item_launches():
    """runtime.bundle: consecutive PreparedLaunch entries become one launch
    list (in order), other callables stay where they are."""
    from pylcm_b200 import runtime

    calls = []

    class FakeLib:
        def lcmx_launch_list(self, arr, n, stream):
            calls.append(("list", [arr[i].kernel for i in range(n)], stream))
            return 0

    class FakeCtx:
        lib = FakeLib()

        def check(self, rc):
            raise AssertionError(rc)

    def prep(name, seed=None):
        return runtime.PreparedLaunch(FakeCtx(), (1, name.encode(), 16, 32, 1, 1, 0, 256, 0, seed))

    def other(stream):
        calls.append(("other", stream))

    ops = [prep("a"), prep("b", seed=3), other, prep("c"), other, other, prep("d")]
    out = runtime.bundle(ops)
    assert len(out) == 6
    for f in out:
        f(7)
    assert calls == [("list", [b"a", b"b"], 7), ("other", 7), ("list", [b"c"], 7), ("other", 7), ("other", 7),
                     ("list", [b"d"], 7)]
