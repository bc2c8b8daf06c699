"""Tracing + CUDA code generation, checked without a GPU.

Every kernel the engine would launch for the test models is generated and
compiled with NVRTC for sm_100a here (NVRTC needs no device)."""

import ctypes
from pathlib import Path

import numpy as np
import pytest

from pylcm_b200 import ir, jnp
from pylcm_b200.engine import SolveEngine
from pylcm_b200.exceptions import TracingError
from tests import models as M

NVRTC = Path("/usr/local/cuda/lib64/libnvrtc.so")


def nvrtc_compile(src: str) -> tuple[int, str]:
    nv = ctypes.CDLL(str(NVRTC))
    prog = ctypes.c_void_p()
    assert nv.nvrtcCreateProgram(ctypes.byref(prog), src.encode(), b"t.cu", 0, None, None) == 0
    opts = [b"--gpu-architecture=sm_100a", b"--std=c++17", b"--device-as-default-execution-space"]
    arr = (ctypes.c_char_p * len(opts))(*opts)
    rc = nv.nvrtcCompileProgram(prog, len(opts), arr)
    n = ctypes.c_size_t()
    nv.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
    log = ctypes.create_string_buffer(n.value)
    nv.nvrtcGetProgramLog(prog, log)
    nv.nvrtcDestroyProgram(ctypes.byref(prog))
    return rc, log.value.decode()


CASES = {
    "regression": (lambda: M.regression_model(4), lambda: M.regression_params(4)),
    "processes": (lambda: M.processes_model(4, "tauchen"), lambda: M.processes_params("tauchen")),
    "retirement": (lambda: M.retirement_model(5), M.retirement_params),
    "stochastic": (lambda: M.stochastic_model(4, 20, 20), M.stochastic_params),
    "hc": (lambda: M.hc_model(3, 10, 4, 4, 8), lambda: M.hc_params(0, 4)),
    **{f"grid_{k}": (lambda k=k: M.grid_kinds_model(k), M.grid_kinds_params)
       for k in ("irreg", "log", "piece_lin", "piece_log")},
}


@pytest.mark.skipif(not NVRTC.exists(), reason="NVRTC not installed")
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_generated_kernels_compile(case, precision):
    mk, mp = CASES[case]
    model, params = mk(), mp()
    eng = SolveEngine(model, precision)
    n = 0
    for s in eng.specs:
        for p in s.active_periods:
            rk = eng.kernels(s, eng.targets_at(s, p), params)
    for rk in eng._kernels.values():
        rc, log = nvrtc_compile(rk.src)
        assert rc == 0, log[:2000]
        n += 1
    assert n >= 1


def test_tracer_builds_shared_nodes():
    x = ir.var("state", "w", "f")
    a = jnp.log(x) + 1.0
    b = jnp.log(x) + 1.0
    assert a is b  # hash-consed


def test_tracer_rejects_python_branching():
    x = ir.var("state", "w", "f")
    with pytest.raises(TracingError):
        if x > 1.0:
            pass


def test_ir_evaluate_matches_numpy():
    x = ir.var("state", "w", "f")
    e = jnp.where(x > 2.0, jnp.log(x) * 3.0, x**2 - 1.0)
    xs = np.linspace(0.5, 4, 9)
    got = ir.evaluate(e, {("state", "w"): xs}, {})
    np.testing.assert_array_equal(got, np.where(xs > 2.0, np.log(xs) * 3.0, xs**2 - 1.0))


def test_phase_split_hoists_utility_out_of_the_state_loop():
    """The utility of the retirement model depends on actions only, so it is
    evaluated once per action into shared memory, not per (state, action)."""
    from pylcm_b200 import codegen as C

    model, params = M.retirement_model(5), M.retirement_params()
    eng = SolveEngine(model, "fp64")
    s = eng.specs[0]
    rk = eng.kernels(s, eng.targets_at(s, 0), params)
    assert C._phase(rk.tr.U) == "A"
    inner = rk.src.split("__device__ __forceinline__ bool lcm_sa0_")[1].split("return true;")[0]
    assert "log(" not in inner
    assert "log(" in rk.src.split("lcm_atab_")[-1]


def test_collapsed_rows_eligibility():
    """The single-precision search reads a target with two continuous axes
    from collapsed rows when one axis is affine in a small action grid and its
    state part does not read the line state; never in double precision or
    when switched off."""
    import dataclasses

    from pylcm_b200.engine import default_config

    model, params = M.hc_model(3, 10, 4, 4, 8), M.hc_params(0, 4)
    alive = next(s for s in model.regime_specs if s.name == "alive")

    def src(precision, **kw):
        cfg = {s.name: dataclasses.replace(default_config(s, precision, 1), **kw) for s in model.regime_specs}
        eng = SolveEngine(model, precision, configs=cfg)
        return eng.kernels(alive, eng.targets_at(alive, 0), params).source()

    s32 = src("fp32")
    assert "lcm_sc1_" in s32 and "lcm_interp1s" in s32 and "nLine" in s32
    assert "lcm_sc1_" not in src("fp32", collapse=False)
    assert "lcm_sc1_" not in src("fp64")


def test_collapsed_rows_refused_when_the_collapsed_axis_reads_the_line_state(monkeypatch):
    """Human capital whose law reads wealth (the line state) cannot be
    interpolated once per line: the search keeps the bilinear read."""
    import dataclasses

    from pylcm_b200 import examples as EX
    from pylcm_b200.engine import default_config

    def next_hc(human_capital, hours, wealth):
        return 0.95 * human_capital + 0.1 * hours + 1e-4 * wealth

    monkeypatch.setattr(EX, "_hc_next_hc", next_hc)
    model, params = EX.hc_model(3, 10, 4, 4, 8), EX.hc_params(0, 4)
    alive = next(s for s in model.regime_specs if s.name == "alive")
    cfg = {s.name: default_config(s, "fp32", 1) for s in model.regime_specs}
    eng = SolveEngine(model, "fp32", configs=cfg)
    src = eng.kernels(alive, eng.targets_at(alive, 0), params).source()
    assert "lcm_sc1_" not in src and "nLine" not in src
