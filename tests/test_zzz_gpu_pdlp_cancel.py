"""PDLP cancellation: settings version 4's `cancel` callback, the counterpart of
GpuPdlp's PdlpParams::cancel (src/cuda/GpuPdlp.hpp:62-67), a flag the caller sets to
stop a running solve. The callback is called once per
restart window, where the host synchronizes anyway, so a non-zero answer stops the
solve after the window that is running, with status 3. A callback that answers zero
changes nothing. (Named to run after every other gpu file, the allocation-free entry
point's included.)"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PERIOD = 64
CANCEL = C.CFUNCTYPE(C.c_int, C.c_void_p)


def _solve(engine, A, inst, flag=None, **fields):
    """flag: a c_int the callback reads through its context pointer; the number of
    calls is counted in calls[0]."""
    s = engine.pdlp_default_settings()
    s.eps_optimal = 1e-6
    s.restart_period = PERIOD
    for k, v in fields.items():
        setattr(s, k, v)
    calls = [0]

    def poll(context):
        calls[0] += 1
        return C.c_int.from_address(context).value

    cb = CANCEL(poll)   # kept alive for the call
    if flag is not None:
        s.cancel = C.cast(cb, C.c_void_p).value
        s.cancel_context = C.addressof(flag)
    rc, x, y, r = engine.pdlp_solve(A, inst, s)
    return rc, x, y, r, calls[0]


def test_zero_flag_changes_nothing(engine, instances):
    inst = instances.lp_uniform(11, 300, 700, 5)
    A = engine.Matrix.from_instance(inst)
    rc0, x0, y0, r0, _ = _solve(engine, A, inst)
    assert rc0 == 0 and r0["status"] == 0 and r0["iterations"] > PERIOD
    clear = C.c_int(0)
    rc, x, y, r, calls = _solve(engine, A, inst, clear)
    assert rc == 0 and r["status"] == 0 and r["iterations"] == r0["iterations"]
    assert np.array_equal(x, x0) and np.array_equal(y, y0)
    assert 1 <= calls <= r["iterations"] // PERIOD   # once per window that did not converge


@pytest.mark.parametrize("variant", ["adaptive_fp64", "adaptive_fp32_refine", "halpern"])
def test_set_flag_stops_after_the_running_window(engine, instances, variant):
    inst = instances.lp_uniform(11, 300, 700, 5)
    A = engine.Matrix.from_instance(inst)
    fields = {"adaptive_fp64": {}, "adaptive_fp32_refine": {"precision": engine.FP32_REFINE},
              "halpern": {"algorithm": engine.PDLP_HALPERN}}[variant]
    stop = C.c_int(1)
    rc, x, y, r, calls = _solve(engine, A, inst, stop, **fields)
    assert rc == 0 and r["status"] == 3, r
    # the FP32 loop formed its first FP64 center (one refinement) before the first window
    assert r["iterations"] == PERIOD and calls == 1
    assert r["refinements"] == (1 if variant == "adaptive_fp32_refine" else 0)
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(y))
