"""The allocation-free entry point, sankhya_b200_lp_pdhg_device_noalloc.

Some callers cannot call cudaMalloc while they solve: runtimes that hand out
all device memory from their own pool, processes with a fixed device-memory
budget that must not grow after start-up, services that cannot take the
device-wide synchronisation cudaMalloc/cudaFree can impose on other streams. This entry point takes device pointers for the model
and the solution and keeps its scratch in a fixed 16 MiB array inside the
library, so a solve allocates nothing. These tests call it through the C ABI and
check it against the allocating entry point, sankhya_cuda_lp_pdhg, on two calls
of the same instance with a solve of a different, larger instance between them:
the array keeps the previous call's contents, so the second compared call starts
on scratch that another problem left behind and checks that everything that must
start at zero is cleared. The file is named to be collected after the rest of the
suite; only the test_zzz_ files follow it."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(engine):
    L = engine.lib()
    f = L.sankhya_b200_lp_pdhg_device_noalloc
    f.argtypes = [C.POINTER(engine.CSR)] + [C.c_void_p] * 5 + [engine.Settings, C.c_void_p,
                                                                C.POINTER(engine.Result)]
    f.restype = C.c_int
    return f


def _device_model(inst):
    import torch
    return {k: torch.tensor(np.asarray(inst[k], dtype=np.float64), device="cuda") for k in ("c", "rl", "ru", "cl", "cu")}


def _solve(f, engine, A, d, n, s):
    import torch
    sol = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    res = engine.Result()
    rc = f(C.byref(A.handle), d["c"].data_ptr(), d["rl"].data_ptr(), d["ru"].data_ptr(), d["cl"].data_ptr(),
           d["cu"].data_ptr(), s, sol.data_ptr(), C.byref(res))
    assert rc == 0, engine.last_error()
    return sol.cpu().numpy(), res.as_dict()


def test_matches_allocating_entry_on_two_calls(engine, instances):
    inst = instances.lp_uniform(41, 500, 1200, 5)
    other = instances.lp_uniform(42, 3000, 7000, 5)   # larger: its scratch covers the first one's
    A = engine.Matrix.from_instance(inst)
    B = engine.Matrix.from_instance(other)
    s = engine.settings(300, 50, 0.05, 0.05, 1.0, 1e-9)
    rc, x_ref, _, r_ref = engine.pdhg(A, inst, s)
    assert rc == 0
    rc, xo_ref, _, ro_ref = engine.pdhg(B, other, s)
    assert rc == 0
    f = _bind(engine)
    d, do = _device_model(inst), _device_model(other)
    for call in range(2):
        x, r = _solve(f, engine, A, d, inst["n"], s)
        # same kernels in the same order: bit-identical to the allocating entry point
        assert np.array_equal(x, x_ref), call
        assert r == r_ref, call
        if call == 0:
            xo, ro = _solve(f, engine, B, do, other["n"], s)
            assert np.array_equal(xo, xo_ref) and ro == ro_ref


def test_converges_like_the_allocating_entry(engine, instances):
    import torch
    inst = instances.small_dense_lp(1, 1, [1.0], [1.0], [1.0], [float("inf")], [0.0], [float("inf")])
    A = engine.Matrix.from_instance(inst)
    s = engine.settings(5000, 10, 0.25, 2.0, 1.0, 1e-5)
    rc, x_ref, _, r_ref = engine.pdhg(A, inst, s)
    f = _bind(engine)
    d = _device_model(inst)
    sol = torch.zeros(1, dtype=torch.float64, device="cuda")
    res = engine.Result()
    assert f(C.byref(A.handle), d["c"].data_ptr(), d["rl"].data_ptr(), d["ru"].data_ptr(), d["cl"].data_ptr(),
             d["cu"].data_ptr(), s, sol.data_ptr(), C.byref(res)) == 0
    assert res.status == 0 and res.iterations == r_ref["iterations"]
    assert abs(sol.item() - 1.0) <= 1e-3


def test_rejects_a_handle_pointing_at_other_arrays(engine, instances):
    """A copy of a handle whose values pointer was moved is not the planned matrix."""
    import torch
    inst = instances.lp_uniform(43, 50, 120, 4)
    A = engine.Matrix.from_instance(inst)
    other_values = torch.tensor(inst["val"] * 2.0, device="cuda")
    h = engine.CSR(A.handle.rows, A.handle.cols, A.handle.nnz, A.handle.device_row_offsets,
                   A.handle.device_column_indices, other_values.data_ptr())
    f = _bind(engine)
    d = _device_model(inst)
    sol = torch.zeros(inst["n"], dtype=torch.float64, device="cuda")
    res = engine.Result()
    rc = f(C.byref(h), d["c"].data_ptr(), d["rl"].data_ptr(), d["ru"].data_ptr(), d["cl"].data_ptr(),
           d["cu"].data_ptr(), engine.settings(10, 5, 0.1, 0.1, 1.0, 1e-6), sol.data_ptr(), C.byref(res))
    assert rc == -1 and "sankhya_cuda_csr_create" in engine.last_error()


def test_rejects_sizes_beyond_the_scratch(engine):
    import torch
    n = 600_000  # 4 * cols doubles alone exceed the 2 Mi-double scratch
    A = engine.Matrix(1, n, [0, n], np.arange(n, dtype=np.int32), np.ones(n))
    f = _bind(engine)
    z = torch.zeros(n, dtype=torch.float64, device="cuda")
    r = torch.zeros(1, dtype=torch.float64, device="cuda")
    res = engine.Result()
    rc = f(C.byref(A.handle), z.data_ptr(), r.data_ptr(), r.data_ptr(), z.data_ptr(), z.data_ptr(),
           engine.settings(10, 5, 0.1, 0.1, 1.0, 1e-6), z.data_ptr(), C.byref(res))
    assert rc == -1 and "too large" in engine.last_error()
