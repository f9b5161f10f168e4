"""The reference's own CUDA known-answer tests (cuda/tests/spmv_smoke.cu,
pdhg_smoke.cu, diagonal_qp_smoke.cu): first the programs themselves, compiled
unchanged against include/sankhya_cuda.h and linked to this library
(oracle/Makefile target ref-tests, built where the reference sources are
present), then the same checks restated through the C ABI from Python."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
INF = float("inf")
ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
REF_PROGRAMS = ("spmv_smoke", "pdhg_smoke", "diagonal_qp_smoke")


@pytest.mark.parametrize("name", REF_PROGRAMS)
def test_reference_program(name, engine):
    """The reference's test program, unmodified, against this library: exit 0."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_" + name)
    if not os.path.exists(exe):
        pytest.skip("reference test programs not built (reference sources absent at build time)")
    ldd = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
    lib = os.path.realpath(os.path.join(ROOT, "the-solver_b200", "lib", "libsankhya_cuda.so"))
    assert any(os.path.realpath(line.split("=>")[1].split("(")[0].strip()) == lib
               for line in ldd.splitlines() if "libsankhya_cuda.so" in line and "=>" in line), ldd
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)


def test_spmv_smoke(engine):
    # spmv_smoke.cu:135-156: [[1,0,2],[0,3,4]] * [2,5,7] = [16,43]; bad inputs rejected
    import torch
    offsets, columns, values = [0, 2, 4], [0, 2, 1, 2], [1.0, 2.0, 3.0, 4.0]
    with pytest.raises(RuntimeError):
        engine.Matrix(2, 3, [0, 3, 2], columns, values)
    with pytest.raises(RuntimeError):
        engine.Matrix(2, 3, offsets, [0, 3, 1, 2], values)
    with pytest.raises(RuntimeError):
        engine.Matrix(2, 3, offsets, columns, [1.0, np.nan, 3.0, 4.0])
    rc, y = engine.spmv_host(2, 3, offsets, columns, values, [2.0, 5.0, 7.0])
    assert rc == 0 and y.tolist() == [16.0, 43.0]
    # :158-180 persistent CSR, queued A x -> A^T y -> A x chain on the default stream
    A = engine.Matrix(2, 3, offsets, columns, values)
    dx = torch.tensor([2.0, 5.0, 7.0], dtype=torch.float64, device="cuda")
    dy = torch.zeros(2, dtype=torch.float64, device="cuda")
    L = engine.lib()
    assert L.sankhya_cuda_spmv_device_f64(A.handle, dx.data_ptr(), dy.data_ptr()) == 0
    assert dy.cpu().tolist() == [16.0, 43.0]
    assert L.sankhya_cuda_spmv_transpose_device_f64(A.handle, dy.data_ptr(), dx.data_ptr()) == 0
    assert L.sankhya_cuda_spmv_device_f64(A.handle, dx.data_ptr(), dy.data_ptr()) == 0
    assert dy.cpu().tolist() == [424.0, 1203.0]
    A.close()


def test_axpy(engine):
    import torch
    rc, y = engine.axpy_host(2.0, [1.0, 2.0, 3.0], [10.0, 20.0, 30.0])
    assert rc == 0 and y.tolist() == [12.0, 24.0, 36.0]
    dx = torch.tensor([1.0, 2.0], dtype=torch.float64, device="cuda")
    dy = torch.tensor([1.0, 1.0], dtype=torch.float64, device="cuda")
    assert engine.lib().sankhya_cuda_axpy_device_f64(2, -1.0, dx.data_ptr(), dy.data_ptr()) == 0
    assert dy.cpu().tolist() == [0.0, -1.0]


def _one(engine, value=1.0):
    return engine.Matrix(1, 1, [0, 1], [0], [value])


def test_pdhg_smoke(engine):
    # pdhg_smoke.cu: min x, x >= 1 (row), x >= 0 -> x = 1
    inst = dict(c=[1.0], rl=[1.0], ru=[INF], cl=[0.0], cu=[INF])
    A = _one(engine)
    s = engine.settings(5000, 10, 0.25, 2.0, 1.0, 1e-5)
    rc, *_ = engine.pdhg(A, inst, s, c=[np.nan])
    assert rc != 0
    big = _one(engine, 1e308)
    rc, x, y, r = engine.pdhg(big, inst, s, rl=[1e308])
    assert rc == -2 and r["status"] == -2
    rc, x, y, r = engine.pdhg(A, inst, s)
    assert rc == 0 and r["status"] == 0
    for k in ("maximum_row_violation", "maximum_kkt_residual", "maximum_dual_residual", "maximum_complementarity"):
        assert np.isfinite(r[k]) and r[k] <= 1e-5
    assert abs(x[0] - 1.0) <= 1e-3


def test_diagonal_qp_smoke(engine):
    # diagonal_qp_smoke.cu: min x^2 - 4x, x >= 1 -> x = 2, obj -4
    inst = dict(c=[-4.0], rl=[1.0], ru=[INF], cl=[0.0], cu=[INF])
    A = _one(engine)
    s = engine.settings(10000, 10, 0.15, 0.5, 1.0, 1e-7)
    rc, x, y, r = engine.pdhg(A, inst, s, qdiag=[2.0])
    assert rc == 0 and r["status"] == 0 and abs(x[0] - 2) <= 1e-5 and abs(r["objective"] + 4) <= 1e-5
    for k in ("maximum_row_violation", "maximum_kkt_residual", "maximum_dual_residual", "maximum_complementarity"):
        assert r[k] <= 1e-7
    s0 = engine.settings(10000, 10, 0.0, 0.0, 1.0, 1e-7)
    rc, x, y, r = engine.pdhg(A, inst, s0, qdiag=[2.0], primal_steps=[0.15], dual_steps=[0.5], want_dual=True)
    assert rc == 0 and r["status"] == 0 and abs(x[0] - 2) <= 1e-5 and abs(y[0]) <= 1e-6
    rc, *_ = engine.pdhg(A, inst, s0, qdiag=[2.0], primal_steps=[0.0], dual_steps=[0.5])
    assert rc != 0


def test_argument_validation(engine):
    """sankhya_cuda_lp.cu:116-153: -1 for each invalid-input class."""
    inst = dict(c=[1.0], rl=[1.0], ru=[INF], cl=[0.0], cu=[INF])
    A = _one(engine)
    good = dict(max_iterations=10, check_every=5, tau=0.1, sigma=0.1, theta=1.0, tolerance=1e-6)
    for bad in (dict(max_iterations=0), dict(check_every=0), dict(theta=1.5), dict(theta=-0.1),
                dict(tolerance=0.0), dict(tau=0.0), dict(time_limit=-1.0)):
        s = engine.settings(**{**good, **bad})
        rc, *_ = engine.pdhg(A, inst, s)
        assert rc == -1, bad
    s = engine.settings(**good)
    for over in (dict(cl=[INF]), dict(cu=[-INF]), dict(cl=[2.0], cu=[1.0]), dict(rl=[np.nan]),
                 dict(rl=[2.0], ru=[1.0])):
        rc, *_ = engine.pdhg(A, inst, s, **over)
        assert rc == -1, over
    rc, *_ = engine.pdhg(A, inst, s, qdiag=[-1.0])
    assert rc == -1
