"""SpMV on the matrix shapes of the reference's GPU SpMV tests
(tests/cuda/test_gpu_spmv.cpp:89-172: diagonal, dense, rectangular, pathologically
sparse with mostly empty rows, dense-ish, large random, and repeated execution on one
handle), through this library's entry points: the device product, the device
transpose product and the host-array product. The reference holds its GPU result to
1e-9 absolute and relative against the CPU product; here every product must meet
that, and every row of up to 32 entries (the owning-lane path) must equal the
sequential sum in stored order bit for bit. (Named to run after every other gpu file, the
allocation-free entry point's included.)"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ABS_TOL = REL_TOL = 1e-9


def _random_csr(rows, cols, density, seed, lo=-10.0, hi=10.0):
    rng = np.random.default_rng(seed)
    mask = rng.random((rows, cols)) < density
    vals = rng.uniform(lo, hi, (rows, cols))
    return _csr(np.where(mask, vals, 0.0), mask)


def _csr(dense, mask=None):
    mask = dense != 0.0 if mask is None else mask
    ptr = np.zeros(dense.shape[0] + 1, np.int32)
    ptr[1:] = np.cumsum(mask.sum(axis=1))
    idx = np.concatenate([np.nonzero(mask[i])[0] for i in range(dense.shape[0])] + [np.zeros(0, np.int64)])
    val = np.concatenate([dense[i, mask[i]] for i in range(dense.shape[0])] + [np.zeros(0)])
    return ptr, idx.astype(np.int32), val.astype(np.float64)


def _sequential(ptr, idx, val, x):
    """Row sums in stored order, one rounding per add (the reference's serial loop)."""
    y = np.zeros(len(ptr) - 1)
    for r in range(len(ptr) - 1):
        s = 0.0
        for p in range(ptr[r], ptr[r + 1]):
            s += float(val[p]) * float(x[idx[p]])
        y[r] = s
    return y


def _transpose(rows, cols, ptr, idx, val):
    """A^T in CSR with each row's entries in ascending source row (the stored order of
    the engine's transpose)."""
    r = np.repeat(np.arange(rows), np.diff(ptr))
    order = np.lexsort((r, idx))
    tptr = np.zeros(cols + 1, np.int32)
    tptr[1:] = np.cumsum(np.bincount(idx, minlength=cols))
    return tptr, r[order].astype(np.int32), val[order]


def _check(got, ptr, ref):
    diff = np.abs(got - ref)
    assert diff.max(initial=0.0) < ABS_TOL
    assert (diff / (1.0 + np.abs(ref))).max(initial=0.0) < REL_TOL
    short = np.diff(ptr) <= 32
    assert np.array_equal(got[short], ref[short])


def _products(engine, rows, cols, ptr, idx, val, xs, ys):
    import torch
    A = engine.Matrix(rows, cols, ptr, idx, val)
    L = engine.lib()
    tptr, tidx, tval = _transpose(rows, cols, ptr, idx, val)
    try:
        for x, y in zip(xs, ys):
            dx = torch.tensor(x, dtype=torch.float64, device="cuda")
            dy = torch.zeros(rows, dtype=torch.float64, device="cuda")
            assert L.sankhya_cuda_spmv_device_f64(A.handle, dx.data_ptr(), dy.data_ptr()) == 0
            _check(dy.cpu().numpy(), ptr, _sequential(ptr, idx, val, x))
            rc, yh = engine.spmv_host(rows, cols, ptr, idx, val, x)
            assert rc == 0
            _check(yh, ptr, _sequential(ptr, idx, val, x))
            dyt = torch.tensor(y, dtype=torch.float64, device="cuda")
            dxt = torch.zeros(cols, dtype=torch.float64, device="cuda")
            assert L.sankhya_cuda_spmv_transpose_device_f64(A.handle, dyt.data_ptr(), dxt.data_ptr()) == 0
            _check(dxt.cpu().numpy(), tptr, _sequential(tptr, tidx, tval, y))
    finally:
        A.close()


@pytest.mark.parametrize("shape", ["diagonal", "dense16", "rectangular", "pathologically_sparse", "dense_ish",
                                   "large_random"])
def test_shapes_match_sequential_product(engine, shape):
    rng = np.random.default_rng(100)
    if shape == "diagonal":
        ptr, idx, val = _csr(np.diag([2.0, 3.0, 4.0]))
        rows = cols = 3
        x = np.ones(3)
    elif shape == "dense16":
        rows = cols = 16
        ptr, idx, val = _csr(rng.uniform(-5.0, 5.0, (16, 16)), np.ones((16, 16), bool))
        x = rng.uniform(-5.0, 5.0, 16)
    elif shape == "rectangular":
        rows, cols = 50, 30
        ptr, idx, val = _random_csr(50, 30, 0.1, 11)
        x = rng.uniform(-4.0, 4.0, 30)
    elif shape == "pathologically_sparse":
        rows = cols = 500
        ptr, idx, val = _random_csr(500, 500, 0.0001, 21)
        assert (np.diff(ptr) == 0).mean() > 0.9        # most rows empty
        x = np.ones(500)
    elif shape == "dense_ish":
        rows = cols = 80
        ptr, idx, val = _random_csr(80, 80, 0.6, 31)
        assert np.diff(ptr).max() > 32                 # rows beyond the owning-lane path
        x = rng.uniform(-2.0, 2.0, 80)
    else:
        rows = cols = 3000
        ptr, idx, val = _random_csr(3000, 3000, 0.002, 41)
        x = np.ones(3000)
    y = rng.uniform(-3.0, 3.0, rows)
    _products(engine, rows, cols, ptr, idx, val, [x], [y])


def test_repeated_execution_on_one_handle(engine):
    """Five different inputs through the same matrix handle: no state leaks between calls."""
    ptr, idx, val = _random_csr(100, 100, 0.05, 51)
    rng = np.random.default_rng(52)
    xs = [rng.uniform(-3.0, 3.0, 100) for _ in range(5)]
    ys = [rng.uniform(-3.0, 3.0, 100) for _ in range(5)]
    _products(engine, 100, 100, ptr, idx, val, xs, ys)
