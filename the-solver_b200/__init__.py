"""Python view of the B200 PDHG engine's C ABI (lib/libsankhya_cuda.so).

The engine itself is C++/CUDA behind the reference's C entry points; this
module only loads the shared library with ctypes and marshals numpy arrays,
for tests and benchmarks. It raises when the library is missing: there is no
Python or CPU fallback.

Import it by path (the folder name is not a Python identifier):
    spec = importlib.util.spec_from_file_location("sankhya_b200", "<repo>/the-solver_b200/__init__.py")
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsankhya_cuda.so")

dptr = C.POINTER(C.c_double)
iptr = C.POINTER(C.c_int)

# Every symbol declared in include/sankhya_cuda.h and include/sankhya_b200.h.
REFERENCE_SYMBOLS = (
    "sankhya_cuda_csr_create", "sankhya_cuda_csr_destroy", "sankhya_cuda_spmv_device_f64",
    "sankhya_cuda_spmv_transpose_device_f64", "sankhya_cuda_axpy_device_f64", "sankhya_cuda_lp_pdhg",
    "sankhya_cuda_qp_pdhg_preconditioned_with_dual", "sankhya_cuda_diagonal_qp_pdhg",
    "sankhya_cuda_sparse_qp_pdhg", "sankhya_cuda_qp_pdhg_preconditioned", "sankhya_cuda_spmv_f64",
    "sankhya_cuda_axpy_f64", "sankhya_cuda_last_error",
)
EXTENSION_SYMBOLS = (
    "sankhya_b200_set_timing", "sankhya_b200_last_timing", "sankhya_b200_pdhg_loop",
    "sankhya_b200_pdlp_default_settings", "sankhya_b200_pdlp_solve", "sankhya_b200_pdlp_solve_qp",
    "sankhya_b200_scale_factors",
    "sankhya_b200_batch_default_settings", "sankhya_b200_batch_pdhg", "sankhya_b200_shared_batch_pdhg",
    "sankhya_b200_lp_pdhg_device_noalloc", "sankhya_b200_gnn_default_settings", "sankhya_b200_gnn_create",
    "sankhya_b200_gnn_destroy", "sankhya_b200_gnn_parameter_count", "sankhya_b200_gnn_get_parameters",
    "sankhya_b200_gnn_set_parameters", "sankhya_b200_gnn_predict", "sankhya_b200_gnn_gradient",
    "sankhya_b200_gnn_train_step", "sankhya_b200_csr_transpose", "sankhya_b200_polish_default_settings",
    "sankhya_b200_pdlp_solve_polished",
)

_lib = None


def build(verbose: bool = False) -> str:
    """Compiles lib/libsankhya_cuda.so for sm_100a with nvcc (make)."""
    out = subprocess.run(["make", "-C", HERE, "-j8"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("building libsankhya_cuda.so failed:\n" + out.stdout + out.stderr)
    if verbose:
        print(out.stdout)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


class CSR(C.Structure):
    """SankhyaCudaCSR."""
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("nnz", C.c_int),
                ("device_row_offsets", C.c_void_p), ("device_column_indices", C.c_void_p),
                ("device_values", C.c_void_p)]


class Settings(C.Structure):
    """SankhyaCudaLPSettings."""
    _fields_ = [("max_iterations", C.c_int), ("check_every", C.c_int), ("tau", C.c_double),
                ("sigma", C.c_double), ("theta", C.c_double), ("tolerance", C.c_double),
                ("time_limit", C.c_double)]


class Result(C.Structure):
    """SankhyaCudaLPResult."""
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("objective", C.c_double),
                ("maximum_row_violation", C.c_double), ("maximum_step", C.c_double),
                ("maximum_kkt_residual", C.c_double), ("maximum_dual_residual", C.c_double),
                ("maximum_complementarity", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Timing(C.Structure):
    """SankhyaB200Timing."""
    _fields_ = [("iterations", C.c_int), ("checkpoints", C.c_int), ("kernel_launches", C.c_int),
                ("per_kernel_samples", C.c_int), ("loop_ms", C.c_double), ("checkpoint_ms", C.c_double),
                ("dual_kernel_ms", C.c_double), ("primal_kernel_ms", C.c_double), ("h2d_ms", C.c_double),
                ("d2h_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LoopResult(C.Structure):
    """SankhyaB200LoopResult."""
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("numeric_failure", C.c_int),
                ("dual_step", C.c_double), ("anorm", C.c_double), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PdlpSettings(C.Structure):
    """SankhyaB200PdlpSettings."""
    _fields_ = [("struct_version", C.c_int), ("max_iterations", C.c_int), ("restart_period", C.c_int),
                ("power_iterations", C.c_int), ("adaptive_step", C.c_int), ("scaling", C.c_int),
                ("ruiz_iterations", C.c_int), ("precision", C.c_int), ("eps_optimal", C.c_double),
                ("time_limit", C.c_double), ("eta_min_factor", C.c_double), ("eta_max_factor", C.c_double),
                ("ruiz_tolerance", C.c_double), ("algorithm", C.c_int), ("reserved", C.c_int),
                ("initial_primal_weight", C.c_double), ("cancel", C.c_void_p), ("cancel_context", C.c_void_p)]


class PdlpResult(C.Structure):
    """SankhyaB200PdlpResult."""
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("restarts", C.c_int),
                ("rejected_steps", C.c_int), ("host_syncs", C.c_int), ("refinements", C.c_int),
                ("primal_objective", C.c_double), ("dual_objective", C.c_double),
                ("relative_primal_residual", C.c_double), ("relative_dual_residual", C.c_double),
                ("relative_gap", C.c_double), ("matrix_norm", C.c_double), ("final_step_size", C.c_double),
                ("primal_weight", C.c_double), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PolishSettings(C.Structure):
    """SankhyaB200PolishSettings."""
    _fields_ = [("struct_version", C.c_int), ("max_polish_iterations", C.c_int),
                ("start_tolerance", C.c_double), ("polish_tolerance", C.c_double)]


class PolishResult(C.Structure):
    """SankhyaB200PolishResult."""
    _fields_ = [("rounds", C.c_int), ("main_iterations", C.c_int), ("primal_iterations", C.c_int),
                ("dual_iterations", C.c_int), ("main_seconds", C.c_double), ("polish_seconds", C.c_double),
                ("main_relative_primal_residual", C.c_double), ("main_relative_dual_residual", C.c_double),
                ("main_relative_gap", C.c_double), ("pair_relative_primal_residual", C.c_double),
                ("pair_relative_dual_residual", C.c_double), ("pair_relative_gap", C.c_double),
                ("pair_primal_objective", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchSettings(C.Structure):
    """SankhyaB200BatchSettings."""
    _fields_ = [("struct_version", C.c_int), ("max_iterations", C.c_int), ("check_every", C.c_int),
                ("schedule", C.c_int), ("primal_tol", C.c_double), ("dual_tol", C.c_double),
                ("time_limit", C.c_double)]


class BatchResult(C.Structure):
    """SankhyaB200BatchResult."""
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("objective", C.c_double),
                ("row_violation", C.c_double), ("step", C.c_double), ("dual_step", C.c_double),
                ("anorm", C.c_double)]


class GnnSettings(C.Structure):
    """SankhyaB200GnnSettings."""
    _fields_ = [("struct_version", C.c_int), ("rounds", C.c_int), ("seed", C.c_ulonglong),
                ("learning_rate", C.c_double), ("y_scale", C.c_double)]


SCALE_RUIZ, SCALE_POCK_CHAMBOLLE, SCALE_POW2 = 1, 2, 4
FP64, FP32_REFINE, BF16_REFINE = 0, 1, 2
PDLP_ADAPTIVE, PDLP_HALPERN = 0, 1


def _declare(L):
    P = C.POINTER
    L.sankhya_cuda_csr_create.argtypes = [P(CSR), C.c_int, C.c_int, C.c_int, iptr, iptr, dptr]
    L.sankhya_cuda_csr_destroy.argtypes = [P(CSR)]
    L.sankhya_cuda_csr_destroy.restype = None
    L.sankhya_cuda_last_error.restype = C.c_char_p
    L.sankhya_cuda_spmv_device_f64.argtypes = [P(CSR), C.c_void_p, C.c_void_p]
    L.sankhya_cuda_spmv_transpose_device_f64.argtypes = [P(CSR), C.c_void_p, C.c_void_p]
    L.sankhya_cuda_axpy_device_f64.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    L.sankhya_cuda_spmv_f64.argtypes = [C.c_int, C.c_int, C.c_int, iptr, iptr, dptr, dptr, dptr]
    L.sankhya_cuda_axpy_f64.argtypes = [C.c_int, C.c_double, dptr, dptr]
    L.sankhya_cuda_lp_pdhg.argtypes = [P(CSR), dptr, dptr, dptr, dptr, dptr, Settings, dptr, P(Result)]
    L.sankhya_cuda_diagonal_qp_pdhg.argtypes = [P(CSR), dptr, dptr, dptr, dptr, dptr, dptr, Settings, dptr,
                                                P(Result)]
    L.sankhya_cuda_sparse_qp_pdhg.argtypes = [P(CSR), P(CSR), dptr, dptr, dptr, dptr, dptr, Settings, dptr,
                                              P(Result)]
    L.sankhya_cuda_qp_pdhg_preconditioned.argtypes = [P(CSR), P(CSR), dptr, dptr, dptr, dptr, dptr, dptr, dptr,
                                                      dptr, Settings, dptr, P(Result)]
    L.sankhya_cuda_qp_pdhg_preconditioned_with_dual.argtypes = [P(CSR), P(CSR), dptr, dptr, dptr, dptr, dptr,
                                                                dptr, dptr, dptr, Settings, dptr, dptr,
                                                                P(Result)]
    L.sankhya_b200_set_timing.argtypes = [C.c_int]
    L.sankhya_b200_set_timing.restype = None
    L.sankhya_b200_last_timing.argtypes = [P(Timing)]
    L.sankhya_b200_last_timing.restype = None
    L.sankhya_b200_pdhg_loop.argtypes = [C.c_void_p, C.c_void_p, dptr, dptr, dptr, P(LoopResult)]
    if hasattr(L, "sankhya_b200_pdlp_solve"):
        L.sankhya_b200_pdlp_default_settings.argtypes = [P(PdlpSettings)]
        L.sankhya_b200_pdlp_default_settings.restype = None
        L.sankhya_b200_pdlp_solve.argtypes = [P(CSR), dptr, dptr, dptr, dptr, dptr, P(PdlpSettings), dptr,
                                              dptr, dptr, dptr, P(PdlpResult)]
        L.sankhya_b200_scale_factors.argtypes = [P(CSR), C.c_int, C.c_int, C.c_double, dptr, dptr]
    if hasattr(L, "sankhya_b200_pdlp_solve_qp"):
        L.sankhya_b200_pdlp_solve_qp.argtypes = [P(CSR), P(CSR), dptr, dptr, dptr, dptr, dptr, dptr,
                                                 P(PdlpSettings), dptr, dptr, dptr, dptr, P(PdlpResult)]
    if hasattr(L, "sankhya_b200_pdlp_solve_polished"):
        L.sankhya_b200_polish_default_settings.argtypes = [P(PolishSettings)]
        L.sankhya_b200_polish_default_settings.restype = None
        L.sankhya_b200_pdlp_solve_polished.argtypes = [P(CSR), dptr, dptr, dptr, dptr, dptr, P(PdlpSettings),
                                                       P(PolishSettings), dptr, dptr, dptr, dptr, P(PdlpResult),
                                                       P(PolishResult)]
    if hasattr(L, "sankhya_b200_batch_pdhg"):
        L.sankhya_b200_batch_default_settings.argtypes = [P(BatchSettings)]
        L.sankhya_b200_batch_default_settings.restype = None
        L.sankhya_b200_batch_pdhg.argtypes = [P(CSR), C.c_int, iptr, iptr, dptr, dptr, dptr, dptr, dptr,
                                              P(BatchSettings), dptr, dptr, P(BatchResult)]
    L.sankhya_b200_csr_transpose.argtypes = [P(CSR), iptr, iptr, dptr]
    if hasattr(L, "sankhya_b200_gnn_create"):
        L.sankhya_b200_gnn_default_settings.argtypes = [P(GnnSettings)]
        L.sankhya_b200_gnn_default_settings.restype = None
        L.sankhya_b200_gnn_create.argtypes = [P(GnnSettings), P(C.c_void_p)]
        L.sankhya_b200_gnn_destroy.argtypes = [C.c_void_p]
        L.sankhya_b200_gnn_destroy.restype = None
        L.sankhya_b200_gnn_parameter_count.argtypes = [C.c_void_p]
        fptr = P(C.c_float)
        L.sankhya_b200_gnn_get_parameters.argtypes = [C.c_void_p, fptr]
        L.sankhya_b200_gnn_set_parameters.argtypes = [C.c_void_p, fptr]
        L.sankhya_b200_gnn_predict.argtypes = [C.c_void_p, P(CSR), dptr, dptr, dptr, dptr, dptr, dptr, dptr]
        L.sankhya_b200_gnn_gradient.argtypes = [C.c_void_p, P(CSR), dptr, dptr, dptr, dptr, dptr, dptr, dptr,
                                                P(C.c_double), fptr]
        L.sankhya_b200_gnn_train_step.argtypes = [C.c_void_p, P(CSR), dptr, dptr, dptr, dptr, dptr, dptr, dptr,
                                                  P(C.c_double)]
    if hasattr(L, "sankhya_b200_shared_batch_pdhg"):
        L.sankhya_b200_shared_batch_pdhg.argtypes = [P(CSR), C.c_int, dptr, C.c_int, dptr, dptr, C.c_int, dptr,
                                                     dptr, C.c_int, P(BatchSettings), dptr, dptr, P(BatchResult)]


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return None if a is None else a.ctypes.data_as(dptr)


def last_error() -> str:
    return lib().sankhya_cuda_last_error().decode()


class Matrix:
    """A device-resident CSR made by sankhya_cuda_csr_create."""

    def __init__(self, rows, cols, ptr, idx, val):
        self.ptr = np.ascontiguousarray(ptr, dtype=np.int32)
        self.idx = np.ascontiguousarray(idx, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        self.handle = CSR()
        rc = lib().sankhya_cuda_csr_create(C.byref(self.handle), int(rows), int(cols), int(self.val.shape[0]),
                                           self.ptr.ctypes.data_as(iptr), self.idx.ctypes.data_as(iptr),
                                           self.val.ctypes.data_as(dptr))
        if rc != 0:
            raise RuntimeError(f"sankhya_cuda_csr_create failed: {last_error()}")

    @classmethod
    def from_instance(cls, inst, hessian=False):
        if hessian:
            return cls(inst["n"], inst["n"], inst["q_ptr"], inst["q_idx"], inst["q_val"])
        return cls(inst["m"], inst["n"], inst["ptr"], inst["idx"], inst["val"])

    def close(self):
        if self.handle is not None:
            lib().sankhya_cuda_csr_destroy(C.byref(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def settings(max_iterations=1000, check_every=10, tau=0.0, sigma=0.0, theta=1.0, tolerance=1e-6,
             time_limit=0.0) -> Settings:
    return Settings(max_iterations, check_every, tau, sigma, theta, tolerance, time_limit)


def _out(buf, length, name):
    """A caller's output array (float64, contiguous, `length` long), or a new one."""
    if buf is None:
        return np.zeros(length)
    if buf.dtype != np.float64 or not buf.flags["C_CONTIGUOUS"] or buf.shape != (length,):
        raise ValueError(f"{name} must be a contiguous float64 array of length {length}")
    return buf


def pdhg(matrix: Matrix, inst, s: Settings, hessian: Matrix | None = None, qdiag=None, primal_steps=None,
         dual_steps=None, want_dual=False, entry: str | None = None, x_out=None, y_out=None, **over):
    """Calls one of the five *_pdhg entry points; returns (rc, x, y, result). x and y
    are written into x_out / y_out when given (for example pinned host arrays, which
    the device-to-host copies reach fastest), else into new arrays."""
    L = lib()
    get = lambda k: _d(over[k]) if k in over else _d(inst[k])
    c, rl, ru, cl, cu = get("c"), get("rl"), get("ru"), get("cl"), get("cu")
    n, m = matrix.handle.cols, matrix.handle.rows
    x = _out(x_out, n, "x_out")
    y = _out(y_out, m, "y_out") if want_dual else None
    res = Result()
    qd, ps, ds = _d(qdiag), _d(primal_steps), _d(dual_steps)
    h = C.byref(hessian.handle) if hessian is not None else None
    if entry is None:
        if ps is not None:
            entry = "with_dual" if want_dual else "preconditioned"
        elif hessian is not None:
            entry = "sparse"
        elif qd is not None:
            entry = "diagonal"
        else:
            entry = "lp"
    if entry != "with_dual":
        y = None  # only the *_with_dual entry point returns multipliers
    M = C.byref(matrix.handle)
    if entry == "lp":
        rc = L.sankhya_cuda_lp_pdhg(M, _p(c), _p(rl), _p(ru), _p(cl), _p(cu), s, _p(x), C.byref(res))
    elif entry == "diagonal":
        rc = L.sankhya_cuda_diagonal_qp_pdhg(M, _p(qd), _p(c), _p(rl), _p(ru), _p(cl), _p(cu), s, _p(x),
                                             C.byref(res))
    elif entry == "sparse":
        rc = L.sankhya_cuda_sparse_qp_pdhg(M, h, _p(c), _p(rl), _p(ru), _p(cl), _p(cu), s, _p(x), C.byref(res))
    elif entry == "preconditioned":
        rc = L.sankhya_cuda_qp_pdhg_preconditioned(M, h, _p(qd), _p(c), _p(rl), _p(ru), _p(cl), _p(cu), _p(ps),
                                                   _p(ds), s, _p(x), C.byref(res))
    elif entry == "with_dual":
        rc = L.sankhya_cuda_qp_pdhg_preconditioned_with_dual(M, h, _p(qd), _p(c), _p(rl), _p(ru), _p(cl), _p(cu),
                                                             _p(ps), _p(ds), s, _p(x), _p(y), C.byref(res))
    else:
        raise ValueError(entry)
    return rc, x, y, res.as_dict()


def set_timing(level: int):
    lib().sankhya_b200_set_timing(int(level))


def last_timing() -> dict:
    t = Timing()
    lib().sankhya_b200_last_timing(C.byref(t))
    return t.as_dict()


def spmv_host(rows, cols, ptr, idx, val, x):
    y = np.zeros(rows)
    ptr = np.ascontiguousarray(ptr, dtype=np.int32)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    val, x = _d(val), _d(x)
    rc = lib().sankhya_cuda_spmv_f64(rows, cols, int(val.shape[0]), ptr.ctypes.data_as(iptr),
                                     idx.ctypes.data_as(iptr), _p(val), _p(x), _p(y))
    return rc, y


def axpy_host(alpha, x, y):
    x, y = _d(x), _d(y).copy()
    rc = lib().sankhya_cuda_axpy_f64(int(x.shape[0]), float(alpha), _p(x), _p(y))
    return rc, y


def pdlp_default_settings() -> PdlpSettings:
    s = PdlpSettings()
    lib().sankhya_b200_pdlp_default_settings(C.byref(s))
    return s


def pdlp_solve(matrix: Matrix, inst, s: PdlpSettings | None = None, x0=None, y0=None, want_dual=True, **over):
    L = lib()
    s = s or pdlp_default_settings()
    get = lambda k: _d(over[k]) if k in over else _d(inst[k])
    c, rl, ru, cl, cu = get("c"), get("rl"), get("ru"), get("cl"), get("cu")
    n, m = matrix.handle.cols, matrix.handle.rows
    x = np.zeros(n)
    y = np.zeros(m) if want_dual else None
    res = PdlpResult()
    rc = L.sankhya_b200_pdlp_solve(C.byref(matrix.handle), _p(c), _p(rl), _p(ru), _p(cl), _p(cu), C.byref(s),
                                   _p(_d(x0)), _p(_d(y0)), _p(x), _p(y), C.byref(res))
    return rc, x, y, res.as_dict()


def pdlp_solve_qp(matrix: Matrix, inst, s: PdlpSettings | None = None, hessian: Matrix | None = None, qdiag=None,
                  x0=None, y0=None, want_dual=True, **over):
    """sankhya_b200_pdlp_solve_qp: the restarted solve with x'Q x / 2 in the objective,
    Q a full symmetric Matrix (hessian) or its diagonal (qdiag)."""
    L = lib()
    s = s or pdlp_default_settings()
    get = lambda k: _d(over[k]) if k in over else _d(inst[k])
    c, rl, ru, cl, cu = get("c"), get("rl"), get("ru"), get("cl"), get("cu")
    n, m = matrix.handle.cols, matrix.handle.rows
    x = np.zeros(n)
    y = np.zeros(m) if want_dual else None
    res = PdlpResult()
    qd = _d(qdiag)
    rc = L.sankhya_b200_pdlp_solve_qp(C.byref(matrix.handle), C.byref(hessian.handle) if hessian is not None else None,
                                      _p(qd), _p(c), _p(rl), _p(ru), _p(cl), _p(cu), C.byref(s), _p(_d(x0)),
                                      _p(_d(y0)), _p(x), _p(y), C.byref(res))
    return rc, x, y, res.as_dict()


def polish_default_settings() -> PolishSettings:
    p = PolishSettings()
    lib().sankhya_b200_polish_default_settings(C.byref(p))
    return p


def pdlp_solve_polished(matrix: Matrix, inst, s: PdlpSettings | None = None, polish: PolishSettings | None = None,
                        x0=None, y0=None, want_dual=True, **over):
    """sankhya_b200_pdlp_solve_polished: the restarted FP64 solve with feasibility
    polishing; returns (rc, x, y, result, polish_result)."""
    L = lib()
    s = s or pdlp_default_settings()
    get = lambda k: _d(over[k]) if k in over else _d(inst[k])
    c, rl, ru, cl, cu = get("c"), get("rl"), get("ru"), get("cl"), get("cu")
    n, m = matrix.handle.cols, matrix.handle.rows
    x = np.zeros(n)
    y = np.zeros(m) if want_dual else None
    res, pres = PdlpResult(), PolishResult()
    rc = L.sankhya_b200_pdlp_solve_polished(C.byref(matrix.handle), _p(c), _p(rl), _p(ru), _p(cl), _p(cu),
                                            C.byref(s), C.byref(polish) if polish is not None else None,
                                            _p(_d(x0)), _p(_d(y0)), _p(x), _p(y), C.byref(res), C.byref(pres))
    return rc, x, y, res.as_dict(), pres.as_dict()


def scale_factors(matrix: Matrix, scaling: int, ruiz_iterations: int = 100, ruiz_tolerance: float = 1e-2):
    """Device equilibration factors (row_scale, col_scale) for a device matrix."""
    r = np.zeros(matrix.handle.rows)
    c = np.zeros(matrix.handle.cols)
    rc = lib().sankhya_b200_scale_factors(C.byref(matrix.handle), int(scaling), int(ruiz_iterations),
                                          float(ruiz_tolerance), _p(r), _p(c))
    return rc, r, c


def block_diagonal(instances_list):
    """Concatenates LP instance dicts into one block-diagonal instance plus the
    row / column segment offsets."""
    ptrs, idxs, vals = [np.zeros(1, dtype=np.int64)], [], []
    rseg, cseg = [0], [0]
    nz = 0
    for inst in instances_list:
        ptrs.append(inst["ptr"][1:].astype(np.int64) + nz)
        idxs.append(inst["idx"].astype(np.int64) + cseg[-1])
        vals.append(inst["val"])
        nz += int(inst["ptr"][-1])
        rseg.append(rseg[-1] + inst["m"])
        cseg.append(cseg[-1] + inst["n"])
    cat = lambda k: np.concatenate([i[k] for i in instances_list])
    out = dict(m=rseg[-1], n=cseg[-1], ptr=np.concatenate(ptrs).astype(np.int32),
               idx=np.concatenate(idxs).astype(np.int32), val=np.concatenate(vals),
               c=cat("c"), rl=cat("rl"), ru=cat("ru"), cl=cat("cl"), cu=cat("cu"))
    return out, np.asarray(rseg, dtype=np.int32), np.asarray(cseg, dtype=np.int32)


def batch_default_settings() -> BatchSettings:
    s = BatchSettings()
    lib().sankhya_b200_batch_default_settings(C.byref(s))
    return s


def batch_pdhg(matrix: Matrix, inst, row_segments, col_segments, s: BatchSettings | None = None, want_dual=False):
    """Batched sk_solve-style PDHG over a block-diagonal matrix; returns (rc, x, y, results list)."""
    s = s or batch_default_settings()
    rseg = np.ascontiguousarray(row_segments, dtype=np.int32)
    cseg = np.ascontiguousarray(col_segments, dtype=np.int32)
    k = rseg.shape[0] - 1
    x = np.zeros(matrix.handle.cols)
    y = np.zeros(matrix.handle.rows) if want_dual else None
    res = (BatchResult * k)()
    rc = lib().sankhya_b200_batch_pdhg(C.byref(matrix.handle), k, rseg.ctypes.data_as(iptr), cseg.ctypes.data_as(iptr),
                                       _p(_d(inst["c"])), _p(_d(inst["rl"])), _p(_d(inst["ru"])), _p(_d(inst["cl"])),
                                       _p(_d(inst["cu"])), C.byref(s), _p(x), _p(y), res)
    return rc, x, y, [{f: getattr(r, f) for f, _ in BatchResult._fields_} for r in res]


def shared_batch_pdhg(matrix: Matrix, batch: int, c, rl, ru, cl, cu, s: BatchSettings | None = None,
                      want_dual=False):
    """Batched sk_solve-style PDHG over LPs sharing `matrix`. Each of c, (rl, ru),
    (cl, cu) is either one vector shared by all LPs or a (batch, len) array.
    Returns (rc, x[batch, n], y[batch, m] or None, results list)."""
    s = s or batch_default_settings()
    m, n = matrix.handle.rows, matrix.handle.cols

    def arr(v, length):
        a = np.ascontiguousarray(v, dtype=np.float64)
        per = a.ndim == 2
        if per:
            assert a.shape == (batch, length)
        else:
            assert a.shape == (length,)
        return a, int(per)

    c_, cp = arr(c, n)
    rl_, rp = arr(rl, m)
    ru_, rp2 = arr(ru, m)
    cl_, kp = arr(cl, n)
    cu_, kp2 = arr(cu, n)
    assert rp == rp2 and kp == kp2, "lower and upper bounds must both be shared or both per LP"
    x = np.zeros((batch, n))
    y = np.zeros((batch, m)) if want_dual else None
    res = (BatchResult * batch)()
    rc = lib().sankhya_b200_shared_batch_pdhg(C.byref(matrix.handle), batch, _p(c_), cp, _p(rl_), _p(ru_), rp,
                                              _p(cl_), _p(cu_), kp, C.byref(s), _p(x), _p(y), res)
    return rc, x, y, [{f: getattr(r, f) for f, _ in BatchResult._fields_} for r in res]



class Gnn:
    """The warm-start network (sankhya_b200_gnn_*): predicts (x, y) for an LP of
    a family that shares one matrix; trained on (instance, solution) pairs."""

    def __init__(self, rounds=4, seed=1, learning_rate=1e-3, y_scale=1.0):
        st = GnnSettings()
        lib().sankhya_b200_gnn_default_settings(C.byref(st))
        st.rounds, st.seed, st.learning_rate, st.y_scale = rounds, seed, learning_rate, y_scale
        self.settings = st
        self.handle = C.c_void_p()
        rc = lib().sankhya_b200_gnn_create(C.byref(st), C.byref(self.handle))
        if rc != 0:
            raise RuntimeError(last_error())
        self.count = lib().sankhya_b200_gnn_parameter_count(self.handle)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and _lib is not None:
            _lib.sankhya_b200_gnn_destroy(h)
            self.handle = None

    def parameters(self):
        out = np.zeros(self.count, dtype=np.float32)
        if lib().sankhya_b200_gnn_get_parameters(self.handle, out.ctypes.data_as(C.POINTER(C.c_float))):
            raise RuntimeError(last_error())
        return out

    def set_parameters(self, theta):
        t = np.ascontiguousarray(theta, dtype=np.float32)
        assert t.shape == (self.count,)
        if lib().sankhya_b200_gnn_set_parameters(self.handle, t.ctypes.data_as(C.POINTER(C.c_float))):
            raise RuntimeError(last_error())

    @staticmethod
    def _model(inst):
        return [_d(inst[k]) for k in ("c", "rl", "ru", "cl", "cu")]

    def predict(self, matrix: Matrix, inst):
        c, rl, ru, cl, cu = self._model(inst)
        x = np.zeros(matrix.handle.cols)
        y = np.zeros(matrix.handle.rows)
        rc = lib().sankhya_b200_gnn_predict(self.handle, C.byref(matrix.handle), _p(c), _p(rl), _p(ru), _p(cl), _p(cu),
                                            _p(x), _p(y))
        if rc != 0:
            raise RuntimeError(last_error())
        return x, y

    def gradient(self, matrix: Matrix, inst, x_target, y_target):
        c, rl, ru, cl, cu = self._model(inst)
        xt, yt = _d(x_target), _d(y_target)
        loss = C.c_double()
        g = np.zeros(self.count, dtype=np.float32)
        rc = lib().sankhya_b200_gnn_gradient(self.handle, C.byref(matrix.handle), _p(c), _p(rl), _p(ru), _p(cl),
                                             _p(cu), _p(xt), _p(yt), C.byref(loss),
                                             g.ctypes.data_as(C.POINTER(C.c_float)))
        if rc != 0:
            raise RuntimeError(last_error())
        return loss.value, g

    def train_step(self, matrix: Matrix, inst, x_target, y_target):
        c, rl, ru, cl, cu = self._model(inst)
        xt, yt = _d(x_target), _d(y_target)
        loss = C.c_double()
        rc = lib().sankhya_b200_gnn_train_step(self.handle, C.byref(matrix.handle), _p(c), _p(rl), _p(ru), _p(cl),
                                               _p(cu), _p(xt), _p(yt), C.byref(loss))
        if rc != 0:
            raise RuntimeError(last_error())
        return loss.value


def csr_transpose(matrix: Matrix):
    """The engine's stored transpose of `matrix` (A in CSC form): (ptr, idx, val)."""
    h = matrix.handle
    ptr = np.zeros(h.cols + 1, dtype=np.int32)
    idx = np.zeros(max(h.nnz, 1), dtype=np.int32)
    val = np.zeros(max(h.nnz, 1))
    rc = lib().sankhya_b200_csr_transpose(C.byref(h), ptr.ctypes.data_as(iptr), idx.ctypes.data_as(iptr), _p(val))
    if rc != 0:
        raise RuntimeError(last_error())
    return ptr, idx[:h.nnz], val[:h.nnz]
