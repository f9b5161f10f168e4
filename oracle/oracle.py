"""ctypes bindings for the checkers in this folder.

TEST INFRASTRUCTURE ONLY. Imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py; the product never imports it.

  liboracle.so                  C restatement of the reference path (pdhg_oracle.c)
  _ref/libsankhya_ref.so        the reference's own C core (sk_solve, sk_verify, ...)
  _ref/libsankhya_ref_omp.so    the same core built with OpenMP (same bits, threaded csc_tmv)
  _ref/libsihps_scaling_ref.so  the reference C++ core's Ruiz / Pock-Chambolle (src/lp/Scaling.cpp)
  _ref/libsihps_pdlp_ref.so     the reference C++ core's GPU PDLP (src/cuda/GpuPdlp.cpp), needs a GPU
  _ref/libsankhya_ref_hooked.so the C core with include/integration/sk_solve_hook.inc applied, calling the engine
  _ref/libsankhya_cuda_ref.so   the reference's CUDA prototype built for sm_100a
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_libs: dict[str, C.CDLL] = {}

dptr = C.POINTER(C.c_double)
iptr = C.POINTER(C.c_int)


def _as_d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _as_i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _p(a, t=dptr):
    return None if a is None else a.ctypes.data_as(t)


def load(name: str) -> C.CDLL:
    if name not in _libs:
        path = {"oracle": os.path.join(HERE, "liboracle.so"),
                "ref": os.path.join(HERE, "_ref", "libsankhya_ref.so"),
                "ref_omp": os.path.join(HERE, "_ref", "libsankhya_ref_omp.so"),
                "ref_scaling": os.path.join(HERE, "_ref", "libsihps_scaling_ref.so"),
                "ref_pdlp": os.path.join(HERE, "_ref", "libsihps_pdlp_ref.so"),
                "ref_hooked": os.path.join(HERE, "_ref", "libsankhya_ref_hooked.so"),
                "ref_milp_hooked": os.path.join(HERE, "_ref", "libsankhya_ref_milp_hooked.so"),
                "ref_lp": os.path.join(HERE, "_ref", "libsihps_lp_ref.so"),
                "ref_lp_hooked": os.path.join(HERE, "_ref", "libsihps_lp_hooked.so"),
                "ref_cuda": os.path.join(HERE, "_ref", "libsankhya_cuda_ref.so"),
                "ref_crossover": os.path.join(HERE, "_ref", "libsk_crossover_ref.so"),
                "ref_sihps_crossover": os.path.join(HERE, "_ref", "libsihps_crossover_ref.so"),
                "ref_lp_cpu": os.path.join(HERE, "_ref", "libsihps_lp_cpu.so"),
                "ref_lp_hybrid_cpu": os.path.join(HERE, "_ref", "libsihps_lp_hybrid_cpu.so")}[name]
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle {'ref' if name != 'oracle' else ''})")
        _libs[name] = C.CDLL(path)
    return _libs[name]


def available(name: str) -> bool:
    try:
        load(name)
        return True
    except (FileNotFoundError, OSError):
        return False


# ---------------------------------------------------------------- oracle structs

class OrcCsr(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("ptr", iptr), ("idx", iptr), ("val", dptr)]


class LPSettings(C.Structure):
    """Layout of SankhyaCudaLPSettings (and orc_settings)."""
    _fields_ = [("max_iterations", C.c_int), ("check_every", C.c_int), ("tau", C.c_double),
                ("sigma", C.c_double), ("theta", C.c_double), ("tolerance", C.c_double),
                ("time_limit", C.c_double)]


class LPResult(C.Structure):
    """Layout of SankhyaCudaLPResult (and orc_result)."""
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("objective", C.c_double),
                ("maximum_row_violation", C.c_double), ("maximum_step", C.c_double),
                ("maximum_kkt_residual", C.c_double), ("maximum_dual_residual", C.c_double),
                ("maximum_complementarity", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SkOut(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("dual_step", C.c_double),
                ("anorm", C.c_double)]


class Verify(C.Structure):
    _fields_ = [("objective", C.c_double), ("primal_infeasibility", C.c_double),
                ("dual_infeasibility", C.c_double), ("complementarity", C.c_double)]


class PdlpParams(C.Structure):
    _fields_ = [("eps_optimal", C.c_double), ("max_iterations", C.c_int),
                ("restart_period", C.c_int), ("power_iterations", C.c_int),
                ("adaptive_step", C.c_int), ("eta_min_factor", C.c_double),
                ("eta_max_factor", C.c_double)]


class PdlpStats(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("restarts", C.c_int),
                ("rejected_steps", C.c_int), ("primal_objective", C.c_double),
                ("dual_objective", C.c_double), ("relative_primal_residual", C.c_double),
                ("relative_dual_residual", C.c_double), ("relative_gap", C.c_double),
                ("matrix_norm", C.c_double), ("final_step_size", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class _Keep:
    """Holds numpy buffers alive while a ctypes struct points into them."""

    def __init__(self):
        self.refs = []

    def d(self, a):
        a = _as_d(a)
        self.refs.append(a)
        return a

    def i(self, a):
        a = _as_i(a)
        self.refs.append(a)
        return a


def _csr(keep: _Keep, rows, cols, ptr, idx, val) -> OrcCsr:
    return OrcCsr(rows, cols, _p(keep.i(ptr), iptr), _p(keep.i(idx), iptr), _p(keep.d(val)))


def inst_csr(keep, inst):
    return _csr(keep, inst["m"], inst["n"], inst["ptr"], inst["idx"], inst["val"])


def hessian_csr(keep, inst):
    if "q_ptr" not in inst:
        return None
    n = inst["n"]
    return _csr(keep, n, n, inst["q_ptr"], inst["q_idx"], inst["q_val"])


def fixed_pdhg(inst, settings: dict, primal_steps=None, dual_steps=None, qdiag=None,
               hessian=False, want_dual=True, **over):
    """orc_fixed_pdhg: the cuda prototype's solve_qp restated. Returns (rc, x, y, result)."""
    lib = load("oracle")
    keep = _Keep()
    a = inst_csr(keep, inst)
    h = hessian_csr(keep, inst) if hessian else None
    get = lambda k: keep.d(over[k]) if k in over else keep.d(inst[k])
    x = np.zeros(inst["n"])
    y = np.zeros(inst["m"]) if want_dual else None
    res = LPResult()
    s = LPSettings(**settings)
    lib.orc_fixed_pdhg.restype = C.c_int
    rc = lib.orc_fixed_pdhg(C.byref(a), C.byref(h) if h is not None else None,
                            _p(keep.d(qdiag)) if qdiag is not None else None,
                            _p(get("c")), _p(get("rl")), _p(get("ru")), _p(get("cl")), _p(get("cu")),
                            s, _p(keep.d(primal_steps)) if primal_steps is not None else None,
                            _p(keep.d(dual_steps)) if dual_steps is not None else None,
                            _p(x), _p(y), C.byref(res))
    return rc, x, y, res.as_dict()


def sk_loop(inst, max_iterations, primal_tol=1e-7, dual_tol=1e-7, time_limit=0.0, quadratic=False):
    lib = load("oracle")
    keep = _Keep()
    a = inst_csr(keep, inst)
    q = hessian_csr(keep, inst) if quadratic else None
    n, m = inst["n"], inst["m"]
    x, y, act = np.zeros(n), np.zeros(m), np.zeros(m)
    out = SkOut()
    rc = lib.orc_sk_loop(C.byref(a), C.byref(q) if q is not None else None,
                         _p(keep.d(inst["c"])), _p(keep.d(inst["rl"])), _p(keep.d(inst["ru"])),
                         _p(keep.d(inst["cl"])), _p(keep.d(inst["cu"])), C.c_int(max_iterations),
                         C.c_double(primal_tol), C.c_double(dual_tol), C.c_double(time_limit),
                         _p(x), _p(y), _p(act), C.byref(out))
    assert rc == 0
    return x, y, act, {k: getattr(out, k) for k, _ in SkOut._fields_}


def sk_verify(inst, x, y, quadratic=False, objshift=0.0):
    lib = load("oracle")
    keep = _Keep()
    a = inst_csr(keep, inst)
    q = hessian_csr(keep, inst) if quadratic else None
    v = Verify()
    lib.orc_sk_verify(C.byref(a), C.byref(q) if q is not None else None, _p(keep.d(inst["c"])),
                      C.c_double(objshift), _p(keep.d(inst["rl"])), _p(keep.d(inst["ru"])),
                      _p(keep.d(inst["cl"])), _p(keep.d(inst["cu"])), _p(keep.d(x)),
                      _p(keep.d(y)) if y is not None else None, C.byref(v))
    return {k: getattr(v, k) for k, _ in Verify._fields_}


def pdlp(inst, eps=1e-8, max_iterations=100000, restart_period=64, power_iterations=30,
         adaptive=True, eta_min_factor=1e-6, eta_max_factor=1e4):
    lib = load("oracle")
    keep = _Keep()
    a = inst_csr(keep, inst)
    p = PdlpParams(eps, max_iterations, restart_period, power_iterations, int(adaptive),
                   eta_min_factor, eta_max_factor)
    x, y = np.zeros(inst["n"]), np.zeros(inst["m"])
    st = PdlpStats()
    lib.orc_pdlp(C.byref(a), _p(keep.d(inst["c"])), _p(keep.d(inst["cl"])), _p(keep.d(inst["cu"])),
                 _p(keep.d(inst["rl"])), _p(keep.d(inst["ru"])), C.byref(p), _p(x), _p(y),
                 C.byref(st))
    return x, y, st.as_dict()


def power_norm(inst, iterations=30):
    lib = load("oracle")
    keep = _Keep()
    a = inst_csr(keep, inst)
    lib.orc_power_norm.restype = C.c_double
    return lib.orc_power_norm(C.byref(a), C.c_int(iterations))


def ruiz(inst, max_iters=100, tol=1e-2):
    lib = load("oracle")
    keep = _Keep()
    a = inst_csr(keep, inst)
    r, c = np.zeros(inst["m"]), np.zeros(inst["n"])
    conv = lib.orc_ruiz(C.byref(a), C.c_int(max_iters), C.c_double(tol), _p(r), _p(c))
    return r, c, bool(conv)


def pock_chambolle(inst, alpha=1.0):
    lib = load("oracle")
    keep = _Keep()
    a = inst_csr(keep, inst)
    r, c = np.zeros(inst["m"]), np.zeros(inst["n"])
    lib.orc_pock_chambolle(C.byref(a), C.c_double(alpha), _p(r), _p(c))
    return r, c


def _ref_scaling_call(name, inst, *args):
    lib = load("ref_scaling")
    keep = _Keep()
    ptr, idx, val = keep.i(inst["ptr"]), keep.i(inst["idx"]), keep.d(inst["val"])
    r, c = np.zeros(inst["m"]), np.zeros(inst["n"])
    fn = getattr(lib, name)
    fn.restype = C.c_int
    rc = fn(C.c_int(inst["m"]), C.c_int(inst["n"]), C.c_int(int(inst["ptr"][-1])), _p(ptr, iptr), _p(idx, iptr),
            _p(val), *args, _p(r), _p(c))
    if rc != 0:
        raise ValueError(f"{name} rejected the matrix")
    return r, c


def ref_ruiz(inst, max_iters=100, tol=1e-2):
    """The reference's compute_ruiz_scaling (src/lp/Scaling.cpp): (row_scale, col_scale)."""
    return _ref_scaling_call("ref_ruiz_scaling", inst, C.c_int(max_iters), C.c_double(tol))


def ref_pock_chambolle(inst, alpha=1.0):
    """The reference's compute_pock_chambolle_scaling (src/lp/Scaling.cpp)."""
    return _ref_scaling_call("ref_pock_chambolle_scaling", inst, C.c_double(alpha))


class RefPdlpParams(C.Structure):
    """RefPdlpParams of ref_pdlp_shim.cpp (the reference's PdlpParams, plus `scale`)."""
    _fields_ = [("eps_optimal", C.c_double), ("max_iterations", C.c_int), ("restart_period", C.c_int),
                ("time_limit_seconds", C.c_double), ("power_iterations", C.c_int), ("adaptive_step", C.c_int),
                ("eta_min_factor", C.c_double), ("eta_max_factor", C.c_double), ("scale", C.c_int),
                ("reserved", C.c_int)]


class RefPdlpStats(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("restarts", C.c_int),
                ("rejected_steps", C.c_int), ("host_syncs", C.c_int), ("reserved", C.c_int),
                ("primal_objective", C.c_double), ("dual_objective", C.c_double),
                ("relative_primal_residual", C.c_double), ("relative_dual_residual", C.c_double),
                ("relative_gap", C.c_double), ("matrix_norm", C.c_double), ("seconds", C.c_double)]


def ref_gpupdlp(inst, eps=1e-8, max_iterations=500000, restart_period=64, power_iterations=30, adaptive=True,
                eta_min_factor=1e-6, eta_max_factor=1e4, time_limit=0.0, scale=True):
    """The reference's own GPU PDLP (GpuPdlp, with run_first_order's scaling when `scale`)
    on the current CUDA device: (x, stats dict). Needs a GPU."""
    lib = load("ref_pdlp")
    keep = _Keep()
    p = RefPdlpParams(eps, max_iterations, restart_period, time_limit, power_iterations, int(adaptive),
                      eta_min_factor, eta_max_factor, int(scale), 0)
    st = RefPdlpStats()
    x = np.zeros(inst["n"])
    fn = lib.ref_gpupdlp_solve
    fn.restype = C.c_int
    rc = fn(C.c_int(inst["m"]), C.c_int(inst["n"]), C.c_int(int(inst["ptr"][-1])), _p(keep.i(inst["ptr"]), iptr),
            _p(keep.i(inst["idx"]), iptr), _p(keep.d(inst["val"])), _p(keep.d(inst["c"])), _p(keep.d(inst["cl"])),
            _p(keep.d(inst["cu"])), _p(keep.d(inst["rl"])), _p(keep.d(inst["ru"])), C.byref(p), _p(x), C.byref(st))
    if rc != 0:
        raise RuntimeError("reference GpuPdlp failed")
    return x, {k: getattr(st, k) for k, _ in RefPdlpStats._fields_}


class RefLpOptions(C.Structure):
    """RefLpOptions of ref_lpsolver_shim.cpp (a subset of sihps::LpSolverOptions)."""
    _fields_ = [("method", C.c_int), ("use_presolve", C.c_int), ("hybrid_row_threshold", C.c_int),
                ("pdlp_max_iterations", C.c_int), ("pdlp_eps", C.c_double), ("pdlp_time_limit", C.c_double),
                ("hybrid_first_order_eps", C.c_double), ("hybrid_first_order_budget", C.c_double),
                ("hybrid_simplex_budget", C.c_double)]


class RefLpResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("used_first_order", C.c_int),
                ("first_order_fallback_used", C.c_int), ("pdlp_converged", C.c_int), ("pdlp_iterations", C.c_int),
                ("objective", C.c_double), ("primal_residual", C.c_double), ("pdlp_relative_gap", C.c_double),
                ("solve_seconds", C.c_double)]


LP_SIMPLEX, LP_FIRST_ORDER, LP_HYBRID = 0, 1, 2
LP_STATUS = ("OPTIMAL", "INFEASIBLE", "UNBOUNDED", "ITERATION_LIMIT", "NUMERICAL_FAILURE")


def ref_solve_lp(inst, method=LP_SIMPLEX, hooked=False, lib_name=None, **opts):
    """The reference C++ core's sihps::solve_lp (src/lp/LpSolver.cpp:126-334) on the
    instance: (x, result dict). `hooked` selects the build whose run_first_order is the
    integration block calling the engine; otherwise FIRST_ORDER runs the reference's own
    GpuPdlp. `lib_name` picks another build ("ref_lp_cpu", "ref_lp_hybrid_cpu": the
    integration blocks over the CPU stand-in engine). Keyword options are RefLpOptions
    fields; the rest keep the core's defaults. SIMPLEX runs on the CPU; FIRST_ORDER and
    HYBRID need a GPU, except through the stand-in builds."""
    lib = load(lib_name or ("ref_lp_hooked" if hooked else "ref_lp"))
    o = RefLpOptions()
    lib.ref_lp_default_options(C.byref(o))
    o.method = method
    for k, v in opts.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    keep = _Keep()
    r = RefLpResult()
    x = np.zeros(inst["n"])
    fn = lib.ref_solve_lp
    fn.restype = C.c_int
    rc = fn(C.c_int(inst["m"]), C.c_int(inst["n"]), C.c_int(int(inst["ptr"][-1])), _p(keep.i(inst["ptr"]), iptr),
            _p(keep.i(inst["idx"]), iptr), _p(keep.d(inst["val"])), _p(keep.d(inst["c"])), _p(keep.d(inst["cl"])),
            _p(keep.d(inst["cu"])), _p(keep.d(inst["rl"])), _p(keep.d(inst["ru"])), C.byref(o), _p(x), C.byref(r))
    if rc != 0:
        raise RuntimeError("reference solve_lp threw")
    out = {k: getattr(r, k) for k, _ in RefLpResult._fields_}
    out["status_name"] = LP_STATUS[out["status"]] if 0 <= out["status"] < len(LP_STATUS) else str(out["status"])
    return x, out


class RefCudaCsr(C.Structure):
    """Layout of the reference's SankhyaCudaCSR (cuda/include/sankhya_cuda.h)."""
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("nnz", C.c_int), ("device_row_offsets", C.c_void_p),
                ("device_column_indices", C.c_void_p), ("device_values", C.c_void_p)]


class RefCudaPrototype:
    """The reference's CUDA prototype (cuda/src/sankhya_cuda*.cu built for sm_100a into
    _ref/libsankhya_cuda_ref.so) holding one matrix on the current device; `pdhg` is its
    sankhya_cuda_qp_pdhg_preconditioned (LP: no Hessian, no diagonal). Needs a GPU."""

    def __init__(self, inst):
        L = load("ref_cuda")
        P = C.POINTER
        L.sankhya_cuda_csr_create.argtypes = [P(RefCudaCsr), C.c_int, C.c_int, C.c_int, iptr, iptr, dptr]
        L.sankhya_cuda_csr_destroy.argtypes = [P(RefCudaCsr)]
        L.sankhya_cuda_csr_destroy.restype = None
        L.sankhya_cuda_qp_pdhg_preconditioned.argtypes = [P(RefCudaCsr), P(RefCudaCsr), dptr, dptr, dptr, dptr,
                                                          dptr, dptr, dptr, dptr, LPSettings, dptr, P(LPResult)]
        L.sankhya_cuda_last_error.restype = C.c_char_p
        self.L = L
        self.keep = _Keep()
        self.h = RefCudaCsr()
        k = self.keep
        rc = L.sankhya_cuda_csr_create(C.byref(self.h), inst["m"], inst["n"], int(inst["ptr"][-1]),
                                       _p(k.i(inst["ptr"]), iptr), _p(k.i(inst["idx"]), iptr), _p(k.d(inst["val"])))
        if rc != 0:
            raise RuntimeError("reference sankhya_cuda_csr_create failed: " + L.sankhya_cuda_last_error().decode())
        self.arrays = {name: k.d(inst[name]) for name in ("c", "rl", "ru", "cl", "cu")}
        self.n = inst["n"]

    def pdhg(self, settings: dict, primal_steps, dual_steps):
        a, k = self.arrays, self.keep
        x = np.zeros(self.n)
        res = LPResult()
        rc = self.L.sankhya_cuda_qp_pdhg_preconditioned(
            C.byref(self.h), None, None, _p(a["c"]), _p(a["rl"]), _p(a["ru"]), _p(a["cl"]), _p(a["cu"]),
            _p(k.d(primal_steps)), _p(k.d(dual_steps)), LPSettings(**settings), _p(x), C.byref(res))
        return rc, x, res.as_dict()

    def close(self):
        if self.h is not None:
            self.L.sankhya_cuda_csr_destroy(C.byref(self.h))
            self.h = None


def pow2_scale(inst, passes=4):
    lib = load("oracle")
    keep = _Keep()
    a = inst_csr(keep, inst)
    r, c = np.zeros(inst["m"]), np.zeros(inst["n"])
    lib.orc_pow2_scale(C.byref(a), C.c_int(passes), _p(r), _p(c))
    return r, c


# ------------------------------------------------------- the reference's C core

class SkCsc(C.Structure):
    _fields_ = [("nrow", C.c_int), ("ncol", C.c_int), ("p", iptr), ("i", iptr), ("x", dptr),
                ("nzmax", C.c_int)]


class SkModel(C.Structure):
    _fields_ = [("nrow", C.c_int), ("ncol", C.c_int), ("A", SkCsc), ("Q", C.POINTER(SkCsc)),
                ("c", dptr), ("rlow", dptr), ("rupp", dptr), ("clow", dptr), ("cupp", dptr),
                ("vartype", C.POINTER(C.c_ubyte)), ("objshift", C.c_double),
                ("objsense", C.c_double), ("rowname", C.c_void_p), ("colname", C.c_void_p),
                ("name", C.c_char_p)]


class SkOptions(C.Structure):
    _fields_ = [("primal_tol", C.c_double), ("dual_tol", C.c_double), ("pivot_tol", C.c_double),
                ("time_limit", C.c_double), ("iteration_limit", C.c_longlong),
                ("node_limit", C.c_longlong), ("presolve", C.c_int), ("scaling", C.c_int),
                ("refactor_interval", C.c_int), ("verbosity", C.c_int), ("threads", C.c_int),
                ("mip_gap_abs", C.c_double), ("mip_gap_rel", C.c_double), ("mip_cuts", C.c_int),
                ("mip_heuristics", C.c_int), ("dual_simplex", C.c_int), ("lp_engine", C.c_int),
                ("random_seed", C.c_ulonglong)]


class SkSolution(C.Structure):
    _fields_ = [("result", C.c_int), ("objective", C.c_double), ("x", dptr), ("y", dptr),
                ("rc", dptr), ("rowact", dptr), ("ncol", C.c_int), ("nrow", C.c_int),
                ("iterations", C.c_longlong), ("nodes", C.c_longlong),
                ("solve_seconds", C.c_double), ("primal_infeasibility", C.c_double),
                ("dual_infeasibility", C.c_double), ("complementarity", C.c_double),
                ("mip_gap", C.c_double), ("dual_bound", C.c_double)]


SK_LP_FIRST_ORDER = 2


def build_sk_model(keep: _Keep, inst, quadratic=False):
    """An sk_model view over an instance dict (A converted to CSC)."""
    import importlib.util
    m, n = inst["m"], inst["n"]
    if "csc" not in inst:
        rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(inst["ptr"]))
        order = np.argsort(inst["idx"], kind="stable")
        cp = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(inst["idx"], minlength=n), out=cp[1:])
        inst["csc"] = (cp.astype(np.int32), rows[order].astype(np.int32), inst["val"][order].copy())
    cp, ci, cx = inst["csc"]
    model = SkModel()
    model.nrow, model.ncol = m, n
    nnz = int(cp[-1])
    model.A = SkCsc(m, n, _p(keep.i(cp), iptr), _p(keep.i(ci), iptr), _p(keep.d(cx)), max(nnz, 1))
    if quadratic and "q_ptr" in inst:
        q = SkCsc(n, n, _p(keep.i(inst["q_ptr"]), iptr), _p(keep.i(inst["q_idx"]), iptr),
                  _p(keep.d(inst["q_val"])), max(int(inst["q_ptr"][-1]), 1))
        keep.refs.append(q)
        model.Q = C.pointer(q)
    for k, f in (("c", "c"), ("rl", "rlow"), ("ru", "rupp"), ("cl", "clow"), ("cu", "cupp")):
        setattr(model, f, _p(keep.d(inst[k])))
    vt = np.zeros(max(n, 1), dtype=np.uint8)
    if "vartype" in inst:   # SK_INTEGER (1) marks the integer columns of a MILP
        vt[:n] = np.asarray(inst["vartype"], dtype=np.uint8)
    keep.refs.append(vt)
    model.vartype = vt.ctypes.data_as(C.POINTER(C.c_ubyte))
    model.objshift = 0.0
    model.objsense = 1.0
    return model


def ref_options(primal_tol=1e-7, dual_tol=1e-7, iteration_limit=0, time_limit=0.0,
                lp_engine=SK_LP_FIRST_ORDER, threads=1, lib_name="ref"):
    lib = load(lib_name)
    o = SkOptions()
    lib.sk_options_default(C.byref(o))
    o.primal_tol, o.dual_tol = primal_tol, dual_tol
    o.iteration_limit, o.time_limit = iteration_limit, time_limit
    o.lp_engine, o.threads, o.verbosity = lp_engine, threads, 0
    return o


def reference_tree():
    """The reference checkout the checkers are built from, or None where it is absent:
    $SANKHYA_REFERENCE, else the location oracle/Makefile builds from by default."""
    import subprocess
    path = os.environ.get("SANKHYA_REFERENCE")
    if not path:
        r = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True)
        path = r.stdout.strip() if r.returncode == 0 else ""
    return path if path and os.path.isfile(os.path.join(path, "c", "src", "sk_solve.c")) else None


def ref_sk_solve(inst, quadratic=False, lib_name="ref", **opts):
    """Runs the reference's sk_solve; returns (status, dict with x, y, rowact, fields).
    lib_name "ref_omp" runs the OpenMP build (give `threads`)."""
    lib = load(lib_name)
    keep = _Keep()
    model = build_sk_model(keep, inst, quadratic)
    o = ref_options(lib_name=lib_name, **opts)
    s = SkSolution()
    lib.sk_solution_init(C.byref(s))
    st = lib.sk_solve(C.byref(model), C.byref(o), C.byref(s))
    out = {k: getattr(s, k) for k, _ in SkSolution._fields_ if k not in ("x", "y", "rc", "rowact")}
    n, m = inst["n"], inst["m"]
    out["x"] = np.ctypeslib.as_array(s.x, (n,)).copy() if s.x and n else np.zeros(n)
    out["y"] = np.ctypeslib.as_array(s.y, (m,)).copy() if s.y and m else np.zeros(m)
    out["rowact"] = np.ctypeslib.as_array(s.rowact, (m,)).copy() if s.rowact and m else np.zeros(m)
    lib.sk_solution_free(C.byref(s))
    return st, out


def ref_sk_verify(inst, x, y, quadratic=False):
    lib = load("ref")
    keep = _Keep()
    model = build_sk_model(keep, inst, quadratic)
    s = SkSolution()
    lib.sk_solution_init(C.byref(s))
    xs = keep.d(x)
    s.x = _p(xs)
    if y is not None:
        s.y = _p(keep.d(y))
    st = lib.sk_verify(C.byref(model), C.byref(s))
    return st, {"objective": s.objective, "primal_infeasibility": s.primal_infeasibility,
                "dual_infeasibility": s.dual_infeasibility, "complementarity": s.complementarity}


def ref_read_mps(path):
    """The reference's own MPS/QPS reader (sk_read_mps, c/src/sk_core.c): the model as
    an instance dict (A in CSR with ascending columns per row, the counting-sort order of
    the reference's apps/*.cu csc_to_csr), plus Q as full symmetric CSR when present.
    Infinite bounds come back as +-inf (the reader's 1e30 sentinels converted)."""
    lib = load("ref")
    model = SkModel()
    lib.sk_model_init(C.byref(model))
    st = lib.sk_read_mps(path.encode(), C.byref(model))
    if st != 0:
        lib.sk_model_free(C.byref(model))
        raise ValueError(f"sk_read_mps({path}) returned {st}")
    try:
        m, n = model.nrow, model.ncol
        nnz = model.A.p[n]
        cp = np.ctypeslib.as_array(model.A.p, (n + 1,)).copy()
        ci = np.ctypeslib.as_array(model.A.i, (nnz,)).copy() if nnz else np.zeros(0, np.int32)
        cx = np.ctypeslib.as_array(model.A.x, (nnz,)).copy() if nnz else np.zeros(0)

        def csr(rows_, cols_, p_, i_, x_):
            cnt = np.bincount(i_, minlength=rows_) if len(i_) else np.zeros(rows_, np.int64)
            ptr = np.zeros(rows_ + 1, np.int32)
            np.cumsum(cnt, out=ptr[1:])
            col = np.repeat(np.arange(cols_, dtype=np.int32), np.diff(p_))
            order = np.argsort(i_, kind="stable")
            return ptr, col[order].astype(np.int32), x_[order].copy()

        def vec(ptr_, k):
            v = np.ctypeslib.as_array(ptr_, (k,)).copy() if k else np.zeros(0)
            v[v >= 1e30] = np.inf
            v[v <= -1e30] = -np.inf
            return v

        ptr, idx, val = csr(m, n, cp, ci, cx)
        inst = dict(m=m, n=n, ptr=ptr, idx=idx, val=val, c=vec(model.c, n), rl=vec(model.rlow, m),
                    ru=vec(model.rupp, m), cl=vec(model.clow, n), cu=vec(model.cupp, n),
                    objshift=model.objshift,
                    integer=np.ctypeslib.as_array(model.vartype, (n,)).copy() if n else np.zeros(0, np.uint8))
        if model.Q:
            q = model.Q.contents
            qn = q.p[n]
            qp = np.ctypeslib.as_array(q.p, (n + 1,)).copy()
            inst["q_ptr"], inst["q_idx"], inst["q_val"] = csr(
                n, n, qp, np.ctypeslib.as_array(q.i, (qn,)).copy(), np.ctypeslib.as_array(q.x, (qn,)).copy())
        return inst
    finally:
        lib.sk_model_free(C.byref(model))


def ref_sk_scale_model(inst, passes=4):
    lib = load("ref")
    keep = _Keep()
    model = build_sk_model(keep, inst)
    r, c = np.zeros(inst["m"]), np.zeros(inst["n"])
    lib.sk_scale_model(C.byref(model), _p(r), _p(c), C.c_int(passes))
    return r, c


class CrossoverStats(C.Structure):
    """sk_b200_crossover_stats (include/integration/sk_crossover.h)."""
    _fields_ = [("rounds", C.c_int), ("fixed_columns", C.c_int), ("released_columns", C.c_int),
                ("full_fallback", C.c_int), ("direct", C.c_int), ("simplex_iterations", C.c_longlong),
                ("seconds", C.c_double)]


def ref_crossover(inst, x, y, fix_tolerance=1e-6, max_rounds=5, primal_tol=1e-7, dual_tol=1e-7):
    """Runs the crossover integration source (built against the reference's C core) from
    the first-order point (x, y); returns (status, dict with the certified x, y, the
    sk_verify residuals and the crossover's counters)."""
    lib = load("ref_crossover")
    ref = load("ref")
    keep = _Keep()
    model = build_sk_model(keep, inst)
    o = ref_options(primal_tol=primal_tol, dual_tol=dual_tol, lp_engine=0)
    s = SkSolution()
    ref.sk_solution_init(C.byref(s))
    st = CrossoverStats()
    rc = lib.sk_b200_crossover(C.byref(model), C.byref(o), _p(keep.d(x)), _p(keep.d(y)),
                               C.c_double(fix_tolerance), C.c_int(max_rounds), C.byref(s), C.byref(st))
    n, m = inst["n"], inst["m"]
    out = {k: getattr(s, k) for k, _ in SkSolution._fields_ if k not in ("x", "y", "rc", "rowact")}
    out.update({k: getattr(st, k) for k, _ in CrossoverStats._fields_})
    out["x"] = np.ctypeslib.as_array(s.x, (n,)).copy() if s.x and n else np.zeros(n)
    out["y"] = np.ctypeslib.as_array(s.y, (m,)).copy() if s.y and m else np.zeros(m)
    ref.sk_solution_free(C.byref(s))
    return rc, out


class RefCrossoverResult(C.Structure):
    """RefCrossoverResult (oracle/ref_crossover_shim.cpp)."""
    _fields_ = [("status", C.c_int), ("used_warm_start", C.c_int), ("dual_iterations", C.c_int),
                ("cold_iterations", C.c_int), ("basic_structurals", C.c_int), ("repaired", C.c_int),
                ("objective", C.c_double), ("primal_residual", C.c_double), ("dual_residual", C.c_double),
                ("seconds", C.c_double)]


def ref_sihps_crossover(inst, x, y, time_budget=0.0):
    """Runs the crossover source for the reference C++ core (a basis from the first-order
    point (x, y) seated in its simplex, time_budget seconds for it, 0: none); returns
    (rc, dict with x, y and the counters)."""
    lib = load("ref_sihps_crossover")
    keep = _Keep()
    n, m = inst["n"], inst["m"]
    x_out, y_out = np.zeros(n), np.zeros(m)
    r = RefCrossoverResult()
    rc = lib.ref_crossover_lp(C.c_int(m), C.c_int(n), C.c_int(int(inst["ptr"][-1])), _p(keep.i(inst["ptr"]), iptr),
                              _p(keep.i(inst["idx"]), iptr), _p(keep.d(inst["val"])), _p(keep.d(inst["c"])),
                              _p(keep.d(inst["cl"])), _p(keep.d(inst["cu"])), _p(keep.d(inst["rl"])),
                              _p(keep.d(inst["ru"])), _p(keep.d(x)), _p(keep.d(y)), C.c_double(time_budget),
                              _p(x_out), _p(y_out), C.byref(r))
    out = {k: getattr(r, k) for k, _ in RefCrossoverResult._fields_}
    out["x"], out["y"] = x_out, y_out
    return rc, out
