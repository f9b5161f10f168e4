"""The C-ABI library loads and exports every symbol the headers declare; the
ctypes mirrors have the C struct sizes. No GPU needed (no compute calls)."""
import ctypes as C
import os
import re

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    names = []
    for h in ("sankhya_cuda.h", "sankhya_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"SANKHYA_CUDA_API\s+[\w\s\*]+?\b(\w+)\s*\(", text)
    return names


def test_headers_declare_the_reference_abi(engine):
    names = declared_symbols()
    for s in engine.REFERENCE_SYMBOLS:
        assert s in names, s
    # the reference header declares exactly these 13 public functions
    assert len(engine.REFERENCE_SYMBOLS) == 13


def test_library_exports_every_declared_symbol(engine):
    L = engine.lib()
    for s in declared_symbols():
        assert hasattr(L, s), f"missing export {s}"


def test_struct_layouts_match_reference():
    import sankhya_b200 as E
    # SankhyaCudaCSR: 3 ints + 3 pointers (with padding after the ints)
    assert C.sizeof(E.CSR) == 4 * 3 + 4 + 8 * 3
    assert C.sizeof(E.Settings) == 4 * 2 + 8 * 5
    assert C.sizeof(E.Result) == 4 * 2 + 8 * 6
    assert E.Settings.time_limit.offset == 40


def test_no_device_is_a_clean_error(engine):
    """Without a GPU the entry points fail with -1 and an error text (no fallback)."""
    import numpy as np
    import torch
    if torch.cuda.is_available():
        return
    rc, y = engine.spmv_host(2, 3, [0, 2, 4], [0, 2, 1, 2], [1.0, 2, 3, 4], [2.0, 5, 7])
    assert rc != 0 and "device" in engine.last_error().lower()


def test_host_spmv_rejects_out_of_bounds_csr_before_device_work(engine):
    """sankhya_cuda_spmv_f64 checks, on the host and before any device query, what
    would send its kernel outside the uploaded buffers: offsets outside [0, nnz],
    decreasing offsets, columns outside [0, cols). Runs the same with or without a GPU."""
    vals, x = [1.0, 2.0, 3.0, 4.0], [2.0, 5.0, 7.0]
    rc, _ = engine.spmv_host(2, 3, [0, 2, 5], [0, 2, 1, 2], vals, x)
    assert rc == -1 and "row-offset endpoints" in engine.last_error()
    rc, _ = engine.spmv_host(2, 3, [-1, 2, 4], [0, 2, 1, 2], vals, x)
    assert rc == -1 and "row-offset endpoints" in engine.last_error()
    rc, _ = engine.spmv_host(2, 3, [0, 3, 2], [0, 2, 1, 2], vals, x)
    assert rc == -1 and "row-offset ordering" in engine.last_error()
    rc, _ = engine.spmv_host(2, 3, [0, 2, 4], [0, 3, 1, 2], vals, x)
    assert rc == -1 and "column index" in engine.last_error()
    rc, _ = engine.spmv_host(2, 3, [0, 2, 4], [0, 2, -1, 2], vals, x)
    assert rc == -1 and "column index" in engine.last_error()


def test_every_solver_entry_fails_without_a_device(engine, instances):
    """No host path behind any solver entry point: without a GPU each returns -1 with
    an error text (checked where this suite runs without one)."""
    import ctypes as C
    import numpy as np
    import torch
    if torch.cuda.is_available():
        return
    L = engine.lib()
    inst = instances.lp_uniform(1, 8, 12, 2)
    csr = engine.CSR()
    p = lambda a, t=C.c_int: np.ascontiguousarray(a, dtype=np.int32 if t is C.c_int else np.float64).ctypes.data_as(
        C.POINTER(t))
    rc = L.sankhya_cuda_csr_create(C.byref(csr), inst["m"], inst["n"], int(inst["ptr"][-1]), p(inst["ptr"]),
                                   p(inst["idx"]), p(inst["val"], C.c_double))
    assert rc != 0 and "device" in engine.last_error().lower()
    net = C.c_void_p()
    assert L.sankhya_b200_gnn_create(None, C.byref(net)) == -1 and not net.value
    assert "device" in engine.last_error().lower()
    s = engine.batch_default_settings()
    x = np.zeros(2 * inst["n"])
    res = (engine.BatchResult * 2)()
    d = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))
    fake = engine.CSR(inst["m"], inst["n"], int(inst["ptr"][-1]), None, None, None)
    rc = L.sankhya_b200_shared_batch_pdhg(C.byref(fake), 2, d(inst["c"]), 0, d(inst["rl"]), d(inst["ru"]), 0,
                                          d(inst["cl"]), d(inst["cu"]), 0, C.byref(s), d(x), None, res)
    assert rc == -1 and "device" in engine.last_error().lower()
    ps = engine.pdlp_default_settings()
    pr = engine.PdlpResult()
    rc = L.sankhya_b200_pdlp_solve(C.byref(fake), d(inst["c"]), d(inst["rl"]), d(inst["ru"]), d(inst["cl"]),
                                   d(inst["cu"]), C.byref(ps), None, None, d(x), None, C.byref(pr))
    assert rc == -1 and "device" in engine.last_error().lower()


def test_loop_hook_validates_the_model_before_device_work(engine, oracle, instances):
    """sankhya_b200_pdhg_loop applies sk_model_validate's checks (c/src/sk_core.c:126-155)
    before any device call: each malformed variant returns SK_ERR_ARG (1). Without a
    GPU, the well-formed models the gpu tests solve get past them and stop at the
    device check (SK_ERR_NUMERIC, 7), so the checks reject none of those."""
    import ctypes as C
    import json
    import numpy as np
    import torch
    L = engine.lib()

    def call(inst, quadratic=False, edit=None):
        keep = oracle._Keep()
        model = oracle.build_sk_model(keep, inst, quadratic)
        if edit:
            edit(model, keep)
        opts = oracle.SkOptions(primal_tol=1e-6, dual_tol=1e-6, iteration_limit=100, threads=1)
        x, y, act = np.zeros(inst["n"]), np.zeros(inst["m"]), np.zeros(inst["m"])
        res = engine.LoopResult()
        return L.sankhya_b200_pdhg_loop(C.byref(model), C.byref(opts), engine._p(x), engine._p(y), engine._p(act),
                                        C.byref(res))

    lp = instances.lp_uniform(12, 60, 150, 4)
    qp = instances.qp_diag_plus_lowrank(3, 40, 80, a_per_col=4, l_per_col=2)
    if not torch.cuda.is_available():
        man = json.load(open(os.path.join(ROOT, "tests", "golden", "manifest.json")))
        for name, seed, m, n, per_col, limits in man["lp"]:
            assert call(instances.lp_uniform(seed, m, n, per_col)) == 7, name
        for name, seed, m, n, limits in man["qp"]:
            assert call(instances.qp_diag_plus_lowrank(seed, m, n, a_per_col=4, l_per_col=2), quadratic=True) == 7, name
        assert call(lp) == 7 and call(qp, quadratic=True) == 7

    def setp(k, v):
        def edit(model, keep):
            arr = np.ctypeslib.as_array(model.A.p, (model.ncol + 1,)).copy()
            arr[k] = v
            model.A.p = oracle._p(keep.i(arr), oracle.iptr)
        return edit

    def seti(k, v):
        def edit(model, keep):
            nnz = model.A.p[model.ncol]
            arr = np.ctypeslib.as_array(model.A.i, (nnz,)).copy()
            arr[k] = v
            model.A.i = oracle._p(keep.i(arr), oracle.iptr)
        return edit

    def setd(field, k, v):
        def edit(model, keep):
            size = model.ncol if field in ("c", "clow", "cupp") else model.nrow
            arr = np.ctypeslib.as_array(getattr(model, field), (size,)).copy()
            arr[k] = v
            setattr(model, field, oracle._p(keep.d(arr)))
        return edit

    nnz = int(lp["ptr"][-1])
    bad = [
        setp(0, 1),                                    # p[0] != 0
        setp(5, 10 ** 6),                              # offset beyond nnz
        setp(lp["n"], nnz + 1),                        # p[ncol] beyond nzmax
        seti(3, lp["m"]),                              # row index out of range
        seti(0, -1),
        setd("c", 2, float("nan")),                    # non-finite cost
        setd("clow", 1, 20.0),                         # crossed column bound (upper 10)
        setd("rlow", 0, float("nan")),                 # NaN row bound
        lambda model, keep: setattr(model.A, "nzmax", nnz - 1),   # nnz beyond nzmax
        lambda model, keep: setattr(model.A, "nrow", lp["m"] + 1),
    ]
    for k, edit in enumerate(bad):
        assert call(lp, edit=edit) == 1, k
        assert "invalid sk model" in engine.last_error(), k

    def bad_q(model, keep):
        q = model.Q.contents
        n = q.ncol
        arr = np.ctypeslib.as_array(q.i, (q.p[n],)).copy()
        arr[0] = n
        q.i = oracle._p(keep.i(arr), oracle.iptr)
    assert call(qp, quadratic=True, edit=bad_q) == 1


MIRRORS = {  # ctypes class in the package -> C struct in include/
    "CSR": "SankhyaCudaCSR", "Settings": "SankhyaCudaLPSettings", "Result": "SankhyaCudaLPResult",
    "Timing": "SankhyaB200Timing", "LoopResult": "SankhyaB200LoopResult",
    "PdlpSettings": "SankhyaB200PdlpSettings", "PdlpResult": "SankhyaB200PdlpResult",
    "BatchSettings": "SankhyaB200BatchSettings", "BatchResult": "SankhyaB200BatchResult",
    "GnnSettings": "SankhyaB200GnnSettings", "PolishSettings": "SankhyaB200PolishSettings",
    "PolishResult": "SankhyaB200PolishResult",
}


def test_ctypes_mirrors_match_the_headers(engine, tmp_path):
    """Every ctypes mirror has the size and field offsets the C compiler gives the
    header's struct (a program built against include/ prints them)."""
    import subprocess
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sankhya_cuda.h"', '#include "sankhya_b200.h"',
             "int main(void) {"]
    for py, cs in MIRRORS.items():
        cls = getattr(engine, py)
        lines.append(f'printf("{py} size %zu\\n", sizeof({cs}));')
        for name, _ in cls._fields_:
            lines.append(f'printf("{py} {name} %zu\\n", offsetof({cs}, {name}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        py, name, value = line.split()
        got[(py, name)] = int(value)
    for py in MIRRORS:
        cls = getattr(engine, py)
        assert C.sizeof(cls) == got[(py, "size")], py
        for name, _ in cls._fields_:
            assert getattr(cls, name).offset == got[(py, name)], (py, name)


def test_pdlp_settings_versions(engine, instances):
    """Settings versions 1 to 4 pass the settings checks (they stop at the device check
    here); other versions are refused. Version 3 callers' structs end before `cancel`,
    version 2 before `initial_primal_weight`, version 1 before `algorithm`."""
    import numpy as np
    import torch
    if torch.cuda.is_available():
        return
    inst = instances.lp_uniform(1, 8, 12, 2)
    fake = engine.CSR(inst["m"], inst["n"], int(inst["ptr"][-1]), None, None, None)
    L = engine.lib()
    d = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))
    s = engine.pdlp_default_settings()
    assert s.struct_version == 4 and not s.cancel
    for version, message in ((1, "device"), (2, "device"), (3, "device"), (4, "device"), (0, "struct_version"),
                             (5, "struct_version")):
        s.struct_version = version
        res = engine.PdlpResult()
        x = np.zeros(inst["n"])
        rc = L.sankhya_b200_pdlp_solve(C.byref(fake), d(inst["c"]), d(inst["rl"]), d(inst["ru"]), d(inst["cl"]),
                                       d(inst["cu"]), C.byref(s), None, None, d(x), None, C.byref(res))
        assert rc == -1 and message in engine.last_error(), (version, engine.last_error())


def test_polishing_settings_checks(engine, instances):
    """The polishing entry point checks its settings before any device work: the
    defaults (and NULL polishing settings) reach the device check; another struct
    version, a non-positive tolerance, a negative budget, or a main loop other than
    the FP64 adaptive one are refused."""
    import numpy as np
    import torch
    if torch.cuda.is_available():
        return
    inst = instances.lp_uniform(1, 8, 12, 2)
    fake = engine.CSR(inst["m"], inst["n"], int(inst["ptr"][-1]), None, None, None)
    L = engine.lib()
    d = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))
    p = engine.polish_default_settings()
    assert (p.struct_version, p.max_polish_iterations, p.start_tolerance, p.polish_tolerance) == (1, 0, 1e-4, 1e-8)

    def call(edit_polish=None, edit_settings=None, null_polish=False):
        s = engine.pdlp_default_settings()
        q = engine.polish_default_settings()
        if edit_polish:
            edit_polish(q)
        if edit_settings:
            edit_settings(s)
        res, pres = engine.PdlpResult(), engine.PolishResult()
        pres.rounds = 99
        x = np.zeros(inst["n"])
        rc = L.sankhya_b200_pdlp_solve_polished(C.byref(fake), d(inst["c"]), d(inst["rl"]), d(inst["ru"]),
                                                d(inst["cl"]), d(inst["cu"]), C.byref(s),
                                                None if null_polish else C.byref(q), None, None, d(x), None,
                                                C.byref(res), C.byref(pres))
        assert rc == -1 and res.status == -1 and pres.rounds == 0
        return engine.last_error()

    assert "device" in call()
    assert "device" in call(null_polish=True)
    assert "struct_version" in call(edit_polish=lambda q: setattr(q, "struct_version", 2))
    for field, value in (("start_tolerance", 0.0), ("polish_tolerance", -1.0), ("polish_tolerance", float("nan")),
                         ("max_polish_iterations", -1)):
        assert "invalid polishing settings" in call(edit_polish=lambda q: setattr(q, field, value)), field
    for field, value in (("precision", engine.FP32_REFINE), ("adaptive_step", 0),
                         ("algorithm", engine.PDLP_HALPERN)):
        assert "FP64 adaptive loop" in call(edit_settings=lambda s: setattr(s, field, value)), field


def test_headers_compile_as_c_and_cxx_and_every_symbol_links(tmp_path):
    """include/*.h are usable from C (C99, -Wall -Werror) and from C++: a program that
    takes the address of every declared function compiles both ways and links against
    the library."""
    import subprocess
    names = declared_symbols()
    body = ["#include \"sankhya_cuda.h\"", "#include \"sankhya_b200.h\"", "#include <stdio.h>",
            "int main(void) {", "    const void* fns[] = {"]
    body += [f"        (const void*)&{n}," for n in names]
    body += ["    };", "    printf(\"%d\\n\", (int)(sizeof(fns) / sizeof(fns[0])));", "    return 0;", "}"]
    lib = os.path.join(ROOT, "the-solver_b200", "lib")
    for lang, compiler, std, ext in (("c", "gcc", "-std=c99", ".c"), ("c++", "g++", "-std=c++17", ".cpp")):
        src = tmp_path / ("abi" + ext)
        src.write_text("\n".join(body) + "\n")
        exe = tmp_path / ("abi_" + lang.replace("+", "x"))
        r = subprocess.run([compiler, std, "-Wall", "-Werror", "-Wno-pedantic", "-I" + os.path.join(ROOT, "include"),
                            str(src), "-L" + lib, "-lsankhya_cuda", "-Wl,-rpath," + lib, "-o", str(exe)],
                           capture_output=True, text=True)
        assert r.returncode == 0, (lang, r.stderr[-3000:])
        out = subprocess.run([str(exe)], capture_output=True, text=True)
        assert out.returncode == 0 and int(out.stdout) == len(names), (lang, out.stdout, out.stderr)
