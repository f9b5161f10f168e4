"""The `sk_solve` integration written in INTEGRATION.md section 2, applied as written.

Where the reference sources are present, the test takes the reference's
c/src/sk_solve.c, inserts the documented hook before the first-order loop of
solve_continuous (at `start = sk_wall_seconds();`) and the `after_loop:` label after
the `performed_iterations` assignment, and pipes the result to gcc on standard
input (no copy of the source is written). It is compiled with the reference's other
C core sources where they lie and this library, then `sk_solve` of the patched core
is compared with the unpatched one (oracle/_ref/libsankhya_ref.so) on an LP through
the first-order engine and on a convex QP. Without a GPU the hook reports no device
and the documented fallback restores the CPU loop's start, so the results must be
identical bit for bit; that checks the snippet compiles, links and leaves the
reference's behaviour intact. With a GPU the hook itself runs; its iterates are
pinned against the reference's sk_solve fixtures in tests/test_gpu_parity.py.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
C_SOURCES = ("sankhya_model.c", "sankhya_lu.c", "sankhya_mps.c", "sankhya_verify.c", "sk_lu.c", "sk_core.c",
             "sk_simplex.c", "sk_scale.c", "sk_milp.c")


def _reference():
    import importlib.util
    spec = importlib.util.spec_from_file_location("graft_entry", os.path.join(ROOT, "__graft_entry__.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.REFERENCE


def _snippet():
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    section = doc.split("## 2.")[1].split("## 3.")[0]
    block = re.search(r"```c\n(.*?)```", section, re.S).group(1)
    include, body = block.split("\n", 1)
    assert include.startswith('#include "sankhya_b200.h"')
    return body


def _patched_source(text, body):
    start = text.index("static sk_status solve_continuous(")
    loop = text.index("\n    start = sk_wall_seconds();\n", start)
    done = text.index("\n    performed_iterations = iteration > maximum_iterations", loop)
    done_end = text.index("\n", done + 1)
    out = text[:loop + 1] + body + text[loop + 1:done_end + 1] + "after_loop:;\n" + text[done_end + 1:]
    return out.replace('#include "sankhya.h"\n', '#include "sankhya.h"\n#include "sankhya_b200.h"\n', 1)


@pytest.fixture(scope="module")
def hooked_core(tmp_path_factory):
    ref = _reference()
    src = os.path.join(ref, "c", "src")
    lib = os.path.join(ROOT, "the-solver_b200", "lib", "libsankhya_cuda.so")
    if not os.path.exists(os.path.join(src, "sk_solve.c")) or not os.path.exists(lib):
        pytest.skip("reference C sources or the engine library absent")
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsankhya_ref.so")):
        pytest.skip("reference C core not built (make -C oracle ref)")
    text = open(os.path.join(src, "sk_solve.c")).read()
    patched = _patched_source(text, _snippet())
    out = str(tmp_path_factory.mktemp("hooked") / "libsk_hooked.so")
    cmd = ["gcc", "-O3", "-DNDEBUG", "-std=gnu11", "-fPIC", "-shared", "-DSANKHYA_WITH_B200",
           "-I" + os.path.join(ref, "c", "include"), "-I" + os.path.join(ROOT, "include"),
           "-x", "c", "-", "-x", "none"] + [os.path.join(src, f) for f in C_SOURCES] + [
           "-L" + os.path.dirname(lib), "-lsankhya_cuda", "-Wl,-rpath," + os.path.dirname(lib), "-o", out, "-lm"]
    r = subprocess.run(cmd, input=patched, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


def test_snippet_anchors_exist_once():
    ref = _reference()
    path = os.path.join(ref, "c", "src", "sk_solve.c")
    if not os.path.exists(path):
        pytest.skip("reference C sources absent")
    text = open(path).read()
    body = text[text.index("static sk_status solve_continuous("):]
    body = body[:body.index("\n}\n")]
    assert body.count("\n    start = sk_wall_seconds();\n") == 1
    assert body.count("\n    performed_iterations = iteration > maximum_iterations") == 1
    patched = _patched_source(text, _snippet())
    assert patched.count("goto after_loop;") == 1 and patched.count("after_loop:;") == 1


@pytest.mark.parametrize("case", ["lp_first_order", "qp"])
def test_patched_sk_solve_matches_reference(hooked_core, oracle, instances, case):
    if case == "lp_first_order":
        inst, quad = instances.lp_uniform(12, 60, 150, 4), False
        opts = dict(primal_tol=1e-6, dual_tol=1e-6, iteration_limit=2000)
    else:
        inst, quad = instances.qp_diag_plus_lowrank(3, 40, 80, a_per_col=4, l_per_col=2), True
        opts = dict(primal_tol=1e-6, dual_tol=1e-6, iteration_limit=3000)
    ref_lib = oracle.load("ref")
    st_ref, out_ref = oracle.ref_sk_solve(inst, quadratic=quad, **opts)
    saved = oracle._libs["ref"]
    try:
        oracle._libs["ref"] = C.CDLL(hooked_core)
        st, out = oracle.ref_sk_solve(inst, quadratic=quad, **opts)
    finally:
        oracle._libs["ref"] = saved
    assert oracle._libs["ref"] is ref_lib
    assert st == st_ref == 0
    assert out["result"] == out_ref["result"] and out["iterations"] == out_ref["iterations"]
    for k in ("x", "y", "rowact"):
        assert np.array_equal(out[k], out_ref[k]), k
    assert out["objective"] == out_ref["objective"]
