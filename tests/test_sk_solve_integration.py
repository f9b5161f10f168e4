"""The `sk_solve` integration (include/integration/sk_solve_hook.inc), applied as written.

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
reference's behaviour intact. The reference's own c/tests programs are then built
against the patched core and must all pass; a counting stand-in for the engine shows
which of them reach the hook. With a GPU the hook itself runs; its iterates are
pinned against the reference's sk_solve fixtures in tests/test_gpu_parity.py.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import hooked_core as H   # oracle/hooked_core.py: applies the block, builds the core

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _reference():
    import oracle as O
    ref = O.reference_tree()
    if ref is None:
        pytest.skip("reference sources absent (set SANKHYA_REFERENCE)")
    return ref


def _build_core(ref, out, lib_dir, lib_name):
    """The patched core as a shared library linked to lib<lib_name>.so in lib_dir."""
    return H.build(ref, out, lib_dir, lib_name)


@pytest.fixture(scope="module")
def hooked_core(tmp_path_factory):
    ref = _reference()
    lib = os.path.join(ROOT, "the-solver_b200", "lib", "libsankhya_cuda.so")
    if not os.path.exists(os.path.join(ref, "c", "src", "sk_solve.c")) or not os.path.exists(lib):
        pytest.skip("reference C sources or the engine library absent")
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsankhya_ref.so")):
        pytest.skip("reference C core not built (make -C oracle ref)")
    out = str(tmp_path_factory.mktemp("hooked") / "libsk_hooked.so")
    return _build_core(ref, out, os.path.dirname(lib), "sankhya_cuda")


# A stand-in for the engine that records each call of the loop hook on stderr and
# answers SK_ERR_NUMERIC (no device), so the core falls back to its own loop.
COUNTING_STUB = r"""
#include <stdio.h>
int sankhya_b200_pdhg_loop(const void* m, const void* o, double* x, double* y, double* a, void* r) {
    (void)m; (void)o; (void)x; (void)y; (void)a; (void)r;
    fprintf(stderr, "sankhya_b200_pdhg_loop called\n");
    return 7;
}
"""


def _c_tests(ref):
    d = os.path.join(ref, "c", "tests")
    return sorted(f[:-2] for f in os.listdir(d) if f.endswith(".c"))


def _run_c_test(ref, core, name, out_dir):
    """Builds the reference's c/tests/<name>.c against `core` and runs it from the
    reference root (some read model files by relative path)."""
    exe = os.path.join(out_dir, name)
    core_dir = os.path.dirname(core)
    lib_name = os.path.basename(core)[3:-3]
    cmd = ["gcc", "-O2", "-std=gnu11", "-I" + os.path.join(ref, "c", "include"), "-I" + os.path.join(ref, "c", "src"),
           os.path.join(ref, "c", "tests", name + ".c"), "-L" + core_dir, "-l" + lib_name, "-Wl,-rpath," + core_dir,
           "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, (name, r.stderr[-2000:])
    return subprocess.run([exe], cwd=ref, capture_output=True, text=True, timeout=300)


def test_reference_c_tests_pass_with_the_block(hooked_core, tmp_path):
    """Every program in the reference's c/tests passes against the core with the block
    applied and linked to this library (here: the fallback path when no device)."""
    ref = _reference()
    names = _c_tests(ref)
    assert len(names) >= 20
    for name in names:
        r = _run_c_test(ref, hooked_core, name, str(tmp_path))
        assert r.returncode == 0, (name, r.returncode, r.stdout[-1000:], r.stderr[-1000:])


def test_which_reference_c_tests_reach_the_loop(hooked_core, tmp_path):
    """Through a counting stand-in for the engine: the reference's C tests that run the
    first-order loop of solve_continuous call the hook exactly once; the others are
    settled by sk_solve's QP shortcuts or the simplex and never reach it."""
    ref = _reference()
    stub_dir = tmp_path / "stub"
    stub_dir.mkdir()
    (stub_dir / "stub.c").write_text(COUNTING_STUB)
    r = subprocess.run(["gcc", "-shared", "-fPIC", str(stub_dir / "stub.c"), "-o", str(stub_dir / "libloopstub.so")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    core = _build_core(ref, str(tmp_path / "libsk_stubbed.so"), str(stub_dir), "loopstub")
    calls = {}
    for name in _c_tests(ref):
        r = _run_c_test(ref, core, name, str(tmp_path))
        assert r.returncode == 0, (name, r.stderr[-1000:])
        calls[name] = r.stderr.count("sankhya_b200_pdhg_loop called")
    assert calls.get("qp_iteration_limit_smoke") == 1 and calls.get("qp_working_set_smoke") == 1, calls
    assert all(v in (0, 1) for v in calls.values()), calls


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
    patched = H.patched_source(text, H.snippet())
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
