"""The callers in include/integration/, compiled inside the reference
translation units they belong to (from standard input; no copy of a source is
written), so the names, types and signatures they use must match both the
reference's code and this library's C ABI:

- the sihps caller: `run_first_order` (src/lp/LpSolver.cpp:62-99) replaced by one
  sankhya_b200_pdlp_solve call, checked with g++ -fsyntax-only against LpProblem,
  CSRMatrix, PdlpParams and PdlpStats (oracle/hooked_lpsolver.py links the spliced
  core and tests/test_gpu_lpsolver_first_order.py runs it);
- the MILP batch caller: the node-relaxation block wrapped in a function appended to
  c/src/sk_milp.c, where the `milp` driver struct it reads (M->m, M->lp_opt) is
  defined, checked with gcc -fsyntax-only."""
import os
import subprocess

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _reference():
    import oracle as O
    ref = O.reference_tree()
    if ref is None:
        pytest.skip("reference sources absent (set SANKHYA_REFERENCE)")
    return ref


INTEGRATION = os.path.join(ROOT, "include", "integration")


def _block():
    return open(os.path.join(INTEGRATION, "lpsolver_run_first_order.inc")).read()


def _milp_block():
    return open(os.path.join(INTEGRATION, "sk_milp_batch.inc")).read()


def _spliced(text, block):
    import hooked_lpsolver
    return hooked_lpsolver.spliced(text, block)


def _compile(ref, source):
    lp = os.path.join(ref, "src", "lp")
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror=return-type", "-iquote", lp,
           "-I" + os.path.join(ref, "src"), "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
           "-x", "c++", "-"]
    return subprocess.run(cmd, input=source, capture_output=True, text=True)


@pytest.fixture(scope="module")
def lp_solver_source():
    ref = _reference()
    path = os.path.join(ref, "src", "lp", "LpSolver.cpp")
    if not os.path.exists(path):
        pytest.skip("reference C++ sources absent")
    return ref, open(path).read()


def test_unmodified_translation_unit_compiles(lp_solver_source):
    """The baseline: the reference's own LpSolver.cpp compiles with these flags."""
    ref, text = lp_solver_source
    r = _compile(ref, text)
    assert r.returncode == 0, r.stderr[-3000:]


def test_replacement_compiles_in_place(lp_solver_source):
    ref, text = lp_solver_source
    block = _block()
    assert "sankhya_b200_pdlp_solve(" in block and "GpuPdlp" not in block
    r = _compile(ref, _spliced(text, block))
    assert r.returncode == 0, r.stderr[-3000:]


def test_a_wrong_field_is_caught(lp_solver_source):
    """The check has teeth: a misspelt PdlpStats field fails to compile."""
    ref, text = lp_solver_source
    broken = _block().replace("stats_out.host_syncs", "stats_out.host_sync_count")
    r = _compile(ref, _spliced(text, broken))
    assert r.returncode != 0 and "host_sync_count" in r.stderr


def test_hybrid_crossover_compiles_in_place(lp_solver_source):
    """HYBRID's simplex step replaced by the crossover block (with run_first_order
    replaced as above): the spliced LpSolver.cpp compiles against the core's Simplex,
    LpResult and PdlpStats and the crossover header."""
    import hooked_lpsolver
    ref, text = lp_solver_source
    body = open(os.path.join(INTEGRATION, "lpsolver_hybrid_crossover.inc")).read()
    assert "sihps_b200::crossover(" in body
    source = hooked_lpsolver.spliced_hybrid(_spliced(text, _block()), body)
    assert source.count("\n        auto try_simplex = [&]() {\n") == 1 and "sihps_crossover.hpp" in source
    lp = os.path.join(ref, "src", "lp")
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror=return-type", "-iquote", lp,
           "-I" + os.path.join(ref, "src"), "-I" + os.path.join(ROOT, "include"), "-I" + INTEGRATION,
           "-I/usr/local/cuda/include", "-x", "c++", "-"]
    r = subprocess.run(cmd, input=source, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    broken = body.replace("crossover_stats, options.hybrid_simplex_budget_seconds",
                          "crossover_stats, options.hybrid_simplex_budget")
    r = subprocess.run(cmd, input=hooked_lpsolver.spliced_hybrid(_spliced(text, _block()), broken),
                       capture_output=True, text=True)
    assert r.returncode != 0 and "hybrid_simplex_budget" in r.stderr


MILP_WRAPPER = """
#include "sankhya_b200.h"
#include <string.h>
static void b200_solve_open_nodes(milp *M, int batch, double **node_low, double **node_upp,
                                  const int *row_ptr, const int *col_idx, const double *val) {
%s
    free(results); free(x_nodes); sankhya_cuda_csr_destroy(&csr);
}
"""


def _compile_c(ref, source):
    cmd = ["gcc", "-std=gnu11", "-fsyntax-only", "-Wall", "-Wno-unused-function", "-I" + os.path.join(ref, "c", "src"),
           "-I" + os.path.join(ref, "c", "include"), "-I" + os.path.join(ROOT, "include"), "-x", "c", "-"]
    return subprocess.run(cmd, input=source, capture_output=True, text=True)


@pytest.fixture(scope="module")
def sk_milp_source():
    ref = _reference()
    path = os.path.join(ref, "c", "src", "sk_milp.c")
    if not os.path.exists(path):
        pytest.skip("reference C sources absent")
    return ref, open(path).read()


def test_milp_batch_caller_compiles_against_the_driver(sk_milp_source):
    ref, text = sk_milp_source
    assert "typedef struct milp {" in text
    r = _compile_c(ref, text + MILP_WRAPPER % _milp_block())
    assert r.returncode == 0, r.stderr[-3000:]
    assert "warning" not in r.stderr.split("b200_solve_open_nodes")[-1], r.stderr[-3000:]


def test_milp_check_has_teeth(sk_milp_source):
    ref, text = sk_milp_source
    broken = _milp_block().replace("M->lp_opt.primal_tol", "M->lp_options.primal_tol")
    r = _compile_c(ref, text + MILP_WRAPPER % broken)
    assert r.returncode != 0 and "lp_options" in r.stderr
