"""The reference C++ core's LP driver (sihps::solve_lp, src/lp/LpSolver.cpp) built
from its own sources by oracle/hooked_lpsolver.py, as it is and with run_first_order
replaced by the integration block (include/integration/lpsolver_run_first_order.inc).
On the CPU: the splice replaces exactly the one function, the hooked build links the
engine's sankhya_b200_pdlp_solve, and the SIMPLEX path (no GPU) of both builds gives the
objective of the reference C core's own simplex (sk_solve with SK_LP_SIMPLEX), which pins
the shim's encoding of two-sided rows. FIRST_ORDER and HYBRID are run by
tests/test_gpu_lpsolver_first_order.py."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _need(oracle, name):
    if not oracle.available(name):
        pytest.skip(f"{name} not built (make -C oracle ref ref-tests)")


def test_splice_replaces_only_run_first_order(oracle):
    import hooked_lpsolver
    ref = oracle.reference_tree()
    if ref is None:
        pytest.skip("reference sources absent")
    text = open(os.path.join(ref, "src", "lp", "LpSolver.cpp")).read()
    out = hooked_lpsolver.spliced(text, hooked_lpsolver.block())
    start = out.index("bool run_first_order(const LpProblem& target")
    body = out[start:out.index("\n}\n", start)]
    assert "sankhya_b200_pdlp_solve(" in body and "GpuPdlp" not in body
    # everything outside the function is the reference's text, plus one include
    assert out.replace('#include "sankhya_b200.h"\n', "", 1).replace(hooked_lpsolver.block(), "") == \
        text.replace(text[text.index("bool run_first_order(const LpProblem& target"):
                          text.index("\n}\n", text.index("bool run_first_order(")) + 3], "")


def test_hooked_build_links_the_engine(oracle):
    _need(oracle, "ref_lp_hooked")
    path = os.path.join(ROOT, "oracle", "_ref", "libsihps_lp_hooked.so")
    nm = subprocess.run(["nm", "-D", path], capture_output=True, text=True).stdout
    assert " U sankhya_b200_pdlp_solve" in nm and " T ref_solve_lp" in nm
    dyn = subprocess.run(["readelf", "-d", path], capture_output=True, text=True).stdout
    assert "libsankhya_cuda.so" in dyn


@pytest.mark.parametrize("seed,m,n", [(3, 60, 150), (8, 200, 500)])
def test_simplex_path_matches_the_c_core(oracle, instances, seed, m, n):
    _need(oracle, "ref_lp")
    _need(oracle, "ref_lp_hooked")
    inst = instances.lp_uniform(seed, m, n, 4)
    st, ref = oracle.ref_sk_solve(inst, lp_engine=1, primal_tol=1e-9, dual_tol=1e-9)
    assert st == 0 and ref["result"] == 0
    for hooked in (False, True):
        x, r = oracle.ref_solve_lp(inst, oracle.LP_SIMPLEX, hooked=hooked)
        assert r["status_name"] == "OPTIMAL" and not r["used_first_order"], r
        assert abs(r["objective"] - ref["objective"]) <= 1e-9 * (1 + abs(ref["objective"])), (r, ref["objective"])
        assert abs(float(inst["c"] @ x) - r["objective"]) <= 1e-9 * (1 + abs(r["objective"]))
        assert r["primal_residual"] <= 1e-6
