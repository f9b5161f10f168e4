"""The reference's command-line programs, apps/sankhya_pdhg.cu and
apps/sankhya_qp_cuda.cu, compiled unchanged against include/sankhya_cuda.h and linked
to this library (oracle/Makefile target ref-tests), run on MPS / QPS files: the
reference's own CLI tests (cuda/CMakeLists.txt:31-48) as written, on its model files,
and seeded instances written by tests/mps_files.py. Each program verifies its own
answer with the reference's C core and exits 0 only when that check passes
(sankhya_pdhg.cu:148, sankhya_qp_cuda.cu:230-237). Beyond that exit code, every run
must agree with the oracle given the steps the program chose: the same stopping
iteration, x bit for bit (LP, printed to 17 digits), the objective to 1e-12 (LP) or
to its 12 printed digits (QP)."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import mps_files as mf

pytestmark = pytest.mark.gpu
ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
REF = os.path.join(ROOT, "oracle", "_ref")
SMOKE = os.path.join(REF, "smoke")
DEFAULTS = dict(max_iterations=100000, check_every=100, theta=1.0, tolerance=1e-6)


def _program(name):
    exe = os.path.join(REF, "ref_" + name)
    if not os.path.exists(exe):
        pytest.skip("reference programs not built (reference sources absent at build time)")
    return exe


def _smoke(name):
    path = os.path.join(SMOKE, name)
    if not os.path.exists(path):
        pytest.skip("reference CLI model files not copied (reference sources absent at build time)")
    return path


def _run(exe, path, *args, expect_ok=True):
    r = subprocess.run([exe, path, *args], capture_output=True, text=True, timeout=300)
    if expect_ok:
        assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return r


def _lp_against_oracle(oracle, out, path, **over):
    """Parses sankhya_pdhg's report and checks it against the oracle run with the
    program's automatic steps; returns (x, objective)."""
    auto = dict(re.findall(r"auto_(\w+)=(\S+)", out))
    status_line = [s for s in out.splitlines() if s.startswith("status=")][0]
    head = dict(re.findall(r"(\w+)=(-?[0-9][^ ]*)", status_line))
    xs = dict(re.findall(r"^x\[(\w+)\]=(\S+)$", out, re.M))
    assert int(head["status"]) == 0
    assert re.search(r"verified_feasible=1", out)
    back = oracle.ref_read_mps(path)
    settings = dict(DEFAULTS, tau=float(auto["tau"]), sigma=float(auto["sigma"]), **over)
    rc, x, _, r = oracle.fixed_pdhg(back, settings, want_dual=False)
    assert rc == 0 and r["status"] == 0
    assert int(head["iterations"]) == r["iterations"]
    obj = float(head["objective"])
    assert abs(obj - r["objective"]) <= 1e-12 * (1 + abs(r["objective"]))
    names = [m.group(1) for m in re.finditer(r"^x\[(\w+)\]=", out, re.M)]
    got = np.array([float(xs[k]) for k in names])
    assert np.array_equal(got, x)
    return got, obj


def _qp_against_oracle(oracle, out, path, **over):
    """Parses sankhya_qp_cuda's JSON report and checks it against the oracle run with
    the program's mass-based steps; returns the report."""
    line = json.loads([s for s in out.splitlines() if s.startswith("{")][-1])
    assert line["status"] == 0 and line["independent_primal_status"] == "ok"
    back = oracle.ref_read_mps(path)
    primal, dual = mf.app_qp_steps(back)
    qd = mf.q_diagonal(back)
    kw = dict(qdiag=qd) if qd is not None else dict(hessian=True)
    rc, x, y, r = oracle.fixed_pdhg(back, dict(DEFAULTS, tau=0.0, sigma=0.0, **over), primal_steps=primal,
                                    dual_steps=dual, want_dual=True, **kw)
    assert rc == 0 and r["status"] == 0
    assert line["iterations"] == r["iterations"]
    assert abs(line["objective"] - r["objective"]) <= 1e-10 * (1 + abs(r["objective"]))
    st, v = oracle.ref_sk_verify(back, x, y, quadratic=True)
    assert st == 0 and abs(line["independent_objective"] - v["objective"]) <= 1e-10 * (1 + abs(v["objective"]))
    return line


# -- the reference's CLI tests, cuda/CMakeLists.txt:31-48, as written ---------------

def test_cli_pdhg_smoke(oracle):
    """sankhya_cuda_pdhg_cli_smoke: unit_lp.mps --iterations 5000 --tolerance 1e-5."""
    exe, path = _program("sankhya_pdhg"), _smoke("unit_lp.mps")
    out = _run(exe, path, "--iterations", "5000", "--tolerance", "1e-5", "--device", "0").stdout
    x, obj = _lp_against_oracle(oracle, out, path, max_iterations=5000, tolerance=1e-5)
    assert abs(x[0] - 1.0) <= 1e-5 and abs(obj - 1.0) <= 1e-5


def test_cli_general_qp_smoke(oracle):
    """sankhya_cuda_general_qp_smoke: tiny_qp.qps (off-diagonal Hessian, a column with
    no constraint entries) --iterations 100000 --tolerance 1e-5: x = (2, 0), obj -4."""
    exe, path = _program("sankhya_qp_cuda"), _smoke("tiny_qp.qps")
    out = _run(exe, path, "--iterations", "100000", "--tolerance", "1e-5", "--device", "0").stdout
    line = _qp_against_oracle(oracle, out, path, max_iterations=100000, tolerance=1e-5)
    assert abs(line["objective"] + 4.0) <= 1e-5


def test_cli_nonconvex_qp_guard():
    """sankhya_cuda_nonconvex_qp_guard (WILL_FAIL): the program must exit non-zero.
    The file has no constraint rows, so the reference's reader rejects it before any
    solve; this library is never called."""
    exe, path = _program("sankhya_qp_cuda"), _smoke("nonconvex_qp.qps")
    assert _run(exe, path, expect_ok=False).returncode != 0


def test_tiny_lp_by_hand(oracle):
    """tiny_lp.mps (L rows, an upper bound) through sankhya_pdhg's defaults:
    x = 3, y = 1, obj -11 by hand."""
    exe, path = _program("sankhya_pdhg"), _smoke("tiny_lp.mps")
    x, obj = _lp_against_oracle(oracle, _run(exe, path).stdout, path)
    assert np.allclose(x, [3.0, 1.0], atol=1e-6) and abs(obj + 11.0) <= 1e-6


# -- seeded instances -----------------------------------------------------------------

def test_sankhya_pdhg_program(tmp_path, oracle):
    exe = _program("sankhya_pdhg")
    inst = mf.lp_instance(5)
    path = str(tmp_path / "lp.mps")
    mf.write_mps(path, inst)
    x, _ = _lp_against_oracle(oracle, _run(exe, path).stdout, path)
    assert len(x) == inst["n"]


@pytest.mark.parametrize("diagonal", [True, False])
def test_sankhya_qp_cuda_program(tmp_path, oracle, diagonal):
    exe = _program("sankhya_qp_cuda")
    inst = mf.qp_instance(5, diagonal=diagonal)
    path = str(tmp_path / "qp.qps")
    mf.write_mps(path, inst)
    _qp_against_oracle(oracle, _run(exe, path).stdout, path)
