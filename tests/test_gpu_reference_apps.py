"""The reference's command-line programs, apps/sankhya_pdhg.cu and
apps/sankhya_qp_cuda.cu, compiled unchanged against include/sankhya_cuda.h and linked
to this library (oracle/Makefile target ref-tests), run on MPS / QPS files of seeded
instances. Each program verifies its own answer with the reference's C core and
exits 0 only when that check passes (sankhya_pdhg.cu:148, sankhya_qp_cuda.cu:230-237).
Beyond that exit code, the run must agree with the oracle given the steps the program
chose: the same stopping iteration, x bit for bit, the objective to 1e-12."""
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
SETTINGS = dict(max_iterations=100000, check_every=100, theta=1.0, tolerance=1e-6)


def _program(name):
    exe = os.path.join(REF, "ref_" + name)
    if not os.path.exists(exe):
        pytest.skip("reference programs not built (reference sources absent at build time)")
    return exe


def _run(exe, path):
    r = subprocess.run([exe, path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def test_sankhya_pdhg_program(tmp_path, oracle):
    exe = _program("sankhya_pdhg")
    inst = mf.lp_instance(5)
    path = str(tmp_path / "lp.mps")
    mf.write_mps(path, inst)
    out = _run(exe, path)
    auto = dict(re.findall(r"auto_(\w+)=(\S+)", out))
    status_line = [s for s in out.splitlines() if s.startswith("status=")][0]
    head = dict(re.findall(r"(\w+)=(-?[0-9][^ ]*)", status_line))
    xs = dict(re.findall(r"^x\[(\w+)\]=(\S+)$", out, re.M))
    assert int(head["status"]) == 0
    assert re.search(r"verified_feasible=1", out)
    tau, sigma = float(auto["tau"]), float(auto["sigma"])
    back = oracle.ref_read_mps(path)
    rc, x, _, r = oracle.fixed_pdhg(back, dict(SETTINGS, tau=tau, sigma=sigma), want_dual=False)
    assert rc == 0 and r["status"] == 0
    assert int(head["iterations"]) == r["iterations"]
    obj = float(head["objective"])
    assert abs(obj - r["objective"]) <= 1e-12 * (1 + abs(r["objective"]))
    got = np.array([float(xs[f"X{j}"]) for j in range(inst["n"])])
    assert np.array_equal(got, x)


@pytest.mark.parametrize("diagonal", [True, False])
def test_sankhya_qp_cuda_program(tmp_path, oracle, diagonal):
    exe = _program("sankhya_qp_cuda")
    inst = mf.qp_instance(5, diagonal=diagonal)
    path = str(tmp_path / "qp.qps")
    mf.write_mps(path, inst)
    out = _run(exe, path)
    line = json.loads([s for s in out.splitlines() if s.startswith("{")][-1])
    assert line["status"] == 0 and line["independent_primal_status"] == "ok"
    back = oracle.ref_read_mps(path)
    primal, dual = mf.app_qp_steps(back)
    kw = dict(qdiag=mf.q_diagonal(back)) if diagonal else dict(hessian=True)
    rc, x, y, r = oracle.fixed_pdhg(back, dict(SETTINGS, tau=0.0, sigma=0.0), primal_steps=primal,
                                    dual_steps=dual, want_dual=True, **kw)
    assert rc == 0 and r["status"] == 0
    assert line["iterations"] == r["iterations"]
    assert abs(line["objective"] - r["objective"]) <= 1e-10 * (1 + abs(r["objective"]))
    st, v = oracle.ref_sk_verify(back, x, y, quadratic=True)
    assert st == 0 and abs(line["independent_objective"] - v["objective"]) <= 1e-10 * (1 + abs(v["objective"]))
