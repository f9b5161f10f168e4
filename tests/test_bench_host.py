"""Host-side pieces of bench.py that need no GPU: the byte accounting of the fused
iteration and the time_to_kkt summary, driven by a stand-in engine, with the result
serialised the way bench.py prints its line (strict JSON)."""
import importlib.util
import json
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bench_under_test"] = mod
    spec.loader.exec_module(mod)
    return mod


class _Settings:
    pass


class _FakeEngine:
    """pdlp_solve answers from a table keyed by (precision, algorithm)."""
    FP64, FP32_REFINE, PDLP_ADAPTIVE, PDLP_HALPERN = 0, 1, 0, 1

    def __init__(self, answers):
        self.answers = answers

    def pdlp_default_settings(self):
        return _Settings()

    def pdlp_solve(self, A, inst, s):
        import time
        time.sleep(0.002)   # wall times are rounded to milliseconds
        status, x = self.answers[(s.precision, s.algorithm)]
        r = {"status": status, "iterations": 640, "refinements": int(s.precision == 1),
             "relative_primal_residual": 1e-7, "relative_dual_residual": 1e-7, "relative_gap": 1e-7}
        return 0, np.asarray(x, dtype=float), None, r


def test_iteration_bytes_are_the_two_launches():
    b = _bench()
    m, n, nnz = 1_000_000, 2_000_000, 20_000_000
    assert b.iteration_bytes(m, n, nnz) == b.dual_bytes(m, n, nnz) + b.primal_bytes(m, n, nnz)
    assert b.dual_bytes(m, n, nnz) == 12 * nnz + 4 * (m + 1) + 8 * n + 32 * m
    assert b.primal_bytes(m, n, nnz) == 12 * nnz + 4 * (n + 1) + 8 * m + 48 * n


def test_time_to_kkt_reports_speedups_and_objective_agreement():
    b = _bench()
    inst = {"c": np.array([1.0, -2.0])}
    E = _FakeEngine({(0, 0): (0, [1.0, 1.0]), (1, 0): (0, [1.0, 1.0 + 1e-7]),
                     (0, 1): (1, [0.0, 0.0]), (1, 1): (0, [np.nan, 0.0])})
    out = b.time_to_kkt(E, None, inst)
    assert out["fp64"]["objective"] == -1.0
    assert abs(out["fp32_refined"]["objective_rel_diff_vs_fp64"] - 2e-7 / 2.0) < 1e-15
    assert "speedup_fp32_refined_vs_fp64" in out
    assert "speedup_halpern_fp64_vs_fp64" not in out          # that run did not converge
    assert out["halpern_fp64"]["objective_rel_diff_vs_fp64"] == 0.5
    assert out["halpern_fp32_refined"]["objective_rel_diff_vs_fp64"] is None   # NaN is not JSON
    json.dumps(out, allow_nan=False)


def test_time_to_kkt_survives_instant_solves():
    """A solve faster than the millisecond rounding gives no speed-up entry, not a
    division by zero."""
    b = _bench()
    E = _FakeEngine({(p, a): (0, [1.0]) for p in (0, 1) for a in (0, 1)})
    E.pdlp_solve = lambda A, inst, s: (0, np.array([1.0]), None,
                                       {"status": 0, "iterations": 64, "refinements": 0,
                                        "relative_primal_residual": 0.0, "relative_dual_residual": 0.0,
                                        "relative_gap": 0.0})
    out = b.time_to_kkt(E, None, {"c": np.array([1.0])})
    assert all(out[k]["objective_rel_diff_vs_fp64"] == 0.0 for k in ("fp32_refined", "halpern_fp64"))
    json.dumps(out, allow_nan=False)


def test_clock_summary_parses_nvidia_smi_rows():
    """The clocks record: median SM clock under load, the maximum, and the throttle
    reasons that were Active in any sample (nvidia-smi csv, noheader, nounits)."""
    b = _bench()
    sampler = b.ClockSampler(0)
    sampler.out = "\n".join([
        "0, 1965, 1965, 612.3, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 998.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 700.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
    ])
    s = sampler.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3
    empty = b.ClockSampler(0)
    empty.out = ""
    assert empty.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}


def test_reference_core_prefers_the_openmp_build():
    b = _bench()
    lib_name, threads = b.reference_core()
    omp = os.path.join(ROOT, "oracle", "_ref", "libsankhya_ref_omp.so")
    if os.path.exists(omp):
        assert lib_name == "ref_omp" and threads == len(os.sched_getaffinity(0))
    else:
        assert (lib_name, threads) == ("ref", 1)
    assert "OpenMP" in b._core_text(("ref_omp", 8)) and "1 thread" in b._core_text(("ref", 1))


def test_committed_traffic_figures_parse_as_the_bench_reads_them():
    """bench.py fills roofline.traffic from profiles/traffic_lp_config1.txt (key=value
    lines, # comments): both launches' figures are there and are integers of the size
    of one launch's DRAM bytes."""
    path = os.path.join(ROOT, "profiles", "traffic_lp_config1.txt")
    figures = dict(line.strip().split("=", 1) for line in open(path)
                   if "=" in line and not line.lstrip().startswith("#"))
    for key in ("primal", "dual"):
        v = int(figures[key])
        assert 1e8 < v < 1e9, (key, v)
