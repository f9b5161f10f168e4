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
    FP64, FP32_REFINE, BF16_REFINE, PDLP_ADAPTIVE, PDLP_HALPERN = 0, 1, 2, 0, 1

    def __init__(self, answers):
        self.answers = answers

    def pdlp_default_settings(self):
        return _Settings()

    def pdlp_solve(self, A, inst, s):
        import time
        time.sleep(0.002)   # wall times are rounded to milliseconds
        status, x = self.answers[(s.precision, s.algorithm)]
        r = {"status": status, "iterations": 640, "restarts": 3, "refinements": 4 * int(s.precision == 1),
             "relative_primal_residual": 1e-7, "relative_dual_residual": 1e-7, "relative_gap": 1e-7}
        return 0, np.asarray(x, dtype=float), None, r


def test_iteration_bytes_are_the_two_launches():
    b = _bench()
    m, n, nnz = 1_000_000, 2_000_000, 20_000_000
    assert b.iteration_bytes(m, n, nnz) == b.dual_bytes(m, n, nnz) + b.primal_bytes(m, n, nnz)
    assert b.dual_bytes(m, n, nnz) == 12 * nnz + 4 * (m + 1) + 8 * n + 32 * m
    assert b.primal_bytes(m, n, nnz) == 12 * nnz + 4 * (n + 1) + 8 * m + 48 * n


def test_time_to_kkt_reports_speedups_and_objective_error(monkeypatch):
    """One row per tolerance: FP64, FP32-refined and bf16-value runs, the speed-up where both
    converged, and each objective's relative error against the oracle value."""
    b = _bench()
    monkeypatch.setattr(b, "oracle_objective", lambda: -1.0)
    inst = {"c": np.array([1.0, -2.0])}
    E = _FakeEngine({(0, 0): (0, [1.0, 1.0]), (1, 0): (0, [1.0, 1.0 + 1e-7]), (2, 0): (0, [1.0, 1.0 + 2e-7]),
                     (0, 1): (1, [0.0, 0.0]), (1, 1): (0, [np.nan, 0.0])})
    out = b.time_to_kkt(E, None, inst, eps_list=(1e-4, 1e-6, 1e-8), halpern=True)
    assert out["oracle_objective"] == -1.0
    for key in ("eps_1e-04", "eps_1e-06", "eps_1e-08"):
        row = out[key]
        assert row["fp64"]["objective"] == -1.0 and row["fp64"]["objective_rel_err_vs_oracle"] == 0.0
        assert abs(row["fp32_refined"]["objective_rel_err_vs_oracle"] - 2e-7 / 2.0) < 1e-15
        assert row["fp32_refined"]["refinements"] == 4
        assert "speedup_fp32_refined_vs_fp64" in row
        assert abs(row["bf16_values_refined"]["objective_rel_err_vs_oracle"] - 4e-7 / 2.0) < 1e-15
        assert "speedup_bf16_values_refined_vs_fp64" in row
    assert "halpern_fp64" in out["eps_1e-06"] and "halpern_fp64" not in out["eps_1e-04"]
    assert "speedup_halpern_fp64_vs_fp64" not in out["eps_1e-06"]     # that run did not converge
    assert out["eps_1e-06"]["halpern_fp64"]["objective_rel_err_vs_oracle"] == 0.5
    json.dumps(out, allow_nan=False)


def test_time_to_kkt_without_oracle_and_nan_objective(monkeypatch):
    """No oracle file: no error entries; a NaN objective is reported as null (strict JSON)."""
    b = _bench()
    monkeypatch.setattr(b, "oracle_objective", lambda: None)
    E = _FakeEngine({(0, 0): (0, [1.0]), (1, 0): (0, [np.nan]), (2, 0): (0, [1.0])})
    out = b.time_to_kkt(E, None, {"c": np.array([1.0])}, eps_list=(1e-6,))
    row = out["eps_1e-06"]
    assert "objective_rel_err_vs_oracle" not in row["fp64"]
    assert row["fp32_refined"]["objective"] is None
    json.dumps(out, allow_nan=False)


def test_time_to_kkt_survives_instant_solves(monkeypatch):
    """A solve faster than the millisecond rounding gives no speed-up entry, not a
    division by zero."""
    b = _bench()
    monkeypatch.setattr(b, "oracle_objective", lambda: 1.0)
    E = _FakeEngine({(p, a): (0, [1.0]) for p in (0, 1) for a in (0, 1)})
    E.pdlp_solve = lambda A, inst, s: (0, np.array([1.0]), None,
                                       {"status": 0, "iterations": 64, "restarts": 0, "refinements": 0,
                                        "relative_primal_residual": 0.0, "relative_dual_residual": 0.0,
                                        "relative_gap": 0.0})
    out = b.time_to_kkt(E, None, {"c": np.array([1.0])}, eps_list=(1e-6,))
    row = out["eps_1e-06"]
    assert "speedup_fp32_refined_vs_fp64" not in row
    assert row["fp32_refined"]["objective_rel_err_vs_oracle"] == 0.0
    json.dumps(out, allow_nan=False)


def test_oracle_objective_file_parses():
    """The committed oracle value (where present) is a finite float the bench can use."""
    b = _bench()
    v = b.oracle_objective()
    if os.path.exists(b.ORACLE_OBJECTIVE):
        assert v is not None and np.isfinite(v)
    else:
        assert v is None


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


def test_config0_leg_reports_each_mode_against_the_simplex(monkeypatch):
    """The config-0 leg: one row per precision with its objective error against the
    simplex golden, the best of the timed solves, and a reference row (here
    unavailable, as on a machine without the reference build)."""
    b = _bench()
    calls = []

    class _I:
        @staticmethod
        def lp_config0(seed):
            return {"c": np.array([1.0, -2.0]), "m": 1, "n": 2}

    class _E(_FakeEngine):
        class Matrix:
            @staticmethod
            def from_instance(inst):
                class _M:
                    def close(self):
                        calls.append("close")
                return _M()

    E = _E({(0, 0): (0, [1.0, 1.0]), (1, 0): (0, [1.0, 1.0]), (2, 0): (0, [1.0, 1.0])})
    import builtins
    import sys
    monkeypatch.setattr(sys, "path", list(sys.path))
    real_import = builtins.__import__

    def no_oracle(name, *a, **k):
        if name == "oracle":
            raise FileNotFoundError("reference build absent")
        return real_import(name, *a, **k)

    monkeypatch.setattr(builtins, "__import__", no_oracle)
    out = b.config0_to_1e8(E, _I, reps=2)
    assert out["eps"] == 1e-8 and calls == ["close"]
    for name in ("fp64", "fp32_refined", "bf16_values_refined"):
        assert out[name]["status"] == 0
        if out["oracle_objective"] is not None:
            assert "objective_rel_err_vs_oracle" in out[name]
    assert "unavailable" in out["reference_gpupdlp"]
    json.dumps(out, allow_nan=False)


def test_polish_legs_report_plain_and_polished_answers(monkeypatch):
    """The --polish legs: per instance the plain 1e-4 solve and one polished solve per
    gap target, each with its quality against the instance (row violation, objective
    error against the oracle value) and the polishing counters, as strict JSON."""
    b = _bench()
    monkeypatch.setattr(b, "oracle_objective", lambda: -3.0)
    solves = []

    def tiny(seed):
        # one row x0 + x1 in [1, 2], boxes [0, 10]
        return {"m": 1, "n": 2, "ptr": np.array([0, 2]), "idx": np.array([0, 1]), "val": np.array([1.0, 1.0]),
                "c": np.array([-1.0, -2.0]), "rl": np.array([1.0]), "ru": np.array([2.0]),
                "cl": np.zeros(2), "cu": np.full(2, 10.0)}

    class _I:
        lp_config1 = staticmethod(tiny)
        lp_config0 = staticmethod(tiny)

    class _E:
        class Matrix:
            @staticmethod
            def from_instance(inst):
                class _M:
                    def close(self):
                        solves.append("close")
                return _M()

        def pdlp_default_settings(self):
            return _Settings()

        def pdlp_solve(self, A, inst, s):
            solves.append(("plain", s.eps_optimal))
            r = {"status": 0, "iterations": 64, "relative_primal_residual": 1e-5, "relative_dual_residual": 0.0,
                 "relative_gap": 9e-5}
            return 0, np.array([0.0, 2.1]), np.zeros(1), r

        def pdlp_solve_polished(self, A, inst, s):
            solves.append(("polished", s.eps_optimal))
            r = {"status": 0, "iterations": 192, "relative_primal_residual": 0.0, "relative_dual_residual": 0.0,
                 "relative_gap": s.eps_optimal / 2}
            pr = {"rounds": 2, "main_iterations": 128, "primal_iterations": 64, "dual_iterations": 0,
                  "main_seconds": 0.01, "polish_seconds": 0.001, "pair_relative_primal_residual": 0.0,
                  "pair_relative_gap": s.eps_optimal / 2, "pair_primal_objective": -4.0,
                  "main_relative_primal_residual": 1e-6, "main_relative_gap": float("nan")}
            return 0, np.array([0.0, 2.0]), np.zeros(1), r, pr

    out = b.polish_legs(_E(), _I, time_limit=1.0)
    assert solves.count("close") == 2
    assert [c for c in solves if c != "close"] == [("plain", 1e-4), ("polished", 1e-4), ("polished", 1e-6),
                                                    ("plain", 1e-4), ("polished", 1e-4), ("polished", 1e-8)]
    c1 = out["lp_config1"]
    assert abs(c1["plain_1e-4"]["row_violation_rel"] - 0.1 / 3.0) < 1e-12
    pol = c1["polished_gap_1e-04"]
    assert pol["row_violation_rel"] == 0.0 and pol["rounds"] == 2 and pol["primal_polish_iterations"] == 64
    assert abs(pol["objective_rel_err_vs_oracle"] - 1.0 / 4.0) < 1e-12
    assert pol["main_at_last_handover"]["relative_gap"] is None    # NaN is not JSON
    assert "polished_gap_1e-08" in out["lp_config0"]
    json.dumps(out, allow_nan=False)


def test_crossover_leg_reaches_the_certified_vertex():
    """The --crossover leg with a stand-in engine that answers with the oracle's PDLP
    point (the engine's algorithm) at config 0's 1e-8: the C++ core's seated basis gives
    the certified optimum through its warm start, and the C core's identified basis is
    certified as it stands (no simplex)."""
    import pytest
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not (O.available("ref_sihps_crossover") and O.available("oracle")):
        pytest.skip("reference cores not built (make -C oracle ref)")
    b = _bench()
    spec = importlib.util.spec_from_file_location("inst_for_bench", os.path.join(ROOT, "the-solver_b200", "instances.py"))
    I = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(I)

    class _E:
        class Matrix:
            @staticmethod
            def from_instance(inst):
                class _M:
                    def close(self):
                        pass
                return _M()

        def pdlp_default_settings(self):
            return _Settings()

        def pdlp_solve(self, A, inst, s):
            x, y, st = O.pdlp(inst, eps=s.eps_optimal, max_iterations=s.max_iterations)
            return 0, x, y, {"status": 0 if st["converged"] else 1, "iterations": st["iterations"]}

    if not O.available("ref_crossover"):
        pytest.skip("reference C core not built (make -C oracle ref)")
    out = b.crossover_legs(_E(), I, O)
    cpp, cc = out["cpp_core_crossover"], out["c_core_crossover"]
    assert out["engine_pdlp"]["status"] == 0
    assert cpp["rc"] == 0 and cpp["status"] == 0 and cpp["used_warm_start"] == 1, cpp
    assert cpp["objective_rel_err_vs_oracle"] < 1e-9 and cpp["dual_pivots"] <= 50, cpp
    assert cc["rc"] == 0 and cc["result"] == 0 and cc["direct"] == 1 and cc["pivots"] == 0, cc
    assert cc["objective_rel_err_vs_oracle"] < 1e-9, cc
    json.dumps(out, allow_nan=False)
