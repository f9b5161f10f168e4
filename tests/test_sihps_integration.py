"""The sihps caller written in INTEGRATION.md section 3: `run_first_order`
(src/lp/LpSolver.cpp:62-99) replaced by one sankhya_b200_pdlp_solve call.

Where the reference sources are present, the test takes the reference's
src/lp/LpSolver.cpp, replaces the body of run_first_order with the documented
function, adds this repository's header, and compiles the translation unit from
standard input with g++ -fsyntax-only (no copy of the source is written): the names,
types and signatures the block uses must match both the reference's C++ core
(LpProblem, CSRMatrix, PdlpParams, PdlpStats) and this library's C ABI. Linking and
running need the rest of the C++ core, which its own CMake project builds; that is not
run here."""
import os
import re
import subprocess

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _reference():
    import importlib.util
    spec = importlib.util.spec_from_file_location("graft_entry", os.path.join(ROOT, "__graft_entry__.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.REFERENCE


def _block():
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    section = doc.split("## 3.")[1].split("## 4.")[0]
    return re.search(r"```cpp\n(.*?)```", section, re.S).group(1)


def _spliced(text, block):
    start = text.index("bool run_first_order(const LpProblem& target")
    end = text.index("\n}\n", start) + 3
    out = text[:start] + block + text[end:]
    anchor = '#include "Scaling.hpp"\n'
    assert anchor in out
    return out.replace(anchor, anchor + '#include "sankhya_b200.h"\n', 1)


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
