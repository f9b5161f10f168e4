"""Every function in the repository's Python files refers only to names that exist: a
name a function reads without binding it must be bound at module level or be a
builtin. Catches a missing import in code paths the CPU suite never runs (the gpu
tests, bench.py's other modes) before a GPU run does."""
import builtins
import os
import subprocess
import symtable

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _undefined(path):
    src = open(path).read()
    top = symtable.symtable(src, path, "exec")
    bound = {s.get_name() for s in top.get_symbols() if s.is_assigned() or s.is_imported() or s.is_namespace()}
    found = []

    def walk(table):
        for sym in table.get_symbols():
            name = sym.get_name()
            if (table.get_type() != "module" and sym.is_referenced() and sym.is_global()
                    and not sym.is_declared_global() and name not in bound and not hasattr(builtins, name)
                    and name not in ("__file__", "__name__")):
                found.append(f"{os.path.relpath(path, ROOT)}: {table.get_name()}(): {name}")
        for child in table.get_children():
            walk(child)

    walk(top)
    return found


def test_no_undefined_names():
    out = subprocess.run(["git", "ls-files", "*.py"], cwd=ROOT, capture_output=True, text=True)
    files = [os.path.join(ROOT, f) for f in out.stdout.split()] if out.returncode == 0 else []
    if not files:   # not a git checkout: walk the tree instead
        for d, _, names in os.walk(ROOT):
            if "/_work" in d or "/.git" in d or "gpurun_out" in d:
                continue
            files += [os.path.join(d, n) for n in names if n.endswith(".py")]
    assert files
    problems = [p for f in files for p in _undefined(f)]
    assert not problems, problems


def test_the_check_finds_a_missing_import(tmp_path):
    planted = tmp_path / "planted.py"
    planted.write_text("import os\n\ndef f():\n    import numpy as np\n    return np.zeros(1)\n\n"
                       "def g():\n    return np.ones(2), os.sep\n")
    assert _undefined(str(planted)) == [f"{os.path.relpath(str(planted), ROOT)}: g(): np"]
