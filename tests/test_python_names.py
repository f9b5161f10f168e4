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


def test_fixture_attributes_used_by_the_tests_exist(engine, oracle, instances, learned):
    """Every `engine.X`, `oracle.X`, `instances.X` and `learned.X` the test files use
    (the gpu ones included, which the CPU suite only imports) exists on the module the
    fixture provides."""
    import ast
    mods = {"engine": engine, "oracle": oracle, "instances": instances, "learned": learned}
    missing = []
    tests_dir = os.path.join(ROOT, "tests")
    for name in sorted(os.listdir(tests_dir)):
        if not name.endswith(".py"):
            continue
        path = os.path.join(tests_dir, name)
        for node in ast.walk(ast.parse(open(path).read(), path)):
            if (isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name) and node.value.id in mods
                    and isinstance(node.ctx, ast.Load) and not hasattr(mods[node.value.id], node.attr)):
                missing.append(f"{name}:{node.lineno}: {node.value.id}.{node.attr}")
    assert not missing, missing


def test_bench_and_trainer_module_attributes_exist(engine, oracle, instances):
    """bench.py reaches the engine, instance and oracle modules as E, I and O, and the
    warm-start trainer (the-solver_b200/learned.py) takes the engine as `engine`; their
    gpu paths never run on CPU: every attribute they use on those modules exists."""
    import ast
    missing = []
    for rel, mods in (("bench.py", {"E": engine, "I": instances, "O": oracle}),
                      (os.path.join("the-solver_b200", "learned.py"), {"engine": engine, "I": instances})):
        path = os.path.join(ROOT, rel)
        missing += [f"{rel}:{n.lineno}: {n.value.id}.{n.attr}"
                    for n in ast.walk(ast.parse(open(path).read(), path))
                    if isinstance(n, ast.Attribute) and isinstance(n.value, ast.Name) and n.value.id in mods
                    and isinstance(n.ctx, ast.Load) and not hasattr(mods[n.value.id], n.attr)]
    assert not missing, missing
