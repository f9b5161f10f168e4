"""TEST INFRASTRUCTURE ONLY: the reference's C core with the sk_solve integration block
(include/integration/sk_solve_hook.inc) applied, and optionally (--milp-node) the
branch-and-bound node block (include/integration/sk_milp_node.inc) in sk_milp.c's
milp_solve_lp.

The block is read from include/integration/sk_solve_hook.inc and inserted into the reference's
c/src/sk_solve.c before the first-order loop of solve_continuous (at
`start = sk_wall_seconds();`), with the `after_loop:` label after the
`performed_iterations` assignment. The patched file goes to gcc on standard input
(no copy of the source is written) and is compiled with the reference's other C core
sources where they lie, into a shared library linked to the engine library. Used by
oracle/Makefile (oracle/_ref/libsankhya_ref_hooked.so, for the gpu tests, which run
sk_solve through it) and by the CPU tests.

    python oracle/hooked_core.py --ref <reference tree> --lib-dir <engine lib dir> --out <.so>
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
C_SOURCES = ("sankhya_model.c", "sankhya_lu.c", "sankhya_mps.c", "sankhya_verify.c", "sk_lu.c", "sk_core.c",
             "sk_simplex.c", "sk_scale.c", "sk_milp.c")


HOOK = os.path.join(ROOT, "include", "integration", "sk_solve_hook.inc")


def snippet() -> str:
    """The integration block as a maintainer pastes it into solve_continuous."""
    return open(HOOK).read()


def patched_source(text: str, body: str) -> str:
    """sk_solve.c with the block before the loop and the label after it."""
    start = text.index("static sk_status solve_continuous(")
    loop = text.index("\n    start = sk_wall_seconds();\n", start)
    done = text.index("\n    performed_iterations = iteration > maximum_iterations", loop)
    done_end = text.index("\n", done + 1)
    out = text[:loop + 1] + body + text[loop + 1:done_end + 1] + "after_loop:;\n" + text[done_end + 1:]
    return out.replace('#include "sankhya.h"\n', '#include "sankhya.h"\n#include "sankhya_b200.h"\n', 1)


MILP_NODE = os.path.join(ROOT, "include", "integration", "sk_milp_node.inc")
MILP_LP_BRANCH = """    } else {
        memset(&ss, 0, sizeof(ss));
        if (sk_simplex_solve(&M->work, &M->lp_opt, &M->ls, &ss) != SK_OK)
            return SK_RESULT_NUMERIC_FAILURE;
        M->st.simplex_iterations += ss.iterations;
    }"""


def milp_node_snippet() -> str:
    """The node block as a maintainer pastes it into milp_solve_lp's LP branch."""
    return open(MILP_NODE).read()


def patched_milp(text: str, body: str) -> str:
    """sk_milp.c with the body of milp_solve_lp's LP branch replaced by `body`."""
    start = text.index("static sk_result milp_solve_lp(")
    at = text.index(MILP_LP_BRANCH, start)
    return text[:at] + "    } else {\n" + body + "    }" + text[at + len(MILP_LP_BRANCH):]


def build(ref: str, out: str, lib_dir: str, lib_name: str = "sankhya_cuda", rpath: str | None = None,
          milp_node: bool = False) -> str:
    """Compiles the patched core into `out`, linked to lib<lib_name>.so in lib_dir. With
    milp_node, sk_milp.c's node relaxations go through the engine as well. Each patched
    file goes to the compiler on standard input; objects go to a temporary directory."""
    import shutil
    import tempfile
    src = os.path.join(ref, "c", "src")
    cc = os.environ.get("CC", "gcc")
    flags = [cc, "-O3", "-DNDEBUG", "-std=gnu11", "-fPIC", "-DSANKHYA_WITH_B200",
             "-I" + os.path.join(ref, "c", "include"), "-I" + src, "-I" + os.path.join(ROOT, "include")]
    patched = {"sk_solve.c": patched_source(open(os.path.join(src, "sk_solve.c")).read(), snippet())}
    if milp_node:
        patched["sk_milp.c"] = patched_milp(open(os.path.join(src, "sk_milp.c")).read(), milp_node_snippet())
    tmp = tempfile.mkdtemp(prefix="sk_hooked_")
    try:
        objs = []
        for name, text in patched.items():
            obj = os.path.join(tmp, name + ".o")
            r = subprocess.run(flags + ["-c", "-x", "c", "-", "-o", obj], input=text, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(name + ": " + r.stderr[-3000:])
            objs.append(obj)
        cmd = flags + ["-shared"] + objs + [os.path.join(src, f) for f in C_SOURCES if f not in patched] + [
            "-L" + lib_dir, "-l" + lib_name, "-Wl,-rpath," + (rpath or lib_dir), "-o", out, "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(r.stderr[-3000:])
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    ap.add_argument("--lib-dir", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--rpath", default=None, help="run-time search path for the engine library")
    ap.add_argument("--milp-node", action="store_true", help="also route sk_milp's node LPs through the engine")
    a = ap.parse_args(argv)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    build(a.ref, a.out, a.lib_dir, rpath=a.rpath, milp_node=a.milp_node)
    return 0


if __name__ == "__main__":
    sys.exit(main())
