"""TEST INFRASTRUCTURE ONLY: the reference's C core with the sk_solve integration block
(include/integration/sk_solve_hook.inc) applied.

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


def build(ref: str, out: str, lib_dir: str, lib_name: str = "sankhya_cuda", rpath: str | None = None) -> str:
    """Compiles the patched core into `out`, linked to lib<lib_name>.so in lib_dir."""
    src = os.path.join(ref, "c", "src")
    patched = patched_source(open(os.path.join(src, "sk_solve.c")).read(), snippet())
    cc = os.environ.get("CC", "gcc")
    cmd = [cc, "-O3", "-DNDEBUG", "-std=gnu11", "-fPIC", "-shared", "-DSANKHYA_WITH_B200",
           "-I" + os.path.join(ref, "c", "include"), "-I" + os.path.join(ROOT, "include"),
           "-x", "c", "-", "-x", "none"] + [os.path.join(src, f) for f in C_SOURCES] + [
           "-L" + lib_dir, "-l" + lib_name, "-Wl,-rpath," + (rpath or lib_dir), "-o", out, "-lm"]
    r = subprocess.run(cmd, input=patched, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-3000:])
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    ap.add_argument("--lib-dir", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--rpath", default=None, help="run-time search path for the engine library")
    a = ap.parse_args(argv)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    build(a.ref, a.out, a.lib_dir, rpath=a.rpath)
    return 0


if __name__ == "__main__":
    sys.exit(main())
