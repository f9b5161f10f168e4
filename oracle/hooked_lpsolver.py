"""TEST INFRASTRUCTURE ONLY: the reference C++ core's LP driver (sihps::solve_lp,
src/lp/LpSolver.cpp) compiled from its own sources with the C entry point of
oracle/ref_lpsolver_shim.cpp, in two builds:

  --hook   run_first_order (src/lp/LpSolver.cpp:62-99) replaced by the integration block
           include/integration/lpsolver_run_first_order.inc, linked to the engine library:
           solve_lp's FIRST_ORDER and HYBRID paths then call sankhya_b200_pdlp_solve, with
           the core's presolve, postsolve, simplex fallback and original-space gate as
           they are;
  (none)   the core unchanged (FIRST_ORDER runs the reference's own GpuPdlp over cuSPARSE).

The spliced LpSolver.cpp goes to the compiler on standard input (no copy of a source
is written); the other sources are compiled where they lie. Objects go to a temporary
directory that is removed afterwards. Used by oracle/Makefile
(oracle/_ref/libsihps_lp_ref.so, oracle/_ref/libsihps_lp_hooked.so) and by the tests.

    python oracle/hooked_lpsolver.py --ref <reference tree> --out <.so> [--hook --lib-dir <engine lib dir>]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BLOCK = os.path.join(ROOT, "include", "integration", "lpsolver_run_first_order.inc")
SHIM = os.path.join(HERE, "ref_lpsolver_shim.cpp")
# The part of the core's library (src/CMakeLists.txt:1-26) that solve_lp needs: sparse
# storage, the CUDA helpers, the GPU pricer and PDLP, the MPS reader, and lp/.
SOURCES = ("memory/MemoryArena.cpp", "sparse/CSRMatrix.cpp", "sparse/CSCMatrix.cpp", "sparse/Convert.cpp",
           "cuda/CudaStream.cpp", "cuda/CudaEvent.cpp", "cuda/CudaDevice.cpp", "cuda/CusparseHandle.cpp",
           "cuda/GpuSpMV.cpp", "cuda/GpuPricer.cpp", "cuda/PricingKernels.cu", "cuda/PdlpKernels.cu",
           "cuda/GpuPdlp.cpp", "io/MpsReader.cpp", "lp/BasisFactorization.cpp", "lp/LpProblem.cpp",
           "lp/Presolve.cpp", "lp/Scaling.cpp", "lp/Simplex.cpp")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def block() -> str:
    return open(BLOCK).read()


def spliced(text: str, body: str) -> str:
    """LpSolver.cpp with run_first_order replaced by `body` and the engine header added
    after the file's own includes."""
    start = text.index("bool run_first_order(const LpProblem& target")
    end = text.index("\n}\n", start) + 3
    out = text[:start] + body + text[end:]
    anchor = '#include "Scaling.hpp"\n'
    if anchor not in out:
        raise ValueError("LpSolver.cpp: include anchor not found")
    return out.replace(anchor, anchor + '#include "sankhya_b200.h"\n', 1)


def spliced_hybrid(text: str, body: str) -> str:
    """LpSolver.cpp with the `try_simplex` lambda of solve_lp's HYBRID branch replaced by
    `body` (include/integration/lpsolver_hybrid_crossover.inc) and the crossover header
    added after the file's own includes."""
    start = text.index("        auto try_simplex = [&]() {")
    end = text.index("\n        };\n", start) + len("\n        };\n")
    out = text[:start] + body + text[end:]
    anchor = '#include "Scaling.hpp"\n'
    if anchor not in out:
        raise ValueError("LpSolver.cpp: include anchor not found")
    return out.replace(anchor, anchor + '#include "sihps_crossover.hpp"\n', 1)


def _run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        raise RuntimeError(" ".join(cmd[:4]) + " ...\n" + r.stderr[-3000:])


def build(ref: str, out: str, hook: bool, lib_dir: str | None = None, rpath: str | None = None,
          hybrid_crossover: bool = False, engine_lib: str = "sankhya_cuda") -> str:
    """hybrid_crossover (with hook): HYBRID's simplex step replaced as well, by
    include/integration/lpsolver_hybrid_crossover.inc, with sihps_crossover.cpp compiled in.
    engine_lib: the library the hook links (lib<engine_lib>.so in lib_dir)."""
    src = os.path.join(ref, "src")
    integration = os.path.join(ROOT, "include", "integration")
    inc = ["-I" + src, "-I" + os.path.join(ROOT, "include"), "-I" + integration, "-I" + os.path.join(CUDA, "include")]
    tmp = tempfile.mkdtemp(prefix="sihps_lp_")
    try:
        def compile_one(rel):
            obj = os.path.join(tmp, rel.replace("/", "_") + ".o")
            path = os.path.join(src, rel)
            if rel.endswith(".cu"):
                _run(["nvcc", "-O3", "-DNDEBUG", "-std=c++17"] + ARCH + ["-Xcompiler", "-fPIC", "-I" + src, "-c", path,
                                                                          "-o", obj])
            else:
                _run(["g++", "-O3", "-DNDEBUG", "-std=c++17", "-fPIC"] + inc + ["-c", path, "-o", obj])
            return obj

        with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
            objs = list(pool.map(compile_one, SOURCES))
        lp_obj = os.path.join(tmp, "lp_LpSolver.cpp.o")
        text = open(os.path.join(src, "lp", "LpSolver.cpp")).read()
        if hook:
            source = spliced(text, block())
            if hybrid_crossover:
                source = spliced_hybrid(source, open(os.path.join(integration, "lpsolver_hybrid_crossover.inc")).read())
                xobj = os.path.join(tmp, "sihps_crossover.o")
                _run(["g++", "-O3", "-DNDEBUG", "-std=c++17", "-fPIC"] + inc +
                     ["-c", os.path.join(integration, "sihps_crossover.cpp"), "-o", xobj])
                objs.append(xobj)
            _run(["g++", "-O3", "-DNDEBUG", "-std=c++17", "-fPIC", "-iquote", os.path.join(src, "lp")] + inc +
                 ["-x", "c++", "-", "-c", "-o", lp_obj], input=source)
        else:
            _run(["g++", "-O3", "-DNDEBUG", "-std=c++17", "-fPIC"] + inc + ["-c", os.path.join(src, "lp", "LpSolver.cpp"),
                                                                             "-o", lp_obj])
        shim_obj = os.path.join(tmp, "shim.o")
        _run(["g++", "-O3", "-DNDEBUG", "-std=c++17", "-fPIC"] + inc + ["-c", SHIM, "-o", shim_obj])
        link = ["nvcc"] + ARCH + ["-shared", "-o", out] + objs + [lp_obj, shim_obj] + [
            "-L" + os.path.join(CUDA, "lib64"), "-lcusparse", "-lcudart",
            "-Xlinker", "-rpath", "-Xlinker", os.path.join(CUDA, "lib64"), "-Xlinker", "--no-undefined"]
        if hook:
            link += ["-L" + lib_dir, "-l" + engine_lib, "-Xlinker", "-rpath", "-Xlinker", rpath or lib_dir]
        _run(link)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--hook", action="store_true")
    ap.add_argument("--lib-dir", default=None)
    ap.add_argument("--rpath", default=None, help="run-time search path for the engine library")
    ap.add_argument("--hybrid-crossover", action="store_true",
                    help="with --hook: HYBRID's simplex step through the crossover as well")
    ap.add_argument("--engine-lib", default="sankhya_cuda", help="with --hook: the library name to link")
    a = ap.parse_args(argv)
    if a.hook and not a.lib_dir:
        ap.error("--hook needs --lib-dir")
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    build(a.ref, a.out, a.hook, a.lib_dir, a.rpath, a.hybrid_crossover, a.engine_lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
