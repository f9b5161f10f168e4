"""The C-ABI library loads and exports every symbol the headers declare; the
ctypes mirrors have the C struct sizes. No GPU needed (no compute calls)."""
import ctypes as C
import os
import re

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    names = []
    for h in ("sankhya_cuda.h", "sankhya_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"SANKHYA_CUDA_API\s+[\w\s\*]+?\b(\w+)\s*\(", text)
    return names


def test_headers_declare_the_reference_abi(engine):
    names = declared_symbols()
    for s in engine.REFERENCE_SYMBOLS:
        assert s in names, s
    # the reference header declares exactly these 13 public functions
    assert len(engine.REFERENCE_SYMBOLS) == 13


def test_library_exports_every_declared_symbol(engine):
    L = engine.lib()
    for s in declared_symbols():
        assert hasattr(L, s), f"missing export {s}"


def test_struct_layouts_match_reference():
    import sankhya_b200 as E
    # SankhyaCudaCSR: 3 ints + 3 pointers (with padding after the ints)
    assert C.sizeof(E.CSR) == 4 * 3 + 4 + 8 * 3
    assert C.sizeof(E.Settings) == 4 * 2 + 8 * 5
    assert C.sizeof(E.Result) == 4 * 2 + 8 * 6
    assert E.Settings.time_limit.offset == 40


def test_no_device_is_a_clean_error(engine):
    """Without a GPU the entry points fail with -1 and an error text (no fallback)."""
    import numpy as np
    import torch
    if torch.cuda.is_available():
        return
    rc, y = engine.spmv_host(2, 3, [0, 2, 4], [0, 2, 1, 2], [1.0, 2, 3, 4], [2.0, 5, 7])
    assert rc != 0 and "device" in engine.last_error().lower()
