"""C-ABI boundary checks that need no GPU: the library builds, loads, exports every symbol
declared in include/rsdft_b200.h, and rejects calls made before initialisation."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from rsdft_develop_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "rsdft_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rsdft_gpu_\w+)\s*\(", src)))


def test_header_matches_exports():
    assert _declared() == sorted(api.EXPORTS)


def _declared_arity():
    src = open(os.path.join(ROOT, "include", "rsdft_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(rsdft_gpu_\w+)\s*\(([^)]*)\)\s*;", src):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else len(args.split(","))
    return out


def test_ctypes_signatures_match_header():
    lib = api.load_library()
    for name, n in _declared_arity().items():
        f = getattr(lib, name)
        assert f.argtypes is not None, name
        assert len(f.argtypes) == n, (name, len(f.argtypes), n)


def test_library_exports_every_declared_symbol():
    lib = api.load_library()
    for name in _declared():
        assert hasattr(lib, name), name


def test_calls_before_init_fail_cleanly():
    lib = api.load_library()
    x = np.zeros(8)
    r = lib.rsdft_gpu_hamiltonian_d(1, 1, C.c_void_p(x.ctypes.data), C.c_void_p(x.ctypes.data), 8, 1, 0)
    assert r == -7  # RSDFT_ERR_STATE
    assert b"rsdft_gpu_init" in lib.rsdft_gpu_last_error()
    assert lib.rsdft_gpu_init(None) == -1
    assert lib.rsdft_gpu_kernel_launches() == 0
    e = np.zeros(2)
    assert lib.rsdft_gpu_xc_pbe(C.c_void_p(x.ctypes.data), C.c_void_p(x.ctypes.data), C.c_void_p(e.ctypes.data)) == -7
    assert b"rsdft_gpu_init" in lib.rsdft_gpu_last_error()


def test_oracle_not_imported_by_product():
    pkg = os.path.join(ROOT, "rsdft_develop_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in txt and "from oracle" not in txt, f
                assert "liborc" not in txt, f
