"""The C-ABI boundary: the in-tree library loads, exports every function that
include/lsvd.h declares, and behaves correctly without a GPU (no compute)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from lie_cliffalg_analog_svd_b200 import _lib as L
from lie_cliffalg_analog_svd_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"LSVD_API\s+[\w\s\*]+?\b(lsvd_\w+)\s*\(", txt))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    B.build()
    return L.load()


def test_header_declares_entry_points():
    names = header_functions()
    for must in ("lsvd_small_solve_f64", "lsvd_micro_solve_f64", "lsvd_svd_batched_f64",
                 "lsvd_metrics_f64", "lsvd_context_create"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (lsvd_\w+)", out))
    missing = [n for n in header_functions() if n not in exported]
    assert not missing, missing
    # the ctypes table covers the header too
    assert set(header_functions()) <= set(L.SIGNATURES) | set(L.OPTIONAL_SIGNATURES)


def test_library_exports_nothing_else(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    ours = set(re.findall(r"\bT (lsvd_\w+)", out))
    assert ours == set(header_functions())


def test_status_strings_and_version(lib):
    assert b"sm_100a" in lib.lsvd_version()
    for s in range(10):
        assert lib.lsvd_status_string(s)


def test_structs_match_header(lib):
    assert C.sizeof(L.Diag) == 48
    assert C.sizeof(L.Rotor) == 16
    assert C.sizeof(L.PolarInfo) == 56
    assert np.dtype(L.DIAG_DTYPE).itemsize == 48
    assert np.dtype(L.ROTOR_DTYPE).itemsize == 16


def test_null_arguments_are_rejected(lib):
    assert lib.lsvd_context_create(0, None) == L.BAD_ARGUMENT
    assert lib.lsvd_context_destroy(None) == L.BAD_ARGUMENT
    assert lib.lsvd_small_solve_f64(None, 4, None, 4, None, 4, None, None, 4, None, None, 0,
                                    None, None, 0) == L.BAD_ARGUMENT


def test_no_device_is_reported_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert lib.lsvd_context_create(0, C.byref(h)) == L.NO_DEVICE


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "lie_cliffalg_analog_svd_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(dirpath, f)).read()
                assert not re.search(r"^\s*(import|from)\s+oracle|lsvd_oracle|oracle/", txt, re.M), f


def _header_text():
    txt = open(os.path.join(ROOT, "include", "lsvd.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return re.sub(r"//[^\n]*", "", txt)


def test_rust_binding_matches_header():
    # rust/lie_svd_gpu/src/ffi.rs declares every export with the header's
    # parameter count, and every struct with the header's fields in order
    # (the crate is source only: no Rust toolchain here)
    rs = open(os.path.join(ROOT, "rust", "lie_svd_gpu", "src", "ffi.rs")).read()
    hdr = _header_text()
    c_fns = {m.group(1): m.group(2) for m in re.finditer(r"LSVD_API[^;(]*?\b(lsvd_\w+)\s*\(([^)]*)\)\s*;", hdr)}
    r_fns = {m.group(1): m.group(2) for m in re.finditer(r"pub fn (lsvd_\w+)\s*\(([^)]*)\)", rs)}
    assert set(r_fns) == set(c_fns) == set(header_functions())

    def arity(args):
        args = " ".join(args.split())
        return 0 if args in ("", "void") else args.count(",") + 1

    for name, args in c_fns.items():
        assert arity(r_fns[name]) == arity(args), name
    c_structs = {m.group(2): re.findall(r"(\w+)\s*(?:\[\w+\])?\s*(?:,|;)", m.group(1))
                 for m in re.finditer(r"typedef struct\s*\w*\s*\{(.*?)\}\s*(\w+);", hdr, flags=re.S)}
    r_structs = {m.group(1): re.findall(r"pub (\w+):", m.group(2))
                 for m in re.finditer(r"pub struct (\w+)\s*\{(.*?)\}", rs, flags=re.S)}
    pairs = {"lsvd_diag": "LsvdDiag", "lsvd_rotor": "LsvdRotor", "lsvd_large_info": "LsvdLargeInfo",
             "lsvd_joint_params": "LsvdJointParams", "lsvd_joint_trace": "LsvdJointTrace",
             "lsvd_triage": "LsvdTriage", "lsvd_polar_info": "LsvdPolarInfo", "lsvd_mzi_phase": "LsvdMziPhase",
             "lsvd_schedule_header": "LsvdScheduleHeader", "lsvd_schedule_record": "LsvdScheduleRecord"}
    assert set(pairs) == set(c_structs)
    for c_name, r_name in pairs.items():
        assert r_structs[r_name] == c_structs[c_name], c_name
