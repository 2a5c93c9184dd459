"""NVTX ranges of the library (csrc/lsvd_trace.h), seen through an NVTX
injection library (tests/nvtx_recorder.c) that logs every range of the
process: each C-ABI entry opens one range in the domain "lsvd", closed on
every return path, and the large solve nests its phases inside its entry.

The reference times its solvers with Instant around each call
(src/lib.rs:56-130); these ranges are the device-side counterpart a profiler
attaches to."""
import os
import shutil
import subprocess
import sys
import textwrap

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(ROOT, "lie_cliffalg_analog_svd_b200", "_lib", "liblsvd_b200.so")
CUDA_INC = "/usr/local/cuda/include"


@pytest.fixture(scope="module")
def recorder(tmp_path_factory):
    gcc = shutil.which("gcc") or shutil.which("cc")
    if not gcc or not os.path.exists(os.path.join(CUDA_INC, "nvtx3", "nvToolsExt.h")):
        pytest.skip("needs a C compiler and the NVTX3 headers")
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    out = str(tmp_path_factory.mktemp("nvtx") / "nvtx_recorder.so")
    subprocess.run([gcc, "-shared", "-fPIC", "-O1", "-I", CUDA_INC, os.path.join(HERE, "nvtx_recorder.c"),
                    "-o", out], check=True)
    return out


def _run(recorder, tmp_path, body, timeout=120):
    log = tmp_path / "nvtx.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=recorder, LSVD_NVTX_LOG=str(log), PYTHONPATH=ROOT)
    script = "import ctypes as C, numpy as np\nlib = C.CDLL(%r)\n" % LIB + textwrap.dedent(body)
    r = subprocess.run([sys.executable, "-c", script], env=env, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout, log.read_text().splitlines() if log.exists() else []


def _ranges(lines):
    """(name, depth) for every push of the lsvd domain; asserts pushes and pops balance."""
    stack, seen = [], []
    for ln in lines:
        if ln.startswith("push "):
            seen.append((ln[5:], len(stack)))
            stack.append(ln[5:])
        elif ln == "pop":
            assert stack, "pop without push"
            stack.pop()
    assert not stack, f"unclosed ranges {stack}"
    return seen


def test_entry_ranges_close_on_every_return_path(recorder, tmp_path):
    out, lines = _run(recorder, tmp_path, """
        vp, i64, i32, u32 = C.c_void_p, C.c_int64, C.c_int32, C.c_uint32
        # argument errors return before any device work: the range still closes
        lib.lsvd_micro_solve_f64.argtypes = [vp, i64, vp, i64, vp, i64, vp, vp, i64, vp, u32]
        print(lib.lsvd_micro_solve_f64(None, 2, None, 2, None, 2, None, None, 2, None, 0))
        lib.lsvd_svd_batched_noalloc_f64.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, u32]
        print(lib.lsvd_svd_batched_noalloc_f64(None, -1, None, None, None, None, None, None, 0))
        # the host encoder of the phase-schedule frame runs to completion on the CPU
        rot = np.zeros(3, dtype=[("i", "<u2"), ("j", "<u2"), ("round", "<u4"), ("theta", "<f8")])
        rot["i"], rot["j"], rot["round"], rot["theta"] = [0, 1, 0], [1, 2, 2], [0, 1, 2], [0.1, -0.2, 0.3]
        lib.lsvd_schedule_binary_from_rotors.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, u32]
        n = C.c_int64(0)
        print(lib.lsvd_schedule_binary_from_rotors(None, rot.ctypes.data, 3, 3, 0, None, 0, C.byref(n), 0))
        buf = np.zeros(n.value, np.uint8)
        print(lib.lsvd_schedule_binary_from_rotors(None, rot.ctypes.data, 3, 3, 0, buf.ctypes.data, n.value,
                                                   C.byref(n), 0))
    """)
    codes = [int(x) for x in out.split()]
    assert codes == [4, 4, 0, 0], codes  # LSVD_BAD_ARGUMENT twice, then LSVD_OK
    assert lines.count("domain lsvd") == 1, lines
    assert _ranges(lines) == [("lsvd_micro_solve_f64", 0), ("lsvd_svd_batched_noalloc_f64", 0),
                              ("lsvd_schedule_binary_from_rotors", 0), ("lsvd_schedule_binary_from_rotors", 0)]


def test_no_tool_no_log(tmp_path):
    # without an injection library the ranges are no-ops and the entries behave the same
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    env = {k: v for k, v in os.environ.items() if k != "NVTX_INJECTION64_PATH"}
    code = ("import ctypes as C\nlib = C.CDLL(%r)\n"
            "lib.lsvd_micro_solve_f64.argtypes = [C.c_void_p, C.c_int64] + [C.c_void_p, C.c_int64] * 2"
            " + [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_uint32]\n"
            "print(lib.lsvd_micro_solve_f64(None, 2, None, 2, None, 2, None, None, 2, None, 0))\n") % LIB
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.split() == ["4"], r.stderr


@pytest.mark.gpu
def test_large_solve_phases_nest_inside_the_entry(recorder, tmp_path):
    out, lines = _run(recorder, tmp_path, """
        from lie_cliffalg_analog_svd_b200 import LieSvdSmall
        a = np.random.default_rng(0).standard_normal((256, 256))
        u, s, vt = LieSvdSmall.solve(a)
        print(float(np.linalg.norm((u * s) @ vt - a) / np.linalg.norm(a)))
    """, timeout=600)
    assert float(out.split()[-1]) < 1e-12
    seen = _ranges(lines)
    names = [nm for nm, _ in seen]
    top = names.index("lsvd_small_solve_f64")
    depth = dict(seen[top + 1:])
    for phase in ("large/polar", "polar/newton_schulz", "large/jacobi_two_sided", "large/outputs"):
        assert phase in depth and depth[phase] > seen[top][1], (phase, seen)
