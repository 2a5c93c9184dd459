"""Builds ``liblsvd_b200.so`` (the C ABI of ``include/lsvd.h``) in-tree with
nvcc for sm_100a.  Objects are cached under ``_build/`` next to this file and
rebuilt when their source, a header or the flags changed (content digests).

    python -m lie_cliffalg_analog_svd_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "liblsvd_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers_digest() -> str:
    h = hashlib.sha256()
    for f in sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                    glob.glob(os.path.join(INCLUDE, "*.h"))):
        h.update(f.encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def _compile(src: str, verbose: bool, extra: list[str], headers: str, reuse: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    # an object is current when it was built from this source, these headers and
    # these flags (content, not timestamps: an edit made while a build runs must
    # not leave an object compiled from the old text looking fresh)
    h = hashlib.sha256()
    with open(src, "rb") as fh:
        h.update(fh.read())
    h.update(headers.encode())
    h.update(" ".join([*ARCH, *NVCC_FLAGS, *extra]).encode())
    sig = h.hexdigest()
    sig_path = obj + ".sig"
    if reuse and os.path.exists(obj) and os.path.exists(sig_path):
        with open(sig_path) as fh:
            if fh.read().strip() == sig:
                return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout, r.stderr, flush=True)
    with open(sig_path, "w") as fh:
        fh.write(sig)
    return obj


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compiles every ``csrc/*.cu`` for sm_100a and links the shared library.
    Returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        headers, reuse = _headers_digest(), not (force or ptxas_verbose)
        objs = list(ex.map(lambda s: _compile(s, verbose or ptxas_verbose, extra, headers, reuse), srcs))
    # relink only when an object is newer than the library (freshness is decided per
    # object against its source and the headers, so an edit made while another build
    # ran is never masked by that build's library)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose, a.ptxas_verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
