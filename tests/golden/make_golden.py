"""Generates ``tests/golden/named_sigma.json``: singular values of the named
test matrices of ``src/lie_svd_benchmarks.rs`` (Kahan, Hilbert, Pei, Frank,
Parter, Cauchy, Vandermonde) computed with mpmath at 60 significant digits
(the cross-check the reference's ``compare/`` crate does with MPFR,
``compare/src/main.rs:121-157``).

The Rust reference cannot be run here (no rustc/cargo), and its own tests
store no golden vectors -- they pin properties and the Pei closed form.  These
high-precision values are the independent ground truth the oracle and the
CUDA library are both checked against.

Run: ``python tests/golden/make_golden.py`` (takes ~1 minute).
"""
import json
import os
import sys

import mpmath as mp

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", ".."))
from lie_cliffalg_analog_svd_b200 import profiles as P  # noqa: E402

mp.mp.dps = 60


def mp_sigma(a):
    m = mp.matrix(a.tolist())
    s = mp.svd_r(m, compute_uv=False)
    vals = sorted((s[i] for i in range(s.rows)), reverse=True)
    return [mp.nstr(v, 40) for v in vals]


CASES = {
    "kahan_16_1.2": lambda: P.kahan_matrix(16, 1.2),
    "kahan_32_1.2": lambda: P.kahan_matrix(32, 1.2),
    "hilbert_6": lambda: P.hilbert_matrix(6),
    "hilbert_8": lambda: P.hilbert_matrix(8),
    "hilbert_10": lambda: P.hilbert_matrix(10),
    "pei_16_0.01": lambda: P.pei_matrix(16, 0.01),
    "frank_8": lambda: P.frank_matrix(8),
    "frank_12": lambda: P.frank_matrix(12),
    "parter_16": lambda: P.parter_matrix(16),
    "cauchy_6": lambda: P.cauchy_matrix(6),
    "vandermonde_6": lambda: P.vandermonde_matrix(6),
}


def main():
    out = {}
    for name, fn in CASES.items():
        a = fn()
        out[name] = {"n": int(a.shape[0]), "sigma": mp_sigma(a)}
        print(name, out[name]["sigma"][0], out[name]["sigma"][-1], flush=True)
    path = os.path.join(os.path.dirname(__file__), "named_sigma.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
