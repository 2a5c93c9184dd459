"""The oracle against the reference's own printed outputs (no GPU).

The reference prints rounding-level statistics (orthogonality, reconstruction
residual, final joint off-diagonal norm) and exact counts (sweeps, accepted
rotations) for inputs it builds without an RNG stream: the RNG-free stress
profiles (src/lib.rs:270-314) and the Phase-JADE / joint-SVD smoke families of
its stress binary (src/bin/stress_cpu.rs:472-500, :597-624, whose
``deterministic_orthogonal`` is a 64-bit LCG).  The oracle, fed the same
inputs, reproduces them to the printed digits: its products follow ndarray's
``dot`` (sequential fused multiply-adds, matrixmultiply 0.3.11) and its
solvers the reference's loops.  Values from ``tests/golden/reference_outputs.json``
(extracted by ``tests/golden/extract_reference_outputs.py``)."""
import json
import os

import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import profiles as P

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))


def rust_e3(x: float) -> str:
    """Rust ``format!("{:.3e}", x)``: no '+' and no zero padding in the exponent."""
    m, e = f"{x:.3e}".split("e")
    return f"{m}e{int(e)}"


def small_metrics(n, profile):
    a = P.generate(n, profile, 17)[0]
    u, s, vt = O.LieSvdSmall.solve(a)
    return O.metrics.compute(a, u, s, vt, None)


@pytest.mark.parametrize("row", GOLD["small_n64"], ids=lambda r: r["profile"])
def test_small_solve_rounding_statistics_n64(row):
    # LieSvdSmall::solve + metrics::compute (src/lib.rs:149-194) at n = 64:
    # all three statistics to the four printed digits
    m = small_metrics(64, row["profile"])
    assert (rust_e3(m.rel_recon), rust_e3(m.orth_u), rust_e3(m.orth_v)) == \
        (row["rel_recon"], row["orth_u"], row["orth_v"])


@pytest.mark.parametrize("row", GOLD["auto_n32"], ids=lambda r: r["profile"])
def test_small_solve_rounding_statistics_n32(row):
    assert rust_e3(small_metrics(32, row["profile"]).rel_recon) == row["rel_recon"]


def jade_family(n):
    # print_joint_phase_jade_smoke (src/bin/stress_cpu.rs:472-486)
    q = O.deterministic_orthogonal(n, [0x9E3779B97F4A7C15])
    base = np.abs(np.sin(np.arange(n) + 1.0))
    return [O.dot(O.dot(q, np.diag(1.0 + k * 0.2 + base)), q.T.copy()) for k in range(6)]


def joint_svd_family(n):
    # print_joint_svd_smoke (src/bin/stress_cpu.rs:597-610)
    st = [0xA24BAED4963EE407]
    u0 = O.deterministic_orthogonal(n, st)
    v0 = O.deterministic_orthogonal(n, st)
    return [O.dot(O.dot(u0, np.diag(1.0 + k * 0.15 + np.arange(n) * 0.05)), v0.T.copy()) for k in range(4)]


@pytest.mark.parametrize("row", GOLD["jade"], ids=lambda r: f"n{r['n']}")
def test_phase_jade_smoke(row):
    n = row["n"]
    _, _, tr = O.LieSvdJoint.diagonalize_symmetric_with_params(jade_family(n),
                                                               O.JointDiagonalizationParams.for_n(n))
    assert rust_e3(tr.initial_offdiag) == row["initial_offdiag"]
    assert tr.sweeps == row["sweeps"] and tr.rejected_rotations == 0
    if n in (64, 128):
        # every printed digit and the exact rotation count
        assert rust_e3(tr.final_offdiag) == row["final_offdiag"] and tr.rotations == row["rotations"]
    else:
        # n = 16 / 256: the final norm within 0.5 % and the count within one rotation (the family's
        # sin() values and the norm's sum order are not bit-identical across libms)
        assert abs(tr.final_offdiag / float(row["final_offdiag"]) - 1) < 5e-3
        assert abs(tr.rotations - row["rotations"]) <= 1


def test_joint_svd_smoke_n64():
    row = next(r for r in GOLD["joint_svd"] if r["n"] == 64)
    _, _, _, tr = O.LieSvdJoint.joint_svd_with_params(joint_svd_family(64), O.JointDiagonalizationParams.for_n(64))
    assert rust_e3(tr.initial_offdiag) == row["initial_offdiag"]
    assert (tr.sweeps, tr.rotations) == (row["sweeps"], row["rotations"])
    assert abs(tr.final_offdiag / float(row["final_offdiag"]) - 1) < 1e-3


NAMED = {"kahan": lambda n: P.kahan_matrix(n, 1.2), "pei": lambda n: P.pei_matrix(n, 0.01),
         "vandermonde": P.vandermonde_matrix, "hilbert": P.hilbert_matrix}


def rust_e1(x: float) -> str:
    m, e = f"{x:.1e}".split("e")
    return f"{m}e{int(e)}"


@pytest.mark.parametrize("row", GOLD["compare_named"], ids=lambda r: f"{r['matrix']}{r['n']}")
def test_named_matrices_on_a_host_without_fma(row):
    # the compare harness (compare/src/main.rs:36-57, matrices of src/lie_svd_benchmarks.rs) ran
    # where matrixmultiply has no FMA kernel: the oracle's multiply-then-add products reproduce it
    O.set_dot_fma(False)
    try:
        a = NAMED[row["matrix"]](row["n"])
        u, s, vt = O.LieSvdSmall.solve(a)
        m = O.metrics.compute(a, u, s, vt, None)
    finally:
        O.set_dot_fma(True)
    assert (rust_e1(m.orth_u), rust_e1(m.rel_recon)) == (row["orth_u"], row["rel_recon"])


def test_pei_closed_form_error_on_a_host_without_fma():
    # compare/src/main.rs:173-186: max relative error of LieSvdSmall's sigma against the
    # Pei closed form (n = 64, alpha = 0.01), printed as 1.0e-12
    row = GOLD["compare_pei_closed_form"]
    O.set_dot_fma(False)
    try:
        _, s, _ = O.LieSvdSmall.solve(P.pei_matrix(row["n"], row["alpha"]))
    finally:
        O.set_dot_fma(True)
    want = np.sort(P.pei_matrix_singular_values(row["n"], row["alpha"]))[::-1]
    got = np.sort(s)[::-1]
    assert rust_e1(float(np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)))) == row["max_rel"]
