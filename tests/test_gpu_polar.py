"""Large Newton-Schulz polar factor (newton_schulz_polar,
src/lie_svd_small.rs:158-183, on large m x n inputs) and its tcgen05 product
kernel.

Bars:
* FP64 GEMM (mma.sync m8n8k4): against numpy's FP64 product, elementwise
  |C - C_ref| <= 4 K eps (|A||B|) (both sum K products in FP64).
* tcgen05 GEMM: against the FP64 product of the same TF32/BF16-rounded
  operands, |C - C_ref| <= K 2^-22 (|A||B|^T) elementwise (FP32 accumulation),
  relative Frobenius error <= 4 sqrt(K) 2^-24.
* FP64 polar: ||Q^T Q - I||_F <= 1e-12 sqrt(n); distance to the exact polar
  factor Q1 Q2^T of A = Q1 diag(s) Q2^T within 2e-14 kappa n (the factor's
  condition grows with kappa); on 64 x 64 inputs the iterate equals the
  oracle's newton_schulz_polar to 1e-12 with the same iteration count +-1.
* Mixed TF32/BF16 + FP64 refinement: ||Q^T Q - I||_F <= 1e-12 sqrt(n) always
  (the refinement restores orthogonality); the distance to A's polar factor
  is set by the low-precision phase, <= 2 u_lo sqrt(n) for kappa <= 1e3
  (u_lo = 2^-11 TF32, 2^-8 BF16).
"""
import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import LsvdError, polar
from lie_cliffalg_analog_svd_b200 import profiles as P
from lie_cliffalg_analog_svd_b200.api import gemm_f64, gemm_nt_lowp

pytestmark = pytest.mark.gpu

U_LO = {"tf32": 2.0 ** -11, "bf16": 2.0 ** -8}


def _round_tf32(x: np.ndarray) -> np.ndarray:
    """cvt.rna.tf32.f32: keep 10 mantissa bits, ties away from zero."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = (b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)
    return r.view(np.float32)


def _round_bf16(x: np.ndarray) -> np.ndarray:
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).to(torch.bfloat16).float().numpy()


@pytest.mark.parametrize("ta,tb", [(False, False), (True, False), (False, True), (True, True)])
@pytest.mark.parametrize("M,N,K", [(128, 128, 16), (1, 1, 1), (7, 9, 5), (130, 257, 33), (300, 200, 1000),
                                   (512, 384, 4096), (64, 1000, 3), (2560, 2312, 96),
                                   (32, 32, 300001), (5, 70, 65537), (130, 64, 100000),
                                   (64, 64, 50001), (3, 17, 9000), (16, 9, 4096)])
def test_gemm_f64(ta, tb, M, N, K):
    # the small shapes run on 128 x 64 tiles, (2560, 2312, 96) on 128 x 128 tiles;
    # the last six split K into slices (few output tiles, K >= 4096; odd K
    # leaves a remainder slice); A B^T with M, N <= 64 takes the CUDA-core
    # slices (T = 4, 2, 2, 1 for the 64, 32, 17 and 16 wide outputs)
    import torch
    rng = np.random.default_rng(M * 13 + N * 5 + K + 2 * ta + tb)
    a = rng.standard_normal((K, M) if ta else (M, K))
    b = rng.standard_normal((N, K) if tb else (K, N))
    c0 = rng.standard_normal((M, N))
    pad = lambda x: np.pad(x, ((0, 0), (0, (-x.shape[1]) % 2)))  # noqa: E731  (even row stride)
    ad = torch.from_numpy(pad(a)).cuda()[:, :a.shape[1]]
    bd = torch.from_numpy(pad(b)).cuda()[:, :b.shape[1]]
    cd = torch.from_numpy(c0.copy()).cuda()
    gemm_f64(ad, bd, ta, tb, alpha=1.5, beta=-0.5, c=cd)
    opa, opb = (a.T if ta else a), (b.T if tb else b)
    ref = 1.5 * (opa @ opb) - 0.5 * c0
    mag = 1.5 * (np.abs(opa) @ np.abs(opb)) + 0.5 * np.abs(c0)
    assert np.all(np.abs(cd.cpu().numpy() - ref) <= 4 * max(K, 1) * 2.2e-16 * mag + 1e-300)
    # beta = 0 must not read C (NaN in C stays out of the result)
    cn = torch.full((M, N), float("nan"), dtype=torch.float64, device="cuda")
    gemm_f64(ad, bd, ta, tb, c=cn)
    assert torch.isfinite(cn).all()


@pytest.mark.parametrize("prec", ["tf32", "bf16"])
@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 512), (1024, 1024, 1024), (512, 128, 4096),
                                   (128, 256, 64), (384, 768, 2048)])
def test_tc_gemm(prec, M, N, K):
    import torch
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    a = rng.standard_normal((M, K)).astype(np.float32)
    b = rng.standard_normal((N, K)).astype(np.float32)
    c = gemm_nt_lowp(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), prec).cpu().numpy()
    rnd = _round_tf32 if prec == "tf32" else _round_bf16
    ar, br = rnd(a).astype(np.float64), rnd(b).astype(np.float64)
    ref = ar @ br.T
    mag = np.abs(ar) @ np.abs(br).T
    assert np.all(np.abs(c - ref) <= K * 2.0 ** -22 * mag)
    assert np.linalg.norm(c - ref) <= 4 * np.sqrt(K) * 2.0 ** -24 * np.linalg.norm(ref)


def _exact(m, n, kappa, seed):
    q1, s, q2 = P.conditioned_factors(m, n, kappa, seed)
    return (q1 * s[None, :]) @ q2.T, q1 @ q2.T


def _orth(q):
    return np.linalg.norm(q.T @ q - np.eye(q.shape[1]))


@pytest.mark.parametrize("m,n", [(256, 256), (384, 128), (200, 136), (96, 96)])
@pytest.mark.parametrize("kappa", [1e2, 1e5, 1e8])
def test_polar_fp64(m, n, kappa):
    a, q_exact = _exact(m, n, kappa, seed=m + n + int(np.log10(kappa)))
    r = polar(a, "fp64")
    assert r.converged and r.iters_lowp == 0 and r.iters_fp64 > 0
    assert _orth(r.q) <= 1e-12 * np.sqrt(n)
    assert abs(r.orth - _orth(r.q)) <= 1e-12 * np.sqrt(n)
    assert np.linalg.norm(r.q - q_exact) <= 2e-14 * kappa * n


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_polar_matches_oracle_64(seed):
    a = P.generate(64, "uniform_random", seed)[0]
    qo, ok, it = O.ns_polar(a)
    r = polar(a, "fp64")
    assert ok and r.converged
    assert abs(r.iters_fp64 - it) <= 1
    assert np.max(np.abs(r.q - qo)) <= 1e-12


@pytest.mark.parametrize("prec", ["tf32", "bf16"])
@pytest.mark.parametrize("m,n", [(256, 256), (512, 256), (1024, 1024)])
@pytest.mark.parametrize("kappa", [1e2, 1e5, 1e8])
def test_polar_mixed(prec, m, n, kappa):
    a, q_exact = _exact(m, n, kappa, seed=m + 2 * n + int(np.log10(kappa)))
    r = polar(a, prec)
    assert r.converged and r.iters_lowp > 0 and r.iters_fp64 > 0
    assert _orth(r.q) <= 1e-12 * np.sqrt(n)
    if kappa <= 1e3:
        assert np.linalg.norm(r.q - q_exact) <= 2 * U_LO[prec] * np.sqrt(n)


def test_polar_device_pointers():
    import torch
    a, q_exact = _exact(512, 256, 1e3, seed=9)
    r = polar(torch.from_numpy(a).cuda(), "tf32")
    q = r.q.cpu().numpy()
    assert r.converged and _orth(q) <= 1e-12 * 16
    assert np.linalg.norm(q - q_exact) <= 2 * U_LO["tf32"] * 16
    r64 = polar(torch.from_numpy(a).cuda(), "fp64")
    assert np.linalg.norm(r64.q.cpu().numpy() - q_exact) <= 2e-14 * 1e3 * 256


def test_polar_rejects():
    with pytest.raises(LsvdError):
        polar(np.ones((4, 8)), "fp64")        # m < n
    with pytest.raises(LsvdError):
        polar(np.eye(200), "tf32")            # not a multiple of 128
