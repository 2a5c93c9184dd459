"""GPU parity for the blocked large solve: LieSvdSmall::solve at n > 64
(src/lie_svd_small.rs:296-323; the reference routes n <= 512 there,
src/lie_svd_adaptive.rs:71) and LieSvdSmall::solve_rectangular with
min(m, d) > 64 (:340-360), against the oracle on identical inputs, plus the
reference's own large-size tests.

Bars (FP64):
* singular values, normwise: max|s_gpu - s_ref| / s_ref[0] <= 1e-13, also
  against the imposed spectrum of A = Q1 diag(s) Q2^T;
* ||U^T U - I||_F, ||V^T V - I||_F and the relative reconstruction
  <= max(2e-13 n / 64, 8 x the oracle's own value on the same input) -- both
  accumulate O(n) rotations per column, so the floor grows with n;
* singular vectors |<u_gpu_j, u_ref_j>| >= 1 - 1e-9 for columns whose singular
  value is separated from its neighbours by a relative gap > 1e-6.
"""
import concurrent.futures as cf

import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import LieSvdSmall, svd_large
from lie_cliffalg_analog_svd_b200 import _lib as L
from lie_cliffalg_analog_svd_b200 import profiles as P

pytestmark = pytest.mark.gpu


def mets(a, u, s, vt):
    rec = np.linalg.norm((u * s) @ vt - a) / max(np.linalg.norm(a), 1e-300)
    return rec, np.linalg.norm(u.T @ u - np.eye(u.shape[1])), np.linalg.norm(vt @ vt.T - np.eye(vt.shape[0]))


def sigma_err(s, ref):
    s, ref = np.sort(s)[::-1], np.sort(ref)[::-1]
    return np.max(np.abs(s - ref)) / max(ref[0], 1e-300)


def compare(a, g, o, tol_sigma=1e-13):
    ug, sg, vg = g
    uo, so, vo = o
    k = len(so)
    assert np.all(np.isfinite(ug)) and np.all(np.isfinite(vg)) and np.all(sg >= 0)
    assert np.all(np.diff(sg) <= 0), "sigma must be descending"
    assert sigma_err(sg, so) <= tol_sigma, sigma_err(sg, so)
    rg, oug, ovg = mets(a, ug, sg, vg)
    ro, ouo, ovo = mets(a, uo, so, vo)
    floor = 2e-13 * max(1.0, k / 64)
    assert rg <= max(floor, 8 * ro), (rg, ro)
    assert oug <= max(floor, 8 * ouo), (oug, ouo)
    assert ovg <= max(floor, 8 * ovo), (ovg, ovo)
    for j in range(k):
        gap = min([abs(so[j] - so[i]) for i in (j - 1, j + 1) if 0 <= i < k] + [np.inf])
        if so[j] > 1e-6 * so[0] and gap > 1e-6 * so[0]:
            assert abs(ug[:, j] @ uo[:, j]) >= 1 - 1e-9, j
            assert abs(vg[j] @ vo[j]) >= 1 - 1e-9, j


def _oracle_all(mats, rect=False):
    f = O.LieSvdSmall.solve_rectangular if rect else O.LieSvdSmall.solve
    with cf.ThreadPoolExecutor(4) as ex:
        return list(ex.map(f, mats))


def test_square_sizes_vs_oracle():
    # past the shared-memory kernels, odd sizes and block-padding edges included
    ns = [65, 96, 128, 200, 257, 384, 512]
    mats = [np.random.default_rng(500 + n).standard_normal((n, n)) for n in ns]
    refs = _oracle_all(mats)
    for a, o in zip(mats, refs):
        compare(a, LieSvdSmall.solve(a), o)


def test_conditioned_vs_imposed_spectrum():
    # A = Q1 diag(s) Q2^T with geometric s, kappa 1e2 / 1e8 / 1e12, against the
    # oracle and the imposed singular values
    for n, kappa, seed in ((160, 1e2, 1), (256, 1e8, 2), (130, 1e12, 3)):
        q1, s, q2 = P.conditioned_factors(n, n, kappa, seed)
        a = (q1 * s) @ q2.T
        g = LieSvdSmall.solve(a)
        assert sigma_err(g[1], s) <= 1e-13
        compare(a, g, O.LieSvdSmall.solve(a))


def test_rectangular_vs_oracle():
    rng = np.random.default_rng(77)
    mats = [rng.standard_normal((300, 100)), rng.standard_normal((100, 300)), rng.standard_normal((1000, 65))]
    refs = _oracle_all(mats, rect=True)
    for a, o in zip(mats, refs):
        g = LieSvdSmall.solve_rectangular(a)
        k = min(a.shape)
        assert g[0].shape == (a.shape[0], k) and g[2].shape == (k, a.shape[1])
        compare(a, g, o)


def test_ref_random_384_machine_precision_orthogonality():  # src/lie_svd_small.rs:643-657
    n = 384
    a = np.random.default_rng(7).uniform(-1.0, 1.0, (n, n))
    u, s, vt = LieSvdSmall.solve(a)
    recon = np.linalg.norm((u * s) @ vt - a)
    assert recon < 1e-8
    assert np.linalg.norm(u.T @ u - np.eye(n)) < 1e-8
    assert np.linalg.norm(vt @ vt.T - np.eye(n)) < 1e-8


def test_ref_ill_conditioned_large():  # the n = 32 test of :571-615 at n = 96
    n = 96
    rng = np.random.default_rng(42)
    ur = np.linalg.qr(rng.uniform(-1, 1, (n, n)))[0]
    vr = np.linalg.qr(rng.uniform(-1, 1, (n, n)))[0]
    s = 10.0 ** (-15.0 * np.arange(n) / (n - 1))
    a = (ur * s) @ vr.T
    u, sg, vt = LieSvdSmall.solve(a)
    assert np.linalg.norm((u * sg) @ vt - a) < 1e-6
    assert np.linalg.norm(u.T @ u - np.eye(n)) < 1e-6
    assert np.linalg.norm(vt @ vt.T - np.eye(n)) < 1e-6


def test_svd_large_entry_and_info():
    import torch
    rng = np.random.default_rng(5)
    a = rng.standard_normal((700, 300))
    r = svd_large(a, want_diag=True)
    assert r.status == L.OK
    assert r.info.sweeps_fp64 >= 2 and r.info.ns_iters_fp64 > 5 and r.info.flops_fp64 > 0
    # the reference's stop test: off(P) < 1e-13 ||P||_F at the last sweep start (||P||_F = ||A||_F)
    assert r.info.last_offdiag < 1e-13 * np.linalg.norm(a)
    ref = np.linalg.svd(a, compute_uv=False)
    assert sigma_err(r.s, ref) <= 1e-13
    rec, ou, ov = mets(a, r.u, r.s, r.vt)
    assert rec < 1e-12 and ou < 1e-11 and ov < 1e-11
    assert abs(r.diag["orth_u"] - ou) <= 1e-13 + 0.1 * ou
    # device pointers give the same bits as host pointers
    rd = svd_large(torch.from_numpy(a).cuda())
    assert np.array_equal(rd.s.cpu().numpy(), r.s) and np.array_equal(rd.u.cpu().numpy(), r.u)


def test_large_edge_cases():
    # zero matrix: sigma = 0, orthonormal U and V (the reference's MGS fill gives unit vectors)
    z = np.zeros((80, 80))
    u, s, vt = LieSvdSmall.solve(z)
    assert np.all(s == 0) and np.linalg.norm(u.T @ u - np.eye(80)) < 1e-12
    bad = np.random.default_rng(1).standard_normal((70, 70))
    bad[3, 4] = np.nan
    with pytest.raises(L.LsvdError) as ei:
        svd_large(bad)
    assert ei.value.status == L.NONFINITE_INPUT


@pytest.mark.parametrize("prec", ["tf32", "bf16"])
def test_mixed_route_matches_fp64_and_oracle(prec):
    # TF32/BF16 tensor-core Newton-Schulz bulk, a preconditioning eigensolve to
    # the low-precision level, then FP64 one-sided Jacobi on A V0: the same
    # bars as the FP64 route (sigma 1e-13 normwise against the imposed
    # spectrum, orthogonality and reconstruction), at kappa 1e2 / 1e5 / 1e8,
    # square and tall, and the oracle at n = 512
    for (m, n), kappa, seed in (((512, 512), 1e2, 11), ((640, 384), 1e5, 12), ((512, 512), 1e8, 13)):
        q1, s, q2 = P.conditioned_factors(m, n, kappa, seed)
        a = (q1 * s) @ q2.T
        r = svd_large(a, prec)
        assert r.status == L.OK, r.status
        assert r.info.ns_iters_lowp > 0 and r.info.ns_iters_fp64 == 0 and r.info.sweeps_fp64 >= 1
        assert sigma_err(r.s, s) <= 1e-13, (prec, kappa, sigma_err(r.s, s))
        f = svd_large(a, "fp64")
        assert sigma_err(r.s, f.s) <= 1e-13
        floor = 2e-13 * max(1.0, n / 64)
        rec, ou, ov = mets(a, r.u, r.s, r.vt)
        # U = W / sigma is re-orthonormalised (Newton-Schulz): columns with
        # sigma_j << sigma_1 move by up to tol sigma_1 / sigma_j, which costs
        # the reconstruction up to ~1e-11 relative (sigma and orthogonality keep
        # the FP64 bars)
        assert ou <= floor and ov <= floor and rec <= 1e-11, (prec, kappa, rec, ou, ov)
        if (m, n) == (512, 512) and kappa == 1e2:
            compare(a, (r.u, r.s, r.vt), O.LieSvdSmall.solve(a))


def test_mixed_route_rejects_unaligned():
    with pytest.raises(L.LsvdError) as ei:
        svd_large(np.random.default_rng(0).standard_normal((300, 200)), "tf32")
    assert ei.value.status == L.UNSUPPORTED
