"""GPU parity of the mixed-precision batched SVD (TF32/BF16 tensor-core bulk,
FP64 refinement and Jacobi cleanup) against the oracle and the imposed
spectra, at the FP64 path's bars:
* singular values, normwise: max|s - s_ref| / s_ref[0] <= 1e-13
* ||U^T U - I||_F, ||V^T V - I||_F <= 4e-13, relative reconstruction <= 1e-13.
"""
import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import svd_batched, unpack
from lie_cliffalg_analog_svd_b200 import _lib as L
from lie_cliffalg_analog_svd_b200 import profiles as P

pytestmark = pytest.mark.gpu


def sigma_err(s, ref):
    s, ref = np.sort(s)[::-1], np.sort(ref)[::-1]
    return np.max(np.abs(s - ref)) / max(ref[0], 1e-300)


@pytest.mark.parametrize("prec", ["tf32", "bf16"])
def test_mixed_batched_accuracy(prec):
    ns, a, sig = P.uneven_batch_workload(2000, seed=21)
    u, s, vt, dg, st = svd_batched(ns, a, precision=prec, want_diag=True)
    assert st == L.OK
    assert np.all(dg["orth_u"] < 4e-13) and np.all(dg["orth_v"] < 4e-13)
    assert np.all(dg["rel_recon"] < 1e-13)
    us, ss, vts, as_ = unpack(ns, u), unpack(ns, s, False), unpack(ns, vt), unpack(ns, a)
    sr = unpack(ns, sig, False)
    for t in range(len(ns)):
        assert sigma_err(ss[t], sr[t]) < 1e-13, (t, ns[t])
    rng = np.random.default_rng(1)
    for t in rng.choice(len(ns), 60, replace=False):
        n = int(ns[t])
        so = O.LieSvdMicro.solve(as_[t])[1] if n <= 4 else O.LieSvdSmall.solve(as_[t])[1]
        assert sigma_err(ss[t], so) < 1e-13
        assert np.all(np.diff(ss[t]) <= 0)
        assert np.linalg.norm((us[t] * ss[t]) @ vts[t] - as_[t]) / np.linalg.norm(as_[t]) < 1e-13


@pytest.mark.parametrize("prec", ["tf32", "bf16"])
def test_mixed_matches_fp64_singular_vectors(prec):
    ns = np.full(200, 40, dtype=np.int32)
    rng = np.random.default_rng(2)
    a = rng.standard_normal(int((ns.astype(np.int64) ** 2).sum()))
    u1, s1, v1, _, _ = svd_batched(ns, a, precision="fp64")
    u2, s2, v2, _, _ = svd_batched(ns, a, precision=prec)
    for x, y, sx in zip(unpack(ns, v1), unpack(ns, v2), unpack(ns, s1, False)):
        assert np.all(np.abs(np.abs(np.sum(x * y, axis=1)) - 1) < 1e-9)
    assert np.max(np.abs(s1 - s2)) < 1e-12


@pytest.mark.parametrize("prec", ["tf32", "bf16"])
def test_mixed_edge_cases(prec):
    ns = np.array([1, 3, 5, 17, 64, 64, 40], dtype=np.int32)
    rng = np.random.default_rng(4)
    mats = [rng.standard_normal((n, n)) for n in ns]
    mats[4][:] = 0.0                                     # zero matrix
    x = rng.standard_normal((64, 2))
    mats[5] = x @ rng.standard_normal((2, 64))           # rank 2
    u0, v0 = P.random_orthogonal(40, rng), P.random_orthogonal(40, rng)
    mats[6] = (u0 * np.repeat([2.0, 1.0], 20)) @ v0.T    # two 20-fold clusters
    a = np.concatenate([m.ravel() for m in mats])
    u, s, vt, dg, st = svd_batched(ns, a, precision=prec, want_diag=True)
    assert st == L.OK
    for m, ut, st_, vtt in zip(mats, unpack(ns, u), unpack(ns, s, False), unpack(ns, vt)):
        ref = np.linalg.svd(m, compute_uv=False)
        if ref[0] > 0:
            assert sigma_err(st_, ref) < 1e-13
        else:
            assert np.all(st_ == 0)
        k = len(st_)
        assert np.linalg.norm(ut.T @ ut - np.eye(k)) < 1e-12
        assert np.linalg.norm(vtt @ vtt.T - np.eye(k)) < 1e-12
        assert np.linalg.norm((ut * st_) @ vtt - m) <= 1e-13 * max(np.linalg.norm(m), 1e-300) + 1e-300
