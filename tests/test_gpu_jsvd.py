"""GPU two-sided joint SVD (LieSvdJoint::joint_svd_with_params,
src/lie_svd_joint.rs:170-261) against the reference's own tests
(src/lie_svd_joint.rs:598-664) and the oracle on identical families.

Bars: the reference's (final off-diagonal < initial * 1e-8 on exactly
jointly diagonalisable square families; final <= initial on rectangular
ones; ||U^T U - I||, ||V V^T - I|| < 1e-10); U^T M_k V equal to
diag(+-sigma_k) within 1e-9 on exact families; sorted |diagonals| equal to
the oracle's within 1e-9 relative to the family norm; on noisy families the
final off-diagonal within 10x of the oracle's (both stop at the same rule,
after a different pair order)."""
import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import JointDiagonalizationParams, LieSvdJoint, LsvdError
from lie_cliffalg_analog_svd_b200 import profiles as P

pytestmark = pytest.mark.gpu


def _square_family(n, k, seed):
    rng = np.random.default_rng(seed)
    u0 = P.random_orthogonal(n, rng)
    v0 = P.random_orthogonal(n, rng)
    return [u0 @ np.diag(1.0 + f * 0.2 + np.arange(n) * 0.11) @ v0.T for f in range(k)]


def _rect_family(rows, cols, k, seed, noise=0.0):
    rng = np.random.default_rng(seed)
    u0 = P.random_orthogonal(rows, rng)
    v0 = P.random_orthogonal(cols, rng)
    out = []
    kk = min(rows, cols)
    for f in range(k):
        s = np.zeros((rows, cols))
        s[np.arange(kk), np.arange(kk)] = 1.0 + f * 0.2 + np.arange(kk) * 0.07
        out.append(u0 @ s @ v0.T + noise * rng.standard_normal((rows, cols)))
    return out


@pytest.mark.parametrize("n,k,seed", [(10, 4, 150), (16, 3, 152), (23, 5, 153), (40, 6, 154)])
def test_ref_joint_svd_square(n, k, seed):  # :598-626
    mats = _square_family(n, k, seed)
    params = JointDiagonalizationParams.for_n(n)
    params.max_sweeps = 36
    u, sig, vt, tr = LieSvdJoint.joint_svd_with_params(mats, params)
    assert tr.final_offdiag < tr.initial_offdiag * 1e-8 and tr.rotations > 0
    assert len(sig) == k
    assert np.linalg.norm(u.T @ u - np.eye(n)) < 1e-10
    assert np.linalg.norm(vt @ vt.T - np.eye(n)) < 1e-10
    for m, s in zip(mats, sig):
        d = u.T @ m @ vt.T
        assert np.allclose(np.abs(d), np.diag(s), atol=1e-9)
    op = O.JointDiagonalizationParams.for_n(n)
    op.max_sweeps = 36
    uo, so, vto, tro = O.LieSvdJoint.joint_svd_with_params(mats, op)
    scale = max(np.linalg.norm(m) for m in mats)
    for s, s2 in zip(sig, so):
        assert np.max(np.abs(np.sort(s) - np.sort(s2))) <= 1e-9 * scale


@pytest.mark.parametrize("rows,cols,seed", [(9, 13, 151), (13, 9, 155), (20, 33, 156), (37, 17, 157)])
def test_ref_joint_svd_rectangular(rows, cols, seed):  # :628-664
    mats = _rect_family(rows, cols, 3, seed)
    params = JointDiagonalizationParams.for_n(min(rows, cols))
    params.max_sweeps = 32
    u, sig, vt, tr = LieSvdJoint.joint_svd_with_params(mats, params)
    assert tr.final_offdiag <= tr.initial_offdiag
    assert len(sig) == 3 and len(sig[0]) == min(rows, cols)
    assert np.linalg.norm(u.T @ u - np.eye(rows)) < 1e-10
    assert np.linalg.norm(vt @ vt.T - np.eye(cols)) < 1e-10
    op = O.JointDiagonalizationParams.for_n(min(rows, cols))
    op.max_sweeps = 32
    _, _, _, tro = O.LieSvdJoint.joint_svd_with_params(mats, op)
    assert tr.final_offdiag <= 10 * tro.final_offdiag + 1e-12 * tro.initial_offdiag


@pytest.mark.parametrize("noise", [1e-8, 1e-4])
def test_joint_svd_noisy_vs_oracle(noise):
    mats = _rect_family(24, 24, 5, 160, noise)
    u, sig, vt, tr = LieSvdJoint.joint_svd(mats)
    _, so, _, tro = O.LieSvdJoint.joint_svd(mats)
    assert tr.final_offdiag <= 10 * tro.final_offdiag + 1e-12 * tro.initial_offdiag
    assert abs(tr.initial_offdiag - tro.initial_offdiag) <= 1e-12 * tro.initial_offdiag
    assert np.linalg.norm(u.T @ u - np.eye(24)) < 1e-10
    # U^T M V reproduces the returned |diagonals|
    for m, s in zip(mats, sig):
        assert np.allclose(np.abs(np.diag(u.T @ m @ vt.T)), s, atol=1e-9)


def test_joint_svd_families_batch_and_edges():
    fams = np.stack([np.stack(_square_family(12, 3, 170 + f)) for f in range(5)])
    u, s, vt, tr = LieSvdJoint.joint_svd_families(fams)
    for f in range(5):
        u1, s1, vt1, tr1 = LieSvdJoint.joint_svd(list(fams[f]))
        assert np.max(np.abs(u[f] - u1)) <= 1e-13 and tr[f].sweeps == tr1.sweeps
    # 1 x n: nothing to rotate (kk = 1), identity bases, |m_00|
    m = np.array([[[-2.0, 1.0, 3.0]]])
    u, sig, vt, tr = LieSvdJoint.joint_svd(list(m))
    assert np.array_equal(u, np.eye(1)) and np.array_equal(vt, np.eye(3))
    assert sig[0][0] == 2.0 and tr.sweeps == 0 and tr.rotations == 0
    with pytest.raises(LsvdError):
        LieSvdJoint.joint_svd([np.zeros((0, 3))])
