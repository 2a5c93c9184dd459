"""GPU Phase-JADE (LieSvdJoint::diagonalize_symmetric_with_params,
src/lie_svd_joint.rs:71-158) against the reference's own tests
(src/lie_svd_joint.rs:547-596) and the oracle on identical families.

Bars: final off-diagonal < initial * 1e-8 on exactly jointly diagonalisable
families (the reference's test); ||V^T V - I||_F < 1e-10; V^T M_k V equal to
diag(d_k) within 1e-9; sorted diagonals equal to the oracle's within 1e-9
(relative to the family norm); on perturbed families the final off-diagonal
within 10x of the oracle's (both stop at the same rule, after a different
pair order)."""
import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import JointDiagonalizationParams, LieSvdJoint
from lie_cliffalg_analog_svd_b200 import profiles as P

pytestmark = pytest.mark.gpu


def _family(n, k, seed):
    rng = np.random.default_rng(seed)
    q = np.linalg.qr(rng.uniform(-0.5, 0.5, (n, n)))[0]
    return [q @ np.diag(1.0 + f * 0.3 + np.arange(n) * 0.17) @ q.T for f in range(k)]


@pytest.mark.parametrize("n,k,seed", [(12, 5, 130), (10, 2, 131), (14, 9, 132)])
def test_ref_jade_family(n, k, seed):  # src/lie_svd_joint.rs:547-585
    mats = _family(n, k, seed)
    params = JointDiagonalizationParams.for_n(n)
    params.max_sweeps = 40
    v, diags, tr = LieSvdJoint.diagonalize_symmetric_with_params(mats, params)
    assert tr.final_offdiag < tr.initial_offdiag * 1e-8
    assert tr.rotations > 0 and len(diags) == k
    assert np.linalg.norm(v.T @ v - np.eye(n)) < 1e-10
    for m, d in zip(mats, diags):
        assert np.allclose(v.T @ m @ v, np.diag(d), atol=1e-9)
    op = O.JointDiagonalizationParams.for_n(n)
    op.max_sweeps = 40
    vo, do, tro = O.LieSvdJoint.diagonalize_symmetric_with_params(mats, op)
    assert abs(tr.initial_offdiag - tro.initial_offdiag) <= 1e-12 * tro.initial_offdiag
    for d, e in zip(diags, do):
        assert np.max(np.abs(np.sort(d) - np.sort(e))) < 1e-9


def test_ref_already_diagonal_family():  # :587-596
    mats = [np.diag(1.0 + np.arange(8) + k) for k in range(4)]
    _, _, tr = LieSvdJoint.diagonalize_symmetric(mats)
    assert tr.final_offdiag <= 1e-14 and tr.rotations == 0


@pytest.mark.parametrize("eps", [0.0, 1e-8, 1e-4])
@pytest.mark.parametrize("n", [24, 40])
def test_jade_families_vs_oracle(eps, n):
    fam = P.jade_family_workload(2, 16, n, eps, seed=7 + n)
    v, d, tr = LieSvdJoint.diagonalize_families(fam)
    for f in range(2):
        vo, do, tro = O.LieSvdJoint.diagonalize_symmetric([fam[f, k] for k in range(16)])
        assert np.linalg.norm(v[f].T @ v[f] - np.eye(n)) < 1e-10
        assert abs(tr[f].initial_offdiag - tro.initial_offdiag) <= 1e-12 * tro.initial_offdiag
        scale = np.sqrt(np.sum(fam[f] ** 2))
        assert tr[f].final_offdiag <= max(10 * tro.final_offdiag, 1e-12 * scale)
        assert abs(tr[f].sweeps - tro.sweeps) <= 3
        if eps == 0.0:
            for k in range(16):
                assert np.max(np.abs(np.sort(d[f, k]) - np.sort(np.asarray(do[k])))) < 1e-9 * scale
        # V^T M V diagonal up to the remaining off-diagonal mass
        off = sum(np.sum((v[f].T @ fam[f, k] @ v[f] - np.diag(d[f, k])) ** 2) for k in range(16))
        assert np.sqrt(off) <= 1e-9 * scale + 2 * tr[f].final_offdiag


def test_jade_trivial_sizes():
    v, d, tr = LieSvdJoint.diagonalize_families(np.full((3, 2, 1, 1), 2.5))
    assert np.all(v == 1.0) and np.all(d == 2.5) and all(t.sweeps == 0 for t in tr)
    mats = _family(3, 2, 5)
    v, diags, tr = LieSvdJoint.diagonalize_symmetric(mats)
    assert np.linalg.norm(v.T @ v - np.eye(3)) < 1e-12


def test_jade_cfg4_size_vs_oracle():
    # the benchmark's family shape (K = 64 symmetric 256 x 256 matrices,
    # A_k = Q diag(d_k) Q^T + eps E_k) at all three eps, one family each,
    # against the oracle: final off-diagonal, sorted diagonals, sweeps (within
    # one) and rejected rotations
    import concurrent.futures as cf
    n, K = 256, 64
    fams = {eps: P.jade_family_workload(1, K, n, eps, seed=4000 + i)
            for i, eps in enumerate((0.0, 1e-8, 1e-4))}

    def run_oracle(eps):
        return eps, O.LieSvdJoint.diagonalize_symmetric([fams[eps][0, k] for k in range(K)])

    with cf.ThreadPoolExecutor(3) as ex:
        ores = dict(ex.map(run_oracle, fams))
    for eps, fam in fams.items():
        v, d, tr = LieSvdJoint.diagonalize_families(fam)
        vo, do, tro = ores[eps]
        scale = np.sqrt(np.sum(fam[0] ** 2))
        assert np.linalg.norm(v[0].T @ v[0] - np.eye(n)) < 1e-10
        assert abs(tr[0].initial_offdiag - tro.initial_offdiag) <= 1e-12 * tro.initial_offdiag
        assert tr[0].final_offdiag <= max(10 * tro.final_offdiag, 1e-12 * scale), (eps, tr[0], tro)
        assert abs(tr[0].sweeps - tro.sweeps) <= 1, (eps, tr[0].sweeps, tro.sweeps)
        assert abs(tr[0].rejected_rotations - tro.rejected_rotations) <= max(2, tro.rejected_rotations // 10), \
            (eps, tr[0].rejected_rotations, tro.rejected_rotations)
        # the joint eigenvalues: equal to the oracle's up to the order of V's columns,
        # within the off-diagonal mass both leave behind
        tol = 1e-9 * scale + 2 * max(tr[0].final_offdiag, tro.final_offdiag)
        for k in range(K):
            assert np.max(np.abs(np.sort(d[0, k]) - np.sort(np.asarray(do[k])))) <= tol, (eps, k)
