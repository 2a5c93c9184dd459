"""Stream-keeping batched SVD and its rotor-replay adjoint.

Forward: sigma equal to the oracle's LieSvdSmall::solve_rectangular
(src/lie_svd_small.rs:340-360) within 1e-12 relative to sigma_1; V rebuilt
from the recorded stream (rounds in order, then the permutation) equal to the
forward's V within 1e-12; U S V^T = A within 4e-13 relative.

Adjoint:
* against the analytic FP64 thin-SVD adjoint restated in numpy on the
  forward's own U, V (F_ij = 1/(s_j^2 - s_i^2), polar term 1/(s_i + s_j)):
  relative Frobenius error <= 1e-9 for singular-value gaps >= 1e-3;
* against FP64 central finite differences (h = 1e-6) of
  L(A) = <Ubar, U> + <Sbar, S> + <Vbar, V> + <Qbar, U V^T> along random
  unit-Frobenius directions D, singular vectors sign-aligned to the
  unperturbed ones: |<Abar, D> - FD| <= 1e-5 ||Abar||_F for gaps >= 1e-2 (the
  FD noise floor is the solver's rounding in V, ~eps sigma_1 / gap, over h);
* with a 1e-6 gap: the polar cotangent still matches finite differences (the
  polar factor is smooth on the scale of sigma_min, sigma is not: its
  curvature there is ~1/gap), sigma + polar cotangents match the analytic
  formula, and gap_tol keeps the U cotangent adjoint finite.
"""
import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import LsvdError, svd_batched_stream, svd_vjp
from lie_cliffalg_analog_svd_b200 import profiles as P

pytestmark = pytest.mark.gpu


def _replay_v(rot, count, perm, n):
    v = np.eye(n)
    for e in rot[:count]:
        i, j, th = int(e["i"]), int(e["j"]), float(e["theta"])
        c, s = np.cos(th), np.sin(th)
        vi, vj = v[:, i].copy(), v[:, j].copy()
        v[:, i] = c * vi - s * vj
        v[:, j] = s * vi + c * vj
    return v[:, perm]


def _numpy_adjoint(u, s, v, ub, sb, vb, qb, gap_tol=0.0):
    n = s.size
    den = s[None, :] ** 2 - s[:, None] ** 2
    close = np.abs(s[None, :] - s[:, None]) <= gap_tol * s.max()
    with np.errstate(divide="ignore"):
        f = np.where((den == 0) | close, 0.0, 1.0 / np.where(den == 0, 1.0, den))
    np.fill_diagonal(f, 0.0)
    g = u.T @ ub
    h = v.T @ vb
    mm = u.T @ qb @ v
    core = (f * (g - g.T)) * s[None, :] + s[:, None] * (f * (h - h.T)) \
        + (mm - mm.T) / (s[:, None] + s[None, :]) + np.diag(sb)
    proj = (ub + qb @ v) - u @ (u.T @ (ub + qb @ v))
    return u @ core @ v.T + (proj / s[None, :]) @ v.T


def _loss(u, s, v, ub, sb, vb, qb):
    return np.sum(ub * u) + np.sum(sb * s) + np.sum(vb * v) + np.sum(qb * (u @ v.T))


def _aligned(fwd, t, v0):
    u = fwd.u[t]
    v = fwd.vt[t].T
    sg = np.sign(np.sum(v * v0, axis=0))
    sg[sg == 0] = 1.0
    return u * sg, fwd.s[t], v * sg


@pytest.mark.parametrize("m,n", [(128, 64), (40, 17), (24, 24), (9, 2)])
def test_stream_forward(m, n):
    a, sig = P.adjoint_workload(4, m, n, seed=m + n, gap=1e-3 if n > 2 else 0.0)
    fwd = svd_batched_stream(a, want_uv=True, want_diag=True)
    assert fwd.status == 0
    for t in range(4):
        so = O.LieSvdSmall.solve_rectangular(a[t])[1]
        assert np.max(np.abs(fwd.s[t] - so)) <= 1e-12 * so[0]
        assert np.max(np.abs(fwd.s[t] - sig[t])) <= 1e-12 * sig[t][0]
        v = _replay_v(fwd.rotors[t], fwd.counts[t], fwd.perm[t], n)
        assert np.max(np.abs(v - fwd.vt[t].T)) <= 1e-12
        rec = (fwd.u[t] * fwd.s[t]) @ fwd.vt[t]
        assert np.linalg.norm(rec - a[t]) <= 4e-13 * np.linalg.norm(a[t])
    assert fwd.stream_bytes() > 0 and fwd.uv_bytes() == 4 * (m * n + n * n) * 8


@pytest.mark.parametrize("m,n", [(128, 64), (40, 17), (24, 24)])
@pytest.mark.parametrize("which", ["u", "s", "v", "q", "all"])
def test_vjp_vs_analytic(m, n, which):
    cnt = 3
    a, _ = P.adjoint_workload(cnt, m, n, seed=7 * m + n, small_gap_frac=0.0)
    fwd = svd_batched_stream(a, want_uv=True)
    rng = np.random.default_rng(m * n)
    ub = rng.standard_normal((cnt, m, n)) if which in ("u", "all") else np.zeros((cnt, m, n))
    sb = rng.standard_normal((cnt, n)) if which in ("s", "all") else np.zeros((cnt, n))
    vb = rng.standard_normal((cnt, n, n)) if which in ("v", "all") else np.zeros((cnt, n, n))
    qb = rng.standard_normal((cnt, m, n)) if which in ("q", "all") else np.zeros((cnt, m, n))
    ab = svd_vjp(fwd, ubar=ub, sbar=sb, vbar=vb, qbar=qb)
    for t in range(cnt):
        ref = _numpy_adjoint(fwd.u[t], fwd.s[t], fwd.vt[t].T, ub[t], sb[t], vb[t], qb[t])
        assert np.linalg.norm(ab[t] - ref) <= 1e-9 * np.linalg.norm(ref)


def test_vjp_stored_v_matches_replay():
    a, _ = P.adjoint_workload(3, 128, 64, seed=21)
    fwd = svd_batched_stream(a, want_uv=True)
    rng = np.random.default_rng(3)
    ub = rng.standard_normal(a.shape); qb = rng.standard_normal(a.shape)
    vb = rng.standard_normal((3, 64, 64))
    ab_r = svd_vjp(fwd, ubar=ub, vbar=vb, qbar=qb)
    ab_s = svd_vjp(fwd, ubar=ub, vbar=vb, qbar=qb, stored_vt=fwd.vt)
    assert np.linalg.norm(ab_r - ab_s) <= 1e-11 * np.linalg.norm(ab_s)


def test_vjp_null_cotangents_match_zeros():
    a, _ = P.adjoint_workload(2, 30, 10, seed=3)
    fwd = svd_batched_stream(a)
    rng = np.random.default_rng(1)
    sb = rng.standard_normal((2, 10))
    z = np.zeros((2, 30, 10))
    ab1 = svd_vjp(fwd, sbar=sb)
    ab2 = svd_vjp(fwd, ubar=z, sbar=sb, vbar=np.zeros((2, 10, 10)), qbar=z)
    assert np.max(np.abs(ab1 - ab2)) <= 1e-13 * np.max(np.abs(ab1))


def _fd_direction(a, d, ub, sb, vb, qb, h=1e-6):
    """Central difference of the loss along d for each matrix of the batch."""
    cnt = a.shape[0]
    base = svd_batched_stream(a, want_uv=True)
    plus = svd_batched_stream(a + h * d, want_uv=True)
    minus = svd_batched_stream(a - h * d, want_uv=True)
    out = np.empty(cnt)
    for t in range(cnt):
        v0 = base.vt[t].T
        lp = _loss(*_aligned(plus, t, v0), ub[t], sb[t], vb[t], qb[t])
        lm = _loss(*_aligned(minus, t, v0), ub[t], sb[t], vb[t], qb[t])
        out[t] = (lp - lm) / (2 * h)
    return out, base


@pytest.mark.parametrize("m,n", [(128, 64), (20, 8)])
def test_vjp_vs_finite_differences(m, n):
    cnt = 4
    a, _ = P.adjoint_workload(cnt, m, n, seed=11 + m, gap=1e-2, small_gap_frac=0.0)
    rng = np.random.default_rng(5 + n)
    ub = rng.standard_normal((cnt, m, n)); sb = rng.standard_normal((cnt, n))
    vb = rng.standard_normal((cnt, n, n)); qb = rng.standard_normal((cnt, m, n))
    for rep in range(2):
        d = rng.standard_normal((cnt, m, n))
        d /= np.linalg.norm(d, axis=(1, 2), keepdims=True)
        fd, base = _fd_direction(a, d, ub, sb, vb, qb)
        ab = svd_vjp(base, ubar=ub, sbar=sb, vbar=vb, qbar=qb)
        an = np.einsum("tij,tij->t", ab, d)
        assert np.all(np.abs(an - fd) <= 1e-5 * np.linalg.norm(ab, axis=(1, 2)))


def test_vjp_small_gap():
    m, n = 64, 16
    a, sig = P.adjoint_workload(3, m, n, seed=99, gap=1e-2, small_gap=1e-6, small_gap_frac=1.0)
    gaps = np.min(-np.diff(sig, axis=1), axis=1)
    assert np.all(gaps < 1e-5)
    rng = np.random.default_rng(2)
    zu = np.zeros((3, m, n)); zv = np.zeros((3, n, n)); zs = np.zeros((3, n))
    sb = rng.standard_normal((3, n)); qb = rng.standard_normal((3, m, n))
    # the polar factor is smooth on the scale of sigma_min, not of the gap:
    # finite differences still apply to a polar-only loss
    d = rng.standard_normal((3, m, n))
    d /= np.linalg.norm(d, axis=(1, 2), keepdims=True)
    fd, base = _fd_direction(a, d, zu, zs, zv, qb)
    ab = svd_vjp(base, qbar=qb)
    an = np.einsum("tij,tij->t", ab, d)
    assert np.all(np.abs(an - fd) <= 1e-5 * np.linalg.norm(ab, axis=(1, 2)))
    # sigma + polar cotangents against the analytic formula (finite for a close pair)
    ab = svd_vjp(base, sbar=sb, qbar=qb)
    for t in range(3):
        ref = _numpy_adjoint(base.u[t], base.s[t], base.vt[t].T, zu[t], sb[t], zv[t], qb[t])
        assert np.linalg.norm(ab[t] - ref) <= 1e-9 * np.linalg.norm(ref)
    # U cotangent: the close pair's 1/(s_j^2 - s_i^2) term is dropped by gap_tol
    ub = rng.standard_normal((3, m, n))
    ab_t = svd_vjp(base, ubar=ub, gap_tol=1e-4)
    assert np.all(np.isfinite(ab_t))
    for t in range(3):
        ref = _numpy_adjoint(base.u[t], base.s[t], base.vt[t].T, ub[t], zs[t], zv[t], zu[t], gap_tol=1e-4)
        assert np.linalg.norm(ab_t[t] - ref) <= 1e-9 * np.linalg.norm(ref)


def test_vjp_device_pointers():
    import torch
    a, _ = P.adjoint_workload(8, 128, 64, seed=4)
    rng = np.random.default_rng(8)
    ub = rng.standard_normal(a.shape); qb = rng.standard_normal(a.shape)
    fwd_h = svd_batched_stream(a)
    ab_h = svd_vjp(fwd_h, ubar=ub, qbar=qb)
    fwd_d = svd_batched_stream(torch.from_numpy(a).cuda())
    ab_d = svd_vjp(fwd_d, ubar=torch.from_numpy(ub).cuda(), qbar=torch.from_numpy(qb).cuda())
    assert np.max(np.abs(ab_d.cpu().numpy() - ab_h)) <= 1e-12 * np.max(np.abs(ab_h))
    assert np.array_equal(fwd_d.counts.cpu().numpy(), fwd_h.counts)


def test_stream_errors():
    a, _ = P.adjoint_workload(2, 32, 16, seed=1)
    with pytest.raises(LsvdError):
        svd_batched_stream(a, rotor_cap=10)          # stream longer than the cap
    with pytest.raises(LsvdError):
        svd_batched_stream(np.ones((1, 4, 8)))       # m < n
    fwd = svd_batched_stream(a)
    fwd.s[0, -1] = 0.0
    with pytest.raises(LsvdError):
        svd_vjp(fwd, sbar=np.ones((2, 16)))          # sigma <= 0
