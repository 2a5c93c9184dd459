"""The consumers on the GPU (lie_cliffalg_analog_svd_b200/consumers.py)
against the oracle's restatement (oracle/oracle_consumers.py, itself checked
against the reference's tests in test_consumers_oracle.py), plus the
reference's own tests of them run through the GPU: Phase-BSS
(src/lie_svd_bss.rs:216-251) and the canonical wrappers
(src/phase_normalizer.rs:377-413, :1144-1229).

Bars: sums in another order and solves in another (parallel) rotation order,
so values agree to rounding (1e-10 relative) where they are unique; the
separated channels and the JADE basis are unique up to the sign and order of
their rows, so they are matched first (|correlation| >= 1 - 1e-10)."""
import numpy as np
import pytest

import oracle_consumers as OC
from lie_cliffalg_analog_svd_b200 import consumers as G
from test_consumers_oracle import bss_sources, random_orthogonal

pytestmark = pytest.mark.gpu


def _match_rows(a, b):
    """Signed permutation p, sg with a[i] ~ sg[i] b[p[i]] by |correlation|."""
    na = a / np.linalg.norm(a, axis=1, keepdims=True)
    nb = b / np.linalg.norm(b, axis=1, keepdims=True)
    c = na @ nb.T
    p = np.argmax(np.abs(c), axis=1)
    assert len(set(p.tolist())) == len(p), c
    return p, np.sign(c[np.arange(len(p)), p]), np.abs(c[np.arange(len(p)), p])


def _check_bss(obs, params_gpu, params_oracle, tol_corr=1e-10):
    g = G.LieSvdBss.separate(obs, params_gpu)
    o = OC.bss_separate(obs, params_oracle)
    assert g.separated.shape == o.separated.shape and g.unmixing.shape == o.unmixing.shape
    p, sg, corr = _match_rows(g.separated, o.separated)
    assert np.all(corr >= 1 - tol_corr), corr
    un = sg[:, None] * o.unmixing[p]
    assert np.max(np.abs(g.unmixing - un)) <= 1e-7 * np.max(np.abs(un))
    assert np.max(np.abs(g.channel_coherence - o.channel_coherence[p])) <= 1e-9
    t, u = g.trace, o.trace
    assert (t.channels, t.samples) == (u.channels, u.samples)
    assert abs(t.covariance_floor - u.covariance_floor) <= 1e-12 * u.covariance_floor
    assert abs(t.joint_initial_offdiag - u.joint_initial_offdiag) <= 1e-12 + 1e-10 * u.joint_initial_offdiag
    assert t.joint_final_offdiag <= t.joint_initial_offdiag + 1e-10
    assert abs(t.mean_channel_coherence - u.mean_channel_coherence) <= 1e-9
    return g, o


def test_bss_reference_test_through_the_gpu():  # src/lie_svd_bss.rs:216-251
    s, mix = bss_sources()
    obs = mix @ s
    before = G.estimate_sir_db(s, obs)
    assert abs(before - OC.estimate_sir_db(s, obs)) <= 1e-9
    g, o = _check_bss(obs, G.PhaseBssParams.for_channels(4), OC.PhaseBssParams.for_channels(4))
    after = G.estimate_sir_db(s, g.separated)
    assert after > before + 3.0, (before, after)
    assert abs(after - OC.estimate_sir_db(s, o.separated)) <= 1e-6
    assert np.isfinite(g.trace.mean_channel_coherence)


@pytest.mark.parametrize("channels,samples,lags", [(3, 6, [0, 7]), (5, 1001, [1, 2, 3, 5]), (16, 4099, [1, 4, 9]),
                                                   (80, 6000, [1, 2, 3, 5])])
def test_bss_shapes_and_lags(channels, samples, lags):
    # odd sample counts (ragged rows on the product kernel), lags beyond the
    # samples (the covariance fallback) and more channels than the reference test;
    # 80 channels take the large solve for the covariance SVD and the tensor-tile
    # split-K products (outputs wider than 64)
    rng = np.random.default_rng(channels)
    t = np.arange(samples, dtype=np.float64)
    # one sinusoid per channel at 0.03 .. 0.43 cycles per sample: well-separated
    # lagged autocorrelations, so the joint basis is well conditioned
    src = np.stack([np.sin(2 * np.pi * (0.03 + 0.4 * k / channels) * t + k) * (1 + 0.1 * k)
                    for k in range(channels)])
    src += 0.05 * rng.standard_normal(src.shape)
    mix = np.eye(channels) + 0.1 * rng.standard_normal((channels, channels))
    pg, po = G.PhaseBssParams.for_channels(channels), OC.PhaseBssParams.for_channels(channels)
    pg.lags, po.lags = list(lags), list(lags)
    _check_bss(mix @ src, pg, po, tol_corr=1e-8)


def test_bss_rejects_empty():
    with pytest.raises(Exception):
        G.LieSvdBss.separate(np.zeros((3, 1)))


def test_canonical_scores_match_the_oracle_and_the_reference_properties():  # :377-413
    rng = np.random.default_rng(1)
    a = rng.random((7, 5)) - 0.5
    sc = G.canonical_row_scores(a)
    assert np.max(np.abs(sc - OC.canonical_row_scores(a))) <= 1e-12 * np.max(np.abs(sc))
    assert np.max(np.abs(G.canonical_row_scores(a @ random_orthogonal(5, rng)) - sc)) < 1e-9
    perm = rng.permutation(7)
    assert np.max(np.abs(G.canonical_row_scores(a[perm]) - sc[perm])) < 1e-9
    cs = G.canonical_column_scores(a)
    assert np.max(np.abs(cs - OC.canonical_column_scores(a))) <= 1e-12 * np.max(np.abs(cs))
    assert np.max(np.abs(G.row_wedge_capacity(a) - OC.row_wedge_capacity_from_gram(a @ a.T))) <= 1e-12


@pytest.mark.parametrize("shape", [(12, 12), (9, 14), (70, 40), (130, 130)])
def test_solve_canonicalized_matches_the_oracle(shape):
    rng = np.random.default_rng(101)
    base = rng.random(shape) - 0.5
    r = G.solve_canonicalized(base)
    u, s, vt, ro, co = OC.solve_canonicalized(base)
    assert r.row_order.order.tolist() == list(ro) and r.col_order.order.tolist() == list(co)
    assert np.max(np.abs(r.sigma - s)) <= 1e-13 * s.max()
    assert np.max(np.abs((r.u * r.sigma) @ r.vt - base)) <= 1e-12 * np.abs(base).max() * max(shape)
    # the reference's invariance test (n = 12 there): shuffled input, same restored result
    rp, cp = rng.permutation(shape[0]), rng.permutation(shape[1])
    r2 = G.solve_canonicalized(base[np.ix_(rp, cp)])
    rec = ((r2.u[np.argsort(rp)] * r2.sigma) @ r2.vt)[:, np.argsort(cp)]
    assert np.max(np.abs(rec - (r.u * r.sigma) @ r.vt)) < 1e-8


def test_diagonalize_symmetric_canonicalized_restores_the_basis():  # :1204-1229
    rng = np.random.default_rng(103)
    n = 6
    q = random_orthogonal(n, rng)
    fam = [q @ np.diag(1.0 + k * 0.4 + np.arange(n) * 0.2) @ q.T for k in range(3)]
    r = G.diagonalize_symmetric_canonicalized(fam)
    for m in fam:
        x = r.basis.T @ m @ r.basis
        assert np.sum(np.abs(x - np.diag(np.diag(x)))) < 1e-6
    v, _, _, order = OC.diagonalize_symmetric_canonicalized(fam)
    assert r.order.order.tolist() == list(order)
    assert r.order.permute_symmetric(r.order.restore_symmetric(fam[0])).tolist() == fam[0].tolist()
